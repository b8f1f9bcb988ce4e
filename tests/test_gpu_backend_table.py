"""The B200 liquid-scheduler backend table against the reference's own CPU table.

Both tables (LiquidSubstepBackend3D, liquid_substep_backend_3d.h:47-260) run
the same operation on the same inputs through oracle/_ref/
libfluidity_backend_check.so: the CPU table is CpuLiquidSubstepBackend3D
compiled from the reference's sources (liquid_substep_3d_cpu.cc:703-859), the
B200 table is fluidity_b200/adapter over the library's FP64 boundary kernels
and its MAC pressure solver. Scene: the bounded 32^3 tank dam break of
tests/backend_tables.py (1024 particles, 80 blocks of 4^3 cells).

Bars: deposit quanta and compatible stencils, normalized faces, forces and the
pressure links (tests/backend_tables.LinkScene) bit-identical; the gather's flags and fallback counts identical and its
values within 1e-12 of the largest magnitude (the ghost fits' hypot is the
device's); predicted faces within 1e-12 relative; the projection within the
solvers' common gate; error codes identical, including which of several
failing particles decides the code.
"""

import numpy as np
import pytest

import backend_tables as bt
from oracle.box_system import box_pressure_system

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not bt.available(), reason="backend harness not built")]

CPU, B200 = bt.CPU, bt.B200


@pytest.fixture(scope="module")
def scene():
    yield bt.Scene()
    bt.release()


@pytest.fixture(scope="module")
def one_sided():
    return bt.Scene(mixed_sides=False)


@pytest.fixture(scope="module")
def deposited(scene):
    code, q, st = bt.deposit(CPU, scene)
    assert code == 0
    return q, st


@pytest.fixture(scope="module")
def histories(one_sided):
    """On the one-sided scene: old history, the CPU table's normalized deposit
    (some faces low-mass); new, the CPU forces on it, perturbed on valid faces
    as a projection would, with missing faces next to the water marked
    predicted."""
    scene = one_sided
    code, q, _ = bt.deposit(CPU, scene)
    assert code == 0
    min_mass = 0.1 * float(scene.particles["mass"][0])
    code, m, v, val = bt.normalize(CPU, q, min_mass)
    assert code == 0
    code, pred = bt.forces(CPU, scene, v)
    assert code == 0
    rng = np.random.default_rng(3)
    new_v = pred + np.where(val == 1, rng.uniform(-0.05, 0.05, len(pred)), 0.0)
    new_val = val.copy()
    missing_inside = np.nonzero((val == 0) & (scene.tags["eligible"] == 1) & (scene.lattice[:, 1] < 10)
                                & (scene.lattice[:, 0] < 6) & (scene.lattice[:, 2] < 6))[0]
    marked = []
    for slot in missing_inside[::2][:40]:
        side = int(scene.tags["side"][slot])
        c, value = bt.predict(CPU, scene, v, val, int(slot), side)
        if c == 0:
            new_v[slot] = value
            new_val[slot] = 2
            marked.append(int(slot))
    assert len(marked) >= 10
    return dict(min_mass=min_mass, old=(v, val), new=(new_v, new_val), masses=m, predicted_slots=marked,
                missing=missing_inside)


def test_tables_fill_the_transfer_and_projection_operations():
    code, cpu = bt.filled(CPU)
    assert code == 0 and cpu == 0x7FF
    code, b200 = bt.filled(B200)
    assert code == 0
    # deposit, normalize, predict, forces, gather, project, links, freeze and wetted piston;
    # no topology or particle update
    assert b200 == 0x73F


def test_deposit_is_bit_identical(scene, deposited):
    q_cpu, st_cpu = deposited
    code, q, st = bt.deposit(B200, scene)
    assert code == 0
    assert np.array_equal(q, q_cpu)
    for f in ("slot", "compatible", "weight", "gradient", "centered"):
        assert np.array_equal(st[f], st_cpu[f]), f
    # the scene exercises partial support: walls, outside faces and mixed sides
    frac = st_cpu["compatible"].mean()
    assert 0.5 < frac < 1.0
    assert np.count_nonzero(q_cpu["mass"]) > 500


def test_normalize_and_forces_are_bit_identical(scene, deposited, histories):
    q, _ = deposited
    cpu = bt.normalize(CPU, q, histories["min_mass"])
    b200 = bt.normalize(B200, q, histories["min_mass"])
    assert cpu[0] == 0 and b200[0] == 0
    for a, b in zip(cpu[1:], b200[1:]):
        assert np.array_equal(a, b)
    val = cpu[3]
    assert {0, 1, 3} <= set(np.unique(val).tolist())  # missing, valid and low-mass faces all occur
    c0, f_cpu = bt.forces(CPU, scene, cpu[2])
    c1, f_b200 = bt.forces(B200, scene, cpu[2])
    assert c0 == 0 and c1 == 0
    assert np.array_equal(f_cpu, f_b200)


def test_predict_missing_face_matches(scene, one_sided, histories):
    v, val = histories["old"]
    checked = 0
    for slot in histories["missing"][:60]:
        for sc, side in ((one_sided, 0), (scene, 0), (scene, 1)):
            c0, a = bt.predict(CPU, sc, v, val, int(slot), side)
            c1, b = bt.predict(B200, sc, v, val, int(slot), side)
            assert c0 == c1, (slot, side)
            if c0 == 0:
                assert abs(a - b) <= 1e-12 * max(abs(a), 1.0), (slot, side, a, b)
                checked += 1
    assert checked >= 60


def test_gather_matches(one_sided, histories):
    c0, g_cpu, n_cpu = bt.gather(CPU, one_sided, histories["old"], histories["new"])
    c1, g, n = bt.gather(B200, one_sided, histories["old"], histories["new"])
    assert c0 == 0 and c1 == 0
    assert np.array_equal(n, n_cpu)
    for f in ("affine", "old_fallback", "new_fallback", "low_mass"):
        assert np.array_equal(g[f], g_cpu[f]), f
    for f in ("new_pic", "increment", "retained", "slopes", "gradient"):
        scale = max(np.abs(g_cpu[f]).max(), 1.0)
        err = np.abs(g[f] - g_cpu[f]).max() / scale
        assert err <= 1e-12, (f, err)
    print(f"gather: fallback counts {n_cpu.tolist()}, affine on {int(g_cpu['affine'].sum())} of {len(g_cpu)}")
    assert n_cpu[0] > 0 and n_cpu[2] > 0 and g_cpu["affine"].sum() > 100


def test_error_codes_follow_the_cpu_order(scene):
    p = scene.particles.copy()
    p["velocity"][700, 1] = np.nan  # InvalidArgument at particle 700
    p["trial"][300, 0] = p["sorted"][300, 0] + 0.75 * bt.H  # moved beyond half a cell: FailedPrecondition at 300
    for which in (CPU, B200):
        assert bt.deposit(which, scene, particles=p)[0] == 9
    p["trial"][300, 0] = p["sorted"][300, 0]
    for which in (CPU, B200):
        assert bt.deposit(which, scene, particles=p)[0] == 3
    assert bt.deposit(CPU, scene, capacity=512)[0] == bt.deposit(B200, scene, capacity=512)[0] == 8
    q = np.zeros(scene.faces, bt.QUANTA)
    q["mass"][5] = -1
    assert bt.normalize(CPU, q, 0.0)[0] == bt.normalize(B200, q, 0.0)[0] == 3
    # a side with no compatible support anywhere in a stencil
    p = scene.particles.copy()
    p["side"][10] = 7
    assert bt.deposit(CPU, scene, particles=p)[0] == bt.deposit(B200, scene, particles=p)[0] == 9


def _dam_break_system():
    import oracle
    from fluidity_b200 import scenes
    from helpers import box_for, soa_to_xvc

    soa, m = scenes.dam_break(32)
    x, v, c = soa_to_xvc(soa)
    box = box_for(32)
    fm, fq = oracle.p2g(box, x, v, c, m)
    u_pred, _ = oracle.normalize_forces(box, fm, fq, 0.0, scenes.DT, scenes.GRAVITY)
    ct = oracle.classify_cells(box, x)
    return box, box_pressure_system(box, ct, u_pred), scenes.DT


def test_project_matches_within_the_gate():
    box, s, dt = _dam_break_system()
    flux = np.full(len(s["faces_idx"]), np.nan)
    sealed = np.nonzero(s["faces_kind"] == 0)[0]
    flux[sealed[::5]] = 1e-7  # explicit wall flux on some sealed faces
    c0, cpu = bt.project(CPU, s, box.h, dt, tolerance_scale=1e-3, face_flux=flux)
    c1, b200 = bt.project(B200, s, box.h, dt, tolerance_scale=1e-3, face_flux=flux)
    assert c0 == 0 and c1 == 0
    np.testing.assert_allclose(b200["rhs"], cpu["rhs"], rtol=1e-12, atol=1e-18)
    rhs_l2 = np.linalg.norm(cpu["rhs"])
    gate = 1e-3 * (2e-6 + 2e-6 * rhs_l2)
    assert cpu["diag"][1] <= gate and b200["diag"][1] <= gate
    pmax = np.abs(cpu["pressure"]).max()
    dp = np.abs(b200["pressure"] - cpu["pressure"]).max() / pmax
    du = np.abs(b200["corrected_u"] - cpu["corrected_u"]).max() / np.abs(cpu["corrected_u"]).max()
    print(f"project: {len(cpu['pressure'])} cells, iterations cpu {cpu['diag'][0]:.0f} b200 {b200['diag'][0]:.0f}, "
          f"max |dp|/|p| {dp:.2e}, max |du|/|u| {du:.2e}")
    assert dp <= 1e-5 and du <= 1e-5
    np.testing.assert_allclose(b200["measure"][:2], cpu["measure"][:2], rtol=1e-12)
    assert abs(b200["measure"][2] - cpu["measure"][2]) <= 1e-12 * max(abs(cpu["measure"][2]), 1e-12)
    assert b200["diag"][4] == cpu["diag"][4] == 0


def test_operations_repeat_bitwise_without_growing_device_memory(one_sided, histories):
    """The B200 table reserves its storage when it is made: repeated attempts
    leave the device's free memory unchanged and repeat bit for bit."""
    import torch

    box, s, dt = _dam_break_system()
    fs, ps = bt.FreezeScene("tank"), bt.PistonScene("union")

    def attempt():
        return (bt.deposit(B200, one_sided)[1], bt.gather(B200, one_sided, histories["old"], histories["new"])[1],
                bt.project(B200, s, box.h, dt)[1]["pressure"], bt.freeze(B200, fs)[2], bt.wetted_piston(B200, ps)[1])

    first = attempt()
    torch.cuda.synchronize()
    free = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        again = attempt()
        for a, b in zip(first, again):
            assert np.array_equal(a, b)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free


def test_links_are_bit_identical():
    s = bt.LinkScene()
    c0, cells_cpu, faces_cpu, low_cpu = bt.links(CPU, s)
    c1, cells, faces, low = bt.links(B200, s)
    assert c0 == 0 and c1 == 0
    assert np.array_equal(cells, cells_cpu)
    assert np.array_equal(faces, faces_cpu, equal_nan=True)
    assert low == low_cpu > 0
    kinds = np.bincount(faces_cpu[:, 0].astype(int), minlength=3)
    assert kinds[0] > 0 and kinds[1] > 0 and kinds[2] > 0
    internal = faces_cpu[:, 0] == 1
    assert np.count_nonzero(faces_cpu[internal, 1]) == len(s.itf_ordinal)  # the interfaces' jumps
    assert np.isfinite(faces_cpu[:, 7]).sum() > 0  # explicit wall fluxes carried through
    # the one-sided mobility of free-surface links where the liquid cell has a predictor density
    assert len(np.unique(faces_cpu[:, 2])) > 2


def test_links_error_codes_match():
    s = bt.LinkScene()
    nf = len(s.face_index)

    def both(**kw):
        a, b = bt.links(CPU, s, **kw)[0], bt.links(B200, s, **kw)[0]
        assert a == b, (kw.keys(), a, b)
        return a

    pred = s.predicted.copy()
    pred[100] = np.nan
    assert both(predicted=pred) == 3
    air_i = np.vstack([s.air_index, s.cell_index[:1]])
    order = np.lexsort((air_i[:, 0], air_i[:, 1], air_i[:, 2]))
    assert both(air_index=air_i[order], air_pressure=np.append(s.air_pressure, 100.0)[order]) == 3
    itf = s.itf_values.copy()
    itf[2, 1] = 1e6  # surface tension so large that the step exceeds the capillary bound
    assert both(itf_values=itf) == 10
    keep = np.ones(nf, bool)
    keep[500] = False
    assert both(face_index=s.face_index[keep], face_slot=s.face_slot[keep], face_values=s.face_values[keep],
                piston=s.piston[keep], predicted=s.predicted[keep], itf_ordinal=np.array([], np.uint64),
                itf_values=np.zeros((0, 4))) == 9
    fv = s.face_values.copy()
    fv[42, 0] = 2 * bt.H * bt.H
    assert both(face_values=fv) == 3
    cv = s.cell_values.copy()
    cv[7, 1] = 0.0
    assert both(cell_values=cv) == 3
    assert both(wetted=np.full(nf, np.nan)) == 0
    wet = np.full(nf, np.nan)
    wet[3] = 1e-6
    assert both(wetted=wet) == 3


def _assert_frozen_equal(cpu, gpu):
    code0, ci0, cv0, fi0, fs0, fv0, bound0 = cpu
    code1, ci1, cv1, fi1, fs1, fv1, bound1 = gpu
    assert code0 == 0 and code1 == 0
    assert np.array_equal(ci1, ci0)  # the kept cells
    assert np.array_equal(cv1[:, :2], cv0[:, :2])  # liquid volumes and centre distances, bitwise
    assert np.array_equal(cv1[:, 2], cv0[:, 2])  # curvature, bitwise
    assert np.array_equal(fi1, fi0) and np.array_equal(fs1, fs0)
    assert np.array_equal(fv1, fv0, equal_nan=True)  # areas, wall velocities, piston fluxes and flags
    assert bound1 == bound0


@pytest.mark.parametrize("obstacle", ["none", "halfspace", "slab", "tank"])
def test_freeze_is_bit_identical(obstacle):
    s = bt.FreezeScene(obstacle)
    cpu, gpu = bt.freeze(CPU, s), bt.freeze(B200, s)
    _assert_frozen_equal(cpu, gpu)
    _, _, cv, _, _, fv, bound = cpu
    vol = cv[:, 0] / bt.H ** 3
    assert (vol < 0.99).sum() > 50 and (vol > 1 - 1e-12).sum() > 10  # cut and whole liquid cells
    assert (cv[:, 2] != 0).sum() > 50 and np.isfinite(bound)  # interface cells with curvature
    if obstacle != "none":
        assert ((fv[:, 0] > 0) & (fv[:, 0] < bt.H ** 2)).sum() > 10  # partly blocked faces
    if obstacle == "tank":
        assert fv[:, 4].sum() > 10 and np.isfinite(fv[:, 3]).all()  # piston faces; every face carries a flux


def test_freeze_with_exact_curvature_and_without_surface_tension():
    _assert_frozen_equal(bt.freeze(CPU, bt.FreezeScene(exact_curvature=1.5)),
                         bt.freeze(B200, bt.FreezeScene(exact_curvature=1.5)))
    cpu = bt.freeze(CPU, bt.FreezeScene(sigma=0.0))
    _assert_frozen_equal(cpu, bt.freeze(B200, bt.FreezeScene(sigma=0.0)))
    assert np.all(cpu[2][:, 2] == 0) and cpu[6] == np.inf


def test_freeze_error_codes_match():
    s = bt.FreezeScene("halfspace")

    def both(**kw):
        a, b = bt.freeze(CPU, s, **kw)[0], bt.freeze(B200, s, **kw)[0]
        assert a == b, (kw.keys(), a, b)
        return a

    swapped = s.cell_index.copy()
    swapped[[10, 11]] = swapped[[11, 10]]
    assert both(cell_index=swapped) == 3
    # a missing centre sample of a candidate (deep in the liquid) and of a curvature stencil
    keep = ~np.all(s.center_index == (5, 1, 5), axis=1)
    assert both(center_index=s.center_index[keep], center_distance=s.center_distance[keep]) == 9
    keep = ~np.all(s.corner_index == (6, 2, 6), axis=1)
    assert both(corner_index=s.corner_index[keep], corner_distance=s.corner_distance[keep]) == 9
    assert both(normal=(0.8, 0.0, 0.61)) == 3  # not a unit normal
    assert both(kind=2, half_width=0.0) == 3
    assert both(density=0.0) == 3
    assert both(step_duration=1.0) == 9  # above the capillary bound
    bad = s.corner_distance.copy()
    bad[3] = np.nan
    assert both(corner_distance=bad) == 3
    many = np.repeat(s.cell_index, 4, axis=0)[:4097]
    assert both(cell_index=many) == 8
    t = bt.FreezeScene("tank")

    def tank(**kw):
        a, b = bt.freeze(CPU, t, **kw)[0], bt.freeze(B200, t, **kw)[0]
        assert a == b, (kw.keys(), a, b)
        return a

    low, high = t.tank[0], t.tank[1]
    assert tank(tank=(high, low) + t.tank[2:]) == 3  # walls out of order
    assert tank(tank=t.tank[:5] + (1e4,)) == 9  # the piston passes the far wall within the step
    assert tank(tank=t.tank[:2] + (np.inf,) + t.tank[3:]) == 3


@pytest.mark.parametrize("obstacle", ["none", "tank"])
def test_freeze_then_links_on_device_match_the_cpu_pipeline(obstacle):
    """The frozen view of each table feeds that table's own link assembly."""
    s = bt.FreezeScene(obstacle)
    out = []
    for which in (CPU, B200):
        code, ci, cv, fi, fs, fv, _ = bt.freeze(which, s)
        assert code == 0
        nc, nf = len(ci), len(fi)
        fields = np.zeros((nc, 4))
        fields[:, 1] = np.inf
        fields[:, 3] = np.nan
        ls = dict(blocks=s.blocks, center_index=s.center_index, center_distance=s.center_distance, cell_index=ci,
                  cell_values=cv, face_index=fi, face_slot=fs, face_values=fv[:, :4],
                  piston=fv[:, 4].astype(np.uint8), step_duration=s.step_duration, density=s.density, sigma=s.sigma,
                  fields=fields, predicted=np.linspace(-0.1, 0.1, nf), ambient=0.0, air_index=np.zeros((0, 3)),
                  air_pressure=np.zeros(0), itf_ordinal=np.zeros(0, np.uint64), itf_values=np.zeros((0, 4)),
                  wetted=None)
        out.append(bt.links(which, bt.LinkScene(), **ls))
    (c0, cells0, faces0, low0), (c1, cells1, faces1, low1) = out
    assert c0 == 0 and c1 == 0
    assert np.array_equal(cells1, cells0) and np.array_equal(faces1, faces0, equal_nan=True) and low1 == low0
    assert (faces0[:, 0] == 2).sum() > 50  # free-surface links with their theta distances


def test_operation_times_against_the_cpu_table(scene, one_sided, histories):
    """Each operation of both tables timed on the host clock around the table
    call alone (the B200 call includes its uploads, kernels, downloads and
    record conversion; the harness's own set-up is excluded), median of 15
    after 3 warm-up calls; printed for the record. The B200 table must not be
    slower than the CPU table on the operations whose work grows with the
    scene (deposit, gather, freeze, project)."""

    box, system, dt = _dam_break_system()
    q = bt.deposit(CPU, scene)[1]
    ls = bt.LinkScene()
    fs = bt.FreezeScene("tank")
    ps = bt.PistonScene("union")
    ops = {
        "deposit (1024 particles)": lambda w: bt.deposit(w, scene),
        "normalize (15360 faces)": lambda w: bt.normalize(w, q, 0.1 * float(scene.particles["mass"][0])),
        "forces (15360 faces)": lambda w: bt.forces(w, one_sided, histories["old"][0]),
        "gather (1024 particles)": lambda w: bt.gather(w, one_sided, histories["old"], histories["new"]),
        "freeze (tank, 1296 candidates)": lambda w: bt.freeze(w, fs),
        "links (864 cells, 2880 faces)": lambda w: bt.links(w, ls),
        "wetted piston (644 particle spheres)": lambda w: bt.wetted_piston(w, ps),
        "project (3375 cells, to the gate)": lambda w: bt.project(w, system, box.h, dt),
    }
    rows = {}
    for name, op in ops.items():
        med = []
        for which in (CPU, B200):
            for _ in range(3):
                assert op(which)[0] == 0
            t = []
            for _ in range(15):
                op(which)
                t.append(bt.last_op_ms())
            med.append(float(np.median(t)))
        rows[name] = med
    print("\noperation | CPU table ms | B200 table ms | ratio")
    for name, (c, g) in rows.items():
        print(f"{name} | {c:.3f} | {g:.3f} | {c / g:.1f}x")
    for name in ("deposit", "gather", "freeze", "project", "wetted"):
        c, g = next(v for k, v in rows.items() if k.startswith(name))
        assert g <= c, (name, c, g)


@pytest.mark.parametrize("field", ["plane", "union"])
def test_wetted_piston_is_bit_identical(field):
    s = bt.PistonScene(field)
    c0, p0, f0, w0, a0 = bt.wetted_piston(CPU, s)
    c1, p1, f1, w1, a1 = bt.wetted_piston(B200, s)
    assert c0 == 0 and c1 == 0
    assert np.array_equal(p1, p0)  # patches: indices, area enclosures, receivers, assigned area and flux
    assert np.array_equal(f1, f0, equal_nan=True)  # each receiver face's summed midpoint flux
    assert np.array_equal(w1, w0) and a1 == a0
    assert a0 > 0 and (p0[:, 4] >= 0).sum() > 20 and w0[0] > 0


def test_wetted_piston_error_codes_match():
    s = bt.PistonScene("union")

    def both(scene=s, **kw):
        a, b = bt.wetted_piston(CPU, scene, **kw)[0], bt.wetted_piston(B200, scene, **kw)[0]
        assert a == b, (kw.keys(), a, b)
        return a

    assert both(bt.PistonScene("sphere")) == 9  # a small sphere's banded enclosure is wider than 1/1000
    assert both(bt.PistonScene("drop")) == 3  # not a field the piston can measure
    assert both(radius=0.0) == 3
    bad = s.positions.copy()
    bad[5, 1] = np.nan
    assert both(positions=bad) == 3
    assert both(tank=(s.tank[1], s.tank[0]) + tuple(s.tank[2:])) == 3
    swapped = s.face_slot.copy()
    swapped[[3, 4]] = swapped[[4, 3]]
    assert both(face_slot=swapped) == 3
    fv = s.face_values.copy()
    receivers = np.nonzero(fv[:, 4] == 1)[0]
    fv[receivers[0], 2] = 0.0  # a receiver face whose wall velocity is not the piston's
    assert both(face_values=fv) == 9
    assert both(positions=np.repeat(s.positions, 2, axis=0)) == 8  # more particles than the bounded workspace


def test_freeze_and_wetted_piston_agree_on_seeded_scenes():
    """Seeded variations: drops of other centres, radii and wobbles under each
    obstacle kind, and tanks of other walls and piston speeds with particle
    unions of other spacings; whenever the CPU table succeeds the B200 table
    gives the same bits, and otherwise the same code."""
    rng = np.random.default_rng(11)
    agreed = pistons = 0
    for trial in range(12):
        kind = ["none", "halfspace", "slab", "tank"][trial % 4]
        s = bt.FreezeScene(kind)
        if kind == "tank":
            t = list(s.tank)
            t[0] = rng.uniform(0.05, 0.9) * bt.H
            t[2] = rng.uniform(0.05, 0.9) * bt.H
            t[5] = rng.uniform(-0.2, 0.2)
            s.tank = tuple(t)
        else:
            c = np.array([rng.uniform(5.0, 7.0), rng.uniform(4.0, 5.0), rng.uniform(5.0, 7.0)])
            r0, wob = rng.uniform(2.5, 3.8), rng.uniform(0.0, 0.4)

            def dist(p):
                r = np.linalg.norm(p - c, axis=1)
                return (r - r0 - wob * np.sin(p[:, 0] / 1.5) * np.cos(p[:, 2] / 2.0)) * bt.H

            s.center_distance = dist(s.center_index + 0.5)
            s.corner_distance = dist(s.corner_index.astype(np.float64))
            if kind == "halfspace":
                a = rng.uniform(0.0, np.pi / 2)
                s.normal, s.coordinate = (np.cos(a), 0.0, np.sin(a)), rng.uniform(4.0, 7.0) * bt.H
            if kind == "slab":
                a = rng.uniform(0.0, np.pi / 2)
                s.normal, s.coordinate = (np.cos(a), 0.0, np.sin(a)), rng.uniform(6.0, 10.0) * bt.H
        cpu, gpu = bt.freeze(CPU, s), bt.freeze(B200, s)
        assert cpu[0] == gpu[0], (trial, kind, cpu[0], gpu[0])
        if cpu[0] == 0:
            _assert_frozen_equal(cpu, gpu)
            agreed += 1
        if kind == "tank" and cpu[0] == 0:
            code, ci, cv, fi, fs, fv, _ = cpu
            ps = bt.PistonScene("union")
            gx, gy, gz = np.meshgrid(s.tank[0] + bt.H * (0.2 + 0.5 * np.arange(4)), bt.H * (0.8 + 0.5 * np.arange(7)),
                                     bt.H * (0.5 + 0.5 * np.arange(23)), indexing="ij")
            over = dict(blocks=s.blocks, tank=s.tank, cell_index=ci, cell_values=cv, face_index=fi, face_slot=fs,
                        face_values=fv, positions=np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1),
                        radius=0.65 * bt.H)
            a, b = bt.wetted_piston(CPU, ps, **over), bt.wetted_piston(B200, ps, **over)
            assert a[0] == b[0], (trial, a[0], b[0])
            if a[0] == 0:
                assert np.array_equal(b[1], a[1]) and np.array_equal(b[2], a[2], equal_nan=True)
                assert np.array_equal(b[3], a[3]) and b[4] == a[4]
                pistons += 1
    assert agreed >= 8 and pistons >= 1
