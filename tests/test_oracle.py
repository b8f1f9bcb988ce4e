"""Pins the oracle: the FP64 restatement (oracle/cpu) against the reference's
golden vectors (tests/golden, generated from its Python fixtures) and against
the reference's own CPU operators compiled from source (oracle/_ref).
CPU only."""

import numpy as np
import pytest

import oracle
from fluidity_b200 import scenes
from helpers import box_for, golden, pressure_case, soa_to_xvc
from oracle.box_system import box_pressure_system, ref_blocks_for_box

CORNER_BLOCKS = np.array([[0, -1, 0], [1, -1, 0], [0, 0, 0], [1, 0, 0], [0, -1, 1], [1, -1, 1], [0, 0, 1], [1, 0, 1]],
                         np.int32)
CORNER_BOX = oracle.Box.make([0.0, 0.0, 0.0], 1.0, [0, -4, 0], [8, 8, 8])
AFFINE = np.array([[2.0, 4.0, -1.0], [-5.0, 1.0, 5.0], [7.0, -2.0, 3.0]])
VEL = np.array([1.0, -2.0, 4.0])
CORNER = np.array([3.75, -0.25, 3.75])

needs_ref = pytest.mark.skipif(oracle.ref() is None, reason="reference operators not built (oracle/ref/Makefile)")


def _dense_face(box, arrays, axis, i, j, k):
    li, lj, lk = i - box.lo[0], j - box.lo[1], k - box.lo[2]
    return arrays[axis][lk, lj, li]


def test_stencil_matches_exact_rational_fixture():
    g = golden("transfer_3d.json")["arrays"]
    pos = np.array(g["position"])
    found = {}
    for axis in range(3):
        faces, vals = oracle.stencil([0, 0, 0], 1.0, axis, pos)
        for f, v in zip(faces, vals):
            found[tuple(int(t) for t in f)] = v
    assert len(g["face_indices"]) == 81
    for idx, w, disp, grad in zip(g["face_indices"], g["weights"], g["face_displacements"], g["weight_gradients"]):
        v = found[tuple(idx)]
        np.testing.assert_allclose(v[0], w, rtol=2e-12, atol=2e-12)
        np.testing.assert_allclose(v[1:4], disp, rtol=2e-12, atol=2e-12)
        np.testing.assert_allclose(v[4:7], grad, rtol=2e-12, atol=2e-12)


def test_p2g_matches_exact_rational_fixture():
    g = golden("transfer_3d.json")["arrays"]
    fm, fq = oracle.p2g(CORNER_BOX, [g["position"]], [g["velocity"]], [np.ravel(g["affine_velocity_fit"])],
                        g["particle_mass"][0])
    for idx, m, q in zip(g["face_indices"], g["expected_mass"], g["expected_pure_momentum"]):
        np.testing.assert_allclose(_dense_face(CORNER_BOX, fm, *idx), m, rtol=2e-12, atol=2e-12)
        np.testing.assert_allclose(_dense_face(CORNER_BOX, fq, *idx), q, rtol=2e-12, atol=2e-12)
    assert np.isclose(sum(a.sum() for a in fm), 3 * g["particle_mass"][0])


@needs_ref
def test_stencil_matches_reference_operator():
    rng = np.random.default_rng(1)
    for _ in range(20):
        pos = rng.uniform(2.0, 6.0, size=3)
        for axis in range(3):
            faces, vals = oracle.stencil([0, 0, 0], 0.5, axis, pos)
            rf = np.zeros((27, 4), np.int32)
            rv = np.zeros((27, 7))
            lib = oracle.ref()
            assert lib.ref_geometry_stencil(oracle._d(np.zeros(3)), 0.5, axis, oracle._d(pos), oracle._d(pos),
                                            oracle._i(rf), oracle._d(rv)) == 0
            np.testing.assert_array_equal(faces, rf)
            np.testing.assert_allclose(vals, rv, rtol=1e-14, atol=1e-15)


def _random_particles(n, rng, lo=1.2, hi=7.8, h=1.0):
    x = rng.uniform(lo, hi, size=(n, 3)) * h
    v = rng.normal(size=(n, 3))
    c = rng.normal(size=(n, 9))
    m = rng.uniform(0.5, 2.0, size=n)
    return x, v, c, m


@needs_ref
def test_p2g_restatement_matches_reference_deposit():
    rng = np.random.default_rng(2)
    x, v, c, m = _random_particles(300, rng)
    blocks = np.array([[i, j, k] for k in range(3) for j in range(3) for i in range(3)], np.int32)
    rm, rq = oracle.ref_deposit([0, 0, 0], 1.0, blocks, oracle.particles_aos(x, v, c, m))
    fi = oracle.ref_face_indices([0, 0, 0], 1.0, blocks)
    box = oracle.Box.make([0, 0, 0], 1.0, [0, 0, 0], [12, 12, 12])
    fm, fq = oracle.p2g(box, x, v, c, m)
    for s, (a, i, j, k) in enumerate(fi):
        if i < 12 and j < 12 and k < 12:
            assert _dense_face(box, fm, a, i, j, k) == pytest.approx(rm[s], rel=1e-13, abs=1e-13)
            assert _dense_face(box, fq, a, i, j, k) == pytest.approx(rq[s], rel=1e-12, abs=1e-12)


@needs_ref
def test_quanta_restatement_matches_reference_bitwise():
    rng = np.random.default_rng(3)
    x, v, c, m = _random_particles(200, rng)
    blocks = np.array([[i, j, k] for k in range(3) for j in range(3) for i in range(3)], np.int32)
    ms, ps = 2.0 ** -30, 2.0 ** -24
    rmq, rpq = oracle.ref_deposit_quanta([0, 0, 0], 1.0, blocks, oracle.particles_aos(x, v, c, m), ms, ps, len(x))
    fi = oracle.ref_face_indices([0, 0, 0], 1.0, blocks)
    box = oracle.Box.make([0, 0, 0], 1.0, [0, 0, 0], [12, 12, 12])
    mq, pq = oracle.p2g_quanta(box, x, v, c, m, ms, ps)
    for s, (a, i, j, k) in enumerate(fi):
        if i < 12 and j < 12 and k < 12:
            assert _dense_face(box, mq, a, i, j, k) == rmq[s]
            assert _dense_face(box, pq, a, i, j, k) == rpq[s]
    # order independence (integer sums)
    mq2, pq2 = oracle.p2g_quanta(box, x[::-1], v[::-1], c[::-1], m[::-1], ms, ps)
    for a in range(3):
        np.testing.assert_array_equal(mq[a], mq2[a])
        np.testing.assert_array_equal(pq[a], pq2[a])


@needs_ref
def test_normalize_restatement_matches_reference():
    """The restatement's normalize (fo_normalize_forces with dt = 0) against the
    reference's NormalizeLiquidMacFaces3D on the same decoded deposits: equal
    masses and velocities, and the same per-face validity (0 missing, 1 valid,
    3 low mass), with a threshold that makes some faces low-mass."""
    rng = np.random.default_rng(7)
    x, v, c, m = _random_particles(300, rng)
    box = oracle.Box.make([0, 0, 0], 1.0, [0, 0, 0], [12, 12, 12])
    ms, ps = 2.0 ** -30, 2.0 ** -24
    mq, pq = oracle.p2g_quanta(box, x, v, c, m, ms, ps)
    m_min = float(np.quantile(np.concatenate([a[a > 0] for a in mq]) * ms, 0.2))
    fm = [a.astype(np.float64) * ms for a in mq]
    fq = [a.astype(np.float64) * ps for a in pq]
    u, valid = oracle.normalize_forces(box, fm, fq, m_min, 0.0, [0.0, 0.0, 0.0])
    seen = set()
    for a in range(3):
        rm, ru, rv = oracle.ref_normalize(mq[a].ravel(), pq[a].ravel(), ms, ps, len(x), m_min)
        np.testing.assert_array_equal(fm[a].ravel(), rm)
        np.testing.assert_allclose(u[a].ravel(), ru, rtol=1e-15, atol=0)
        np.testing.assert_array_equal(valid[a].ravel(), rv)
        seen |= set(np.unique(rv).tolist())
    assert seen == {0, 1, 3}


def test_quanta_ties_round_to_even():
    """Known answers of the reference's tie test (test_transfers_3d.cc:800-862):
    at the X face (3,-1,3) of a particle at (3.5, 0, 4) each axis weight is 1/2."""
    pos = np.array([[3.5, 0.0, 4.0]])
    expected = {-2.5: -2, -1.5: -2, -0.5: 0, 0.5: 0, 1.5: 2, 2.5: 2}
    for vel, q in expected.items():
        mq, pq = oracle.p2g_quanta(CORNER_BOX, pos, [[vel, 0, 0]], np.zeros((1, 9)), 8.0, 1.0, 1.0)
        assert _dense_face(CORNER_BOX, mq, 0, 3, -1, 3) == 1
        assert _dense_face(CORNER_BOX, pq, 0, 3, -1, 3) == q
    mq, pq = oracle.p2g_quanta(CORNER_BOX, np.repeat(pos, 2, 0), [[1.0, 0, 0]] * 2, np.zeros((2, 9)), 4.0, 1.0, 1.0)
    assert _dense_face(CORNER_BOX, mq, 0, 3, -1, 3) == 0
    assert _dense_face(CORNER_BOX, pq, 0, 3, -1, 3) == 0


def _affine_fields(box, p, rows, vel, old):
    u_new, u_old = [], []
    for a in range(3):
        shape = box.face_shape(a)
        k, j, i = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
        anchor = [(i + box.lo[0] + (0 if a == 0 else 0.5)) * box.h + box.origin[0],
                  (j + box.lo[1] + (0 if a == 1 else 0.5)) * box.h + box.origin[1],
                  (k + box.lo[2] + (0 if a == 2 else 0.5)) * box.h + box.origin[2]]
        u_new.append(vel[a] + sum(rows[a][d] * (anchor[d] - p[d]) for d in range(3)))
        u_old.append(np.full(shape, old[a]))
    return u_new, u_old


def test_g2p_reproduces_affine_field_at_corner():
    """test_transfers_3d.cc:110-143: fitted slopes == gradient == C, PIC == v."""
    for origin, h in (([0.0, 0.0, 0.0], 1.0), ([1.0, -3.0, 5.0], 2.0)):
        box = oracle.Box.make(origin, h, [0, -4, 0], [8, 8, 8])
        p = np.array(origin) + h * CORNER
        un, uo = _affine_fields(box, p, AFFINE, VEL, [2.0, 3.0, -4.0])
        out = oracle.g2p(box, [p], un, uo)[0]
        np.testing.assert_allclose(out[0:3], VEL, rtol=2e-12, atol=2e-12)
        np.testing.assert_allclose(out[3:6], [-1.0, -5.0, 8.0], rtol=2e-12, atol=2e-12)
        np.testing.assert_allclose(out[6:15].reshape(3, 3), AFFINE, rtol=2e-12, atol=2e-12)
        np.testing.assert_allclose(out[15:24].reshape(3, 3), AFFINE, rtol=2e-12, atol=2e-12)


def test_g2p_quadratic_row_separates_fit_and_gradient():
    """test_transfers_3d.cc:205-245: a displacement-squared field gives PIC 1/4 h^2-scaled
    and fitted slope -3/16 (h=1) / -3/8 (h=2), with zero gradient at the particle."""
    for origin, h, pic, slope in (([0.0, 0.0, 0.0], 1.0, 0.25, -0.1875), ([1.0, -3.0, 5.0], 2.0, 1.0, -0.375)):
        box = oracle.Box.make(origin, h, [0, -4, 0], [8, 8, 8])
        p = np.array(origin) + h * CORNER
        un = []
        for a in range(3):
            shape = box.face_shape(a)
            idx = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")[2 - a]
            anchor = (idx + box.lo[a]) * h + origin[a]
            un.append((anchor - p[a]) ** 2)
        out = oracle.g2p(box, [p], un)[0]
        np.testing.assert_allclose(out[0:3], pic, rtol=2e-12, atol=2e-12)
        np.testing.assert_allclose(out[6:15].reshape(3, 3), np.diag([slope] * 3), rtol=2e-12, atol=2e-12)
        np.testing.assert_allclose(out[15:24], 0.0, atol=2e-12)


def test_g2p_matches_reference_transport_sampler():
    """Velocity and true gradient vs mac_transport_3d.sample_mac_transport (quadratic)."""
    t = golden("transport_3d.json")
    h = t["h"]
    box = oracle.Box.make([0, 0, 0], h, [0, 0, 0], [16, 16, 16])
    un = []
    for a in range(3):
        c0, g, q = t["coefficients"][a]
        g, q = np.array(g), np.array(q)
        shape = box.face_shape(a)
        k, j, i = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
        X = np.stack([(i + (0 if a == 0 else 0.5)) * h, (j + (0 if a == 1 else 0.5)) * h,
                      (k + (0 if a == 2 else 0.5)) * h], -1)
        un.append(c0 + X @ g + np.einsum("...i,ij,...j->...", X, q, X))
    out = oracle.g2p(box, np.array(t["positions"]), un)
    np.testing.assert_allclose(out[:, 0:3], t["velocity"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(out[:, 15:24].reshape(-1, 3, 3), t["gradient"], rtol=1e-12, atol=1e-12)


@needs_ref
def test_g2p_restatement_matches_reference_gather():
    rng = np.random.default_rng(4)
    x, v, c, m = _random_particles(100, rng)
    blocks = np.array([[i, j, k] for k in range(3) for j in range(3) for i in range(3)], np.int32)
    fi = oracle.ref_face_indices([0, 0, 0], 1.0, blocks)
    uo, un = rng.normal(size=len(fi)), rng.normal(size=len(fi))
    ref = oracle.ref_gather([0, 0, 0], 1.0, blocks, oracle.particles_aos(x, v, c, m), uo, un)
    box = oracle.Box.make([0, 0, 0], 1.0, [0, 0, 0], [12, 12, 12])
    dn = [np.zeros(box.face_shape(a)) for a in range(3)]
    do = [np.zeros(box.face_shape(a)) for a in range(3)]
    for s, (a, i, j, k) in enumerate(fi):
        if i < 13 and j < 13 and k < 13:
            sh = box.face_shape(a)
            if k < sh[0] and j < sh[1] and i < sh[2]:
                dn[a][k, j, i] = un[s]
                do[a][k, j, i] = uo[s]
    out = oracle.g2p(box, x, dn, do)
    np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("case", range(8))
def test_pressure_restatement_matches_dense_fixture(case):
    g = golden("pressure_3d.json")
    ci, cv, fi, fk, fv, dt, ex = pressure_case(g["arrays"], case)
    out = oracle.pressure_solve(ci, cv, fi, fk, fv, 1.0, dt, rel_tol=1e-15, max_iterations=200)
    tol = dict(rtol=2e-12, atol=2e-12)
    np.testing.assert_allclose(out["pressure"], ex["expected_cell_pressures"], **tol)
    np.testing.assert_allclose(out["rhs"], ex["expected_integrated_rhs"], **tol)
    np.testing.assert_allclose(out["residual"], ex["expected_true_residuals"], **tol)
    np.testing.assert_allclose(out["defect"], ex["expected_cell_constraint_defects"], **tol)
    np.testing.assert_allclose(out["corrected_u"], ex["expected_corrected_face_velocities"], **tol)
    assert out["diag"]["gauge_count"] == len(ex["gauges"])


@needs_ref
@pytest.mark.parametrize("case", range(8))
def test_reference_build_matches_dense_fixture(case):
    """Pins the compiled reference itself (ProjectMacPressure3D) against the Python fixture."""
    g = golden("pressure_3d.json")
    ci, cv, fi, fk, fv, dt, ex = pressure_case(g["arrays"], case)
    blocks = sorted({(x // 4, y // 4, z // 4) for (_, x, y, z) in fi} | {(x // 4, y // 4, z // 4) for x, y, z in ci})
    out = oracle.ref_project([0, 0, 0], 1.0, np.array(blocks, np.int32), dt, ci, cv, fi, fk, fv,
                             tolerance_scale=1e-12)
    np.testing.assert_allclose(out["pressure"], ex["expected_cell_pressures"], rtol=2e-9, atol=2e-9)
    np.testing.assert_allclose(out["corrected_u"], ex["expected_corrected_face_velocities"], rtol=2e-9, atol=2e-9)


@needs_ref
def test_pressure_restatement_matches_reference_on_dam_break():
    """The 32^3 dam break's first projection (3375 fluid cells, under the
    reference's 4096-cell cap): same system, same answer."""
    n = 32
    soa, m = scenes.dam_break(n)
    x, v, c = soa_to_xvc(soa)
    box = box_for(n)
    fm, fq = oracle.p2g(box, x, v, c, m)
    u_pred, _ = oracle.normalize_forces(box, fm, fq, 0.0, scenes.DT, scenes.GRAVITY)
    ct = oracle.classify_cells(box, x)
    sysm = box_pressure_system(box, ct, u_pred)
    assert len(sysm["cells_idx"]) == 3375
    mine = oracle.pressure_solve(sysm["cells_idx"], sysm["cells_val"], sysm["faces_idx"], sysm["faces_kind"],
                                 sysm["faces_val"], box.h, scenes.DT, rel_tol=1e-12)
    ref = oracle.ref_project([0, 0, 0], box.h, ref_blocks_for_box(n), scenes.DT, sysm["cells_idx"],
                             sysm["cells_val"], sysm["faces_idx"], sysm["faces_kind"], sysm["faces_val"],
                             tolerance_scale=1e-6)
    np.testing.assert_allclose(mine["rhs"], ref["rhs"], rtol=1e-12, atol=1e-18)
    assert np.abs(mine["pressure"] - ref["pressure"]).max() <= 1e-6 * np.abs(ref["pressure"]).max()
    np.testing.assert_allclose(mine["corrected_u"], ref["corrected_u"], rtol=1e-6, atol=1e-9)


def test_vcycle_is_symmetric_positive():
    n = 32
    soa, _ = scenes.dam_break(n)
    x, _, _ = soa_to_xvc(soa)
    box = box_for(n)
    ct = oracle.classify_cells(box, x)
    rng = np.random.default_rng(5)
    a = rng.normal(size=ct.shape) * (ct == 1)
    b = rng.normal(size=ct.shape) * (ct == 1)
    ma = oracle.vcycle(box, ct, a)
    mb = oracle.vcycle(box, ct, b)
    assert np.vdot(ma, b) == pytest.approx(np.vdot(a, mb), rel=1e-10)
    assert np.vdot(ma, a) > 0


def test_oracle_step_conserves_mass_and_projects():
    n = 32
    soa, m = scenes.dam_break(n)
    x, v, c = soa_to_xvc(soa)
    box = box_for(n)
    r = oracle.step(box, x, v, c, scenes.DT)
    assert r["diag"]["true_residual_l2"] <= 1e-6 * r["diag"]["rhs_l2"]
    un, ct = r["u_new"], r["cell_type"]
    div = (un[0][:, :, 1:] - un[0][:, :, :-1]) + (un[1][:, 1:, :] - un[1][:, :-1, :]) + (un[2][1:] - un[2][:-1])
    assert np.abs(div[ct == 1]).max() / n <= 1e-4
    assert np.all(r["x"] >= box.h) and np.all(r["x"] <= 1 - box.h)


def test_scenes_are_seeded_and_sized():
    a, ma = scenes.dam_break(32)
    b, mb = scenes.dam_break(32)
    np.testing.assert_array_equal(a, b)
    assert a.shape == (15, 8 * 15 ** 3) and ma == pytest.approx(1000.0 / 32 ** 3 / 8)
    c, _ = scenes.dam_break(32, seed=1)
    assert not np.array_equal(a[:3], c[:3])
    s, _ = scenes.splash(64)
    assert (s[3] > 0).sum() > 0 and (s[3] < 0).sum() == (s[3] > 0).sum()
