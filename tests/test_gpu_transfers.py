"""GPU parity of the transfer operators through the C-ABI, against the
reference's compiled CPU operators (oracle/_ref), the FP64 restatement and the
exact-rational golden fixture. FP32 hot path: 1e-5 norm-wise relative
(max |gpu - ref| / max |ref|); FP64 quantized path: bit-exact."""

import numpy as np
import pytest

import fluidity_b200 as fb
import oracle
from helpers import golden

pytestmark = pytest.mark.gpu

TOL = 1e-5
CORNER_BLOCKS = np.array([[0, -1, 0], [1, -1, 0], [0, 0, 0], [1, 0, 0], [0, -1, 1], [1, -1, 1], [0, 0, 1], [1, 0, 1]],
                         np.int32)


def ref_slot(blocks, axis, x, y, z):
    """Owned-slot index in the reference's 4^3 layout (sparse_mac_grid_3d.cc:388-409)."""
    order = sorted(range(len(blocks)), key=lambda i: (blocks[i][2], blocks[i][1], blocks[i][0]))
    ordinal = {tuple(blocks[i]): r for r, i in enumerate(order)}
    b = (x // 4, y // 4, z // 4)
    return ordinal[b] * 192 + axis * 64 + ((z - 4 * b[2]) * 4 + (y - 4 * b[1])) * 4 + (x - 4 * b[0])


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def _cube_blocks(k):
    return np.array([[i, j, l] for l in range(k) for j in range(k) for i in range(k)], np.int32)


def _random_particles(n, rng, lo, hi, h):
    x = rng.uniform(lo, hi, size=(n, 3)) * h
    return x, rng.normal(size=(n, 3)), rng.normal(size=(n, 9)), rng.uniform(0.5, 2.0, size=n)


def test_deposit_corner_matches_exact_rational_fixture():
    g = golden("transfer_3d.json")["arrays"]
    parts = oracle.particles_aos([g["position"]], [g["velocity"]], [np.ravel(g["affine_velocity_fit"])],
                                 g["particle_mass"][0])
    m, q, meas = fb.deposit_mac_3d([0, 0, 0], 1.0, CORNER_BLOCKS, parts)
    assert meas.compiled_architecture == 1000
    touched = np.zeros(len(m), bool)
    for (a, x, y, z), em, eq in zip(g["face_indices"], g["expected_mass"], g["expected_pure_momentum"]):
        s = ref_slot(CORNER_BLOCKS.tolist(), a, x, y, z)
        touched[s] = True
        assert m[s] == pytest.approx(em, rel=1e-6, abs=1e-7)
        assert q[s] == pytest.approx(eq, rel=1e-5, abs=1e-6)
    assert np.all(m[~touched] == 0.0) and np.all(q[~touched] == 0.0)


def test_deposit_matches_reference_operator():
    rng = np.random.default_rng(10)
    h = 1.0 / 32
    blocks = _cube_blocks(8)
    x, v, c, m = _random_particles(20000, rng, 1.5, 30.5, h)
    parts = oracle.particles_aos(x, v, c, m * h ** 3)
    rm, rq = oracle.ref_deposit([0, 0, 0], h, blocks, parts)
    gm, gq, _ = fb.deposit_mac_3d([0, 0, 0], h, blocks, parts)
    assert _rel(gm, rm) <= TOL
    assert _rel(gq, rq) <= TOL


def test_quanta_deposit_is_bitwise_reference():
    rng = np.random.default_rng(11)
    blocks = _cube_blocks(4)
    x, v, c, m = _random_particles(3000, rng, 1.5, 14.5, 1.0)
    parts = oracle.particles_aos(x, v, c, m)
    ms, ps = 2.0 ** -30, 2.0 ** -24
    rm, rq = oracle.ref_deposit_quanta([0, 0, 0], 1.0, blocks, parts, ms, ps, len(x))
    gm, gq, meas = fb.deposit_mac_quanta_3d([0, 0, 0], 1.0, blocks, parts, ms, ps, len(x))
    np.testing.assert_array_equal(gm, rm)
    np.testing.assert_array_equal(gq, rq)
    # order independence: the reversed batch gives identical integer sums
    gm2, gq2, _ = fb.deposit_mac_quanta_3d([0, 0, 0], 1.0, blocks, parts[::-1].copy(), ms, ps, len(x))
    np.testing.assert_array_equal(gm2, gm)
    np.testing.assert_array_equal(gq2, gq)


def test_quanta_ties_round_to_even_on_device():
    """Known answers of test_transfers_3d.cc:800-862 (expected quanta {-2,-2,0,0,2,2})."""
    slot = ref_slot(CORNER_BLOCKS.tolist(), 0, 3, -1, 3)
    for vel, expect in {-2.5: -2, -1.5: -2, -0.5: 0, 0.5: 0, 1.5: 2, 2.5: 2}.items():
        p = oracle.particles_aos([[3.5, 0.0, 4.0]], [[vel, 0, 0]], np.zeros((1, 9)), 8.0)
        gm, gq, _ = fb.deposit_mac_quanta_3d([0, 0, 0], 1.0, CORNER_BLOCKS, p, 1.0, 1.0, 1)
        assert gm[slot] == 1 and gq[slot] == expect


def test_quanta_translated_geometry_matches_reference():
    rng = np.random.default_rng(12)
    origin, h = [1.0, -3.0, 5.0], 2.0
    cells = np.stack([rng.uniform(1.5, 6.4, 64), rng.uniform(1.5, 2.4, 64), rng.uniform(1.5, 6.4, 64)], 1)
    x = np.array(origin) + h * cells  # inside blocks (0..1, 0, 0..1) with complete support
    v, c, m = rng.normal(size=(64, 3)), rng.normal(size=(64, 9)), rng.uniform(0.5, 2.0, size=64)
    parts = oracle.particles_aos(x, v, c, m)
    rm, rq = oracle.ref_deposit_quanta(origin, h, CORNER_BLOCKS[[2, 3, 6, 7]], parts, 2.0 ** -20, 2.0 ** -20, 64)
    gm, gq, _ = fb.deposit_mac_quanta_3d(origin, h, CORNER_BLOCKS[[2, 3, 6, 7]], parts, 2.0 ** -20, 2.0 ** -20, 64)
    np.testing.assert_array_equal(gm, rm)
    np.testing.assert_array_equal(gq, rq)


def test_gather_matches_reference_operator():
    rng = np.random.default_rng(13)
    h = 1.0 / 32
    blocks = _cube_blocks(8)
    x, v, c, m = _random_particles(20000, rng, 1.5, 30.5, h)
    parts = oracle.particles_aos(x, v, c, m)
    fc = 192 * len(blocks)
    uo, un = rng.normal(size=fc), rng.normal(size=fc)
    ref = oracle.ref_gather([0, 0, 0], h, blocks, parts, uo, un)
    got, meas = fb.gather_mac_3d([0, 0, 0], h, blocks, parts, uo, un)
    assert meas.compiled_architecture == 1000
    for lo, hi in ((0, 3), (3, 6), (6, 15), (15, 24)):
        assert _rel(got[:, lo:hi], ref[:, lo:hi]) <= TOL, (lo, hi)


def test_gather_reproduces_affine_field():
    for origin, h in (([0.0, 0.0, 0.0], 1.0), ([1.0, -3.0, 5.0], 2.0)):
        fi = oracle.ref_face_indices(origin, h, CORNER_BLOCKS)
        p = np.array(origin) + h * np.array([3.75, -0.25, 3.75])
        rows = np.array([[2.0, 4.0, -1.0], [-5.0, 1.0, 5.0], [7.0, -2.0, 3.0]])
        vel = np.array([1.0, -2.0, 4.0])
        un = np.zeros(len(fi))
        for s, (a, i, j, k) in enumerate(fi):
            anchor = np.array(origin) + h * (np.array([i, j, k], float) + np.where(np.arange(3) == a, 0.0, 0.5))
            un[s] = vel[a] + rows[a] @ (anchor - p)
        uo = np.tile([2.0, 3.0, -4.0], 1)[fi[:, 0]]
        parts = oracle.particles_aos([p], [[0, 0, 0]], np.zeros((1, 9)), 1.0)
        got, _ = fb.gather_mac_3d(origin, h, CORNER_BLOCKS, parts, uo, un)
        np.testing.assert_allclose(got[0, 0:3], vel, rtol=TOL, atol=TOL * 10)
        np.testing.assert_allclose(got[0, 3:6], [-1.0, -5.0, 8.0], rtol=TOL, atol=TOL * 10)
        np.testing.assert_allclose(got[0, 6:15].reshape(3, 3), rows, rtol=TOL, atol=TOL * 50)
        np.testing.assert_allclose(got[0, 15:24].reshape(3, 3), rows, rtol=TOL, atol=TOL * 50)


def test_rejections_preserve_error_codes():
    p = oracle.particles_aos([[3.5, 0.0, 4.0]], [[np.nan, 0, 0]], np.zeros((1, 9)), 1.0)
    with pytest.raises(fb.FluidityError) as e:
        fb.deposit_mac_3d([0, 0, 0], 1.0, CORNER_BLOCKS, p)
    assert e.value.code == fb.INVALID_ARGUMENT
    far = oracle.particles_aos([[3.5, 0.0, 4.0]], [[0, 0, 0]], np.zeros((1, 9)), 1.0,
                               trial=[[4.2, 0.0, 4.0]])  # motion beyond h/2
    with pytest.raises(fb.FluidityError) as e:
        fb.deposit_mac_3d([0, 0, 0], 1.0, CORNER_BLOCKS, far)
    assert e.value.code == fb.FAILED_PRECONDITION
    edge = oracle.particles_aos([[0.2, -3.9, 0.2]], [[0, 0, 0]], np.zeros((1, 9)), 1.0)  # support leaves the blocks
    with pytest.raises(fb.FluidityError) as e:
        fb.deposit_mac_3d([0, 0, 0], 1.0, CORNER_BLOCKS, edge)
    assert e.value.code == fb.FAILED_PRECONDITION
    with pytest.raises(fb.FluidityError) as e:
        fb.deposit_mac_quanta_3d([0, 0, 0], 1.0, CORNER_BLOCKS, p, 3.0, 1.0, 1)
    assert e.value.code == fb.INVALID_ARGUMENT
    with pytest.raises(fb.FluidityError) as e:
        fb.deposit_mac_quanta_3d([0, 0, 0], 1.0, CORNER_BLOCKS, p, 1.0, 1.0, (1 << 20) + 1)
    assert e.value.code == fb.RESOURCE_EXHAUSTED


def test_empty_batch_clears_faces():
    m, q, _ = fb.deposit_mac_3d([0, 0, 0], 1.0, CORNER_BLOCKS, np.zeros((0, 19)))
    assert np.all(m == 0) and np.all(q == 0) and len(m) == 192 * 8


def test_normalized_p2g_reports_face_validity():
    """fl_p2g_normalized on the sorted 32^3 dam break with a minimum face mass
    that makes part of the faces low-mass: the validity bytes equal the FP64
    restatement's NormalizeCore validity (pinned against the reference's
    NormalizeLiquidMacFaces3D), and the velocities the fused normalize's."""
    import ctypes

    import torch

    from fluidity_b200 import scenes
    from helpers import box_for, soa_to_xvc

    n = 32
    soa, mass = scenes.dam_break(n)
    count = soa.shape[1]
    ctx = fb.LiquidContext(n, capacity=count)
    src = [torch.from_numpy(np.ascontiguousarray(soa[k])).cuda() for k in range(15)]
    dst = [torch.empty_like(t) for t in src]

    def parts(ts):
        p = fb.Particles()
        for d in range(3):
            p.x[d], p.v[d] = ts[d].data_ptr(), ts[3 + d].data_ptr()
        for d in range(9):
            p.c[d] = ts[6 + d].data_ptr()
        p.mass, p.count = None, count
        return p

    lib, rep = fb.library(), fb.Report()
    pin, pout = parts(src), parts(dst)
    assert lib.fl_topology_from_particles(ctx.handle, ctypes.byref(pin), None, ctypes.byref(rep)) == fb.OK
    assert lib.fl_sort_particles_by_block(ctx.handle, ctypes.byref(pin), ctypes.byref(pout), None,
                                          ctypes.byref(rep)) == fb.OK
    blocks = ctx.active_blocks()
    nb = len(blocks)
    # the FP64 face masses; a threshold between two well-separated masses
    x, v, c = soa_to_xvc(soa)
    box = box_for(n)
    fm, fq = oracle.p2g(box, x, v, c, mass)
    masses = np.unique(np.concatenate([a[a > 0] for a in fm]))
    gaps = np.nonzero(masses[1:] > masses[:-1] * (1 + 1e-3))[0]
    k = gaps[np.searchsorted(gaps, len(masses) // 4)]
    m_min = 0.5 * (masses[k] + masses[k + 1])
    tp = fb.transfer_params(scenes.DT, mass, min_face_mass=m_min)
    u = [torch.zeros(nb * 512, device="cuda") for _ in range(3)]
    fmass = [torch.zeros(nb * 512, device="cuda") for _ in range(3)]
    val = [torch.full((nb * 512,), 200, dtype=torch.uint8, device="cuda") for _ in range(3)]
    arr = lambda ts: (ctypes.c_void_p * 3)(*[t.data_ptr() for t in ts])
    assert lib.fl_p2g_normalized(ctx.handle, ctypes.byref(pout), ctypes.byref(tp), arr(u), arr(fmass), arr(val), None,
                                 ctypes.byref(rep)) == fb.OK and rep.error == 0
    want_u, want_val = oracle.normalize_forces(box, fm, fq, m_min, scenes.DT, scenes.GRAVITY)
    seen = set()
    for a in range(3):
        got = fb.sparse_faces_to_dense(blocks, val[a].cpu().numpy(), (n, n, n), a, fill=255)
        have = got != 255
        np.testing.assert_array_equal(got[have], want_val[a][have])
        assert np.all(want_val[a][~have] == 0)  # faces outside the active blocks have no mass
        seen |= set(np.unique(got[have]).tolist())
    assert seen == {0, 1, 3}
    ctx.close()
