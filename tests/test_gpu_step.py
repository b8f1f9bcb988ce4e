"""GPU parity of the full liquid substep (sort -> P2G + normalize + gravity ->
MGPCG projection -> G2P + advection) against the FP64 oracle on the seeded dam
break, at 32^3 (steps 1 and 10, oracle replayed from the GPU state) and 128^3.

Tolerances: grid and particle fields 1e-5 norm-wise relative (FP32 transfers
vs FP64 oracle); pressure 1e-5 relative (both solves stop at a 1e-6 relative
FP64 residual); the GPU pressure's own FP64 residual, re-evaluated by the
oracle, <= 1e-6 ||b||."""

import ctypes

import numpy as np
import pytest

import fluidity_b200 as fb
import oracle
from fluidity_b200 import scenes
from helpers import box_for, dam_break_context, read_fields, rel_err, soa_to_xvc, sort_permutation
from oracle.box_system import box_pressure_system

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _compare_step(ctx, n, state_in, precision=0, levels=0, pre=1, post=2):
    """Runs one GPU step from state_in and one oracle step; returns errors."""
    ctx.upload(state_in)
    code, diag = ctx.step(fb.transfer_params(scenes.DT, scenes.DENSITY / n ** 3 / 8),
                          fb.default_pressure_options(precision=precision, levels=levels, pre=pre, post=post))
    assert code == fb.OK, diag.as_dict()
    f = read_fields(ctx, n)
    out = ctx.download()
    x, v, c = soa_to_xvc(state_in)
    box = box_for(n)
    r = oracle.step(box, x, v, c, scenes.DT)
    perm = sort_permutation(state_in, n)
    errs = {}
    for a in range(3):
        have = ~np.isnan(f["u_pred"][a])
        errs[f"u_pred{a}"] = rel_err(f["u_pred"][a], r["u_pred"][a], have)
        errs[f"u_new{a}"] = rel_err(f["u_new"][a], r["u_new"][a], have)
    fluid = r["cell_type"] == 1
    known = f["cell_type"] != 255
    assert np.array_equal(f["cell_type"][known], r["cell_type"][known])
    assert not np.any(fluid & ~known)
    errs["pressure"] = rel_err(f["pressure"], r["pressure"], fluid)
    errs["x"] = float(np.abs(out[0:3].T - r["x"][perm]).max() / n)  # in cells
    errs["v"] = rel_err(out[3:6].T, r["v"][perm])
    errs["C"] = rel_err(out[6:15].T, r["c"][perm])
    return errs, diag, f, out


@pytest.mark.parametrize("precision", [0, 1])
def test_dam_break_32_first_step_matches_oracle(precision):
    ctx, soa, _ = dam_break_context(32)
    errs, diag, _, _ = _compare_step(ctx, 32, soa, precision)
    assert diag.relative_residual <= 1e-6
    for k, e in errs.items():
        assert e <= TOL, (k, e, errs)


def test_dam_break_32_step_10_matches_oracle_replay():
    ctx, soa, m = dam_break_context(32)
    tp = fb.transfer_params(scenes.DT, m)
    opt = fb.default_pressure_options()
    for _ in range(9):
        code, _ = ctx.step(tp, opt)
        assert code == fb.OK
    state9 = ctx.download()
    errs, diag, _, _ = _compare_step(ctx, 32, state9)
    for k, e in errs.items():
        assert e <= TOL, (k, e, errs)


def test_dam_break_32_step_100_matches_oracle_replay():
    """Config 1 runs 100 steps: the 100th step, replayed by the oracle from the GPU state."""
    ctx, soa, m = dam_break_context(32)
    tp = fb.transfer_params(scenes.DT, m)
    opt = fb.default_pressure_options()
    for _ in range(99):
        code, _ = ctx.step(tp, opt)
        assert code == fb.OK
    errs, diag, _, _ = _compare_step(ctx, 32, ctx.download())
    assert diag.relative_residual <= 1e-6
    for k, e in errs.items():
        assert e <= TOL, (k, e, errs)


def test_dam_break_128_steps_10_and_200_match_oracle_replay():
    """Config 2 (128^3, 4-level V-cycle): steps 10 and 200, each replayed by the
    oracle from the GPU state of the step before."""
    ctx, soa, m = dam_break_context(128)
    tp = fb.transfer_params(scenes.DT, m)
    opt = fb.default_pressure_options(levels=4, pre=2, post=2)
    done = 0
    for check in (10, 200):
        while done < check - 1:
            code, _ = ctx.step(tp, opt)
            assert code == fb.OK
            done += 1
        errs, diag, _, _ = _compare_step(ctx, 128, ctx.download(), levels=4, pre=2, post=2)
        done += 1
        assert diag.relative_residual <= 1e-6
        for k, e in errs.items():
            assert e <= TOL, (check, k, e, errs)


def test_dam_break_128_first_step_matches_oracle():
    """128^3 with the 4-level V-cycle (2 pre + 2 post red-black sweeps)."""
    ctx, soa, _ = dam_break_context(128)
    errs, diag, _, _ = _compare_step(ctx, 128, soa, levels=4, pre=2, post=2)
    assert diag.levels == 4
    for k, e in errs.items():
        assert e <= TOL, (k, e, errs)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("warm_start", [0, 2])
def test_pressure_meets_fp64_residual_checked_by_oracle(precision, warm_start):
    """The GPU pressure, re-evaluated in FP64 by the oracle on the same system
    (built from the GPU's own predicted velocities), meets 1e-6 ||b||, and the
    reference's own gate is reported; from p = 0 and from the pressure
    extrapolated from the last two projections."""
    n = 64
    ctx, soa, m = dam_break_context(n)
    opt = fb.default_pressure_options(precision=precision, warm_start=warm_start)
    for _ in range(3):
        ctx.step(fb.transfer_params(scenes.DT, m), opt)
    code, diag = ctx.step(fb.transfer_params(scenes.DT, m), opt)
    assert code == fb.OK
    f = read_fields(ctx, n)
    box = box_for(n)
    u_pred = [np.nan_to_num(f["u_pred"][a].astype(np.float64)) for a in range(3)]
    ct = np.where(f["cell_type"] == 255, 2, f["cell_type"]).astype(np.uint8)
    sysm = box_pressure_system(box, ct, u_pred)
    ci = sysm["cells_idx"]
    p = f["pressure"][ci[:, 2], ci[:, 1], ci[:, 0]]
    ev = oracle.pressure_evaluate(sysm["cells_idx"], sysm["cells_val"], sysm["faces_idx"], sysm["faces_kind"],
                                  sysm["faces_val"], box.h, scenes.DT, p)
    assert ev["diag"]["true_residual_l2"] <= 1.0001e-6 * ev["diag"]["rhs_l2"]
    assert diag.true_residual_l2 == pytest.approx(ev["diag"]["true_residual_l2"], rel=1e-3)
    assert diag.true_residual_l2 <= diag.reference_limit


def test_step_is_bitwise_reproducible():
    ctx, soa, m = dam_break_context(32)
    tp, opt = fb.transfer_params(scenes.DT, m), fb.default_pressure_options()
    outs = []
    for _ in range(2):
        ctx.upload(soa)
        for _ in range(3):
            ctx.step(tp, opt)
        f = read_fields(ctx, 32)
        outs.append((ctx.download(), f["u_new"], f["pressure"]))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    for a in range(3):
        np.testing.assert_array_equal(outs[0][1][a], outs[1][1][a])
    np.testing.assert_array_equal(outs[0][2], outs[1][2])


@pytest.mark.parametrize("precision,tol", [(0, 1e-5), (1, 3e-2)])
@pytest.mark.parametrize("n,levels", [(32, 4), (64, 5)])
def test_vcycle_matches_fp64_restatement(precision, tol, n, levels):
    """One V-cycle against the FP64 restatement. At 64^3 with 5 levels the last
    dense level (8^3) and the coarsest (4^3) run in the one-CTA coarse tail."""
    ctx, soa, m = dam_break_context(n)
    ctx.step(fb.transfer_params(scenes.DT, m), fb.default_pressure_options())
    blocks = ctx.active_blocks()
    nb = len(blocks)
    f = read_fields(ctx, n)
    ct = np.where(f["cell_type"] == 255, 2, f["cell_type"]).astype(np.uint8)
    rng = np.random.default_rng(7)
    r_dense = rng.normal(size=ct.shape) * (ct == 1)
    # dense -> sparse layout
    loc = np.arange(512)
    gx = (blocks[:, 0:1] * 8 + (loc & 7)).ravel()
    gy = (blocks[:, 1:2] * 8 + ((loc >> 3) & 7)).ravel()
    gz = (blocks[:, 2:3] * 8 + (loc >> 6)).ravel()
    r_sparse = r_dense[gz, gy, gx].astype(np.float32)
    lib = fb.library()
    import torch
    r_dev = torch.from_numpy(r_sparse).cuda()
    z_dev = torch.zeros_like(r_dev)
    opt = fb.default_pressure_options(precision=precision, levels=levels)
    assert lib.fl_apply_vcycle(ctx.handle, ctypes.c_void_p(r_dev.data_ptr()), ctypes.c_void_p(z_dev.data_ptr()),
                               ctypes.byref(opt), None) == fb.OK
    torch.cuda.synchronize()
    z = fb.sparse_cells_to_dense(blocks, z_dev.cpu().numpy(), (n, n, n))
    zo = oracle.vcycle(box_for(n), ct, r_dense, levels=levels, pre=opt.pre_sweeps, post=opt.post_sweeps,
                       coarse_sweeps=opt.coarse_sweeps)
    assert rel_err(z, zo, ct == 1) <= tol


def test_sort_is_a_stable_cell_permutation():
    n = 32
    ctx, soa, m = dam_break_context(n)
    rng = np.random.default_rng(3)
    shuffled = soa[:, rng.permutation(soa.shape[1])].copy()
    ctx.upload(shuffled)
    ctx.step(fb.transfer_params(0.0, m, gravity=(0, 0, 0)), fb.default_pressure_options())
    out = ctx.download()
    perm = sort_permutation(shuffled, n)
    # dt = 0: positions only move by the wall clamp (<= 1e-3 h); the order is the stable cell sort
    np.testing.assert_allclose(out[0:3], shuffled[0:3, perm], rtol=0, atol=1.01e-3 / n)
    f = ctx.fields()
    nb = len(ctx.active_blocks())
    cs = fb.copy_to_host(f["cell_start"], nb * 512 + 1, np.int32)
    assert cs[0] == 0 and cs[-1] == soa.shape[1] and np.all(np.diff(cs) >= 0)


def test_sort_handles_crowded_blocks():
    """A block holding more particles than the sort stages in shared memory
    (12,288) sorts its cells in place; the order is still the stable cell sort,
    next to a block that takes the staged path."""
    n = 32
    rng = np.random.default_rng(5)
    crowded, normal = 20000, 3000
    x = np.concatenate([rng.uniform(8.0 / n, 16.0 / n, size=(3, crowded)),
                        rng.uniform([[16.0 / n], [8.0 / n], [8.0 / n]], [[24.0 / n], [16.0 / n], [16.0 / n]],
                                    size=(3, normal))], axis=1)
    soa = np.zeros((15, crowded + normal), np.float32)
    soa[0:3] = x[:, rng.permutation(x.shape[1])]
    soa[3:6] = rng.normal(scale=0.1, size=(3, soa.shape[1]))
    ctx = fb.LiquidContext(n, capacity=soa.shape[1])
    ctx.upload(soa)
    code, diag = ctx.step(fb.transfer_params(0.0, 1.0 / (8 * n ** 3), gravity=(0, 0, 0)),
                          fb.default_pressure_options())
    assert code == fb.OK
    out = ctx.download()
    perm = sort_permutation(soa, n)
    np.testing.assert_array_equal(out[0:3], soa[0:3, perm])  # dt = 0, far from the walls: x unchanged
    f = ctx.fields()
    nb = len(ctx.active_blocks())
    cs = fb.copy_to_host(f["cell_start"], nb * 512 + 1, np.int32)
    assert cs[0] == 0 and cs[-1] == soa.shape[1] and np.all(np.diff(cs) >= 0)
    ctx.close()


def test_empty_and_invalid_particles():
    ctx = fb.LiquidContext(32, capacity=64)
    ctx.upload(np.zeros((15, 0), np.float32))
    code, diag = ctx.step(fb.transfer_params(scenes.DT, 1.0), fb.default_pressure_options())
    assert code == fb.OK
    bad = np.zeros((15, 2), np.float32)
    bad[0:3] = 0.5
    bad[0, 1] = 2.0  # outside the box lattice
    ctx.upload(bad)
    with pytest.raises(fb.FluidityError) as e:
        ctx.step(fb.transfer_params(scenes.DT, 1.0), fb.default_pressure_options())
    assert e.value.code == fb.FAILED_PRECONDITION
    bad[0, 1] = np.nan
    ctx.upload(bad)
    with pytest.raises(fb.FluidityError) as e:
        ctx.step(fb.transfer_params(scenes.DT, 1.0), fb.default_pressure_options())
    assert e.value.code == fb.OUT_OF_RANGE
    with pytest.raises(fb.FluidityError) as e:
        ctx.upload(np.zeros((15, 65), np.float32))
    assert e.value.code == fb.RESOURCE_EXHAUSTED
