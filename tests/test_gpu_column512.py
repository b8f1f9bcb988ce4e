"""The 512^3 column drop (column [0.1,0.3]x[0.1,0.8]x[0.1,0.3] falling into a
pool y <= 0.15, 8 particles per fluid cell, ~190M particles) at full size.

Checked on the device with torch as the checker: the step's sort is the stable
cell order of its input; every projection meets the FP64 gate of 1e-6 ||b||
(the solver's own FP64 true residual) and the reference's gate; two runs from
the same state are bitwise equal. One step is also replayed by the FP64 oracle
on a 64^3 sub-box that holds the pool surface and the foot of the column: the
oracle deposits the sub-box's particles, corrects with the GPU's pressure and
gathers, and the faces and particles far enough inside the sub-box that only
those particles reach them are compared at 1e-5."""

import numpy as np
import pytest

import fluidity_b200 as fb
import oracle
from fluidity_b200 import scenes
from helpers import device_cell_order, state_views

pytestmark = pytest.mark.gpu

N = 512
SUB_LO = (96, 48, 96)  # cells; the sub-box spans 64 cells on each axis
SUB_N = 64


@pytest.fixture(scope="module")
def column():
    return scenes.column_drop(N)


def test_column_512_sort_is_the_stable_cell_order(column):
    import torch

    soa, mass = column
    assert np.all(soa[3:] == 0.0)  # the scene starts at rest
    ctx = fb.LiquidContext(N, capacity=soa.shape[1])
    ctx.upload(soa)
    x_in = [torch.from_numpy(soa[d]).cuda() for d in range(3)]
    # at rest and without gravity the velocities stay zero and positions move only by the wall clamp
    code, _ = ctx.step(fb.transfer_params(1e-6, mass, gravity=(0, 0, 0)), fb.default_pressure_options(precision=1))
    assert code == fb.OK
    perm = device_cell_order(x_in, N)
    out = state_views(ctx)
    for d in range(3):
        assert float((out[d] - x_in[d][perm]).abs().max()) <= 1.01e-3 / N
    ctx.close()


def _sub_fields(ctx, lo, n):
    """The GPU's step fields on the sub-box: dense u_pred, u_new (n+1 along the
    normal), cell pressure and cell type (255 outside the active blocks)."""
    blocks = ctx.active_blocks()
    f = ctx.fields()
    nb = len(blocks)
    lo = np.array(lo)
    sel = np.nonzero(np.all((blocks * 8 + 8 > lo) & (blocks * 8 <= lo + n), axis=1))[0]
    local = blocks[sel] * 8 - lo  # block origin in sub-box cells (may be negative)
    loc = np.arange(512)
    lx, ly, lz = loc & 7, (loc >> 3) & 7, loc >> 6
    gx = (local[:, 0:1] + lx).ravel()
    gy = (local[:, 1:2] + ly).ravel()
    gz = (local[:, 2:3] + lz).ravel()
    idx = (sel[:, None] * 512 + loc[None, :]).ravel()

    def pick(ptr, dtype):
        import torch

        from helpers import device_view

        v = device_view(ptr, nb * 512, dtype)
        return v[torch.from_numpy(idx).cuda()].cpu().numpy()

    out = {}
    for name in ("u_pred", "u_new"):
        arrs = []
        for a in range(3):
            shape = [n, n, n]
            shape[2 - a] += 1
            dense = np.full(shape, np.nan, np.float32)
            val = pick(f[name][a], np.float32)
            ok = (gx >= 0) & (gy >= 0) & (gz >= 0) & (gx < shape[2]) & (gy < shape[1]) & (gz < shape[0])
            dense[gz[ok], gy[ok], gx[ok]] = val[ok]
            arrs.append(dense)
        out[name] = arrs
    ok = (gx >= 0) & (gy >= 0) & (gz >= 0) & (gx < n) & (gy < n) & (gz < n)
    p = np.full((n, n, n), np.nan)
    p[gz[ok], gy[ok], gx[ok]] = pick(f["pressure"], np.float64)[ok]
    t = np.full((n, n, n), 255, np.uint8)
    t[gz[ok], gy[ok], gx[ok]] = pick(f["cell_type"], np.uint8)[ok]
    out["pressure"], out["cell_type"] = p, t
    return out


def test_column_512_gate_repeat_and_subbox_replay(column):
    import torch

    soa, mass = column
    tp = fb.transfer_params(scenes.DT, mass)
    opt = fb.default_pressure_options(precision=1, warm_start=1)
    ctx = fb.LiquidContext(N, capacity=soa.shape[1])
    runs = []
    for run in range(2):
        ctx.upload(soa)
        for k in range(3):
            if run == 0 and k == 2:
                before = [t.clone() for t in state_views(ctx)]
            code, d = ctx.step(tp, opt)
            assert code == fb.OK
            assert d.relative_residual <= 1e-6 and d.true_residual_l2 <= d.reference_limit, d.as_dict()
        if run == 0:
            fields = _sub_fields(ctx, SUB_LO, SUB_N)
        runs.append([t.clone() for t in state_views(ctx)])
    for a, b in zip(*runs):
        assert torch.equal(a, b)
    after = runs[0]
    ctx.close()
    # FP64 replay of the third step on the sub-box
    lo, n = np.array(SUB_LO), SUB_N
    cell = [torch.floor(before[d] * np.float32(N)).to(torch.int64) for d in range(3)]
    inside = torch.ones_like(cell[0], dtype=torch.bool)
    for d in range(3):
        inside &= (cell[d] >= int(lo[d]) + 1) & (cell[d] <= int(lo[d]) + n - 2)
    sel = torch.nonzero(inside).squeeze(1)
    state = torch.stack([t[sel] for t in before]).cpu().numpy()
    box = oracle.Box.make([0.0, 0.0, 0.0], 1.0 / N, lo, [n, n, n])
    r = oracle.step_replay(box, state, np.nan_to_num(fields["pressure"]), scenes.DT, stride=1)
    # faces whose stencil particles are all in the sub-box, particles whose stencil faces are all such faces
    errs = {}
    for a in range(3):
        shape = r["u_pred"][a].shape
        kk, jj, ii = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
        inner = np.ones(shape, bool)
        for c, dd in ((ii, 0), (jj, 1), (kk, 2)):
            inner &= (c >= 3) & (c <= n - 3)
        have = inner & ~np.isnan(fields["u_pred"][a])
        for name in ("u_pred", "u_new"):
            g, w = fields[name][a][have].astype(np.float64), r[name][a][have]
            errs[f"{name}{a}"] = float(np.abs(g - w).max() / max(np.abs(w).max(), 1e-300))
    known = (fields["cell_type"] != 255)[2:-2, 2:-2, 2:-2]
    assert np.array_equal(fields["cell_type"][2:-2, 2:-2, 2:-2][known], r["cell_type"][2:-2, 2:-2, 2:-2][known])
    # the GPU wrote the step's output in the stable cell order of `before`
    perm = device_cell_order(before[:3], N)
    where = torch.empty_like(perm)
    where[perm] = torch.arange(len(perm), device="cuda")
    c_sel = np.floor(state[0:3].T.astype(np.float32) * np.float32(N)).astype(np.int64)
    deep = np.all((c_sel >= lo + 4) & (c_sel <= lo + n - 5), axis=1)
    got_idx = where[sel[torch.from_numpy(np.nonzero(deep)[0]).cuda()]]
    got = torch.stack([t[got_idx] for t in after]).cpu().numpy().T.astype(np.float64)
    want = r["sample"][deep]
    for name, sl in (("x", slice(0, 3)), ("v", slice(3, 6)), ("C", slice(6, 15))):
        errs[name] = float(np.abs(got[:, sl] - want[:, sl]).max() / max(np.abs(want[:, sl]).max(), 1e-300))
    print(f"column drop 512 sub-box step 3: {errs}, {int(deep.sum())} particles, {len(state[0])} deposited")
    assert deep.sum() > 100000
    for k, e in errs.items():
        assert e <= 1e-5, (k, errs)
