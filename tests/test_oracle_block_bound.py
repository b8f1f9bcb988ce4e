"""What a block-local correction can add to the V-cycle, on the CPU.

The learned preconditioner maps the residual on one 8^3 block (plus a one-cell
halo) to a correction on that block, so the best it can do is the exact solve
of the pressure operator restricted to the block. This test runs flexible CG
(FP64, numpy) on the 64^3 dam break's first projection with the FP64
restatement of the GPU's V-cycle (oracle.vcycle) as the preconditioner, and
with the V-cycle followed by exact 8^3 block solves of its residual: the block
solves save at most one iteration, and on their own they need an order of
magnitude more. This bounds what any block-local network can gain over the
V-cycle on these scenes."""

import numpy as np
import pytest

import oracle
from fluidity_b200 import scenes
from helpers import box_for, soa_to_xvc

sp = pytest.importorskip("scipy.sparse")
spla = pytest.importorskip("scipy.sparse.linalg")


def _system(n):
    soa, m = scenes.dam_break(n)
    x, v, c = soa_to_xvc(soa)
    box = box_for(n)
    r = oracle.step(box, x, v, c, scenes.DT)
    fm, fq = oracle.p2g(box, r["x"], r["v"], r["c"], m)
    u, _ = oracle.normalize_forces(box, fm, fq, 0.0, scenes.DT, scenes.GRAVITY)
    ct = oracle.classify_cells(box, r["x"])
    fluid = ct == 1
    idx = -np.ones(ct.shape, int)
    idx[fluid] = np.arange(fluid.sum())
    K, J, I = np.nonzero(fluid)
    rows, cols, vals = [], [], []
    diag = np.zeros(len(K))
    for dk, dj, di in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        t = ct[K + dk, J + dj, I + di]
        f = t == 1
        rows += list(idx[K, J, I][f])
        cols += list(idx[(K + dk)[f], (J + dj)[f], (I + di)[f]])
        vals += [-1.0] * int(f.sum())
        diag += (t == 1) + (t == 2)  # unit conductance to fluid and air, none to solid
    N = len(K)
    A = sp.csr_matrix((vals + list(diag), (rows + list(range(N)), cols + list(range(N)))), shape=(N, N))
    for a in range(3):  # stationary walls, as the step applies them
        kk, jj, ii = np.meshgrid(*[np.arange(s) for s in u[a].shape], indexing="ij")
        head, tail = [ii, jj, kk], [ii.copy(), jj.copy(), kk.copy()]
        tail[a] = tail[a] - 1

        def typ(q):
            ok = (q[0] >= 0) & (q[1] >= 0) & (q[2] >= 0) & (q[0] < n) & (q[1] < n) & (q[2] < n)
            t = np.zeros(q[0].shape, int)
            t[ok] = ct[q[2][ok], q[1][ok], q[0][ok]]
            return t

        u[a][(typ(head) == 0) | (typ(tail) == 0)] = 0.0
    ux, uy, uz = u
    div = (ux[:, :, 1:] - ux[:, :, :-1]) + (uy[:, 1:, :] - uy[:, :-1, :]) + (uz[1:, :, :] - uz[:-1, :, :])
    b = -div[fluid]
    return box, ct, fluid, (K, J, I), A, b


def _fcg(A, b, prec, tol=1e-6, maxit=500):
    x, r = np.zeros_like(b), b.copy()
    bn, last, it = np.linalg.norm(b), None, 0
    while np.linalg.norm(r) > tol * bn and it < maxit:
        z = prec(r)
        d = z.copy()
        if last is not None:
            d -= (z @ last[1]) / last[2] * last[0]
        q = A @ d
        dq = d @ q
        alpha = (d @ r) / dq
        x += alpha * d
        r -= alpha * q
        last, it = (d, q, dq), it + 1
    return it


def test_exact_block_solves_add_at_most_one_iteration_to_the_vcycle():
    n = 64
    box, ct, fluid, (K, J, I), A, b = _system(n)

    def vcycle(r):
        dense = np.zeros(ct.shape)
        dense[fluid] = r
        return oracle.vcycle(box, ct, dense, levels=4)[fluid]

    blk = (K // 8) * (n // 8) ** 2 + (J // 8) * (n // 8) + I // 8
    solves = []
    for bb in np.unique(blk):
        ids = np.nonzero(blk == bb)[0]
        solves.append((ids, spla.splu(A[ids][:, ids].tocsc())))

    def block(r):
        z = np.zeros_like(r)
        for ids, lu in solves:
            z[ids] = lu.solve(r[ids])
        return z

    def composite(r):
        z = vcycle(r)
        return z + block(r - A @ z)

    it_v, it_c, it_b = _fcg(A, b, vcycle), _fcg(A, b, composite), _fcg(A, b, block)
    print(f"64^3 dam break: V-cycle {it_v}, V-cycle + exact block solves {it_c}, block solves alone {it_b}")
    assert it_v - 1 <= it_c <= it_v
    assert it_b >= 5 * it_v
