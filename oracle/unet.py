"""FP64 numpy oracle of the learned block preconditioner (test infrastructure).

No reference counterpart exists (FluidiTy has no learned pressure solver); this
is the checker for the CUDA forward/backward/Adam kernels in
fluidity_b200/csrc/fl_unet.cu. Parity here is "unpinned" by the reference: it
pins the CUDA kernels to this restatement and to finite differences.

Network (per 8^3 block, input 10^3 = block + 1-cell halo, 2 channels):
    e1a = relu(conv3(x, 2->16, valid))            10^3 -> 8^3
    s1  = relu(conv3(e1a, 16->16, same))          8^3
    p1  = avgpool2(s1)                            4^3
    e2a = relu(conv3(p1, 16->32, same))
    s2  = relu(conv3(e2a, 32->32, same))          4^3
    p2  = avgpool2(s2)                            2^3
    bt  = relu(conv3(p2, 32->64, same))           2^3
    u2  = relu(conv1(up2(bt), 64->32) + s2)       4^3
    d2  = relu(conv3(u2, 32->32, same))
    u1  = relu(conv1(up2(d2), 32->16) + s1)       8^3
    d1  = relu(conv3(u1, 16->16, same))
    y   = conv1(d1, 16->1)                        8^3
Layout: activations [batch, channel, z, y, x]; a conv3 weight is [Cout, Cin, 3, 3, 3]
(taps in (dz, dy, dx) order), a conv1 weight [Cout, Cin]; parameters are flattened
layer by layer as weight then bias.
"""

from __future__ import annotations

import numpy as np

LAYERS = [  # name, kind, cin, cout
    ("e1a", "conv3v", 2, 16),
    ("e1b", "conv3", 16, 16),
    ("e2a", "conv3", 16, 32),
    ("e2b", "conv3", 32, 32),
    ("bt", "conv3", 32, 64),
    ("u2", "conv1", 64, 32),
    ("d2", "conv3", 32, 32),
    ("u1", "conv1", 32, 16),
    ("d1", "conv3", 16, 16),
    ("out", "conv1", 16, 1),
]


def layer_sizes():
    out = []
    for name, kind, cin, cout in LAYERS:
        k = 27 if kind.startswith("conv3") else 1
        out.append((name, cout * cin * k, cout))
    return out


def param_count():
    return sum(w + b for _, w, b in layer_sizes())


def unpack(theta):
    params, off = {}, 0
    for (name, kind, cin, cout), (_, nw, nb) in zip(LAYERS, layer_sizes()):
        k = (3, 3, 3) if kind.startswith("conv3") else ()
        params[name] = (theta[off:off + nw].reshape((cout, cin) + k), theta[off + nw:off + nw + nb])
        off += nw + nb
    return params


def pack(grads):
    return np.concatenate([np.concatenate([grads[name][0].ravel(), grads[name][1].ravel()]) for name, *_ in LAYERS])


def init_params(seed=0):
    """He-uniform weights from a seeded generator, zero biases (matches fl_unet_init_params' rule,
    not its random stream)."""
    rng = np.random.default_rng(seed)
    chunks = []
    for name, kind, cin, cout in LAYERS:
        fan_in = cin * (27 if kind.startswith("conv3") else 1)
        bound = np.sqrt(6.0 / fan_in)
        chunks.append(rng.uniform(-bound, bound, size=cout * cin * (27 if kind.startswith("conv3") else 1)))
        chunks.append(np.zeros(cout))
    return np.concatenate(chunks)


def _conv3(x, w, b, pad):
    n, cin, d, _, _ = x.shape
    cout = w.shape[0]
    xp = np.pad(x, ((0, 0), (0, 0), (pad, pad), (pad, pad), (pad, pad))) if pad else x
    do = xp.shape[2] - 2
    y = np.zeros((n, cout, do, do, do))
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                patch = xp[:, :, dz:dz + do, dy:dy + do, dx:dx + do]
                y += np.einsum("ncxyz,oc->noxyz", patch, w[:, :, dz, dy, dx])
    return y + b[None, :, None, None, None]


def _conv3_back(x, w, dy, pad):
    xp = np.pad(x, ((0, 0), (0, 0), (pad, pad), (pad, pad), (pad, pad))) if pad else x
    do = dy.shape[2]
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for dz in range(3):
        for dyy in range(3):
            for dx in range(3):
                patch = xp[:, :, dz:dz + do, dyy:dyy + do, dx:dx + do]
                dw[:, :, dz, dyy, dx] = np.einsum("ncxyz,noxyz->oc", patch, dy)
                dxp[:, :, dz:dz + do, dyy:dyy + do, dx:dx + do] += np.einsum("noxyz,oc->ncxyz", dy, w[:, :, dz, dyy, dx])
    dx_ = dxp[:, :, pad:-pad, pad:-pad, pad:-pad] if pad else dxp
    return dx_, dw, dy.sum(axis=(0, 2, 3, 4))


def _conv1(x, w, b):
    return np.einsum("ncxyz,oc->noxyz", x, w) + b[None, :, None, None, None]


def _conv1_back(x, w, dy):
    return np.einsum("noxyz,oc->ncxyz", dy, w), np.einsum("ncxyz,noxyz->oc", x, dy), dy.sum(axis=(0, 2, 3, 4))


def _pool(x):
    n, c, d, _, _ = x.shape
    return x.reshape(n, c, d // 2, 2, d // 2, 2, d // 2, 2).mean(axis=(3, 5, 7))


def _pool_back(dy):
    return np.repeat(np.repeat(np.repeat(dy, 2, 2), 2, 3), 2, 4) / 8.0


def _up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 2), 2, 3), 2, 4)


def _up_back(dy):
    n, c, d, _, _ = dy.shape
    return dy.reshape(n, c, d // 2, 2, d // 2, 2, d // 2, 2).sum(axis=(3, 5, 7))


def forward(theta, x):
    """x: (batch, 2, 10, 10, 10) -> y (batch, 1, 8, 8, 8) and the cache for backward."""
    P = unpack(theta)
    c = {"x": x}
    c["e1a"] = np.maximum(_conv3(x, *P["e1a"], 0), 0)
    c["s1"] = np.maximum(_conv3(c["e1a"], *P["e1b"], 1), 0)
    c["p1"] = _pool(c["s1"])
    c["e2a"] = np.maximum(_conv3(c["p1"], *P["e2a"], 1), 0)
    c["s2"] = np.maximum(_conv3(c["e2a"], *P["e2b"], 1), 0)
    c["p2"] = _pool(c["s2"])
    c["bt"] = np.maximum(_conv3(c["p2"], *P["bt"], 1), 0)
    c["ubt"] = _up(c["bt"])
    c["u2"] = np.maximum(_conv1(c["ubt"], *P["u2"]) + c["s2"], 0)
    c["d2"] = np.maximum(_conv3(c["u2"], *P["d2"], 1), 0)
    c["ud2"] = _up(c["d2"])
    c["u1"] = np.maximum(_conv1(c["ud2"], *P["u1"]) + c["s1"], 0)
    c["d1"] = np.maximum(_conv3(c["u1"], *P["d1"], 1), 0)
    y = _conv1(c["d1"], *P["out"])
    return y, c


def backward(theta, cache, dy):
    """Gradient of sum(dy * y) with respect to the flattened parameters."""
    P = unpack(theta)
    c = cache
    g = {}
    dd1, dw, db = _conv1_back(c["d1"], P["out"][0], dy)
    g["out"] = (dw, db)
    dd1 = dd1 * (c["d1"] > 0)
    du1, dw, db = _conv3_back(c["u1"], P["d1"][0], dd1, 1)
    g["d1"] = (dw, db)
    du1 = du1 * (c["u1"] > 0)
    ds1 = du1.copy()
    dud2, dw, db = _conv1_back(c["ud2"], P["u1"][0], du1)
    g["u1"] = (dw, db)
    dd2 = _up_back(dud2) * (c["d2"] > 0)
    du2, dw, db = _conv3_back(c["u2"], P["d2"][0], dd2, 1)
    g["d2"] = (dw, db)
    du2 = du2 * (c["u2"] > 0)
    ds2 = du2.copy()
    dubt, dw, db = _conv1_back(c["ubt"], P["u2"][0], du2)
    g["u2"] = (dw, db)
    dbt = _up_back(dubt) * (c["bt"] > 0)
    dp2, dw, db = _conv3_back(c["p2"], P["bt"][0], dbt, 1)
    g["bt"] = (dw, db)
    ds2 = (ds2 + _pool_back(dp2)) * (c["s2"] > 0)
    de2a, dw, db = _conv3_back(c["e2a"], P["e2b"][0], ds2, 1)
    g["e2b"] = (dw, db)
    de2a = de2a * (c["e2a"] > 0)
    dp1, dw, db = _conv3_back(c["p1"], P["e2a"][0], de2a, 1)
    g["e2a"] = (dw, db)
    ds1 = (ds1 + _pool_back(dp1)) * (c["s1"] > 0)
    de1a, dw, db = _conv3_back(c["e1a"], P["e1b"][0], ds1, 1)
    g["e1b"] = (dw, db)
    de1a = de1a * (c["e1a"] > 0)
    _, dw, db = _conv3_back(c["x"], P["e1a"][0], de1a, 0)
    g["e1a"] = (dw, db)
    return pack(g)


def masked_mse(y, target, mask, relative=False):
    """Loss and dL/dy of the masked squared error over items of 512 cells:
    global mean over masked cells, or (relative) the mean over the items with
    target energy sum m t^2 > 0 of sum m (y - t)^2 / sum m t^2."""
    y, target, mask = (np.asarray(a, np.float64).reshape(-1, 512) for a in (y, target, mask))
    d = (y - target) * mask
    if relative:
        energy = (mask * target * target).sum(axis=1, keepdims=True)
        valid = energy > 0
        w = np.where(valid, 1.0 / np.where(valid, energy, 1.0), 0.0) / max(1, int(valid.sum()))
    else:
        w = 1.0 / max(1.0, float(mask.sum()))
    return float((d * d * w).sum()), 2.0 * d * w


def block_operator(mask):
    """A_b of one item as a dense (512, 512) matrix over the block's cells: the
    level-0 pressure operator on the block's fluid cells (unit conductance to
    fluid and air neighbours, none to solid ones), the block's neighbours held
    at zero; rows and columns of non-fluid cells are zero. mask: (10, 10, 10)."""
    A = np.zeros((512, 512))
    for cz in range(8):
        for cy in range(8):
            for cx in range(8):
                c = (cz * 8 + cy) * 8 + cx
                if mask[cz + 1, cy + 1, cx + 1] != 1.0:
                    continue
                for dz, dy, dx in ((0, 0, -1), (0, 0, 1), (0, -1, 0), (0, 1, 0), (-1, 0, 0), (1, 0, 0)):
                    mk = mask[cz + 1 + dz, cy + 1 + dy, cx + 1 + dx]
                    if mk >= 0.0:
                        A[c, c] += 1.0
                    nz, ny, nx = cz + dz, cy + dy, cx + dx
                    if mk == 1.0 and 0 <= nz < 8 and 0 <= ny < 8 and 0 <= nx < 8:
                        A[c, (nz * 8 + ny) * 8 + nx] -= 1.0
    return A


def block_residual_loss(y, x):
    """Loss (1/V) sum |r_b - A_b y|^2 / max(|r_b|^2, 1) over the V items with
    r_b != 0 and its gradient with respect to y. y: (batch, 512); x: (batch, 2,
    10, 10, 10), the window scaled to max |r| = 1."""
    batch = y.shape[0]
    ops, rs = [], []
    for b in range(batch):
        mask = x[b, 1]
        r = np.where(mask == 1.0, x[b, 0], 0.0)[1:9, 1:9, 1:9].reshape(512)
        ops.append(block_operator(mask))
        rs.append(r)
    dens = np.array([r @ r for r in rs])
    valid = int((dens > 0).sum())
    loss, grad = 0.0, np.zeros_like(y, dtype=np.float64)
    for b in range(batch):
        if dens[b] <= 0:
            continue
        fluid = np.diag(ops[b]) > 0
        yb = np.where(fluid, y[b], 0.0)
        rho = np.where(fluid, rs[b] - ops[b] @ yb, 0.0)
        den = valid * max(dens[b], 1.0)
        loss += (rho @ rho) / den
        grad[b] = -2.0 * (ops[b] @ rho) / den
    return loss, grad


def adam(theta, grad, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v
