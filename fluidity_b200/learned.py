"""Training driver of the learned block preconditioner.

Pairs come from the context's own MGPCG solves (fl_collect_training_pairs):
for a dam-break state, the converged pressure p* and the iterates p_k stopped
after k flexible-CG iterations give, per block holding fluid, the input
(r_k / s, cell mask) on the block plus a one-cell halo and the target
(p* - p_k) / s, s = max |r_k| over the window. Training runs entirely in the
library's kernels (fl_unet_forward / fl_unet_backward / fl_unet_block_residual_loss
or fl_unet_masked_mse / fl_adam_step) on batches of 64 items with Adam at lr
1e-3, the convolutions as BF16 tensor-core GEMMs with FP32 accumulation. The default loss is the block residual |r_b - A_b y|^2 / |r_b|^2: the
network learns to invert the pressure operator on its block, a target it can
see in its window (the error p* - p_k is dominated by global modes that a
block-local network cannot see, and training on it ends at the zero
predictor). torch only holds the device buffers and draws the batch indices.

    python -m fluidity_b200.learned --grid 128 --pairs 10000 --steps 2000 --out weights.npy
"""

from __future__ import annotations

import argparse
import time

import numpy as np

import fluidity_b200 as fb
from fluidity_b200 import scenes

DEFAULT_CAPS = (0, 1, 2, 3, 4, 5, 6, 8, 10, 12)


def collect_pairs(n: int = 128, pairs: int = 10000, steps_between: int = 4, caps=DEFAULT_CAPS, precision: int = 0,
                  seed_steps: int = 2, max_states: int = 40, after_vcycle: bool = False):
    """Dam break at n^3 (the 8-particles-per-cell scene); after `seed_steps` steps and
    then every `steps_between` steps, adds the pairs of that step's projection until
    `pairs` items are collected. after_vcycle: the inputs are the residuals left by
    one V-cycle (what the composite preconditioner's network sees). Returns device
    tensors (inputs, targets, masks)."""
    import torch

    soa, m = scenes.dam_break(n)
    ctx = fb.LiquidContext(n, capacity=soa.shape[1])
    ctx.upload(soa)
    params = fb.transfer_params(scenes.DT, m)
    opt = fb.default_pressure_options(precision=precision)
    collect = fb.default_pressure_options(precision=precision)
    collect.preconditioner = 2 if after_vcycle else 0
    inputs = torch.zeros((pairs, 2, 10, 10, 10), dtype=torch.float32, device="cuda")
    targets = torch.zeros((pairs, 512), dtype=torch.float32, device="cuda")
    masks = torch.zeros((pairs, 512), dtype=torch.float32, device="cuda")
    got = 0
    for _ in range(seed_steps):
        ctx.step(params, opt)
    for _ in range(max_states):
        if got >= pairs:
            break
        got += ctx.collect_training_pairs(params, collect, list(caps), inputs[got:], targets[got:], masks[got:])
        for _ in range(steps_between):
            ctx.step(params, opt)
    ctx.close()
    return inputs[:got], targets[:got], masks[:got]


def train(inputs, targets, masks, steps: int = 2000, batch: int = 64, lr: float = 1e-3, seed: int = 0,
          params=None, loss_kind: str = "residual", tensor_cores: bool = True):
    """Adam on batches of the pairs; returns (params, losses per step).
    tensor_cores: the 3x3x3 convolutions of the forward and backward passes as BF16 GEMMs
    with FP32 accumulation on the tensor cores (the configured training precision); False
    runs them in FP32 kernels.
    loss_kind "residual": |r_b - A_b y|^2 / |r_b|^2 per item (fl_unet_block_residual_loss: the network
    learns the inverse of the pressure operator on its block; the zero output scores 1);
    "error": the per-item relative squared error against the targets p* - p_k (fl_unet_masked_mse)."""
    import torch

    n = inputs.shape[0]
    batch = min(batch, n)
    net = fb.UNet(batch, tensor_cores=tensor_cores)
    P = params if params is not None else torch.empty(fb.UNet.param_count(), dtype=torch.float32, device="cuda")
    if params is None:
        fb.UNet.init_params(P, seed)
    G = torch.zeros_like(P)
    M = torch.zeros_like(P)
    V = torch.zeros_like(P)
    y = torch.zeros((batch, 512), dtype=torch.float32, device="cuda")
    gy = torch.zeros_like(y)
    loss = torch.zeros(steps, dtype=torch.float32, device="cuda")
    gen = torch.Generator(device="cpu").manual_seed(seed)
    order = torch.randperm(n, generator=gen)
    pos = 0
    xb = torch.empty((batch, 2, 10, 10, 10), dtype=torch.float32, device="cuda")
    tb = torch.empty((batch, 512), dtype=torch.float32, device="cuda")
    mb = torch.empty((batch, 512), dtype=torch.float32, device="cuda")
    for step in range(1, steps + 1):
        if pos + batch > n:
            order = torch.randperm(n, generator=gen)
            pos = 0
        idx = order[pos:pos + batch].to("cuda")
        pos += batch
        torch.index_select(inputs, 0, idx, out=xb)
        torch.index_select(targets, 0, idx, out=tb)
        torch.index_select(masks, 0, idx, out=mb)
        net.forward(P, xb, y)
        if loss_kind == "residual":
            fb.UNet.block_residual_loss(y, xb, loss[step - 1:step], gy)
        else:
            fb.UNet.masked_mse(y, tb, mb, loss[step - 1:step], gy, relative=1)
        net.backward(P, gy, G)
        fb.UNet.adam_step(P, G, M, V, step, lr=lr)
    torch.cuda.synchronize()
    net.close()
    return P, loss.cpu().numpy()


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--pairs", type=int, default=10000)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--out", default="")
    a = ap.parse_args()
    t0 = time.time()
    x, t, m = collect_pairs(a.grid, a.pairs)
    t1 = time.time()
    P, losses = train(x, t, m, a.steps)
    t2 = time.time()
    print(f"pairs {x.shape[0]} in {t1 - t0:.1f} s; {a.steps} Adam steps in {t2 - t1:.1f} s; "
          f"loss first {losses[:20].mean():.4g} last {losses[-20:].mean():.4g}")
    if a.out:
        np.save(a.out, P.cpu().numpy())
    del torch


if __name__ == "__main__":
    main()
