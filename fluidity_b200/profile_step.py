"""Runs a few liquid substeps of a seeded scene, for profiling (ncu, CUDA events).

    python -m fluidity_b200.profile_step --scene splash --grid 256 --steps 2 [--precision 1] [--levels 0]
        [--warm-start 1] [--inner-rtol 1e-3] [--snapshot] [--unet N]
    python -m fluidity_b200.profile_step --train-batch 256 [--train-reps 20]

Prints, per step, the status, FCG iterations, FP64 relative residual, the
CUDA-event phase times (topology+sort, P2G, pressure, G2P; ms) and the running
kernel-launch counts. With --snapshot every step's state also goes through the
asynchronous snapshot queue (device check + D2H), whose copy time is printed.
With --unet N the learned preconditioner (He-uniform weights, seed 1) is then
applied to a random vector on the last step's cells through the tensor-core
kernels: 3 untimed applications, then N timed with CUDA events.
With --train-batch B no scene is run: one training forward + backward of the
learned preconditioner on B random items (He-uniform weights, seed 1) is timed
with the FP32 convolution kernels and with the tensor-core convolutions, 3
untimed then --train-reps timed with CUDA events each.
"""

from __future__ import annotations

import argparse

import fluidity_b200 as fb
from fluidity_b200 import scenes


def time_training(batch: int, reps: int):
    import torch

    gen = torch.Generator(device="cuda").manual_seed(0)
    params = torch.empty(fb.UNet.param_count(), dtype=torch.float32, device="cuda")
    fb.UNet.init_params(params, 1)
    x = torch.randn((batch, 2000), generator=gen, device="cuda")
    gy = torch.randn((batch, 512), generator=gen, device="cuda")
    y = torch.empty((batch, 512), device="cuda")
    grads = torch.empty_like(params)
    for tc in (False, True):
        net = fb.UNet(batch, tensor_cores=tc)
        for _ in range(3):
            net.forward(params, x, y)
            net.backward(params, gy, grads)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            net.forward(params, x, y)
            net.backward(params, gy, grads)
        e1.record()
        torch.cuda.synchronize()
        net.close()
        print(f"training forward+backward, {batch} items, {'tensor cores' if tc else 'FP32 kernels'}: "
              f"{e0.elapsed_time(e1) / reps:.3f} ms", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="splash", choices=sorted(scenes.SCENES))
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--levels", type=int, default=0)
    ap.add_argument("--warm-start", type=int, default=1)
    ap.add_argument("--inner-rtol", type=float, default=1e-3)
    ap.add_argument("--snapshot", action="store_true")
    ap.add_argument("--unet", type=int, default=0)
    ap.add_argument("--train-batch", type=int, default=0)
    ap.add_argument("--train-reps", type=int, default=20)
    args = ap.parse_args()
    if args.train_batch > 0:
        return time_training(args.train_batch, args.train_reps)
    soa, mass = scenes.SCENES[args.scene](args.grid)
    ctx = fb.LiquidContext(args.grid, capacity=soa.shape[1])
    ctx.upload(soa)
    tp = fb.transfer_params(scenes.DT, mass)
    opt = fb.default_pressure_options(precision=args.precision, levels=args.levels, warm_start=args.warm_start,
                                      inner_rtol=args.inner_rtol)
    queue = fb.SnapshotQueue(ctx) if args.snapshot else None
    for s in range(args.steps):
        code, d = ctx.step(tp, opt)
        print(s, code, d.iterations, f"{d.relative_residual:.3e}", ctx.step_timings().round(4).tolist(),
              fb.kernel_launches(), flush=True)
        if queue is not None:
            t = queue.begin(s + 1, s + 1, (s + 1) * scenes.DT)
            queue.wait(t)
            _, view = queue.finish(t)
            print("  snapshot", view.count, f"{view.copy_ms:.3f} ms", flush=True)
            queue.release(t)
    if queue is not None:
        queue.close()
    if args.unet > 0:
        import torch

        params = torch.empty(fb.UNet.param_count(), dtype=torch.float32, device="cuda")
        fb.UNet.init_params(params, 1)
        ctx.set_learned_preconditioner(params)
        nb = len(ctx.active_blocks())
        r = torch.randn(nb * 512, device="cuda", generator=torch.Generator(device="cuda").manual_seed(0))
        z = torch.zeros_like(r)
        for _ in range(3):
            ctx.apply_learned(r, z, kernels=0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.unet):
            ctx.apply_learned(r, z, kernels=0)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.unet
        print(f"unet {nb} blocks {ms:.4f} ms per application, {nb * 25.6e6 / (ms * 1e-3) / 1e12:.1f} TFLOP/s",
              flush=True)
    ctx.close()


if __name__ == "__main__":
    main()
