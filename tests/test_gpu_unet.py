"""GPU checks of the learned block preconditioner through the C-ABI.

* forward, backward (parameter gradients), masked MSE and Adam of the FP32
  training kernels against the FP64 numpy oracle (oracle/unet.py), which is
  itself pinned by finite differences: 1e-4 max-norm relative per layer; the
  tensor-core training path (BF16 operands, FP32 accumulation) at BF16
  tolerances: 1e-2 on the output, 3e-2 per layer on the gradients of a
  backward from the FP32 forward's cache, cosine 0.98 for the whole BF16 pass;
* a training step is bitwise reproducible (fixed-order reductions);
* training on pairs from the context's own MGPCG solves lowers the loss;
* flexible CG preconditioned by the trained network reaches the 1e-6 relative
  FP64 residual, and an untrained network stalls and falls back to the V-cycle
  (still converging)."""

import numpy as np
import pytest

import fluidity_b200 as fb
from fluidity_b200 import learned, scenes
from helpers import dam_break_context
from oracle import unet as U

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _t(a):
    import torch

    return torch.tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _inputs(rng, n):
    x = rng.normal(size=(n, 2, 10, 10, 10))
    x[:, 1] = rng.integers(-1, 2, size=(n, 10, 10, 10))
    return x


@pytest.fixture(scope="module")
def net():
    n = fb.UNet(8)
    yield n
    n.close()


def test_forward_and_backward_match_oracle(net):
    import torch

    rng = np.random.default_rng(0)
    th = U.init_params(5) + 0.02 * rng.normal(size=U.param_count())
    x = _inputs(rng, 5)
    y_ref, cache = U.forward(th, x)
    dy = rng.normal(size=y_ref.shape)
    g_ref = U.backward(th, cache, dy)
    P, X = _t(th), _t(x)
    Y = torch.zeros((5, 512), device="cuda")
    G = torch.zeros_like(P)
    net.forward(P, X, Y)
    net.backward(P, _t(dy.reshape(5, 512)), G)
    torch.cuda.synchronize()
    assert _rel(Y.cpu().numpy(), y_ref.reshape(5, 512)) <= TOL
    g = G.cpu().numpy()
    off = 0
    for name, nw, nb in U.layer_sizes():
        assert _rel(g[off:off + nw], g_ref[off:off + nw]) <= TOL, name
        assert _rel(g[off + nw:off + nw + nb], g_ref[off + nw:off + nw + nb]) <= TOL, name
        off += nw + nb


def test_tensor_core_training_matches_oracle_at_bf16_tolerance():
    """The tensor-core convolutions against the FP64 oracle.

    The forward output is checked directly. The backward is checked from the
    FP32 forward's cache, so that every ReLU mask is the oracle's: with a
    random output gradient each parameter gradient is a sum of terms of random
    sign that nearly cancel, and the few masks that a BF16 forward flips near
    zero would dominate its error. The whole BF16 forward + backward is held to
    the direction of the oracle's gradient (cosine).
    """
    import torch

    rng = np.random.default_rng(0)
    th = U.init_params(5) + 0.02 * rng.normal(size=U.param_count())
    x = _inputs(rng, 5)
    y_ref, cache = U.forward(th, x)
    dy = rng.normal(size=y_ref.shape)
    g_ref = U.backward(th, cache, dy)
    P, X, DY = _t(th), _t(x), _t(dy.reshape(5, 512))
    Y = torch.zeros((5, 512), device="cuda")
    G = torch.zeros_like(P)
    net = fb.UNet(8)
    net.forward(P, X, Y)  # FP32 forward: the oracle's masks
    net.set_tensor_cores(True)
    net.backward(P, DY, G)
    torch.cuda.synchronize()
    g = G.cpu().numpy()
    net.forward(P, X, Y)  # BF16 forward, then BF16 backward
    G2 = torch.zeros_like(P)
    net.backward(P, DY, G2)
    torch.cuda.synchronize()
    net.close()
    ey = _rel(Y.cpu().numpy(), y_ref.reshape(5, 512))
    g2 = G2.cpu().numpy()
    cos = float(g2 @ g_ref / (np.linalg.norm(g2) * np.linalg.norm(g_ref)))
    off, errs = 0, {}
    for name, nw, nb in U.layer_sizes():
        errs[name] = (_rel(g[off:off + nw], g_ref[off:off + nw]), _rel(g[off + nw:off + nw + nb], g_ref[off + nw:off + nw + nb]))
        off += nw + nb
    print(f"tensor cores vs FP64 oracle: output {ey:.2e}, full-BF16 gradient cosine {cos:.6f}, "
          f"backward per layer {({k: (round(a, 5), round(b, 5)) for k, (a, b) in errs.items()})}")
    assert ey <= 1e-2
    assert cos >= 0.98
    for name, (ew, eb) in errs.items():
        assert ew <= 3e-2 and eb <= 3e-2, (name, ew, eb)


def test_masked_mse_and_adam_match_oracle():
    import torch

    rng = np.random.default_rng(1)
    y, t = rng.normal(size=(3, 512)), rng.normal(size=(3, 512))
    m = (rng.uniform(size=(3, 512)) > 0.4).astype(np.float64)
    t[1] = 0.0  # an item without target energy
    for relative in (0, 1):
        loss_ref, grad_ref = U.masked_mse(y, t, m, relative=bool(relative))
        loss = torch.zeros(1, device="cuda")
        grad = torch.zeros((3, 512), device="cuda")
        fb.UNet.masked_mse(_t(y), _t(t), _t(m), loss, grad, relative=relative)
        assert abs(loss.item() - loss_ref) <= 1e-6 * loss_ref
        assert _rel(grad.cpu().numpy(), grad_ref) <= 1e-6
    th, gr = rng.normal(size=1000), rng.normal(size=1000)
    mm, vv = np.zeros(1000), np.zeros(1000)
    P, G, M, V = _t(th), _t(gr), _t(mm), _t(vv)
    for step in (1, 2, 3):
        th, mm, vv = U.adam(th, gr, mm, vv, step)
        fb.UNet.adam_step(P, G, M, V, step)
    np.testing.assert_allclose(P.cpu().numpy(), th, rtol=0, atol=1e-6)


def test_init_params_follow_he_uniform_rule():
    import torch

    P = torch.empty(fb.UNet.param_count(), device="cuda")
    fb.UNet.init_params(P, 7)
    p = P.cpu().numpy()
    off = 0
    for (name, kind, cin, cout), (_, nw, nb) in zip(U.LAYERS, U.layer_sizes()):
        bound = np.sqrt(6.0 / (cin * (27 if kind.startswith("conv3") else 1)))
        w = p[off:off + nw]
        assert np.all(np.abs(w) <= bound) and np.all(p[off + nw:off + nw + nb] == 0.0), name
        if nw >= 1000:
            assert abs(w.std() - bound / np.sqrt(3)) < 0.05 * bound, name
        off += nw + nb


def test_training_step_is_bitwise_reproducible():
    """Three Adam steps, twice, on the tensor-core path (the default)."""
    import torch

    rng = np.random.default_rng(2)
    x = _t(_inputs(rng, 64))
    t = _t(rng.normal(size=(64, 512)))
    m = _t((rng.uniform(size=(64, 512)) > 0.5).astype(np.float32))
    outs = []
    for _ in range(2):
        P, losses = learned.train(x, t, m, steps=3, batch=64, seed=3)
        outs.append((P.cpu().numpy(), losses))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])


@pytest.fixture(scope="module")
def trained():
    x, t, m = learned.collect_pairs(64, pairs=3000, steps_between=3, seed_steps=2, max_states=6)
    P, losses = learned.train(x, t, m, steps=1500, batch=64, seed=0)
    return x.shape[0], P, losses


def test_training_on_solver_pairs_lowers_the_loss(trained):
    """The block-residual loss |r_b - A_b y|^2 / max(|r_b|^2, 1): the zero
    correction scores at most 1; the trained network must end below half of
    that (it learns to invert the pressure operator on its block)."""
    count, P, losses = trained
    assert count >= 500
    assert np.all(np.isfinite(losses))
    assert losses[-40:].mean() < 0.5
    assert losses[-40:].mean() < 0.1 * losses[:40].mean()


def test_block_residual_loss_matches_oracle():
    import torch

    rng = np.random.default_rng(11)
    x = _inputs(rng, 5)
    x[:, 1] = rng.choice([1.0, 0.0, -1.0], p=[0.7, 0.2, 0.1], size=(5, 10, 10, 10))
    x[3, 0, 1:9, 1:9, 1:9] = 0.0  # an item without residual on its block: skipped
    y = rng.normal(size=(5, 512))
    want_loss, want_grad = U.block_residual_loss(y, x)
    loss = torch.zeros(1, device="cuda")
    grad = torch.zeros((5, 512), device="cuda")
    fb.UNet.block_residual_loss(_t(y), _t(x), loss, grad)
    assert float(loss) == pytest.approx(want_loss, rel=1e-5)
    assert _rel(grad.cpu().numpy(), want_grad) <= 1e-5
    assert np.all(grad.cpu().numpy()[3] == 0.0)


def _held_out(scene, n, steps=7):
    soa, mass = scenes.SCENES[scene](n)
    ctx = fb.LiquidContext(n, capacity=soa.shape[1])
    ctx.upload(soa)
    tp = fb.transfer_params(scenes.DT, mass)
    for _ in range(steps):
        code, _ = ctx.step(tp, fb.default_pressure_options(precision=1))
        assert code == fb.OK
    return ctx, tp


def test_trained_network_gains_over_the_vcycle_alone(trained):
    """The composite preconditioner (V-cycle, then the network's correction from
    the V-cycle's residual) on two held-out states (scenes and sizes the network
    was not trained on): never more flexible-CG iterations to the 1e-6 FP64
    residual than the V-cycle alone, and fewer on at least one; every iteration
    uses the network (no fallback). Without the network (the zero network) the
    composite is the V-cycle itself."""
    import torch

    _, P, _ = trained
    gains = []
    for scene, n in (("splash", 64), ("dam_break", 128)):
        ctx, tp = _held_out(scene, n)
        code, v = ctx.project(tp, fb.default_pressure_options(rel_tol=1e-6, warm_start=0, precision=1))
        assert code == fb.OK
        ctx.set_learned_preconditioner(torch.zeros(fb.UNet.param_count(), device="cuda"))
        code, z = ctx.project(tp, fb.default_pressure_options(rel_tol=1e-6, warm_start=0, precision=1,
                                                              preconditioner=2))
        assert code == fb.OK and z.iterations == v.iterations
        ctx.set_learned_preconditioner(P)
        code, c = ctx.project(tp, fb.default_pressure_options(rel_tol=1e-6, warm_start=0, precision=1,
                                                              preconditioner=2))
        assert code == fb.OK, c.as_dict()
        assert c.relative_residual <= 1e-6 and c.fell_back == 0 and c.learned_iterations == c.iterations
        gains.append((scene, n, v.iterations, c.iterations))
        ctx.close()
    print("V-cycle vs composite iterations:", gains)
    assert all(ci <= vi for _, _, vi, ci in gains), gains
    assert any(ci < vi for _, _, vi, ci in gains), gains


def test_learned_fcg_reaches_fp64_residual(trained):
    _, P, _ = trained
    ctx, _, m = dam_break_context(64)
    params = fb.transfer_params(scenes.DT, m)
    ctx.step(params, fb.default_pressure_options())
    ctx.set_learned_preconditioner(P)
    for prec in (0, 1):
        opt = fb.default_pressure_options(precision=prec, preconditioner=1, max_iterations=2000)
        code, d = ctx.step(params, opt)
        assert code == fb.OK, d.as_dict()
        assert d.relative_residual <= 1e-6 and d.learned_iterations > 0
    ctx.close()


def _identity_params():
    """Weights for which the network returns its residual input (z = r): a
    correction no better than plain CG."""
    P = {name: [w.copy(), b.copy()] for name, (w, b) in U.unpack(np.zeros(U.param_count())).items()}
    P["e1a"][0][0, 0, 1, 1, 1], P["e1a"][0][1, 0, 1, 1, 1] = 1.0, -1.0
    for name in ("e1b", "d1"):
        P[name][0][0, 0, 1, 1, 1] = P[name][0][1, 1, 1, 1, 1] = 1.0
    P["out"][0][0, 0], P["out"][0][0, 1] = 1.0, -1.0
    return U.pack(P)


def test_identity_network_is_exact_through_the_kernels(net):
    import torch

    rng = np.random.default_rng(4)
    x = _inputs(rng, 3)
    Y = torch.zeros((3, 512), device="cuda")
    net.forward(_t(_identity_params()), _t(x), Y)
    np.testing.assert_allclose(Y.cpu().numpy().reshape(3, 8, 8, 8), x[:, 0, 1:9, 1:9, 1:9], rtol=1e-6, atol=1e-6)


def test_tensor_core_inference_matches_fp32_forward():
    """The tcgen05 implicit-GEMM inference (BF16 activations, FP32 accumulation)
    against the FP32 training forward on the same solver windows: 3e-2 max-norm
    relative for a random network; the identity network returns r on fluid cells
    to BF16 rounding (4e-3 of max |r|)."""
    import torch

    ctx, _, m = dam_break_context(32)
    params = fb.transfer_params(scenes.DT, m)
    ctx.step(params, fb.default_pressure_options())
    nb = len(ctx.active_blocks())
    rng = np.random.default_rng(6)
    r = _t(rng.normal(size=nb * 512))
    z_tc = torch.zeros(nb * 512, device="cuda")
    z_ref = torch.zeros_like(z_tc)
    th = U.init_params(9) + 0.01 * rng.normal(size=U.param_count())
    ctx.set_learned_preconditioner(_t(th))
    ctx.apply_learned(r, z_tc, kernels=0)
    ctx.apply_learned(r, z_ref, kernels=1)
    a, b = z_tc.cpu().numpy(), z_ref.cpu().numpy()
    assert np.any(b != 0.0)
    assert _rel(a, b) <= 3e-2
    ctx.set_learned_preconditioner(_t(_identity_params()))
    ctx.apply_learned(r, z_tc, kernels=0)
    ctx.apply_learned(r, z_ref, kernels=1)
    a, b = z_tc.cpu().numpy(), z_ref.cpu().numpy()
    fluid = b != 0.0
    np.testing.assert_allclose(b[fluid], r.cpu().numpy()[fluid], rtol=1e-6, atol=1e-6)
    assert np.all(a[~fluid] == 0.0)
    assert np.abs(a - b).max() <= 4e-3 * np.abs(b).max()
    ctx.close()


def test_stalled_network_falls_back_to_the_vcycle():
    ctx, _, m = dam_break_context(32)
    params = fb.transfer_params(scenes.DT, m)
    ctx.step(params, fb.default_pressure_options())
    ctx.set_learned_preconditioner(_t(_identity_params()))
    # stall_ratio 0.01: every learned iteration counts as stalled -> fallback after exactly 3
    code, d = ctx.step(params, fb.default_pressure_options(preconditioner=1, stall_ratio=0.01))
    assert code == fb.OK
    assert d.fell_back == 1 and d.learned_iterations == 3
    assert d.relative_residual <= 1e-6
    ctx.close()


def test_zero_network_breaks_down_and_falls_back_at_once():
    import torch

    ctx, _, m = dam_break_context(32)
    params = fb.transfer_params(scenes.DT, m)
    ctx.step(params, fb.default_pressure_options())
    ctx.set_learned_preconditioner(torch.zeros(fb.UNet.param_count(), device="cuda"))  # z = 0, z.r = 0
    code, d = ctx.step(params, fb.default_pressure_options(preconditioner=1))
    assert code == fb.OK
    assert d.fell_back == 1 and d.learned_iterations == 0
    assert d.relative_residual <= 1e-6
    ctx.close()
