"""The FP64 numpy restatement of the learned block preconditioner (oracle/unet.py)
against central finite differences, layer by layer. No reference counterpart
exists, so these checks are what pin the oracle that the GPU kernels are tested
against. CPU only."""

import numpy as np

from oracle import unet as U


def test_parameter_count_and_layout():
    assert U.param_count() == 141937
    th = U.init_params(3)
    P = U.unpack(th)
    assert P["e1a"][0].shape == (16, 2, 3, 3, 3) and P["bt"][0].shape == (64, 32, 3, 3, 3)
    assert P["out"][0].shape == (1, 16) and np.all(P["d1"][1] == 0.0)
    np.testing.assert_array_equal(U.pack({k: v for k, v in P.items()}), th)


def test_forward_shapes_and_positive_homogeneity_without_bias():
    rng = np.random.default_rng(1)
    th = U.init_params(1)  # zero biases: the network is positively homogeneous of degree 1
    x = rng.normal(size=(2, 2, 10, 10, 10))
    y, _ = U.forward(th, x)
    assert y.shape == (2, 1, 8, 8, 8)
    y2, _ = U.forward(th, 2.5 * x)
    np.testing.assert_allclose(y2, 2.5 * y, rtol=1e-12, atol=1e-12)


def test_backward_matches_finite_differences_per_layer():
    rng = np.random.default_rng(0)
    th = U.init_params(1) + 0.01 * rng.normal(size=U.param_count())  # non-zero biases too
    x = rng.normal(size=(1, 2, 10, 10, 10))
    y, cache = U.forward(th, x)
    dy = rng.normal(size=y.shape)
    g = U.backward(th, cache, dy)
    off = 0
    eps = 1e-6
    for _, nw, nb in U.layer_sizes():
        for lo, hi in ((off, off + nw), (off + nw, off + nw + nb)):
            d = np.zeros_like(th)
            d[lo:hi] = rng.normal(size=hi - lo)
            fd = ((U.forward(th + eps * d, x)[0] * dy).sum() - (U.forward(th - eps * d, x)[0] * dy).sum()) / (2 * eps)
            assert abs(fd - g @ d) <= 1e-6 * max(1.0, abs(fd)), (lo, hi, fd, g @ d)
        off += nw + nb


def test_masked_mse_gradient_and_adam():
    rng = np.random.default_rng(2)
    y, t = rng.normal(size=(3, 512)), rng.normal(size=(3, 512))
    m = (rng.uniform(size=(3, 512)) > 0.3).astype(float)
    loss, grad = U.masked_mse(y, t, m)
    assert np.isclose(loss, ((y - t) ** 2 * m).sum() / m.sum())
    eps = 1e-6
    d = rng.normal(size=y.shape)
    fd = (U.masked_mse(y + eps * d, t, m)[0] - U.masked_mse(y - eps * d, t, m)[0]) / (2 * eps)
    assert np.isclose(fd, (grad * d).sum(), rtol=1e-7)
    loss, grad = U.masked_mse(y, t, m, relative=True)
    per_item = [((y[b] - t[b]) ** 2 * m[b]).sum() / (m[b] * t[b] ** 2).sum() for b in range(3)]
    assert np.isclose(loss, np.mean(per_item))
    fd = (U.masked_mse(y + eps * d, t, m, True)[0] - U.masked_mse(y - eps * d, t, m, True)[0]) / (2 * eps)
    assert np.isclose(fd, (grad * d).sum(), rtol=1e-7)
    t0 = t.copy()
    t0[2] = 0.0  # no target energy: the item is left out
    loss, grad = U.masked_mse(y, t0, m, relative=True)
    assert np.isclose(loss, np.mean(per_item[:2])) and np.all(grad[2] == 0.0)
    th, gr = rng.normal(size=10), rng.normal(size=10)
    th1, m1, v1 = U.adam(th, gr, np.zeros(10), np.zeros(10), 1)
    np.testing.assert_allclose(th1, th - 1e-3 * np.sign(gr), rtol=0, atol=1e-9)  # first step moves lr*sign(g)


def test_block_residual_loss_gradient_matches_finite_differences():
    """The block-residual loss of the learned preconditioner (oracle restatement
    of fl_unet_block_residual_loss): gradient by central differences, and the
    zero correction scores |r_b|^2 / max(|r_b|^2, 1) <= 1."""
    rng = np.random.default_rng(3)
    x = np.zeros((3, 2, 10, 10, 10))
    x[:, 0] = rng.normal(size=(3, 10, 10, 10))
    x[:, 1] = rng.choice([1.0, 0.0, -1.0], p=[0.7, 0.2, 0.1], size=(3, 10, 10, 10))
    y = rng.normal(size=(3, 512))
    loss, grad = U.block_residual_loss(y, x)
    eps = 1e-6
    for k in rng.choice(3 * 512, 12, replace=False):
        b, c = divmod(int(k), 512)
        yp, ym = y.copy(), y.copy()
        yp[b, c] += eps
        ym[b, c] -= eps
        fd = (U.block_residual_loss(yp, x)[0] - U.block_residual_loss(ym, x)[0]) / (2 * eps)
        assert abs(fd - grad[b, c]) <= 1e-7 * np.abs(grad).max()
    zero, _ = U.block_residual_loss(np.zeros_like(y), x)
    assert 0.0 < zero <= 1.0
