"""The bench workload at full size (256^3 splash, 29.6M particles): one step
after the warm-up replayed field by field by the FP64 oracle (u_pred, u_new,
v, C, x at 1e-5; the GPU pressure judged by its FP64 true residual on the
step's own system), for both V-cycle storages; and properties that do not
depend on the size: the sort is the stable cell order, every projection meets
the FP64 gate, and the step is reproducible bit for bit."""

import numpy as np
import pytest

import fluidity_b200 as fb
import oracle
from fluidity_b200 import scenes
from helpers import read_fields, sort_permutation
from oracle.replay import step_parity

pytestmark = pytest.mark.gpu

N = 256


@pytest.fixture(scope="module")
def splash():
    soa, mass = scenes.splash(N)
    return soa, mass


def test_splash_256_sort_is_the_stable_cell_order(splash):
    soa, mass = splash
    soa = soa.copy()
    soa[3:] = 0.0  # at rest and without gravity: the velocities stay exactly zero
    ctx = fb.LiquidContext(N, capacity=soa.shape[1])
    ctx.upload(soa)
    # The state after the step is the input in stable cell order (positions move only by the wall
    # clamp, at most 1e-3 h). A positive dt keeps the projection defined (its right-hand side
    # scales as 1/dt) and is exactly zero here.
    code, _ = ctx.step(fb.transfer_params(1e-6, mass, gravity=(0, 0, 0)), fb.default_pressure_options(precision=1))
    assert code == fb.OK
    out = ctx.download()
    perm = sort_permutation(soa, N)
    np.testing.assert_allclose(out[0:3], soa[0:3, perm], rtol=0, atol=1.01e-3 / N)
    f = ctx.fields()
    nb = len(ctx.active_blocks())
    cs = fb.copy_to_host(f["cell_start"], nb * 512 + 1, np.int32)
    assert cs[0] == 0 and cs[-1] == soa.shape[1] and np.all(np.diff(cs) >= 0)
    ctx.close()


def test_splash_256_projection_gate_and_reproducibility(splash):
    soa, mass = splash
    tp = fb.transfer_params(scenes.DT, mass)
    opt = fb.default_pressure_options(precision=1, warm_start=1)
    ctx = fb.LiquidContext(N, capacity=soa.shape[1])
    runs = []
    for _ in range(2):
        ctx.upload(soa)
        for _ in range(3):
            code, d = ctx.step(tp, opt)
            assert code == fb.OK
            assert d.relative_residual <= 1e-6 and d.true_residual_l2 <= d.reference_limit
        out = ctx.download()
        assert np.all(np.isfinite(out))
        runs.append(out)
    np.testing.assert_array_equal(runs[0], runs[1])
    ctx.close()


@pytest.mark.parametrize("precision", [1, 0])
def test_splash_256_step_matches_fp64_oracle_replay(splash, precision):
    """Step 6 of the bench scene (after five steps as warm-up), BF16 and FP32
    V-cycle storage: grid and particle fields within 1e-5 of the FP64 oracle,
    the GPU pressure meeting 1e-6 ||b|| in FP64."""
    soa, mass = splash
    tp = fb.transfer_params(scenes.DT, mass)
    opt = fb.default_pressure_options(precision=precision, warm_start=1)
    ctx = fb.LiquidContext(N, capacity=soa.shape[1])
    ctx.upload(soa)
    for _ in range(5):
        code, _ = ctx.step(tp, opt)
        assert code == fb.OK
    state = ctx.download()
    ctx.upload(state)
    code, diag = ctx.step(tp, opt)
    assert code == fb.OK and diag.relative_residual <= 1e-6, diag.as_dict()
    fields = read_fields(ctx, N)
    out = ctx.download()
    ctx.close()
    errs = step_parity(N, state, out, fields, scenes.DT)
    print(f"splash 256 step 6, precision {precision}: {errs}")
    assert errs["cell_types_agree"], errs
    assert errs["pressure_relative_residual"] <= 1.0001e-6, errs
    for k in ("u_pred0", "u_pred1", "u_pred2", "u_new0", "u_new1", "u_new2", "v", "C", "x"):
        assert errs[k] <= 1e-5, (k, errs)
