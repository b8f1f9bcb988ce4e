"""Asynchronous device-to-host snapshots (fl_snapshot_*), the B200 counterpart
of the reference's CudaLiquidSnapshotQueue3D
(native/include/fluidity/host/cuda_liquid_snapshot_3d.h:56-110,
native/cuda/liquid_snapshot_3d_host.cc:228-380).

Checked: a finished snapshot is bit for bit the state it was taken from, also
while later steps run and write the copied buffer (the fence), the pipelined
upload -> step -> snapshot loop returns what the synchronous host step returns,
the slot state machine's status codes, and the device check's DATA_LOSS for a
state with a non-finite value or a position outside the lattice."""

import ctypes

import numpy as np
import pytest

import fluidity_b200 as fb
from fluidity_b200 import scenes

pytestmark = pytest.mark.gpu


def _setup(n, scene="dam_break"):
    soa, mass = scenes.SCENES[scene](n)
    ctx = fb.LiquidContext(n, capacity=soa.shape[1])
    tp = fb.transfer_params(scenes.DT, mass)
    opt = fb.default_pressure_options(precision=1, warm_start=1)
    return ctx, soa, tp, opt


def _code(fn, *args):
    with pytest.raises(fb.FluidityError) as e:
        fn(*args)
    return e.value.code


def test_snapshot_is_the_state_it_was_taken_from():
    ctx, soa, tp, opt = _setup(32)
    q = fb.SnapshotQueue(ctx)
    assert q.last_valid() is None
    ctx.upload(soa)
    ctx.step(tp, opt)
    want = ctx.download()
    t = q.begin(1, frame_ordinal=1, time=scenes.DT)
    assert q.wait(t) == fb.SNAPSHOT_READY
    got, view = q.finish(t)
    np.testing.assert_array_equal(got, want)
    assert view.count == soa.shape[1] and view.epoch.generation == 1 and view.copy_ms > 0
    q.release(t)
    last, lv = q.last_valid()  # kept after the release
    np.testing.assert_array_equal(last, want)
    assert lv.epoch.frame_ordinal == 1
    q.close()
    ctx.close()


def test_snapshot_is_fenced_against_the_steps_after_it():
    """The copy of the state after step 1 runs while steps 2 and 3 are queued;
    step 3's G2P writes the copied buffer and must wait for the copy."""
    ctx, soa, tp, opt = _setup(128, "splash")
    ctx.upload(soa)
    states = []
    for _ in range(3):
        ctx.step(tp, opt)
        states.append(ctx.download())
    q = fb.SnapshotQueue(ctx)
    ctx.upload(soa)
    ctx.step(tp, opt)
    t = q.begin(1)
    ctx.step(tp, opt)
    ctx.step(tp, opt)
    assert q.wait(t) == fb.SNAPSHOT_READY
    got, _ = q.finish(t)
    np.testing.assert_array_equal(got, states[0])
    np.testing.assert_array_equal(ctx.download(), states[2])  # the fence did not disturb the steps
    q.release(t)
    q.close()
    ctx.close()


def test_pipelined_host_loop_matches_the_synchronous_host_step():
    """upload -> step -> begin, finishing the previous snapshot while the next
    step's input is copied in: each snapshot equals fl_step_host's output."""
    ctx, soa, tp, opt = _setup(64, "splash")
    host_in = np.ascontiguousarray(soa, np.float32)
    want = np.empty_like(host_in)
    ctx.step_host(host_in, want, tp, opt)
    q = fb.SnapshotQueue(ctx)
    prev = None
    for gen in range(1, 5):
        ctx.upload(host_in)
        ctx.step(tp, opt)
        t = q.begin(gen, gen, gen * scenes.DT)
        if prev is not None:
            assert q.wait(prev) == fb.SNAPSHOT_READY
            got, _ = q.finish(prev)
            np.testing.assert_array_equal(got, want)
            q.release(prev)
        prev = t
    assert q.wait(prev) == fb.SNAPSHOT_READY
    got, _ = q.finish(prev)
    np.testing.assert_array_equal(got, want)
    q.release(prev)
    q.close()
    ctx.close()


def test_snapshot_slot_state_machine():
    ctx, soa, tp, opt = _setup(32)
    ctx.upload(soa)
    ctx.step(tp, opt)
    q = fb.SnapshotQueue(ctx)
    assert _code(q.begin, 0) == fb.INVALID_ARGUMENT
    t1 = q.begin(1)
    assert _code(q.begin, 1) == fb.ALREADY_EXISTS
    t2 = q.begin(2)
    assert _code(q.begin, 3) == fb.UNAVAILABLE  # both reservations held
    assert _code(q.finish, t1) == fb.FAILED_PRECONDITION  # not observed READY yet
    assert q.wait(t2) == fb.SNAPSHOT_READY
    q.finish(t2)
    assert _code(q.poll, t2) == fb.FAILED_PRECONDITION  # a writer lease is not polled
    assert q.wait(t1) == fb.SNAPSHOT_READY
    assert _code(q.finish, t1) == fb.FAILED_PRECONDITION  # older than the last finished generation
    q.cancel(t1)  # READY: freed at once
    assert _code(q.poll, t1) == fb.FAILED_PRECONDITION  # stale ticket
    assert _code(q.begin, 2) == fb.FAILED_PRECONDITION  # generation not above the last finished
    t4 = q.begin(4)
    q.cancel(t4)  # PENDING until a poll observes the completed copy
    assert q.wait(t4) == fb.SNAPSHOT_CANCELED
    assert _code(q.poll, t4) == fb.FAILED_PRECONDITION
    q.release(t2)
    assert _code(q.release, t2) == fb.FAILED_PRECONDITION
    assert q.last_valid()[1].epoch.generation == 2
    lib = fb.library()
    assert lib.fl_context_destroy(ctx.handle) == fb.FAILED_PRECONDITION  # a queue is live
    # the three pinned buffers rotate: many begin/finish/release cycles stay valid
    want = ctx.download()
    for gen in range(5, 12):
        t = q.begin(gen)
        q.wait(t)
        got, _ = q.finish(t)
        np.testing.assert_array_equal(got, want)
        q.release(t)
    q.close()
    ctx.close()


@pytest.mark.parametrize("where", ["nonfinite", "outside"])
def test_snapshot_device_check_reports_data_loss(where):
    ctx, soa, tp, opt = _setup(32)
    bad = np.array(soa, np.float32)
    k = bad.shape[1] // 3
    if where == "nonfinite":
        bad[4, k] = np.nan  # a velocity
    else:
        bad[0, k] = 1.5  # x beyond the unit box's block lattice
    ctx.upload(bad)
    q = fb.SnapshotQueue(ctx)
    t = q.begin(1)
    assert q.wait(t) == fb.SNAPSHOT_READY
    assert _code(q.finish, t) == fb.DATA_LOSS
    assert _code(q.begin, 2) == fb.INTERNAL  # the queue is poisoned
    assert q.last_valid() is None
    q.close()
    ctx.close()


def test_snapshot_of_an_empty_state():
    ctx, soa, tp, opt = _setup(32)
    ctx.upload(soa[:, :0])
    q = fb.SnapshotQueue(ctx)
    t = q.begin(1)
    assert q.wait(t) == fb.SNAPSHOT_READY
    got, view = q.finish(t)
    assert got.shape == (15, 0) and view.count == 0
    q.release(t)
    q.close()
    ctx.close()


def test_staged_inputs_pipeline_matches_the_synchronous_host_step():
    """stage(k + 1) -> step(k) -> begin(k), finishing snapshot k - 1: each step
    starts from its staged input (as if uploaded) while the next one is copied."""
    ctx, soa, tp, opt = _setup(64, "splash")
    host_in = np.ascontiguousarray(soa, np.float32)
    want = np.empty_like(host_in)
    ctx.step_host(host_in, want, tp, opt)
    q = fb.SnapshotQueue(ctx)
    ctx.stage(host_in)
    prev = None
    for gen in range(1, 6):
        if gen < 5:
            ctx.stage(host_in)
        ctx.step(tp, opt)
        t = q.begin(gen)
        if prev is not None:
            assert q.wait(prev) == fb.SNAPSHOT_READY
            got, _ = q.finish(prev)
            np.testing.assert_array_equal(got, want)
            q.release(prev)
        prev = t
    assert q.wait(prev) == fb.SNAPSHOT_READY
    got, _ = q.finish(prev)
    np.testing.assert_array_equal(got, want)
    q.release(prev)
    # at most two inputs wait; an upload drops them and becomes the state
    ctx.stage(host_in)
    ctx.stage(host_in)
    assert _code(ctx.stage, host_in) == fb.UNAVAILABLE
    ctx.upload(host_in)
    ctx.step(tp, opt)
    np.testing.assert_array_equal(ctx.download(), want)
    q.close()
    ctx.close()


def test_steps_continue_from_the_state_after_staging():
    """With four buffers a step without a staged input advances the current
    state exactly as the two-buffer path does."""
    ctx, soa, tp, opt = _setup(64, "splash")
    host_in = np.ascontiguousarray(soa, np.float32)
    ctx.upload(host_in)
    for _ in range(3):
        ctx.step(tp, opt)
    want = ctx.download()
    ctx.stage(host_in)
    for _ in range(3):
        ctx.step(tp, opt)
    np.testing.assert_array_equal(ctx.download(), want)
    ctx.close()
