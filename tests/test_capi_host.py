"""Host-side checks of the entry points that validate before touching a device
(CPU only): the general pressure operator's input rules and capacity limits
(mac_pressure_3d.h:88-100), the snapshot queue's and the staging call's
argument checks, and the no-device refusal of a valid request."""

import ctypes

import numpy as np
import pytest

import fluidity_b200 as fb
from helpers import closed_system


def _on_b200():
    info = fb.runtime_info()
    return info["device_count"] > 0 and info["major"] == 10


def _two_cells():
    """Two unit cells joined by one open internal face; their ten other faces sealed."""
    ci = np.array([[0, 0, 0], [1, 0, 0]], np.int32)
    cv = np.array([[1.0, 0.0, 0.0, 0.0, 0.0]] * 2)
    fi, fk, fv = closed_system(ci, {(0, 1, 0, 0): (1, [1.0, 1e-3, 1.0, 0.0, 0.0, 0.0])})
    return ci, cv, fi, fk, fv


def _internal(fi):
    return int(np.nonzero((fi == [0, 1, 0, 0]).all(1))[0][0])


def _code(*args, **kw):
    with pytest.raises(fb.FluidityError) as e:
        fb.project_mac_pressure_3d(*args, **kw)
    return e.value.code


def test_pressure_operator_rejects_malformed_systems_before_the_device():
    ci, cv, fi, fk, fv = _two_cells()
    assert _code(ci[::-1], cv, fi, fk, fv, 1.0, 0.01) == fb.INVALID_ARGUMENT  # not (z,y,x)-sorted
    assert _code(ci[[0, 0]], cv, fi, fk, fv, 1.0, 0.01) == fb.INVALID_ARGUMENT  # duplicate cell
    k = _internal(fi)
    fi1, fk1, fv1 = closed_system(ci[:1], {})
    fk1[:] = 1
    assert _code(ci[:1], cv[:1], fi1, fk1, fv1, 1.0, 0.01) == fb.INVALID_ARGUMENT  # internal faces, one cell
    kind = fk.copy()
    kind[k] = 2
    assert _code(ci, cv, fi, kind, fv, 1.0, 0.01) == fb.INVALID_ARGUMENT  # Dirichlet, two cells
    kind[:] = 0
    kind[0] = 2
    assert _code(ci, cv, fi, kind, fv, 1.0, 0.01) == fb.INVALID_ARGUMENT  # Dirichlet with a closed aperture
    kind = fk.copy()
    kind[k] = 0
    assert _code(ci, cv, fi, kind, fv, 1.0, 0.01) == fb.INVALID_ARGUMENT  # open sealed face
    wide = fv.copy()
    wide[k, 0] = 1.0 + 1e-9
    assert _code(ci, cv, fi, fk, wide, 1.0, 0.01) == fb.INVALID_ARGUMENT  # aperture above h^2
    neg = fv.copy()
    neg[(k + 1) % len(fv), 0] = -0.0 - 1e-300
    assert _code(ci, cv, fi, fk, neg, 1.0, 0.01) == fb.INVALID_ARGUMENT  # negative aperture
    bad = cv.copy()
    bad[0, 0] = 0.0
    assert _code(ci, bad, fi, fk, fv, 1.0, 0.01) == fb.INVALID_ARGUMENT  # no fluid volume
    bad = cv.copy()
    bad[1, 3] = np.nan
    assert _code(ci, bad, fi, fk, fv, 1.0, 0.01) == fb.INVALID_ARGUMENT  # non-finite value
    assert _code(ci, cv, fi, fk, fv, 1.0, 0.0) == fb.INVALID_ARGUMENT  # dt
    assert _code(ci, cv, fi, fk, fv, 1.0, 0.01, max_iterations=0) == fb.INVALID_ARGUMENT
    assert _code(ci, cv, fi, fk, fv, 1.0, 0.01, rel_tol=-1.0) == fb.INVALID_ARGUMENT
    # the faces must be exactly the incident faces, unique, in owned-slot order
    dup = np.concatenate([np.arange(k + 1), np.arange(k, len(fi))])
    assert _code(ci, cv, fi[dup], fk[dup], fv[dup], 1.0, 0.01) == fb.INVALID_ARGUMENT  # duplicated face
    miss = np.delete(np.arange(len(fi)), 0)
    assert _code(ci, cv, fi[miss], fk[miss], fv[miss], 1.0, 0.01) == fb.INVALID_ARGUMENT  # missing face
    swap = np.arange(len(fi))
    swap[[0, 1]] = [1, 0]
    assert _code(ci, cv, fi[swap], fk[swap], fv[swap], 1.0, 0.01) == fb.INVALID_ARGUMENT  # out of slot order
    extra = np.vstack([fi, [[2, 5, 5, 5]]]).astype(np.int32)
    assert _code(ci, cv, extra, np.append(fk, 0), np.vstack([fv, np.zeros((1, 6))]), 1.0, 0.01) == \
        fb.INVALID_ARGUMENT  # a face of no cell
    many = np.stack(np.meshgrid(np.arange(17), np.arange(17), np.arange(15), indexing="ij"), -1).reshape(-1, 3)
    many = many[np.lexsort((many[:, 0], many[:, 1], many[:, 2]))]
    assert _code(many, np.tile(cv[0], (len(many), 1)), fi[:0], fk[:0], fv[:0], 1.0, 0.01) == fb.RESOURCE_EXHAUSTED


def test_pressure_operator_refuses_without_a_b200():
    if _on_b200():
        pytest.skip("a B200 is present")
    assert _code(*_two_cells(), 1.0, 0.01) == fb.FAILED_PRECONDITION


def test_snapshot_and_staging_calls_check_their_arguments():
    lib = fb.library()
    out = ctypes.c_void_p()
    assert lib.fl_snapshot_queue_create(None, ctypes.byref(out)) == fb.INVALID_ARGUMENT
    assert lib.fl_snapshot_queue_destroy(None) == fb.OK
    ticket, view, progress = fb.SnapshotTicket(), fb.SnapshotView(), ctypes.c_int()
    epoch = fb.Epoch(1, 1, 0.0)
    assert lib.fl_snapshot_begin(None, ctypes.byref(epoch), None, ctypes.byref(ticket)) == fb.INVALID_ARGUMENT
    assert lib.fl_snapshot_poll(None, ctypes.byref(ticket), ctypes.byref(progress)) == fb.FAILED_PRECONDITION
    assert lib.fl_snapshot_wait(None, ctypes.byref(ticket), ctypes.byref(progress)) == fb.FAILED_PRECONDITION
    assert lib.fl_snapshot_finish(None, ctypes.byref(ticket), ctypes.byref(view)) == fb.FAILED_PRECONDITION
    assert lib.fl_snapshot_release(None, ctypes.byref(ticket)) == fb.FAILED_PRECONDITION
    assert lib.fl_snapshot_cancel(None, ctypes.byref(ticket)) == fb.FAILED_PRECONDITION
    assert lib.fl_snapshot_last_valid(None, ctypes.byref(view)) == fb.INVALID_ARGUMENT
    assert lib.fl_stage_particles(None, None, 0) == fb.INVALID_ARGUMENT
