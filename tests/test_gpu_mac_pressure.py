"""ProjectMacPressure3D on the GPU (fl_project_mac_pressure_3d) against the
reference's manufactured pressure fixtures (tests/golden/pressure_3d.json,
re-expressed from the reference's pressure_3d_fixtures.py) and the FP64 oracle
(oracle/cpu/fl_oracle.c, fo_pressure_solve).

The right-hand side is summed per cell in the reference's order with
compensated sums and no fused products, so it equals the oracle's bit for bit;
pressures and corrected velocities agree within the solve tolerances written
below. Status codes follow mac_pressure_3d.h:88-100."""

import ctypes

import numpy as np
import pytest

import fluidity_b200 as fb
import oracle
from fluidity_b200 import scenes
from helpers import box_for, closed_system, golden, pressure_case, soa_to_xvc
from oracle.box_system import box_pressure_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", range(8))
def test_manufactured_fixture(case):
    ci, cv, fi, fk, fv, dt, ex = pressure_case(golden("pressure_3d.json")["arrays"], case)
    out = fb.project_mac_pressure_3d(ci, cv, fi, fk, fv, 1.0, dt, rel_tol=1e-15, max_iterations=200)
    tol = dict(rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(out["pressure"], ex["expected_cell_pressures"], **tol)
    np.testing.assert_allclose(out["rhs"], ex["expected_integrated_rhs"], **tol)
    np.testing.assert_allclose(out["residual"], ex["expected_true_residuals"], **tol)
    np.testing.assert_allclose(out["defect"], ex["expected_cell_constraint_defects"], **tol)
    np.testing.assert_allclose(out["corrected_u"], ex["expected_corrected_face_velocities"], **tol)
    np.testing.assert_array_equal(out["gauges"], ex["gauges"])
    ref = oracle.pressure_solve(ci, cv, fi, fk, fv, 1.0, dt, rel_tol=1e-15, max_iterations=200)
    np.testing.assert_array_equal(out["rhs"], ref["rhs"])
    assert out["compiled_architecture"] == 1000


def _dam_break_system(n=32):
    soa, m = scenes.dam_break(n)
    x, v, c = soa_to_xvc(soa)
    box = box_for(n)
    fm, fq = oracle.p2g(box, x, v, c, m)
    u_pred, _ = oracle.normalize_forces(box, fm, fq, 0.0, scenes.DT, scenes.GRAVITY)
    ct = oracle.classify_cells(box, x)
    return box, box_pressure_system(box, ct, u_pred)


def test_dam_break_32_first_projection_matches_oracle():
    """3375 fluid cells (under the 4096-cell cap), Dirichlet air faces and sealed walls."""
    box, s = _dam_break_system()
    args = (s["cells_idx"], s["cells_val"], s["faces_idx"], s["faces_kind"], s["faces_val"], box.h, scenes.DT)
    out = fb.project_mac_pressure_3d(*args, rel_tol=1e-12, max_iterations=4000)
    ref = oracle.pressure_solve(*args, rel_tol=1e-12, max_iterations=4000)
    np.testing.assert_array_equal(out["rhs"], ref["rhs"])
    # both stop at ||b - Ap|| <= 1e-12 ||b||
    assert np.abs(out["pressure"] - ref["pressure"]).max() <= 1e-8 * np.abs(ref["pressure"]).max()
    np.testing.assert_allclose(out["corrected_u"], ref["corrected_u"], rtol=1e-8, atol=1e-10)
    assert out["diag"]["true_residual_l2"] <= 1e-12 * out["diag"]["rhs_l2"] * 1.000001
    assert out["diag"]["gauge_count"] == 0  # every component touches air
    # the reference's own gate: ||b - Ap|| <= 2e-6 + 2e-6 ||b||
    gate = fb.project_mac_pressure_3d(*args, rel_tol=0.0, max_iterations=4000)
    assert gate["diag"]["true_residual_l2"] <= 2e-6 + 2e-6 * gate["diag"]["rhs_l2"]
    assert gate["diag"]["iterations"] <= out["diag"]["iterations"]


def _call_raw(ci, cv, fi, fk, fv, h, dt, max_iterations, rel_tol, sentinel=7.0):
    nc, nf = len(ci), len(fi)
    ci, cv = np.ascontiguousarray(ci, np.int32), np.ascontiguousarray(cv, np.float64)
    fi, fk, fv = (np.ascontiguousarray(fi, np.int32).reshape(-1, 4), np.ascontiguousarray(fk, np.int32),
                  np.ascontiguousarray(fv, np.float64).reshape(-1, 6))
    outs = [np.full(nc, sentinel) for _ in range(4)] + [np.full(max(nf, 1), sentinel)]
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int32)
    code = fb.library().fl_project_mac_pressure_3d(
        h, dt, ci.ctypes.data_as(ip), cv.ctypes.data_as(dp), nc, fi.ctypes.data_as(ip), fk.ctypes.data_as(ip),
        fv.ctypes.data_as(dp), nf, max_iterations, rel_tol, outs[0].ctypes.data_as(dp), outs[4].ctypes.data_as(dp),
        outs[1].ctypes.data_as(dp), outs[2].ctypes.data_as(dp), outs[3].ctypes.data_as(dp), None, None, None)
    return code, outs


def _two_cells(divergence):
    """Two cells joined by one open internal face, every other face sealed."""
    ci = np.array([[0, 0, 0], [1, 0, 0]], np.int32)
    cv = np.array([[1.0, divergence, 0.0, 0.0, 0.0]] * 2)
    fi, fk, fv = closed_system(ci, {(0, 1, 0, 0): (1, [1.0, 1e-3, 1.0, 0.0, 0.0, 0.0])})
    return ci, cv, fi, fk, fv


def test_status_codes_and_no_publication_on_failure():
    ci, cv, fi, fk, fv = _two_cells(0.0)
    code, outs = _call_raw(ci, cv, fi, fk, fv, 1.0, 0.01, 50, 1e-12)
    assert code == fb.OK and outs[0][0] == 0.0  # a closed, balanced pair: the gauge pins cell 0
    # an unanchored component with a net source is incompatible
    code, outs = _call_raw(*_two_cells(1.0), 1.0, 0.01, 50, 1e-12)
    assert code == fb.FAILED_PRECONDITION and np.all(outs[0] == 7.0)
    with pytest.raises(oracle.OracleError) as e:
        oracle.pressure_solve(*_two_cells(1.0), 1.0, 0.01, rel_tol=1e-12)
    assert e.value.code == fb.FAILED_PRECONDITION
    # cells out of (z,y,x) order, a bad iteration budget, an internal face missing a cell
    assert _call_raw(ci[::-1], cv, fi, fk, fv, 1.0, 0.01, 50, 1e-12)[0] == fb.INVALID_ARGUMENT
    assert _call_raw(ci, cv, fi, fk, fv, 1.0, 0.01, 0, 1e-12)[0] == fb.INVALID_ARGUMENT
    assert _call_raw(ci[:1], cv[:1], fi, fk, fv, 1.0, 0.01, 50, 1e-12)[0] == fb.INVALID_ARGUMENT
    # a face listed twice, one left out
    dup = np.concatenate([[0], np.arange(len(fi))])
    assert _call_raw(ci, cv, fi[dup], fk[dup], fv[dup], 1.0, 0.01, 50, 1e-12)[0] == fb.INVALID_ARGUMENT
    assert _call_raw(ci, cv, fi[1:], fk[1:], fv[1:], 1.0, 0.01, 50, 1e-12)[0] == fb.INVALID_ARGUMENT
    # above the 4096-cell cap
    big = np.stack(np.meshgrid(np.arange(17), np.arange(17), np.arange(15), indexing="ij"), -1).reshape(-1, 3)
    big = big[np.lexsort((big[:, 0], big[:, 1], big[:, 2]))]
    cvb = np.tile([1.0, 0.0, 0.0, 0.0, 0.0], (len(big), 1))
    assert len(big) > 4096
    assert _call_raw(big, cvb, fi[:0], fk[:0], fv[:0], 1.0, 0.01, 50, 1e-12)[0] == fb.RESOURCE_EXHAUSTED
    # a budget too small for the gate: aborted, nothing published
    box, s = _dam_break_system()
    code, outs = _call_raw(s["cells_idx"], s["cells_val"], s["faces_idx"], s["faces_kind"], s["faces_val"], box.h,
                           scenes.DT, 2, 1e-12)
    assert code == fb.ABORTED and np.all(outs[0] == 7.0) and np.all(outs[4] == 7.0)


def test_solves_are_bitwise_reproducible():
    box, s = _dam_break_system()
    args = (s["cells_idx"], s["cells_val"], s["faces_idx"], s["faces_kind"], s["faces_val"], box.h, scenes.DT)
    a = fb.project_mac_pressure_3d(*args, rel_tol=1e-12, max_iterations=4000)
    b = fb.project_mac_pressure_3d(*args, rel_tol=1e-12, max_iterations=4000)
    for k in ("pressure", "rhs", "residual", "defect", "corrected_u"):
        np.testing.assert_array_equal(a[k], b[k])
    assert a["diag"]["iterations"] == b["diag"]["iterations"] == 95  # as the FP64 oracle
