"""Oracle helper (test infrastructure, the checker): field-by-field errors of
one device step against its FP64 replay (fo_step_replay in oracle/cpu).

The device step ran from `state` (FP32 SoA, 15 x np) and produced `out` (the
state after the step, in the stable cell order of `state`) and the dense box
fields of that step (u_pred, u_new per axis, cell pressure, cell type with 255
for cells outside the active blocks). The oracle repeats the step in FP64 with
the device's pressure given instead of solved, so every difference is the
transfers' and the correction's own; the pressure itself is judged by the FP64
true residual of the device pressure on the system built from the device's
own predicted velocities (mac_pressure_3d_arithmetic.h:404-503)."""

from __future__ import annotations

import numpy as np

import oracle
from oracle.box_system import box_pressure_system


def _rel(a, b, mask=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _cell_order(state, n):
    """The device's stable sort by (8^3 block, local cell) for a box of n cells."""
    X = state[0:3].astype(np.float32) * np.float32(n)
    cell = np.floor(X).astype(np.int64)
    nbk = n // 8
    key = ((((cell[2] >> 3) * nbk + (cell[1] >> 3)) * nbk + (cell[0] >> 3)) * 512 + (cell[2] & 7) * 64 +
           (cell[1] & 7) * 8 + (cell[0] & 7))
    return np.argsort(key, kind="stable")


def step_parity(n, state, out, fields, dt, stride=61, density=1000.0, gravity=(0.0, -9.81, 0.0)):
    """Per-field errors (norm-wise relative, max |device - fp64| / max |fp64|;
    x also as the largest difference in cells) of one device step on the n^3 box scene, with the G2P fields
    checked on every `stride`-th particle."""
    box = oracle.Box.make([0.0, 0.0, 0.0], 1.0 / n, [0, 0, 0], [n, n, n])
    pressure = np.nan_to_num(fields["pressure"])
    r = oracle.step_replay(box, state, pressure, dt, stride=stride, density=density, gravity=gravity)
    known = fields["cell_type"] != 255
    errs = {"cell_types_agree": bool(np.array_equal(fields["cell_type"][known], r["cell_type"][known])
                                     and not np.any((r["cell_type"] == 1) & ~known))}
    for a in range(3):
        have = ~np.isnan(fields["u_pred"][a])
        errs[f"u_pred{a}"] = _rel(fields["u_pred"][a], r["u_pred"][a], have)
        errs[f"u_new{a}"] = _rel(fields["u_new"][a], r["u_new"][a], have)
    perm = _cell_order(state, n)
    where = np.empty_like(perm)
    where[perm] = np.arange(len(perm))
    got = out[:, where[r["sample_index"]]].T.astype(np.float64)
    want = r["sample"]
    errs["x"] = _rel(got[:, 0:3], want[:, 0:3])
    errs["x_cells"] = float(np.abs(got[:, 0:3] - want[:, 0:3]).max() * n)  # FP32 position rounding shows here
    errs["v"] = _rel(got[:, 3:6], want[:, 3:6])
    errs["C"] = _rel(got[:, 6:15], want[:, 6:15])
    ct = np.where(fields["cell_type"] == 255, 2, fields["cell_type"]).astype(np.uint8)
    sysm = box_pressure_system(box, ct, [np.nan_to_num(fields["u_pred"][a].astype(np.float64)) for a in range(3)],
                               density=density)
    ci = sysm["cells_idx"]
    ev = oracle.pressure_evaluate(sysm["cells_idx"], sysm["cells_val"], sysm["faces_idx"], sysm["faces_kind"],
                                  sysm["faces_val"], box.h, dt, pressure[ci[:, 2], ci[:, 1], ci[:, 0]])
    errs["pressure_relative_residual"] = ev["diag"]["true_residual_l2"] / ev["diag"]["rhs_l2"]
    errs["post_projection_divergence_max_per_s"] = ev["diag"]["max_volume_scaled_residual"]
    errs["replayed_fluid_cells"] = int(len(ci))
    errs["sampled_particles"] = int(len(want))
    return errs
