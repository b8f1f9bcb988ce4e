"""Shared test helpers: scene setup, host replica of the stable cell sort, and
GPU state read-back into dense box arrays for comparison with the oracle."""

import json
from pathlib import Path

import numpy as np

import fluidity_b200 as fb
import oracle
from fluidity_b200 import scenes

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden(name):
    return json.loads((GOLDEN / name).read_text())


def soa_to_xvc(soa):
    x = soa[0:3].T.astype(np.float64)
    v = soa[3:6].T.astype(np.float64)
    c = soa[6:15].T.astype(np.float64)
    return x, v, c


def box_for(n):
    return oracle.Box.make([0.0, 0.0, 0.0], 1.0 / n, [0, 0, 0], [n, n, n])


def sort_permutation(soa, n):
    """Replica of the device's stable sort key (block, local cell) for a box of n cells."""
    X = soa[0:3].astype(np.float32) * np.float32(n)
    cell = np.floor(X).astype(np.int64)
    nbk = n // 8
    key = ((((cell[2] >> 3) * nbk + (cell[1] >> 3)) * nbk + (cell[0] >> 3)) * 512 + (cell[2] & 7) * 64 +
           (cell[1] & 7) * 8 + (cell[0] & 7))
    return np.argsort(key, kind="stable")


def read_fields(ctx, n):
    blocks = ctx.active_blocks()
    nb = len(blocks)
    f = ctx.fields()
    nn = (n, n, n)
    out = {"blocks": blocks}
    out["u_pred"] = [fb.sparse_faces_to_dense(blocks, fb.copy_to_host(f["u_pred"][a], nb * 512, np.float32), nn, a,
                                              fill=np.nan) for a in range(3)]
    out["u_new"] = [fb.sparse_faces_to_dense(blocks, fb.copy_to_host(f["u_new"][a], nb * 512, np.float32), nn, a,
                                             fill=np.nan) for a in range(3)]
    out["pressure"] = fb.sparse_cells_to_dense(blocks, fb.copy_to_host(f["pressure"], nb * 512, np.float64), nn,
                                               fill=np.nan)
    out["cell_type"] = fb.sparse_cells_to_dense(blocks, fb.copy_to_host(f["cell_type"], nb * 512, np.uint8), nn,
                                                fill=255)
    return out


def rel_err(a, b, mask=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def dam_break_context(n, capacity=None):
    soa, m = scenes.dam_break(n)
    ctx = fb.LiquidContext(n, capacity=capacity or soa.shape[1])
    ctx.upload(soa)
    return ctx, soa, m


def pressure_case(arr, case):
    """One case of tests/golden/pressure_3d.json in the record layout of the oracle and the C-ABI."""
    co, fo, go = arr["case_cell_offsets"], arr["case_face_offsets"], arr["case_gauge_offsets"]
    cs, ce, fs, fe = co[case], co[case + 1], fo[case], fo[case + 1]
    cells_idx = np.array(arr["cell_indices"][cs:ce], np.int32)
    cells_val = np.stack([arr["cell_fluid_volumes"][cs:ce], arr["target_cell_divergences"][cs:ce],
                          arr["cell_bulk_moduli"][cs:ce], arr["previous_cell_pressures"][cs:ce],
                          np.zeros(ce - cs)], 1)
    faces_idx = np.array(arr["face_indices"][fs:fe], np.int32)
    faces_kind = np.array(arr["face_link_kinds"][fs:fe], np.int32)
    faces_val = np.stack([arr["face_open_areas"][fs:fe], arr["face_inverse_densities"][fs:fe],
                          arr["face_pressure_gradient_distances"][fs:fe], arr["predicted_face_velocities"][fs:fe],
                          arr["wall_face_velocities"][fs:fe], arr["face_pressure_lifts"][fs:fe]], 1)
    expect = {k: np.array(arr[k][cs:ce]) for k in ("expected_cell_pressures", "expected_integrated_rhs",
                                                     "expected_true_residuals", "expected_cell_constraint_defects")}
    expect["expected_corrected_face_velocities"] = np.array(arr["expected_corrected_face_velocities"][fs:fe])
    expect["gauges"] = np.array(arr["expected_gauge_cell_ordinals"][go[case]:go[case + 1]])
    return cells_idx, cells_val, faces_idx, faces_kind, faces_val, arr["step_durations"][case], expect


def closed_system(cells_idx, open_faces):
    """Every incident face of the cells (shared faces once) in the reference's
    owned-slot order: sealed with zero values, except the faces named in
    open_faces ({(axis, x, y, z): (kind, 6 values)})."""
    from oracle.box_system import owned_slot_order

    faces = set()
    for x, y, z in np.asarray(cells_idx).tolist():
        for a in range(3):
            hi = [x, y, z]
            hi[a] += 1
            faces.add((a, x, y, z))
            faces.add((a, *hi))
    fi = np.array(sorted(faces), np.int32)
    fi = fi[owned_slot_order(fi)]
    fk = np.zeros(len(fi), np.int32)
    fv = np.zeros((len(fi), 6))
    for f, key in enumerate(map(tuple, fi.tolist())):
        if key in open_faces:
            fk[f], fv[f] = open_faces[key][0], open_faces[key][1]
    return fi, fk, fv


class _DeviceArray:
    """A raw device pointer seen through __cuda_array_interface__ (for torch views of library buffers)."""

    def __init__(self, ptr, count, dtype):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def device_view(ptr, count, dtype):
    """A torch tensor aliasing `count` elements of library device memory at `ptr`."""
    import torch

    return torch.as_tensor(_DeviceArray(ptr, count, dtype), device="cuda")


def state_views(ctx):
    """torch views of the context's current particle state: 15 arrays (x[3], v[3], C[9])."""
    pv = ctx.particles_view()
    n = pv.count
    return [device_view(pv.x[d], n, np.float32) for d in range(3)] + \
        [device_view(pv.v[d], n, np.float32) for d in range(3)] + [device_view(pv.c[d], n, np.float32) for d in range(9)]


def device_cell_order(x, n):
    """The device's stable sort by (8^3 block, local cell) computed with torch on
    device positions x (3 tensors): the permutation, as a torch int64 tensor."""
    import torch

    cell = [torch.floor(x[d] * np.float32(n)).to(torch.int64) for d in range(3)]
    nbk = n // 8
    key = ((((cell[2] >> 3) * nbk + (cell[1] >> 3)) * nbk + (cell[0] >> 3)) * 512 + (cell[2] & 7) * 64 +
           (cell[1] & 7) * 8 + (cell[0] & 7))
    return torch.sort(key, stable=True).indices
