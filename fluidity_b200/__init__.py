"""fluidity_b200: B200-native APIC transfers and MGPCG pressure projection.

The compute path is the CUDA library ``_lib/libfluidity_b200.so`` (sm_100a),
reached through its C-ABI (``include/fluidity_b200.h``). This module is a thin
ctypes mirror of that interface plus host helpers (scene generation, sparse to
dense field views). There is no CPU fallback: importing works without a GPU,
but every compute call raises ``FluidityError`` unless the CUDA library loads
and a B200 is present.

Reference-shaped operators mirror FluidiTy's operator API
(native/include/fluidity/host/transfers_3d.h:23-61):

* :func:`deposit_mac_3d`        <-> ``DepositMac3D``
* :func:`deposit_mac_quanta_3d` <-> ``DepositMacQuanta3D`` / ``CudaDepositMacQuanta3D``
* :func:`gather_mac_3d`         <-> ``GatherMac3D`` / ``CudaGatherMac3D``

and :class:`LiquidContext` drives the resident substep
(topology -> sort -> P2G -> pressure -> G2P) the way the reference's
``LiquidSubstepBackend3D`` table does (liquid_substep_backend_3d.h:47-260).
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import scenes  # noqa: F401  (re-exported helper)

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_lib" / "libfluidity_b200.so"

OK, INVALID_ARGUMENT, RESOURCE_EXHAUSTED, FAILED_PRECONDITION, ABORTED, OUT_OF_RANGE, INTERNAL = 0, 3, 8, 9, 10, 11, 13
ALREADY_EXISTS, UNAVAILABLE, DATA_LOSS = 6, 14, 15
STATUS_NAMES = {0: "OK", 3: "INVALID_ARGUMENT", 6: "ALREADY_EXISTS", 8: "RESOURCE_EXHAUSTED", 9: "FAILED_PRECONDITION",
                10: "ABORTED", 11: "OUT_OF_RANGE", 13: "INTERNAL", 14: "UNAVAILABLE", 15: "DATA_LOSS"}
SNAPSHOT_PENDING, SNAPSHOT_READY, SNAPSHOT_CANCELED = 0, 1, 2


class FluidityError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {STATUS_NAMES.get(code, code)} ({code})")
        self.code = code


_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lp = ctypes.POINTER(ctypes.c_int64)


class Report(ctypes.Structure):
    _fields_ = [("compiled_architecture", ctypes.c_int), ("error", ctypes.c_int),
                ("first_bad_index", ctypes.c_ulonglong)]


class Measurement(ctypes.Structure):
    _fields_ = [("compiled_architecture", ctypes.c_int), ("kernel_ms", ctypes.c_float)]


class GridDesc(ctypes.Structure):
    _fields_ = [("origin", ctypes.c_double * 3), ("h", ctypes.c_double), ("block_lo", ctypes.c_int32 * 3),
                ("block_dim", ctypes.c_int32 * 3), ("solid_lo", ctypes.c_int32 * 3), ("solid_hi", ctypes.c_int32 * 3)]


class Particles(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p * 3), ("v", ctypes.c_void_p * 3), ("c", ctypes.c_void_p * 9),
                ("mass", ctypes.c_void_p), ("count", ctypes.c_uint64)]


class TransferParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("particle_mass", ctypes.c_double), ("gravity", ctypes.c_double * 3),
                ("min_face_mass", ctypes.c_double), ("density", ctypes.c_double)]


class PressureOptions(ctypes.Structure):
    _fields_ = [("levels", ctypes.c_int), ("pre_sweeps", ctypes.c_int), ("post_sweeps", ctypes.c_int),
                ("coarse_sweeps", ctypes.c_int), ("precision", ctypes.c_int), ("max_iterations", ctypes.c_int),
                ("max_refinements", ctypes.c_int), ("warm_start", ctypes.c_int), ("rel_tol", ctypes.c_double),
                ("inner_rtol", ctypes.c_double), ("preconditioner", ctypes.c_int), ("stall_limit", ctypes.c_int),
                ("stall_ratio", ctypes.c_double)]


class PressureDiagnostics(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int), ("refinements", ctypes.c_int),
                ("levels", ctypes.c_int), ("fluid_cells", ctypes.c_int), ("active_blocks", ctypes.c_int),
                ("rhs_l2", ctypes.c_double), ("true_residual_l2", ctypes.c_double),
                ("relative_residual", ctypes.c_double), ("reference_limit", ctypes.c_double),
                ("max_volume_residual", ctypes.c_double), ("max_divergence", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("learned_iterations", ctypes.c_int), ("fell_back", ctypes.c_int)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


EXPORTS = [
    "fl_context_create", "fl_context_destroy", "fl_topology_from_particles", "fl_topology_from_blocks",
    "fl_active_blocks", "fl_sort_particles_by_block", "fl_p2g", "fl_pressure_project", "fl_g2p", "fl_step",
    "fl_upload_particles", "fl_download_particles", "fl_state_particles", "fl_state_fields", "fl_step_host",
    "fl_deposit_mac_3d", "fl_deposit_mac_quanta_3d", "fl_gather_mac_3d", "fl_copy_to_host", "fl_copy_to_device",
    "fl_runtime_info", "fl_apply_vcycle", "fl_step_timings", "fl_kernel_launches", "fl_unet_param_count",
    "fl_unet_create", "fl_unet_destroy", "fl_unet_init_params", "fl_unet_forward", "fl_unet_backward",
    "fl_unet_masked_mse", "fl_adam_step", "fl_collect_training_pairs", "fl_set_learned_preconditioner",
    "fl_apply_learned",
]

class MacPressureDiagnostics(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint64), ("true_residual_l2", ctypes.c_double),
                ("max_volume_scaled_residual", ctypes.c_double), ("max_cell_constraint_defect", ctypes.c_double),
                ("rhs_l2", ctypes.c_double), ("gauge_count", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StaticGrid(ctypes.Structure):
    """fl_static_grid: the caller-owned block layout of fl_p2g_static_scratch."""
    _fields_ = [("origin", ctypes.c_double * 3), ("h", ctypes.c_double), ("solid_lo", ctypes.c_int32 * 3),
                ("solid_hi", ctypes.c_int32 * 3), ("block_coords", ctypes.c_void_p), ("neighbors", ctypes.c_void_p),
                ("cell_start", ctypes.c_void_p), ("block_count", ctypes.c_uint64)]


class Epoch(ctypes.Structure):
    _fields_ = [("generation", ctypes.c_uint64), ("frame_ordinal", ctypes.c_uint64), ("time", ctypes.c_double)]


class SnapshotTicket(ctypes.Structure):
    _fields_ = [("slot", ctypes.c_uint32), ("reservation", ctypes.c_uint64), ("epoch", Epoch)]


class SnapshotView(ctypes.Structure):
    _fields_ = [("soa", ctypes.c_void_p), ("count", ctypes.c_uint64), ("epoch", Epoch), ("copy_ms", ctypes.c_float)]


_lib = None


def library():
    """Load the CUDA library (raises FluidityError when it is missing)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FluidityError(FAILED_PRECONDITION, f"CUDA library not built: {LIB_PATH}")
        lib = ctypes.CDLL(str(LIB_PATH))
        vp = ctypes.c_void_p
        lib.fl_context_create.argtypes = [ctypes.POINTER(GridDesc), ctypes.c_uint64, ctypes.POINTER(vp)]
        lib.fl_context_destroy.argtypes = [vp]
        lib.fl_topology_from_particles.argtypes = [vp, ctypes.POINTER(Particles), vp, ctypes.POINTER(Report)]
        lib.fl_topology_from_blocks.argtypes = [vp, _ip, ctypes.c_uint64]
        lib.fl_active_blocks.argtypes = [vp, _ip, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
        lib.fl_sort_particles_by_block.argtypes = [vp, ctypes.POINTER(Particles), ctypes.POINTER(Particles), vp,
                                                   ctypes.POINTER(Report)]
        lib.fl_p2g.argtypes = [vp, ctypes.POINTER(Particles), ctypes.POINTER(TransferParams), ctypes.c_int,
                               vp * 3, vp * 3, vp, ctypes.POINTER(Report)]
        lib.fl_p2g_normalized.argtypes = [vp, ctypes.POINTER(Particles), ctypes.POINTER(TransferParams), vp * 3,
                                          vp * 3, vp * 3, vp, ctypes.POINTER(Report)]
        lib.fl_p2g_static_scratch.argtypes = [ctypes.POINTER(StaticGrid), ctypes.POINTER(Particles),
                                              ctypes.POINTER(TransferParams), ctypes.c_int, vp * 3, vp * 3, vp,
                                              ctypes.POINTER(Report)]
        lib.fl_pressure_project.argtypes = [vp, vp * 3, vp * 3, ctypes.POINTER(TransferParams),
                                            ctypes.POINTER(PressureOptions), ctypes.POINTER(PressureDiagnostics),
                                            vp, vp]
        lib.fl_g2p.argtypes = [vp, ctypes.POINTER(Particles), vp * 3, vp * 3, ctypes.c_float, vp, vp,
                               ctypes.POINTER(Report)]
        lib.fl_step.argtypes = [vp, ctypes.POINTER(TransferParams), ctypes.POINTER(PressureOptions),
                                ctypes.POINTER(PressureDiagnostics), vp, ctypes.POINTER(Report)]
        lib.fl_upload_particles.argtypes = [vp, _fp, ctypes.c_uint64, vp]
        lib.fl_download_particles.argtypes = [vp, _fp, vp]
        lib.fl_stage_particles.argtypes = [vp, _fp, ctypes.c_uint64]
        lib.fl_state_particles.argtypes = [vp, ctypes.POINTER(Particles)]
        lib.fl_state_fields.argtypes = [vp, vp * 3, vp * 3, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                        ctypes.POINTER(vp)]
        lib.fl_step_host.argtypes = [vp, _fp, _fp, ctypes.c_uint64, ctypes.POINTER(TransferParams),
                                     ctypes.POINTER(PressureOptions), ctypes.POINTER(PressureDiagnostics), vp]
        lib.fl_deposit_mac_3d.argtypes = [_dp, ctypes.c_double, _ip, ctypes.c_uint64, _dp, ctypes.c_uint64, _dp, _dp,
                                          ctypes.POINTER(Measurement)]
        lib.fl_deposit_mac_quanta_3d.argtypes = [_dp, ctypes.c_double, _ip, ctypes.c_uint64, _dp, ctypes.c_uint64,
                                                 ctypes.c_double, ctypes.c_double, ctypes.c_uint64, _lp, _lp,
                                                 ctypes.POINTER(Measurement)]
        lib.fl_gather_mac_3d.argtypes = [_dp, ctypes.c_double, _ip, ctypes.c_uint64, _dp, ctypes.c_uint64, _dp, _dp,
                                         _dp, ctypes.POINTER(Measurement)]
        lib.fl_copy_to_host.argtypes = [vp, vp, ctypes.c_uint64]
        lib.fl_copy_to_device.argtypes = [vp, vp, ctypes.c_uint64]
        lib.fl_runtime_info.argtypes = [ctypes.POINTER(ctypes.c_int)] * 4
        lib.fl_apply_vcycle.argtypes = [vp, vp, vp, ctypes.POINTER(PressureOptions), vp]
        lib.fl_step_timings.argtypes = [vp, _fp]
        lib.fl_kernel_launches.argtypes = [ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong)]
        lib.fl_unet_param_count.restype = ctypes.c_int64
        lib.fl_unet_param_count.argtypes = []
        lib.fl_unet_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
        lib.fl_unet_destroy.argtypes = [vp]
        lib.fl_unet_set_tensor_cores.argtypes = [vp, ctypes.c_int]
        lib.fl_unet_init_params.argtypes = [vp, ctypes.c_uint64, vp]
        lib.fl_unet_forward.argtypes = [vp, vp, vp, ctypes.c_int, vp, vp]
        lib.fl_unet_backward.argtypes = [vp, vp, vp, ctypes.c_int, vp, vp]
        lib.fl_unet_masked_mse.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp]
        lib.fl_unet_block_residual_loss.argtypes = [vp, vp, ctypes.c_int, vp, vp, vp]
        lib.fl_adam_step.argtypes = [vp, vp, vp, vp, ctypes.c_uint64, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_float, vp]
        lib.fl_collect_training_pairs.argtypes = [vp, ctypes.POINTER(TransferParams), ctypes.POINTER(PressureOptions),
                                                  _ip, ctypes.c_int, vp, vp, vp, ctypes.c_uint64,
                                                  ctypes.POINTER(ctypes.c_uint64)]
        lib.fl_set_learned_preconditioner.argtypes = [vp, vp, vp]
        lib.fl_apply_learned.argtypes = [vp, vp, vp, ctypes.c_int, vp]
        lib.fl_project_mac_pressure_3d.argtypes = [ctypes.c_double, ctypes.c_double, _ip, _dp, ctypes.c_uint64, _ip, _ip,
                                                   _dp, ctypes.c_uint64, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp,
                                                   _dp, _dp, ctypes.POINTER(ctypes.c_uint64),
                                                   ctypes.POINTER(MacPressureDiagnostics), ctypes.POINTER(Measurement)]
        tk, ip = ctypes.POINTER(SnapshotTicket), ctypes.POINTER(ctypes.c_int)
        lib.fl_snapshot_queue_create.argtypes = [vp, ctypes.POINTER(vp)]
        lib.fl_snapshot_queue_destroy.argtypes = [vp]
        lib.fl_snapshot_begin.argtypes = [vp, ctypes.POINTER(Epoch), vp, tk]
        lib.fl_snapshot_poll.argtypes = [vp, tk, ip]
        lib.fl_snapshot_wait.argtypes = [vp, tk, ip]
        lib.fl_snapshot_finish.argtypes = [vp, tk, ctypes.POINTER(SnapshotView)]
        lib.fl_snapshot_release.argtypes = [vp, tk]
        lib.fl_snapshot_cancel.argtypes = [vp, tk]
        lib.fl_snapshot_last_valid.argtypes = [vp, ctypes.POINTER(SnapshotView)]
        _lib = lib
    return _lib


def _check(code: int, what: str):
    if code != OK:
        raise FluidityError(code, what)


def runtime_info():
    vals = [ctypes.c_int() for _ in range(4)]
    library().fl_runtime_info(*[ctypes.byref(v) for v in vals])
    return dict(compiled_architecture=vals[0].value, device_count=vals[1].value, major=vals[2].value,
                minor=vals[3].value)


def default_pressure_options(precision: int = 0, rel_tol: float = 1e-6, levels: int = 0, pre: int = 1,
                             post: int = 2, coarse_sweeps: int = 4, max_iterations: int = 400,
                             max_refinements: int = 6, inner_rtol: float = 1e-3,
                             warm_start: int = 0, preconditioner: int = 0, stall_limit: int = 3,
                             stall_ratio: float = 0.9) -> PressureOptions:
    """Solver options. One pre-smoothing and two post-smoothing sweeps per level: fewer V-cycle
    kernels for slightly more flexible-CG iterations, the fastest of the sweep counts measured
    (3.09 vs 3.24 ms per projection at the 256^3 splash, 1.19 vs 1.30 ms at the 128^3 dam break,
    against two and two)."""
    o = PressureOptions()
    o.warm_start = warm_start
    o.preconditioner, o.stall_limit, o.stall_ratio = preconditioner, stall_limit, stall_ratio
    o.levels, o.pre_sweeps, o.post_sweeps, o.coarse_sweeps = levels, pre, post, coarse_sweeps
    o.precision, o.max_iterations, o.max_refinements = precision, max_iterations, max_refinements
    o.rel_tol, o.inner_rtol = rel_tol, inner_rtol
    return o


def transfer_params(dt: float, particle_mass: float, gravity=(0.0, -9.81, 0.0), min_face_mass: float = 0.0,
                    density: float = 1000.0) -> TransferParams:
    t = TransferParams()
    t.dt, t.particle_mass = dt, particle_mass
    t.gravity[:] = list(gravity)
    t.min_face_mass, t.density = min_face_mass, density
    return t


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _d(a):
    return a.ctypes.data_as(_dp)


# ----------------------------------------------------------------------------- reference-shaped operators


def deposit_mac_3d(origin, h, blocks, particles):
    """GPU DepositMac3D: returns (face_mass, face_pure_momentum) in the
    reference's owned 4^3 slot order, plus the CUDA-event measurement."""
    blocks = np.ascontiguousarray(blocks, np.int32)
    parts = _f64(particles)
    fc = 192 * len(blocks)
    m, q = np.zeros(fc), np.zeros(fc)
    meas = Measurement()
    _check(library().fl_deposit_mac_3d(_d(_f64(origin)), float(h), blocks.ctypes.data_as(_ip), len(blocks), _d(parts),
                                       len(parts), _d(m), _d(q), ctypes.byref(meas)), "fl_deposit_mac_3d")
    return m, q, meas


def deposit_mac_quanta_3d(origin, h, blocks, particles, mass_per_quantum, momentum_per_quantum, capacity):
    blocks = np.ascontiguousarray(blocks, np.int32)
    parts = _f64(particles)
    fc = 192 * len(blocks)
    m, q = np.zeros(fc, np.int64), np.zeros(fc, np.int64)
    meas = Measurement()
    _check(library().fl_deposit_mac_quanta_3d(_d(_f64(origin)), float(h), blocks.ctypes.data_as(_ip), len(blocks),
                                              _d(parts), len(parts), float(mass_per_quantum),
                                              float(momentum_per_quantum), int(capacity), m.ctypes.data_as(_lp),
                                              q.ctypes.data_as(_lp), ctypes.byref(meas)), "fl_deposit_mac_quanta_3d")
    return m, q, meas


def project_mac_pressure_3d(cells_idx, cells_val, faces_idx, faces_kind, faces_val, h, dt, rel_tol=0.0,
                            max_iterations=256):
    """ProjectMacPressure3D on the GPU (fl_project_mac_pressure_3d): cells (n, 3) int32 with
    (n, 5) values, faces (m, 4) int32 with kinds (m,) and (m, 6) values, in the record
    layout of include/fluidity_b200.h. Returns pressure, rhs, residual, defect,
    corrected_u, gauges, diag and kernel_ms; raises FluidityError on a failed status."""
    ci = np.ascontiguousarray(cells_idx, np.int32)
    cv = np.ascontiguousarray(cells_val, np.float64)
    fi = np.ascontiguousarray(faces_idx, np.int32).reshape(-1, 4)
    fk = np.ascontiguousarray(faces_kind, np.int32).reshape(-1)
    fv = np.ascontiguousarray(faces_val, np.float64).reshape(-1, 6)
    nc, nf = ci.shape[0], fi.shape[0]
    p, b, r, d = np.zeros(nc), np.zeros(nc), np.zeros(nc), np.zeros(nc)
    u = np.zeros(max(nf, 1))
    g = np.zeros(max(nc, 1), np.uint64)
    diag, meas = MacPressureDiagnostics(), Measurement()
    code = library().fl_project_mac_pressure_3d(float(h), float(dt), ci.ctypes.data_as(_ip), cv.ctypes.data_as(_dp),
                                                nc, fi.ctypes.data_as(_ip), fk.ctypes.data_as(_ip),
                                                fv.ctypes.data_as(_dp), nf, int(max_iterations), float(rel_tol),
                                                p.ctypes.data_as(_dp), u.ctypes.data_as(_dp), b.ctypes.data_as(_dp),
                                                r.ctypes.data_as(_dp), d.ctypes.data_as(_dp),
                                                g.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                                ctypes.byref(diag), ctypes.byref(meas))
    if code != OK:
        raise FluidityError(code, f"fl_project_mac_pressure_3d ({diag.as_dict()})")
    return dict(pressure=p, rhs=b, residual=r, defect=d, corrected_u=u[:nf], gauges=g[:diag.gauge_count],
                diag=diag.as_dict(), kernel_ms=meas.kernel_ms, compiled_architecture=meas.compiled_architecture)


def gather_mac_3d(origin, h, blocks, particles, old_u, new_u):
    blocks = np.ascontiguousarray(blocks, np.int32)
    parts = _f64(particles)
    out = np.zeros((len(parts), 24))
    meas = Measurement()
    _check(library().fl_gather_mac_3d(_d(_f64(origin)), float(h), blocks.ctypes.data_as(_ip), len(blocks), _d(parts),
                                      len(parts), _d(_f64(old_u)), _d(_f64(new_u)), _d(out), ctypes.byref(meas)),
           "fl_gather_mac_3d")
    return out, meas


# ----------------------------------------------------------------------------- resident liquid context


class LiquidContext:
    """Resident device arena for the box scene: particles, sparse 8^3-block grid,
    solver buffers (fl_context_* in the C-ABI)."""

    def __init__(self, n, h=None, capacity=0, origin=(0.0, 0.0, 0.0), walls=True):
        n = tuple(int(v) for v in (n if np.iterable(n) else (n, n, n)))
        if any(v % 8 for v in n):
            raise ValueError("box cells per axis must be a multiple of 8")
        self.n = n
        self.h = float(h if h is not None else 1.0 / n[0])
        self.origin = tuple(float(v) for v in origin)
        d = GridDesc()
        d.origin[:] = list(self.origin)
        d.h = self.h
        d.block_lo[:] = [0, 0, 0]
        d.block_dim[:] = [v // 8 for v in n]
        if walls:
            d.solid_lo[:] = [1, 1, 1]
            d.solid_hi[:] = [v - 2 for v in n]
        else:
            d.solid_lo[:] = [-(2 ** 31)] * 3
            d.solid_hi[:] = [2 ** 31 - 1] * 3
        self.desc = d
        self.capacity = int(capacity)
        self._ctx = ctypes.c_void_p()
        _check(library().fl_context_create(ctypes.byref(d), self.capacity, ctypes.byref(self._ctx)),
               "fl_context_create")
        self.count = 0

    def close(self):
        if self._ctx:
            _check(library().fl_context_destroy(self._ctx), "fl_context_destroy (close its snapshot queues first)")
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._ctx

    def upload(self, soa: np.ndarray, stream=None):
        """soa: float32 array (15, count): x, y, z, vx, vy, vz, C rows."""
        soa = np.ascontiguousarray(soa, np.float32)
        self.count = soa.shape[1]
        _check(library().fl_upload_particles(self._ctx, soa.ctypes.data_as(_fp), self.count, stream),
               "fl_upload_particles")

    def stage(self, soa: np.ndarray):
        """Queues soa (float32 (15, count), pinned for an asynchronous copy) as the input of
        the next step that has none staged before it (fl_stage_particles)."""
        if soa.dtype != np.float32 or not soa.flags.c_contiguous:
            raise ValueError("stage needs a C-contiguous float32 (15, count) array")
        _check(library().fl_stage_particles(self._ctx, soa.ctypes.data_as(_fp), soa.shape[1]),
               "fl_stage_particles")

    def download(self, stream=None) -> np.ndarray:
        self.count = self.particles_view().count  # a staged input may have changed it
        out = np.zeros((15, self.count), np.float32)
        _check(library().fl_download_particles(self._ctx, out.ctypes.data_as(_fp), stream), "fl_download_particles")
        return out

    def step(self, params: TransferParams, options: PressureOptions, stream=None):
        diag = PressureDiagnostics()
        rep = Report()
        code = library().fl_step(self._ctx, ctypes.byref(params), ctypes.byref(options), ctypes.byref(diag), stream,
                                 ctypes.byref(rep))
        if code not in (OK, ABORTED):
            raise FluidityError(code, f"fl_step (report error {rep.error} at {rep.first_bad_index})")
        return code, diag

    def step_host(self, host_in: np.ndarray, host_out: np.ndarray, params, options, stream=None):
        diag = PressureDiagnostics()
        code = library().fl_step_host(self._ctx, host_in.ctypes.data_as(_fp), host_out.ctypes.data_as(_fp),
                                      host_in.shape[1], ctypes.byref(params), ctypes.byref(options),
                                      ctypes.byref(diag), stream)
        if code not in (OK, ABORTED):
            raise FluidityError(code, "fl_step_host")
        return code, diag

    def step_timings(self):
        """CUDA-event ms of the last step: topology+sort, P2G, pressure, G2P."""
        ms = np.zeros(4, np.float32)
        _check(library().fl_step_timings(self._ctx, ms.ctypes.data_as(_fp)), "fl_step_timings")
        return ms

    def active_blocks(self) -> np.ndarray:
        cnt = ctypes.c_uint64()
        library().fl_active_blocks(self._ctx, None, 0, ctypes.byref(cnt))
        out = np.zeros((cnt.value, 3), np.int32)
        if cnt.value:
            _check(library().fl_active_blocks(self._ctx, out.ctypes.data_as(_ip), cnt.value, ctypes.byref(cnt)),
                   "fl_active_blocks")
        return out

    def fields(self):
        """Device pointers of the last step's face fields, pressure, cell type and cell ranges."""
        up, un = (ctypes.c_void_p * 3)(), (ctypes.c_void_p * 3)()
        p, t, cs = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _check(library().fl_state_fields(self._ctx, up, un, ctypes.byref(p), ctypes.byref(t), ctypes.byref(cs)),
               "fl_state_fields")
        return dict(u_pred=list(up), u_new=list(un), pressure=p.value, cell_type=t.value, cell_start=cs.value)

    def particles_view(self) -> Particles:
        p = Particles()
        _check(library().fl_state_particles(self._ctx, ctypes.byref(p)), "fl_state_particles")
        return p

    def project(self, params: TransferParams, options: PressureOptions, stream=None):
        """Re-runs the pressure projection of the last step (its predicted velocities and
        cells) with `options`; returns (status code, diagnostics)."""
        f = self.fields()
        up = (ctypes.c_void_p * 3)(*f["u_pred"])
        un = (ctypes.c_void_p * 3)(*f["u_new"])
        diag = PressureDiagnostics()
        code = library().fl_pressure_project(self._ctx, up, un, ctypes.byref(params), ctypes.byref(options),
                                             ctypes.byref(diag), None, stream)
        if code not in (OK, ABORTED):
            raise FluidityError(code, "fl_pressure_project")
        return code, diag

    def collect_training_pairs(self, params: TransferParams, options: PressureOptions, iterations, inputs, targets,
                               masks) -> int:
        """(residual, error) items of the last step's projection into device tensors
        inputs (cap, 2, 10, 10, 10), targets and masks (cap, 512); returns the count."""
        its = np.ascontiguousarray(iterations, np.int32)
        cap = min(inputs.shape[0], targets.shape[0], masks.shape[0])
        written = ctypes.c_uint64()
        _check(library().fl_collect_training_pairs(self._ctx, ctypes.byref(params), ctypes.byref(options),
                                                   its.ctypes.data_as(_ip), len(its), inputs.data_ptr(),
                                                   targets.data_ptr(), masks.data_ptr(), cap, ctypes.byref(written)),
               "fl_collect_training_pairs")
        return written.value

    def set_learned_preconditioner(self, params, stream=None):
        """Loads FP32 network parameters (a device tensor) for options.preconditioner = 1."""
        _check(library().fl_set_learned_preconditioner(self._ctx, params.data_ptr(), stream),
               "fl_set_learned_preconditioner")

    def apply_learned(self, r, z, kernels: int = 0, stream=None):
        """z = U(r) on the cells of the last sort (device tensors, active_blocks*512 floats, natural
        order); kernels 0 = tensor-core inference, 1 = FP32 training forward."""
        _check(library().fl_apply_learned(self._ctx, r.data_ptr(), z.data_ptr(), int(kernels), stream),
               "fl_apply_learned")


class SnapshotQueue:
    """Asynchronous device-to-host snapshots of a context's particle state
    (fl_snapshot_* in the C-ABI; the reference's CudaLiquidSnapshotQueue3D,
    native/include/fluidity/host/cuda_liquid_snapshot_3d.h:56-110).

    ``begin`` queues the check and the copy of the state after the work queued
    on ``stream`` and returns a ticket; ``poll``/``wait`` report progress;
    ``finish`` validates the copy and returns a (15, count) float32 array that
    views the pinned slot memory until ``release``. The last finished snapshot
    stays readable through ``last_valid`` until the next finish. Error statuses
    raise FluidityError with the C-ABI code (UNAVAILABLE: both slots held)."""

    def __init__(self, ctx: LiquidContext):
        self._q = ctypes.c_void_p()
        self._ctx = ctx  # the context must outlive the queue
        _check(library().fl_snapshot_queue_create(ctx.handle, ctypes.byref(self._q)), "fl_snapshot_queue_create")

    def close(self):
        if self._q:
            library().fl_snapshot_queue_destroy(self._q)
            self._q = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def begin(self, generation: int, frame_ordinal: int = 0, time: float = 0.0, stream=None) -> SnapshotTicket:
        t = SnapshotTicket()
        e = Epoch(generation, frame_ordinal, time)
        _check(library().fl_snapshot_begin(self._q, ctypes.byref(e), stream, ctypes.byref(t)), "fl_snapshot_begin")
        return t

    def poll(self, ticket: SnapshotTicket) -> int:
        p = ctypes.c_int()
        _check(library().fl_snapshot_poll(self._q, ctypes.byref(ticket), ctypes.byref(p)), "fl_snapshot_poll")
        return p.value

    def wait(self, ticket: SnapshotTicket) -> int:
        p = ctypes.c_int()
        _check(library().fl_snapshot_wait(self._q, ctypes.byref(ticket), ctypes.byref(p)), "fl_snapshot_wait")
        return p.value

    @staticmethod
    def _array(v: SnapshotView) -> np.ndarray:
        if v.count == 0:
            return np.zeros((15, 0), np.float32)
        buf = (ctypes.c_float * (15 * v.count)).from_address(v.soa)
        return np.ctypeslib.as_array(buf).reshape(15, v.count)

    def finish(self, ticket: SnapshotTicket):
        """(state view (15, count), SnapshotView) of a READY ticket."""
        v = SnapshotView()
        _check(library().fl_snapshot_finish(self._q, ctypes.byref(ticket), ctypes.byref(v)), "fl_snapshot_finish")
        return self._array(v), v

    def release(self, ticket: SnapshotTicket):
        _check(library().fl_snapshot_release(self._q, ctypes.byref(ticket)), "fl_snapshot_release")

    def cancel(self, ticket: SnapshotTicket):
        _check(library().fl_snapshot_cancel(self._q, ctypes.byref(ticket)), "fl_snapshot_cancel")

    def last_valid(self):
        """(state view, SnapshotView) of the last finished snapshot, or None before the first."""
        v = SnapshotView()
        code = library().fl_snapshot_last_valid(self._q, ctypes.byref(v))
        if code == FAILED_PRECONDITION:
            return None
        _check(code, "fl_snapshot_last_valid")
        return self._array(v), v


class UNet:
    """Training handle of the learned block preconditioner (fl_unet_*). Tensors are
    device tensors (torch, float32, contiguous); calls are ordered on `stream`."""

    def __init__(self, max_batch: int, tensor_cores: bool = False):
        h = ctypes.c_void_p()
        _check(library().fl_unet_create(int(max_batch), ctypes.byref(h)), "fl_unet_create")
        self._h = h
        self.max_batch = int(max_batch)
        if tensor_cores:
            self.set_tensor_cores(True)

    def set_tensor_cores(self, enable: bool):
        """fl_unet_set_tensor_cores: the 3x3x3 training convolutions as BF16 GEMMs with
        FP32 accumulation on the tensor cores (True) or the FP32 kernels (False)."""
        _check(library().fl_unet_set_tensor_cores(self._h, 1 if enable else 0), "fl_unet_set_tensor_cores")

    @staticmethod
    def param_count() -> int:
        return int(library().fl_unet_param_count())

    @staticmethod
    def init_params(params, seed: int = 0, stream=None):
        _check(library().fl_unet_init_params(params.data_ptr(), int(seed), stream), "fl_unet_init_params")

    def forward(self, params, inputs, outputs, stream=None):
        _check(library().fl_unet_forward(self._h, params.data_ptr(), inputs.data_ptr(), inputs.shape[0],
                                         outputs.data_ptr(), stream), "fl_unet_forward")

    def backward(self, params, grad_outputs, grads, stream=None):
        _check(library().fl_unet_backward(self._h, params.data_ptr(), grad_outputs.data_ptr(), grad_outputs.shape[0],
                                          grads.data_ptr(), stream), "fl_unet_backward")

    @staticmethod
    def masked_mse(outputs, targets, masks, loss, grad_outputs, relative: int = 0, stream=None):
        _check(library().fl_unet_masked_mse(outputs.data_ptr(), targets.data_ptr(), masks.data_ptr(), outputs.shape[0],
                                            int(relative), loss.data_ptr(), grad_outputs.data_ptr(), stream),
               "fl_unet_masked_mse")

    @staticmethod
    def block_residual_loss(outputs, inputs, loss, grad_outputs, stream=None):
        """fl_unet_block_residual_loss: |r_b - A_b y|^2 / |r_b|^2 averaged over the items."""
        _check(library().fl_unet_block_residual_loss(outputs.data_ptr(), inputs.data_ptr(), outputs.shape[0],
                                                     loss.data_ptr(), grad_outputs.data_ptr(), stream),
               "fl_unet_block_residual_loss")

    @staticmethod
    def adam_step(params, grads, m, v, step: int, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999,
                  eps: float = 1e-8, stream=None):
        _check(library().fl_adam_step(params.data_ptr(), grads.data_ptr(), m.data_ptr(), v.data_ptr(), params.numel(),
                                      int(step), lr, beta1, beta2, eps, stream), "fl_adam_step")

    def close(self):
        if self._h:
            library().fl_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kernel_launches():
    own, libc = ctypes.c_ulonglong(), ctypes.c_ulonglong()
    library().fl_kernel_launches(ctypes.byref(own), ctypes.byref(libc))
    return own.value, libc.value


def copy_to_host(ptr, count, dtype) -> np.ndarray:
    out = np.zeros(count, dtype)
    if count:
        _check(library().fl_copy_to_host(out.ctypes.data, ptr, out.nbytes), "fl_copy_to_host")
    return out


def sparse_faces_to_dense(blocks: np.ndarray, sparse: np.ndarray, n, axis: int, fill=0.0) -> np.ndarray:
    """Scatter an owned-face array (nb*512, 8^3 layout) into a dense (z,y,x) box
    array with n[axis]+1 faces along the normal."""
    n = tuple(n)
    shape = [n[2], n[1], n[0]]
    shape[2 - axis] += 1
    dense = np.full(shape, fill, dtype=sparse.dtype)
    nb = len(blocks)
    loc = np.arange(512)
    lx, ly, lz = loc & 7, (loc >> 3) & 7, loc >> 6
    gx = (blocks[:, 0:1] * 8 + lx[None, :]).ravel()
    gy = (blocks[:, 1:2] * 8 + ly[None, :]).ravel()
    gz = (blocks[:, 2:3] * 8 + lz[None, :]).ravel()
    ok = (gx < shape[2]) & (gy < shape[1]) & (gz < shape[0])
    dense[gz[ok], gy[ok], gx[ok]] = sparse[: nb * 512][ok]
    return dense


def sparse_cells_to_dense(blocks: np.ndarray, sparse: np.ndarray, n, fill=0) -> np.ndarray:
    n = tuple(n)
    dense = np.full((n[2], n[1], n[0]), fill, dtype=sparse.dtype)
    loc = np.arange(512)
    lx, ly, lz = loc & 7, (loc >> 3) & 7, loc >> 6
    gx = (blocks[:, 0:1] * 8 + lx[None, :]).ravel()
    gy = (blocks[:, 1:2] * 8 + ly[None, :]).ravel()
    gz = (blocks[:, 2:3] * 8 + lz[None, :]).ravel()
    dense[gz, gy, gx] = sparse[: len(blocks) * 512]
    return dense
