"""The oracle: CPU checkers for the CUDA liquid-step path.

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / --impl reference legs import this package, always as the checker
or the timed CPU baseline, never as the thing measured or shipped.

Two checkers live here:

* ``cpu`` -- an FP64 restatement in C (oracle/cpu/fl_oracle.c) of the
  reference's stencil, P2G, normalize/forces, G2P and integrated pressure
  system, plus the geometric V-cycle the CUDA preconditioner implements.
* ``ref`` -- the reference's own CPU operators (DepositMac3D,
  DepositMacQuanta3D, GatherMac3D, ProjectMacPressure3D, ...) compiled from the
  FluidiTy sources by oracle/ref/Makefile into oracle/_ref/libfluidity_ref.so.
  The reference caps these at 2^20 quantized particles and 4096 pressure cells.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
CPU_LIB = HERE / "_lib" / "libfl_oracle.so"
REF_LIB = HERE / "_ref" / "libfluidity_ref.so"
# The FluidiTy sources: $FLUIDITY_REFERENCE, else a checkout beside this repository.
REFERENCE_ROOT = Path(os.environ.get("FLUIDITY_REFERENCE", str(HERE.parent.parent / "reference")))

_cpu = None
_ref = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lp = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build(force: bool = False) -> None:
    """Compile the C restatement, and the reference operators when the FluidiTy
    sources are present (a machine without those sources uses the prebuilt files)."""
    (HERE / "_lib").mkdir(exist_ok=True)
    src = HERE / "cpu" / "fl_oracle.c"
    if force or not CPU_LIB.exists() or CPU_LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.check_call(
            ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-o", str(CPU_LIB), str(src), "-lm"]
        )
    if (REFERENCE_ROOT / "native" / "src").is_dir():
        subprocess.check_call(
            ["make", "-s", "-C", str(HERE / "ref"), f"REF={REFERENCE_ROOT}", "-j8"]
        )


class Box(ctypes.Structure):
    _fields_ = [
        ("origin", ctypes.c_double * 3),
        ("h", ctypes.c_double),
        ("lo", ctypes.c_int32 * 3),
        ("n", ctypes.c_int32 * 3),
    ]

    @staticmethod
    def make(origin, h, lo, n) -> "Box":
        b = Box()
        b.origin[:] = [float(v) for v in origin]
        b.h = float(h)
        b.lo[:] = [int(v) for v in lo]
        b.n[:] = [int(v) for v in n]
        return b

    def face_shape(self, axis: int):
        nx, ny, nz = (self.n[d] + (1 if d == axis else 0) for d in range(3))
        return (nz, ny, nx)


class PressureInputs(ctypes.Structure):
    _fields_ = [
        ("nc", ctypes.c_size_t),
        ("nf", ctypes.c_size_t),
        ("cell_index", _ip),
        ("cell_values", _dp),
        ("face_index", _ip),
        ("face_kind", _ip),
        ("face_values", _dp),
        ("h", ctypes.c_double),
        ("dt", ctypes.c_double),
    ]


class PressureDiag(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_double),
        ("true_residual_l2", ctypes.c_double),
        ("max_volume_scaled_residual", ctypes.c_double),
        ("max_defect", ctypes.c_double),
        ("rhs_l2", ctypes.c_double),
        ("gauge_count", ctypes.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class StepParams(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double),
        ("density", ctypes.c_double),
        ("gravity", ctypes.c_double * 3),
        ("m_min", ctypes.c_double),
        ("rel_tol", ctypes.c_double),
        ("clamp_margin", ctypes.c_double),
        ("max_iterations", ctypes.c_size_t),
    ]


def cpu():
    """The FP64 C restatement (built on first use when missing)."""
    global _cpu
    if _cpu is None:
        if not CPU_LIB.exists():
            build()
        lib = ctypes.CDLL(str(CPU_LIB))
        lib.fo_stencil.argtypes = [_dp, ctypes.c_double, ctypes.c_int, _dp, _ip, _dp]
        lib.fo_p2g.argtypes = [ctypes.POINTER(Box), _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_size_t,
                               _dp * 3, _dp * 3]
        lib.fo_p2g_quanta.argtypes = [ctypes.POINTER(Box), _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_size_t,
                                      ctypes.c_double, ctypes.c_double, _lp * 3, _lp * 3]
        lib.fo_normalize_forces.argtypes = [ctypes.POINTER(Box), _dp * 3, _dp * 3, ctypes.c_double,
                                            ctypes.c_double, _dp, _dp * 3, _u8p * 3]
        lib.fo_g2p.argtypes = [ctypes.POINTER(Box), _dp, ctypes.c_size_t, ctypes.c_void_p, _dp * 3, _dp]
        lib.fo_pressure_solve.argtypes = [ctypes.POINTER(PressureInputs), ctypes.c_double, ctypes.c_size_t,
                                          _dp, _dp, _dp, _dp, _dp, ctypes.POINTER(PressureDiag)]
        lib.fo_pressure_evaluate.argtypes = [ctypes.POINTER(PressureInputs), _dp, _dp, _dp, _dp, _dp,
                                             ctypes.POINTER(PressureDiag)]
        lib.fo_classify_cells.argtypes = [ctypes.POINTER(Box), _dp, ctypes.c_size_t, _u8p]
        lib.fo_step.argtypes = [ctypes.POINTER(Box), ctypes.POINTER(StepParams), _dp, _dp, _dp, ctypes.c_size_t,
                                _dp * 3, _dp * 3, _dp, _u8p, ctypes.POINTER(PressureDiag)]
        lib.fo_step_replay.argtypes = [ctypes.POINTER(Box), ctypes.POINTER(StepParams), ctypes.POINTER(ctypes.c_float),
                                       ctypes.c_size_t, _dp, ctypes.c_size_t, ctypes.c_size_t, _dp * 3, _dp * 3, _u8p,
                                       ctypes.POINTER(PressureDiag), _dp]
        lib.fo_vcycle.argtypes = [ctypes.POINTER(Box), _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, _dp, _dp]
        _cpu = lib
    return _cpu


def ref():
    """The reference's own compiled CPU operators, or None when not built."""
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            return None
        lib = ctypes.CDLL(str(REF_LIB))
        lib.ref_grid_face_count.restype = ctypes.c_longlong
        lib.ref_grid_face_count.argtypes = [_dp, ctypes.c_double, _ip, ctypes.c_size_t]
        lib.ref_grid_face_indices.argtypes = [_dp, ctypes.c_double, _ip, ctypes.c_size_t, _ip]
        lib.ref_particle_sort_bin.argtypes = [_dp, ctypes.c_double, _dp, _ip]
        lib.ref_geometry_stencil.argtypes = [_dp, ctypes.c_double, ctypes.c_int, _dp, _dp, _ip, _dp]
        lib.ref_deposit_mac_3d.argtypes = [_dp, ctypes.c_double, _ip, ctypes.c_size_t, _dp, ctypes.c_size_t,
                                           _dp, _dp]
        lib.ref_deposit_mac_quanta_3d.argtypes = [_dp, ctypes.c_double, _ip, ctypes.c_size_t, _dp,
                                                  ctypes.c_size_t, ctypes.c_double, ctypes.c_double,
                                                  ctypes.c_size_t, _lp, _lp]
        lib.ref_gather_mac_3d.argtypes = [_dp, ctypes.c_double, _ip, ctypes.c_size_t, _dp, ctypes.c_size_t,
                                          _dp, _dp, _dp]
        lib.ref_normalize_liquid_mac_faces_3d.argtypes = [_lp, _lp, ctypes.c_size_t, ctypes.c_double, ctypes.c_double,
                                                          ctypes.c_size_t, ctypes.c_double, _dp, _dp, _u8p]
        lib.ref_project_mac_pressure_3d.argtypes = [
            _dp, ctypes.c_double, _ip, ctypes.c_size_t, ctypes.c_double, _ip, _dp, ctypes.c_size_t, _ip, _ip,
            _dp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_double, _dp, _dp, _dp, _dp, _dp, _dp]
        _ref = lib
    return _ref


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _l(a):
    return a.ctypes.data_as(_lp)


def _u8(a):
    return a.ctypes.data_as(_u8p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OracleError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what} failed with status {code}")
        self.code = code


def _check(code: int, what: str):
    if code != 0:
        raise OracleError(code, what)


# --------------------------------------------------------------------------- restatement


def stencil(origin, h, axis, pos):
    faces = np.zeros((27, 4), np.int32)
    vals = np.zeros((27, 7), np.float64)
    _check(cpu().fo_stencil(_d(_f64(origin)), float(h), int(axis), _d(_f64(pos)), _i(faces), _d(vals)), "stencil")
    return faces, vals


def p2g(box: Box, x, v, c, mass):
    x, v, c = _f64(x), _f64(v), _f64(c)
    mass = _f64(np.atleast_1d(mass))
    stride = 0 if mass.size == 1 else 1
    fm = [np.zeros(box.face_shape(a)) for a in range(3)]
    fq = [np.zeros(box.face_shape(a)) for a in range(3)]
    _check(cpu().fo_p2g(ctypes.byref(box), _d(x), _d(v), _d(c), _d(mass), stride, x.shape[0],
                        (_dp * 3)(*[_d(a) for a in fm]), (_dp * 3)(*[_d(a) for a in fq])), "p2g")
    return fm, fq


def p2g_quanta(box: Box, x, v, c, mass, mass_per_quantum, momentum_per_quantum):
    x, v, c = _f64(x), _f64(v), _f64(c)
    mass = _f64(np.atleast_1d(mass))
    stride = 0 if mass.size == 1 else 1
    mq = [np.zeros(box.face_shape(a), np.int64) for a in range(3)]
    pq = [np.zeros(box.face_shape(a), np.int64) for a in range(3)]
    _check(cpu().fo_p2g_quanta(ctypes.byref(box), _d(x), _d(v), _d(c), _d(mass), stride, x.shape[0],
                               float(mass_per_quantum), float(momentum_per_quantum),
                               (_lp * 3)(*[_l(a) for a in mq]), (_lp * 3)(*[_l(a) for a in pq])), "p2g_quanta")
    return mq, pq


def normalize_forces(box: Box, fm, fq, m_min, dt, g):
    u = [np.zeros(box.face_shape(a)) for a in range(3)]
    valid = [np.zeros(box.face_shape(a), np.uint8) for a in range(3)]
    cpu().fo_normalize_forces(ctypes.byref(box), (_dp * 3)(*[_d(a) for a in fm]), (_dp * 3)(*[_d(a) for a in fq]),
                              float(m_min), float(dt), _d(_f64(g)), (_dp * 3)(*[_d(a) for a in u]),
                              (_u8p * 3)(*[_u8(a) for a in valid]))
    return u, valid


def g2p(box: Box, x, u_new, u_old=None):
    x = _f64(x)
    out = np.zeros((x.shape[0], 24))
    un = [_f64(a) for a in u_new]
    old = None
    if u_old is not None:
        uo = [_f64(a) for a in u_old]
        old = ctypes.cast((_dp * 3)(*[_d(a) for a in uo]), ctypes.c_void_p)
    _check(cpu().fo_g2p(ctypes.byref(box), _d(x), x.shape[0], old, (_dp * 3)(*[_d(a) for a in un]), _d(out)), "g2p")
    return out


def classify_cells(box: Box, x):
    x = _f64(x)
    t = np.zeros((box.n[2], box.n[1], box.n[0]), np.uint8)
    cpu().fo_classify_cells(ctypes.byref(box), _d(x), x.shape[0], _u8(t))
    return t


def _pressure_inputs(cells_idx, cells_val, faces_idx, faces_kind, faces_val, h, dt):
    keep = [np.ascontiguousarray(cells_idx, np.int32), _f64(cells_val), np.ascontiguousarray(faces_idx, np.int32),
            np.ascontiguousarray(faces_kind, np.int32), _f64(faces_val)]
    pi = PressureInputs(len(keep[0]), len(keep[2]), _i(keep[0]), _d(keep[1]), _i(keep[2]), _i(keep[3]),
                        _d(keep[4]), float(h), float(dt))
    return pi, keep


def pressure_solve(cells_idx, cells_val, faces_idx, faces_kind, faces_val, h, dt, rel_tol=0.0, max_iterations=10000):
    """FP64 solve of the integrated MAC pressure system (see fl_oracle.h)."""
    pi, keep = _pressure_inputs(cells_idx, cells_val, faces_idx, faces_kind, faces_val, h, dt)
    nc, nf = pi.nc, pi.nf
    p, r, d, b, u = (np.zeros(nc), np.zeros(nc), np.zeros(nc), np.zeros(nc), np.zeros(nf))
    diag = PressureDiag()
    code = cpu().fo_pressure_solve(ctypes.byref(pi), float(rel_tol), int(max_iterations), _d(p), _d(r), _d(d), _d(b),
                                   _d(u), ctypes.byref(diag))
    _check(code, "pressure_solve")
    return dict(pressure=p, residual=r, defect=d, rhs=b, corrected_u=u, diag=diag.as_dict())


def pressure_evaluate(cells_idx, cells_val, faces_idx, faces_kind, faces_val, h, dt, pressure):
    pi, keep = _pressure_inputs(cells_idx, cells_val, faces_idx, faces_kind, faces_val, h, dt)
    nc, nf = pi.nc, pi.nf
    r, d, b, u = (np.zeros(nc), np.zeros(nc), np.zeros(nc), np.zeros(nf))
    diag = PressureDiag()
    p = _f64(pressure)
    _check(cpu().fo_pressure_evaluate(ctypes.byref(pi), _d(p), _d(r), _d(d), _d(b), _d(u), ctypes.byref(diag)),
           "pressure_evaluate")
    return dict(residual=r, defect=d, rhs=b, corrected_u=u, diag=diag.as_dict())


def step(box: Box, x, v, c, dt, density=1000.0, gravity=(0.0, -9.81, 0.0), m_min=0.0, rel_tol=1e-6,
         clamp_margin=1e-3, max_iterations=20000):
    """One FP64 APIC liquid step on the box scene; x, v, c updated copies are returned."""
    x, v, c = _f64(x).copy(), _f64(v).copy(), _f64(c).copy()
    prm = StepParams()
    prm.dt, prm.density = dt, density
    prm.gravity[:] = list(gravity)
    prm.m_min, prm.rel_tol, prm.clamp_margin, prm.max_iterations = m_min, rel_tol, clamp_margin, max_iterations
    u_pred = [np.zeros(box.face_shape(a)) for a in range(3)]
    u_new = [np.zeros(box.face_shape(a)) for a in range(3)]
    cp = np.zeros((box.n[2], box.n[1], box.n[0]))
    ct = np.zeros((box.n[2], box.n[1], box.n[0]), np.uint8)
    diag = PressureDiag()
    _check(cpu().fo_step(ctypes.byref(box), ctypes.byref(prm), _d(x), _d(v), _d(c), x.shape[0],
                         (_dp * 3)(*[_d(a) for a in u_pred]), (_dp * 3)(*[_d(a) for a in u_new]), _d(cp), _u8(ct),
                         ctypes.byref(diag)), "step")
    return dict(x=x, v=v, c=c, u_pred=u_pred, u_new=u_new, pressure=cp, cell_type=ct, diag=diag.as_dict())


def step_replay(box: Box, soa, cell_pressure, dt, first=0, stride=1, density=1000.0, gravity=(0.0, -9.81, 0.0),
                m_min=0.0, clamp_margin=1e-3):
    """One FP64 step from the FP32 SoA state `soa` (15 x np) with the pressure
    given (dense over the box) instead of solved: returns the predicted and
    corrected face velocities, the cell types, the FP64 evaluation of the given
    pressure on the step's own system (true residual, ||b||), and x, v, C after
    the step for the particles first, first + stride, ... ((n_sample, 15))."""
    soa = np.ascontiguousarray(soa, np.float32)
    np_ = soa.shape[1]
    prm = StepParams()
    prm.dt, prm.density = dt, density
    prm.gravity[:] = list(gravity)
    prm.m_min, prm.rel_tol, prm.clamp_margin, prm.max_iterations = m_min, 0.0, clamp_margin, 0
    u_pred = [np.zeros(box.face_shape(a)) for a in range(3)]
    u_new = [np.zeros(box.face_shape(a)) for a in range(3)]
    ct = np.zeros((box.n[2], box.n[1], box.n[0]), np.uint8)
    cp = _f64(cell_pressure)
    nsample = len(range(first, np_, stride)) if stride > 0 else 0
    sample = np.zeros((max(nsample, 1), 15))
    diag = PressureDiag()
    _check(cpu().fo_step_replay(ctypes.byref(box), ctypes.byref(prm), soa.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                np_, _d(cp), int(first), int(stride), (_dp * 3)(*[_d(a) for a in u_pred]),
                                (_dp * 3)(*[_d(a) for a in u_new]), _u8(ct), ctypes.byref(diag), _d(sample)),
           "step_replay")
    return dict(u_pred=u_pred, u_new=u_new, cell_type=ct, diag=diag.as_dict(), sample=sample[:nsample],
                sample_index=np.arange(first, np_, stride) if stride > 0 else np.zeros(0, np.int64))


def vcycle(box: Box, cell_type, r, levels=4, pre=2, post=2, coarse_sweeps=8):
    ct = np.ascontiguousarray(cell_type, np.uint8)
    r = _f64(r)
    z = np.zeros_like(r)
    _check(cpu().fo_vcycle(ctypes.byref(box), _u8(ct), levels, pre, post, coarse_sweeps, _d(r), _d(z)), "vcycle")
    return z


# --------------------------------------------------------------------------- reference operators


def particles_aos(x, v, c, mass, trial=None):
    """Pack MacTransferParticle3D records (19 doubles each)."""
    x = _f64(x)
    n = x.shape[0]
    out = np.zeros((n, 19))
    out[:, 0:3] = x
    out[:, 3:6] = x if trial is None else _f64(trial)
    out[:, 6] = np.broadcast_to(_f64(mass), (n,))
    out[:, 7:10] = _f64(v)
    out[:, 10:19] = _f64(c).reshape(n, 9)
    return out


def ref_face_indices(origin, h, blocks):
    lib = ref()
    blocks = np.ascontiguousarray(blocks, np.int32)
    count = lib.ref_grid_face_count(_d(_f64(origin)), float(h), _i(blocks), len(blocks))
    if count < 0:
        raise OracleError(int(-count), "ref_grid_face_count")
    out = np.zeros((count, 4), np.int32)
    _check(lib.ref_grid_face_indices(_d(_f64(origin)), float(h), _i(blocks), len(blocks), _i(out)), "face_indices")
    return out


def ref_deposit(origin, h, blocks, particles):
    lib = ref()
    blocks = np.ascontiguousarray(blocks, np.int32)
    fc = lib.ref_grid_face_count(_d(_f64(origin)), float(h), _i(blocks), len(blocks))
    m, q = np.zeros(fc), np.zeros(fc)
    parts = _f64(particles)
    _check(lib.ref_deposit_mac_3d(_d(_f64(origin)), float(h), _i(blocks), len(blocks), _d(parts), len(parts), _d(m),
                                  _d(q)), "DepositMac3D")
    return m, q


def ref_deposit_quanta(origin, h, blocks, particles, mass_per_quantum, momentum_per_quantum, capacity):
    lib = ref()
    blocks = np.ascontiguousarray(blocks, np.int32)
    fc = lib.ref_grid_face_count(_d(_f64(origin)), float(h), _i(blocks), len(blocks))
    m, q = np.zeros(fc, np.int64), np.zeros(fc, np.int64)
    parts = _f64(particles)
    _check(lib.ref_deposit_mac_quanta_3d(_d(_f64(origin)), float(h), _i(blocks), len(blocks), _d(parts), len(parts),
                                         float(mass_per_quantum), float(momentum_per_quantum), int(capacity), _l(m),
                                         _l(q)), "DepositMacQuanta3D")
    return m, q


def ref_normalize(mass_q, momentum_q, mass_per_quantum, momentum_per_quantum, capacity, minimum_face_mass):
    """NormalizeLiquidMacFaces3D: decoded face masses, velocities and validity bytes."""
    lib = ref()
    mq, pq = np.ascontiguousarray(mass_q, np.int64), np.ascontiguousarray(momentum_q, np.int64)
    n = len(mq)
    m, u, val = np.zeros(n), np.zeros(n), np.zeros(n, np.uint8)
    _check(lib.ref_normalize_liquid_mac_faces_3d(_l(mq), _l(pq), n, float(mass_per_quantum), float(momentum_per_quantum),
                                                 int(capacity), float(minimum_face_mass), _d(m), _d(u), _u8(val)),
           "NormalizeLiquidMacFaces3D")
    return m, u, val


def ref_gather(origin, h, blocks, particles, old_u, new_u):
    lib = ref()
    blocks = np.ascontiguousarray(blocks, np.int32)
    parts = _f64(particles)
    out = np.zeros((len(parts), 24))
    _check(lib.ref_gather_mac_3d(_d(_f64(origin)), float(h), _i(blocks), len(blocks), _d(parts), len(parts),
                                 _d(_f64(old_u)), _d(_f64(new_u)), _d(out)), "GatherMac3D")
    return out


def ref_project(origin, h, blocks, dt, cells_idx, cells_val, faces_idx, faces_kind, faces_val, max_iterations=256,
                tolerance_scale=1.0):
    lib = ref()
    blocks = np.ascontiguousarray(blocks, np.int32)
    ci, cv = np.ascontiguousarray(cells_idx, np.int32), _f64(cells_val)
    fi, fk, fv = np.ascontiguousarray(faces_idx, np.int32), np.ascontiguousarray(faces_kind, np.int32), _f64(faces_val)
    nc, nf = len(ci), len(fi)
    p, r, d, b, u, diag = np.zeros(nc), np.zeros(nc), np.zeros(nc), np.zeros(nc), np.zeros(nf), np.zeros(5)
    _check(lib.ref_project_mac_pressure_3d(_d(_f64(origin)), float(h), _i(blocks), len(blocks), float(dt), _i(ci),
                                           _d(cv), nc, _i(fi), _i(fk), _d(fv), nf, int(max_iterations),
                                           float(tolerance_scale), _d(p), _d(r), _d(d), _d(b), _d(u), _d(diag)),
           "ProjectMacPressure3D")
    return dict(pressure=p, residual=r, defect=d, rhs=b, corrected_u=u,
                diag=dict(iterations=diag[0], levels=diag[1], true_residual_l2=diag[2],
                          max_volume_scaled_residual=diag[3], max_defect=diag[4]))
