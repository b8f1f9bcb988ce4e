"""ctypes view of the backend-table harness (oracle/_ref/libfluidity_backend_check.so)
and the bounded 32^3 tank dam break the table tests run on.

The harness runs one LiquidSubstepBackend3D operation through the reference's
own CPU table (which=0) or the B200 table (which=1) on the same inputs. The
numpy record dtypes below are the reference's record layouts
(liquid_boundary_transfer_types_3d.h:4-45, mac_transfer_types_3d.h:7-30).

Scene: a 32^3 tank (h = 1/32 m, walls on the lattice planes 0 and 32) with a
4 x 8 x 4-cell water column in its low corner, 8 particles per cell (1024,
the boundary path's particle cap), small seeded velocities and APIC slopes,
trial positions moved less than half a cell. Faces inside the tank are
structurally eligible; faces on or beyond the tank's walls are ineligible and
carry a prescribed wall at rest (the inward normal of the first low wall they
lie on or beyond). With mixed_sides the column's top two cell layers (y >= 6)
carry side tag 1, as do the faces and walls there, so the compatible-support
masks mix sides; a ghost of one side next to the other side's walls then has
no support, so the gather runs on the one-sided scene. Active 4^3 blocks: x, z in [-1, 2],
y in [-1, 3] (80 blocks, 15360 face slots).
"""

from __future__ import annotations

import ctypes

import numpy as np

import oracle

LIB_PATH = oracle.HERE / "_ref" / "libfluidity_backend_check.so"

PARTICLE = np.dtype([("sorted", "<f8", 3), ("trial", "<f8", 3), ("mass", "<f8"), ("velocity", "<f8", 3),
                     ("slopes", "<f8", 9), ("side", "<i8"), ("affine", "u1"), ("pad", "u1", 7)])
TAG = np.dtype([("side", "<i8"), ("eligible", "u1"), ("pad", "u1", 7)])
QUANTA = np.dtype([("mass", "<i8"), ("momentum", "<i8"), ("stress", "<i8")])
SAMPLE = np.dtype([("slot", "<u8"), ("compatible", "u1"), ("pad", "u1", 7), ("weight", "<f8"),
                   ("gradient", "<f8", 3), ("centered", "<f8", 3)])
WALL = np.dtype([("available", "u1"), ("pad", "u1", 7), ("side", "<i8"), ("normal", "<f8", 3),
                 ("velocity", "<f8", 3)])
GATHERED = np.dtype([("new_pic", "<f8", 3), ("increment", "<f8", 3), ("retained", "<f8", 3), ("slopes", "<f8", 9),
                     ("gradient", "<f8", 9), ("affine", "u1"), ("old_fallback", "u1"), ("new_fallback", "u1"),
                     ("low_mass", "u1"), ("pad", "u1", 4)])
assert (PARTICLE.itemsize, TAG.itemsize, QUANTA.itemsize, SAMPLE.itemsize, WALL.itemsize, GATHERED.itemsize) == (
    168, 16, 24, 72, 64, 224)

CPU, B200 = 0, 1
MASS_Q = 2.0 ** -40
MOMENTUM_Q = 2.0 ** -40
N = 32
H = 1.0 / N
DT = 1.0 / 240.0
GRAVITY = (0.0, -9.81, 0.0)


def available() -> bool:
    return LIB_PATH.exists()


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(LIB_PATH))
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _d3(v):
    return (ctypes.c_double * 3)(*[float(x) for x in v])


def last_op_ms() -> float:
    """Host time of the harness's last table operation alone, ms."""
    f = lib().bk_last_op_ms
    f.restype = ctypes.c_double
    return float(f())


def filled(which):
    m = ctypes.c_uint32(0)
    code = lib().bk_filled(ctypes.c_int(which), ctypes.byref(m))
    return code, m.value


class Scene:
    """The bounded tank dam break, its face tags and walls."""

    def __init__(self, seed: int = 7, mixed_sides: bool = True):
        rng = np.random.default_rng(seed)
        self.origin = np.zeros(3)
        bz, by, bx = np.meshgrid(np.arange(-1, 3), np.arange(-1, 4), np.arange(-1, 3), indexing="ij")
        self.blocks = np.stack([bx.ravel(), by.ravel(), bz.ravel()], 1).astype(np.int32)  # (z,y,x) order
        self.faces = 192 * len(self.blocks)
        cz, cy, cx = np.meshgrid(np.arange(4), np.arange(8), np.arange(4), indexing="ij")
        cells = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], 1).astype(np.float64)
        sub = np.array([[i, j, k] for k in (0.25, 0.75) for j in (0.25, 0.75) for i in (0.25, 0.75)])
        pos = (cells[:, None, :] + sub[None] + rng.uniform(-0.2, 0.2, (len(cells), 8, 3))).reshape(-1, 3)
        n = len(pos)
        p = np.zeros(n, PARTICLE)
        p["sorted"] = pos * H
        trial = pos + rng.uniform(-0.3, 0.3, pos.shape)
        trial = np.clip(trial, 0.02, None)
        trial = np.minimum(np.maximum(trial, pos - 0.45), pos + 0.45)
        p["trial"] = trial * H
        p["mass"] = 1000.0 * H ** 3 / 8
        p["velocity"] = rng.uniform(-0.5, 0.5, (n, 3))
        p["slopes"] = rng.uniform(-2.0, 2.0, (n, 9))
        p["side"] = (pos[:, 1] >= 6.0).astype(np.int64) if mixed_sides else 0
        p["affine"] = (np.arange(n) % 16 != 5).astype(np.uint8)
        self.particles = p
        # face slots: block ordinal, axis, local (z,y,x)
        slot = np.arange(self.faces)
        blk = self.blocks[slot // 192]
        axis = (slot % 192) // 64
        local = slot % 64
        lat = blk * 4 + np.stack([local % 4, (local // 4) % 4, local // 16], 1)
        self.axis, self.lattice = axis, lat
        inside = np.ones(self.faces, bool)
        for a in range(3):
            on = axis == a
            inside &= np.where(on, (lat[:, a] > 0) & (lat[:, a] < N), (lat[:, a] >= 0) & (lat[:, a] < N))
        tags = np.zeros(self.faces, TAG)
        tags["eligible"] = inside.astype(np.uint8)
        tags["side"] = (lat[:, 1] >= 6).astype(np.int64) if mixed_sides else 0
        self.tags = tags
        # every ineligible face is a prescribed wall at rest, its normal the
        # inward normal of the first low tank wall it lies on or beyond
        walls = np.zeros(self.faces, WALL)
        walls["available"] = (~inside).astype(np.uint8)
        walls["side"] = tags["side"]
        normal_axis = np.full(self.faces, -1)
        for a in (2, 1, 0):
            low = np.where(axis == a, lat[:, a] <= 0, lat[:, a] < 0)
            normal_axis = np.where(low, a, normal_axis)
        normal_axis = np.where((normal_axis < 0) & ~inside, axis, normal_axis)
        rows = np.nonzero(~inside)[0]
        walls["normal"][rows, normal_axis[rows]] = 1.0
        self.walls = walls

    def grid_args(self):
        return (_d3(self.origin), ctypes.c_double(H), _p(self.blocks), ctypes.c_uint64(len(self.blocks)))


def deposit(which, s: Scene, particles=None, tags=None, capacity=1024):
    particles = s.particles if particles is None else particles
    tags = s.tags if tags is None else tags
    q = np.zeros(s.faces, QUANTA)
    st = np.zeros((len(particles), 3, 27), SAMPLE)
    code = lib().bk_deposit(ctypes.c_int(which), *s.grid_args(), _p(particles), ctypes.c_uint64(len(particles)),
                            _p(tags), ctypes.c_double(MASS_Q), ctypes.c_double(MOMENTUM_Q), ctypes.c_uint64(capacity),
                            _p(q), _p(st))
    return code, q, st


def normalize(which, quanta, min_mass, capacity=1024):
    n = len(quanta)
    m, v, val = np.zeros(n), np.zeros(n), np.zeros(n, np.uint8)
    code = lib().bk_normalize(ctypes.c_int(which), _p(quanta), ctypes.c_uint64(n), ctypes.c_double(MASS_Q),
                              ctypes.c_double(MOMENTUM_Q), ctypes.c_uint64(capacity), ctypes.c_double(min_mass),
                              _p(m), _p(v), _p(val))
    return code, m, v, val


def forces(which, s: Scene, old, acceleration=GRAVITY, dt=DT):
    out = np.zeros(s.faces)
    code = lib().bk_forces(ctypes.c_int(which), *s.grid_args(), _p(np.ascontiguousarray(old)), _d3(acceleration),
                           ctypes.c_double(dt), _p(out))
    return code, out


def predict(which, s: Scene, velocities, validity, slot, side, acceleration=GRAVITY, dt=DT, time=0.0):
    out = ctypes.c_double(np.nan)
    code = lib().bk_predict(ctypes.c_int(which), *s.grid_args(), ctypes.c_double(time), _p(velocities),
                            _p(validity), _p(s.tags), _p(s.walls), ctypes.c_uint64(slot), ctypes.c_int64(side),
                            _d3(acceleration), ctypes.c_double(dt), ctypes.byref(out))
    return code, out.value


def gather(which, s: Scene, old, new, t0=0.0, t1=DT, particles=None):
    """old/new: (velocities, validity) per slot; tags and walls are the scene's."""
    particles = s.particles if particles is None else particles
    out = np.zeros(len(particles), GATHERED)
    counts = (ctypes.c_uint64 * 3)()
    code = lib().bk_gather(ctypes.c_int(which), *s.grid_args(), _p(particles), ctypes.c_uint64(len(particles)),
                           ctypes.c_double(t0), ctypes.c_double(t1), _p(old[0]), _p(old[1]), _p(s.tags),
                           _p(s.walls), _p(new[0]), _p(new[1]), _p(s.tags), _p(s.walls), _p(out), counts)
    return code, out, np.array(counts[:], np.uint64)


def project(which, system, h, dt, max_iterations=256, tolerance_scale=1.0, face_flux=None):
    """system: oracle.box_system.box_pressure_system output (faces in owned-slot order)."""
    ci, cv = system["cells_idx"], system["cells_val"]
    fi, fk, fv = system["faces_idx"], system["faces_kind"], system["faces_val"]
    lat = fi[:, 1:4].astype(np.int64)
    owners = np.unique(np.floor_divide(lat, 4), axis=0)
    owners = owners[np.lexsort((owners[:, 0], owners[:, 1], owners[:, 2]))].astype(np.int32)
    nc, nf = len(ci), len(fi)
    outs = [np.zeros(nc), np.zeros(nf), np.zeros(nc), np.zeros(nc), np.zeros(nc)]
    diag, meas = (ctypes.c_double * 5)(), (ctypes.c_double * 3)()
    flux = None if face_flux is None else np.ascontiguousarray(face_flux, np.float64)
    code = lib().bk_project(ctypes.c_int(which), _d3((0, 0, 0)), ctypes.c_double(h), _p(owners),
                            ctypes.c_uint64(len(owners)), ctypes.c_double(dt), _p(np.ascontiguousarray(ci, np.int32)),
                            _p(np.ascontiguousarray(cv, np.float64)), ctypes.c_uint64(nc),
                            _p(np.ascontiguousarray(fi, np.int32)), _p(np.ascontiguousarray(fk, np.int32)),
                            _p(np.ascontiguousarray(fv, np.float64)), _p(flux), ctypes.c_uint64(nf),
                            ctypes.c_uint64(max_iterations), ctypes.c_double(tolerance_scale), *map(_p, outs), diag,
                            meas)
    keys = ("pressure", "corrected_u", "rhs", "residual", "defect")
    return code, dict(zip(keys, outs), diag=np.array(diag[:]), measure=np.array(meas[:]))


def release():
    if _lib is not None:
        _lib.bk_release()


def _owned_slot(blocks, axis, lat):
    """Owned slot of face (axis, lattice) in the sorted 4^3-block list, or -1."""
    b = np.floor_divide(lat, 4)
    key = {tuple(v): i for i, v in enumerate(blocks.tolist())}
    o = key.get((int(b[0]), int(b[1]), int(b[2])), -1)
    if o < 0:
        return -1
    loc = lat - 4 * b
    return o * 192 + axis * 64 + int((loc[2] * 4 + loc[1]) * 4 + loc[0])


class LinkScene:
    """A pool in a 12 x 32 x 12-cell tank frozen for the pressure-link
    assembly: cells x, z in [0, 12), y in [0, 6) (864 cells), a free surface
    in the top cell layer at a seeded height per column (so theta runs from
    0.01 to 0.95 and some air links are regularized to 0.05 h) with small
    seeded curvatures, tank walls at the lattice
    planes x, z = 0 and 12 and y = 0 (sealed, some with explicit wall fluxes
    or a wall velocity), every incident face in
    owned-slot order, centre samples on every cell within one of the pool,
    predictor densities on the cells x < 3 (so faces between them can carry
    certified internal interfaces), a few air cells with their own gas
    pressure, surface tension 0.072 N/m."""

    def __init__(self, seed: int = 5):
        rng = np.random.default_rng(seed)
        n, ny = 12, 6
        bz, by, bx = np.meshgrid(np.arange(-1, 4), np.arange(-1, 3), np.arange(-1, 4), indexing="ij")
        self.blocks = np.stack([bx.ravel(), by.ravel(), bz.ravel()], 1).astype(np.int32)
        cz, cy, cx = np.meshgrid(np.arange(n), np.arange(ny), np.arange(n), indexing="ij")
        ci = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], 1).astype(np.int32)  # (z,y,x) order
        self.cell_index = ci
        # the surface height of each column: the top cells' theta (surface - 5.5) runs from 0.01 to 0.95
        surf = 5.5 + rng.uniform(0.01, 0.95, (n + 2, n + 2))
        height = lambda x, z: surf[np.clip(x, -1, n) + 1, np.clip(z, -1, n) + 1]  # noqa: E731
        dist = (ci[:, 1] + 0.5 - height(ci[:, 0], ci[:, 2])) * H
        curv = np.where(ci[:, 1] == ny - 1, rng.uniform(-3.0, 3.0, len(ci)), 0.0)
        self.cell_values = np.stack([np.full(len(ci), H ** 3), dist, curv], 1)
        cells = {tuple(v) for v in ci.tolist()}
        # centre samples: every cell within one of a pool cell, (z,y,x) sorted
        near = set()
        for x, y, z in ci.tolist():
            for dz in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        near.add((x + dx, y + dy, z + dz))
        near = sorted(near, key=lambda c: (c[2], c[1], c[0]))
        self.center_index = np.array(near, np.int32)
        ce = self.center_index
        self.center_distance = (ce[:, 1] + 0.5 - height(ce[:, 0], ce[:, 2])) * H
        # incident faces in owned-slot order
        faces = set()
        for x, y, z in ci.tolist():
            for a in range(3):
                for side in (0, 1):
                    lat = [x, y, z]
                    lat[a] += side
                    faces.add((a, *lat))
        recs = []
        for a, x, y, z in faces:
            slot = _owned_slot(self.blocks, a, np.array([x, y, z]))
            assert slot >= 0
            recs.append((slot, a, x, y, z))
        recs.sort()
        self.face_slot = np.array([r[0] for r in recs], np.uint64)
        self.face_index = np.array([r[1:] for r in recs], np.int32)
        nf = len(recs)
        fv = np.zeros((nf, 4))
        fv[:, 3] = np.nan
        for f, (slot, a, x, y, z) in enumerate(recs):
            wall = [x, y, z][a] == 0 or (a != 1 and [x, y, z][a] == n)
            fv[f, 0] = 0.0 if wall else H * H
            fv[f, 1] = H * H - fv[f, 0]
            if wall and f % 7 == 0:
                fv[f, 3] = 1e-8 * ((f % 3) - 1)
            if wall and f % 11 == 0:
                fv[f, 2] = 0.01
        self.face_values = fv
        self.piston = np.zeros(nf, np.uint8)
        self.step_duration, self.density, self.sigma = DT, 1000.0, 0.072
        fields = np.zeros((len(ci), 4))
        fields[:, 0] = rng.uniform(-0.1, 0.1, len(ci))
        fields[:, 1] = np.inf
        fields[:, 2] = rng.uniform(0.0, 50.0, len(ci))
        fields[:, 3] = np.where(ci[:, 0] < 3, 1000.0 + rng.uniform(-5.0, 5.0, len(ci)), np.nan)
        fields[ci[:, 0] == 5, 1] = 2.2e9  # a compliant column
        self.fields = fields
        self.predicted = rng.uniform(-0.3, 0.3, nf)
        self.ambient = 101.0
        air = [c for c in near if c[1] >= ny and 0 <= c[0] < n and 0 <= c[2] < n][::13]
        self.air_index = np.array(air, np.int32).reshape(-1, 3)
        self.air_pressure = rng.uniform(90.0, 110.0, len(air))
        # interfaces on x-faces between two cells x < 3 (both with densities)
        ords = [f for f, (slot, a, x, y, z) in enumerate(recs) if a == 0 and 1 <= x <= 2 and (x - 1, y, z) in cells
                and y < ny - 1][::5]
        self.itf_ordinal = np.array(ords, np.uint64)
        self.itf_values = np.stack([rng.uniform(0.0, 1.0, len(ords)), np.full(len(ords), 0.05),
                                    rng.uniform(-2.0, 2.0, len(ords)), rng.uniform(-1.0, 1.0, len(ords))], 1)
        self.wetted = None


def links(which, s: LinkScene, **override):
    """The table's .links on the scene (fields overridable by keyword)."""
    a = dict(s.__dict__)
    a.update(override)
    nc, nf = len(a["cell_index"]), len(a["face_index"])
    cells_out = np.zeros((nc, 5))
    faces_out = np.zeros((nf, 8))
    lower = ctypes.c_uint64(0)
    c = lambda x, t: np.ascontiguousarray(x, t)  # noqa: E731
    wet = None if a["wetted"] is None else c(a["wetted"], np.float64)
    code = lib().bk_links(
        ctypes.c_int(which), _d3((0, 0, 0)), ctypes.c_double(H), _p(c(a["blocks"], np.int32)),
        ctypes.c_uint64(len(a["blocks"])), _p(c(a["center_index"], np.int32)), _p(c(a["center_distance"], np.float64)),
        ctypes.c_uint64(len(a["center_index"])), _p(c(a["cell_index"], np.int32)), _p(c(a["cell_values"], np.float64)),
        ctypes.c_uint64(nc), _p(c(a["face_index"], np.int32)), _p(c(a["face_slot"], np.uint64)),
        _p(c(a["face_values"], np.float64)), _p(c(a["piston"], np.uint8)), ctypes.c_uint64(nf),
        ctypes.c_double(a["step_duration"]), ctypes.c_double(a["density"]), ctypes.c_double(a["sigma"]),
        _p(c(a["fields"], np.float64)), _p(c(a["predicted"], np.float64)), ctypes.c_double(a["ambient"]), _p(wet),
        _p(c(a["air_index"], np.int32)), _p(c(a["air_pressure"], np.float64)), ctypes.c_uint64(len(a["air_index"])),
        _p(c(a["itf_ordinal"], np.uint64)), _p(c(a["itf_values"], np.float64)), ctypes.c_uint64(len(a["itf_ordinal"])),
        _p(cells_out), _p(faces_out), ctypes.byref(lower))
    return code, cells_out, faces_out, lower.value


class FreezeScene:
    """Candidate cells of a 12 x 9 x 12-cell region (x, z in [0, 12), y in
    [0, 9): 1296 candidates) holding a wobbly drop: the signed distance, in
    cells, is |p - (6, 4.5, 6)| - 3.7 - 0.25 sin(2x/3) cos(z/2), times h,
    sampled at every cell centre within one of the region and at every lattice
    corner of the candidates. The region's outer cells are air, so every face
    of a liquid cell opens onto a liquid or an air cell. Obstacles: none, a
    translating halfspace whose plane cuts the drop's low-x, low-z side, or a
    translating slab 2.4 h thick across it (thicker than a cell's diagonal, so
    no cell holds liquid on both of its sides); with the open tank the liquid
    is instead a pool filling a tank whose walls and floor cut the lattice
    cells. Active 4^3 blocks: x, z in [-1, 3], y in [-1, 2]."""

    def __init__(self, obstacle: str = "none", sigma: float = 0.072, exact_curvature: float = float("nan")):
        n, ny = 12, 9
        self.tank = (0.0,) * 6
        bz, by, bx = np.meshgrid(np.arange(-1, 4), np.arange(-1, 3), np.arange(-1, 4), indexing="ij")
        self.blocks = np.stack([bx.ravel(), by.ravel(), bz.ravel()], 1).astype(np.int32)

        def distance(p):
            r = np.sqrt((p[:, 0] - 6.0) ** 2 + (p[:, 1] - 4.5) ** 2 + (p[:, 2] - 6.0) ** 2)
            return (r - 3.7 - 0.25 * np.sin(p[:, 0] / 1.5) * np.cos(p[:, 2] / 2.0)) * H

        cz, cy, cx = np.meshgrid(np.arange(n), np.arange(ny), np.arange(n), indexing="ij")
        self.cell_index = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], 1).astype(np.int32)
        ez, ey, ex = np.meshgrid(np.arange(-1, n + 1), np.arange(-1, ny + 1), np.arange(-1, n + 1), indexing="ij")
        self.center_index = np.stack([ex.ravel(), ey.ravel(), ez.ravel()], 1).astype(np.int32)
        self.center_distance = distance(self.center_index + 0.5)
        kz, ky, kx = np.meshgrid(np.arange(n + 1), np.arange(ny + 1), np.arange(n + 1), indexing="ij")
        self.corner_index = np.stack([kx.ravel(), ky.ravel(), kz.ravel()], 1).astype(np.int32)
        self.corner_distance = distance(self.corner_index.astype(np.float64))
        self.kind, self.normal, self.coordinate, self.half_width = 0, (0.0, 0.0, 0.0), 0.0, 0.0
        self.velocity = (0.0, 0.0, 0.0)
        if obstacle == "halfspace":  # solid where n . x <= c
            self.kind, self.normal, self.coordinate = 1, (0.8, 0.0, 0.6), 5.3 * H
            self.velocity = (0.05, 0.0, -0.02)
        elif obstacle == "slab":
            self.kind, self.normal, self.coordinate, self.half_width = 2, (0.6, 0.0, 0.8), 8.1 * H, 1.2 * H
            self.velocity = (0.0, 0.0, 0.1)
        elif obstacle == "tank":
            # a pool filling an open tank whose walls and floor cut the lattice
            # cells (low x moves as a piston): distance (y - s(x, z)) h
            self.kind, self.tank = 3, (0.3 * H, 11.6 * H, 0.45 * H, 0.2 * H, 11.7 * H, 0.05)
            surface = lambda x, z: 4.4 + 0.7 * np.sin(x / 2.0) * np.cos(0.4 * z)  # noqa: E731
            c = self.center_index + 0.5
            self.center_distance = (c[:, 1] - surface(c[:, 0], c[:, 2])) * H
            k = self.corner_index.astype(np.float64)
            self.corner_distance = (k[:, 1] - surface(k[:, 0], k[:, 2])) * H
        self.step_duration, self.density, self.sigma = DT, 1000.0, sigma
        self.exact_curvature = exact_curvature


def freeze(which, s: FreezeScene, **override):
    """The table's .freeze on the scene: (code, cell indices, cell values
    (volume, centre distance, curvature), face indices (axis, x, y, z), face
    slots, face values (open, blocked, wall velocity, prescribed wall flux or
    NaN, piston flag), capillary bound)."""
    a = dict(s.__dict__)
    a.update(override)
    n = len(a["cell_index"])
    ci = np.zeros((n, 3), np.int32)
    cv = np.zeros((n, 3))
    fi = np.zeros((6 * n, 4), np.int32)
    fs = np.zeros(6 * n, np.uint64)
    fv = np.zeros((6 * n, 5))
    nc, nf, bound = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_double(0.0)
    c = lambda x, t: np.ascontiguousarray(x, t)  # noqa: E731
    code = lib().bk_freeze(
        ctypes.c_int(which), _d3((0, 0, 0)), ctypes.c_double(H), _p(c(a["blocks"], np.int32)),
        ctypes.c_uint64(len(a["blocks"])), _p(c(a["cell_index"], np.int32)), ctypes.c_uint64(n),
        _p(c(a["center_index"], np.int32)), _p(c(a["center_distance"], np.float64)),
        ctypes.c_uint64(len(a["center_index"])), _p(c(a["corner_index"], np.int32)),
        _p(c(a["corner_distance"], np.float64)), ctypes.c_uint64(len(a["corner_index"])), ctypes.c_int(a["kind"]),
        _d3(a["normal"]), ctypes.c_double(a["coordinate"]), ctypes.c_double(a["half_width"]), _d3(a["velocity"]),
        (ctypes.c_double * 6)(*[float(v) for v in a["tank"]]), ctypes.c_double(a["step_duration"]), ctypes.c_double(a["density"]), ctypes.c_double(a["sigma"]),
        ctypes.c_double(a["exact_curvature"]), _p(ci), _p(cv), ctypes.byref(nc), _p(fi), _p(fs), _p(fv),
        ctypes.byref(nf), ctypes.byref(bound))
    k, m = nc.value, nf.value
    return code, ci[:k], cv[:k], fi[:m], fs[:m], fv[:m], bound.value


class PistonScene:
    """The open-tank pool frozen by the CPU table (FreezeScene("tank")) and a
    liquid field over the low-x piston: a horizontal plane at 4.4 cells, an
    analytic sphere of radius 3 cells centred 1.5 cells inside the piston, or
    a union of 0.6-cell particle spheres on a 0.5-cell lattice in the 1.7
    cells next to the piston (4 x 7 x 23 = 644 particles)."""

    def __init__(self, field: str = "plane"):
        fs = FreezeScene("tank")
        code, ci, cv, fi, fslot, fv, _ = freeze(CPU, fs)
        assert code == 0
        self.blocks, self.tank = fs.blocks, fs.tank
        self.cell_index, self.cell_values = ci, cv
        self.face_index, self.face_slot, self.face_values = fi, fslot, fv
        self.kind, self.center, self.radius, self.plane_y = 2, (0.0, 0.0, 0.0), 1.0, 4.4 * H
        self.positions = np.zeros((0, 3))
        x0 = fs.tank[0]
        if field == "sphere":
            self.kind, self.center, self.radius = 0, (x0 + 1.5 * H, 3.0 * H, 6.0 * H), 3.0 * H
        elif field == "union":
            self.kind, self.radius = 1, 0.6 * H
            gx, gy, gz = np.meshgrid(x0 + H * (0.2 + 0.5 * np.arange(4)), H * (0.8 + 0.5 * np.arange(7)),
                                     H * (0.5 + 0.5 * np.arange(23)), indexing="ij")
            self.positions = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1)
        elif field == "drop":
            self.kind = 3


def wetted_piston(which, s: PistonScene, **override):
    """The table's .wetted_piston: (code, patches (n, 9), face fluxes (NaN
    for none), whole area and flux enclosures (4,), attached count)."""
    a = dict(s.__dict__)
    a.update(override)
    nf = len(a["face_index"])
    patches = np.zeros((24576, 9))
    fluxes = np.zeros(max(nf, 1))
    whole = (ctypes.c_double * 4)()
    npatch, attached = ctypes.c_uint64(0), ctypes.c_uint64(0)
    c = lambda x, t: np.ascontiguousarray(x, t)  # noqa: E731
    pos = c(a["positions"], np.float64).reshape(-1, 3)
    code = lib().bk_wetted_piston(
        ctypes.c_int(which), _d3((0, 0, 0)), ctypes.c_double(H), _p(c(a["blocks"], np.int32)),
        ctypes.c_uint64(len(a["blocks"])), _p(c(a["cell_index"], np.int32)), _p(c(a["cell_values"], np.float64)),
        ctypes.c_uint64(len(a["cell_index"])), _p(c(a["face_index"], np.int32)), _p(c(a["face_slot"], np.uint64)),
        _p(c(a["face_values"], np.float64)), ctypes.c_uint64(nf), ctypes.c_int(a["kind"]), _d3(a["center"]),
        ctypes.c_double(a["radius"]), ctypes.c_double(a["plane_y"]), _p(pos), ctypes.c_uint64(len(pos)),
        (ctypes.c_double * 6)(*[float(v) for v in a["tank"]]), _p(patches), ctypes.byref(npatch), _p(fluxes), whole,
        ctypes.byref(attached))
    return code, patches[:npatch.value], fluxes[:nf], np.array(whole[:]), attached.value
