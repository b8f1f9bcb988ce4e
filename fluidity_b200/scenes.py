"""Seeded synthetic liquid scenes on the unit cube (host-side initial state).

Every scene is a box of n^3 MAC cells (h = 1/n, origin 0) with one-cell solid
walls on all six faces. Fluid cells are the non-wall cells whose centre lies in
the scene's liquid region; each receives 8 particles, one per 2x2x2 sub-cell
stratum, uniformly jittered inside its stratum. The jitter is a counter-based
SplitMix64 stream keyed by (seed, cell linear index, stratum, axis), so the same
scene is generated bit-for-bit by every consumer (GPU path, oracle, bench).

Scenes (sizes as in the workloads this library is measured on):
* ``dam_break(n)``: fluid in [0, 0.5]^3, at rest.
* ``splash(n)``: pool y <= 0.2 over the whole floor plus two spheres of radius
  0.15 at (0.35, 0.6, 0.5) and (0.65, 0.6, 0.5) moving at +2 and -2 m/s in x.
* ``column_drop(n)``: column [0.1,0.3]x[0.1,0.8]x[0.1,0.3] over a pool y <= 0.15.
"""

from __future__ import annotations

import numpy as np

DENSITY = 1000.0
DT = 1.0 / 240.0
GRAVITY = (0.0, -9.81, 0.0)

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _uniform(seed: int, key: np.ndarray) -> np.ndarray:
    """Uniform [0,1) doubles with 53 random bits from (seed, key)."""
    with np.errstate(over="ignore"):
        x = _splitmix64(key.astype(np.uint64) * np.uint64(0x2545F4914F6CDD1D) + np.uint64(seed))
    return (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def seed_particles(n: int, cells: np.ndarray, seed: int = 0, velocity=None):
    """Particles for the given fluid cells ((k, j, i) triples, shape (m, 3)).

    Returns an FP32 SoA array (15, 8m): x, y, z, vx, vy, vz and nine zero
    affine entries, plus the particle mass rho h^3 / 8.
    """
    h = 1.0 / n
    cells = np.asarray(cells, dtype=np.int64)
    m = len(cells)
    k, j, i = cells[:, 0], cells[:, 1], cells[:, 2]
    lin = (k * n + j) * n + i
    strata = np.arange(8, dtype=np.int64)
    sx, sy, sz = strata & 1, (strata >> 1) & 1, strata >> 2
    key = (lin[:, None] * 8 + strata[None, :]) * 3
    ux = _uniform(seed, key)
    uy = _uniform(seed, key + 1)
    uz = _uniform(seed, key + 2)
    x = (i[:, None] + (sx[None, :] + ux) * 0.5) * h
    y = (j[:, None] + (sy[None, :] + uy) * 0.5) * h
    z = (k[:, None] + (sz[None, :] + uz) * 0.5) * h
    soa = np.zeros((15, 8 * m), np.float32)
    # Rounded to FP32 inside the particle's own cell: a jitter just below the
    # cell's upper edge would otherwise round onto the edge, into the next cell.
    for d, (pos, cell) in enumerate(((x, i), (y, j), (z, k))):
        edge = np.nextafter(((cell[:, None] + 1) * h).astype(np.float32), np.float32(0.0))
        soa[d] = np.minimum(pos.astype(np.float32), edge).ravel()
    if velocity is not None:
        vel = np.asarray(velocity, np.float64).reshape(-1, 3)
        if len(vel) == 1:
            vel = np.repeat(vel, m, axis=0)
        for d in range(3):
            soa[3 + d] = np.repeat(vel[:, d], 8)
    mass = DENSITY * h ** 3 / 8.0
    return soa, mass


def seed_scene(n: int, inside, velocity_of=None, seed: int = 0, slab: int = 32):
    """Particles of every interior cell whose centre satisfies inside(X, Y, Z),
    generated z-slab by z-slab into one preallocated FP32 SoA array: the same
    particles in the same order as seed_particles over all the cells at once,
    with host memory bounded by one slab (a 512^3 scene holds ~190M particles).
    velocity_of(X, Y, Z) -> (m, 3) gives the velocity of the selected cells."""
    h = 1.0 / n
    idx = np.arange(1, n - 1)
    c = (idx + 0.5) / n
    J2, I2 = np.meshgrid(idx, idx, indexing="ij")
    Y2, X2 = np.meshgrid(c, c, indexing="ij")
    slabs = [idx[k0:k0 + slab] for k0 in range(0, len(idx), slab)]

    def cells_of(ks):
        Z = np.repeat(((ks + 0.5) / n)[:, None, None], len(idx), 1).repeat(len(idx), 2)
        X = np.broadcast_to(X2, Z.shape)
        Y = np.broadcast_to(Y2, Z.shape)
        mask = inside(X, Y, Z)
        K = np.broadcast_to(ks[:, None, None], Z.shape)
        J = np.broadcast_to(J2, Z.shape)
        I = np.broadcast_to(I2, Z.shape)
        return np.stack([K[mask], J[mask], I[mask]], axis=1), (X[mask], Y[mask], Z[mask])

    total = sum(int(inside(np.broadcast_to(X2, (len(ks), *X2.shape)), np.broadcast_to(Y2, (len(ks), *X2.shape)),
                           np.broadcast_to(((ks + 0.5) / n)[:, None, None], (len(ks), *X2.shape))).sum())
                for ks in slabs)
    out = np.zeros((15, 8 * total), np.float32)
    at = 0
    for ks in slabs:
        cells, xyz = cells_of(ks)
        if len(cells) == 0:
            continue
        vel = velocity_of(*xyz) if velocity_of is not None else None
        part, _ = seed_particles(n, cells, seed, vel)
        out[:, at:at + part.shape[1]] = part
        at += part.shape[1]
    return out, DENSITY * h ** 3 / 8.0


def _interior_centres(n: int):
    idx = np.arange(1, n - 1)
    c = (idx + 0.5) / n
    return idx, c


def _cells_where(n: int, inside):
    idx, c = _interior_centres(n)
    K, J, I = np.meshgrid(idx, idx, idx, indexing="ij")
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    mask = inside(X, Y, Z)
    return np.stack([K[mask], J[mask], I[mask]], axis=1), mask, (X, Y, Z)


def dam_break(n: int, seed: int = 0):
    cells, _, _ = _cells_where(n, lambda X, Y, Z: (X <= 0.5) & (Y <= 0.5) & (Z <= 0.5))
    return seed_particles(n, cells, seed)


def splash(n: int, seed: int = 0):
    c1, c2, r = (0.35, 0.6, 0.5), (0.65, 0.6, 0.5), 0.15

    def in_sphere(X, Y, Z, c):
        return (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r

    cells, mask, (X, Y, Z) = _cells_where(
        n, lambda X, Y, Z: (Y <= 0.2) | in_sphere(X, Y, Z, c1) | in_sphere(X, Y, Z, c2))
    Xs, Ys, Zs = X[mask], Y[mask], Z[mask]
    vel = np.zeros((len(cells), 3))
    pool = Ys <= 0.2
    s1 = in_sphere(Xs, Ys, Zs, c1) & ~pool
    s2 = in_sphere(Xs, Ys, Zs, c2) & ~pool & ~s1
    vel[s1, 0] = 2.0
    vel[s2, 0] = -2.0
    return seed_particles(n, cells, seed, vel)


def column_drop(n: int, seed: int = 0):
    return seed_scene(
        n, lambda X, Y, Z: (Y <= 0.15) | ((X >= 0.1) & (X <= 0.3) & (Y >= 0.1) & (Y <= 0.8) & (Z >= 0.1) & (Z <= 0.3)),
        seed=seed)


SCENES = {"dam_break": dam_break, "splash": splash, "column_drop": column_drop}
