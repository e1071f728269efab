"""Seeded synthetic cloth workloads (triangle soups in the reference's (F, 3, 3) layout).

The reference evaluates on no public dataset; these generators build the five measured
configurations from their stated shapes and value distributions:

* ``static_fold``   — 64x64 crumpled cloth, half folded through itself (7,938 triangles, fp32)
* ``cloth_sphere``  — 128x128 cloth falling 0.03 onto an icosphere (level 5) 0.02 below it
                      (52,738 triangles, fp64)
* ``impulse_fold``  — 256x256 jittered cloth with a folded half (130,050 triangles, fp64)
* ``batched``       — many cloth+sphere meshes of log-uniform size
* ``served``        — a Poisson request stream of impulse solves

All randomness comes from ``numpy.random.Generator(PCG64(seed))``.
"""
from __future__ import annotations

import functools
import math

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def grid(nx: int, ny: int, x0=0.0, x1=1.0, y0=0.0, y1=1.0):
    """Regular nx-by-ny vertex grid, two triangles per cell with a consistent diagonal."""
    xs = np.linspace(x0, x1, nx)
    ys = np.linspace(y0, y1, ny)
    X, Y = np.meshgrid(xs, ys, indexing="xy")          # row-major over y then x
    verts = np.stack([X.ravel(), Y.ravel(), np.zeros(nx * ny)], axis=1)
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="xy")
    v00 = (j * nx + i).ravel()
    v10 = v00 + 1
    v01 = v00 + nx
    v11 = v01 + 1
    f0 = np.stack([v00, v10, v11], axis=1)
    f1 = np.stack([v00, v11, v01], axis=1)
    faces = np.stack([f0, f1], axis=1).reshape(-1, 3)
    return verts, faces.astype(np.int64)


@functools.lru_cache(maxsize=8)
def _icosphere_unit(level: int):
    return icosphere_build(level)


def icosphere(level: int, radius: float = 1.0):
    """Subdivided icosahedron projected onto a sphere (20 * 4^level faces)."""
    v, f = _icosphere_unit(level)
    return v * radius, f.copy()


def icosphere_build(level: int):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int64)


def soup(verts, faces):
    return np.ascontiguousarray(verts[faces])


def sinusoid_height(g, x, y, n=8, amp=0.05):
    f = g.uniform(1.0, 6.0, n)
    th = g.uniform(0.0, 2 * math.pi, n)
    ph = g.uniform(0.0, 2 * math.pi, n)
    z = np.zeros_like(x)
    for k in range(n):
        z += amp * np.sin(2 * math.pi * f[k] * (x * math.cos(th[k]) + y * math.sin(th[k])) + ph[k])
    return z


def static_fold(seed: int = 0, n: int = 64, dtype=np.float32):
    """Crumpled cloth folded across x = 0.5 so the halves intersect: (1, F, 3, 3)."""
    g = rng(seed)
    verts, faces = grid(n, n)
    x, y = verts[:, 0], verts[:, 1]
    verts[:, 2] = sinusoid_height(g, x, y)
    m = x > 0.5
    verts[m, 0] = 1.0 - x[m]
    return soup(verts, faces)[None].astype(dtype)


def cloth_sphere(seed: int = 0, nx: int = 128, ny: int = 128, level: int = 5, drop=0.03, sigma=0.005,
                 gap=0.02, dtype=np.float64):
    """Cloth 'gap' above the pole of a unit icosphere moving 'drop' down: (x0, x1) each (1, F, 3, 3).

    The cloth spans [-0.5, 0.5]^2 scaled by the grid aspect; the sphere is static.
    """
    g = rng(seed)
    sx = 1.0
    sy = (ny - 1) / (nx - 1) if nx != ny else 1.0
    cv, cf = grid(nx, ny, -0.5 * sx, 0.5 * sx, -0.5 * sy, 0.5 * sy)
    cv[:, 2] = 1.0 + gap
    cv1 = cv.copy()
    cv1[:, 2] -= drop
    cv1 += g.normal(0.0, sigma, cv.shape)
    sv, sf = icosphere(level)
    x0 = np.concatenate([soup(cv, cf), soup(sv, sf)], axis=0)
    x1 = np.concatenate([soup(cv1, cf), soup(sv, sf)], axis=0)
    return x0[None].astype(dtype), x1[None].astype(dtype)


def impulse_fold(seed: int = 0, n: int = 256, dtype=np.float64):
    """Jittered cloth with the x > 0.5 half folded 0.005 above the rest, moving down 0.01.

    Returns (x0, x1, masses) with masses (1, F, 3) = 1.
    """
    g = rng(seed)
    verts, faces = grid(n, n)
    verts[:, 2] = g.normal(0.0, 0.01, verts.shape[0])
    m = verts[:, 0] > 0.5
    verts[m, 0] = 1.0 - verts[m, 0]
    verts[m, 2] += 0.005
    v1 = verts.copy()
    v1[:, 2] -= 0.01
    v1 += g.normal(0.0, 0.002, verts.shape)
    x0 = soup(verts, faces)[None].astype(dtype)
    x1 = soup(v1, faces)[None].astype(dtype)
    masses = np.ones(x0.shape[:3], dtype=dtype)
    return x0, x1, masses


def jittered_fold(seed: int, nx: int = 8, ny: int = 8, noise: float = 0.02, drop: float = 0.05,
                  dtype=np.float64, fold: bool = True):
    """Small jittered grid folded over itself with a random displacement: (x0, x1, masses).

    Each soup is (F, 3, 3) built from an indexed mesh, so neighbouring triangles share
    vertices exactly (the reference detects shared vertices by coordinate equality).
    masses (F, 3) are per-corner, uniform in [0.5, 2].
    """
    g = rng(seed)
    v, f = grid(nx, ny)
    v[:, 2] = g.normal(0, noise, v.shape[0])
    if fold:
        m = v[:, 0] > 0.5
        v[m, 0] = 1.0 - v[m, 0]
        v[m, 2] += 0.01
    v1 = v.copy()
    v1[:, 2] -= drop
    v1 += g.normal(0, noise, v.shape)
    x0 = soup(v, f).astype(dtype)
    x1 = soup(v1, f).astype(dtype)
    masses = g.uniform(0.5, 2.0, (x0.shape[0], 3)).astype(dtype)
    return x0, x1, masses


def grid_for_count(g, tris: int):
    """nx, ny with aspect U[0.5, 2] and 2 (nx-1)(ny-1) close to 'tris'."""
    aspect = g.uniform(0.5, 2.0)
    cells = tris / 2.0
    nxm1 = max(1, int(round(math.sqrt(cells * aspect))))
    nym1 = max(1, int(round(cells / nxm1)))
    return nxm1 + 1, nym1 + 1


def batched(num_meshes: int = 64, lo: float = 1e3, hi: float = 1e5, seed0: int = 1000, level: int = 5,
            dtype=np.float64):
    """List of (x0, x1) cloth+sphere meshes, each (F_i, 3, 3); the i-th uses seed seed0 + i."""
    out = []
    for i in range(num_meshes):
        g = rng(seed0 + i)
        tris = math.exp(g.uniform(math.log(lo), math.log(hi)))
        nx, ny = grid_for_count(g, tris)
        x0, x1 = cloth_sphere(seed=seed0 + i, nx=nx, ny=ny, level=level, dtype=dtype)
        out.append((x0[0], x1[0]))
    return out


# A fold whose layers start apart (heights N(0, 0.002^2), the upper half 0.02 above) and
# whose upper half moves 0.03 down through the lower one: every triangle of the fold collides
# in the first check, and the impulse loop separates them in a few iterations.
SEPARATED_FOLD = dict(noise=0.002, gap=0.02, drop=0.0, drop_noise=0.002, fold_drop=0.03)


def impulse_fold_mesh(seed: int = 0, nx: int = 256, ny: int = 256, dtype=np.float64, noise: float = 0.01,
                      gap: float = 0.005, drop: float = 0.01, drop_noise: float = 0.002, fold_drop: float = 0.0):
    """Indexed form of the impulse workload (jittered cloth with heights N(0, noise^2), the
    x > 0.5 half folded gap above the rest, everything moving drop down (the folded half
    fold_drop more) with N(0, drop_noise^2) noise; by default a fold whose layers already
    interpenetrate) on an nx-by-ny grid scaled to the grid's aspect: verts0 (V, 3), verts1
    (V, 3), vel (V, 3) = verts1 - verts0, faces (F, 3) int32, per-corner unit masses (F, 3)."""
    g = rng(seed)
    sy = (ny - 1) / (nx - 1)
    verts, faces = grid(nx, ny, 0.0, 1.0, 0.0, sy)
    verts[:, 2] = g.normal(0.0, noise, verts.shape[0])
    m = verts[:, 0] > 0.5
    verts[m, 0] = 1.0 - verts[m, 0]
    verts[m, 2] += gap
    v1 = verts.copy()
    v1[:, 2] -= drop
    v1[m, 2] -= fold_drop
    v1 += g.normal(0.0, drop_noise, verts.shape)
    masses = np.ones((faces.shape[0], 3), dtype=dtype)
    return (verts.astype(dtype), v1.astype(dtype), (v1 - verts).astype(dtype), faces.astype(np.int32), masses)


def served_stream(num_requests: int = 256, rate: float = 2000.0, lo: float = 2e3, hi: float = 2e5,
                  seed: int = 0, seed0: int = 1000, dtype=np.float64):
    """Poisson request stream: (arrival seconds, request seed, nx, ny) per request.

    Inter-arrival times are exponential with the given rate (seed `seed`); request i has
    log-uniform triangle count in [lo, hi] and builds its mesh with impulse_fold_mesh(seed0 + i).
    """
    g = rng(seed)
    t = np.cumsum(g.exponential(1.0 / rate, num_requests))
    out = []
    for i in range(num_requests):
        gi = rng(seed0 + i)
        tris = math.exp(gi.uniform(math.log(lo), math.log(hi)))
        nx, ny = grid_for_count(gi, tris)
        out.append((float(t[i]), seed0 + i, nx, ny))
    return out
