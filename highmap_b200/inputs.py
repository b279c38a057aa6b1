"""Seeded synthetic heightmaps for the solvers' tests and benchmarks.

Input preparation only (not part of the erosion path).  The structure
follows HighMap's ``noise_fbm`` (HighMap/src/primitives/coherent_noise/
noise.cpp:41-75, HighMap/src/functions/fbm_functions.cpp:17-53,396-406):

* coordinates x_i = i / nx, y_j = j / ny on the unit square
  (``grid_xy_vector`` with endpoint=false, operator/fill_array.cpp:13-23);
* octave k samples the base noise at (kw * lacunarity^k) * (x, y) with
  seed + k;
* amplitude starts at amp0 = 1 / sum_k persistence^k and after each octave
  is multiplied by ((1 - weight) + weight * min(value + 1, 2) / 2) and by
  persistence;
* ``remap`` to [0, 1] (range/range.cpp:342-361).

The base noise is 2-D Perlin gradient noise written from Perlin's published
"improved noise" method (quintic fade 6t^5 - 15t^4 + 10t^3, a seeded
permutation of 256 lattice hashes, 8 unit gradient directions).  It is not
FastNoiseLite's field; tests and benchmarks upload the same bytes to every
path, so only the statistics (an fBm terrain in [0, 1]) matter.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

_GRAD = np.array(
    [[1.0, 0.0], [-1.0, 0.0], [0.0, 1.0], [0.0, -1.0],
     [0.70710678, 0.70710678], [-0.70710678, 0.70710678],
     [0.70710678, -0.70710678], [-0.70710678, -0.70710678]],
    dtype=np.float32,
)


def _fade(t):
    return t * t * t * (t * (t * 6.0 - 15.0) + 10.0)


def _tables(seed: int):
    rng = np.random.default_rng(int(seed) & 0xFFFFFFFF)
    perm = rng.permutation(256).astype(np.int32)
    perm = np.concatenate([perm, perm, perm])
    gsel = rng.integers(0, 8, size=256, dtype=np.int32)
    g = _GRAD[gsel[perm[:512]]]  # gradient of hash value k, for k < 512
    return perm, np.ascontiguousarray(g[:, 0]), np.ascontiguousarray(g[:, 1])


def perlin2(x: np.ndarray, y: np.ndarray, seed: int) -> np.ndarray:
    """Perlin gradient noise on the outer grid x (nx,) by y (ny,); returns
    an (ny, nx) float32 field in about [-1, 1]."""
    perm, gx, gy = _tables(seed)
    xf = np.floor(x)
    yf = np.floor(y)
    xi = (xf.astype(np.int64) & 255).astype(np.int32)
    yi = (yf.astype(np.int64) & 255).astype(np.int32)
    tx = (x - xf).astype(np.float32)
    ty = (y - yf).astype(np.float32)
    u = _fade(tx)[None, :]
    v = _fade(ty)[:, None]

    def corner(dx, dy):
        h = perm[xi + dx][None, :] + (yi + dy)[:, None]  # < 512
        return gx[h] * (tx[None, :] - dx) + gy[h] * (ty[:, None] - dy)

    n00 = corner(0, 0)
    n10 = corner(1, 0)
    nx0 = n00 + u * (n10 - n00)
    n01 = corner(0, 1)
    n11 = corner(1, 1)
    nx1 = n01 + u * (n11 - n01)
    return (np.float32(1.41421356) * (nx0 + v * (nx1 - nx0))).astype(np.float32)


def remap(a: np.ndarray, vmin: float = 0.0, vmax: float = 1.0) -> np.ndarray:
    lo = float(a.min())
    hi = float(a.max())
    if hi == lo:
        return np.full_like(a, vmin)
    return ((a - lo) / (hi - lo) * (vmax - vmin) + vmin).astype(np.float32)


def _fbm_rows(nx, ny, j0, j1, seed, kw, octaves, weight, persistence, lacunarity):
    x = np.arange(nx, dtype=np.float64) / nx
    y = np.arange(j0, j1, dtype=np.float64) / ny
    amp0 = 1.0 / sum(persistence ** k for k in range(octaves))
    total = np.zeros((j1 - j0, nx), dtype=np.float32)
    amp = np.full((j1 - j0, nx), amp0, dtype=np.float32)
    freq = float(kw)
    for k in range(octaves):
        value = perlin2(freq * x, freq * y, seed + k)
        total += value * amp
        amp *= np.float32(1.0 - weight) + np.float32(weight) * np.minimum(value + np.float32(1.0),
                                                                         np.float32(2.0)) * np.float32(0.5)
        amp *= np.float32(persistence)
        freq *= lacunarity
    return total


def fbm(nx: int, ny: int, seed: int, kw: float = 4.0, octaves: int = 8,
        weight: float = 0.7, persistence: float = 0.5, lacunarity: float = 2.0,
        remap01: bool = True) -> np.ndarray:
    """fBm heightmap of shape (ny, nx), float32, remapped to [0, 1].  Rows
    are computed in bands on a thread pool; the result does not depend on
    the number of threads."""
    band = max(16, (1 << 20) // max(nx, 1))
    starts = list(range(0, ny, band))
    args = (seed, kw, octaves, weight, persistence, lacunarity)
    if len(starts) == 1:
        total = _fbm_rows(nx, ny, 0, ny, *args)
    else:
        with ThreadPoolExecutor(max_workers=min(len(starts), os.cpu_count() or 1)) as ex:
            parts = list(ex.map(lambda j0: _fbm_rows(nx, ny, j0, min(ny, j0 + band), *args), starts))
        total = np.concatenate(parts, axis=0)
    return remap(total) if remap01 else total
