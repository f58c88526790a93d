"""Seeded synthetic point sets and vectors for the H-matrix workloads.

One portable generator (SplitMix64, Steele/Lea/Flood 2014) so that Python and
C++ harnesses produce identical inputs:

* uniform double = (u >> 11) * 2^-53,
* points are drawn point-major (x0, y0[, z0], x1, ...) and returned SoA
  (``coords[d, i]``),
* right-hand sides are U[-1, 1] drawn from seed + 1000.

The reference (kadircs/hmglib) draws its points with cuRAND or GSL Halton
(``src/hmglib_test.cu:68-75``, ``src/paper_benchmark.cu:26-57``); those streams
are not reproducible off-GPU, so every harness here uses this generator instead.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, start: int = 0) -> np.ndarray:
    """Outputs ``start .. start+count-1`` of the SplitMix64 stream for ``seed``."""
    with np.errstate(over="ignore"):
        idx = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + idx * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, count: int, start: int = 0) -> np.ndarray:
    u = splitmix64(seed, count, start)
    return (u >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform_points(n: int, dim: int, seed: int) -> np.ndarray:
    """``n`` points i.i.d. uniform in [0,1]^dim, SoA ``(dim, n)`` float64."""
    u = uniform01(seed, n * dim)
    return np.ascontiguousarray(u.reshape(n, dim).T)


def gmm_points(n: int, dim: int, seed: int, components: int = 16,
               std_lo: float = 0.02, std_hi: float = 0.1) -> np.ndarray:
    """Gaussian mixture: means U[0,1]^dim, per-component std U[std_lo, std_hi],
    equal weights, Box-Muller normals; one stream for everything."""
    head = uniform01(seed, components * (dim + 1))
    means = head[: components * dim].reshape(components, dim)
    stds = std_lo + (std_hi - std_lo) * head[components * dim:]
    body = uniform01(seed, n * (1 + 2 * dim), start=components * (dim + 1))
    comp = np.minimum((body[:n] * components).astype(np.int64), components - 1)
    u1 = body[n:n + n * dim].reshape(n, dim)
    u2 = body[n + n * dim:].reshape(n, dim)
    z = np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)
    pts = means[comp] + stds[comp, None] * z
    return np.ascontiguousarray(pts.T)


def rhs_vector(n: int, seed: int, nrhs: int = 1) -> np.ndarray:
    """U[-1,1] right-hand side(s) from ``seed + 1000``; shape (n,) or (nrhs, n)."""
    u = uniform01(seed + 1000, n * nrhs) * 2.0 - 1.0
    return u if nrhs == 1 else u.reshape(nrhs, n)


def group_sets(count: int = 512, seed: int = 3, log2_lo: float = 10.0, log2_hi: float = 16.0,
               l2_lo: float = 0.01, l2_hi: float = 0.2):
    """Many independent point sets: sizes round(2^U[log2_lo, log2_hi]), dimension
    alternating 2, 3, points uniform in the unit box, Gaussian length^2 U[l2_lo, l2_hi].
    Returns a list of (points (dim, n), squared length scale)."""
    head = uniform01(seed, 2 * count)
    out = []
    for i in range(count):
        n = int(round(2.0 ** (log2_lo + (log2_hi - log2_lo) * head[2 * i])))
        l2 = l2_lo + (l2_hi - l2_lo) * head[2 * i + 1]
        dim = 2 if i % 2 == 0 else 3
        out.append((uniform_points(n, dim, (seed << 20) + i + 1), float(l2)))
    return out
