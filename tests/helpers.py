"""Shared helpers of the parity tests: one workload description, built both by the
engine (through the C ABI) and by the CPU oracle."""
from __future__ import annotations

import numpy as np

from hmglib_b200 import synth


def make_points(gen, n, dim, seed, scale=1.0):
    if gen == "uniform":
        p = synth.uniform_points(n, dim, seed)
    elif gen == "gmm":
        p = synth.gmm_points(n, dim, seed)
    elif gen == "line":
        # all points share every coordinate but the first (max == min in those dimensions)
        p = np.full((dim, n), 0.5)
        p[0] = synth.uniform01(seed, n)
    elif gen == "lattice":
        nx = int(round(n ** (1.0 / dim)))
        g = np.stack(np.meshgrid(*[np.arange(nx, dtype=np.float64)] * dim, indexing="ij"), 0)
        p = g.reshape(dim, -1)
        p = np.repeat(p, max(1, n // p.shape[1]), axis=1)[:, :n]
    else:
        raise ValueError(gen)
    return np.ascontiguousarray(p * scale)


def bits_for(dim):
    return 32 if dim == 2 else 20


def engine(hmg, p1, p2, eta, c_leaf, rule=0, max_level=50):
    dim = p1.shape[0]
    H = hmg.HMatrix(p1.shape[1], p2.shape[1], dim)
    H.set_points(0, p1)
    H.set_points(1, p2)
    H.setup(eta, c_leaf, max_level=max_level, rule=rule)
    return H


def oracle_setup(O, p1, p2, eta, c_leaf, rule=0, max_level=50):
    dim = p1.shape[0]
    s1, o1, z1 = O.order_points(p1, bits_for(dim))
    s2, o2, z2 = O.order_points(p2, bits_for(dim))
    blocks = O.tree(z1, s1, z2, s2, eta, c_leaf, max_level=max_level, rule=rule)
    return dict(codes1=s1, order1=o1, z1=z1, codes2=s2, order2=o2, z2=z2, blocks=blocks)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
