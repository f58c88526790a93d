"""ctypes front end of the CPU oracle (oracle/hmg_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU baseline.  The product path (hmglib_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libhmg_oracle.so")
_lib = None

KERNEL_GAUSSIAN_REF = 1
KERNEL_MATERN_REF = 2
KERNEL_GAUSSIAN = 3
KERNEL_MATERN32 = 4
WT_ACA = 1
WT_DENSE = 2

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    L.orc_minmax.argtypes = [_dp, C.c_int, C.c_int, _dp, _dp]
    L.orc_morton.argtypes = [_dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _u64p]
    L.orc_sort.argtypes = [_u64p, C.c_int, _u64p, _i64p]
    L.orc_reorder.argtypes = [_dp, C.c_int, C.c_int, _i64p, _dp]
    L.orc_tree.restype = C.c_void_p
    L.orc_tree.argtypes = [_dp, _u64p, C.c_int, _dp, _u64p, C.c_int, C.c_int, C.c_double,
                           C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    L.orc_blocks_count.argtypes = [C.c_void_p]
    L.orc_blocks_levels.argtypes = [C.c_void_p]
    L.orc_blocks_get.argtypes = [C.c_void_p, _ip, _ip, _ip, _ip, _ip, _ip, _ip]
    L.orc_blocks_free.argtypes = [C.c_void_p]
    L.orc_entry.restype = C.c_double
    L.orc_entry.argtypes = [C.c_int, C.c_double, C.c_double, _dp, C.c_int, _dp, C.c_int,
                            C.c_int, C.c_int, C.c_int]
    aca_common = [C.c_int, C.c_double, C.c_double, _dp, C.c_int, _dp, C.c_int, C.c_int,
                  C.c_int, _ip, _ip, _ip, _ip, C.c_int]
    L.orc_aca_fixed.argtypes = aca_common + [_i64p, _i64p, _dp, _dp, _ip]
    L.orc_aca_adaptive.argtypes = aca_common + [C.c_double, _i64p, _i64p, _dp, _dp, _ip]
    L.orc_hmatvec.argtypes = [C.c_int, C.c_double, C.c_double, _dp, C.c_int, _dp, C.c_int,
                              C.c_int, C.c_int, _ip, _ip, _ip, _ip, _ip, _i64p, _i64p, _dp,
                              _dp, _ip, _dp, _dp]
    L.orc_direct.argtypes = [C.c_int, C.c_double, C.c_double, _dp, C.c_int, _dp, C.c_int,
                             C.c_int, _dp, C.c_void_p, C.c_int, _dp, C.c_int]
    L.orc_gaussian_rhs.argtypes = [_dp, C.c_int, C.c_int, _dp]
    _lib = L
    return L


def kernel_param(kind: int, value: float) -> float:
    """Host-side parameter as the engine passes it: 1/l^2 (Gaussian), sqrt(3)/rho (Matern-3/2)."""
    if kind == KERNEL_GAUSSIAN:
        return 1.0 / value
    if kind == KERNEL_MATERN32:
        return float(np.sqrt(3.0)) / value
    return 0.0


def minmax(coords):
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    dim, n = coords.shape
    mn = np.empty(dim); mx = np.empty(dim)
    lib().orc_minmax(coords, n, dim, mn, mx)
    return mn, mx


def morton(coords, bits):
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    dim, n = coords.shape
    mn, mx = minmax(coords)
    codes = np.empty(n, dtype=np.uint64)
    lib().orc_morton(coords, n, dim, bits, mn, mx, codes)
    return codes


def sort_codes(codes):
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    n = codes.shape[0]
    s = np.empty(n, dtype=np.uint64); o = np.empty(n, dtype=np.int64)
    lib().orc_sort(codes, n, s, o)
    return s, o


def order_points(coords, bits):
    """Morton codes, stable sort and gather: (sorted codes, order, Z-ordered coords)."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    codes = morton(coords, bits)
    s, o = sort_codes(codes)
    return s, o, np.ascontiguousarray(coords[:, o])


class Blocks:
    """Leaf list of the block-cluster tree (bounds inclusive, like work_item)."""

    def __init__(self, s1l, s1u, s2l, s2u, typ, lev1, lev2, levels):
        self.s1l, self.s1u, self.s2l, self.s2u = s1l, s1u, s2l, s2u
        self.type, self.lev1, self.lev2, self.levels = typ, lev1, lev2, levels

    def __len__(self):
        return int(self.s1l.shape[0])

    @property
    def m1(self):
        return self.s1u - self.s1l + 1

    @property
    def m2(self):
        return self.s2u - self.s2l + 1

    def subset(self, mask):
        return Blocks(self.s1l[mask].copy(), self.s1u[mask].copy(), self.s2l[mask].copy(),
                      self.s2u[mask].copy(), self.type[mask].copy(), self.lev1[mask].copy(),
                      self.lev2[mask].copy(), self.levels)


def tree(c1, codes1, c2, codes2, eta, c_leaf, max_level=50, root_levels=(0, 0), rule=0,
         sort_dense_first=True) -> Blocks:
    c1 = np.ascontiguousarray(c1, dtype=np.float64)
    c2 = np.ascontiguousarray(c2, dtype=np.float64)
    codes1 = np.ascontiguousarray(codes1, dtype=np.uint64)
    codes2 = np.ascontiguousarray(codes2, dtype=np.uint64)
    dim, n1 = c1.shape
    n2 = c2.shape[1]
    L = lib()
    h = L.orc_tree(c1, codes1, n1, c2, codes2, n2, dim, float(eta), int(c_leaf),
                   int(max_level), int(root_levels[0]), int(root_levels[1]), int(rule),
                   1 if sort_dense_first else 0)
    try:
        nb = L.orc_blocks_count(h)
        arrs = [np.empty(nb, dtype=np.int32) for _ in range(7)]
        if nb:
            L.orc_blocks_get(h, *arrs)
        levels = L.orc_blocks_levels(h)
    finally:
        L.orc_blocks_free(h)
    return Blocks(*arrs, levels)


def _factor_offsets(m, kb):
    sizes = m.astype(np.int64) * kb.astype(np.int64)
    off = np.zeros(len(sizes), dtype=np.int64)
    if len(sizes) > 1:
        off[1:] = np.cumsum(sizes)[:-1]
    return off, int(sizes.sum())


class Factors:
    def __init__(self, blocks, kb, uoff, voff, U, V, ranks):
        self.blocks, self.kb, self.uoff, self.voff = blocks, kb, uoff, voff
        self.U, self.V, self.ranks = U, V, ranks


def aca(kind, param, reg, c1, c2, blocks: Blocks, k, eps=None) -> Factors:
    """Fixed-rank reference ACA (eps None) or the adaptive eps mode on ``blocks``."""
    c1 = np.ascontiguousarray(c1, dtype=np.float64)
    c2 = np.ascontiguousarray(c2, dtype=np.float64)
    dim, n1 = c1.shape
    n2 = c2.shape[1]
    m1, m2 = blocks.m1, blocks.m2
    kb = np.minimum(np.minimum(m1, m2), k).astype(np.int64)
    uoff, us = _factor_offsets(m1, kb)
    voff, vs = _factor_offsets(m2, kb)
    U = np.zeros(max(us, 1)); V = np.zeros(max(vs, 1))
    ranks = np.zeros(len(blocks), dtype=np.int32)
    args = (int(kind), float(param), float(reg), c1, n1, c2, n2, dim, len(blocks),
            blocks.s1l, blocks.s1u, blocks.s2l, blocks.s2u, int(k))
    if eps is None:
        lib().orc_aca_fixed(*args, uoff, voff, U, V, ranks)
    else:
        lib().orc_aca_adaptive(*args, float(eps), uoff, voff, U, V, ranks)
    return Factors(blocks, kb, uoff, voff, U, V, ranks)


def hmatvec(kind, param, reg, c1, c2, blocks: Blocks, fac: Factors, xs):
    """H-matvec in Z order. ``fac`` covers the ACA blocks of ``blocks`` (same order)."""
    c1 = np.ascontiguousarray(c1, dtype=np.float64)
    c2 = np.ascontiguousarray(c2, dtype=np.float64)
    dim, n1 = c1.shape
    n2 = c2.shape[1]
    nb = len(blocks)
    uoff = np.zeros(nb, dtype=np.int64); voff = np.zeros(nb, dtype=np.int64)
    ranks = np.zeros(nb, dtype=np.int32)
    aca_idx = np.nonzero(blocks.type == WT_ACA)[0]
    if fac is not None and len(aca_idx):
        uoff[aca_idx] = fac.uoff; voff[aca_idx] = fac.voff; ranks[aca_idx] = fac.ranks
        U, V = fac.U, fac.V
    else:
        U = np.zeros(1); V = np.zeros(1)
    ys = np.empty(n1)
    lib().orc_hmatvec(int(kind), float(param), float(reg), c1, n1, c2, n2, dim, nb,
                      blocks.s1l, blocks.s1u, blocks.s2l, blocks.s2u, blocks.type, uoff, voff,
                      U, V, ranks, np.ascontiguousarray(xs, dtype=np.float64), ys)
    return ys


def direct(kind, param, reg, c1, c2, xs, rows=None, nthreads=0):
    """FP64 direct sum in Z order (all rows, or the listed rows)."""
    c1 = np.ascontiguousarray(c1, dtype=np.float64)
    c2 = np.ascontiguousarray(c2, dtype=np.float64)
    dim, n1 = c1.shape
    n2 = c2.shape[1]
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    if rows is None:
        y = np.empty(n1)
        lib().orc_direct(int(kind), float(param), float(reg), c1, n1, c2, n2, dim, xs, None,
                         0, y, int(nthreads))
    else:
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        y = np.empty(rows.shape[0])
        lib().orc_direct(int(kind), float(param), float(reg), c1, n1, c2, n2, dim, xs,
                         rows.ctypes.data, rows.shape[0], y, int(nthreads))
    return y


def gaussian_rhs(coords):
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    dim, n = coords.shape
    b = np.empty(n)
    lib().orc_gaussian_rhs(coords, n, dim, b)
    return b
