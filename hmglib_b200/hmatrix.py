"""Host-side mirror of the reference's H-matrix interface (src/hmglib.h:29-121).

``HMatrix`` keeps the reference's life cycle -- init, setup, precompute_aca,
precompute_dense, apply, apply_full, destroy -- and argument meaning, on top of
the C ABI in include/hmg.h.  Vectors may be NumPy arrays (host; copied in and out
inside the call) or CUDA tensors / any object exposing ``data_ptr()`` (device;
stream-ordered on the handle's stream, which is the legacy default stream unless
``stream`` is given).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def _ptr(a):
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


class HMatrix:
    """An H-matrix between point sets 1 (rows) and 2 (columns)."""

    def __init__(self, n1: int, n2: int, dim: int, bits: int = 0, stream: int | None = None):
        self._lib = L.lib()
        h = C.c_void_p()
        L.check(self._lib.hmg_create(C.byref(h), int(n1), int(n2), int(dim), int(bits),
                                     C.c_void_p(stream or 0)), "hmg_create")
        self._h = h
        self.n1, self.n2, self.dim = int(n1), int(n2), int(dim)

    # -- life cycle ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.hmg_destroy(self._h)
            self._h = None

    destroy = close

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, name, *args):
        L.check(getattr(self._lib, name)(self._h, *args), name)

    # -- construction ----------------------------------------------------------
    def set_points(self, which: int, coords):
        """coords: (dim, n) float64, host array or device tensor (SoA)."""
        if hasattr(coords, "data_ptr"):
            assert tuple(coords.shape) == (self.dim, (self.n1, self.n2)[which])
            self._call("hmg_set_points", int(which), _ptr(coords), 1)
        else:
            c = np.ascontiguousarray(coords, dtype=np.float64)
            assert c.shape == (self.dim, (self.n1, self.n2)[which]), c.shape
            self._call("hmg_set_points", int(which), _ptr(c), 0)

    def setup(self, eta: float, c_leaf: int, max_level: int = 50, root_levels=(0, 0),
              rule: int = L.ADMISSIBLE_MAX):
        self._call("hmg_setup", float(eta), int(c_leaf), int(max_level), int(root_levels[0]),
                   int(root_levels[1]), int(rule))

    def set_kernel(self, kind: int, param: float = 0.0, regularization: float = 0.0):
        self._call("hmg_set_kernel", int(kind), float(param), float(regularization))

    def precompute_aca(self, k: int, eps: float = 0.0, precision: int = L.PREC_FP64):
        self._call("hmg_precompute_aca", int(k), float(eps), int(precision))

    def precompute_dense(self, precision: int = L.PREC_FP64):
        self._call("hmg_precompute_dense", int(precision))

    def set_near_mode(self, mode: int):
        self._call("hmg_set_near_mode", int(mode))

    # -- products --------------------------------------------------------------
    def matvec(self, x, y=None):
        """y = H x.  Host arrays: synchronous.  Device tensors: asynchronous."""
        if hasattr(x, "data_ptr"):
            assert y is not None, "pass a device output tensor"
            self._call("hmg_matvec", _ptr(x), _ptr(y))
            return y
        xh = np.ascontiguousarray(x, dtype=np.float64)
        yh = np.empty(self.n1) if y is None else y
        self._call("hmg_matvec_host", _ptr(xh), _ptr(yh))
        return yh

    apply = matvec

    def matvec_multi(self, X, Y):
        """Y = H X for device FP64 tensors X (n2 x nrhs) and Y (n1 x nrhs), column-major
        (a tensor of shape (nrhs, n) row-major is the column-major (n, nrhs) matrix);
        asynchronous."""
        nrhs = int(X.shape[0])
        self._call("hmg_matvec_multi", nrhs, _ptr(X), int(X.stride(0)), _ptr(Y), int(Y.stride(0)))
        return Y

    def matvec_unbatched(self, x, y):
        """y = H x one block per launch on device tensors (hmg_matvec_unbatched, the
        reference's sequential_h_matrix_mvp_without_batching); asynchronous."""
        self._call("hmg_matvec_unbatched", _ptr(x), _ptr(y))
        return y

    def matvec_device(self, x_ptr: int, y_ptr: int):
        self._call("hmg_matvec", C.c_void_p(x_ptr), C.c_void_p(y_ptr))

    def full_matvec(self, x, y):
        """FP64 direct product on device tensors (apply_full_mvp)."""
        self._call("hmg_full_matvec", _ptr(x), _ptr(y))
        return y

    def full_matvec_rows(self, x, rows, y):
        self._call("hmg_full_matvec_rows", _ptr(x), _ptr(rows), int(rows.shape[0]), _ptr(y))
        return y

    def cg_solve(self, b, x, shift: float, tol: float = 1e-8, maxit: int = 1000, refine: bool = True):
        """Solve (H + shift I) x = b on device tensors; x is the initial guess.
        Returns (iterations, final relative residual)."""
        it = C.c_int(0)
        rel = C.c_double(0.0)
        self._call("hmg_cg_solve", float(shift), _ptr(b), _ptr(x), float(tol), int(maxit),
                   1 if refine else 0, C.byref(it), C.byref(rel))
        return it.value, rel.value

    def cg_solve_multi(self, B, X, shift: float, tol: float = 1e-8, maxit: int = 1000, refine: bool = True):
        """Solve (H + shift I) X = B for the rows of device tensors B, X of shape
        (nrhs, n) (column-major n x nrhs); X holds the initial guesses.  Returns
        (iterations, per-column final relative residuals)."""
        nrhs = int(B.shape[0])
        it = C.c_int(0)
        rel = np.zeros(nrhs)
        self._call("hmg_cg_solve_multi", nrhs, float(shift), _ptr(B), int(B.stride(0)), _ptr(X),
                   int(X.stride(0)), float(tol), int(maxit), 1 if refine else 0, C.byref(it), _ptr(rel))
        return it.value, rel

    def cg_multi(self, B, X, shift: float, tol: float = 1e-8, maxit: int = 1000, refine: bool = True):
        """A step-driven block CG solve (hmg_cg_multi_*): see CgMulti."""
        return CgMulti(self, B, X, shift, tol, maxit, refine)

    def gaussian_rhs(self, b):
        self._call("hmg_gaussian_rhs", _ptr(b))
        return b

    def synchronize(self):
        self._call("hmg_synchronize")

    def set_matvec_variant(self, variant: int):
        """0: streaming (bulk-copy) product kernels, 1: plain-load kernels."""
        self._call("hmg_set_matvec_variant", int(variant))

    def autotune(self, reps: int = 3) -> dict:
        """Choose the product's V^T task size and grid by timing them (hmg_autotune)."""
        piece, ctas, ms = C.c_int(0), C.c_int(0), C.c_double(0.0)
        self._call("hmg_autotune", int(reps), C.byref(piece), C.byref(ctas), C.byref(ms))
        return {"piece_bytes": piece.value, "ctas_per_sm": ctas.value, "ms": ms.value}

    def set_graphs(self, on: bool = True):
        """Replay products as a captured CUDA graph (hmg_set_graphs)."""
        self._call("hmg_set_graphs", int(bool(on)))

    def build_bf16_factors(self, near: int = L.PREC_BF16):
        """BF16 tcgen05 operands of the FP32 factors for tensor-core multi-vector products
        (hmg_build_tensor_core_operands); the near field on the tensor cores too
        (near=PREC_BF16), in FP32 on the CUDA cores (near=PREC_FP32), or every operand
        as a BF16 hi + lo pair (near=PREC_BF16X3, ~5e-6) or as three BF16 parts
        (near=PREC_BF16X6, 24 bits)."""
        self._call("hmg_build_tensor_core_operands", int(near))

    def save(self, path: str):
        """Write the H-matrix to `path` (hmg_save)."""
        self._call("hmg_save", str(path).encode())

    def offsets(self, which: int = 0) -> np.ndarray:
        """Group handles: first row (which=0) or column (1) of every set, then n."""
        cnt = self.info()["group_count"]
        out = np.zeros(cnt + 1, dtype=np.int64)
        self._call("hmg_group_offsets", int(which), _ptr(out))
        return out

    def set_tensor_core_min_vectors(self, nrhs: int):
        """With on-chip tensor-core operands, multi-vector products of fewer than nrhs
        vectors (default 17) run on the CUDA cores (hmg_set_tensor_core_min_vectors)."""
        self._call("hmg_set_tensor_core_min_vectors", int(nrhs))

    def set_product_precision(self, precision: int):
        """Arithmetic of products over FP32/mixed storage: PREC_FP32 (default) or PREC_FP64."""
        self._call("hmg_set_product_precision", int(precision))

    def set_profiling(self, on: bool = True):
        self._call("hmg_set_profiling", 1 if on else 0)

    def profile(self) -> dict:
        """Device milliseconds of the last product's phases."""
        out = np.zeros(4)
        self._call("hmg_get_profile", _ptr(out))
        return {"gather_ms": out[0], "vtx_ms": out[1], "tiles_ms": out[2], "total_ms": out[3]}

    # -- inspection --------------------------------------------------------------
    def info(self) -> dict:
        i = L.Info()
        self._call("hmg_get_info", C.byref(i))
        return i.as_dict()

    def codes(self, which: int) -> np.ndarray:
        n = (self.n1, self.n2)[which]
        out = np.empty(n, dtype=np.uint64)
        self._call("hmg_get_codes", int(which), _ptr(out))
        return out

    def order(self, which: int) -> np.ndarray:
        n = (self.n1, self.n2)[which]
        out = np.empty(n, dtype=np.int64)
        self._call("hmg_get_order", int(which), _ptr(out))
        return out

    def points(self, which: int) -> np.ndarray:
        n = (self.n1, self.n2)[which]
        out = np.empty((self.dim, n), dtype=np.float64)
        self._call("hmg_get_points", int(which), _ptr(out))
        return out

    def blocks(self):
        """(s1l, s1u, s2l, s2u, type): the leaf list in the reference's order."""
        nb = self.info()["block_count"]
        arrs = [np.empty(nb, dtype=np.int32) for _ in range(5)]
        self._call("hmg_get_blocks", *[_ptr(a) for a in arrs])
        return tuple(arrs)

    def ranks(self) -> np.ndarray:
        nb = self.info()["block_count"]
        out = np.empty(nb, dtype=np.int32)
        self._call("hmg_get_ranks", _ptr(out))
        return out

    def factors(self, block: int, m1: int, m2: int, rank: int):
        U = np.zeros((max(rank, 1), m1))
        V = np.zeros((max(rank, 1), m2))
        self._call("hmg_get_factors", int(block), _ptr(U), _ptr(V))
        return U[:rank], V[:rank]


class CgMulti:
    """(H + shift I) X = B advanced one enqueued piece of work at a time: ``advance()``
    enqueues at most one CG iteration (or a true residual and restart) on the
    H-matrix's stream without waiting for the GPU and returns whether it did;
    ``poll()`` returns (done, iterations, relative residuals) without blocking;
    ``close()`` waits for the stream and frees the work vectors.  B and X (device
    tensors of shape (nrhs, n)) must stay alive until then."""

    def __init__(self, H: HMatrix, B, X, shift, tol, maxit, refine):
        self._lib = H._lib
        self._s = C.c_void_p()
        self.nrhs = int(B.shape[0])
        self._keep = (H, B, X)
        L.check(self._lib.hmg_cg_multi_begin(C.byref(self._s), H._h, self.nrhs, float(shift), _ptr(B),
                                             int(B.stride(0)), _ptr(X), int(X.stride(0)), float(tol), int(maxit),
                                             1 if refine else 0), "hmg_cg_multi_begin")

    def advance(self) -> bool:
        e = C.c_int(0)
        L.check(self._lib.hmg_cg_multi_advance(self._s, C.byref(e)), "hmg_cg_multi_advance")
        return bool(e.value)

    def poll(self):
        done, it = C.c_int(0), C.c_int(0)
        rel = np.zeros(self.nrhs)
        L.check(self._lib.hmg_cg_multi_poll(self._s, C.byref(done), C.byref(it), _ptr(rel)), "hmg_cg_multi_poll")
        return bool(done.value), it.value, rel

    def close(self):
        if self._s:
            self._lib.hmg_cg_multi_end(self._s)
            self._s = None
            self._keep = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load(path: str, stream: int | None = None) -> "HMatrix":
    """An H-matrix written by HMatrix.save (hmg_load)."""
    lib = L.lib()
    h = C.c_void_p()
    L.check(lib.hmg_load(C.byref(h), str(path).encode(), C.c_void_p(stream or 0)), "hmg_load")
    H = HMatrix.__new__(HMatrix)
    H._lib = lib
    H._h = h
    i = H.info()
    H.n1, H.n2, H.dim = i["n1"], i["n2"], i["dim"]
    return H


def group(sets, stream: int | None = None) -> "HMatrix":
    """The block-diagonal union of set-up HMatrix objects (hmg_group_create): one
    handle whose products cover every set in the same launches.  Vectors are the
    concatenation of the sets' vectors; `offsets(0)` gives each set's first row."""
    lib = L.lib()
    arr = (C.c_void_p * len(sets))(*[hm._h.value for hm in sets])
    h = C.c_void_p()
    L.check(lib.hmg_group_create(C.byref(h), arr, len(sets), C.c_void_p(stream or 0)), "hmg_group_create")
    g = HMatrix.__new__(HMatrix)
    g._lib = lib
    g._h = h
    g.n1 = sum(hm.n1 for hm in sets)
    g.n2 = sum(hm.n2 for hm in sets)
    g.dim = max(hm.dim for hm in sets)
    return g


def group_setup(sets, eta: float, c_leaf, max_level: int = 50, rule: int = L.ADMISSIBLE_MAX,
                stream: int | None = None) -> "HMatrix":
    """The block-diagonal union of HMatrix objects that have points and a kernel but
    need not be set up (hmg_group_setup): every set is ordered and clustered in the same
    kernel launches.  `c_leaf` is one leaf size for all sets or one per set.  Equal, bit
    for bit, to `group` over the sets after `setup(eta, c_leaf[i], max_level,
    rule=rule)` on each."""
    lib = L.lib()
    leaf = [int(c_leaf)] * len(sets) if np.isscalar(c_leaf) else [int(c) for c in c_leaf]
    if len(leaf) != len(sets):
        raise ValueError("c_leaf: one value, or one per set")
    arr = (C.c_void_p * len(sets))(*[hm._h.value for hm in sets])
    lv = (C.c_int * len(sets))(*leaf)
    h = C.c_void_p()
    L.check(lib.hmg_group_setup(C.byref(h), arr, len(sets), float(eta), lv, int(max_level), int(rule),
                                C.c_void_p(stream or 0)), "hmg_group_setup")
    g = HMatrix.__new__(HMatrix)
    g._lib = lib
    g._h = h
    g.n1 = sum(hm.n1 for hm in sets)
    g.n2 = sum(hm.n2 for hm in sets)
    g.dim = max(hm.dim for hm in sets)
    return g


def radix_sort_u64(keys_ptr: int, vals_ptr: int, n: int, key_bits: int = 64, stream: int = 0):
    L.check(L.lib().hmg_radix_sort_u64(C.c_void_p(keys_ptr), C.c_void_p(vals_ptr), int(n),
                                       int(key_bits), C.c_void_p(stream)), "hmg_radix_sort_u64")


def morton_codes(coords_ptr: int, n: int, dim: int, bits: int, codes_ptr: int, stream: int = 0):
    L.check(L.lib().hmg_morton_codes(C.c_void_p(coords_ptr), int(n), int(dim), int(bits),
                                     C.c_void_p(codes_ptr), C.c_void_p(stream)), "hmg_morton_codes")
