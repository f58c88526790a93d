"""ctypes binding of libhmg.so (include/hmg.h).

The library is built in-tree by ``python -m hmglib_b200.build``; importing this
module never falls back to anything else: a missing library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhmg.so")

HMG_OK = 0
STATUS_NAMES = {0: "HMG_OK", 1: "HMG_ERR_INVALID", 2: "HMG_ERR_CUDA", 3: "HMG_ERR_NOMEM",
                4: "HMG_ERR_STATE", 5: "HMG_ERR_UNSUPPORTED"}

KERNEL_GAUSSIAN_REF = 1
KERNEL_MATERN_REF = 2
KERNEL_GAUSSIAN = 3
KERNEL_MATERN32 = 4
ADMISSIBLE_MAX = 0
ADMISSIBLE_MIN = 1
PREC_FP64 = 0
PREC_FP32 = 1
PREC_MIXED = 2
PREC_BF16 = 3
PREC_BF16X3 = 4
PREC_BF16X6 = 5
PREC_BF16X6_ONCHIP = 6
NEAR_STORED = 0
NEAR_ONTHEFLY = 1


class HmgError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Info(C.Structure):
    _fields_ = [("n1", C.c_int), ("n2", C.c_int), ("dim", C.c_int), ("bits", C.c_int),
                ("block_count", C.c_int), ("dense_count", C.c_int), ("aca_count", C.c_int),
                ("levels", C.c_int), ("tile_count", C.c_int), ("max_rank", C.c_int),
                ("near_entries", C.c_int64), ("far_entries", C.c_int64), ("far_rows", C.c_int64),
                ("near_bytes", C.c_int64), ("far_bytes", C.c_int64), ("matvec_bytes", C.c_int64),
                ("near_precision", C.c_int), ("far_precision", C.c_int), ("near_mode", C.c_int),
                ("far_u_bytes", C.c_int64), ("far_v_bytes", C.c_int64), ("matvec_launches", C.c_int),
                ("group_count", C.c_int), ("tc_parts", C.c_int), ("tc_bytes", C.c_int64),
                ("tc_onchip", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

_vp = C.c_void_p
_PROTOS = {
    "hmg_last_error": (C.c_char_p, []),
    "hmg_version": (C.c_int, []),
    "hmg_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    "hmg_set_points": (C.c_int, [_vp, C.c_int, _vp, C.c_int]),
    "hmg_setup": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "hmg_set_kernel": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double]),
    "hmg_precompute_aca": (C.c_int, [_vp, C.c_int, C.c_double, C.c_int]),
    "hmg_precompute_dense": (C.c_int, [_vp, C.c_int]),
    "hmg_set_near_mode": (C.c_int, [_vp, C.c_int]),
    "hmg_matvec": (C.c_int, [_vp, _vp, _vp]),
    "hmg_matvec_host": (C.c_int, [_vp, _vp, _vp]),
    "hmg_matvec_unbatched": (C.c_int, [_vp, _vp, _vp]),
    "hmg_matvec_multi": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, C.c_int]),
    "hmg_group_create": (C.c_int, [C.POINTER(_vp), C.POINTER(_vp), C.c_int, _vp]),
    "hmg_group_setup": (C.c_int, [C.POINTER(_vp), C.POINTER(_vp), C.c_int, C.c_double, C.POINTER(C.c_int),
                                  C.c_int, C.c_int, _vp]),
    "hmg_group_offsets": (C.c_int, [_vp, C.c_int, _vp]),
    "hmg_save": (C.c_int, [_vp, C.c_char_p]),
    "hmg_build_bf16_factors": (C.c_int, [_vp]),
    "hmg_build_tensor_core_operands": (C.c_int, [_vp, C.c_int]),
    "hmg_set_graphs": (C.c_int, [_vp, C.c_int]),
    "hmg_autotune": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "hmg_load": (C.c_int, [C.POINTER(_vp), C.c_char_p, _vp]),
    "hmg_full_matvec": (C.c_int, [_vp, _vp, _vp]),
    "hmg_full_matvec_rows": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp]),
    "hmg_gaussian_rhs": (C.c_int, [_vp, _vp]),
    "hmg_cg_solve": (C.c_int, [_vp, C.c_double, _vp, _vp, C.c_double, C.c_int, C.c_int,
                               C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "hmg_cg_solve_multi": (C.c_int, [_vp, C.c_int, C.c_double, _vp, C.c_int, _vp, C.c_int, C.c_double,
                                     C.c_int, C.c_int, C.POINTER(C.c_int), _vp]),
    "hmg_cg_multi_begin": (C.c_int, [C.POINTER(_vp), _vp, C.c_int, C.c_double, _vp, C.c_int, _vp, C.c_int,
                                     C.c_double, C.c_int, C.c_int]),
    "hmg_cg_multi_advance": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "hmg_cg_multi_poll": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), _vp]),
    "hmg_cg_multi_end": (C.c_int, [_vp]),
    "hmg_synchronize": (C.c_int, [_vp]),
    "hmg_set_profiling": (C.c_int, [_vp, C.c_int]),
    "hmg_get_profile": (C.c_int, [_vp, _vp]),
    "hmg_set_matvec_variant": (C.c_int, [_vp, C.c_int]),
    "hmg_set_product_precision": (C.c_int, [_vp, C.c_int]),
    "hmg_set_tensor_core_min_vectors": (C.c_int, [_vp, C.c_int]),
    "hmg_destroy": (C.c_int, [_vp]),
    "hmg_get_info": (C.c_int, [_vp, C.POINTER(Info)]),
    "hmg_get_codes": (C.c_int, [_vp, C.c_int, _vp]),
    "hmg_get_order": (C.c_int, [_vp, C.c_int, _vp]),
    "hmg_get_points": (C.c_int, [_vp, C.c_int, _vp]),
    "hmg_get_blocks": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hmg_get_ranks": (C.c_int, [_vp, _vp]),
    "hmg_get_factors": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "hmg_radix_sort_u64": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _vp]),
    "hmg_morton_codes": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp]),
}


def lib():
    """Load libhmg.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m hmglib_b200.build`")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in _PROTOS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int, where: str):
    if status != HMG_OK:
        msg = lib().hmg_last_error()
        raise HmgError(status, where, msg.decode() if msg else "")
