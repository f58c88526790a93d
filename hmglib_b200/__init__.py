"""B200-native H-matrix engine with the kadircs/hmglib interface.

The compute path is libhmg.so (hand-written sm_100a CUDA behind the C ABI of
include/hmg.h and the reference's entry points in include/hmglib.h).  This
package holds the ctypes binding, the host-side mirror of the reference's
interface (``HMatrix``), the in-tree build and the synthetic input generators.
"""
from ._lib import (ADMISSIBLE_MAX, ADMISSIBLE_MIN, KERNEL_GAUSSIAN, KERNEL_GAUSSIAN_REF,  # noqa: F401
                   KERNEL_MATERN32, KERNEL_MATERN_REF, NEAR_ONTHEFLY, NEAR_STORED, PREC_FP32,
                   PREC_BF16, PREC_BF16X3, PREC_BF16X6, PREC_BF16X6_ONCHIP, PREC_FP64, PREC_MIXED,
                   HmgError, lib)
from .hmatrix import CgMulti, HMatrix, group, group_setup, load, morton_codes, radix_sort_u64  # noqa: F401
