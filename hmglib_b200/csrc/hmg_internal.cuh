// hmg_internal.cuh -- shared device/host definitions of the B200 H-matrix engine.
//
// Data layout in HBM (one handle = one H-matrix between point sets 1 and 2):
//   * points: SoA double coords[d][i], Z-ordered after setup; perm[i] = original
//     index of Z-ordered point i (int32), iperm its inverse.
//   * blocks: SoA int32 (r0, m1, c0, m2, type) in the reference's work-list order
//     (DENSE blocks first, each group in traversal order).
//   * row tiles: the finest row partition induced by all block row ranges, split
//     into pieces of at most HMG_TILE_ROWS rows; each tile is padded to a multiple
//     of 4 rows (16 bytes of FP32) in every stored slice.
//   * near field: per dense block, its tile slices back to back, each column-major
//     (s_pad x m2).
//   * far field: per admissible block, U_b as tile slices (s_pad x r_b column-major)
//     and V_b^T as r_b rows of m2p (= m2 rounded up to 4) entries.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>

#define HMG_TILE_ROWS 128
#define HMG_WT_ACA 1
#define HMG_WT_DENSE 2

#define HMG_KERNEL_GAUSSIAN_REF 1
#define HMG_KERNEL_MATERN_REF 2
#define HMG_KERNEL_GAUSSIAN 3
#define HMG_KERNEL_MATERN32 4

namespace hmg {

struct KernelSpec {
    int kind;       // HMG_KERNEL_*
    int dim;        // point dimension
    double param;   // 1/l^2 (GAUSSIAN) or sqrt(3)/rho (MATERN32); unused otherwise
    double reg;     // added when the Z-ordered row and column indices coincide
    double matern_ref_denom;  // 2^{d/2} Gamma(1+d/2) for MATERN_REF
};

struct PointsView {
    const double* c1[3];  // Z-ordered coordinates of set 1, per dimension
    const double* c2[3];
    int n1, n2;
};

// Squared distance with the contraction nvcc applies to the reference's
// `result += t*t` (kernel_system_assembler.h:42-45): fma(t, t, s) per dimension.
__device__ __forceinline__ double sqdist(const PointsView& P, int dim, int i, int j)
{
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (d < dim) {
            double t = P.c1[d][i] - P.c2[d][j];
            s = __fma_rn(t, t, s);
        }
    }
    return s;
}

// One kernel entry K(i, j) in FP64 (kernel_system_assembler.h:33-52, 77-96).
__device__ __forceinline__ double kernel_from_sq(const KernelSpec& K, double s)
{
    switch (K.kind) {
    case HMG_KERNEL_GAUSSIAN_REF: {
        double r = sqrt(s);
        return exp(-r * r);
    }
    case HMG_KERNEL_MATERN_REF: {
        double r = sqrt(s);
        return (yn(1, r + 1.0e-15) * r) / K.matern_ref_denom;
    }
    case HMG_KERNEL_GAUSSIAN:
        return exp(-(s * K.param));
    case HMG_KERNEL_MATERN32: {
        double a = sqrt(s) * K.param;
        return (1.0 + a) * exp(-a);
    }
    default:
        return 0.0;
    }
}

__device__ __forceinline__ double kernel_entry(const KernelSpec& K, const PointsView& P, int i,
                                               int j)
{
    double v = kernel_from_sq(K, sqdist(P, K.dim, i, j));
    if (i == j) v += K.reg;
    return v;
}

// ---------------------------------------------------------------------------
// Host-side error handling: every C-ABI entry returns a status and records a
// message retrievable with hmg_last_error().
// ---------------------------------------------------------------------------
void set_error(const char* fmt, ...);

#define HMG_CUDA_TRY(expr)                                                                  \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess) {                                                            \
            ::hmg::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,                    \
                             cudaGetErrorString(_e));                                       \
            return HMG_ERR_CUDA;                                                            \
        }                                                                                   \
    } while (0)

#define HMG_LAUNCH_CHECK() HMG_CUDA_TRY(cudaGetLastError())

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
inline int round_up4(int x) { return (x + 3) & ~3; }

}  // namespace hmg
