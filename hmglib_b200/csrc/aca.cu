// aca.cu -- batched ACA of all admissible blocks, one CTA per block, FP64.
//
// The reference (linear_algebra.cu:3684-4012) advances all blocks in lock step:
// every rank step is ~10 kernel launches, Thrust reduce_by_key calls and a host
// synchronisation, over "batched" vectors that concatenate all blocks.  Here one
// CTA owns one block for its whole ACA: the residual row / column, the pivot
// searches and the norms are CTA reductions, and the only traffic is the block's
// own U/V panels (L2-resident for all but the largest blocks).
//
// Two modes:
//   * fixed (eps <= 0): the reference's semantics -- rank k_b = min(k,m1,m2)
//     (:769-787), row pivots taken in index order skipping residual rows of norm
//     < 1e-13 (:2009-2024, :2091, :1213-1230), column pivot = LAST index of the
//     largest |v| (tuple_absolute_maximum, :991-1018), v scaled by the pivot
//     (:963-986), residual updates with fused multiply-adds (:918-959, :1091-1147).
//     The reference's scaling kernel reads the pivot entry while other threads
//     overwrite it (:983); here the pivot is read once before any write.
//   * adaptive (eps > 0): standard partial pivoting -- next row = largest |u_r| over
//     unused rows, column = FIRST index of the largest |v| -- stopping when
//     |u_r| |v_r| <= eps ||S_r||_F with the Frobenius norm of the approximant
//     updated exactly (the criterion the reference keeps dormant at
//     :1595-1755, without its (1-eta) factor, which is negative for eta > 1).
//
// Factors are computed into FP64 scratch per batch of blocks and then compacted
// (converted to the storage precision, laid out as tile slices for U and as
// padded rows of V^T) into one allocation per batch.
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <vector>

#include "hmg_matrix.cuh"

namespace hmg {

static constexpr int ACA_THREADS = 256;
static constexpr int ACA_WARPS = ACA_THREADS / 32;
static constexpr int ACA_KMAX = 512;

struct AcaBatch {
    const int* blocks;       // block indices of this batch
    const long long* uoff;   // FP64 scratch offsets
    const long long* voff;
    double* U;
    double* V;
    int* rank_out;           // per batch entry
    double* s2_out;          // per batch entry: |U V^T|_F^2 (adaptive mode), may be null
};

struct BlockGeom {
    const int *r0, *m1, *c0, *m2;
    const double* param;  // per-block kernel parameter (grouped H-matrices), else null
};

__device__ __forceinline__ double block_sum(double v, double* red)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < ACA_WARPS; w++) s += red[w];
    return s;
}

// (value, index) argmax; last = true: ties go to the larger index, else the smaller.
__device__ __forceinline__ bool better(double a, int i, double b, int j, bool last)
{
    if (a != b) return a > b;
    return last ? i > j : i < j;
}

__device__ __forceinline__ void block_argmax(double& a, int& i, bool last, double* reda,
                                             int* redi)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double b = __shfl_xor_sync(0xffffffffu, a, o);
        int j = __shfl_xor_sync(0xffffffffu, i, o);
        if (better(b, j, a, i, last)) { a = b; i = j; }
    }
    __syncthreads();
    if (lane == 0) { reda[warp] = a; redi[warp] = i; }
    __syncthreads();
    a = reda[0];
    i = redi[0];
#pragma unroll
    for (int w = 1; w < ACA_WARPS; w++)
        if (better(reda[w], redi[w], a, i, last)) { a = reda[w]; i = redi[w]; }
}

// four CTAs an SM: the rank steps are latency-bound, so occupancy sets their pace
__global__ void __launch_bounds__(ACA_THREADS, 4)
k_aca(BlockGeom g, KernelSpec K0, PointsView P, AcaBatch B, int k, double eps, const int* elist)
{
    __shared__ double coef[ACA_KMAX];
    __shared__ double red[ACA_WARPS];
    __shared__ double reda[ACA_WARPS];
    __shared__ int redi[ACA_WARPS];
    extern __shared__ unsigned used[];  // adaptive mode: one bit per row

    const int e = elist ? elist[blockIdx.x] : blockIdx.x;
    const int b = B.blocks[e];
    KernelSpec K = K0;
    if (g.param) K.param = g.param[b];
    const int r0 = g.r0[b], m1 = g.m1[b], c0 = g.c0[b], m2 = g.m2[b];
    int kb = k < m1 ? k : m1;
    kb = kb < m2 ? kb : m2;
    double* U = B.U + B.uoff[e];
    double* V = B.V + B.voff[e];
    const int tid = threadIdx.x;
    const bool adaptive = eps > 0.0;
    int rank = 0;
    double S2 = 0.0;  // adaptive mode: squared Frobenius norm of the approximant

    if (!adaptive) {
        int ir = -1;
        for (int r = 0; r < kb; r++) {
            bool found = false;
            for (;;) {
                if (ir >= m1 - 1) break;
                ir += 1;
                for (int l = tid; l < r; l += ACA_THREADS) coef[l] = U[ir + (size_t)l * m1];
                __syncthreads();
                double ss = 0.0;
                for (int j = tid; j < m2; j += ACA_THREADS) {
                    double val = kernel_entry(K, P, r0 + ir, c0 + j);
                    for (int l = 0; l < r; l++)
                        val = __fma_rn(-coef[l], V[j + (size_t)l * m2], val);
                    V[j + (size_t)r * m2] = val;
                    ss += val * val;
                }
                double n2 = block_sum(ss, red);
                if (sqrt(n2) >= 1.0e-13) { found = true; break; }
                __syncthreads();
            }
            if (!found) break;
            double best = -1.0;
            int jr = 0;
            for (int j = tid; j < m2; j += ACA_THREADS) {
                double a = fabs(V[j + (size_t)r * m2]);
                if (better(a, j, best, jr, true)) { best = a; jr = j; }
            }
            block_argmax(best, jr, true, reda, redi);
            const double piv = V[jr + (size_t)r * m2];
            __syncthreads();
            for (int j = tid; j < m2; j += ACA_THREADS)
                V[j + (size_t)r * m2] = V[j + (size_t)r * m2] / piv;
            for (int l = tid; l < r; l += ACA_THREADS) coef[l] = V[jr + (size_t)l * m2];
            __syncthreads();
            for (int i = tid; i < m1; i += ACA_THREADS) {
                double val = kernel_entry(K, P, r0 + i, c0 + jr);
                for (int l = 0; l < r; l++) val = __fma_rn(-coef[l], U[i + (size_t)l * m1], val);
                U[i + (size_t)r * m1] = val;
            }
            rank = r + 1;
            __syncthreads();
        }
    } else {
        const int nwords = (m1 + 31) >> 5;
        for (int w = tid; w < nwords; w += ACA_THREADS) used[w] = 0u;
        __syncthreads();
        int ir = 0, nused = 0;
        for (int r = 0; r < kb; r++) {
            int jr = -1;
            double piv = 0.0;
            bool have = false;
            for (;;) {
                if (tid == 0) used[ir >> 5] |= 1u << (ir & 31);
                nused++;
                for (int l = tid; l < r; l += ACA_THREADS) coef[l] = U[ir + (size_t)l * m1];
                __syncthreads();
                double best = -1.0;
                int bj = 0x7fffffff;
                for (int j = tid; j < m2; j += ACA_THREADS) {
                    double val = kernel_entry(K, P, r0 + ir, c0 + j);
                    for (int l = 0; l < r; l++)
                        val = __fma_rn(-coef[l], V[j + (size_t)l * m2], val);
                    V[j + (size_t)r * m2] = val;
                    double a = fabs(val);
                    if (better(a, j, best, bj, false)) { best = a; bj = j; }
                }
                block_argmax(best, bj, false, reda, redi);
                if (best > 0.0) {
                    jr = bj;
                    have = true;
                    break;
                }
                // zero residual row: the next unused row in index order
                int cand = 0x7fffffff;
                for (int i = tid; i < m1; i += ACA_THREADS)
                    if (!((used[i >> 5] >> (i & 31)) & 1u)) { cand = i; break; }
                double dummy = 0.0;
                block_argmax(dummy, cand, false, reda, redi);
                if (cand == 0x7fffffff) break;
                ir = cand;
                __syncthreads();
            }
            if (!have) break;
            piv = V[jr + (size_t)r * m2];
            __syncthreads();
            double pv = 0.0;
            for (int j = tid; j < m2; j += ACA_THREADS) {
                double v = V[j + (size_t)r * m2] / piv;
                V[j + (size_t)r * m2] = v;
                pv += v * v;
            }
            for (int l = tid; l < r; l += ACA_THREADS) coef[l] = V[jr + (size_t)l * m2];
            __syncthreads();
            double pu = 0.0, bu = -1.0;
            int bi = 0x7fffffff;
            for (int i = tid; i < m1; i += ACA_THREADS) {
                double val = kernel_entry(K, P, r0 + i, c0 + jr);
                for (int l = 0; l < r; l++) val = __fma_rn(-coef[l], U[i + (size_t)l * m1], val);
                U[i + (size_t)r * m1] = val;
                pu += val * val;
                if (!((used[i >> 5] >> (i & 31)) & 1u)) {
                    double a = fabs(val);
                    if (better(a, i, bu, bi, false)) { bu = a; bi = i; }
                }
            }
            double nv2 = block_sum(pv, red);
            double nu2 = block_sum(pu, red);
            block_argmax(bu, bi, false, reda, redi);
            // cross terms sum_l (u_r . U_l)(v_r . V_l): warp w takes columns l = w mod 8 whole
            // (coalesced dot products, a fixed-order warp reduction), warp 0 sums the
            // products over l in order.  Few registers per thread, so several CTAs share an SM.
            {
                const int warp = tid >> 5, lane = tid & 31;
                const double* ur = U + (size_t)r * m1;
                const double* vr = V + (size_t)r * m2;
                for (int l = warp; l < r; l += ACA_WARPS) {
                    const double* ul = U + (size_t)l * m1;
                    const double* vl = V + (size_t)l * m2;
                    double a = 0.0, c = 0.0;
                    for (int i = lane; i < m1; i += 32) a = __fma_rn(ur[i], ul[i], a);
                    for (int j = lane; j < m2; j += 32) c = __fma_rn(vr[j], vl[j], c);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        a += __shfl_xor_sync(0xffffffffu, a, o);
                        c += __shfl_xor_sync(0xffffffffu, c, o);
                    }
                    if (lane == 0) coef[l] = a * c;
                }
                __syncthreads();
                if (warp == 0) {
                    double p = 0.0;
                    for (int l = lane; l < r; l += 32) p += coef[l];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
                    if (lane == 0) red[0] = p;
                }
                __syncthreads();
            }
            const double cross = red[0];
            __syncthreads();
            S2 = S2 + 2.0 * cross + nu2 * nv2;
            rank = r + 1;
            if (sqrt(nu2 * nv2) <= eps * sqrt(fabs(S2))) break;
            if (nused >= m1) break;
            if (bi == 0x7fffffff) break;
            ir = bi;
            __syncthreads();
        }
    }
    if (tid == 0) {
        B.rank_out[e] = rank;
        if (B.s2_out) B.s2_out[e] = S2;
    }
}


// ---------------------------------------------------------------------------
// The adaptive ACA of a small block (m1, m2 <= ACA_WSMALL) by one warp: the steps of
// k_aca's adaptive mode with warp shuffles in place of CTA reductions and no CTA
// barriers.  Most admissible blocks are small (at N = 2^20, 925k of 1.16M have
// m1 + m2 < 512); a CTA of 256 threads per block would leave most lanes idle and
// synchronise six times a rank step.
// ---------------------------------------------------------------------------
static constexpr int ACA_WSMALL = 512;              // largest m1 and m2 of the warp variant
static constexpr int ACA_WPC = 8;                   // warps (blocks) per CTA

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// (value, index) argmax over the warp; ties go to the smaller index
__device__ __forceinline__ void warp_argmax_first(double& a, int& i)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double b = __shfl_xor_sync(0xffffffffu, a, o);
        const int j = __shfl_xor_sync(0xffffffffu, i, o);
        if (better(b, j, a, i, false)) { a = b; i = j; }
    }
}

__global__ void __launch_bounds__(ACA_WPC * 32, 4)
k_aca_warp(BlockGeom g, KernelSpec K0, PointsView P, AcaBatch B, int k, double eps, const int* elist, int nlist)
{
    __shared__ double coefs[ACA_WPC][ACA_WSMALL];
    __shared__ unsigned usedw[ACA_WPC][ACA_WSMALL / 32];
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = blockIdx.x * ACA_WPC + wi;
    if (slot >= nlist) return;
    const int e = elist[slot];
    const int b = B.blocks[e];
    KernelSpec K = K0;
    if (g.param) K.param = g.param[b];
    const int r0 = g.r0[b], m1 = g.m1[b], c0 = g.c0[b], m2 = g.m2[b];
    int kb = k < m1 ? k : m1;
    kb = kb < m2 ? kb : m2;
    double* U = B.U + B.uoff[e];
    double* V = B.V + B.voff[e];
    double* coef = coefs[wi];
    unsigned* used = usedw[wi];
    for (int w = lane; w < ACA_WSMALL / 32; w += 32) used[w] = 0u;
    __syncwarp();
    int rank = 0, ir = 0, nused = 0;
    double S2 = 0.0;
    for (int r = 0; r < kb; r++) {
        int jr = -1;
        bool have = false;
        for (;;) {
            if (lane == 0) used[ir >> 5] |= 1u << (ir & 31);
            nused++;
            for (int l = lane; l < r; l += 32) coef[l] = U[ir + (size_t)l * m1];
            __syncwarp();
            double best = -1.0;
            int bj = 0x7fffffff;
            for (int j = lane; j < m2; j += 32) {
                double val = kernel_entry(K, P, r0 + ir, c0 + j);
                for (int l = 0; l < r; l++) val = __fma_rn(-coef[l], V[j + (size_t)l * m2], val);
                V[j + (size_t)r * m2] = val;
                const double a = fabs(val);
                if (better(a, j, best, bj, false)) { best = a; bj = j; }
            }
            warp_argmax_first(best, bj);
            if (best > 0.0) {
                jr = bj;
                have = true;
                break;
            }
            // zero residual row: the next unused row in index order
            int cand = 0x7fffffff;
            for (int i = lane; i < m1; i += 32)
                if (!((used[i >> 5] >> (i & 31)) & 1u)) { cand = i; break; }
            double dummy = 0.0;
            warp_argmax_first(dummy, cand);
            if (cand == 0x7fffffff) break;
            ir = cand;
            __syncwarp();
        }
        if (!have) break;
        __syncwarp();  // every lane's V[., r] written
        const double piv = V[jr + (size_t)r * m2];
        double pv = 0.0;
        for (int j = lane; j < m2; j += 32) {
            const double v = V[j + (size_t)r * m2] / piv;
            V[j + (size_t)r * m2] = v;
            pv += v * v;
        }
        __syncwarp();
        for (int l = lane; l < r; l += 32) coef[l] = V[jr + (size_t)l * m2];
        __syncwarp();
        double pu = 0.0, bu = -1.0;
        int bi = 0x7fffffff;
        for (int i = lane; i < m1; i += 32) {
            double val = kernel_entry(K, P, r0 + i, c0 + jr);
            for (int l = 0; l < r; l++) val = __fma_rn(-coef[l], U[i + (size_t)l * m1], val);
            U[i + (size_t)r * m1] = val;
            pu += val * val;
            if (!((used[i >> 5] >> (i & 31)) & 1u)) {
                const double a = fabs(val);
                if (better(a, i, bu, bi, false)) { bu = a; bi = i; }
            }
        }
        const double nv2 = warp_sum(pv), nu2 = warp_sum(pu);
        warp_argmax_first(bu, bi);
        __syncwarp();  // every lane's U[., r] written
        // cross terms sum_l (u_r . U_l)(v_r . V_l), in l order
        double cross = 0.0;
        const double* ur = U + (size_t)r * m1;
        const double* vr = V + (size_t)r * m2;
        for (int l = 0; l < r; l++) {
            const double* ul = U + (size_t)l * m1;
            const double* vl = V + (size_t)l * m2;
            double a = 0.0, c = 0.0;
            for (int i = lane; i < m1; i += 32) a = __fma_rn(ur[i], ul[i], a);
            for (int j = lane; j < m2; j += 32) c = __fma_rn(vr[j], vl[j], c);
            cross += warp_sum(a) * warp_sum(c);
        }
        S2 = S2 + 2.0 * cross + nu2 * nv2;
        rank = r + 1;
        if (sqrt(nu2 * nv2) <= eps * sqrt(fabs(S2))) break;
        if (nused >= m1) break;
        if (bi == 0x7fffffff) break;
        ir = bi;
        __syncwarp();
    }
    if (lane == 0) {
        B.rank_out[e] = rank;
        if (B.s2_out) B.s2_out[e] = S2;
    }
}

// Write the FP64 scratch factors of one block into its final storage:
// U as tile slices (s_pad x r column-major, padding rows zero) and V^T as r rows
// of m2p entries (padding zero).
template <typename T>
__global__ void k_aca_compact(BlockGeom g, AcaBatch B, const int* tile_r0, const int* tile_s,
                              const int* tile_pstart, const int* tfirst, const int* tlast,
                              T* const* ptrU, T* const* ptrV)
{
    const int e = blockIdx.x;
    const int b = B.blocks[e];
    const int r0 = g.r0[b], m1 = g.m1[b], m2 = g.m2[b];
    const int r = B.rank_out[e];
    if (r == 0) return;
    const double* U = B.U + B.uoff[e];
    const double* V = B.V + B.voff[e];
    T* dU = ptrU[b];
    T* dV = ptrV[b];
    const int m2p = (m2 + 3) & ~3;
    for (long long idx = threadIdx.x; idx < (long long)r * m2p; idx += blockDim.x) {
        int l = (int)(idx / m2p), j = (int)(idx % m2p);
        dV[idx] = j < m2 ? (T)V[j + (size_t)l * m2] : (T)0;
    }
    const int p0 = tile_pstart[tfirst[b]];
    for (int t = tfirst[b]; t <= tlast[b]; t++) {
        int s = tile_s[t], sp = (s + 3) & ~3, tr = tile_r0[t] - r0;
        T* dst = dU + (size_t)(tile_pstart[t] - p0) * r;
        for (int idx = threadIdx.x; idx < sp * r; idx += blockDim.x) {
            int l = idx / sp, i = idx % sp;
            dst[idx] = i < s ? (T)U[(size_t)l * m1 + tr + i] : (T)0;
        }
    }
}

// ---------------------------------------------------------------------------
// Mixed-precision storage of the low-rank terms.
//
// The ACA terms u_l v_l^T of a block decay roughly geometrically.  A term whose
// rounding to a short format adds an error far below the ACA accuracy does not need
// FP32: with sigma_l = |u_l| |v_l| and S = |U V^T|_F, the terms l with
// sum_{l' >= l} sigma_l' <= TAU16 * S are stored in FP16 (unit roundoff 4.9e-4,
// error <~ 1e-3 TAU16 S) and those with a tail below TAU8 * S in FP8 e4m3 (error
// <~ 0.07 TAU8 S).  The FP8 count is rounded down to a multiple of 4 and the FP16
// count to a multiple of 2 (the remainder moves up a tier): short terms are stored
// interleaved in pairs (FP16) and quads (FP8), so that every 16-byte chunk of every
// tier holds four consecutive rows (U) or columns (V^T) of 1, 2 or 4 terms.  Each
// short term is scaled (u by su, v by sv: to [-1, 1] in FP16, to [-448, 448] in FP8)
// and su*sv is folded into t_l = v_l^T x.
// ---------------------------------------------------------------------------
static constexpr double TAU16 = 1e-4;
static constexpr double TAU8 = 1.5e-6;

struct TierOut {
    int* r32;          // per batch entry: terms kept in FP32
    int* r16;          // terms in FP16 (the rest, up to the rank, in FP8)
    const long long* soff;  // per batch entry: offset into the scale arrays
    float* su;         // per term: scale of u_l
    float* sv;         // per term: scale of v_l
};

__global__ void __launch_bounds__(256) k_aca_tiers(BlockGeom g, AcaBatch B, TierOut T)
{
    __shared__ double sig[ACA_KMAX];
    __shared__ double mu[ACA_KMAX];
    __shared__ double mv[ACA_KMAX];
    const int e = blockIdx.x;
    const int b = B.blocks[e];
    const int m1 = g.m1[b], m2 = g.m2[b];
    const int r = B.rank_out[e];
    const double* U = B.U + B.uoff[e];
    const double* V = B.V + B.voff[e];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int l = warp; l < r; l += 8) {
        double su = 0.0, mx_u = 0.0, sv = 0.0, mx_v = 0.0;
        for (int i = lane; i < m1; i += 32) {
            double u = U[(size_t)l * m1 + i];
            su = fma(u, u, su);
            mx_u = fmax(mx_u, fabs(u));
        }
        for (int j = lane; j < m2; j += 32) {
            double v = V[(size_t)l * m2 + j];
            sv = fma(v, v, sv);
            mx_v = fmax(mx_v, fabs(v));
        }
        for (int o = 16; o > 0; o >>= 1) {
            su += __shfl_xor_sync(0xffffffffu, su, o);
            sv += __shfl_xor_sync(0xffffffffu, sv, o);
            mx_u = fmax(mx_u, __shfl_xor_sync(0xffffffffu, mx_u, o));
            mx_v = fmax(mx_v, __shfl_xor_sync(0xffffffffu, mx_v, o));
        }
        if (lane == 0) {
            sig[l] = sqrt(su) * sqrt(sv);
            mu[l] = mx_u;
            mv[l] = mx_v;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double S = sqrt(fmax(B.s2_out[e], 0.0));
        int s16 = r, s8 = r;
        double tail = 0.0;
        for (int l = r - 1; l >= 0; l--) {
            tail += sig[l];
            if (tail <= TAU16 * S) s16 = l;
            if (tail <= TAU8 * S) s8 = l;
        }
        if (s8 < s16) s8 = s16;
        s8 = r - ((r - s8) & ~3);          // FP8 terms: a multiple of 4
        s16 = s8 - ((s8 - s16) & ~1);      // FP16 terms: a multiple of 2
        T.r32[e] = s16;
        T.r16[e] = s8 - s16;
        const long long so = T.soff[e];
        for (int l = 0; l < r; l++) {
            float a = 1.0f, c = 1.0f;
            if (l >= s8) {
                a = (float)(mu[l] / 448.0);
                c = (float)(mv[l] / 448.0);
            } else if (l >= s16) {
                a = (float)mu[l];
                c = (float)mv[l];
            }
            if (!(a > 0.0f)) a = 1.0f;
            if (!(c > 0.0f)) c = 1.0f;
            T.su[so + l] = a;
            T.sv[so + l] = c;
        }
    }
}

// Mixed storage of one block (m2p = m2 rounded up to 4, s_pad = tile rows rounded up
// to 4).  V^T: r32 FP32 rows of m2p; r16/2 FP16 pair rows, element (j, t) of pair g
// at half index (g m2p + j) 2 + t; r8/4 FP8 quad rows, element (j, t) of quad g at
// byte (g m2p + j) 4 + t; then r FP32 factors su_l sv_l (1 for FP32 terms).  U tile
// slices: s_pad x r32 FP32 column-major, then the pairs [g][i][2] in FP16 and the
// quads [g][i][4] in FP8; a slice takes s_pad * (4 r32 + 2 r16 + r8) bytes.
__global__ void __launch_bounds__(256)
k_aca_compact_mixed(BlockGeom g, AcaBatch B, TierOut T, const int* tile_r0, const int* tile_s,
                    const int* tile_pstart, const int* tfirst, const int* tlast, void* const* ptrU,
                    void* const* ptrV)
{
    const int e = blockIdx.x;
    const int b = B.blocks[e];
    const int r0 = g.r0[b], m1 = g.m1[b], m2 = g.m2[b];
    const int r = B.rank_out[e];
    if (r == 0) return;
    const int r32 = T.r32[e], r16 = T.r16[e], r8 = r - r32 - r16;
    const long long so = T.soff[e];
    const double* U = B.U + B.uoff[e];
    const double* V = B.V + B.voff[e];
    const int m2p = (m2 + 3) & ~3;
    // V^T
    float* v32 = static_cast<float*>(ptrV[b]);
    __half* v16 = reinterpret_cast<__half*>(v32 + (size_t)r32 * m2p);
    __nv_fp8_storage_t* v8 = reinterpret_cast<__nv_fp8_storage_t*>(v16 + (size_t)r16 * m2p);
    float* scal = reinterpret_cast<float*>(v8 + (size_t)r8 * m2p);
    for (long long idx = threadIdx.x; idx < (long long)r32 * m2p; idx += blockDim.x) {
        const int l = (int)(idx / m2p), j = (int)(idx % m2p);
        v32[idx] = j < m2 ? (float)V[j + (size_t)l * m2] : 0.0f;
    }
    for (long long idx = threadIdx.x; idx < (long long)r16 * m2p; idx += blockDim.x) {
        const int t = (int)(idx & 1), j = (int)((idx >> 1) % m2p), gp = (int)((idx >> 1) / m2p);
        const int l = r32 + 2 * gp + t;
        const float v = j < m2 ? (float)(V[j + (size_t)l * m2] / (double)T.sv[so + l]) : 0.0f;
        v16[idx] = __float2half_rn(v);
    }
    for (long long idx = threadIdx.x; idx < (long long)r8 * m2p; idx += blockDim.x) {
        const int t = (int)(idx & 3), j = (int)((idx >> 2) % m2p), gq = (int)((idx >> 2) / m2p);
        const int l = r32 + r16 + 4 * gq + t;
        const float v = j < m2 ? (float)(V[j + (size_t)l * m2] / (double)T.sv[so + l]) : 0.0f;
        v8[idx] = __nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
    }
    for (int l = threadIdx.x; l < r; l += blockDim.x) scal[l] = T.su[so + l] * T.sv[so + l];
    // U tile slices
    const int bpr = 4 * r32 + 2 * r16 + r8;
    const int p0 = tile_pstart[tfirst[b]];
    char* ubase = static_cast<char*>(ptrU[b]);
    for (int t = tfirst[b]; t <= tlast[b]; t++) {
        const int s = tile_s[t], sp = (s + 3) & ~3, tr = tile_r0[t] - r0;
        char* slice = ubase + (size_t)(tile_pstart[t] - p0) * bpr;
        float* u32 = reinterpret_cast<float*>(slice);
        __half* u16 = reinterpret_cast<__half*>(slice + (size_t)sp * 4 * r32);
        __nv_fp8_storage_t* u8 = reinterpret_cast<__nv_fp8_storage_t*>(slice + (size_t)sp * (4 * r32 + 2 * r16));
        for (int idx = threadIdx.x; idx < sp * r32; idx += blockDim.x) {
            const int l = idx / sp, i = idx % sp;
            u32[idx] = i < s ? (float)U[(size_t)l * m1 + tr + i] : 0.0f;
        }
        for (int idx = threadIdx.x; idx < sp * r16; idx += blockDim.x) {
            const int q = idx & 1, i = (idx >> 1) % sp, gp = (idx >> 1) / sp;
            const int l = r32 + 2 * gp + q;
            const float u = i < s ? (float)(U[(size_t)l * m1 + tr + i] / (double)T.su[so + l]) : 0.0f;
            u16[idx] = __float2half_rn(u);
        }
        for (int idx = threadIdx.x; idx < sp * r8; idx += blockDim.x) {
            const int q = idx & 3, i = (idx >> 2) % sp, gq = (idx >> 2) / sp;
            const int l = r32 + r16 + 4 * gq + q;
            const float u = i < s ? (float)(U[(size_t)l * m1 + tr + i] / (double)T.su[so + l]) : 0.0f;
            u8[idx] = __nv_cvt_float_to_fp8(u, __NV_SATFINITE, __NV_E4M3);
        }
    }
}

void free_far(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    free_tc(h);
    for (void* p : h->far_chunks) cudaFree(p);
    h->far_chunks.clear();
    h->far_chunk_bytes.clear();
    dfree(h->rank, s);
    dfree(h->rank_off, s);
    dfree(h->ptrU, s);
    dfree(h->ptrV, s);
    dfree(h->tbuf, s);
    dfree(h->far_list, s);
    dfree(h->tier32, s);
    dfree(h->tier16, s);
    h->h_r32.clear();
    h->h_r16.clear();
    h->far_alg_u = h->far_alg_v = 0;
    h->nfar_list = 0;
    h->far_prec = -1;
    h->desc_near_mode = -1;
    h->rank_total = h->far_entries = h->far_rows = h->far_stored = 0;
    h->max_rank = 0;
    h->h_rank.clear();
}

hmg_status run_aca(hmg_matrix* h, int k, double eps, int precision)
{
    cudaStream_t s = h->stream;
    hmg_status st = HMG_OK;
    if (k < 1) { set_error("ACA rank bound k must be >= 1 (got %d)", k); return HMG_ERR_INVALID; }
    if (k > ACA_KMAX) {
        set_error("ACA rank bound k=%d exceeds the engine's limit %d", k, ACA_KMAX);
        return HMG_ERR_UNSUPPORTED;
    }
    const bool mixed = precision == HMG_PREC_MIXED;
    if (mixed && !(eps > 0.0)) {
        set_error("mixed-precision factors need the adaptive ACA (eps > 0)");
        return HMG_ERR_INVALID;
    }
    free_far(h);
    const int nb = h->nblocks;
    const size_t esz = precision == HMG_PREC_FP64 ? 8 : 4;
    std::vector<int> rank(nb, 0), r32v(nb, 0), r16v(nb, 0);
    std::vector<void*> pU(nb, nullptr), pV(nb, nullptr);
    long long alg_u = 0, alg_v = 0;
    if ((st = dalloc((int**)&h->rank, (size_t)nb, s)) ||
        (st = dalloc((long long**)&h->rank_off, (size_t)nb + 1, s)) ||
        (st = dalloc((void***)&h->ptrU, (size_t)nb, s)) ||
        (st = dalloc((void***)&h->ptrV, (size_t)nb, s)) ||
        (st = dalloc(&h->tier32, (size_t)nb, s)) || (st = dalloc(&h->tier16, (size_t)nb, s)))
        return st;

    // batches of admissible blocks whose FP64 scratch fits the budget
    size_t free_b = 0, total_b = 0;
    HMG_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    size_t budget = free_b / 4;
    if (budget > ((size_t)16 << 30)) budget = (size_t)16 << 30;
    if (budget < ((size_t)64 << 20)) budget = (size_t)64 << 20;

    BlockGeom g{h->blk_r0, h->blk_m1, h->blk_c0, h->blk_m2, h->blk_param};
    PointsView P{};
    for (int d = 0; d < h->dim; d++) {
        P.c1[d] = h->zpts[0] + (size_t)d * h->n[0];
        P.c2[d] = h->zpts[1] + (size_t)d * h->n[1];
    }
    P.n1 = h->n[0];
    P.n2 = h->n[1];

    // Scratch of the batches, grown to the largest batch and reused across batches: the
    // stream-ordered pool hands freed memory back at every synchronisation, so
    // allocating it per batch would map gigabytes afresh for each one.
    int* d_idx = nullptr;
    long long *d_uo = nullptr, *d_vo = nullptr, *d_so = nullptr;
    double *dU = nullptr, *dV = nullptr, *d_s2 = nullptr;
    int *d_rank = nullptr, *d_r32 = nullptr, *d_r16 = nullptr, *d_list = nullptr;
    float *d_su = nullptr, *d_sv = nullptr;
    size_t cap_ne = 0, cap_u = 0, cap_v = 0, cap_sc = 0;
    auto free_batch = [&]() {
        dfree(d_idx, s); dfree(d_uo, s); dfree(d_vo, s); dfree(dU, s); dfree(dV, s);
        dfree(d_rank, s); dfree(d_s2, s); dfree(d_so, s); dfree(d_r32, s); dfree(d_r16, s);
        dfree(d_su, s); dfree(d_sv, s); dfree(d_list, s);
        cap_ne = cap_u = cap_v = cap_sc = 0;
    };
    int bstart = h->ndense;
    while (bstart < nb) {
        std::vector<int> idx;
        std::vector<long long> uo, vo;
        long long us = 0, vs = 0;
        int maxm1 = 1;
        int b = bstart;
        for (; b < nb; b++) {
            int m1 = h->h_m1[b], m2 = h->h_m2[b];
            int kb = std::min(k, std::min(m1, m2));
            long long need = ((long long)m1 + m2) * kb * 8;
            if (!idx.empty() && (us + vs) * 8 + need > (long long)budget) break;
            idx.push_back(b);
            uo.push_back(us);
            vo.push_back(vs);
            us += (long long)m1 * kb;
            vs += (long long)m2 * kb;
            maxm1 = std::max(maxm1, m1);
        }
        bstart = b;
        int ne = (int)idx.size();
        std::vector<long long> so(ne);
        long long nscale = 0;
        for (int e = 0; e < ne; e++) {
            so[e] = nscale;
            nscale += std::min(k, std::min(h->h_m1[idx[e]], h->h_m2[idx[e]]));
        }
        if ((size_t)ne > cap_ne) {
            dfree(d_idx, s); dfree(d_uo, s); dfree(d_vo, s); dfree(d_rank, s); dfree(d_s2, s);
            dfree(d_so, s); dfree(d_r32, s); dfree(d_r16, s); dfree(d_list, s);
            cap_ne = (size_t)ne;
            if ((st = dalloc(&d_idx, cap_ne, s)) || (st = dalloc(&d_uo, cap_ne, s)) || (st = dalloc(&d_vo, cap_ne, s)) ||
                (st = dalloc(&d_rank, cap_ne, s)) || (st = dalloc(&d_s2, cap_ne, s)) || (st = dalloc(&d_list, cap_ne, s)) ||
                (mixed && ((st = dalloc(&d_so, cap_ne, s)) || (st = dalloc(&d_r32, cap_ne, s)) ||
                           (st = dalloc(&d_r16, cap_ne, s))))) {
                free_batch();
                return st;
            }
        }
        if ((size_t)us > cap_u) {
            dfree(dU, s);
            cap_u = (size_t)us;
            if ((st = dalloc(&dU, cap_u, s))) {
                free_batch();
                return st;
            }
        }
        if ((size_t)vs > cap_v) {
            dfree(dV, s);
            cap_v = (size_t)vs;
            if ((st = dalloc(&dV, cap_v, s))) {
                free_batch();
                return st;
            }
        }
        if (mixed && (size_t)nscale > cap_sc) {
            dfree(d_su, s);
            dfree(d_sv, s);
            cap_sc = (size_t)nscale;
            if ((st = dalloc(&d_su, cap_sc, s)) || (st = dalloc(&d_sv, cap_sc, s))) {
                free_batch();
                return st;
            }
        }
        HMG_CUDA_TRY(cudaMemcpyAsync(d_idx, idx.data(), sizeof(int) * ne, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(d_uo, uo.data(), sizeof(long long) * ne, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(d_vo, vo.data(), sizeof(long long) * ne, cudaMemcpyHostToDevice, s));
        if (mixed) HMG_CUDA_TRY(cudaMemcpyAsync(d_so, so.data(), sizeof(long long) * ne, cudaMemcpyHostToDevice, s));
        AcaBatch B{d_idx, d_uo, d_vo, dU, dV, d_rank, d_s2};
        TierOut T{d_r32, d_r16, d_so, d_su, d_sv};
        size_t dyn = eps > 0.0 ? (size_t)((maxm1 + 31) / 32) * 4 : 0;
        if (dyn > 200 * 1024) {
            set_error("block with %d rows exceeds the adaptive ACA's row-mask capacity", maxm1);
            free_batch();
            return HMG_ERR_UNSUPPORTED;
        }
        if (dyn > 48 * 1024)
            HMG_CUDA_TRY(cudaFuncSetAttribute(k_aca, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)dyn));
        if (eps > 0.0) {
            // adaptive mode: small blocks one warp each, the others one CTA each
            std::vector<int> small, large;
            for (int e = 0; e < ne; e++) {
                const int bb = idx[e];
                ((h->h_m1[bb] <= ACA_WSMALL && h->h_m2[bb] <= ACA_WSMALL) ? small : large).push_back(e);
            }
            if (!small.empty())
                HMG_CUDA_TRY(cudaMemcpyAsync(d_list, small.data(), sizeof(int) * small.size(), cudaMemcpyHostToDevice, s));
            if (!large.empty())
                HMG_CUDA_TRY(cudaMemcpyAsync(d_list + small.size(), large.data(), sizeof(int) * large.size(),
                                             cudaMemcpyHostToDevice, s));
            if (!small.empty()) {
                const int ns = (int)small.size();
                k_aca_warp<<<ceil_div(ns, ACA_WPC), ACA_WPC * 32, 0, s>>>(g, h->kspec, P, B, k, eps, d_list, ns);
                HMG_LAUNCH_CHECK();
            }
            if (!large.empty()) {
                k_aca<<<(unsigned)large.size(), ACA_THREADS, dyn, s>>>(g, h->kspec, P, B, k, eps, d_list + small.size());
                HMG_LAUNCH_CHECK();
            }
            HMG_CUDA_TRY(cudaStreamSynchronize(s));  // the host vectors go out of scope
        } else {
            k_aca<<<ne, ACA_THREADS, dyn, s>>>(g, h->kspec, P, B, k, eps, nullptr);
            HMG_LAUNCH_CHECK();
        }
        if (mixed) {
            k_aca_tiers<<<ne, 256, 0, s>>>(g, B, T);
            HMG_LAUNCH_CHECK();
        }
        std::vector<int> br(ne), b32(ne, 0), b16(ne, 0);
        HMG_CUDA_TRY(cudaMemcpyAsync(br.data(), d_rank, sizeof(int) * ne, cudaMemcpyDeviceToHost, s));
        if (mixed) {
            HMG_CUDA_TRY(cudaMemcpyAsync(b32.data(), d_r32, sizeof(int) * ne, cudaMemcpyDeviceToHost, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(b16.data(), d_r16, sizeof(int) * ne, cudaMemcpyDeviceToHost, s));
        }
        HMG_CUDA_TRY(cudaStreamSynchronize(s));
        // final storage of this batch
        long long bytes = 0;
        std::vector<long long> ofsU(ne), ofsV(ne);
        for (int e = 0; e < ne; e++) {
            int bb = idx[e], r = br[e];
            rank[bb] = r;
            const long long rows_p = h->h_tile_pstart[h->h_blk_tlast[bb] + 1] -
                                     h->h_tile_pstart[h->h_blk_tfirst[bb]];
            const long long m1 = h->h_m1[bb], m2 = h->h_m2[bb];
            ofsU[e] = bytes;
            if (mixed) {
                const int r32 = b32[e], r16 = b16[e], r8 = r - r32 - r16;
                r32v[bb] = r32;
                r16v[bb] = r16;
                const long long bpr = 4 * r32 + 2 * r16 + r8;
                bytes += rows_p * bpr;
                bytes = (bytes + 255) & ~255ll;
                ofsV[e] = bytes;
                bytes += ((m2 + 3) & ~3) * bpr + 4ll * r;
                alg_u += m1 * (4ll * r32 + 2ll * r16 + r8);
                alg_v += m2 * (4ll * r32 + 2ll * r16 + r8);
            } else {
                r32v[bb] = r;
                bytes += rows_p * r * (long long)esz;
                bytes = (bytes + 255) & ~255ll;
                ofsV[e] = bytes;
                bytes += (long long)r * ((m2 + 3) & ~3) * (long long)esz;
                alg_u += m1 * r * (long long)esz;
                alg_v += m2 * r * (long long)esz;
            }
            bytes = (bytes + 255) & ~255ll;
        }
        char* chunk = nullptr;
        if (bytes > 0) {
            cudaError_t ce = cudaMalloc((void**)&chunk, (size_t)bytes);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                set_error("allocating %lld bytes of low-rank factors failed: %s", bytes,
                          cudaGetErrorString(ce));
                return ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
            }
            h->far_chunks.push_back(chunk);
            h->far_chunk_bytes.push_back((size_t)bytes);
            h->far_stored += bytes;
            for (int e = 0; e < ne; e++) {
                pU[idx[e]] = chunk + ofsU[e];
                pV[idx[e]] = chunk + ofsV[e];
            }
            // the batch is a contiguous block range
            HMG_CUDA_TRY(cudaMemcpyAsync(h->ptrU + idx[0], pU.data() + idx[0], sizeof(void*) * ne,
                                         cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->ptrV + idx[0], pV.data() + idx[0], sizeof(void*) * ne,
                                         cudaMemcpyHostToDevice, s));
            if (mixed)
                k_aca_compact_mixed<<<ne, 256, 0, s>>>(g, B, T, h->tile_r0, h->tile_s, h->tile_pstart,
                                                       h->blk_tfirst, h->blk_tlast, h->ptrU, h->ptrV);
            else if (precision == HMG_PREC_FP64)
                k_aca_compact<double><<<ne, 256, 0, s>>>(g, B, h->tile_r0, h->tile_s, h->tile_pstart,
                                                         h->blk_tfirst, h->blk_tlast,
                                                         (double* const*)h->ptrU, (double* const*)h->ptrV);
            else
                k_aca_compact<float><<<ne, 256, 0, s>>>(g, B, h->tile_r0, h->tile_s, h->tile_pstart,
                                                        h->blk_tfirst, h->blk_tlast,
                                                        (float* const*)h->ptrU, (float* const*)h->ptrV);
            HMG_LAUNCH_CHECK();
        }
        HMG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    free_batch();

    // ranks and their offsets
    std::vector<long long> roff(nb + 1, 0);
    h->far_entries = h->far_rows = 0;
    h->max_rank = 0;
    for (int b = 0; b < nb; b++) {
        roff[b + 1] = roff[b] + rank[b];
        if (h->h_type[b] == HMG_WT_ACA) {
            h->far_entries += (long long)(h->h_m1[b] + h->h_m2[b]) * rank[b];
            h->far_rows += h->h_m1[b] + h->h_m2[b];
            h->max_rank = std::max(h->max_rank, rank[b]);
        }
    }
    h->rank_total = roff[nb];
    HMG_CUDA_TRY(cudaMemcpyAsync(h->rank, rank.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(h->tier32, r32v.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(h->tier16, r16v.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
    h->h_r32 = r32v;
    h->h_r16 = r16v;
    h->far_alg_u = alg_u;
    h->far_alg_v = alg_v;
    HMG_CUDA_TRY(cudaMemcpyAsync(h->rank_off, roff.data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice, s));
    // padded and zeroed: the streaming product copies 16-byte-aligned supersets of t_b
    if ((st = dalloc((char**)&h->tbuf, (size_t)(h->rank_total + 32) * 8, s))) return st;
    HMG_CUDA_TRY(cudaMemsetAsync(h->tbuf, 0, (size_t)(h->rank_total + 32) * 8, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    h->h_rank = rank;
    h->far_prec = precision;
    h->aca_k = k;
    h->aca_eps = eps;
    return HMG_OK;
}

}  // namespace hmg
