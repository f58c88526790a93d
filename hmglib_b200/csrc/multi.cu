// multi.cu -- H-matvec with several right-hand sides, Y = H X (1 <= nrhs <= 32).
//
// The reference multiplies one vector per call (apply_h_matrix_mvp, hmglib.cu:271-286);
// a caller with several vectors pays the whole stored H-matrix once per vector.  Here
// the factors and the near field are read once for all vectors: bytes per product are
// those of one single-vector product plus 8 (N1 + N2) per vector, and each stored
// value feeds nrhs multiply-adds.
//
// X (caller order, column-major, FP64) is gathered into Z order as R values per
// point (R = nrhs rounded up to a power of two), in the storage's arithmetic type.
//   K1m  t_b = V_b^T X_b for every admissible block: a warp per K1 piece; its lanes
//        are G = 32/R groups of R lanes (one lane per vector), the groups stride over
//        the row's 16-byte chunks, 4 rows at a time; the groups' partials are summed
//        by a fixed xor butterfly.
//   K2m  one CTA per row tile, one warp per 16 rows: lane (g, j) owns 16/G rows of
//        vector j and walks every pair of the tile, FP32/FP64 products per pair added
//        in FP64; Y written once per row and vector, in the caller's order.
// Deterministic (fixed summation orders, no atomics).  FP32 and FP64 storage with a
// stored near field; mixed storage and on-the-fly near fields use one product per
// vector.
#include <algorithm>

#include "hmg_matrix.cuh"
#include "stream.cuh"

namespace hmg {

template <typename T>
__global__ void k_gather_multi(const double* X, int ldx, int nrhs, const int* perm2, int n, int lgR, T* xm)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= ((long long)n << lgR)) return;
    const int i = (int)(idx >> lgR), j = (int)(idx & ((1 << lgR) - 1));
    xm[idx] = j < nrhs ? (T)X[perm2[i] + (size_t)j * ldx] : (T)0;
}

template <typename S> struct Lanes;
template <> struct Lanes<float> {
    static constexpr int NC = 4;
    __device__ static void get(const uint4& u, float* o)
    {
        o[0] = __uint_as_float(u.x); o[1] = __uint_as_float(u.y);
        o[2] = __uint_as_float(u.z); o[3] = __uint_as_float(u.w);
    }
};
template <> struct Lanes<double> {
    static constexpr int NC = 2;
    __device__ static void get(const uint4& u, double* o)
    {
        o[0] = __hiloint2double((int)u.y, (int)u.x);
        o[1] = __hiloint2double((int)u.w, (int)u.z);
    }
};

template <typename S, int R>
__global__ void __launch_bounds__(256) k_vtx_multi(const K1Desc* __restrict__ descs, int n,
                                                   const S* __restrict__ xm, S* __restrict__ tm)
{
    constexpr int G = 32 / R, NC = Lanes<S>::NC;
    const int lane = threadIdx.x & 31, g = lane / R, j = lane % R;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int u = gw; u < n; u += nw) {
        const K1Desc d = descs[u];
        const int cpr = d.row_bytes >> 4;
        const char* vb = static_cast<const char*>(d.v);
        for (int row = 0; row < d.nrows; row += 4) {
            S acc[4] = {(S)0, (S)0, (S)0, (S)0};
            for (int c = g; c < cpr; c += G) {
                uint4 raw[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    raw[k] = make_uint4(0u, 0u, 0u, 0u);
                    if (row + k < d.nrows) raw[k] = ld_stream(vb + (size_t)(row + k) * d.row_bytes + (size_t)c * 16);
                }
                S xv[NC];
#pragma unroll
                for (int q = 0; q < NC; q++) {
                    const int e = c * NC + q;
                    xv[q] = e < d.m2 ? xm[(size_t)(d.c0 + e) * R + j] : (S)0;
                }
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    S f[NC];
                    Lanes<S>::get(raw[k], f);
#pragma unroll
                    for (int q = 0; q < NC; q++) acc[k] = fma(f[q], xv[q], acc[k]);
                }
            }
#pragma unroll
            for (int o = R; o < 32; o <<= 1)
#pragma unroll
                for (int k = 0; k < 4; k++) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
            if (g == 0)
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (row + k < d.nrows) tm[(size_t)(d.tout + row + k) * R + j] = acc[k];
        }
    }
}

// RL consecutive slice values (rows r0..r0+RL-1 of one column) with 16-byte loads;
// rows at or past sp are not read (their value is 0).
template <typename S, int RL>
__device__ __forceinline__ void load_rows(const S* p, int r0, int sp, S* o)
{
    constexpr int NC = Lanes<S>::NC;
    if constexpr (RL >= NC) {
#pragma unroll
        for (int v = 0; v < RL / NC; v++) {
            uint4 raw = make_uint4(0u, 0u, 0u, 0u);
            if (r0 + v * NC < sp) raw = ld_stream(p + v * NC);
            Lanes<S>::get(raw, o + v * NC);
        }
    } else {
#pragma unroll
        for (int q = 0; q < RL; q++) o[q] = r0 + q < sp ? p[q] : (S)0;
    }
}

template <typename S, int R>
__global__ void __launch_bounds__(256) k_tile_multi(const PairDesc* __restrict__ desc, const int* tile_pair_start,
                                                    const int* tile_r0, const int* tile_s, const int* perm1,
                                                    const S* __restrict__ xm, const S* __restrict__ tm,
                                                    const char* tbase, int nrhs, double* Y, int ldy)
{
    constexpr int G = 32 / R, RL = 16 / G;
    const int t = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / R, j = lane % R;
    const int s = tile_s[t], sp = (s + 3) & ~3, tr0 = tile_r0[t];
    if (warp * 16 >= sp) return;
    const int r0 = warp * 16 + g * RL;
    double acc64[RL];
#pragma unroll
    for (int q = 0; q < RL; q++) acc64[q] = 0.0;
    const int pend = tile_pair_start[t + 1];
    for (int p = tile_pair_start[t]; p < pend; p++) {
        const PairDesc d = desc[p];
        if (r0 >= sp) continue;
        const S* src = d.kind == PAIR_STORED
                           ? xm + (size_t)d.c0 * R + j
                           : tm + (size_t)((static_cast<const char*>(d.w) - tbase) / (long long)sizeof(S)) * R + j;
        const S* base = static_cast<const S*>(d.data) + r0;
        S acc[RL];
#pragma unroll
        for (int q = 0; q < RL; q++) acc[q] = (S)0;
        for (int k = 0; k < d.ncol; k++) {
            const S wk = src[(size_t)k * R];
            S u[RL];
            load_rows<S, RL>(base + (size_t)k * sp, r0, sp, u);
#pragma unroll
            for (int q = 0; q < RL; q++) acc[q] = fma(u[q], wk, acc[q]);
        }
#pragma unroll
        for (int q = 0; q < RL; q++) acc64[q] += (double)acc[q];
    }
    if (j < nrhs)
#pragma unroll
        for (int q = 0; q < RL; q++)
            if (r0 + q < s) Y[perm1[tr0 + r0 + q] + (size_t)j * ldy] = acc64[q];
}

template <typename S, int R>
static hmg_status launch_multi(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy, S* xm, S* tm)
{
    cudaStream_t s = h->stream;
    constexpr int LGR = R == 32 ? 5 : (R == 16 ? 4 : (R == 8 ? 3 : (R == 4 ? 2 : 1)));
    k_gather_multi<S><<<ceil_div((long long)h->n[1] * R, 256), 256, 0, s>>>(X, ldx, nrhs, h->perm[1], h->n[1],
                                                                            LGR, xm);
    HMG_LAUNCH_CHECK();
    const int n0 = h->k1_count[0];
    if (n0 > 0) {
        k_vtx_multi<S, R><<<std::min(ceil_div(n0, 8), 148 * 8), 256, 0, s>>>(
            static_cast<const K1Desc*>(h->k1_units), n0, xm, tm);
        HMG_LAUNCH_CHECK();
    }
    if (h->ntiles > 0) {
        k_tile_multi<S, R><<<h->ntiles, 256, 0, s>>>(static_cast<const PairDesc*>(h->pair_desc),
                                                     h->tile_pair_start, h->tile_r0, h->tile_s, h->perm[0], xm, tm,
                                                     static_cast<const char*>(h->tbuf), nrhs, Y, ldy);
        HMG_LAUNCH_CHECK();
    }
    return HMG_OK;
}

template <typename S>
static hmg_status multi_typed(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    int R = 2;
    while (R < nrhs) R <<= 1;
    // descriptors built for this element type: t_b of block b starts at rank_off[b]
    if ((st = ensure_desc(h, (int)sizeof(S)))) return st;
    S* xm = nullptr;
    S* tm = nullptr;
    if ((st = dalloc(&xm, (size_t)h->n[1] * R, s)) || (st = dalloc(&tm, (size_t)(h->rank_total + 1) * R, s))) {
        dfree(xm, s);
        return st;
    }
    switch (R) {
    case 2: st = launch_multi<S, 2>(h, nrhs, X, ldx, Y, ldy, xm, tm); break;
    case 4: st = launch_multi<S, 4>(h, nrhs, X, ldx, Y, ldy, xm, tm); break;
    case 8: st = launch_multi<S, 8>(h, nrhs, X, ldx, Y, ldy, xm, tm); break;
    case 16: st = launch_multi<S, 16>(h, nrhs, X, ldx, Y, ldy, xm, tm); break;
    default: st = launch_multi<S, 32>(h, nrhs, X, ldx, Y, ldy, xm, tm); break;
    }
    dfree(xm, s);
    dfree(tm, s);
    return st;
}

hmg_status matvec_multi(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    const bool per_vector = nrhs == 1 || h->far_prec == HMG_PREC_MIXED || h->near_mode != HMG_NEAR_STORED ||
                            (h->naca > 0 && h->near_prec != h->far_prec) || h->arith_prec == HMG_PREC_FP64;
    if (per_vector) {
        for (int j = 0; j < nrhs; j++) {
            hmg_status st = matvec_device(h, X + (size_t)j * ldx, Y + (size_t)j * ldy);
            if (st) return st;
        }
        return HMG_OK;
    }
    const bool fp64 = h->naca > 0 ? h->far_prec == HMG_PREC_FP64 : h->near_prec == HMG_PREC_FP64;
    return fp64 ? multi_typed<double>(h, nrhs, X, ldx, Y, ldy) : multi_typed<float>(h, nrhs, X, ldx, Y, ldy);
}

}  // namespace hmg
