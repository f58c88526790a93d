// matvec.cu -- near-field storage and the H-matvec.
//
// The reference multiplies per "batch": it rebuilds index maps with Thrust on every
// call, gathers x per block, runs MAGMA dgemv_vbatched for dense blocks and twice
// for U (V^T x), and adds every block's result into y with double-CAS atomics
// (linear_algebra.cu:1152-1181, 1429-1591, 2817-3137, 4292-4379).
//
// Here one product is three kernels and no host work:
//   K0  x in Z order (and an FP32 copy);
//   K1  t_b = V_b^T x_b for all admissible blocks, a warp per row of V_b^T, work
//       split into pieces of at most ~64 KB so large blocks spread over many warps;
//   K2  one CTA per row tile: every dense block slice and every U_b slice touching
//       the tile is multiplied with x (dense) or t_b (low rank), FP32 products
//       summed per slice and accumulated in FP64 across slices, the CTA's warp
//       partials summed in a fixed order, and y written once, in the caller's
//       order.  No atomics: y is deterministic.
// Each stored byte is read exactly once per product (the HBM roofline's minimum).
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "hmg_matrix.cuh"
#include "stream.cuh"

namespace hmg {


// ---------------------------------------------------------------------------
// near-field fill (precompute_batched_dense_magma, linear_algebra.cu:3140-3342):
// one CTA per dense block, entries written tile slice by tile slice.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_fill_near(const int* blocks_r0, const int* blocks_c0, const int* blocks_m2,
                            const long long* near_off, const int* tfirst, const int* tlast,
                            const int* tile_r0, const int* tile_s, const int* tile_pstart,
                            KernelSpec K, PointsView P, const double* bparam, T* out)
{
    const int b = blockIdx.x;
    if (bparam) K.param = bparam[b];
    const int c0 = blocks_c0[b], m2 = blocks_m2[b];
    (void)blocks_r0;
    T* base = out + near_off[b];
    const int p0 = tile_pstart[tfirst[b]];
    for (int t = tfirst[b]; t <= tlast[b]; t++) {
        const int s = tile_s[t], sp = (s + 3) & ~3, tr = tile_r0[t];
        T* dst = base + (size_t)(tile_pstart[t] - p0) * m2;
        for (int idx = threadIdx.x; idx < sp * m2; idx += blockDim.x) {
            int i = idx % sp, j = idx / sp;
            dst[idx] = i < s ? (T)kernel_entry(K, P, tr + i, c0 + j) : (T)0;
        }
    }
}

void free_near(hmg_matrix* h)
{
    if (h->near_data) cudaFree(h->near_data);
    h->near_data = nullptr;
    dfree(h->near_off, h->stream);
    h->near_prec = -1;
    h->near_stored = 0;
    h->desc_near_mode = -1;
    if (h->near_mode == HMG_NEAR_STORED) h->near_mode = HMG_NEAR_ONTHEFLY;
    free_tc(h);  // its BF16 near slices are copies of this storage
}

static PointsView points_view(hmg_matrix* h)
{
    PointsView P{};
    for (int d = 0; d < h->dim; d++) {
        P.c1[d] = h->zpts[0] + (size_t)d * h->n[0];
        P.c2[d] = h->zpts[1] + (size_t)d * h->n[1];
    }
    P.n1 = h->n[0];
    P.n2 = h->n[1];
    return P;
}

hmg_status fill_near(hmg_matrix* h, int precision)
{
    cudaStream_t s = h->stream;
    free_near(h);
    const int nd = h->ndense;
    const size_t esz = precision == HMG_PREC_FP64 ? 8 : 4;
    std::vector<long long> off(nd > 0 ? nd : 1, 0);
    long long tot = 0, entries = 0;
    for (int b = 0; b < nd; b++) {
        off[b] = tot;
        long long rows_p = h->h_tile_pstart[h->h_blk_tlast[b] + 1] - h->h_tile_pstart[h->h_blk_tfirst[b]];
        tot += rows_p * h->h_m2[b];
        entries += (long long)h->h_m1[b] * h->h_m2[b];
    }
    h->near_entries = entries;
    hmg_status st = dalloc(&h->near_off, (size_t)(nd > 0 ? nd : 1), s);
    if (st) return st;
    if (nd > 0) {
        cudaError_t ce = cudaMalloc(&h->near_data, (size_t)tot * esz);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            h->near_data = nullptr;
            set_error("allocating %lld bytes of near-field blocks failed: %s", tot * (long long)esz,
                      cudaGetErrorString(ce));
            return ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
        }
        HMG_CUDA_TRY(cudaMemcpyAsync(h->near_off, off.data(), sizeof(long long) * nd, cudaMemcpyHostToDevice, s));
        PointsView P = points_view(h);
        if (precision == HMG_PREC_FP64)
            k_fill_near<double><<<nd, 256, 0, s>>>(h->blk_r0, h->blk_c0, h->blk_m2, h->near_off,
                                                   h->blk_tfirst, h->blk_tlast, h->tile_r0, h->tile_s,
                                                   h->tile_pstart, h->kspec, P, h->blk_param, (double*)h->near_data);
        else
            k_fill_near<float><<<nd, 256, 0, s>>>(h->blk_r0, h->blk_c0, h->blk_m2, h->near_off,
                                                  h->blk_tfirst, h->blk_tlast, h->tile_r0, h->tile_s,
                                                  h->tile_pstart, h->kspec, P, h->blk_param, (float*)h->near_data);
        HMG_LAUNCH_CHECK();
    }
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    h->near_stored = tot;
    h->near_prec = precision;
    h->near_mode = HMG_NEAR_STORED;
    return HMG_OK;
}

// ---------------------------------------------------------------------------
// descriptors of the product (rebuilt when storage or modes change)
// ---------------------------------------------------------------------------
__global__ void k_build_desc(const int* tile_pair_start, int ntiles, const int* pair_block,
                             const int* tile_pstart, const int* blk_type, const int* blk_c0,
                             const int* blk_m2, const int* tfirst, const long long* near_off,
                             const void* near_data, int near_esz, int near_mode,
                             const int* rank, const long long* rank_off, void* const* ptrU,
                             const void* tbuf, int far_esz, const void* xs, int x_esz,
                             const int* tier32, const int* tier16, int mixed, PairDesc* desc)
// x_esz is the arithmetic element size: x and t_b are read in that type
{
    int t = blockIdx.x;
    if (t >= ntiles) return;
    int pt = tile_pstart[t];
    for (int p = tile_pair_start[t] + threadIdx.x; p < tile_pair_start[t + 1]; p += blockDim.x) {
        int b = pair_block[p];
        PairDesc d;
        int slice_row = pt - tile_pstart[tfirst[b]];
        d.c0 = blk_c0[b];
        d.pad = 0;
        if (blk_type[b] == HMG_WT_DENSE) {
            d.ncol = blk_m2[b];
            d.w = (const char*)xs + (size_t)blk_c0[b] * x_esz;
            if (near_mode == HMG_NEAR_STORED) {
                d.kind = PAIR_STORED;
                d.data = (const char*)near_data +
                         (size_t)(near_off[b] + (long long)slice_row * d.ncol) * near_esz;
            } else {
                d.kind = PAIR_ONTHEFLY;
                d.data = nullptr;
            }
        } else if (mixed) {
            // FP32 / FP16 / FP8 terms; a tile slice takes s_pad * bpr bytes
            const int r = rank[b], r32 = tier32[b], r16 = tier16[b], r8 = r - r32 - r16;
            const int bpr = 4 * r32 + 2 * r16 + r8;
            d.kind = PAIR_FAR_MIXED;
            d.ncol = r32;
            d.c0 = r16;
            d.pad = r8;
            d.w = (const char*)tbuf + (size_t)rank_off[b] * x_esz;
            d.data = (const char*)ptrU[b] + (size_t)slice_row * bpr;
        } else {
            d.kind = PAIR_FAR;
            d.ncol = rank[b];
            d.w = (const char*)tbuf + (size_t)rank_off[b] * x_esz;
            d.data = (const char*)ptrU[b] + (size_t)slice_row * d.ncol * far_esz;
        }
        desc[p] = d;
    }
}

__global__ void k_build_k1desc(const K1Unit* units, int n, const int* blk_c0, const int* blk_m2,
                               const int* rank, const int* tier32, const int* tier16, const long long* rank_off,
                               void* const* ptrV, int esz, int mixed, K1Desc* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const K1Unit un = units[i];
    const int b = un.b, m2 = blk_m2[b], r = rank[b];
    const int r32 = mixed ? tier32[b] : r, r16 = mixed ? tier16[b] : 0, r8 = r - r32 - r16;
    const size_t m2p = (m2 + 3) & ~3;
    const char* V = static_cast<const char*>(ptrV[b]);
    const size_t b32 = (size_t)r32 * m2p * esz, b16 = (size_t)r16 * m2p * 2;
    // rows of a piece: single terms (tier 0), interleaved pairs (FP16), quads (FP8)
    K1Desc d;
    if (un.tier == 0) {
        d.row_bytes = (int)(m2p * esz);
        d.v = V + (size_t)un.l0 * d.row_bytes;
        d.nrows = un.l1 - un.l0;
    } else if (un.tier == 1) {
        d.row_bytes = (int)(m2p * 4);
        d.v = V + b32 + (size_t)((un.l0 - r32) >> 1) * d.row_bytes;
        d.nrows = (un.l1 - un.l0) >> 1;
    } else {
        d.row_bytes = (int)(m2p * 4);
        d.v = V + b32 + b16 + (size_t)((un.l0 - r32 - r16) >> 2) * d.row_bytes;
        d.nrows = (un.l1 - un.l0) >> 2;
    }
    d.scal = un.tier == 0 ? nullptr
                          : reinterpret_cast<const float*>(V + b32 + b16 + (size_t)r8 * m2p) + un.l0;
    d.tout = rank_off[b] + un.l0;
    d.c0 = blk_c0[b];
    d.m2 = m2;
    d.pad[0] = d.pad[1] = 0;
    out[i] = d;
}

// K1 step shape per tier: rows per step R = 4 / (terms per row) so that a lane holds
// four term sums, and K1_NCH = 8 / R chunks per row, so that a lane has eight 16-byte
// loads in flight whatever the tier.
static constexpr int k1_nch(int tier) { return tier == 0 ? 2 : (tier == 1 ? 4 : 8); }

hmg_status ensure_desc(hmg_matrix* h, int elem)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    // dense-pair descriptors point into the x buffers: they must exist first
    if ((st = ensure_xs(h))) return st;
    if (!h->pair_desc) {
        PairDesc* d = nullptr;
        if ((st = dalloc(&d, (size_t)(h->npairs > 0 ? h->npairs : 1), s))) return st;
        h->pair_desc = d;
        h->desc_near_mode = -1;
    }
    if (h->desc_near_mode == h->near_mode && h->desc_near_prec == h->near_prec &&
        h->desc_far_prec == h->far_prec && h->desc_elem == elem)
        return HMG_OK;
    const void* xs = elem == 8 ? (const void*)h->xs64 : (const void*)h->xs32;
    int near_esz = h->near_prec == HMG_PREC_FP64 ? 8 : 4;
    int far_esz = h->far_prec == HMG_PREC_FP64 ? 8 : 4;
    if (h->ntiles > 0) {
        k_build_desc<<<h->ntiles, 128, 0, s>>>(
            h->tile_pair_start, h->ntiles, h->pair_block, h->tile_pstart, h->blk_type, h->blk_c0,
            h->blk_m2, h->blk_tfirst, h->near_off, h->near_data, near_esz, h->near_mode, h->rank,
            h->rank_off, h->ptrU, h->tbuf, far_esz, xs, elem, h->tier32, h->tier16,
            h->far_prec == HMG_PREC_MIXED ? 1 : 0, (PairDesc*)h->pair_desc);
        HMG_LAUNCH_CHECK();
    }
    // K1 pieces: terms of V_b^T of one storage tier, in runs of at most k1_piece_bytes
    // (64 KB unless hmg_autotune chose otherwise).  Each
    // piece gets the widest lane group 2^LG (LG 2..5) whose lanes still get k1_nch
    // chunks of a row each; pieces are ordered by tier, then by LG (one launch per
    // tier; a warp takes 32 / 2^LG pieces of one class at a time).
    dfree(h->k1_units, s);
    std::vector<K1Unit> units[3][4];
    const bool mixed = h->far_prec == HMG_PREC_MIXED;
    for (int b = h->ndense; b < h->nblocks; b++) {
        const int r = h->h_rank[b];
        if (r == 0) continue;
        const long long m2 = h->h_m2[b];
        const int r32 = mixed ? h->h_r32[b] : r, r16 = mixed ? h->h_r16[b] : 0;
        const int lo[3] = {0, r32, r32 + r16}, hi[3] = {r32, r32 + r16, r};
        // bytes of one piece row: a term (tier 0), a pair of FP16 or a quad of FP8 terms
        const long long rb[3] = {((m2 + 3) & ~3ll) * far_esz, ((m2 + 3) & ~3ll) * 4, ((m2 + 3) & ~3ll) * 4};
        const int tg[3] = {1, 2, 4};
        for (int tier = 0; tier < 3; tier++) {
            if (lo[tier] == hi[tier]) continue;
            const long long per_lane = rb[tier] / 16 / k1_nch(tier);  // chunks per lane at 1 lane
            int lg = 2;
            while (lg < 5 && (1ll << (lg + 1)) <= per_lane) lg++;
            const int per = (int)std::max(1ll, (long long)h->k1_piece_bytes / rb[tier]) * tg[tier];
            for (int l = lo[tier]; l < hi[tier]; l += per)
                units[tier][lg - 2].push_back({b, l, std::min(hi[tier], l + per), tier});
        }
    }
    std::vector<K1Unit> all;
    for (int tier = 0; tier < 3; tier++) {
        const int first = (int)all.size();
        int tasks = 0;
        for (int c = 0; c < 4; c++) {
            h->k1_piece_start[tier][c] = (int)all.size();
            h->k1_task_start[tier][c] = tasks;
            all.insert(all.end(), units[tier][c].begin(), units[tier][c].end());
            const int g = 32 >> (c + 2);
            tasks += ((int)units[tier][c].size() + g - 1) / g;
        }
        h->k1_piece_start[tier][4] = (int)all.size();
        h->k1_task_start[tier][4] = tasks;
        h->k1_count[tier] = (int)all.size() - first;
    }
    h->nk1 = (int)all.size();
    K1Desc* dd = nullptr;
    K1Unit* du = nullptr;
    if ((st = dalloc(&dd, all.size() > 0 ? all.size() : 1, s))) return st;
    h->k1_units = dd;
    if (!all.empty()) {
        if ((st = dalloc(&du, all.size(), s))) return st;
        HMG_CUDA_TRY(cudaMemcpyAsync(du, all.data(), sizeof(K1Unit) * all.size(), cudaMemcpyHostToDevice, s));
        k_build_k1desc<<<ceil_div(h->nk1, 256), 256, 0, s>>>(du, h->nk1, h->blk_c0, h->blk_m2, h->rank,
                                                            h->tier32, h->tier16, h->rank_off, h->ptrV,
                                                            far_esz, mixed ? 1 : 0, dd);
        HMG_LAUNCH_CHECK();
        dfree(du, s);
    }
    // the streaming V^T x kernel works on whole blocks
    dfree(h->far_list, s);
    std::vector<int> fl;
    for (int b = h->ndense; b < h->nblocks; b++)
        if (h->h_rank[b] > 0) fl.push_back(b);
    h->nfar_list = (int)fl.size();
    if ((st = dalloc(&h->far_list, fl.size() > 0 ? fl.size() : 1, s))) return st;
    if (!fl.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->far_list, fl.data(), sizeof(int) * fl.size(), cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    h->desc_near_mode = h->near_mode;
    h->desc_near_prec = h->near_prec;
    h->desc_far_prec = h->far_prec;
    h->desc_elem = elem;
    return HMG_OK;
}

// ---------------------------------------------------------------------------
// the product kernels
// ---------------------------------------------------------------------------
__global__ void k_gather_x(const double* x, const int* perm2, int n, double* xs64, float* xs32)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double v = x[perm2[j]];
    xs64[j] = v;
    xs32[j] = (float)v;
}

template <typename V4> __device__ __forceinline__ V4 ld_stream_as(const void* p)
{
    const uint4 u = ld_stream(p);
    return *reinterpret_cast<const V4*>(&u);
}

template <typename T> struct Vec;
template <> struct Vec<float> { typedef float4 type; static constexpr int N = 4; };
template <> struct Vec<double> { typedef double2 type; static constexpr int N = 2; };

__device__ __forceinline__ void vec_get(const float4& v, float* o) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
__device__ __forceinline__ void vec_get(const double2& v, double* o) { o[0] = v.x; o[1] = v.y; }

// 16 bytes of FP16 (8 values) or FP8 e4m3 (16 values) to floats
__device__ __forceinline__ void unpack16(const uint4& u, float* o)
{
    const __half2* h = reinterpret_cast<const __half2*>(&u);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float2 f = __half22float2(h[k]);
        o[2 * k] = f.x;
        o[2 * k + 1] = f.y;
    }
}

__device__ __forceinline__ float2 fp8x2_to_float2(unsigned short v)
{
    __half2_raw hr = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)v, __NV_E4M3);
    return __half22float2(*reinterpret_cast<const __half2*>(&hr));
}

__device__ __forceinline__ void unpack8(const uint4& u, float* o)
{
    const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float2 a = fp8x2_to_float2((unsigned short)(w[k] & 0xffffu));
        float2 b = fp8x2_to_float2((unsigned short)(w[k] >> 16));
        o[4 * k] = a.x; o[4 * k + 1] = a.y; o[4 * k + 2] = b.x; o[4 * k + 3] = b.y;
    }
}

// 16 bytes of one tier to values, [column][term]: FP32 4 x 1, FP64 2 x 1, FP16 pairs
// 4 x 2, FP8 e4m3 quads 4 x 4
template <typename T, int TIER> struct Chunk;
template <> struct Chunk<float, 0> {
    static constexpr int NC = 4, TG = 1;
    __device__ static void get(const uint4& u, float* o)
    {
        o[0] = __uint_as_float(u.x); o[1] = __uint_as_float(u.y);
        o[2] = __uint_as_float(u.z); o[3] = __uint_as_float(u.w);
    }
};
template <> struct Chunk<double, 0> {
    static constexpr int NC = 2, TG = 1;
    __device__ static void get(const uint4& u, double* o)
    {
        o[0] = __hiloint2double((int)u.y, (int)u.x);
        o[1] = __hiloint2double((int)u.w, (int)u.z);
    }
};
template <> struct Chunk<float, 1> {
    static constexpr int NC = 4, TG = 2;
    __device__ static void get(const uint4& u, float* o) { unpack16(u, o); }
};
template <> struct Chunk<float, 2> {
    static constexpr int NC = 4, TG = 4;
    __device__ static void get(const uint4& u, float* o) { unpack8(u, o); }
};

// K1: t_b[l] = s_l sum_j V_b^T[l][j] x[c0_b + j] over the pieces of one storage tier.
//
// A 16-byte chunk holds NC consecutive columns of TG terms (FP32: 4 x 1, FP64: 2 x 1,
// FP16 pairs: 4 x 2, FP8 quads: 4 x 4), so every tier is read with the same chunk
// loads and every x value loaded serves 4 terms of a lane.  A warp takes a task: up
// to 32 / LPR pieces of one lane-group class, one per group of LPR = 2^LG lanes, so
// that short pieces (the FP16/FP8 tails of small blocks) still keep 32 lanes x 8
// loads in flight.  Each group steps through its piece R rows (4 terms) at a time
// with NCH chunks per row per lane, then sums the four term partials over its lanes
// with a transposing butterfly in a fixed order: t is deterministic.
struct K1Classes {
    int piece_start[5];  // first piece of each class (LG = 2..5), then the end
    int task_start[5];   // first task of each class, then the task count
};

// Sum of the R partials of an LPR-lane group: a transposing butterfly (log2 R halving
// exchanges, then plain ones).  Afterwards lane `sub` holds the total of partial
// sub / (LPR / R); the summation order is fixed.
template <int R, int LPR, typename T>
__device__ __forceinline__ T rows_butterfly(T (&acc)[R], int sub)
{
    constexpr int LOGR = R == 8 ? 3 : (R == 4 ? 2 : 1);
#pragma unroll
    for (int st = 0; st < LOGR; st++) {
        const int h = (R / 2) >> st, o = (LPR / 2) >> st;
        const bool up = (sub & o) != 0;
#pragma unroll
        for (int i = 0; i < h; i++) {
            const T send = up ? acc[i] : acc[i + h];
            const T keep = up ? acc[i + h] : acc[i];
            acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    T a = acc[0];
#pragma unroll
    for (int o = LPR / (2 * R); o >= 1; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    return a;
}

// One task's share of a group: piece d (when `have`), group lanes `sub` of 2^LG.
template <typename S, typename T, int TIER, int LG>
__device__ __forceinline__ void vtx_group(const K1Desc& d, bool have, const T* __restrict__ xs,
                                          T* __restrict__ tbuf, int lane)
{
    typedef Chunk<S, TIER> C;
    constexpr int NC = C::NC, TG = C::TG;
    constexpr int R = 4 / TG, NCH = k1_nch(TIER);
    constexpr int LPR = 1 << LG;
    const int sub = lane & (LPR - 1);
    const int nrows = have ? d.nrows : 0;
    const int cpr = have ? (d.row_bytes >> 4) : 0;
    const char* vb = static_cast<const char*>(d.v);
    for (int row = 0; __any_sync(0xffffffffu, row < nrows); row += R) {
        T acc[4] = {(T)0, (T)0, (T)0, (T)0};
        for (int c = sub; c < cpr; c += NCH * LPR) {
            uint4 raw[NCH][R];
#pragma unroll
            for (int k = 0; k < R; k++) {
                const uint4* rp = reinterpret_cast<const uint4*>(vb + (size_t)(row + k) * d.row_bytes);
#pragma unroll
                for (int hh = 0; hh < NCH; hh++) {
                    raw[hh][k] = make_uint4(0u, 0u, 0u, 0u);
                    if (row + k < nrows && c + hh * LPR < cpr) raw[hh][k] = ld_stream(rp + c + hh * LPR);
                }
            }
#pragma unroll
            for (int hh = 0; hh < NCH; hh++) {
                T xv[NC];
                const int e0 = (c + hh * LPR) * NC;
#pragma unroll
                // the bound test also covers the chunks past the row that a step skips
                for (int q = 0; q < NC; q++) xv[q] = e0 + q < d.m2 ? xs[d.c0 + e0 + q] : (T)0;
#pragma unroll
                for (int k = 0; k < R; k++) {
                    S f[NC * TG];
                    C::get(raw[hh][k], f);
#pragma unroll
                    for (int q = 0; q < NC; q++)
#pragma unroll
                        for (int t = 0; t < TG; t++) acc[k * TG + t] = fma((T)f[q * TG + t], xv[q], acc[k * TG + t]);
                }
            }
        }
        T a = rows_butterfly<4, LPR>(acc, sub);
        const int k = sub / (LPR / 4);  // partial k: row row + k / TG, term k % TG
        if (sub % (LPR / 4) == 0 && row + k / TG < nrows) {
            if (TIER != 0) a *= d.scal[row * TG + k];
            tbuf[d.tout + row * TG + k] = a;
        }
    }
}

// S: the tier's decoded type (FP64 storage: double, else float); T: arithmetic type.
// FP64 arithmetic over FP32 storage needs more registers: two CTAs per SM there.
template <typename S, typename T, int TIER>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 && sizeof(S) == 4) ? 2 : 3)
k_vtx(const K1Desc* __restrict__ descs, K1Classes cls, const T* __restrict__ xs, T* __restrict__ tbuf)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int ntasks = cls.task_start[4];
    const int last = cls.piece_start[4] - 1;
    // class, and this lane's piece, of a task
    auto locate = [&](int task, int& c, int& piece) {
        c = 0;
        while (c < 3 && task >= cls.task_start[c + 1]) c++;
        piece = cls.piece_start[c] + (task - cls.task_start[c]) * (32 >> (c + 2)) + (lane >> (c + 2));
    };
    if (gw >= ntasks) return;
    int c, piece;
    locate(gw, c, piece);
    K1Desc d = descs[min(piece, last)];
    for (int task = gw; task < ntasks; task += nw) {
        int cn = c, pn = piece;
        if (task + nw < ntasks) locate(task + nw, cn, pn);
        // unconditional (clamped) so that nothing waits on it before the end of the task
        const K1Desc next = descs[min(pn, last)];
        const bool have = piece < cls.piece_start[c + 1];
        switch (c) {
        case 0: vtx_group<S, T, TIER, 2>(d, have, xs, tbuf, lane); break;
        case 1: vtx_group<S, T, TIER, 3>(d, have, xs, tbuf, lane); break;
        case 2: vtx_group<S, T, TIER, 4>(d, have, xs, tbuf, lane); break;
        default: vtx_group<S, T, TIER, 5>(d, have, xs, tbuf, lane); break;
        }
        c = cn;
        piece = pn;
        d = next;
    }
}

// The rows row0..row0+3 of a mixed-storage tile slice times t_b.  The slice is a
// uniform run of chunk columns of s_pad * 4 bytes -- r32 FP32 columns, r16/2 FP16
// pairs, r8/4 FP8 quads -- so the lane's 16-byte loads are issued eight at a time
// whatever the tier, and only the decode branches (uniformly across the warp).
template <typename T>
__device__ __forceinline__ void mixed_slice(const PairDesc& d, int sp, int row0, T (&acc)[4])
{
    const char* base = static_cast<const char*>(d.data) + (size_t)row0 * 4;
    const T* w = static_cast<const T*>(d.w);
    const int n32 = d.ncol, n16 = d.c0 >> 1, n8 = d.pad >> 2;
    const int nch = n32 + n16 + n8;
    for (int k0 = 0; k0 < nch; k0 += 8) {
        uint4 raw[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            raw[u] = make_uint4(0u, 0u, 0u, 0u);
            if (k0 + u < nch) raw[u] = ld_stream(base + (size_t)(k0 + u) * sp * 4);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int k = k0 + u;
            if (k >= nch) break;
            if (k < n32) {
                const T wv = w[k];
                acc[0] = fma((T)__uint_as_float(raw[u].x), wv, acc[0]);
                acc[1] = fma((T)__uint_as_float(raw[u].y), wv, acc[1]);
                acc[2] = fma((T)__uint_as_float(raw[u].z), wv, acc[2]);
                acc[3] = fma((T)__uint_as_float(raw[u].w), wv, acc[3]);
            } else if (k < n32 + n16) {
                const int t = n32 + 2 * (k - n32);
                const T wa = w[t], wb = w[t + 1];
                const __half2* h2 = reinterpret_cast<const __half2*>(&raw[u]);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float2 f = __half22float2(h2[q]);
                    acc[q] = fma((T)f.y, wb, fma((T)f.x, wa, acc[q]));
                }
            } else {
                const int t = n32 + 2 * n16 + 4 * (k - n32 - n16);
                const T w0 = w[t], w1 = w[t + 1], w2 = w[t + 2], w3 = w[t + 3];
                const unsigned wd[4] = {raw[u].x, raw[u].y, raw[u].z, raw[u].w};
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float2 f0 = fp8x2_to_float2((unsigned short)(wd[q] & 0xffffu));
                    const float2 f1 = fp8x2_to_float2((unsigned short)(wd[q] >> 16));
                    acc[q] = fma((T)f1.y, w3, fma((T)f1.x, w2, fma((T)f0.y, w1, fma((T)f0.x, w0, acc[q]))));
                }
            }
        }
    }
}

// K2: one CTA (8 warps) per row tile.  A group of RW warps covers the tile's padded
// rows with 16-byte loads (4 FP32 or 2 FP64 rows per lane); the 8/RW groups take
// the tile's pairs round robin.
// S: storage type of the stored near field and of the FP32/FP64 terms; T: arithmetic
// type of a pair's products (float, or double for FP64 arithmetic over FP32 storage).
template <typename S, typename T>
__global__ void __launch_bounds__(256, (sizeof(T) == 8 && sizeof(S) == 4) ? 2 : 3)
k_tile_matvec(const PairDesc* desc, const int* tile_pair_start, const int* tile_r0, const int* tile_s,
              const int* perm1, KernelSpec K, PointsView P, const double* xs64, double* y)
{
    typedef typename Vec<S>::type V4;
    constexpr int NV = Vec<S>::N;
    __shared__ double red[8][HMG_TILE_ROWS];
    const int t = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = tile_s[t], sp = (s + 3) & ~3, tr0 = tile_r0[t];
    const int lanes_needed = sp / NV;
    const int RW = lanes_needed > 32 ? 2 : 1;  // sp <= 128 rows
    const int G = 8 / RW;
    const int g = warp / RW, rw = warp % RW;
    const int row0 = (rw * 32 + lane) * NV;
    const bool active = row0 < sp;
    double acc64[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) acc64[q] = 0.0;

    const int pbeg = tile_pair_start[t], pend = tile_pair_start[t + 1];
    for (int p = pbeg + g; p < pend; p += G) {
        const PairDesc d = desc[p];
        T acc[NV];
#pragma unroll
        for (int q = 0; q < NV; q++) acc[q] = 0;
        if (d.kind != PAIR_ONTHEFLY) {
            const S* base = (const S*)d.data + row0;
            const T* w = (const T*)d.w;
            bool done = !active;
            if constexpr (sizeof(S) == 4) {
                if (active && d.kind == PAIR_FAR_MIXED) {
                    mixed_slice<T>(d, sp, row0, acc);
                    done = true;
                }
            }
            if (!done) {
                int j = 0;
                for (; j + 4 <= d.ncol; j += 4) {
                    V4 v0 = ld_stream_as<V4>(base + (size_t)(j + 0) * sp);
                    V4 v1 = ld_stream_as<V4>(base + (size_t)(j + 1) * sp);
                    V4 v2 = ld_stream_as<V4>(base + (size_t)(j + 2) * sp);
                    V4 v3 = ld_stream_as<V4>(base + (size_t)(j + 3) * sp);
                    T w0 = w[j], w1 = w[j + 1], w2 = w[j + 2], w3 = w[j + 3];
                    S a[NV];
                    vec_get(v0, a);
#pragma unroll
                    for (int q = 0; q < NV; q++) acc[q] = fma((T)a[q], w0, acc[q]);
                    vec_get(v1, a);
#pragma unroll
                    for (int q = 0; q < NV; q++) acc[q] = fma((T)a[q], w1, acc[q]);
                    vec_get(v2, a);
#pragma unroll
                    for (int q = 0; q < NV; q++) acc[q] = fma((T)a[q], w2, acc[q]);
                    vec_get(v3, a);
#pragma unroll
                    for (int q = 0; q < NV; q++) acc[q] = fma((T)a[q], w3, acc[q]);
                }
                for (; j < d.ncol; j++) {
                    V4 v0 = ld_stream_as<V4>(base + (size_t)j * sp);
                    S a[NV];
                    vec_get(v0, a);
                    T w0 = w[j];
#pragma unroll
                    for (int q = 0; q < NV; q++) acc[q] = fma((T)a[q], w0, acc[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < NV; q++) acc64[q] += (double)acc[q];
        } else if (active) {
            // dense block regenerated from the points, FP64
            double a64[NV];
#pragma unroll
            for (int q = 0; q < NV; q++) a64[q] = 0.0;
            for (int j = 0; j < d.ncol; j++) {
                double xv = xs64[d.c0 + j];
#pragma unroll
                for (int q = 0; q < NV; q++)
                    if (row0 + q < s) a64[q] = fma(kernel_entry(K, P, tr0 + row0 + q, d.c0 + j), xv, a64[q]);
            }
#pragma unroll
            for (int q = 0; q < NV; q++) acc64[q] += a64[q];
        }
    }
    // fixed-order reduction of the groups' partial rows
    if (active) {
#pragma unroll
        for (int q = 0; q < NV; q++) red[g][row0 + q] = acc64[q];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < s; i += blockDim.x) {
        double v = 0.0;
        for (int gg = 0; gg < G; gg++) v += red[gg][i];
        y[perm1[tr0 + i]] = v;
    }
}

// Z-ordered x in FP64 and FP32, padded and zeroed: the streaming kernels copy
// 16-byte-aligned supersets of x pieces.
hmg_status ensure_xs(hmg_matrix* h)
{
    if (h->xs64) return HMG_OK;
    cudaStream_t s = h->stream;
    hmg_status st;
    const size_t n = (size_t)h->n[1] + 32;
    if ((st = dalloc(&h->xs64, n, s)) || (st = dalloc(&h->xs32, n, s))) return st;
    HMG_CUDA_TRY(cudaMemsetAsync(h->xs64, 0, sizeof(double) * n, s));
    HMG_CUDA_TRY(cudaMemsetAsync(h->xs32, 0, sizeof(float) * n, s));
    return HMG_OK;
}

static hmg_status launch_product(hmg_matrix* h, const double* x, double* y, bool fp64, bool arith64, bool bulk_k1,
                                 bool bulk_k2);
static hmg_status launch_product_graph(hmg_matrix* h, const double* x, double* y, bool fp64, bool arith64);

hmg_status matvec_device(hmg_matrix* h, const double* x, double* y, bool fp64_arith)
{
    hmg_status st;
    if (h->group_count && h->ndense > 0 && (h->near_mode != HMG_NEAR_STORED || h->near_prec < 0)) {
        set_error("a group handle multiplies a stored near field: call hmg_precompute_dense first");
        return HMG_ERR_STATE;
    }
    if ((st = ensure_xs(h))) return st;
    const bool mixed = h->far_prec == HMG_PREC_MIXED;
    // storage element type of the stored near field and the FP32/FP64 terms
    const bool fp64 = h->far_prec == HMG_PREC_FP64 ||
                      (h->naca == 0 && h->near_prec != HMG_PREC_FP32);
    // arithmetic type of the products
    const bool arith64 = fp64 || fp64_arith || h->arith_prec == HMG_PREC_FP64;
    // stored near field and factors are read by one kernel instance: same element type
    const int far_elem_prec = mixed ? HMG_PREC_FP32 : h->far_prec;
    if (h->near_mode == HMG_NEAR_STORED && h->naca > 0 && h->near_prec != far_elem_prec) {
        set_error("stored near field (precision %d) and factors (precision %d) differ", h->near_prec,
                  h->far_prec);
        return HMG_ERR_UNSUPPORTED;
    }
    const int elem = arith64 ? 8 : 4;
    if ((st = ensure_desc(h, elem))) return st;
    // the streaming kernels read FP32/FP64 storage in its own arithmetic only
    const bool plain_types = !mixed && arith64 == fp64;
    const bool bulk_k1 = h->matvec_variant == 0 && plain_types && h->max_rank <= K1_MAXRANK;
    const bool bulk_k2 = h->matvec_variant == 0 && plain_types &&
                         (h->near_mode == HMG_NEAR_STORED || h->ndense == 0);
    h->last_variant_k1 = bulk_k1 ? 0 : 1;
    h->last_variant_k2 = bulk_k2 ? 0 : 1;
    if (h->use_graphs && !h->profiling && !bulk_k1 && !bulk_k2) return launch_product_graph(h, x, y, fp64, arith64);
    return launch_product(h, x, y, fp64, arith64, bulk_k1, bulk_k2);
}

// Everything a product's launches depend on besides the contents of device memory: two
// products with equal keys issue the same launches with the same arguments, so the
// graph captured for one replays the other.
struct ProductKey {
    const double* x;
    double* y;
    int fp64, arith64, ntiles, nk1, near_mode, near_prec, far_prec;
    int k1_task_start[3][5], k1_piece_start[3][5];
    const void *k1_units, *tbuf, *pair_desc, *xs64, *xs32;
    const int *tile_pair_start, *tile_r0, *tile_s, *perm0, *perm1;
    KernelSpec kspec;
    PointsView P;
};

static ProductKey product_key(hmg_matrix* h, const double* x, double* y, bool fp64, bool arith64)
{
    ProductKey k;
    memset(&k, 0, sizeof(k));  // padding included: keys are compared bytewise
    k.x = x;
    k.y = y;
    k.fp64 = fp64;
    k.arith64 = arith64;
    k.ntiles = h->ntiles;
    k.nk1 = h->nk1;
    k.near_mode = h->near_mode;
    k.near_prec = h->near_prec;
    k.far_prec = h->far_prec;
    memcpy(k.k1_task_start, h->k1_task_start, sizeof(k.k1_task_start));
    memcpy(k.k1_piece_start, h->k1_piece_start, sizeof(k.k1_piece_start));
    k.k1_units = h->k1_units;
    k.tbuf = h->tbuf;
    k.pair_desc = h->pair_desc;
    k.xs64 = h->xs64;
    k.xs32 = h->xs32;
    k.tile_pair_start = h->tile_pair_start;
    k.tile_r0 = h->tile_r0;
    k.tile_s = h->tile_s;
    k.perm0 = h->perm[0];
    k.perm1 = h->perm[1];
    k.kspec = h->kspec;
    k.P = points_view(h);
    return k;
}

void free_product_graph(hmg_matrix* h)
{
    if (h->graph_exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(h->graph_exec));
    h->graph_exec = nullptr;
    free(h->graph_key);
    h->graph_key = nullptr;
}

// The product as one CUDA graph: captured on the first call with a new key, replayed
// with cudaGraphLaunch while the key holds (one graph per handle).
static hmg_status launch_product_graph(hmg_matrix* h, const double* x, double* y, bool fp64, bool arith64)
{
    cudaStream_t s = h->stream;
    const ProductKey key = product_key(h, x, y, fp64, arith64);
    if (!h->graph_exec || memcmp(h->graph_key, &key, sizeof(key)) != 0) {
        free_product_graph(h);
        // captured on a stream of its own (the handle's may be the legacy default stream,
        // which cannot be captured); capturing runs nothing
        if (!h->capture_stream) {
            cudaStream_t cs = nullptr;
            HMG_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            h->capture_stream = cs;
        }
        cudaStream_t cs = static_cast<cudaStream_t>(h->capture_stream);
        HMG_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        h->stream = cs;
        const hmg_status st = launch_product(h, x, y, fp64, arith64, false, false);
        h->stream = s;
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(cs, &g);
        if (st || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            if (!st) set_error("capturing the product graph failed: %s", cudaGetErrorString(ce));
            return st ? st : HMG_ERR_CUDA;
        }
        cudaGraphExec_t ex = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            cudaGetLastError();
            set_error("instantiating the product graph failed: %s", cudaGetErrorString(ie));
            return HMG_ERR_CUDA;
        }
        h->graph_exec = ex;
        h->graph_key = malloc(sizeof(key));
        memcpy(h->graph_key, &key, sizeof(key));
    }
    HMG_CUDA_TRY(cudaGraphLaunch(static_cast<cudaGraphExec_t>(h->graph_exec), s));
    return HMG_OK;
}

// The launches of one product (x gather, V^T x per storage tier, tile kernel).
static hmg_status launch_product(hmg_matrix* h, const double* x, double* y, bool fp64, bool arith64, bool bulk_k1,
                                 bool bulk_k2)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    PointsView P = points_view(h);
    if (h->profiling) HMG_CUDA_TRY(cudaEventRecord(h->ev[0], s));
    k_gather_x<<<ceil_div(h->n[1], 256), 256, 0, s>>>(x, h->perm[1], h->n[1], h->xs64, h->xs32);
    HMG_LAUNCH_CHECK();
    if (h->profiling) HMG_CUDA_TRY(cudaEventRecord(h->ev[1], s));
    if (bulk_k1 && h->nfar_list > 0) {
        if ((st = launch_vtx_bulk(h, fp64))) return st;
    } else if (h->nk1 > 0) {
        const K1Desc* dd = static_cast<const K1Desc*>(h->k1_units);
        double* t64 = static_cast<double*>(h->tbuf);
        float* t32 = static_cast<float*>(h->tbuf);
        // The tiers write disjoint t_b entries: the FP16 and FP8 tiers run on two side
        // streams beside the FP32 one (forked from and joined back into the handle's
        // stream), so the FP8 tier's conversion-bound warps share the SMs with the FP32
        // tier's load-bound ones and the three launches' tails overlap.
        const bool fork = h->k1_task_start[1][4] > 0 || h->k1_task_start[2][4] > 0;
        if (fork) {
            for (int i = 0; i < 2; i++)
                if (!h->k1_aux[i]) HMG_CUDA_TRY(cudaStreamCreateWithFlags(&h->k1_aux[i], cudaStreamNonBlocking));
            for (int i = 0; i < 3; i++)
                if (!h->k1_ev[i]) HMG_CUDA_TRY(cudaEventCreateWithFlags(&h->k1_ev[i], cudaEventDisableTiming));
            HMG_CUDA_TRY(cudaEventRecord(h->k1_ev[0], s));
            for (int i = 0; i < 2; i++) HMG_CUDA_TRY(cudaStreamWaitEvent(h->k1_aux[i], h->k1_ev[0], 0));
        }
        for (int tier = 0; tier < 3; tier++) {
            const cudaStream_t ts = (fork && tier > 0) ? h->k1_aux[tier - 1] : s;
            K1Classes cls;
            for (int c = 0; c < 5; c++) {
                cls.piece_start[c] = h->k1_piece_start[tier][c];
                cls.task_start[c] = h->k1_task_start[tier][c];
            }
            const int ntasks = cls.task_start[4];
            if (ntasks == 0) continue;
            const int grid = std::min(ceil_div(ntasks, 8), h->nsm * h->k1_ctas_per_sm);
            if (tier == 0) {
                if (fp64)
                    k_vtx<double, double, 0><<<grid, 256, 0, ts>>>(dd, cls, h->xs64, t64);
                else if (arith64)
                    k_vtx<float, double, 0><<<grid, 256, 0, ts>>>(dd, cls, h->xs64, t64);
                else
                    k_vtx<float, float, 0><<<grid, 256, 0, ts>>>(dd, cls, h->xs32, t32);
            } else if (tier == 1) {
                if (arith64)
                    k_vtx<float, double, 1><<<grid, 256, 0, ts>>>(dd, cls, h->xs64, t64);
                else
                    k_vtx<float, float, 1><<<grid, 256, 0, ts>>>(dd, cls, h->xs32, t32);
            } else {
                if (arith64)
                    k_vtx<float, double, 2><<<grid, 256, 0, ts>>>(dd, cls, h->xs64, t64);
                else
                    k_vtx<float, float, 2><<<grid, 256, 0, ts>>>(dd, cls, h->xs32, t32);
            }
            HMG_LAUNCH_CHECK();
        }
        if (fork)
            for (int i = 0; i < 2; i++) {
                HMG_CUDA_TRY(cudaEventRecord(h->k1_ev[1 + i], h->k1_aux[i]));
                HMG_CUDA_TRY(cudaStreamWaitEvent(s, h->k1_ev[1 + i], 0));
            }
    }
    if (h->profiling) HMG_CUDA_TRY(cudaEventRecord(h->ev[2], s));
    if (h->ntiles > 0 && bulk_k2) {
        if ((st = launch_tiles_bulk(h, fp64, y))) return st;
    } else if (h->ntiles > 0) {
        const PairDesc* pd = static_cast<const PairDesc*>(h->pair_desc);
        if (fp64)
            k_tile_matvec<double, double><<<h->ntiles, 256, 0, s>>>(pd, h->tile_pair_start, h->tile_r0, h->tile_s,
                                                                    h->perm[0], h->kspec, P, h->xs64, y);
        else if (arith64)
            k_tile_matvec<float, double><<<h->ntiles, 256, 0, s>>>(pd, h->tile_pair_start, h->tile_r0, h->tile_s,
                                                                   h->perm[0], h->kspec, P, h->xs64, y);
        else
            k_tile_matvec<float, float><<<h->ntiles, 256, 0, s>>>(pd, h->tile_pair_start, h->tile_r0, h->tile_s,
                                                                  h->perm[0], h->kspec, P, h->xs64, y);
        HMG_LAUNCH_CHECK();
    }
    if (h->profiling) HMG_CUDA_TRY(cudaEventRecord(h->ev[3], s));
    return HMG_OK;
}

// ---------------------------------------------------------------------------
// FP64 direct summation (apply_full_mvp, hmglib.cu:351-401, without the N^2 matrix)
// ---------------------------------------------------------------------------
static constexpr int DS_THREADS = 256;
static constexpr int DS_CHUNK = 512;

__global__ void __launch_bounds__(DS_THREADS)
k_direct(KernelSpec K, PointsView P, const double* xs, const int* zrows, int nrows, const int* out_perm,
         double* y)
{
    __shared__ double cx[3][DS_CHUNK];
    __shared__ double xv[DS_CHUNK];
    const int t = blockIdx.x * DS_THREADS + threadIdx.x;
    const bool valid = t < nrows;
    const int i = valid ? (zrows ? zrows[t] : t) : 0;
    double pi[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < K.dim; d++) pi[d] = P.c1[d][i];
    double acc = 0.0;
    for (int j0 = 0; j0 < P.n2; j0 += DS_CHUNK) {
        int nc = P.n2 - j0 < DS_CHUNK ? P.n2 - j0 : DS_CHUNK;
        __syncthreads();
        for (int c = threadIdx.x; c < nc; c += DS_THREADS) {
            for (int d = 0; d < K.dim; d++) cx[d][c] = P.c2[d][j0 + c];
            xv[c] = xs[j0 + c];
        }
        __syncthreads();
        if (valid) {
            for (int c = 0; c < nc; c++) {
                double sq = 0.0;
                for (int d = 0; d < K.dim; d++) {
                    double q = pi[d] - cx[d][c];
                    sq = __fma_rn(q, q, sq);
                }
                double k = kernel_from_sq(K, sq);
                if (i == j0 + c) k += K.reg;
                acc = fma(k, xv[c], acc);
            }
        }
    }
    if (valid) y[out_perm ? out_perm[i] : t] = acc;
}

__global__ void k_rows_to_z(const int* rows, int n, const int* iperm, int* z)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) z[t] = iperm[rows[t]];
}

hmg_status direct_matvec(hmg_matrix* h, const double* x, const int* rows, int nrows, double* y)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    if ((st = ensure_xs(h))) return st;
    k_gather_x<<<ceil_div(h->n[1], 256), 256, 0, s>>>(x, h->perm[1], h->n[1], h->xs64, h->xs32);
    HMG_LAUNCH_CHECK();
    PointsView P = points_view(h);
    if (!rows) {
        k_direct<<<ceil_div(h->n[0], DS_THREADS), DS_THREADS, 0, s>>>(h->kspec, P, h->xs64, nullptr, h->n[0],
                                                                      h->perm[0], y);
        HMG_LAUNCH_CHECK();
        return HMG_OK;
    }
    int* z = nullptr;
    if ((st = dalloc(&z, (size_t)(nrows > 0 ? nrows : 1), s))) return st;
    if (nrows > 0) {
        k_rows_to_z<<<ceil_div(nrows, 256), 256, 0, s>>>(rows, nrows, h->iperm[0], z);
        HMG_LAUNCH_CHECK();
        k_direct<<<ceil_div(nrows, DS_THREADS), DS_THREADS, 0, s>>>(h->kspec, P, h->xs64, z, nrows, nullptr, y);
        HMG_LAUNCH_CHECK();
    }
    dfree(z, s);
    return HMG_OK;
}

// set_gaussian_kernel_rhs (hmglib.cu:403-439), evaluated in the caller's order
__global__ void k_gaussian_rhs(const double* pts, int n, int dim, double* b)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double pi = 3.14159265358979323846;
    double r = 1.0;
    for (int d = 0; d < dim; d++) {
        double x = pts[(size_t)d * n + i];
        r = r * sqrt(pi) * (erf(1.0 - x) - erf(0.0 - x)) / 2.0;
    }
    b[i] = r;
}

hmg_status gaussian_rhs(hmg_matrix* h, double* b)
{
    k_gaussian_rhs<<<ceil_div(h->n[0], 256), 256, 0, h->stream>>>(h->pts[0], h->n[0], h->dim, b);
    HMG_LAUNCH_CHECK();
    return HMG_OK;
}

// ---------------------------------------------------------------------------
// autotuning of the product's launch shapes (hmg_autotune)
// ---------------------------------------------------------------------------
// Times the single-vector product on this handle's own H-matrix for each pair of
// V^T piece size (the unit of K1's warp tasks) and K1 grid (CTAs per SM), with CUDA
// events around `reps` products after one untimed product (the first after a piece
// size change also rebuilds the descriptors), and keeps the fastest.  x is the
// handle's device staging vector (its values do not change the work).
hmg_status autotune(hmg_matrix* h, int reps, int* best_piece, int* best_ctas, double* best_ms)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    if (!h->dev_x) {
        if ((st = dalloc(&h->dev_x, (size_t)h->n[1], s)) || (st = dalloc(&h->dev_y, (size_t)h->n[0], s))) return st;
        HMG_CUDA_TRY(cudaMemsetAsync(h->dev_x, 0, sizeof(double) * h->n[1], s));
    }
    static const int pieces[] = {32768, 65536, 131072};
    static const int ctas[] = {4, 8, 16};
    cudaEvent_t e0, e1;
    HMG_CUDA_TRY(cudaEventCreate(&e0));
    HMG_CUDA_TRY(cudaEventCreate(&e1));
    const bool prof = h->profiling;
    h->profiling = false;
    const int piece0 = h->k1_piece_bytes, ctas0 = h->k1_ctas_per_sm;
    double best = 1e300;
    int bp = piece0, bc = ctas0;
    st = HMG_OK;
    for (int pi = 0; pi < 3 && !st; pi++)
        for (int ci = 0; ci < 3 && !st; ci++) {
            if (h->k1_piece_bytes != pieces[pi]) {
                h->k1_piece_bytes = pieces[pi];
                h->desc_near_mode = -1;  // rebuild the K1 pieces
            }
            h->k1_ctas_per_sm = ctas[ci];
            if ((st = matvec_device(h, h->dev_x, h->dev_y))) break;
            cudaEventRecord(e0, s);
            for (int r = 0; r < reps && !st; r++) st = matvec_device(h, h->dev_x, h->dev_y);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) st = HMG_ERR_CUDA;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (!st && ms / reps < best) {
                best = ms / reps;
                bp = pieces[pi];
                bc = ctas[ci];
            }
        }
    h->profiling = prof;
    if (h->k1_piece_bytes != bp) h->desc_near_mode = -1;
    h->k1_piece_bytes = st ? piece0 : bp;
    h->k1_ctas_per_sm = st ? ctas0 : bc;
    if (st) h->desc_near_mode = -1;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if (best_piece) *best_piece = bp;
    if (best_ctas) *best_ctas = bc;
    if (best_ms) *best_ms = best;
    return HMG_OK;
}

}  // namespace hmg
