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
#include <cuda_fp16.h>
#include <cuda_fp8.h>

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

// 16-byte asynchronous copy global -> shared; an invalid source copies nothing and
// zeroes the 16 destination bytes.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    const int n = valid ? 16 : 0;  // 0 source bytes: the 16 destination bytes are zeroed
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
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

static constexpr int K1M_STAGES = 4;
static constexpr size_t K1M_SMEM = 8 * K1M_STAGES * 4 * 128 * sizeof(float);  // 64 KB per CTA

// FP32 storage, R = 8, 16 or 32 vectors: t_b = V_b^T X_b with V rows streamed through
// per-warp shared memory (cp.async, 4 rows x 128 columns per stage, four in flight),
// so every lane's copies are distinct coalesced 16-byte transfers.  Lane (cg, rg)
// computes 4 rows x 4 vectors over every CGN-th group of 4 columns of a stage (V
// from shared memory, X from global/L1), and the CGN column groups are summed by a
// fixed xor butterfly at the end of each 4-row block.
// {a0, a1} += s * {b0, b1}: one packed FP32 multiply-add (two vectors of one stored
// value), each lane rounded as fmaf would round it
__device__ __forceinline__ void fma2s(float& a0, float& a1, float s, float b0, float b1)
{
    uint32_t x0 = __float_as_uint(a0), x1 = __float_as_uint(a1);
    asm("{\n\t.reg .b64 a, b, d;\n\tmov.b64 a, {%2, %2};\n\tmov.b64 b, {%3, %4};\n\tmov.b64 d, {%0, %1};\n\t"
        "fma.rn.f32x2 d, a, b, d;\n\tmov.b64 {%0, %1}, d;\n\t}"
        : "+r"(x0), "+r"(x1) : "r"(__float_as_uint(s)), "r"(__float_as_uint(b0)), "r"(__float_as_uint(b1)));
    a0 = __uint_as_float(x0);
    a1 = __uint_as_float(x1);
}

// 16 bytes of a K1 piece row of tier TIER as [column q][term t] floats: 4 columns of
// TG = 1 (FP32), 2 (FP16 pairs) or 4 (FP8 quads) terms
template <int TIER>
__device__ __forceinline__ void tier_chunk(const uint4& u, float* o)
{
    if constexpr (TIER == 0) {
        o[0] = __uint_as_float(u.x); o[1] = __uint_as_float(u.y);
        o[2] = __uint_as_float(u.z); o[3] = __uint_as_float(u.w);
    } else {
        const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if constexpr (TIER == 1) {
                const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[q]));
                o[2 * q] = f.x;
                o[2 * q + 1] = f.y;
            } else {
                __half2_raw lo = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[q] & 0xffffu), __NV_E4M3);
                __half2_raw hi = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[q] >> 16), __NV_E4M3);
                const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&lo));
                const float2 c = __half22float2(*reinterpret_cast<const __half2*>(&hi));
                o[4 * q] = a.x; o[4 * q + 1] = a.y; o[4 * q + 2] = c.x; o[4 * q + 3] = c.y;
            }
        }
    }
}

template <int R, int TIER>
__global__ void __launch_bounds__(256) k_vtx_multi_smem(const K1Desc* __restrict__ descs, int n,
                                                        const float* __restrict__ xm, float* __restrict__ tm)
{
    constexpr int RG = R / 4, CGN = 32 / RG, SC = 128;  // vector groups, column groups, stage columns
    constexpr int NS = K1M_STAGES;                      // stages in flight per warp
    constexpr int TG = TIER == 0 ? 1 : (TIER == 1 ? 2 : 4), NR = 4 / TG;  // terms per row, rows per block
    extern __shared__ __align__(16) float k1m_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float (*Vs)[4][SC] = reinterpret_cast<float (*)[4][SC]>(k1m_smem + (size_t)warp * NS * 4 * SC);
    const int rg = lane % RG, cg = lane / RG;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int u = gw; u < n; u += nw) {
        const K1Desc d = descs[u];
        const int cpr = d.row_bytes >> 4;  // 16-byte chunks per row
        const int nst = (cpr + SC / 4 - 1) / (SC / 4);  // stages per block of 4 terms
        const char* vb = static_cast<const char*>(d.v);
        const int total = ((d.nrows + NR - 1) / NR) * nst;
        auto issue = [&](int it) {
            if (it < total) {
                const int blk = it / nst, st = it - blk * nst;
                const int ch = st * (SC / 4) + lane;  // this lane's chunk of each row
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    const int row = blk * NR + k;
                    const bool v = row < d.nrows && ch < cpr;
                    cp_async16(&Vs[it % NS][k][lane * 4], v ? vb + (size_t)row * d.row_bytes + (size_t)ch * 16 : vb, v);
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
        float acc[4][4];  // [term of the block][vector]
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[a][c] = 0.0f;
#pragma unroll
        for (int it = 0; it < NS - 1; it++) issue(it);
        for (int it = 0; it < total; it++) {
            issue(it + NS - 1);
            asm volatile("cp.async.wait_group %0;" ::"n"(NS - 1) : "memory");
            __syncwarp();
            const int b = it % NS;
            const int blk = it / nst, st = it - blk * nst;
            const int cbase = st * SC;  // first column of the stage
#pragma unroll
            for (int sub = 0; sub < SC / 4 / CGN; sub++) {
                const int c4 = (sub * CGN + cg) * 4;  // first of this lane's 4 columns
                const int col = cbase + c4;
                float4 xv[4];
#pragma unroll
                for (int q = 0; q < 4; q++)
                    xv[q] = col + q < d.m2 ? *reinterpret_cast<const float4*>(xm + (size_t)(d.c0 + col + q) * R + rg * 4)
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int k = 0; k < NR; k++) {
                    float f[4 * TG];
                    tier_chunk<TIER>(*reinterpret_cast<const uint4*>(&Vs[b][k][c4]), f);
#pragma unroll
                    for (int q = 0; q < 4; q++)
#pragma unroll
                        for (int tt = 0; tt < TG; tt++) {
                            const float vv = f[q * TG + tt];
                            float* ac = acc[k * TG + tt];
                            fma2s(ac[0], ac[1], vv, xv[q].x, xv[q].y);
                            fma2s(ac[2], ac[3], vv, xv[q].z, xv[q].w);
                        }
                }
            }
            __syncwarp();  // this buffer is refilled NS - 1 stages on
            if (st == nst - 1) {
                // the block's 4 terms are complete: sum the column groups, scale, write, reset
#pragma unroll
                for (int o = RG; o < 32; o <<= 1)
#pragma unroll
                    for (int k = 0; k < 4; k++)
#pragma unroll
                        for (int c = 0; c < 4; c++) acc[k][c] += __shfl_xor_sync(0xffffffffu, acc[k][c], o);
                if (cg == 0)
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const int term = blk * 4 + k;
                        if (term < d.nrows * TG) {
                            const float sc = TIER == 0 ? 1.0f : d.scal[term];
                            *reinterpret_cast<float4*>(tm + (size_t)(d.tout + term) * R + rg * 4) =
                                make_float4(acc[k][0] * sc, acc[k][1] * sc, acc[k][2] * sc, acc[k][3] * sc);
                        }
                    }
#pragma unroll
                for (int k = 0; k < 4; k++)
#pragma unroll
                    for (int c = 0; c < 4; c++) acc[k][c] = 0.0f;
            }
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncwarp();
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

// FP32 storage, R = 8, 16 or 32 vectors: the tile's slices are streamed through
// shared memory in stages of 16 columns (cp.async, four stages in flight across pairs), and
// each thread keeps a (R/8 rows) x (4 vectors) register tile, so every shared value
// it reads feeds R/8 or 4 multiply-adds.  Products per pair in FP32, added in FP64.

template <int R>
__global__ void __launch_bounds__(256) k_tile_multi_smem(const PairDesc* __restrict__ desc,
                                                         const int* tile_pair_start, const int* tile_r0,
                                                         const int* tile_s, const int* perm1,
                                                         const float* __restrict__ xm, const float* __restrict__ tm,
                                                         const char* tbase, int nrhs, double* Y, int ldy,
                                                         int only_kind)
{
    constexpr int KC = 16, NS = 4, CG = R / 4, TR = R / 8;  // NS stages in flight
    __shared__ __align__(16) float Us[NS][KC][HMG_TILE_ROWS];
    __shared__ __align__(16) float Ts[NS][KC][R];
    const int t = blockIdx.x, tid = threadIdx.x;
    const int cg = tid % CG, rg = tid / CG;
    const int s = tile_s[t], sp = (s + 3) & ~3, tr0 = tile_r0[t];
    const int pbeg = tile_pair_start[t], pend = tile_pair_start[t + 1];
    const int sp4 = sp >> 2;

    // stage (pair p, first column k0) into buffer b
    auto issue = [&](int b, int p, int k0) {
        const PairDesc d = desc[p];
        const float* data = static_cast<const float*>(d.data);
        for (int idx = tid; idx < KC * sp4; idx += 256) {
            const int kk = idx / sp4, r4 = idx - kk * sp4;
            const bool v = k0 + kk < d.ncol;
            cp_async16(&Us[b][kk][r4 * 4], v ? data + (size_t)(k0 + kk) * sp + r4 * 4 : data, v);
        }
        const float* src = d.kind == PAIR_STORED
                               ? xm + (size_t)d.c0 * R
                               : tm + (size_t)((static_cast<const char*>(d.w) - tbase) / 4) * R;
        for (int idx = tid; idx < KC * (R / 4); idx += 256) {
            const int kk = idx / (R / 4), c4 = idx - kk * (R / 4);
            const bool v = k0 + kk < d.ncol;
            cp_async16(&Ts[b][kk][c4 * 4], v ? src + (size_t)(k0 + kk) * R + c4 * 4 : src, v);
        }
    };
    // the flattened sequence of (pair, column chunk) stages, skipping empty pairs and
    // (only_kind >= 0) pairs of another kind
    auto skip = [&](int q) { return desc[q].ncol == 0 || (only_kind >= 0 && desc[q].kind != only_kind); };
    auto advance = [&](int& q, int& kq) {
        kq += KC;
        if (kq >= desc[q].ncol) {
            q++;
            kq = 0;
            while (q < pend && skip(q)) q++;
        }
    };
    int p = pbeg, k0 = 0;
    while (p < pend && skip(p)) p++;
    int pp = p, kp = 0;  // producer cursor, NS - 1 stages ahead
    for (int st = 0; st < NS - 1; st++) {
        if (pp < pend) {
            issue(st, pp, kp);
            advance(pp, kp);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }

    double acc64[TR][4];
    float acc[TR][4];
#pragma unroll
    for (int i = 0; i < TR; i++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc64[i][c] = 0.0, acc[i][c] = 0.0f;

    for (int it = 0; p < pend; it++) {
        if (pp < pend) {
            issue((it + NS - 1) % NS, pp, kp);
            advance(pp, kp);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group %0;" ::"n"(NS - 1) : "memory");
        __syncthreads();
        const int buf = it % NS;
        const int kmax = min(KC, desc[p].ncol - k0);
        for (int k = 0; k < kmax; k++) {
            float u[TR];
            if constexpr (TR == 4) {
                const float4 v = *reinterpret_cast<const float4*>(&Us[buf][k][rg * 4]);
                u[0] = v.x; u[1] = v.y; u[2] = v.z; u[3] = v.w;
            } else if constexpr (TR == 2) {
                const float2 v = *reinterpret_cast<const float2*>(&Us[buf][k][rg * 2]);
                u[0] = v.x; u[1] = v.y;
            } else {
                u[0] = Us[buf][k][rg];
            }
            const float4 w = *reinterpret_cast<const float4*>(&Ts[buf][k][cg * 4]);
#pragma unroll
            for (int i = 0; i < TR; i++) {
                fma2s(acc[i][0], acc[i][1], u[i], w.x, w.y);
                fma2s(acc[i][2], acc[i][3], u[i], w.z, w.w);
            }
        }
        int pn = p, kn = k0;
        advance(pn, kn);
        if (pn != p) {
#pragma unroll
            for (int i = 0; i < TR; i++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc64[i][c] += (double)acc[i][c], acc[i][c] = 0.0f;
        }
        __syncthreads();  // this buffer is refilled NS - 1 stages on
        p = pn;
        k0 = kn;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
    for (int i = 0; i < TR; i++) {
        const int row = rg * TR + i;
        if (row < s)
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int j = cg * 4 + c;
                if (j < nrhs) Y[perm1[tr0 + row] + (size_t)j * ldy] = acc64[i][c];
            }
    }
}

// Mixed storage (FP32 / FP16-pair / FP8-quad chunk columns), R = 8, 16 or 32
// vectors: the tile kernel above with each chunk column decoded at use.  A chunk
// column holds TG = 1, 2 or 4 terms for 4 rows per 16 bytes; the stage carries the TG
// vector rows (t_b, already scaled) that multiply it.  A thread keeps VT vectors of its
// rows (8 for R = 8, in blocks of 128 threads, so that each decoded value feeds four
// packed multiply-adds; else 4, in blocks of 256).
template <int R>
constexpr size_t mixed_tile_smem()
{
    return (size_t)4 * 16 * (HMG_TILE_ROWS + 4 * R) * sizeof(float) + 4 * 16 * sizeof(int);
}

template <int R, int VT>
__global__ void __launch_bounds__(256) k_tile_multi_mixed(const PairDesc* __restrict__ desc,
                                                          const int* tile_pair_start, const int* tile_r0,
                                                          const int* tile_s, const int* perm1,
                                                          const float* __restrict__ xm, const float* __restrict__ tm,
                                                          const char* tbase, int nrhs, double* Y, int ldy)
{
    constexpr int KC = 16, NS = 4, CG = R / VT, TR = R / 8, NT = 1024 / VT;  // VT vectors a thread
    extern __shared__ __align__(16) float mx_smem[];
    float (*Us)[KC][HMG_TILE_ROWS] = reinterpret_cast<float (*)[KC][HMG_TILE_ROWS]>(mx_smem);
    float (*Ts)[KC][4][R] = reinterpret_cast<float (*)[KC][4][R]>(mx_smem + NS * KC * HMG_TILE_ROWS);
    int (*Tg)[KC] = reinterpret_cast<int (*)[KC]>(mx_smem + NS * KC * (HMG_TILE_ROWS + 4 * R));
    const int t = blockIdx.x, tid = threadIdx.x;
    const int cg = tid % CG, rg = tid / CG;
    const int s = tile_s[t], sp = (s + 3) & ~3, tr0 = tile_r0[t];
    const int pbeg = tile_pair_start[t], pend = tile_pair_start[t + 1];
    const int sp4 = sp >> 2;
    // chunk columns of a pair
    auto cols = [&](const PairDesc& d) {
        return d.kind == PAIR_FAR_MIXED ? d.ncol + (d.c0 >> 1) + (d.pad >> 2) : d.ncol;
    };
    auto issue = [&](int b, int p, int k0) {
        const PairDesc d = desc[p];
        const int nc = cols(d);
        const char* data = static_cast<const char*>(d.data);
        for (int idx = tid; idx < KC * sp4; idx += NT) {
            const int kk = idx / sp4, r4 = idx - kk * sp4;
            const bool v = k0 + kk < nc;
            cp_async16(&Us[b][kk][r4 * 4], v ? data + ((size_t)(k0 + kk) * sp + r4 * 4) * 4 : data, v);
        }
        const bool far = d.kind == PAIR_FAR_MIXED;
        const float* tb = far ? tm + (size_t)((static_cast<const char*>(d.w) - tbase) / 4) * R : xm + (size_t)d.c0 * R;
        const int n32 = d.ncol, n16 = d.c0 >> 1;
        for (int idx = tid; idx < KC * 4 * (R / 4); idx += NT) {
            const int kk = idx / (4 * (R / 4)), rem = idx - kk * (4 * (R / 4));
            const int tt = rem / (R / 4), c4 = rem - tt * (R / 4);
            const int k = k0 + kk;
            int tg = 1, term = k;
            if (far) {
                if (k >= n32 + n16) tg = 4, term = n32 + 2 * n16 + 4 * (k - n32 - n16);
                else if (k >= n32) tg = 2, term = n32 + 2 * (k - n32);
            }
            const bool v = k < nc && tt < tg;
            cp_async16(&Ts[b][kk][tt][c4 * 4], v ? tb + (size_t)(term + tt) * R + c4 * 4 : tb, v);
            if (tt == 0 && c4 == 0) Tg[b][kk] = tg;
        }
    };
    auto skip = [&](int q) { return cols(desc[q]) == 0; };
    auto advance = [&](int& q, int& kq) {
        kq += KC;
        if (kq >= cols(desc[q])) {
            q++;
            kq = 0;
            while (q < pend && skip(q)) q++;
        }
    };
    int p = pbeg, k0 = 0;
    while (p < pend && skip(p)) p++;
    int pp = p, kp = 0;
    for (int st = 0; st < NS - 1; st++) {
        if (pp < pend) {
            issue(st, pp, kp);
            advance(pp, kp);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    double acc64[TR][VT];
    float acc[TR][VT];
#pragma unroll
    for (int i = 0; i < TR; i++)
#pragma unroll
        for (int c = 0; c < VT; c++) acc64[i][c] = 0.0, acc[i][c] = 0.0f;
    for (int it = 0; p < pend; it++) {
        if (pp < pend) {
            issue((it + NS - 1) % NS, pp, kp);
            advance(pp, kp);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group %0;" ::"n"(NS - 1) : "memory");
        __syncthreads();
        const int buf = it % NS;
        const int kmax = min(KC, cols(desc[p]) - k0);
        for (int k = 0; k < kmax; k++) {
            unsigned w[TR];
            if constexpr (TR == 4) {
                const uint4 v = *reinterpret_cast<const uint4*>(&Us[buf][k][rg * 4]);
                w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
            } else if constexpr (TR == 2) {
                const uint2 v = *reinterpret_cast<const uint2*>(&Us[buf][k][rg * 2]);
                w[0] = v.x; w[1] = v.y;
            } else {
                w[0] = __float_as_uint(Us[buf][k][rg]);
            }
            const int tg = Tg[buf][k];
            if (tg == 1) {
#pragma unroll
                for (int hh = 0; hh < VT / 4; hh++) {
                    const float4 x = *reinterpret_cast<const float4*>(&Ts[buf][k][0][cg * VT + 4 * hh]);
#pragma unroll
                    for (int i = 0; i < TR; i++) {
                        const float u = __uint_as_float(w[i]);
                        fma2s(acc[i][4 * hh], acc[i][4 * hh + 1], u, x.x, x.y);
                        fma2s(acc[i][4 * hh + 2], acc[i][4 * hh + 3], u, x.z, x.w);
                    }
                }
            } else if (tg == 2) {
                float4 x0[VT / 4], x1[VT / 4];
#pragma unroll
                for (int hh = 0; hh < VT / 4; hh++) {
                    x0[hh] = *reinterpret_cast<const float4*>(&Ts[buf][k][0][cg * VT + 4 * hh]);
                    x1[hh] = *reinterpret_cast<const float4*>(&Ts[buf][k][1][cg * VT + 4 * hh]);
                }
#pragma unroll
                for (int i = 0; i < TR; i++) {
                    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[i]));
#pragma unroll
                    for (int hh = 0; hh < VT / 4; hh++) {
                        fma2s(acc[i][4 * hh], acc[i][4 * hh + 1], f.x, x0[hh].x, x0[hh].y);
                        fma2s(acc[i][4 * hh + 2], acc[i][4 * hh + 3], f.x, x0[hh].z, x0[hh].w);
                        fma2s(acc[i][4 * hh], acc[i][4 * hh + 1], f.y, x1[hh].x, x1[hh].y);
                        fma2s(acc[i][4 * hh + 2], acc[i][4 * hh + 3], f.y, x1[hh].z, x1[hh].w);
                    }
                }
            } else {
                float4 x[4][VT / 4];
#pragma unroll
                for (int tt = 0; tt < 4; tt++)
#pragma unroll
                    for (int hh = 0; hh < VT / 4; hh++)
                        x[tt][hh] = *reinterpret_cast<const float4*>(&Ts[buf][k][tt][cg * VT + 4 * hh]);
#pragma unroll
                for (int i = 0; i < TR; i++) {
                    __half2_raw lo = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[i] & 0xffffu), __NV_E4M3);
                    __half2_raw hi = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[i] >> 16), __NV_E4M3);
                    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&lo));
                    const float2 c = __half22float2(*reinterpret_cast<const __half2*>(&hi));
                    const float f[4] = {a.x, a.y, c.x, c.y};
#pragma unroll
                    for (int tt = 0; tt < 4; tt++)
#pragma unroll
                        for (int hh = 0; hh < VT / 4; hh++) {
                            fma2s(acc[i][4 * hh], acc[i][4 * hh + 1], f[tt], x[tt][hh].x, x[tt][hh].y);
                            fma2s(acc[i][4 * hh + 2], acc[i][4 * hh + 3], f[tt], x[tt][hh].z, x[tt][hh].w);
                        }
                }
            }
        }
        int pn = p, kn = k0;
        advance(pn, kn);
        if (pn != p) {
#pragma unroll
            for (int i = 0; i < TR; i++)
#pragma unroll
                for (int c = 0; c < VT; c++) acc64[i][c] += (double)acc[i][c], acc[i][c] = 0.0f;
        }
        __syncthreads();  // this buffer is refilled NS - 1 stages on
        p = pn;
        k0 = kn;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
    for (int i = 0; i < TR; i++) {
        const int row = rg * TR + i;
        if (row < s)
#pragma unroll
            for (int c = 0; c < VT; c++) {
                const int j = cg * VT + c;
                if (j < nrhs) Y[perm1[tr0 + row] + (size_t)j * ldy] = acc64[i][c];
            }
    }
}

// mixed storage, 8, 16 or 32 vectors per pass
template <int R>
static hmg_status launch_multi_mixed(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy,
                                     float* xm, float* tm)
{
    cudaStream_t s = h->stream;
    constexpr int LGR = R == 32 ? 5 : (R == 16 ? 4 : 3);
    k_gather_multi<float><<<ceil_div((long long)h->n[1] * R, 256), 256, 0, s>>>(X, ldx, nrhs, h->perm[1], h->n[1],
                                                                                LGR, xm);
    HMG_LAUNCH_CHECK();
    const K1Desc* dd = static_cast<const K1Desc*>(h->k1_units);
    const int cnt[3] = {h->k1_count[0], h->k1_count[1], h->k1_count[2]};
    int first = 0;
    for (int tier = 0; tier < 3; tier++) {
        if (cnt[tier] > 0) {
            const int grid = std::min(ceil_div(cnt[tier], 8), h->nsm * 3);
            if (tier == 0) {
                HMG_CUDA_TRY(cudaFuncSetAttribute(k_vtx_multi_smem<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K1M_SMEM));
                k_vtx_multi_smem<R, 0><<<grid, 256, K1M_SMEM, s>>>(dd + first, cnt[tier], xm, tm);
            } else if (tier == 1) {
                HMG_CUDA_TRY(cudaFuncSetAttribute(k_vtx_multi_smem<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K1M_SMEM));
                k_vtx_multi_smem<R, 1><<<grid, 256, K1M_SMEM, s>>>(dd + first, cnt[tier], xm, tm);
            } else {
                HMG_CUDA_TRY(cudaFuncSetAttribute(k_vtx_multi_smem<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K1M_SMEM));
                k_vtx_multi_smem<R, 2><<<grid, 256, K1M_SMEM, s>>>(dd + first, cnt[tier], xm, tm);
            }
            HMG_LAUNCH_CHECK();
        }
        first += cnt[tier];
    }
    if (h->ntiles > 0) {
        constexpr int VT = R == 8 ? 8 : 4;
        HMG_CUDA_TRY(cudaFuncSetAttribute(k_tile_multi_mixed<R, VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)mixed_tile_smem<R>()));
        k_tile_multi_mixed<R, VT><<<h->ntiles, 1024 / VT, mixed_tile_smem<R>(), s>>>(
            static_cast<const PairDesc*>(h->pair_desc), h->tile_pair_start, h->tile_r0, h->tile_s, h->perm[0], xm, tm,
            static_cast<const char*>(h->tbuf), nrhs, Y, ldy);
        HMG_LAUNCH_CHECK();
    }
    return HMG_OK;
}

static hmg_status multi_mixed(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    int R = 8;
    while (R < nrhs) R <<= 1;
    if ((st = ensure_desc(h, 4))) return st;
    float* xm = nullptr;
    float* tm = nullptr;
    if ((st = dalloc(&xm, (size_t)h->n[1] * R, s)) || (st = dalloc(&tm, (size_t)(h->rank_total + 1) * R, s))) {
        dfree(xm, s);
        return st;
    }
    switch (R) {
    case 8: st = launch_multi_mixed<8>(h, nrhs, X, ldx, Y, ldy, xm, tm); break;
    case 16: st = launch_multi_mixed<16>(h, nrhs, X, ldx, Y, ldy, xm, tm); break;
    default: st = launch_multi_mixed<32>(h, nrhs, X, ldx, Y, ldy, xm, tm); break;
    }
    dfree(xm, s);
    dfree(tm, s);
    return st;
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
        const K1Desc* dd = static_cast<const K1Desc*>(h->k1_units);
        if constexpr (sizeof(S) == 4 && R >= 8) {
            HMG_CUDA_TRY(cudaFuncSetAttribute(k_vtx_multi_smem<R, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)K1M_SMEM));
            k_vtx_multi_smem<R, 0><<<std::min(ceil_div(n0, 8), h->nsm * 3), 256, K1M_SMEM, s>>>(dd, n0, xm, tm);
        }
        else
            k_vtx_multi<S, R><<<std::min(ceil_div(n0, 8), h->nsm * 8), 256, 0, s>>>(dd, n0, xm, tm);
        HMG_LAUNCH_CHECK();
    }
    if (h->ntiles > 0) {
        const PairDesc* pd = static_cast<const PairDesc*>(h->pair_desc);
        const char* tb = static_cast<const char*>(h->tbuf);
        if constexpr (sizeof(S) == 4 && R >= 8)
            k_tile_multi_smem<R><<<h->ntiles, 256, 0, s>>>(pd, h->tile_pair_start, h->tile_r0, h->tile_s,
                                                           h->perm[0], xm, tm, tb, nrhs, Y, ldy, -1);
        else
            k_tile_multi<S, R><<<h->ntiles, 256, 0, s>>>(pd, h->tile_pair_start, h->tile_r0, h->tile_s,
                                                         h->perm[0], xm, tm, tb, nrhs, Y, ldy);
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

// Y = the near-field part of H X for up to 32 vectors, FP32 stored near field, FP32
// products summed in FP64 (the tensor-core path with its near field on the CUDA cores)
hmg_status launch_tile_multi32_dense(hmg_matrix* h, const float* xm, int nrhs, double* Y, int ldy)
{
    if (h->ntiles <= 0) return HMG_OK;
    k_tile_multi_smem<32><<<h->ntiles, 256, 0, h->stream>>>(
        static_cast<const PairDesc*>(h->pair_desc), h->tile_pair_start, h->tile_r0, h->tile_s, h->perm[0], xm,
        nullptr, static_cast<const char*>(h->tbuf), nrhs, Y, ldy, PAIR_STORED);
    HMG_LAUNCH_CHECK();
    return HMG_OK;
}

void launch_gather_multi32(hmg_matrix* h, const double* X, int ldx, int nrhs, float* xm)
{
    k_gather_multi<float><<<ceil_div((long long)h->n[1] * 32, 256), 256, 0, h->stream>>>(X, ldx, nrhs, h->perm[1],
                                                                                        h->n[1], 5, xm);
}

hmg_status matvec_multi(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    // tensor cores, operands converted on chip from the stored factors and near field;
    // a pass costs about the same for 2 to 32 vectors, so fewer than tcm_min_nrhs
    // (hmg_set_tensor_core_min_vectors; 17: the CUDA-core kernels below take up to 16
    // vectors a pass faster, and 17 to 32 at the cost of 32) run on the CUDA cores
    if (h->tcm_ready && nrhs >= 2 && nrhs >= h->tcm_min_nrhs && h->arith_prec == HMG_PREC_FP32 &&
        (h->ndense == 0 || (h->near_mode == HMG_NEAR_STORED && h->near_prec == HMG_PREC_FP32)))
        return matvec_multi_tcm(h, nrhs, X, ldx, Y, ldy);
    // tensor cores: a BF16 copy of the FP32 factors and an FP32 stored near field (up to 64 vectors a pass)
    if (h->tc_ready && nrhs >= 2 && h->far_prec == HMG_PREC_FP32 && h->near_mode == HMG_NEAR_STORED &&
        (h->ndense == 0 || h->near_prec == HMG_PREC_FP32) && h->arith_prec == HMG_PREC_FP32)
        return matvec_multi_tc(h, nrhs, X, ldx, Y, ldy);
    if (nrhs > 32) {  // the CUDA-core kernels take 32 vectors a pass
        hmg_status st = matvec_multi(h, 32, X, ldx, Y, ldy);
        return st ? st : matvec_multi(h, nrhs - 32, X + (size_t)32 * ldx, ldx, Y + (size_t)32 * ldy, ldy);
    }
    if (nrhs > 1 && h->far_prec == HMG_PREC_MIXED && h->near_mode == HMG_NEAR_STORED &&
        (h->ndense == 0 || h->near_prec == HMG_PREC_FP32) && h->arith_prec == HMG_PREC_FP32)
        return multi_mixed(h, nrhs, X, ldx, Y, ldy);
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
