// tcm.cu -- multi-vector products on the tensor cores with operands converted on chip
// from the stored H-matrix (hmg_build_tensor_core_operands with HMG_PREC_BF16X6_ONCHIP).
//
// tc.cu multiplies BF16 copies of the factors and near field that sit beside the FP32
// storage; with three parts (24 bits) those copies take 1.73x the FP32 bytes, so at
// N = 2^20 they do not fit.  Here nothing is copied: the pass kernels read the
// handle's own storage -- FP32 near-field slices and FP32 or mixed FP32 / FP16 / FP8
// factors (the layouts of hmg_internal.cuh) -- and converter warps split every value
// into three BF16 parts (hi, the rounding of what hi misses, the rounding of what both
// miss) in shared memory, in the canonical K-major core layout of the MMA:
//
//   pass 1 (k_tcm_pass<0>): per stack of V_b^T with the same columns (M = stacked
//     terms <= 128, K = the columns, N = the vectors): t_b = V_b^T X_b, times the
//     terms' scales (FP16 / FP8 terms are stored scaled), written as BF16 operand cores
//     of pass 2 (three parts);
//   pass 2 (k_tcm_pass<1>): per row tile (M = 128 rows), the sum over its pairs of
//     U_slice t_b (K = terms) and D_slice X_b (K = columns), written to Y rows.
//
// A step is 32 K positions (4 K cores) of one pair or stack.  Roles of a CTA (one per
// SM, persistent, 10 warps):
//   warps 6-9, the converters: warp g converts the steps i = g (mod 4) into stage i mod
//     5 -- coalesced loads from HBM (several items' loads in flight per lane), the 3-part
//     split on the CUDA cores, 16-byte shared stores, a proxy fence, then an arrival on
//     the stage's "full" barrier; four steps' loads are in flight per SM;
//   warp 4, lane 0: the B operand of each step (3-part X or t_b cores, mostly L2) by one
//     bulk copy into the same stage, counted on the same barrier;
//   warp 5, lane 0: the MMAs of a step (per K16: hi*hi into one accumulator and the
//     correction terms into another -- 5 of them when the step holds FP32 values, 2 when
//     it holds FP16 terms only, none for FP8 terms only, whose BF16 parts are exact with
//     fewer), then tcgen05.commit frees the stage and signals the accumulators;
//   warps 0-3: drain both accumulators after every step (tcgen05.ld) and keep the sums
//     in FP32 registers, so no tensor-core accumulation runs longer than one step.
// Every wait is bounded (pipeline.cuh); on a time-out the CTA records an error code in
// the handle's flag, waits for its own copies and MMAs and frees tensor memory.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <queue>
#include <vector>

#include "hmg_matrix.cuh"
#include "pipeline.cuh"
#include "stream.cuh"
#include "tc_common.cuh"

namespace hmg {

static constexpr int TCM_NMAX = 64;                         // vectors per pass at most
static constexpr int TCM_STAGES = 5;                        // stages of the converted-operand ring
static constexpr int TCM_KC = 4;                            // K cores per step (32 K positions)
static constexpr int TCM_PARTS = 3;                         // BF16 parts of every operand
static constexpr int TCM_AST = TCM_KC * TCM_PARTS * 16 * 128;        // A of a step: 128 rows, 24 KB
static constexpr int TCM_BST = TCM_KC * TCM_PARTS * TCM_NMAX * 16;   // B of a step at 64 vectors, 12 KB
static constexpr int TCM_GROUPS = 4;                        // converter groups (steps in conversion at once)
static constexpr int TCM_GWARPS = 1;                        // warps per converter group
static constexpr int TCM_THREADS = (6 + TCM_GROUPS * TCM_GWARPS) * 32;
static constexpr int TCM_MAXMEM = 8;                        // blocks of a pass-1 stack (ranks rounded to 16)

struct TcmStep {
    long long b_kc;  // first K core of B in the operand buffer (X cores, then t_b cores)
    int src;         // pass 1: stack index; pass 2: pair index
    int kp0;         // first K position of the step
    int meta;        // bits 0-1: K16 groups (1 or 2); bit 8: first step of a job; bit 9: last;
                     // bits 12-15: MMAs per K16 (1, 3 or 6)
    int rows;        // rows of the job's M (tile rows or stack rows)
};
static_assert(sizeof(TcmStep) == 24, "TcmStep layout");

// pass-1 job: the V^T of blocks with the same columns, one under the other
struct TcmStack {
    int c0, m2, rows, nmem;
    int blk[TCM_MAXMEM];
    int off[TCM_MAXMEM];  // first stack row of each block (a multiple of 16)
};

struct TcmJob {
    int r0;    // pass 2: first Z row of the tile; pass 1: the stack
    int rows;  // pass 2: rows of the tile; pass 1: stack rows
};

struct TcmSmem {
    unsigned char a[TCM_STAGES][TCM_AST];
    unsigned char b[TCM_STAGES][TCM_BST];
    __nv_bfloat16 stg[4][32 * TCM_NMAX];  // pass 1 epilogue: 4 K cores of t_b per warp
    uint64_t full[TCM_STAGES], empty[TCM_STAGES], accf[2], acce[2], fin;
    uint32_t tmem;
    int fail;
};
static_assert(sizeof(TcmSmem) <= 227 * 1024, "TcmSmem exceeds the shared memory of a CTA");

// ---------------------------------------------------------------------------
// decoding the stored values
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fp8_value(unsigned byte)
{
    const __half_raw h = __nv_cvt_fp8_to_halfraw((__nv_fp8_storage_t)byte, __NV_E4M3);
    return __half2float(__half(h));
}

__device__ __forceinline__ float half_value(unsigned word, int hi)
{
    const unsigned short u = (unsigned short)(hi ? word >> 16 : word & 0xffffu);
    __half_raw r;
    r.x = u;
    return __half2float(__half(r));
}

// the three BF16 parts of 8 values of one operand row, one uint4 (8 K positions) each
__device__ __forceinline__ void split3(const float (&v)[8], uint4& p0, uint4& p1, uint4& p2)
{
    uint32_t w0[4], w1[4], w2[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float a = v[2 * k], b = v[2 * k + 1];
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        const float2 hf = __bfloat1622float2(h);
        const float ra = a - hf.x, rb = b - hf.y;
        const __nv_bfloat162 l = __floats2bfloat162_rn(ra, rb);
        const float2 lf = __bfloat1622float2(l);
        const __nv_bfloat162 l2 = __floats2bfloat162_rn(ra - lf.x, rb - lf.y);
        w0[k] = *reinterpret_cast<const uint32_t*>(&h);
        w1[k] = *reinterpret_cast<const uint32_t*>(&l);
        w2[k] = *reinterpret_cast<const uint32_t*>(&l2);
    }
    p0 = make_uint4(w0[0], w0[1], w0[2], w0[3]);
    p1 = make_uint4(w1[0], w1[1], w1[2], w1[3]);
    p2 = make_uint4(w2[0], w2[1], w2[2], w2[3]);
}

// row `m` of K core `kc` of a step's A stage: part q at ((kc * 3 + q) * 16 + m / 8) * 128 + (m % 8) * 16
__device__ __forceinline__ void store_row(unsigned char* stage, int kc, int m, const float (&v)[8])
{
    uint4 p0, p1, p2;
    split3(v, p0, p1, p2);
    unsigned char* base = stage + ((size_t)(kc * TCM_PARTS) * 16 + (m >> 3)) * 128 + (m & 7) * 16;
    *reinterpret_cast<uint4*>(base) = p0;
    *reinterpret_cast<uint4*>(base + 16 * 128) = p1;
    *reinterpret_cast<uint4*>(base + 2 * 16 * 128) = p2;
}

// Pass 2: a converter warp's items of a step, an item being 4 consecutive rows of one
// K core (8 K positions x 4 rows, one 16-byte load per K position).  Near slices are
// FP32 column-major (s_pad rows, column j at K position a + j, a = c0 mod 8); U slices
// are chunk columns of s_pad * 4 bytes: r32 FP32 terms, r16 / 2 FP16 pairs, r8 / 4 FP8
// quads.  Two items per lane are loaded before either is converted (16 loads in flight).
__device__ __forceinline__ void convert_pass2(const PairDesc& d, int rows, int kp0, int nkc, unsigned char* stage,
                                              int lane)
{
    const int sp = (rows + 3) & ~3, nq = sp >> 2, n = nq * nkc;
    const bool near = d.kind == PAIR_STORED;
    const bool mixed = d.kind == PAIR_FAR_MIXED;
    const int a = d.c0 & 7, m2 = d.ncol;
    const int r32 = d.ncol, r16 = mixed ? d.c0 : 0, r = r32 + r16 + (mixed ? d.pad : 0);
    const char* slice = static_cast<const char*>(d.data);
    const char* s16 = slice + (size_t)sp * 4 * r32;
    const char* s8 = s16 + (size_t)sp * 2 * r16;
    // tier of K position kp: 0 FP32 (or near), 1 FP16, 2 FP8, 3 none (zero)
    auto tier_of = [&](int kp) -> int {
        if (near) return (kp - a >= 0 && kp - a < m2) ? 0 : 3;
        return kp < r32 ? 0 : (kp < r32 + r16 ? 1 : (kp < r ? 2 : 3));
    };
    for (int base = 0; base < n; base += 64) {
        uint4 w[2][8];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int it = base + 32 * u + lane;
            const int kc = it / nq, i4 = it - kc * nq;
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int kp = kp0 + kc * 8 + e, t = it < n ? tier_of(kp) : 3;
                const char* p = nullptr;
                if (t == 0) p = near ? slice + ((size_t)(kp - a) * sp + 4 * i4) * 4 : slice + ((size_t)kp * sp + 4 * i4) * 4;
                else if (t == 1) p = s16 + ((size_t)((kp - r32) >> 1) * sp + 4 * i4) * 4;
                else if (t == 2) p = s8 + ((size_t)((kp - r32 - r16) >> 2) * sp + 4 * i4) * 4;
                w[u][e] = t == 0 ? ld_stream(p) : (t < 3 ? __ldg(reinterpret_cast<const uint4*>(p)) : make_uint4(0u, 0u, 0u, 0u));
            }
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int it = base + 32 * u + lane;
            if (it >= n) continue;
            const int kc = it / nq, i4 = it - kc * nq;
            float v[4][8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int kp = kp0 + kc * 8 + e, t = tier_of(kp);
                const unsigned ww[4] = {w[u][e].x, w[u][e].y, w[u][e].z, w[u][e].w};
                const int q = t == 1 ? ((kp - r32) & 1) : ((kp - r32 - r16) & 3);
#pragma unroll
                for (int ii = 0; ii < 4; ii++)
                    v[ii][e] = t == 0 ? __uint_as_float(ww[ii])
                                      : (t == 1 ? half_value(ww[ii], q) : (t == 2 ? fp8_value((ww[ii] >> (8 * q)) & 255u) : 0.0f));
            }
#pragma unroll
            for (int ii = 0; ii < 4; ii++)
                if (4 * i4 + ii < rows) store_row(stage, kc, 4 * i4 + ii, v[ii]);
        }
    }
}

// Pass 1: items are (stack row, K core): 8 columns of one term of V_b^T, read as three
// aligned 16-byte quads of 32-bit words (columns j0 - sh .. j0 - sh + 11, sh = j0 mod 4,
// the same for the whole step).  V_b^T holds r32 FP32 rows of m2p words, then r16 / 2
// FP16 pair rows (word (g m2p + j) holds column j of terms 2g, 2g+1), then r8 / 4 FP8
// quad rows (word (g m2p + j): column j of terms 4g..4g+3).  Four items per lane are
// loaded before any is converted.
__device__ __forceinline__ void convert_pass1(const TcmStack& sk, void* const* ptrV, const int* rank,
                                              const int* tier32, const int* tier16, int kp0, int nkc,
                                              unsigned char* stage, int lane)
{
    const int a = sk.c0 & 7, m2 = sk.m2, m2p = (m2 + 3) & ~3, n = sk.rows * nkc;
    const int sh = (4 - (a & 3)) & 3;  // j0 mod 4 for every item (kp0 and 8 kc are multiples of 4)
    for (int base = 0; base < n; base += 128) {
        uint4 w[4][3];
        int tier[4], sel[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int it = base + 32 * u + lane;
            const int m = it / nkc, kc = it - m * nkc;
            tier[u] = 3;
            sel[u] = 0;
            const uint4* row = nullptr;
            if (it < n) {
                int k = 0;
                while (k + 1 < sk.nmem && sk.off[k + 1] <= m) k++;
                const int b = sk.blk[k], l = m - sk.off[k];
                const int r = rank[b], r32 = tier32[b], r16 = tier16[b];
                const char* V = static_cast<const char*>(ptrV[b]);
                if (l < r32) {
                    tier[u] = 0;
                    row = reinterpret_cast<const uint4*>(V + (size_t)l * m2p * 4);
                } else if (l < r32 + r16) {
                    tier[u] = 1;
                    sel[u] = (l - r32) & 1;
                    row = reinterpret_cast<const uint4*>(V + (size_t)r32 * m2p * 4 + (size_t)((l - r32) >> 1) * m2p * 4);
                } else if (l < r) {
                    tier[u] = 2;
                    sel[u] = (l - r32 - r16) & 3;
                    row = reinterpret_cast<const uint4*>(V + (size_t)r32 * m2p * 4 + (size_t)r16 * m2p * 2 +
                                                         (size_t)((l - r32 - r16) >> 2) * m2p * 4);
                }
            }
            const int qs = kp0 + kc * 8 - a - sh;  // first column of the first quad (a multiple of 4)
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const int c = qs + 4 * k;
                w[u][k] = (row && c >= 0 && c < m2p) ? __ldg(row + (c >> 2)) : make_uint4(0u, 0u, 0u, 0u);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int it = base + 32 * u + lane;
            if (it >= n) continue;
            const int m = it / nkc, kc = it - m * nkc;
            const int j0 = kp0 + kc * 8 - a;
            const unsigned words[12] = {w[u][0].x, w[u][0].y, w[u][0].z, w[u][0].w, w[u][1].x, w[u][1].y,
                                        w[u][1].z, w[u][1].w, w[u][2].x, w[u][2].y, w[u][2].z, w[u][2].w};
            float v[8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                // sh is the same for every lane: the compiler selects among four unrolled copies
                unsigned wd;
                switch (sh) {
                case 0: wd = words[e]; break;
                case 1: wd = words[e + 1]; break;
                case 2: wd = words[e + 2]; break;
                default: wd = words[e + 3]; break;
                }
                const bool in = j0 + e >= 0 && j0 + e < m2;
                const int t = in ? tier[u] : 3;
                v[e] = t == 0 ? __uint_as_float(wd)
                              : (t == 1 ? half_value(wd, sel[u]) : (t == 2 ? fp8_value((wd >> (8 * sel[u])) & 255u) : 0.0f));
            }
            store_row(stage, kc, m, v);
        }
    }
}

// the scale of stack row m's term (FP16 / FP8 terms of mixed storage), else 1
__device__ __forceinline__ float stack_scale(const TcmStack& sk, void* const* ptrV, const int* rank, const int* tier32,
                                             const int* tier16, int m)
{
    int k = 0;
    while (k + 1 < sk.nmem && sk.off[k + 1] <= m) k++;
    const int b = sk.blk[k], l = m - sk.off[k];
    const int r = rank[b], r32 = tier32[b], r16 = tier16[b];
    if (l < r32 || l >= r) return 1.0f;
    const size_t m2p = (sk.m2 + 3) & ~3;
    const char* V = static_cast<const char*>(ptrV[b]);
    const float* scal = reinterpret_cast<const float*>(V + m2p * (4 * (size_t)r32 + 2 * (size_t)r16 + (size_t)(r - r32 - r16)));
    return scal[l];
}

// ---------------------------------------------------------------------------
// the pass kernel
// ---------------------------------------------------------------------------
// Steps of CTA c: [cta[c].y, cta[c+1].y); its jobs: [cta[c].x, cta[c+1].x).  MODE 0
// (pass 1) writes t_b cores: K core kc of stack j to B K core tb_kc + map[16 j + kc];
// MODE 1 (pass 2) writes tile row i to Y row map[r0 + i].
template <int MODE, int NV>
__global__ void __launch_bounds__(TCM_THREADS, 1)
    k_tcm_pass(const TcmStep* __restrict__ steps, const TcmJob* __restrict__ jobs, const int2* __restrict__ cta,
               const PairDesc* __restrict__ desc, const TcmStack* __restrict__ stacks, void* const* ptrV,
               const int* __restrict__ rank, const int* __restrict__ tier32, const int* __restrict__ tier16,
               char* Bbuf, long long tb_kc, const int* __restrict__ map, int nrhs, double* Y, int ldy, int* err)
{
    constexpr int P = TCM_PARTS;
    constexpr int KB = NV * 16 * P;  // bytes of a B K core, all parts
    constexpr int TMEM_COLS = 4 * NV;  // two buffers of hi*hi and correction accumulators
    extern __shared__ __align__(1024) unsigned char tcm_raw[];
    TcmSmem& sm = *reinterpret_cast<TcmSmem*>(tcm_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int2 lo = cta[blockIdx.x], hi = cta[blockIdx.x + 1];
    const int nsteps = hi.y - lo.y;
    const TcmStep* my_steps = steps + lo.y;
    volatile int* fail = &sm.fail;
    if (tid == 0) {
        for (int s = 0; s < TCM_STAGES; s++) {
            mbar_init(&sm.full[s], 1 + TCM_GWARPS);
            mbar_init(&sm.empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&sm.accf[b], 1);
            mbar_init(&sm.acce[b], 4);
        }
        mbar_init(&sm.fin, 1);
        sm.fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)),
                     "n"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem;

    if (warp >= 6) {
        // ---- converters: group g takes steps g, g + 4, ... ----
        const int g = (warp - 6) / TCM_GWARPS, gt = tid - (6 + g * TCM_GWARPS) * 32;
        for (int i = g; i < nsteps; i += TCM_GROUPS) {
            const int slot = i % TCM_STAGES;
            if (i >= TCM_STAGES) {
                bool ok = true;
                if (lane == 0) ok = !*fail && mbar_wait(&sm.empty[slot], ((i / TCM_STAGES) - 1) & 1, err, 21);
                if (!__shfl_sync(~0u, ok, 0)) {
                    *fail = 1;
                    break;
                }
            }
            const TcmStep st = my_steps[i];
            const int nkc = 2 * (st.meta & 3);
            if (MODE == 1)
                convert_pass2(desc[st.src], st.rows, st.kp0, nkc, sm.a[slot], gt);
            else
                convert_pass1(stacks[st.src], ptrV, rank, tier32, tier16, st.kp0, nkc, sm.a[slot], gt);
            // the generic-proxy stores become visible to the tensor cores' (async) proxy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.full[slot]);
        }
    } else if (warp == 4) {
        // ---- B operand of every step: one bulk copy, lane 0 ----
        if (lane == 0) {
            int issued = 0;
            for (int i = 0; i < nsteps; i++) {
                const int slot = i % TCM_STAGES;
                if (i >= TCM_STAGES &&
                    (*fail || !mbar_wait(&sm.empty[slot], ((i / TCM_STAGES) - 1) & 1, err, 22))) {
                    *fail = 1;
                    break;
                }
                const TcmStep st = my_steps[i];
                const unsigned bytes = (unsigned)(2 * (st.meta & 3)) * KB;
                mbar_arrive_expect_tx(&sm.full[slot], bytes);
                bulk_g2s(sm.b[slot], Bbuf + st.b_kc * KB, bytes, &sm.full[slot]);
                issued++;
            }
            // the last copy into every stage has landed before the CTA leaves
            for (int s = 0; s < TCM_STAGES && s < issued; s++)
                mbar_wait(&sm.full[s], ((issued - 1 - s) / TCM_STAGES) & 1, err, 23);
        }
        __syncwarp();
    } else if (warp == 5) {
        // ---- MMAs, lane 0 ----
        if (lane == 0) {
            constexpr uint32_t LBA = P * 16 * 128, LBB = KB;  // K-core strides of A and B
            for (int i = 0; i < nsteps; i++) {
                const int slot = i % TCM_STAGES, buf = i & 1;
                if (*fail || !mbar_wait(&sm.full[slot], (i / TCM_STAGES) & 1, err, 24)) {
                    *fail = 1;
                    break;
                }
                if (i >= 2) {  // the epilogue has read this buffer's previous step
                    if (!mbar_wait(&sm.acce[buf], ((i >> 1) - 1) & 1, err, 25)) {
                        *fail = 1;
                        break;
                    }
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const int meta = my_steps[i].meta, nk = meta & 3, mode = (meta >> 12) & 15;
                const uint32_t d = tmem + (uint32_t)(buf * 2 * NV);
                uint64_t ad = smem_desc(smem_u32(sm.a[slot]), LBA, 128), bd = smem_desc(smem_u32(sm.b[slot]), LBB, 128);
                const uint64_t da = (2 * LBA) >> 4, db = (2 * LBB) >> 4;
                const uint64_t alo = (16 * 128) >> 4, blo = (NV * 16) >> 4;  // part q: + q alo / q blo
                for (int k = 0; k < nk; k++) {
                    const uint32_t acc = k > 0 ? 1u : 0u;
                    tc_mma(d, ad, bd, tc_idesc<NV>(), acc);
                    if (mode >= 3) {
                        tc_mma(d + NV, ad, bd + blo, tc_idesc<NV>(), acc);
                        tc_mma(d + NV, ad + alo, bd, tc_idesc<NV>(), 1u);
                    }
                    if (mode >= 6) {
                        tc_mma(d + NV, ad, bd + 2 * blo, tc_idesc<NV>(), 1u);
                        tc_mma(d + NV, ad + 2 * alo, bd, tc_idesc<NV>(), 1u);
                        tc_mma(d + NV, ad + alo, bd + blo, tc_idesc<NV>(), 1u);
                    }
                    ad += da;
                    bd += db;
                }
                tc_commit(&sm.empty[slot]);
                tc_commit(&sm.accf[buf]);
            }
            tc_commit(&sm.fin);  // every MMA issued here has completed before tensor memory is freed
            mbar_wait(&sm.fin, 0, err, 26);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w owns accumulator rows 32w..32w+31 ----
        const int row = warp * 32 + lane;
        float f[NV];
        const int njobs = hi.x - lo.x;
        const TcmJob* my_jobs = jobs + lo.x;
        int jc = 0, rows = 0, yrow = 0, tdst[4] = {0, 0, 0, 0};
        float scale = 1.0f;
        bool ok = true;
        for (int i0 = 0; i0 < nsteps && ok; i0 += 32) {
            const int mt = i0 + lane < nsteps ? my_steps[i0 + lane].meta : 0;
            const int cnt = min(32, nsteps - i0);
            for (int k = 0; k < cnt; k++) {
                const int i = i0 + k, meta = __shfl_sync(~0u, mt, k), buf = i & 1;
                const bool first = meta & 256, last = meta & 512;
                const int mode = (meta >> 12) & 15;
                if (first) {
                    const TcmJob jb = jc < njobs ? my_jobs[jc] : TcmJob{0, 0};
                    rows = jb.rows;
                    if (MODE == 1) {
                        yrow = row < rows ? map[jb.r0 + row] : 0;
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            tdst[q] = (warp * 4 + q < (rows >> 3)) ? map[jb.r0 * 16 + warp * 4 + q] : 0;
                        scale = row < rows ? stack_scale(stacks[jb.r0], ptrV, rank, tier32, tier16, row) : 1.0f;
                    }
                }
                if (!__all_sync(~0u, !*fail && mbar_wait(&sm.accf[buf], (i >> 1) & 1, err, 27))) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t taddr = tmem + (uint32_t)(buf * 2 * NV) + ((uint32_t)(warp * 32) << 16);
                // 16 columns at a time: the running sums f[NV] stay in registers beside them
#pragma unroll
                for (int h = 0; h < NV / 16; h++) {
                    uint32_t v[16], c[16];
                    tc_ld16(taddr + 16 * h, v);
                    if (mode > 1) tc_ld16(taddr + NV + 16 * h, c);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int q = 0; q < 16; q++) {
                        const float tv = __uint_as_float(v[q]) + (mode > 1 ? __uint_as_float(c[q]) : 0.0f);
                        f[16 * h + q] = first ? tv : f[16 * h + q] + tv;
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&sm.acce[buf]);
                if (!last) continue;
                jc++;
                if (MODE == 1) {
                    if (row < rows) {
                        double* y = Y + yrow;
#pragma unroll
                        for (int q = 0; q < NV; q++)
                            if (q < nrhs) y[(size_t)q * ldy] = (double)f[q];
                    }
                } else {
                    // term row -> 3-part B cores of pass 2 (see tc.cu's pass-1 epilogue):
                    // lanes 2p, 2p+1 pair their terms into 32-bit words; staging row u
                    // (K core u / NV, vector u % NV) at u ^ (2 (u / NV)) spreads the banks
                    uint32_t* stg = reinterpret_cast<uint32_t*>(sm.stg[warp]);
                    const bool odd = lane & 1;
#pragma unroll
                    for (int q = 0; q < NV; q++) f[q] *= scale;
#pragma unroll
                    for (int part = 0; part < P; part++) {
#pragma unroll
                        for (int t = 0; t < NV / 2; t++) {
                            float v0 = f[2 * t], v1 = f[2 * t + 1];
#pragma unroll
                            for (int pp = 0; pp < part; pp++) {
                                v0 -= __bfloat162float(__float2bfloat16_rn(v0));
                                v1 -= __bfloat162float(__float2bfloat16_rn(v1));
                            }
                            const float x = __shfl_xor_sync(~0u, odd ? v0 : v1, 1);
                            const int q = odd ? 2 * t + 1 : 2 * t;
                            const uint32_t w = odd ? pack_bf16(x, v1) : pack_bf16(v0, x);
                            const int u = (lane >> 3) * NV + q;
                            stg[(u ^ ((lane >> 3) * 2)) * 4 + ((lane & 7) >> 1)] = w;
                        }
                        __syncwarp();
                        uint4* dst = reinterpret_cast<uint4*>(Bbuf);
                        const uint4* src = reinterpret_cast<const uint4*>(stg);
#pragma unroll
                        for (int it = 0; it < NV / 8; it++) {
                            // staging row u = it * 32 + lane: K core kcl (a constant after unrolling,
                            // NV being a multiple of 32), vector vq
                            constexpr int per = NV / 32;
                            const int kcl = it / per, vq = (it % per) * 32 + lane, u = it * 32 + lane;
                            if (warp * 4 + kcl < (rows >> 3))
                                dst[((size_t)(tb_kc + tdst[kcl]) * P + part) * NV + vq] = src[u ^ (kcl * 2)];
                        }
                        __syncwarp();
                    }
                }
            }
        }
        if (!ok) *fail = 1;
    }
    __syncthreads();
    if (warp == 5) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(TMEM_COLS));
    }
}

// ---------------------------------------------------------------------------
// host side: plan (once) and product
// ---------------------------------------------------------------------------
void free_tcm(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    if (h->tcm_bbuf) {
        cudaStreamSynchronize(s);  // a product in flight may still read it
        cudaFree(h->tcm_bbuf);
    }
    h->tcm_bbuf = nullptr;
    {
        char* p = static_cast<char*>(h->tcm_stacks);
        dfree(p, s);
        h->tcm_stacks = nullptr;
    }
    dfree(h->tcm_kmap, s);
    for (int q = 0; q < 2; q++) {
        dfree(h->tcm_steps[q], s);
        dfree(h->tcm_jobs[q], s);
        dfree(h->tcm_cta[q], s);
        h->tcm_njobs[q] = 0;
    }
    h->tcm_ready = false;
    h->tcm_xkc = h->tcm_tkc = 0;
    h->tcm_all_tiles = false;
}

namespace {

struct TcmPlan {
    std::vector<TcmStep> steps;
    std::vector<int> step0;  // per job: first step (then the end)
    std::vector<TcmJob> jobs;
    std::vector<double> cost;
    void begin(TcmJob j)
    {
        step0.push_back((int)steps.size());
        jobs.push_back(j);
        cost.push_back(0.0);
    }
    // K positions [0, kw) (a multiple of 16) of one source in steps of 32
    void add(int src, int kw, long long b_kc, int rows, int mode_of_first, int r32, int r16, bool far, double bytes_per_k)
    {
        for (int kp0 = 0; kp0 < kw; kp0 += 32) {
            const int nk = std::min(2, (kw - kp0) / 16);
            int mode = mode_of_first;
            if (far) mode = kp0 < r32 ? 6 : (kp0 < r32 + r16 ? 3 : 1);
            steps.push_back(TcmStep{b_kc + kp0 / 8, src, kp0, nk | (mode << 12), rows});
            cost.back() += bytes_per_k * 16 * nk + 2048.0 * mode * nk;
        }
    }
    void finish()
    {
        step0.push_back((int)steps.size());
        for (size_t j = 0; j + 1 < step0.size(); j++) {
            if (step0[j] == step0[j + 1]) continue;
            steps[step0[j]].meta |= 256;
            steps[step0[j + 1] - 1].meta |= 512;
        }
    }
};

// longest job first onto the least loaded CTA; steps and jobs CTA by CTA
hmg_status upload_plan(hmg_matrix* h, int q, const TcmPlan& L, int grid)
{
    cudaStream_t s = h->stream;
    const int nj = (int)L.jobs.size();
    std::vector<int> order;
    for (int j = 0; j < nj; j++)
        if (L.step0[j] < L.step0[j + 1]) order.push_back(j);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return L.cost[a] > L.cost[b]; });
    using Load = std::pair<double, int>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int c = 0; c < grid; c++) heap.push({0.0, c});
    std::vector<std::vector<int>> mine(grid);
    for (int j : order) {
        Load l = heap.top();
        heap.pop();
        mine[l.second].push_back(j);
        heap.push({l.first + L.cost[j] + 4096.0, l.second});
    }
    std::vector<TcmStep> steps;
    std::vector<TcmJob> jobs;
    std::vector<int2> cta(grid + 1);
    steps.reserve(L.steps.size());
    for (int c = 0; c < grid; c++) {
        cta[c] = make_int2((int)jobs.size(), (int)steps.size());
        for (int j : mine[c]) {
            jobs.push_back(L.jobs[j]);
            for (int i = L.step0[j]; i < L.step0[j + 1]; i++) steps.push_back(L.steps[i]);
        }
    }
    cta[grid] = make_int2((int)jobs.size(), (int)steps.size());
    hmg_status st;
    if ((st = dalloc(&h->tcm_steps[q], std::max(steps.size(), (size_t)1) * sizeof(TcmStep), s)) ||
        (st = dalloc(&h->tcm_jobs[q], std::max(jobs.size(), (size_t)1) * sizeof(TcmJob), s)) ||
        (st = dalloc(&h->tcm_cta[q], (size_t)(grid + 1) * sizeof(int2), s)))
        return st;
    if (!steps.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tcm_steps[q], steps.data(), steps.size() * sizeof(TcmStep), cudaMemcpyHostToDevice, s));
    if (!jobs.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tcm_jobs[q], jobs.data(), jobs.size() * sizeof(TcmJob), cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(h->tcm_cta[q], cta.data(), cta.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));  // the host vectors go out of scope
    h->tcm_njobs[q] = (int)jobs.size();
    return HMG_OK;
}

}  // namespace

hmg_status build_tcm(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    free_tc(h);  // also drops an earlier plan
    if (h->naca > 0 && h->far_prec != HMG_PREC_FP32 && h->far_prec != HMG_PREC_MIXED) {
        set_error("hmg_build_tensor_core_operands: on-chip operands need FP32 or mixed factors "
                  "(hmg_precompute_aca with HMG_PREC_FP32 or HMG_PREC_MIXED)");
        return HMG_ERR_STATE;
    }
    if (h->ndense > 0 && !(h->near_mode == HMG_NEAR_STORED && h->near_prec == HMG_PREC_FP32)) {
        set_error("hmg_build_tensor_core_operands: needs an FP32 stored near field (hmg_precompute_dense with HMG_PREC_FP32)");
        return HMG_ERR_STATE;
    }
    for (int b = h->ndense; b < h->nblocks; b++)
        if (((h->h_rank[b] + 15) & ~15) > 128) {
            set_error("hmg_build_tensor_core_operands: block %d has rank %d (> 128)", b, h->h_rank[b]);
            return HMG_ERR_UNSUPPORTED;
        }
    if ((st = ensure_desc(h, 4))) return st;
    const int np = h->npairs, nt = h->ntiles, nb = h->nblocks, grid = h->nsm;
    std::vector<int> tps(nt + 1), pblock(np), ts(nt), tr0(nt);
    HMG_CUDA_TRY(cudaMemcpy(tps.data(), h->tile_pair_start, sizeof(int) * (nt + 1), cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(pblock.data(), h->pair_block, sizeof(int) * np, cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(ts.data(), h->tile_s, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(tr0.data(), h->tile_r0, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    const bool mixed = h->far_prec == HMG_PREC_MIXED;
    const long long xkc = (h->n[1] + 7) / 8 + 4;  // X K cores (8 Z-ordered columns each), with slack
    // pass 1: stacks of blocks with the same columns, ranks rounded to 16, first fit
    std::vector<long long> toff(nb, -1);  // first 16-term group of each block's t_b
    long long tgroups = 0;
    std::vector<TcmStack> stacks;
    std::vector<int> kmap;
    TcmPlan p1, p2;
    {
        std::vector<int> far;
        for (int b = h->ndense; b < nb; b++)
            if (h->h_rank[b] > 0) far.push_back(b);
        std::stable_sort(far.begin(), far.end(), [&](int x, int y) {
            if (h->h_c0[x] != h->h_c0[y]) return h->h_c0[x] < h->h_c0[y];
            if (h->h_m2[x] != h->h_m2[y]) return h->h_m2[x] < h->h_m2[y];
            return h->h_rank[x] > h->h_rank[y];
        });
        for (size_t g0 = 0; g0 < far.size();) {
            size_t g1 = g0;
            while (g1 < far.size() && h->h_c0[far[g1]] == h->h_c0[far[g0]] && h->h_m2[far[g1]] == h->h_m2[far[g0]]) g1++;
            std::vector<std::vector<int>> members;
            std::vector<int> fill;
            for (size_t i = g0; i < g1; i++) {
                const int b = far[i], r16 = (h->h_rank[b] + 15) & ~15;
                size_t k = 0;
                while (k < members.size() && fill[k] + r16 > 128) k++;
                if (k == members.size()) {
                    members.emplace_back();
                    fill.push_back(0);
                }
                members[k].push_back(b);
                fill[k] += r16;
            }
            const int c0 = h->h_c0[far[g0]], m2 = h->h_m2[far[g0]], kw = ((c0 & 7) + m2 + 15) & ~15;
            for (size_t k = 0; k < members.size(); k++) {
                TcmStack sk{};
                sk.c0 = c0;
                sk.m2 = m2;
                sk.rows = fill[k];
                sk.nmem = (int)members[k].size();
                const int job = (int)stacks.size();
                kmap.resize(kmap.size() + 16, 0);
                int off = 0;
                for (int u = 0; u < sk.nmem; u++) {
                    const int b = members[k][u], r16 = (h->h_rank[b] + 15) & ~15;
                    sk.blk[u] = b;
                    sk.off[u] = off;
                    toff[b] = tgroups;
                    for (int kc = 0; kc < r16 / 8; kc++) kmap[job * 16 + off / 8 + kc] = (int)(tgroups * 2 + kc);
                    tgroups += r16 / 16;
                    off += r16;
                }
                stacks.push_back(sk);
                p1.begin(TcmJob{job, sk.rows});
                p1.add(job, kw, c0 >> 3, sk.rows, 6, 0, 0, false, 4.0 * sk.rows);
            }
            g0 = g1;
        }
    }
    // pass 2: per tile, its near pairs (B = X) and low-rank pairs (B = t_b)
    bool all_tiles = true;
    for (int t = 0; t < nt; t++) {
        bool started = false;
        const int sp = (ts[t] + 3) & ~3;
        for (int p = tps[t]; p < tps[t + 1]; p++) {
            const int b = pblock[p];
            const bool dense = b < h->ndense;
            if (!dense && h->h_rank[b] == 0) continue;
            if (!started) {
                p2.begin(TcmJob{tr0[t], ts[t]});
                started = true;
            }
            if (dense) {
                const int a = h->h_c0[b] & 7, kw = (a + h->h_m2[b] + 15) & ~15;
                p2.add(p, kw, h->h_c0[b] >> 3, ts[t], 6, 0, 0, false, 4.0 * sp);
            } else {
                const int r = h->h_rank[b], r16 = (r + 15) & ~15;
                const int r32 = mixed ? h->h_r32[b] : r, rr16 = mixed ? h->h_r16[b] : 0;
                p2.add(p, r16, xkc + toff[b] * 2, ts[t], 6, r32, rr16, true, 4.0 * sp);
            }
        }
        all_tiles = all_tiles && started;
    }
    p1.finish();
    p2.finish();
    // every step's B copy inside the operand buffer, every row count within 128 rows
    const long long bkc = xkc + tgroups * 2;
    for (const TcmPlan* L : {&p1, &p2})
        for (const TcmStep& sp : L->steps) {
            const int nk = sp.meta & 3;
            if (nk < 1 || nk > 2 || sp.b_kc < 0 || sp.b_kc + 2 * nk > bkc || sp.rows < 1 || sp.rows > 128 ||
                sp.src < 0 || sp.src >= (L == &p1 ? (int)stacks.size() : np)) {
                set_error("hmg_build_tensor_core_operands: internal error: a converted-operand step leaves its buffers");
                return HMG_ERR_UNSUPPORTED;
            }
        }
    for (int v : kmap)
        if (v < 0 || v >= tgroups * 2) {
            set_error("hmg_build_tensor_core_operands: internal error: a t_b core lies outside its buffer");
            return HMG_ERR_UNSUPPORTED;
        }
    // operand buffer of a product: X cores then t_b cores, three parts, 64 vectors
    const size_t bbytes = (size_t)bkc * 16 * TCM_NMAX * TCM_PARTS;
    cudaError_t ce = cudaMalloc(&h->tcm_bbuf, bbytes);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        h->tcm_bbuf = nullptr;
        set_error("hmg_build_tensor_core_operands: allocating %zu bytes of X and t_b operands failed: %s", bbytes,
                  cudaGetErrorString(ce));
        return ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
    }
    if ((st = dalloc(reinterpret_cast<char**>(&h->tcm_stacks), std::max(stacks.size(), (size_t)1) * sizeof(TcmStack), s)) ||
        (st = dalloc(&h->tcm_kmap, std::max(kmap.size(), (size_t)1), s))) {
        free_tcm(h);
        return st;
    }
    if (!stacks.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tcm_stacks, stacks.data(), stacks.size() * sizeof(TcmStack), cudaMemcpyHostToDevice, s));
    if (!kmap.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tcm_kmap, kmap.data(), kmap.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    if ((st = upload_plan(h, 0, p1, grid)) || (st = upload_plan(h, 1, p2, grid))) {
        free_tcm(h);
        return st;
    }
    h->tcm_xkc = xkc;
    h->tcm_tkc = tgroups * 2;
    h->tcm_all_tiles = all_tiles;
    h->tcm_ready = true;
    return HMG_OK;
}

template <int NV>
static hmg_status tcm_product(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    cudaStream_t s = h->stream;
    char* bbuf = static_cast<char*>(h->tcm_bbuf);
    const long long xkc = h->tcm_xkc;
    k_tc_x<NV><<<(unsigned)((xkc * NV + 255) / 256), 256, 0, s>>>(X, ldx, nrhs, h->perm[1], h->n[1], xkc,
                                                                    reinterpret_cast<uint4*>(bbuf), TCM_PARTS);
    HMG_LAUNCH_CHECK();
    const size_t smem = sizeof(TcmSmem);
    HMG_CUDA_TRY(cudaFuncSetAttribute(k_tcm_pass<0, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HMG_CUDA_TRY(cudaFuncSetAttribute(k_tcm_pass<1, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const PairDesc* desc = static_cast<const PairDesc*>(h->pair_desc);
    const TcmStack* stacks = static_cast<const TcmStack*>(h->tcm_stacks);
    if (h->tcm_njobs[0] > 0) {
        k_tcm_pass<0, NV><<<h->nsm, TCM_THREADS, smem, s>>>(
            reinterpret_cast<const TcmStep*>(h->tcm_steps[0]), reinterpret_cast<const TcmJob*>(h->tcm_jobs[0]),
            reinterpret_cast<const int2*>(h->tcm_cta[0]), desc, stacks, h->ptrV, h->rank, h->tier32, h->tier16, bbuf,
            xkc, h->tcm_kmap, 0, nullptr, 0, h->dev_err);
        HMG_LAUNCH_CHECK();
    }
    if (!h->tcm_all_tiles)  // rows of tiles without products (all their blocks of rank 0) are zero
        HMG_CUDA_TRY(cudaMemset2DAsync(Y, sizeof(double) * ldy, 0, sizeof(double) * h->n[0], nrhs, s));
    if (h->tcm_njobs[1] > 0) {
        k_tcm_pass<1, NV><<<h->nsm, TCM_THREADS, smem, s>>>(
            reinterpret_cast<const TcmStep*>(h->tcm_steps[1]), reinterpret_cast<const TcmJob*>(h->tcm_jobs[1]),
            reinterpret_cast<const int2*>(h->tcm_cta[1]), desc, stacks, h->ptrV, h->rank, h->tier32, h->tier16, bbuf,
            0, h->perm[0], nrhs, Y, ldy, h->dev_err);
        HMG_LAUNCH_CHECK();
    }
    return HMG_OK;
}

// 2..64 vectors in one pass: MMAs of N = 32 for up to 32 vectors, N = 64 above
hmg_status matvec_multi_tcm(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    hmg_status st = ensure_desc(h, 4);  // the pair descriptors the converters read
    if (st) return st;
    return nrhs > 32 ? tcm_product<64>(h, nrhs, X, ldx, Y, ldy) : tcm_product<32>(h, nrhs, X, ldx, Y, ldy);
}

}  // namespace hmg
