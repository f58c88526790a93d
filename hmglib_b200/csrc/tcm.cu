// tcm.cu -- multi-vector products on the tensor cores with operands converted on chip
// from the stored H-matrix (hmg_build_tensor_core_operands with HMG_PREC_BF16X6_ONCHIP).
//
// tc.cu multiplies BF16 copies of the factors and near field that sit beside the FP32
// storage; with three parts (24 bits) those copies take 1.73x the FP32 bytes, so at
// N = 2^20 they do not fit.  Here nothing is copied: the pass kernels read the
// handle's own storage -- FP32 near-field slices and FP32 or mixed FP32 / FP16 / FP8
// factors (the layouts of hmg_internal.cuh) -- and split every value on chip into
// three BF16 parts (hi, then what hi misses, then what both miss), in the canonical
// K-major core layout of the MMA:
//
//   pass 1 (k_tcm_pass<0>): per stack of V_b^T with the same columns (M = stacked
//     terms <= 128, K = the columns, N = the vectors): t_b = V_b^T X_b, times the
//     terms' scales (FP16 / FP8 terms are stored scaled), written as the three-part
//     BF16 operand cores of pass 2;
//   pass 2 (k_tcm_pass<1>): per row tile (M <= 128 rows), the sum over its pairs of
//     U_slice t_b (K = terms) and D_slice X_b (K = columns), written to Y rows.
//
// A step is 32 K positions (4 K cores) of one pair or stack.  Roles of a CTA (one per
// SM, persistent, 16 warps), each a ring of stages with its own full / empty barriers:
//   warp 10, the raw producer: copies the stored bytes of a step (pass 2: one run of
//     whole slice columns; pass 1: 9 16-byte chunks of every V row of the stack, the
//     out-of-range ones zero-filled) into one of 5 raw stages with 16-byte cp.async,
//     L2 evict-first, and writes the step's header (geometry, pass 1's row table);
//   warps 11-15, the converters: all five share each step, an item being 32 rows x 1
//     K core (one 16-byte row of each part per lane): they read the raw stage
//     (conflict-free), decode FP16 / FP8 with warp-uniform branches, split, and store
//     the parts into one of 3 A stages in shared memory;
//   warp 8, lane 0: the B operand of each step (3-part X or t_b cores) by one bulk
//     copy into one of 3 B stages;
//   warp 9, lane 0: the MMAs of a step.  The parts of a B K core lie side by side
//     along N, so per K16 one MMA of N = 2 NV gives A0 B0 (hi) and A0 B1 (the first
//     correction), and four of N = NV add A1 B0, A0 B2, A2 B0 and A1 B1 to the
//     correction: two accumulators (hi, c).  A step that starts in the FP16 terms (A
//     exact in two parts) runs A0 [B0 B1] and A1 B0; one in the FP8 terms (exact in one
//     part) A0 B0.  tcgen05.commit then frees the A and B stages and signals the
//     accumulators;
//   warps 0-7: drain the accumulators after every step (tcgen05.ld; warp w reads
//     lanes 32 (w mod 4) .. + 31, half w / 4 of the vectors) and keep the sums hi + c
//     in FP32 registers (packed FP32 adds), so no tensor-core accumulation runs longer
//     than one step.
// Every role reads its per-step records 32 at a time (one per lane) and the epilogue
// prefetches the next job's rows, so no role waits on a global load per step.  Every
// wait is bounded (pipeline.cuh); on a time-out the CTA records an error code in the
// handle's flag, waits for its own copies and MMAs and frees tensor memory.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <functional>
#include <memory>
#include <queue>
#include <thread>
#include <vector>

#include "hmg_matrix.cuh"
#include "pipeline.cuh"
#include "stream.cuh"
#include "tc_common.cuh"

namespace hmg {

static constexpr int TCM_NMAX = 64;                          // vectors per pass at most
static constexpr int TCM_KC = 4;                             // K cores per step (32 K positions)
static constexpr int TCM_PARTS = 3;                          // BF16 parts of every operand
static constexpr int TCM_NR = 5;                             // raw stages
static constexpr int TCM_NA = 3;                             // converted A stages
static constexpr int TCM_NB = 3;                             // B stages
static constexpr int TCM_RROW = 144;                         // pass 1: bytes of a raw V row (9 chunks)
static constexpr int TCM_RAW = 128 * TCM_RROW;               // a raw stage (>= 32 columns x 128 rows x 4)
static constexpr int TCM_AST = TCM_KC * TCM_PARTS * 16 * 128;       // A of a step: 128 rows, 24 KB
static constexpr int TCM_BST = TCM_KC * TCM_PARTS * TCM_NMAX * 16;  // B of a step at 64 vectors, 12 KB
static constexpr int TCM_TMEM_COLS = 256;                    // two buffers of 2 NV accumulator columns (hi, c)
static constexpr int TCM_EPI = 8;                            // epilogue warps (4 or 8): 0 .. TCM_EPI - 1
static constexpr int TCM_WB = TCM_EPI;                       // B producer warp
static constexpr int TCM_WMMA = TCM_EPI + 1;                 // MMA warp
static constexpr int TCM_WRAW = TCM_EPI + 2;                 // raw producer warp
static constexpr int TCM_CONV = 8;                           // converter warps, from TCM_EPI + 3
static constexpr int TCM_THREADS = (TCM_EPI + 3 + TCM_CONV) * 32;
static constexpr int TCM_MAXMEM = 8;                         // blocks of a pass-1 stack (ranks rounded to 16)
static constexpr int TCM_STGR = 40;                          // pass 1 epilogue staging: row stride (BF16)
static_assert(2 * 2 * TCM_NMAX <= TCM_TMEM_COLS, "accumulators exceed the tensor memory allocation");
static_assert(TCM_EPI == 4 || TCM_EPI == 8, "4 or 8 epilogue warps");

// The K layout of a low-rank block's terms (t_b rows, U slice K positions, stack rows
// of pass 1): its FP32, FP16 and FP8 terms each start a run of 8 K positions, so that
// every K core holds terms of one storage tier (the padding positions are zero); the
// block takes tcm_kw of them, a multiple of 16.  A block whose padded runs would pass
// 128 positions (ranks near 128) keeps its terms back to back instead ("compact"),
// and its K cores may then mix tiers.
struct TcmTerms {
    int r32, r16, r8;     // terms per tier
    int r32p, r16p, r8p;  // the positions of each run
    bool compact;
};
__host__ __device__ inline TcmTerms tcm_terms(int r, int r32, int r16)
{
    TcmTerms t;
    t.r32 = r32;
    t.r16 = r16;
    t.r8 = r - r32 - r16;
    t.r32p = (r32 + 7) & ~7;
    t.r16p = (r16 + 7) & ~7;
    t.r8p = (t.r8 + 7) & ~7;
    t.compact = t.r32p + t.r16p + t.r8p > 128;
    if (t.compact) {
        t.r32p = t.r32;
        t.r16p = t.r16;
        t.r8p = t.r8;
    }
    return t;
}
__host__ __device__ inline int tcm_kw(const TcmTerms& t) { return (t.r32p + t.r16p + t.r8p + 15) & ~15; }

// One step.  Pass 2 (one pair): raw = first byte of its raw copy, n16 chunks of 16
// bytes; cc0 = the slice's chunk column there (a column of s_pad FP32 rows, a column of
// FP16 pairs or of FP8 quads); near pair: t0 = a = c0 mod 8 (K position of column 0),
// t1 = m2, t2 = -1; low-rank pair (the K layout of TcmTerms): t0 = r32 | r32p << 16,
// t1 = r16 | r16p << 16, t2 = r8 | compact << 16.  Pass 1 (one stack): n16 = the stack, cc0 = first 16-byte chunk of the step's
// columns in a V row (may be negative), t0 = a, t1 = 16-byte chunks of a V row.
struct TcmStep {
    const char* raw;
    long long b_kc;  // first K core of B in the operand buffer (X cores, then t_b cores)
    int meta;        // bits 0-1: K16 groups (1 or 2); bit 8: first step of a job; bit 9: last;
                     // bits 12-15: MMAs per K16 (1, 3 or 6)
    int rows;        // rows of the job's M (tile rows or stack rows)
    int kp0;         // first K position of the step
    int n16;
    int cc0;
    int t0, t1, t2;
};
static_assert(sizeof(TcmStep) == 48, "TcmStep layout");

// pass-1 job: the V^T of blocks with the same columns, one under the other.  A block's
// V^T is a run of 16-byte-aligned rows of m2p words -- r32 FP32 term rows, r16 / 2 FP16
// pair rows, r8 / 4 FP8 quad rows -- and raw row q of the stack is row q - qb[k] of
// member k.  rtab lists the 128 stack rows sorted by storage tier, so that most 32-row
// groups of it decode one tier: entry i = stack row m (bits 0-7), its raw row (bits
// 8-15), tier (bits 16-17: 0 FP32, 1 FP16, 2 FP8, 3 none) and the term's place in its
// pair or quad (bits 18-19).
struct TcmStack {
    const char* vptr[TCM_MAXMEM];
    int qb[TCM_MAXMEM];
    int nmem, nq, m2p4, pad;
    uint32_t rtab[128];
};
static_assert(sizeof(TcmStack) == 624, "TcmStack layout");

struct TcmJob {
    int r0;    // pass 2: first Z row of the tile; pass 1: first t_b term of the stack
    int rows;  // pass 2: rows of the tile; pass 1: stack rows
};

// a step's geometry as the converters keep it in registers (read once per step)
struct TcmGeo {
    int cc0, t0, t1, t2;
};

// written by the raw producer beside each raw stage
struct TcmHdr {
    int kp0, meta, rows, cc0, t0, t1, t2, pad;
    uint32_t rtab[128];
};

struct TcmSmem {
    unsigned char raw[TCM_NR][TCM_RAW];
    unsigned char a[TCM_NA][TCM_AST];
    unsigned char b[TCM_NB][TCM_BST];
    __nv_bfloat16 stg[4][TCM_NMAX * TCM_STGR];  // pass 1 epilogue: per warp, [vector][row] of t_b
    TcmHdr hdr[TCM_NR];
    const char* rowptr[128];                    // raw producer, pass 1: the stack's V rows
    uint64_t raw_full[TCM_NR], raw_empty[TCM_NR], a_full[TCM_NA], a_empty[TCM_NA], b_full[TCM_NB], b_empty[TCM_NB];
    uint64_t accf[2], acce[2], fin;
    uint32_t tmem;
    int fail;
};
static_assert(sizeof(TcmSmem) <= 227 * 1024, "TcmSmem exceeds the shared memory of a CTA");

// ---------------------------------------------------------------------------
// copies and decoding
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cpa16(void* dst, const void* src, unsigned n, uint64_t pol)
{
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2, %3;" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(n), "l"(pol)
                 : "memory");
}

// arrives on bar once every cp.async this thread issued so far has landed
__device__ __forceinline__ void cpa_arrive(uint64_t* bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ float2 h2f2(unsigned w)
{
    __half2 h;
    *reinterpret_cast<unsigned*>(&h) = w;
    return __half22float2(h);
}

__device__ __forceinline__ float2 e4m3x2_f2(unsigned w16)
{
    const __half2_raw hr = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w16 & 0xffffu), __NV_E4M3);
    return __half22float2(*reinterpret_cast<const __half2*>(&hr));
}

// 8 FP8 values starting at byte p (0..3) of the 12 bytes w0 w1 w2
__device__ __forceinline__ void fp8_run(unsigned w0, unsigned w1, unsigned w2, int p, float (&v)[8])
{
    const unsigned sel = 0x3210u + 0x1111u * (unsigned)p;
    const unsigned lo = __byte_perm(w0, w1, sel), hi = __byte_perm(w1, w2, sel);
    const float2 a = e4m3x2_f2(lo), b = e4m3x2_f2(lo >> 16), c = e4m3x2_f2(hi), d = e4m3x2_f2(hi >> 16);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    v[4] = c.x; v[5] = c.y; v[6] = d.x; v[7] = d.y;
}

// the parts of 8 values of one operand row, one uint4 (8 K positions) each: part 0 is
// the BF16 rounding, each further part the rounding of what the parts before miss.
// Every difference is exact in FP32, and what two parts miss has at most 8 significant
// bits, so three parts hold an FP32 value exactly.
__device__ __forceinline__ void store_parts(unsigned char* stage, int kc, int m, const float (&v)[8], int nparts)
{
    uint32_t w0[4], w1[4], w2[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float a = v[2 * k], b = v[2 * k + 1];
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        w0[k] = *reinterpret_cast<const uint32_t*>(&h);
        if (nparts > 1) {
            const float2 hf = __bfloat1622float2(h);
            const float ra = a - hf.x, rb = b - hf.y;
            const __nv_bfloat162 l = __floats2bfloat162_rn(ra, rb);
            w1[k] = *reinterpret_cast<const uint32_t*>(&l);
            if (nparts > 2) {
                const float2 lf = __bfloat1622float2(l);
                const __nv_bfloat162 l2 = __floats2bfloat162_rn(ra - lf.x, rb - lf.y);
                w2[k] = *reinterpret_cast<const uint32_t*>(&l2);
            }
        }
    }
    // row m of K core kc, part q: ((kc * 3 + q) * 16 + m / 8) * 128 + (m % 8) * 16
    unsigned char* base = stage + ((size_t)(kc * TCM_PARTS) * 16 + (m >> 3)) * 128 + (m & 7) * 16;
    *reinterpret_cast<uint4*>(base) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
    if (nparts > 1) *reinterpret_cast<uint4*>(base + 16 * 128) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
    if (nparts > 2) *reinterpret_cast<uint4*>(base + 2 * 16 * 128) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
}

// Pass 2, a K core of a compact low-rank block (TcmTerms), whose tiers may meet inside
// it: position by position
__device__ __forceinline__ void load_pass2_compact(const unsigned* rw, int sp, int m, int cc0, int k0, int r32, int r16,
                                                   int r8, float (&v)[8])
{
    auto word = [&](int c) -> unsigned { return rw[(c - cc0) * sp + m]; };
    const int e16 = r32 + r16, r = e16 + r8, c8 = r32 + (r16 >> 1);
#pragma unroll
    for (int e = 0; e < 8; e++) {
        const int kp = k0 + e;
        float x = 0.0f;
        if (kp < r32) {
            x = __uint_as_float(word(kp));
        } else if (kp < e16) {
            const float2 f = h2f2(word(r32 + ((kp - r32) >> 1)));
            x = ((kp - r32) & 1) ? f.y : f.x;
        } else if (kp < r) {
            const float2 f = e4m3x2_f2(word(c8 + ((kp - e16) >> 2)) >> (8 * ((kp - e16) & 2)));
            x = ((kp - e16) & 1) ? f.y : f.x;
        }
        v[e] = x;
    }
}

// Pass 2, one item: row m (lane) of K core kc.  Word (c, m) of raw chunk column c is at
// rw[(c - cc0) * sp + m]: consecutive lanes read consecutive words.
__device__ __forceinline__ void load_pass2(const TcmGeo H, const unsigned* rw, int sp, int m, int k0, float (&v)[8])
{
    const int cc0 = H.cc0;
    auto word = [&](int c) -> unsigned { return rw[(c - cc0) * sp + m]; };
    if (H.t2 < 0) {  // near slice: FP32 columns [0, m2) at K positions a ..
        const int j0 = k0 - H.t0, m2 = H.t1;
        if (j0 >= 0 && j0 + 8 <= m2) {
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] = __uint_as_float(word(j0 + e));
        } else {
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] = (j0 + e >= 0 && j0 + e < m2) ? __uint_as_float(word(j0 + e)) : 0.0f;
        }
        return;
    }
    // low-rank slice: one tier per K core (TcmTerms); chunk columns r32 FP32 terms, then
    // r16 / 2 FP16 pairs, then r8 / 4 FP8 quads
    const int r32 = H.t0 & 0xffff, r32p = H.t0 >> 16, r16 = H.t1 & 0xffff, r16p = H.t1 >> 16, r8 = H.t2 & 0xffff;
    if (H.t2 >> 16) {
        load_pass2_compact(rw, sp, m, cc0, k0, r32, r16, r8, v);
        return;
    }
    if (k0 < r32p) {
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] = k0 + e < r32 ? __uint_as_float(word(k0 + e)) : 0.0f;
    } else if (k0 < r32p + r16p) {
        // FP16 pairs: term 2g + t of the tier in half t of word g
        const int g0 = (k0 - r32p) >> 1;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float2 f = 2 * (g0 + i) < r16 ? h2f2(word(r32 + g0 + i)) : make_float2(0.0f, 0.0f);
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    } else {
        // FP8 quads: term 4g + t of the tier in byte t of word g
        const int g0 = (k0 - r32p - r16p) >> 2, c8 = r32 + (r16 >> 1);
        const unsigned w0 = 4 * g0 < r8 ? word(c8 + g0) : 0u, w1 = 4 * (g0 + 1) < r8 ? word(c8 + g0 + 1) : 0u;
        fp8_run(w0, w1, 0u, 0, v);
    }
}

// Pass 1, one item: stack row m (lane) of K core kc: the 8 words at sh + 8 kc of its raw
// row (three 16-byte reads; rows 144 bytes apart, so 8 consecutive rows hit 8 distinct
// bank groups), decoded by the row's tier.
__device__ __forceinline__ void load_pass1(const unsigned ent, const unsigned char* raw, int sh, int kc, float (&v)[8])
{
    const int tier = (ent >> 16) & 3, sel = (ent >> 18) & 3;
#pragma unroll
    for (int e = 0; e < 8; e++) v[e] = 0.0f;
    if (tier == 3) return;
    const uint4* rr = reinterpret_cast<const uint4*>(raw + ((ent >> 8) & 255) * TCM_RROW) + 2 * kc;
    const uint4 c0 = rr[0], c1 = rr[1], c2 = rr[2];
    const unsigned words[12] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w, c2.x, c2.y, c2.z, c2.w};
    unsigned w[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
        // sh is the same for every lane of the step
        switch (sh) {
        case 0: w[e] = words[e]; break;
        case 1: w[e] = words[e + 1]; break;
        case 2: w[e] = words[e + 2]; break;
        default: w[e] = words[e + 3]; break;
        }
    }
    if (tier == 0) {
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] = __uint_as_float(w[e]);
    } else if (tier == 1) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float2 f = h2f2(__byte_perm(w[2 * i], w[2 * i + 1], sel ? 0x7632u : 0x5410u));
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    } else {
        const unsigned s2 = (unsigned)sel | ((unsigned)sel + 4u) << 4;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float2 f = e4m3x2_f2(__byte_perm(w[2 * i], w[2 * i + 1], s2));
            v[2 * i] = f.x;
            v[2 * i + 1] = f.y;
        }
    }
}

// ---------------------------------------------------------------------------
// the pass kernel
// ---------------------------------------------------------------------------
// Steps of CTA c: [cta[c].y, cta[c+1].y); its jobs: [cta[c].x, cta[c+1].x).  MODE 0
// (pass 1) writes t_b cores: K core kc of the stack whose first t_b term is r0 to B K core
// tb_kc + r0 / 8 + kc, times tscale per term; MODE 1 (pass 2) writes tile row i to Y
// row map[r0 + i].
template <int MODE, int NV>
__global__ void __launch_bounds__(TCM_THREADS, 1)
    k_tcm_pass(const TcmStep* __restrict__ steps, const TcmJob* __restrict__ jobs, const int2* __restrict__ cta,
               const TcmStack* __restrict__ stacks, char* Bbuf, long long tb_kc, const float* __restrict__ tscale,
               const int* __restrict__ map, int nrhs, double* Y, int ldy, int* err)
{
    constexpr int P = TCM_PARTS;
    constexpr int KB = NV * 16 * P;  // bytes of a B K core, all parts
    extern __shared__ __align__(1024) unsigned char tcm_raw[];
    TcmSmem& sm = *reinterpret_cast<TcmSmem*>(tcm_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int2 lo = cta[blockIdx.x], hi = cta[blockIdx.x + 1];
    const int nsteps = hi.y - lo.y;
    const TcmStep* my_steps = steps + lo.y;
    volatile int* fail = &sm.fail;
    if (tid == 0) {
        for (int s = 0; s < TCM_NR; s++) {
            mbar_init(&sm.raw_full[s], 33);  // the 32 producer lanes' copies + the header
            mbar_init(&sm.raw_empty[s], TCM_CONV);
        }
        for (int s = 0; s < TCM_NA; s++) {
            mbar_init(&sm.a_full[s], TCM_CONV);
            mbar_init(&sm.a_empty[s], 1);
        }
        for (int s = 0; s < TCM_NB; s++) {
            mbar_init(&sm.b_full[s], 1);
            mbar_init(&sm.b_empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&sm.accf[b], 1);
            mbar_init(&sm.acce[b], TCM_EPI);
        }
        mbar_init(&sm.fin, 1);
        sm.fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == TCM_WMMA) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)),
                     "n"(TCM_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem;

    if (warp >= TCM_WRAW + 1) {
        // ---- converters: every step, items (32 rows, 1 K core) dealt over the warps ----
        const int cw = warp - (TCM_WRAW + 1);
        for (int i = 0; i < nsteps; i++) {
            const int slot = i % TCM_NR, as = i % TCM_NA;
            bool ok = !*fail && mbar_wait(&sm.raw_full[slot], (i / TCM_NR) & 1, err, 31);
            if (ok && i >= TCM_NA) ok = mbar_wait(&sm.a_empty[as], ((i / TCM_NA) - 1) & 1, err, 32);
            if (!__all_sync(~0u, ok)) {
                *fail = 1;
                break;
            }
            const TcmHdr& H = sm.hdr[slot];
            const int meta = H.meta, rows = H.rows, kp0 = H.kp0;
            const TcmGeo G{H.cc0, H.t0, H.t1, H.t2};
            const int lg = (meta & 3) == 2 ? 2 : 1, nkc = 1 << lg;  // K cores of the step
            const int mode = (meta >> 12) & 15, nparts = MODE == 0 ? 3 : (mode >= 6 ? 3 : (mode >= 3 ? 2 : 1));
            const int nitems = ((rows + 31) >> 5) << lg;
            unsigned char* stage = sm.a[as];
            if (MODE == 1) {
                const int sp = (rows + 3) & ~3;
                const unsigned* rw = reinterpret_cast<const unsigned*>(sm.raw[slot]);
#pragma unroll 1
                for (int it = cw; it < nitems; it += TCM_CONV) {
                    const int kc = it & (nkc - 1), m = (it >> lg) * 32 + lane;
                    float v[8];
                    load_pass2(G, rw, sp, m, kp0 + 8 * kc, v);
                    store_parts(stage, kc, m, v, nparts);
                }
            } else {
                const int sh = (kp0 - G.t0) & 3;
                // the row-table entries of this warp's items (stack rows in tier order), read
                // before any item is stored
                unsigned ent[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int it = cw + j * TCM_CONV;
                    ent[j] = it < nitems ? H.rtab[(it >> lg) * 32 + lane] : (3u << 16);
                }
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int it = cw + j * TCM_CONV;
                    if (it >= nitems) break;
                    const int kc = it & (nkc - 1), m = ent[j] & 255;
                    float v[8];
                    load_pass1(ent[j], sm.raw[slot], sh, kc, v);
                    store_parts(stage, kc, m, v, 3);
                }
            }
            // the generic-proxy stores become visible to the tensor cores' (async) proxy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&sm.a_full[as]);
                mbar_arrive(&sm.raw_empty[slot]);
            }
        }
    } else if (warp == TCM_WRAW) {
        // ---- raw producer: the stored bytes of every step, 16-byte cp.async per lane ----
        uint64_t pol;
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
        int cur_stack = -1, nq = 0, m2p4 = 0;
        const TcmStack* sk = nullptr;
        const char** rowptr = sm.rowptr;
        bool ok = true;
        for (int i0 = 0; i0 < nsteps && ok; i0 += 32) {
            TcmStep rec{};
            if (i0 + lane < nsteps) rec = my_steps[i0 + lane];
            const int cnt = min(32, nsteps - i0);
            for (int k = 0; k < cnt; k++) {
                const int i = i0 + k, slot = i % TCM_NR;
                const long long rawp = __shfl_sync(~0u, (long long)rec.raw, k);
                const int meta = __shfl_sync(~0u, rec.meta, k), rows = __shfl_sync(~0u, rec.rows, k);
                const int kp0 = __shfl_sync(~0u, rec.kp0, k), n16 = __shfl_sync(~0u, rec.n16, k);
                const int cc0 = __shfl_sync(~0u, rec.cc0, k), t0 = __shfl_sync(~0u, rec.t0, k);
                const int t1 = __shfl_sync(~0u, rec.t1, k), t2 = __shfl_sync(~0u, rec.t2, k);
                if (MODE == 0 && n16 != cur_stack) {
                    // the stack's V rows: member k's rows from vptr[k], m2p4 chunks each
                    cur_stack = n16;
                    sk = stacks + n16;
                    nq = sk->nq;
                    m2p4 = sk->m2p4;
                    const int nmem = sk->nmem;
                    const char* vp = lane < nmem ? sk->vptr[lane] : nullptr;
                    const int qb = lane < nmem ? sk->qb[lane] : 0x7fffffff;
                    for (int q = lane; q < 128; q += 32) {
                        int kk = 0;
                        for (int u = 1; u < nmem; u++)
                            if (__shfl_sync(~0u, qb, u) <= q) kk = u;
                        const char* base = reinterpret_cast<const char*>(__shfl_sync(~0u, (long long)vp, kk));
                        const int q0 = __shfl_sync(~0u, qb, kk);
                        rowptr[q] = base + (size_t)(q - q0) * m2p4 * 16;
                    }
                    __syncwarp();
                }
                if (i >= TCM_NR) {
                    bool w = true;
                    if (lane == 0) w = !*fail && mbar_wait(&sm.raw_empty[slot], ((i / TCM_NR) - 1) & 1, err, 33);
                    if (!__shfl_sync(~0u, w, 0)) {
                        *fail = 1;
                        ok = false;
                        break;
                    }
                }
                TcmHdr& H = sm.hdr[slot];
                if (lane == 0) {
                    H.kp0 = kp0; H.meta = meta; H.rows = rows; H.cc0 = cc0;
                    H.t0 = t0; H.t1 = t1; H.t2 = t2;
                }
                unsigned char* dst = sm.raw[slot];
                if (MODE == 1) {
                    const char* src = reinterpret_cast<const char*>(rawp);
                    for (int c = lane; c < n16; c += 32) cpa16(dst + 16 * c, src + 16 * c, 16, pol);
                } else {
                    cpa16(&H.rtab[4 * lane], &sk->rtab[4 * lane], 16, pol);
                    // chunk c: V row c / 9, chunk c mod 9, walked without division (32 = 3 * 9 + 5);
                    // four chunks a round, their row pointers read before any copy is issued
                    const int nch = nq * 9;
                    int r = lane / 9, kk = lane - 9 * (lane / 9);
                    for (int c = lane; c < nch; c += 128) {
                        int rr[4], kq[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            rr[u] = r;
                            kq[u] = kk;
                            r += 3;
                            kk += 5;
                            if (kk >= 9) {
                                kk -= 9;
                                r += 1;
                            }
                        }
                        const char* rp[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) rp[u] = rowptr[min(rr[u], 127)];
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            if (c + 32 * u < nch) {
                                const int ch = cc0 + kq[u];
                                const bool in = ch >= 0 && ch < m2p4;
                                cpa16(dst + rr[u] * TCM_RROW + 16 * kq[u], in ? rp[u] + 16 * ch : rp[u], in ? 16u : 0u, pol);
                            }
                        }
                    }
                }
                cpa_arrive(&sm.raw_full[slot]);
                __syncwarp();
                if (lane == 0) mbar_arrive(&sm.raw_full[slot]);
            }
        }
        // every copy of this warp has landed before the CTA leaves
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
    } else if (warp == TCM_WB) {
        // ---- B operand of every step: one bulk copy, lane 0 ----
        int issued = 0;
        bool ok = true;
        for (int i0 = 0; i0 < nsteps && ok; i0 += 32) {
            int mt = 0;
            long long bk = 0;
            if (i0 + lane < nsteps) {
                mt = my_steps[i0 + lane].meta;
                bk = my_steps[i0 + lane].b_kc;
            }
            const int cnt = min(32, nsteps - i0);
            for (int k = 0; k < cnt; k++) {
                const int i = i0 + k, slot = i % TCM_NB;
                const int meta = __shfl_sync(~0u, mt, k);
                const long long b_kc = __shfl_sync(~0u, bk, k);
                bool w = true;
                if (lane == 0) {
                    if (i >= TCM_NB) w = !*fail && mbar_wait(&sm.b_empty[slot], ((i / TCM_NB) - 1) & 1, err, 34);
                    if (w) {
                        const unsigned bytes = (unsigned)(2 * (meta & 3)) * KB;
                        mbar_arrive_expect_tx(&sm.b_full[slot], bytes);
                        bulk_g2s(sm.b[slot], Bbuf + b_kc * KB, bytes, &sm.b_full[slot]);
                        issued++;
                    }
                }
                if (!__shfl_sync(~0u, w, 0)) {
                    *fail = 1;
                    ok = false;
                    break;
                }
            }
        }
        // the last copy into every stage has landed before the CTA leaves
        if (lane == 0)
            for (int s = 0; s < TCM_NB && s < issued; s++)
                mbar_wait(&sm.b_full[(issued - 1 - s) % TCM_NB], ((issued - 1 - s) / TCM_NB) & 1, err, 35);
        __syncwarp();
    } else if (warp == TCM_WMMA) {
        // ---- MMAs, lane 0: A0 over the B parts side by side along N, then the corrections ----
        constexpr uint32_t LBA = P * 16 * 128, LBB = KB;  // K-core strides of A and B
        bool ok = true;
        for (int i0 = 0; i0 < nsteps && ok; i0 += 32) {
            const int mt = i0 + lane < nsteps ? my_steps[i0 + lane].meta : 0;
            const int cnt = min(32, nsteps - i0);
            for (int k = 0; k < cnt; k++) {
                const int i = i0 + k, as = i % TCM_NA, bs = i % TCM_NB, buf = i & 1;
                const int meta = __shfl_sync(~0u, mt, k);
                bool w = true;
                if (lane == 0) {
                    w = !*fail && mbar_wait(&sm.a_full[as], (i / TCM_NA) & 1, err, 36) &&
                        mbar_wait(&sm.b_full[bs], (i / TCM_NB) & 1, err, 37);
                    // the epilogue has read this buffer's previous step
                    if (w && i >= 2) w = mbar_wait(&sm.acce[buf], ((i >> 1) - 1) & 1, err, 38);
                    if (w) {
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const int nk = meta & 3, mode = (meta >> 12) & 15;
                        const uint32_t d = tmem + (uint32_t)(buf * 2 * NV);  // hi, c
                        uint64_t ad = smem_desc(smem_u32(sm.a[as]), LBA, 128), bd = smem_desc(smem_u32(sm.b[bs]), LBB, 128);
                        const uint64_t da = (2 * LBA) >> 4, db = (2 * LBB) >> 4;
                        const uint64_t alo = (16 * 128) >> 4;  // part q of A: + q alo
                        for (int kk = 0; kk < nk; kk++) {
                            const uint32_t acc = kk > 0 ? 1u : 0u;
                            if (mode >= 6) {
                                const uint64_t blo = (NV * 16) >> 4;
                                tc_mma(d, ad, bd, tc_idesc<2 * NV>(), acc);
                                tc_mma(d + NV, ad + alo, bd, tc_idesc<NV>(), 1u);
                                tc_mma(d + NV, ad, bd + 2 * blo, tc_idesc<NV>(), 1u);
                                tc_mma(d + NV, ad + 2 * alo, bd, tc_idesc<NV>(), 1u);
                                tc_mma(d + NV, ad + alo, bd + blo, tc_idesc<NV>(), 1u);
                            } else if (mode >= 3) {
                                tc_mma(d, ad, bd, tc_idesc<2 * NV>(), acc);
                                tc_mma(d + NV, ad + alo, bd, tc_idesc<NV>(), 1u);
                            } else {
                                tc_mma(d, ad, bd, tc_idesc<NV>(), acc);
                            }
                            ad += da;
                            bd += db;
                        }
                        tc_commit(&sm.a_empty[as]);
                        tc_commit(&sm.b_empty[bs]);
                        tc_commit(&sm.accf[buf]);
                    }
                }
                if (!__shfl_sync(~0u, w, 0)) {
                    *fail = 1;
                    ok = false;
                    break;
                }
            }
        }
        if (lane == 0) {
            tc_commit(&sm.fin);  // every MMA issued here has completed before tensor memory is freed
            mbar_wait(&sm.fin, 0, err, 39);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w owns accumulator rows 32 (w mod 4) .. + 31 and vectors
        // HV (w / 4) .. + HV - 1 (HV = NV with 4 epilogue warps, NV / 2 with 8) ----
        constexpr int HV = NV * 4 / TCM_EPI;
        static_assert(HV % 2 == 0, "pairs of vectors per epilogue thread");
        const int q4 = warp & 3, hv = warp >> 2;
        const int row = q4 * 32 + lane;
        float f[HV];
        const int njobs = hi.x - lo.x;
        const TcmJob* my_jobs = jobs + lo.x;
        // job jc's rows, first row / term and per-row value (Y row or term scale) are
        // loaded while job jc - 1 runs; the record of job jc + 1 one job earlier still
        auto row_value = [&](const TcmJob& jb) -> unsigned {
            if (row >= jb.rows) return 0u;
            return MODE == 1 ? (unsigned)map[jb.r0 + row] : __float_as_uint(tscale[jb.r0 + row]);
        };
        TcmJob cur = njobs > 0 ? my_jobs[0] : TcmJob{0, 0};
        unsigned cur_val = njobs > 0 ? row_value(cur) : 0u;
        TcmJob nxt = njobs > 1 ? my_jobs[1] : TcmJob{0, 0};
        int jc = 0, rows = 0, r0 = 0;
        unsigned val = 0u;
        bool ok = true;
        int mt_next = lane < nsteps ? my_steps[lane].meta : 0;
        for (int i0 = 0; i0 < nsteps && ok; i0 += 32) {
            const int mt = mt_next;
            mt_next = i0 + 32 + lane < nsteps ? my_steps[i0 + 32 + lane].meta : 0;
            const int cnt = min(32, nsteps - i0);
            for (int k = 0; k < cnt; k++) {
                const int i = i0 + k, meta = __shfl_sync(~0u, mt, k), buf = i & 1;
                const bool first = meta & 256, last = meta & 512;
                const int mode = (meta >> 12) & 15;
                if (first) {
                    rows = cur.rows;
                    r0 = cur.r0;
                    val = cur_val;
                    cur = nxt;
                    cur_val = jc + 1 < njobs ? row_value(cur) : 0u;
                    nxt = jc + 2 < njobs ? my_jobs[jc + 2] : TcmJob{0, 0};
                }
                if (!__all_sync(~0u, !*fail && mbar_wait(&sm.accf[buf], (i >> 1) & 1, err, 40))) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t taddr = tmem + (uint32_t)(buf * 2 * NV + hv * HV) + ((uint32_t)(q4 * 32) << 16);
                // 16 columns of each accumulator at a time: the running sums f[HV] stay in
                // registers beside them
#pragma unroll
                for (int h = 0; h < HV / 16; h++) {
                    uint32_t v[16], c1[16];
                    tc_ld16(taddr + 16 * h, v);
                    if (mode > 1) tc_ld16(taddr + NV + 16 * h, c1);

                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    // hi + c, then into the running sums: packed pairs, uniform branches

                    if (mode > 1) {
#pragma unroll
                        for (int q = 0; q < 16; q += 2) add_f32x2(v[q], v[q + 1], c1[q], c1[q + 1]);
                    }
                    if (first) {
#pragma unroll
                        for (int q = 0; q < 16; q++) f[16 * h + q] = __uint_as_float(v[q]);
                    } else {
#pragma unroll
                        for (int q = 0; q < 16; q += 2) add_f32x2(f[16 * h + q], f[16 * h + q + 1], v[q], v[q + 1]);
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&sm.acce[buf]);
                if (!last) continue;
                jc++;
                if (MODE == 1) {
                    if (row < rows) {
                        double* y = Y + (int)val + (size_t)(hv * HV) * ldy;
#pragma unroll
                        for (int q = 0; q < HV; q++)
                            if (hv * HV + q < nrhs) y[(size_t)q * ldy] = (double)f[q];
                    }
                } else {
                    // term row -> 3-part B cores of pass 2 through the quarter's staging
                    // array [vector][row] (rows padded to 40: the 16-byte reads of 8
                    // consecutive vectors hit distinct bank groups); the two warps of a
                    // quarter fill and read disjoint vectors of it
                    __nv_bfloat16* stg = sm.stg[q4];
                    const float scale = __uint_as_float(val);
#pragma unroll
                    for (int q = 0; q < HV; q++) f[q] *= scale;
                    // part p: the BF16 rounding of what parts 0..p-1 miss, f keeping the rest
                    // (one packed rounding per pair of vectors, reused for the residual)
                    unsigned short* stg16 = reinterpret_cast<unsigned short*>(stg);
#pragma unroll 1
                    for (int part = 0; part < P; part++) {
#pragma unroll
                        for (int q = 0; q < HV; q += 2) {
                            const uint32_t h = pack_bf16(f[q], f[q + 1]);
                            if (part + 1 < P) {
                                f[q] -= __uint_as_float(h << 16);
                                f[q + 1] -= __uint_as_float(h & 0xffff0000u);
                            }
                            stg16[(hv * HV + q) * TCM_STGR + lane] = (unsigned short)(h & 0xffffu);
                            stg16[(hv * HV + q + 1) * TCM_STGR + lane] = (unsigned short)(h >> 16);
                        }
                        __syncwarp();
                        uint4* dst = reinterpret_cast<uint4*>(Bbuf);
#pragma unroll 1
                        for (int u = lane; u < 4 * HV; u += 32) {
                            // K core kcl (rows 8 kcl .. 8 kcl + 7 of the quarter) of vector vq
                            const int kcl = u / HV, vq = hv * HV + u % HV;
                            if (q4 * 4 + kcl < (rows >> 3))
                                dst[((size_t)(tb_kc + (r0 >> 3) + q4 * 4 + kcl) * P + part) * NV + vq] =
                                    *reinterpret_cast<const uint4*>(stg + vq * TCM_STGR + 8 * kcl);
                        }
                        __syncwarp();
                    }
                }
            }
        }
        if (!ok) *fail = 1;
    }
    __syncthreads();
    if (warp == TCM_WMMA) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(TCM_TMEM_COLS));
    }
}

// scale of every t_b term (K position of TcmTerms): su_l sv_l for the FP16 / FP8 terms
// of mixed storage, else 1 (padding included); one warp per block
__global__ void k_tcm_scales(const int* __restrict__ far, int nfar, const int* __restrict__ rank,
                             const int* __restrict__ tier32, const int* __restrict__ tier16,
                             const int* __restrict__ blk_m2, void* const* ptrV, const long long* __restrict__ tterm,
                             int mixed, float* __restrict__ tscale)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nfar) return;
    const int b = far[w], r = rank[b];
    const TcmTerms T = tcm_terms(r, tier32[b], tier16[b]);
    const size_t m2p = (size_t)((blk_m2[b] + 3) & ~3);
    const float* scal = reinterpret_cast<const float*>(static_cast<const char*>(ptrV[b]) +
                                                       m2p * (4 * (size_t)T.r32 + 2 * (size_t)T.r16 + (size_t)T.r8));
    for (int k = lane; k < tcm_kw(T); k += 32) {
        int l = -1;
        if (k >= T.r32p && k < T.r32p + T.r16) l = T.r32 + (k - T.r32p);
        else if (k >= T.r32p + T.r16p && k < T.r32p + T.r16p + T.r8) l = T.r32 + T.r16 + (k - T.r32p - T.r16p);
        tscale[tterm[w] + k] = (mixed && l >= 0) ? scal[l] : 1.0f;
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
    dfree(h->tcm_tscale, s);
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
    void add(const TcmStep& st, double raw_bytes)
    {
        steps.push_back(st);
        const int nk = st.meta & 3, mode = (st.meta >> 12) & 15;
        // copy bytes plus the MMA issue time (~46 cycles a 128 x N x 16 MMA) in bytes
        cost.back() += raw_bytes + 2048.0 * mode * nk;
    }
    // src's jobs after this plan's (before finish)
    void append(const TcmPlan& src)
    {
        const int base = (int)steps.size();
        for (int x : src.step0) step0.push_back(base + x);
        steps.insert(steps.end(), src.steps.begin(), src.steps.end());
        jobs.insert(jobs.end(), src.jobs.begin(), src.jobs.end());
        cost.insert(cost.end(), src.cost.begin(), src.cost.end());
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

// host threads for building a plan
int plan_threads()
{
    return (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
}

// Jobs onto CTAs: the few large ones first, longest first, then the rest in plan order
// (row tiles / column clusters in Z order), each onto the least loaded CTA, so that the
// CTAs work through neighbouring tiles at the same time and share X in L2.
hmg_status upload_plan(hmg_matrix* h, int q, const TcmPlan& L, int grid)
{
    cudaStream_t s = h->stream;
    const int nj = (int)L.jobs.size();
    double total = 0.0;
    for (int j = 0; j < nj; j++) total += L.cost[j];
    const double big = total / (4.0 * grid);
    std::vector<int> order;
    for (int j = 0; j < nj; j++)
        if (L.step0[j] < L.step0[j + 1] && L.cost[j] > big) order.push_back(j);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return L.cost[a] > L.cost[b]; });
    for (int j = 0; j < nj; j++)
        if (L.step0[j] < L.step0[j + 1] && !(L.cost[j] > big)) order.push_back(j);
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
    std::vector<TcmJob> jobs;
    std::vector<int2> cta(grid + 1);
    size_t nsteps = 0;
    for (int c = 0; c < grid; c++) {
        cta[c] = make_int2((int)jobs.size(), (int)nsteps);
        for (int j : mine[c]) {
            jobs.push_back(L.jobs[j]);
            nsteps += (size_t)(L.step0[j + 1] - L.step0[j]);
        }
    }
    cta[grid] = make_int2((int)jobs.size(), (int)nsteps);
    // the steps in CTA order, each CTA's range copied on one of a few host threads
    std::unique_ptr<TcmStep[]> steps(new TcmStep[std::max(nsteps, (size_t)1)]);
    {
        auto copy = [&](int c0, int c1) {
            for (int c = c0; c < c1; c++) {
                size_t o = (size_t)cta[c].y;
                for (int j : mine[c]) {
                    const size_t k = (size_t)(L.step0[j + 1] - L.step0[j]);
                    std::copy(L.steps.begin() + L.step0[j], L.steps.begin() + L.step0[j + 1], steps.get() + o);
                    o += k;
                }
            }
        };
        const int nth = std::min(8, plan_threads());
        std::vector<std::thread> th;
        for (int k = 1; k < nth; k++) th.emplace_back(copy, grid * k / nth, grid * (k + 1) / nth);
        copy(0, grid / nth);
        for (std::thread& x : th) x.join();
    }
    hmg_status st;
    if ((st = dalloc(&h->tcm_steps[q], std::max(nsteps, (size_t)1) * sizeof(TcmStep), s)) ||
        (st = dalloc(&h->tcm_jobs[q], std::max(jobs.size(), (size_t)1) * sizeof(TcmJob), s)) ||
        (st = dalloc(&h->tcm_cta[q], (size_t)(grid + 1) * sizeof(int2), s)))
        return st;
    if (nsteps > 0)
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tcm_steps[q], steps.get(), nsteps * sizeof(TcmStep), cudaMemcpyHostToDevice, s));
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
        if (h->h_rank[b] > 0 &&
            tcm_kw(tcm_terms(h->h_rank[b], h->far_prec == HMG_PREC_MIXED ? h->h_r32[b] : h->h_rank[b],
                             h->far_prec == HMG_PREC_MIXED ? h->h_r16[b] : 0)) > 128) {
            set_error("hmg_build_tensor_core_operands: block %d has rank %d (> 128)", b, h->h_rank[b]);
            return HMG_ERR_UNSUPPORTED;
        }
    if ((st = ensure_desc(h, 4))) return st;
    const int np = h->npairs, nt = h->ntiles, nb = h->nblocks, grid = h->nsm;
    std::vector<int> tps(nt + 1), pblock(np), ts(nt), tr0(nt);
    std::vector<PairDesc> desc(np);
    std::vector<void*> pv(nb, nullptr);
    HMG_CUDA_TRY(cudaMemcpy(tps.data(), h->tile_pair_start, sizeof(int) * (nt + 1), cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(pblock.data(), h->pair_block, sizeof(int) * np, cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(ts.data(), h->tile_s, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(tr0.data(), h->tile_r0, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    if (np > 0) HMG_CUDA_TRY(cudaMemcpy(desc.data(), h->pair_desc, sizeof(PairDesc) * np, cudaMemcpyDeviceToHost));
    if (h->naca > 0 && h->ptrV) HMG_CUDA_TRY(cudaMemcpy(pv.data(), h->ptrV, sizeof(void*) * nb, cudaMemcpyDeviceToHost));
    const bool mixed = h->far_prec == HMG_PREC_MIXED;
    const long long xkc = (h->n[1] + 7) / 8 + 4;  // X K cores (8 Z-ordered columns each), with slack
    // pass 1: stacks of blocks with the same columns, ranks rounded to 16, first fit
    std::vector<long long> toff(nb, -1);  // first 16-term group of each block's t_b
    long long tgroups = 0;
    std::vector<TcmStack> stacks;
    std::vector<int> far_blocks;
    std::vector<long long> far_term;
    TcmPlan p1, p2;
    {
        std::vector<int> far;
        for (int b = h->ndense; b < nb; b++)
            if (h->h_rank[b] > 0) far.push_back(b);
        auto terms = [&](int b) {
            return tcm_terms(h->h_rank[b], mixed ? h->h_r32[b] : h->h_rank[b], mixed ? h->h_r16[b] : 0);
        };
        std::stable_sort(far.begin(), far.end(), [&](int x, int y) {
            if (h->h_c0[x] != h->h_c0[y]) return h->h_c0[x] < h->h_c0[y];
            if (h->h_m2[x] != h->h_m2[y]) return h->h_m2[x] < h->h_m2[y];
            return h->h_rank[x] > h->h_rank[y];
        });
        // the column clusters (runs of equal c0 and m2 in `far`) are planned in contiguous
        // ranges on several host threads with range-local stack and t_b numbering, and
        // joined in order with those numbers shifted: the plan does not depend on the split
        std::vector<size_t> gs;  // first entry of every column cluster, then far.size()
        for (size_t g = 0; g < far.size(); g++)
            if (g == 0 || h->h_c0[far[g]] != h->h_c0[far[g - 1]] || h->h_m2[far[g]] != h->h_m2[far[g - 1]])
                gs.push_back(g);
        gs.push_back(far.size());
        const int ncl = (int)gs.size() - 1;
        struct Part {
            std::vector<TcmStack> stacks;
            std::vector<int> far_blocks;
            std::vector<long long> far_term;
            TcmPlan plan;
            long long tgroups = 0;
        };
        auto plan_clusters = [&](int k0, int k1, Part& P) {
            std::vector<std::vector<int>> members;  // the stacks of one cluster (first fit)
            std::vector<int> fill;
            for (int gk = k0; gk < k1; gk++) {
                const size_t g0 = gs[gk], g1 = gs[gk + 1];
                size_t nstk = 0;
                for (size_t i = g0; i < g1; i++) {
                    const int b = far[i], kwb = tcm_kw(terms(b));
                    size_t k = 0;
                    while (k < nstk && fill[k] + kwb > 128) k++;
                    if (k == nstk) {
                        if (nstk == members.size()) {
                            members.emplace_back();
                            fill.push_back(0);
                        }
                        members[nstk].clear();
                        fill[nstk] = 0;
                        nstk++;
                    }
                    members[k].push_back(b);
                    fill[k] += kwb;
                }
                const int c0 = h->h_c0[far[g0]], m2 = h->h_m2[far[g0]], a = c0 & 7, kw = (a + m2 + 15) & ~15;
                const int m2p4 = ((m2 + 3) & ~3) / 4;
                for (size_t k = 0; k < nstk; k++) {
                    TcmStack sk{};
                    sk.nmem = (int)members[k].size();
                    sk.m2p4 = m2p4;
                    uint32_t row_ent[128];  // per stack row: raw row | tier | place, as rtab without the row
                    for (int m = 0; m < 128; m++) row_ent[m] = 3u << 16;
                    const long long tg0 = P.tgroups;
                    int off = 0, q = 0;
                    for (int u = 0; u < sk.nmem; u++) {
                        const int b = members[k][u];
                        const TcmTerms T = terms(b);
                        const int kwb = tcm_kw(T);
                        sk.vptr[u] = static_cast<const char*>(pv[b]);
                        sk.qb[u] = q;
                        // stack rows in the K layout of TcmTerms: FP32 term rows, FP16 pair rows
                        // (two terms each), FP8 quad rows (four terms each), padding rows zero
                        for (int t = 0; t < T.r32; t++) row_ent[off + t] = (uint32_t)(q + t) << 8;
                        for (int t = 0; t < T.r16; t++)
                            row_ent[off + T.r32p + t] = (uint32_t)(q + T.r32 + t / 2) << 8 | 1u << 16 | (uint32_t)(t & 1) << 18;
                        for (int t = 0; t < T.r8; t++)
                            row_ent[off + T.r32p + T.r16p + t] =
                                (uint32_t)(q + T.r32 + T.r16 / 2 + t / 4) << 8 | 2u << 16 | (uint32_t)(t & 3) << 18;
                        toff[b] = P.tgroups;
                        P.far_blocks.push_back(b);
                        P.far_term.push_back(P.tgroups * 16);
                        P.tgroups += kwb / 16;
                        off += kwb;
                        q += T.r32 + T.r16 / 2 + T.r8 / 4;
                    }
                    sk.nq = q;
                    // rows in tier order (FP32, FP16, FP8, none), each carrying its row number
                    // (a counting sort: row order kept within a tier)
                    {
                        int start[4] = {0, 0, 0, 0};
                        for (int m = 0; m < 128; m++) start[(row_ent[m] >> 16) & 3]++;
                        for (int t = 3, acc = 128; t >= 0; t--) {
                            acc -= start[t];
                            start[t] = acc;
                        }
                        for (int m = 0; m < 128; m++) sk.rtab[start[(row_ent[m] >> 16) & 3]++] = row_ent[m] | (uint32_t)m;
                    }
                    const int job = (int)P.stacks.size();
                    P.stacks.push_back(sk);
                    P.plan.begin(TcmJob{(int)(tg0 * 16), off});
                    for (int kp0 = 0; kp0 < kw; kp0 += 32) {
                        const int nk = std::min(2, (kw - kp0) / 16);
                        TcmStep stp{};
                        stp.raw = nullptr;
                        stp.b_kc = (c0 >> 3) + kp0 / 8;
                        stp.meta = nk | (6 << 12);
                        stp.rows = off;
                        stp.kp0 = kp0;
                        stp.n16 = job;
                        stp.cc0 = (kp0 - a) >= 0 ? (kp0 - a) / 4 : -((a - kp0 + 3) / 4);
                        stp.t0 = a;
                        stp.t1 = m2p4;
                        stp.t2 = 0;
                        P.plan.add(stp, 144.0 * q);
                    }
                }
            }
        };
        const int parts = std::max(1, std::min(plan_threads(), ncl / 256));
        std::vector<int> cut(parts + 1, ncl);
        cut[0] = 0;
        for (int k = 1, g = 0; k < parts; k++) {  // about far.size() / parts blocks a range
            const size_t goal = far.size() * k / parts;
            while (g < ncl && gs[g] < goal) g++;
            cut[k] = std::max(g, cut[k - 1]);
        }
        std::vector<Part> part(parts);
        std::vector<std::thread> th;
        for (int k = 1; k < parts; k++) th.emplace_back(plan_clusters, cut[k], cut[k + 1], std::ref(part[k]));
        plan_clusters(cut[0], cut[1], part[0]);
        for (std::thread& x : th) x.join();
        for (int k = 0; k < parts; k++) {
            Part& P = part[k];
            const int base_stack = (int)stacks.size();
            const long long base_tg = tgroups;
            for (TcmStep& stp : P.plan.steps) stp.n16 += base_stack;
            for (TcmJob& j : P.plan.jobs) j.r0 = (int)((long long)j.r0 + base_tg * 16);
            for (size_t i = 0; i < P.far_blocks.size(); i++) {
                toff[P.far_blocks[i]] += base_tg;
                P.far_term[i] += base_tg * 16;
            }
            stacks.insert(stacks.end(), P.stacks.begin(), P.stacks.end());
            far_blocks.insert(far_blocks.end(), P.far_blocks.begin(), P.far_blocks.end());
            far_term.insert(far_term.end(), P.far_term.begin(), P.far_term.end());
            p1.append(P.plan);
            tgroups += P.tgroups;
            P = Part();
        }
    }
    if (tgroups * 16 > 0x7fffffffll) {
        set_error("hmg_build_tensor_core_operands: %lld t_b terms exceed the plan's 32-bit term index", tgroups * 16);
        return HMG_ERR_UNSUPPORTED;
    }
    // pass 2: per tile, its near pairs (B = X) and low-rank pairs (B = t_b); tiles are
    // independent, so contiguous ranges of them are planned on several host threads and
    // the parts joined in tile order (the plan does not depend on the split)
    auto plan_tile = [&](int t, TcmPlan& P) -> bool {
        bool started = false;
        const int sp = (ts[t] + 3) & ~3;
        for (int p = tps[t]; p < tps[t + 1]; p++) {
            const int b = pblock[p];
            const bool dense = b < h->ndense;
            if (!dense && h->h_rank[b] == 0) continue;
            if (!started) {
                P.begin(TcmJob{tr0[t], ts[t]});
                started = true;
            }
            const PairDesc& d = desc[p];
            const char* data = static_cast<const char*>(d.data);
            if (dense) {
                const int a = h->h_c0[b] & 7, m2 = h->h_m2[b], kw = (a + m2 + 15) & ~15;
                for (int kp0 = 0; kp0 < kw; kp0 += 32) {
                    const int nk = std::min(2, (kw - kp0) / 16);
                    const int cc0 = std::max(kp0 - a, 0), ce = std::min(kp0 - a + 32, m2);
                    TcmStep stp{};
                    stp.raw = data + (size_t)cc0 * sp * 4;
                    stp.b_kc = (h->h_c0[b] >> 3) + kp0 / 8;
                    stp.meta = nk | (6 << 12);
                    stp.rows = ts[t];
                    stp.kp0 = kp0;
                    stp.n16 = (ce - cc0) * sp / 4;
                    stp.cc0 = cc0;
                    stp.t0 = a;
                    stp.t1 = m2;
                    stp.t2 = -1;
                    P.add(stp, 16.0 * stp.n16);
                }
            } else {
                const TcmTerms T = tcm_terms(h->h_rank[b], mixed ? h->h_r32[b] : h->h_rank[b], mixed ? h->h_r16[b] : 0);
                const int kw = tcm_kw(T);
                // chunk column of K position k, or -1 for a padding position
                auto chunk = [&](int k) -> int {
                    if (k < T.r32p) return k < T.r32 ? k : -1;
                    k -= T.r32p;
                    if (k < T.r16p) return k < T.r16 ? T.r32 + k / 2 : -1;
                    k -= T.r16p;
                    return k < T.r8 ? T.r32 + T.r16 / 2 + k / 4 : -1;
                };
                for (int kp0 = 0; kp0 < kw; kp0 += 32) {
                    const int nk = std::min(2, (kw - kp0) / 16);
                    const int mode = kp0 < T.r32p ? 6 : (kp0 < T.r32p + T.r16p ? 3 : 1);
                    int cc0 = 1 << 30, ce = -1;
                    for (int k = kp0; k < kp0 + 16 * nk; k++) {
                        const int c = chunk(k);
                        if (c >= 0) {
                            cc0 = std::min(cc0, c);
                            ce = std::max(ce, c + 1);
                        }
                    }
                    TcmStep stp{};
                    stp.raw = ce > cc0 ? data + (size_t)cc0 * sp * 4 : nullptr;
                    stp.b_kc = xkc + toff[b] * 2 + kp0 / 8;
                    stp.meta = nk | (mode << 12);
                    stp.rows = ts[t];
                    stp.kp0 = kp0;
                    stp.n16 = ce > cc0 ? (ce - cc0) * sp / 4 : 0;
                    stp.cc0 = cc0;
                    stp.t0 = T.r32 | T.r32p << 16;
                    stp.t1 = T.r16 | T.r16p << 16;
                    stp.t2 = T.r8 | (T.compact ? 1 << 16 : 0);
                    P.add(stp, 16.0 * stp.n16);
                }
            }
        }
        return started;
    };
    bool all_tiles = true;
    {
        const int parts = std::max(1, std::min(plan_threads(), nt / 64));
        std::vector<int> cut(parts + 1, nt);
        cut[0] = 0;
        for (int k = 1, t = 0; k < parts; k++) {  // about np / parts pairs a range
            const long long goal = (long long)np * k / parts;
            while (t < nt && tps[t] < goal) t++;
            cut[k] = std::max(t, cut[k - 1]);
        }
        std::vector<TcmPlan> part(parts);
        std::vector<char> all(parts, 1);
        auto run = [&](int k) {
            for (int t = cut[k]; t < cut[k + 1]; t++)
                if (!plan_tile(t, part[k])) all[k] = 0;
        };
        std::vector<std::thread> th;
        for (int k = 1; k < parts; k++) th.emplace_back(run, k);
        run(0);
        for (std::thread& x : th) x.join();
        for (int k = 0; k < parts; k++) {
            p2.append(part[k]);
            all_tiles = all_tiles && all[k];
            part[k] = TcmPlan();
        }
    }
    p1.finish();
    p2.finish();
    // every step's B copy inside the operand buffer, its raw copy inside a raw stage,
    // every row count within 128 rows, every stack row table inside its rows
    const long long bkc = xkc + tgroups * 2;
    for (const TcmPlan* L : {&p1, &p2})
        for (const TcmStep& sp : L->steps) {
            const int nk = sp.meta & 3;
            bool bad = nk < 1 || nk > 2 || sp.b_kc < 0 || sp.b_kc + 2 * nk > bkc || sp.rows < 1 || sp.rows > 128;
            if (L == &p1)
                bad = bad || sp.n16 < 0 || sp.n16 >= (int)stacks.size() || stacks[sp.n16].nq > 128;
            else  // whole slice columns of s_pad rows, at most 32 of them
                bad = bad || sp.n16 < 1 || (4 * sp.n16) % ((sp.rows + 3) & ~3) != 0 ||
                      (4 * sp.n16) / ((sp.rows + 3) & ~3) > 32 || sp.raw == nullptr;
            if (bad) {
                set_error("hmg_build_tensor_core_operands: internal error: a converted-operand step leaves its buffers");
                return HMG_ERR_UNSUPPORTED;
            }
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
    int* d_far = nullptr;
    long long* d_term = nullptr;
    if ((st = dalloc(reinterpret_cast<char**>(&h->tcm_stacks), std::max(stacks.size(), (size_t)1) * sizeof(TcmStack), s)) ||
        (st = dalloc(&h->tcm_tscale, (size_t)std::max(tgroups * 16, 1ll), s)) ||
        (st = dalloc(&d_far, std::max(far_blocks.size(), (size_t)1), s)) ||
        (st = dalloc(&d_term, std::max(far_term.size(), (size_t)1), s))) {
        dfree(d_far, s);
        dfree(d_term, s);
        free_tcm(h);
        return st;
    }
    if (!stacks.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tcm_stacks, stacks.data(), stacks.size() * sizeof(TcmStack), cudaMemcpyHostToDevice, s));
    if (!far_blocks.empty()) {
        HMG_CUDA_TRY(cudaMemcpyAsync(d_far, far_blocks.data(), far_blocks.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(d_term, far_term.data(), far_term.size() * sizeof(long long), cudaMemcpyHostToDevice, s));
        const int nf = (int)far_blocks.size();
        k_tcm_scales<<<ceil_div(nf, 8), 256, 0, s>>>(d_far, nf, h->rank, h->tier32, h->tier16, h->blk_m2, h->ptrV, d_term,
                                                      mixed ? 1 : 0, h->tcm_tscale);
        HMG_LAUNCH_CHECK();
    }
    dfree(d_far, s);
    dfree(d_term, s);
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
    const TcmStack* stacks = static_cast<const TcmStack*>(h->tcm_stacks);
    if (h->tcm_njobs[0] > 0) {
        k_tcm_pass<0, NV><<<h->nsm, TCM_THREADS, smem, s>>>(
            reinterpret_cast<const TcmStep*>(h->tcm_steps[0]), reinterpret_cast<const TcmJob*>(h->tcm_jobs[0]),
            reinterpret_cast<const int2*>(h->tcm_cta[0]), stacks, bbuf, xkc, h->tcm_tscale, nullptr, 0, nullptr, 0,
            h->dev_err);
        HMG_LAUNCH_CHECK();
    }
    if (!h->tcm_all_tiles)  // rows of tiles without products (all their blocks of rank 0) are zero
        HMG_CUDA_TRY(cudaMemset2DAsync(Y, sizeof(double) * ldy, 0, sizeof(double) * h->n[0], nrhs, s));
    if (h->tcm_njobs[1] > 0) {
        k_tcm_pass<1, NV><<<h->nsm, TCM_THREADS, smem, s>>>(
            reinterpret_cast<const TcmStep*>(h->tcm_steps[1]), reinterpret_cast<const TcmJob*>(h->tcm_jobs[1]),
            reinterpret_cast<const int2*>(h->tcm_cta[1]), stacks, bbuf, 0, nullptr, h->perm[0], nrhs, Y, ldy,
            h->dev_err);
        HMG_LAUNCH_CHECK();
    }
    return HMG_OK;
}

// 2..64 vectors in one pass: MMAs of N = 32 for up to 32 vectors, N = 64 above
hmg_status matvec_multi_tcm(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    return nrhs > 32 ? tcm_product<64>(h, nrhs, X, ldx, Y, ldy) : tcm_product<32>(h, nrhs, X, ldx, Y, ldy);
}

}  // namespace hmg
