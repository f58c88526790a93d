// tc.cu -- multi-vector products on the tensor cores (tcgen05), BF16 operands.
//
// hmg_build_bf16_factors converts the FP32 low-rank factors and the FP32 stored near
// field of a handle into BF16 tcgen05 operands; hmg_matvec_multi then multiplies 2..64
// vectors per pass with them, every product on the tensor cores:
//
//   pass 1 (k_tc_pass<0>): per admissible block, t_b = V_b^T X_b (M = rank rounded to
//     16, padded to 128; N = 32 or 64 vectors; K = the block's columns), written as BF16
//     operand cores of pass 2;
//   pass 2 (k_tc_pass<1>): per row tile (M = 128 rows), the sum over its pairs of
//     U_slice * t_b (low rank; K = rank) and D_slice * X_b (near field; K = columns),
//     accumulated in tensor memory and written to the tile's rows of Y (caller order).
//
// Both passes run one persistent kernel: one CTA per SM walks a job list balanced on
// the host (longest job first onto the least loaded CTA).  A job (a block in pass 1, a
// tile in pass 2) is a run of "steps", each an A chunk (<= 48 KB) and the B chunk it
// multiplies (<= 32 KB).  Warp 4 copies steps with bulk copies (cp.async.bulk,
// completion counted on the step slot's mbarrier) into a 208 KB byte ring that holds up
// to 16 steps of any size; warp 5 issues the MMAs (one elected lane, accumulating in one
// of two tensor-memory buffers) and frees each step's bytes with tcgen05.commit; warps
// 0-3 drain a finished buffer (tcgen05.ld, one 32-row quarter each) while the next job
// (split operands: the next step) accumulates in the other.
//
// Operand layout (no swizzle, K-major core matrices of 8 rows x 16 bytes), K cores
// outermost so that every K range of an operand is one contiguous byte range:
//   A (U slice, near slice or V_b^T): core (kc, mc) at (kc * rc + mc) * 128 bytes, rc
//     = stored row cores (tile rows or rank rounded to 8).  The MMA's M is 128: rows
//     past 8 rc read the next K core's bytes (or the rest of the stage) and only reach
//     accumulator rows that are never read back.
//   B (X or t_b): core (nc, kc) = vectors 8nc..8nc+7, K 8kc..8kc+7 at (kc * N / 8 + nc) * 128.
//   X is kept over the Z-ordered column index with 8 columns per K core; a block whose
//   columns start at c0 reads K cores from c0 / 8 on, and its A operand carries
//   c0 mod 8 leading zero columns so the K positions line up.
//   Split operands (P = 2 or 3 BF16 parts) are interleaved by K core: K core kc holds
//   part 0's cores, then part 1's, then part 2's (A: P * rc row cores per K core; B: P *
//   N * 16 bytes per K core), so that one copy brings every part of a K range.
// Descriptors: leading byte offset = stride between K cores (A: P * rc * 128, B: P * N *
// 16), stride byte offset = stride between row cores (128); part q starts q * rc * 128
// (A) or q * N * 16 (B) bytes into each K core.  Instruction kind::f16 with BF16 A/B,
// FP32 D, M 128, N 32 (up to 32 vectors) or 64.
// Every wait is bounded (pipeline.cuh): on a time-out the waiting role records an error
// code in the handle's flag, leaves its loop, and the CTA waits for its own copies and
// MMAs before freeing tensor memory.  BF16 rounding of factors, near field, X and t_b
// (~4e-3 per entry) bounds the accuracy: products agree with FP32 ones to ~1e-3.  Split
// operands (2 or 3 BF16 parts, 3 or 6 MMAs per K step) accumulate hi*hi and the
// correction terms apart and drain both after every step (the tensor cores' own FP32
// accumulation loses accuracy over long chains); the epilogue sums the steps in FP32:
// ~7e-6 with two parts, ~4e-7 with three.
#include <cuda_bf16.h>

#include <algorithm>
#include <queue>
#include <vector>

#include "hmg_matrix.cuh"
#include "pipeline.cuh"
#include "stream.cuh"
#include "tc_common.cuh"

namespace hmg {

static constexpr int TC_NMAX = 64;         // vectors per pass at most (MMA N: 32 or 64)
static constexpr int TC_MAXR16 = 128;      // largest rank rounded to 16 (pass 1's M)
static constexpr int TC_SLOTS = 16;        // steps in flight per CTA at most
static constexpr int TC_RING = 204800;     // bytes of the operand ring (200 KB)
static constexpr int TC_ISSUERS = 8;       // lanes of the copy warp issuing at once
static constexpr int TC_ABYTES = 49152;    // A chunk of a step: at most 384 core matrices
static constexpr int TC_BBYTES = 32768;    // B chunks of a step: at most 32 K cores x 8 vector cores
static constexpr int TC_MAXSTEP = 16;      // MMAs per step
static constexpr int TC_MAXSUB = 4;        // sub-steps (B copies) per step
static constexpr int TC_THREADS = 192;     // warps 0-3 epilogue, 4 copies, 5 MMAs
// B operands (X and t_b) are addressed in K cores: 8 columns or terms x NV vectors, NV * 16 bytes

// A step: one copy of A (the A chunks of up to TC_MAXSUB sub-steps, one after another in
// the A arena) and one copy of B per sub-step (X or t_b cores), placed after A in the ring.
struct TcStep {
    long long a_off;               // bytes into the A arena
    long long b_off[TC_MAXSUB];    // first K core in the B buffer (X cores, then t_b cores), per sub-step
    int meta;                      // bits 0-7: row cores of A (its K-core stride / 128); bit 8: first step
                                   // of a job; bit 9: last; bits 10-11: sub-steps - 1; bits 16-23: MMAs
    int kss;                       // MMAs (of K = 16) of sub-step j, minus 1, in bits 4j..4j+3
};
static_assert(sizeof(TcStep) == 48, "TcStep layout");

struct TcJob {
    int r0;    // pass 2: first Z row of the tile; pass 1: t_b's first 16-term group
    int rows;  // pass 2: rows of the tile; pass 1: rank rounded to 16
};

// ---------------------------------------------------------------------------
// conversion of the FP32 factors and near field (once, by hmg_build_bf16_factors)
// ---------------------------------------------------------------------------
// An operand's BF16 parts: part 0 is the BF16 rounding of a value, part p the BF16
// rounding of what parts 0..p-1 miss (each difference is exact in FP32), so that 1, 2
// or 3 parts carry 8, 16 or 24 significant bits of it.  The parts are interleaved by K
// core: K core kc of an operand with rc row cores holds part 0's rc cores, then part
// 1's, then part 2's, so that one copy brings every part of a K range.  Element
// `within` (core mc * 64 + position) of K core kc, part q, sits at
// base + ((kc * parts + q) * rc) * 64 + within.
__device__ __forceinline__ void store_parts(__nv_bfloat16* out, int parts, long long base, long long kc, int rc,
                                            int within, float v)
{
#pragma unroll
    for (int q = 0; q < 3; q++)
        if (q < parts) {
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            out[base + ((kc * parts + q) * rc) * 64 + within] = h;
            v -= __bfloat162float(h);
        }
}

// far pair: U slice (s_pad x r, column-major) -> A cores, rc = s8 / 8, K = r16
__global__ void k_tc_u(const PairDesc* desc, const int* plist, const long long* aoff, const int* ptile,
                       const int* tile_s, int n, __nv_bfloat16* out, int parts)
{
    const int u = blockIdx.x;
    if (u >= n) return;
    const int p = plist[u];
    const PairDesc d = desc[p];
    const int s = tile_s[ptile[u]], sp = (s + 3) & ~3, s8 = (s + 7) & ~7;
    const int r = d.ncol, r16 = (r + 15) & ~15;
    const float* src = static_cast<const float*>(d.data);
    const long long base = aoff[u] / 2;
    const int rc = s8 / 8;
    for (int idx = threadIdx.x; idx < s8 * r16; idx += blockDim.x) {
        const int core = idx >> 6, e = idx & 63;
        const int kc = core / rc, mc = core - kc * rc;
        const int i = mc * 8 + (e >> 3), k = kc * 8 + (e & 7);
        store_parts(out, parts, base, kc, rc, mc * 64 + e, (i < s && k < r) ? src[(size_t)k * sp + i] : 0.0f);
    }
}

// near pair: slice (s_pad x m2, column-major) -> A cores with c0 mod 8 leading zero columns
__global__ void k_tc_near(const PairDesc* desc, const int* plist, const long long* aoff, const int* ptile,
                          const int* tile_s, int n, __nv_bfloat16* out, int parts)
{
    const int u = blockIdx.x;
    if (u >= n) return;
    const PairDesc d = desc[plist[u]];
    const int s = tile_s[ptile[u]], sp = (s + 3) & ~3, s8 = (s + 7) & ~7;
    const int m2 = d.ncol, a = d.c0 & 7, kw = (a + m2 + 15) & ~15;
    const float* src = static_cast<const float*>(d.data);
    const long long base = aoff[u] / 2;
    const int rc = s8 / 8;
    for (long long idx = threadIdx.x; idx < (long long)s8 * kw; idx += blockDim.x) {
        const int core = (int)(idx >> 6), e = (int)(idx & 63);
        const int kc = core / rc, mc = core - kc * rc;
        const int i = mc * 8 + (e >> 3), c = kc * 8 + (e & 7) - a;
        store_parts(out, parts, base, kc, rc, mc * 64 + e, (i < s && c >= 0 && c < m2) ? src[(size_t)c * sp + i] : 0.0f);
    }
}

// admissible block: V_b^T (rows of m2p FP32 entries per term) -> its rows of a stack's A
// cores.  A stack holds the V^T of blocks with the same columns, one under the other
// (vaux: stack row cores << 8 | the block's first row core in the stack).
__global__ void k_tc_v(const int* blist, const long long* voff, const int* vaux, int n, void* const* ptrV,
                       const int* rank, const int* blk_c0, const int* blk_m2, __nv_bfloat16* out, int parts)
{
    const int u = blockIdx.x;
    if (u >= n) return;
    const int b = blist[u], rc = vaux[u] >> 8, off8 = vaux[u] & 255;
    const int r = rank[b], r16 = (r + 15) & ~15, m2 = blk_m2[b], m2p = (m2 + 3) & ~3;
    const int a = blk_c0[b] & 7, kw = (a + m2 + 15) & ~15;
    const float* V = static_cast<const float*>(ptrV[b]);
    const long long base = voff[u] / 2;
    const int rb = r16 / 8;
    for (long long idx = threadIdx.x; idx < (long long)r16 * kw; idx += blockDim.x) {
        const int core = (int)(idx >> 6), e = (int)(idx & 63);
        const int kc = core / rb, mc = core - kc * rb;
        const int m = mc * 8 + (e >> 3), c = kc * 8 + (e & 7) - a;
        store_parts(out, parts, base, kc, rc, (off8 + mc) * 64 + e,
                    (m < r && c >= 0 && c < m2) ? V[(size_t)m * m2p + c] : 0.0f);
    }
}

// ---------------------------------------------------------------------------
// the persistent pass kernel
// ---------------------------------------------------------------------------
struct TcSmem {
    unsigned char ring[TC_RING];   // operand ring: each step's A chunk, then its B chunk
    __nv_bfloat16 stg[4][32 * TC_NMAX];  // pass 1 epilogue: 4 K cores of t_b per warp (also
                                         // takes the MMA's reads of unused A rows past the ring)
    uint64_t full[TC_SLOTS], empty[TC_SLOTS], accf[2], acce[2], fin;
    uint32_t slot_a[TC_SLOTS], slot_b[TC_SLOTS];  // shared addresses of a step's A and B
    int slot_meta[TC_SLOTS];                       // a step's meta word
    int slot_pos[TC_SLOTS];                        // ring offset of a step (copy warp only)
    int step_bytes[32];                            // bytes of the copy warp's current 32 steps
    uint32_t tmem;
    int fail;
};

static_assert(sizeof(TcSmem) <= 227 * 1024, "TcSmem exceeds the shared memory of a CTA");

__device__ __forceinline__ TcStep load_step(const TcStep* steps, int i, int n)
{
    TcStep st{};
    if (i < n) st = steps[i];
    return st;
}

// Steps of CTA c: [cta[c].y, cta[c+1].y); its jobs: [cta[c].x, cta[c+1].x).  NV vectors per
// pass (MMA N); B K cores are NV * 16 bytes.  Pass 1 (MODE 0) writes t_b cores, K core kc of
// job j (a stack) to B K core tb_kc + map[16 j + kc]; pass 2 (MODE 1) writes (add_y: adds
// to) rows of Y, tile row i to Y row map[r0 + i].  PARTS > 1 (split operands): every
// operand comes as PARTS BF16 parts interleaved by K core (A: a step's row cores field
// counts the row cores of all parts; B: a K core is PARTS * NV * 16 bytes), and each K
// step runs hi*hi plus the correction terms down to 2^-16 of it: hi*lo + lo*hi (2
// parts), and hi*lo2 + lo2*hi + lo*lo (3 parts).
template <int MODE, int NV, int PARTS>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_tc_pass(const TcStep* __restrict__ steps, const TcJob* __restrict__ jobs, const int2* __restrict__ cta,
              const char* __restrict__ A, char* Bbuf, long long tb_kc, const int* __restrict__ map, int nrhs,
              double* Y, int ldy, int add_y, int* err)
{
    constexpr int KB = NV * 16 * PARTS;  // bytes of a B K core, all parts
    constexpr bool SPLIT = PARTS > 1;
    // two accumulator buffers; split: each holds hi*hi (columns 0..NV-1) and the
    // correction terms (NV..2NV-1)
    constexpr int TMEM_COLS = SPLIT ? 4 * NV : 2 * NV;
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem& sm = *reinterpret_cast<TcSmem*>(tc_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int2 lo = cta[blockIdx.x], hi = cta[blockIdx.x + 1];
    const int nsteps = hi.y - lo.y;
    const TcStep* my_steps = steps + lo.y;
    volatile int* fail = &sm.fail;
    if (tid == 0) {
        for (int s = 0; s < TC_SLOTS; s++) {
            mbar_init(&sm.full[s], 1);
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

    if (warp == 4) {
        // ---- copies.  Lane l holds step i0 + l (the next 32 are loaded meanwhile).  In
        // rounds, lane 0 places up to TC_ISSUERS steps at the ring's head (after the steps
        // they would overwrite, oldest first, have been freed by their MMAs) and the lanes
        // holding them issue their copies side by side: one thread issues one bulk copy
        // every few hundred cycles, so small steps need several issuers to keep HBM busy. ----
        uint64_t pol;
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
        int issued = 0, tail = 0, head = 0;  // lane 0's ring state
        bool ok = true;
        TcStep nxt = load_step(my_steps, lane, nsteps);
        for (int i0 = 0; i0 < nsteps && ok; i0 += 32) {
            const TcStep mine = nxt;
            nxt = load_step(my_steps, i0 + 32 + lane, nsteps);
            const int cnt = min(32, nsteps - i0);
            const int ks_all = (mine.meta >> 16) & 0xff;
            const int ab = ks_all * 2 * (mine.meta & 0xff) * 128, bb = ks_all * 2 * KB;
            __syncwarp();
            sm.step_bytes[lane] = ab + bb;
            __syncwarp();
            for (int k = 0; k < cnt && ok;) {
                int m = 0;
                if (lane == 0) {
                    while (k + m < cnt && m < TC_ISSUERS) {
                        const int i = i0 + k + m, z = sm.step_bytes[k + m];
                        int pos = -1;
                        if (tail == i) {
                            pos = 0;  // nothing in flight
                        } else if (i - tail < TC_SLOTS) {
                            const int tpos = sm.slot_pos[tail % TC_SLOTS];  // oldest step in flight
                            if (tpos < head) {                              // in flight: [tpos, head)
                                if (head + z <= TC_RING) pos = head;
                                else if (z <= tpos) pos = 0;
                            } else if (head + z <= tpos) {                  // in flight: [tpos, end) + [0, head)
                                pos = head;
                            }
                        }
                        if (pos >= 0) {
                            sm.slot_pos[i % TC_SLOTS] = pos;
                            head = pos + z;
                            m++;
                            continue;
                        }
                        if (mbar_test_wait(&sm.empty[tail % TC_SLOTS], (tail / TC_SLOTS) & 1)) {
                            tail++;  // the oldest step's MMAs are done: its bytes and slot are free
                            continue;
                        }
                        if (m > 0) break;  // issue what is placed; wait in the next round
                        if (*fail || !mbar_wait(&sm.empty[tail % TC_SLOTS], (tail / TC_SLOTS) & 1, err, 11)) {
                            ok = false;
                            break;
                        }
                        tail++;
                    }
                    issued += m;
                }
                m = __shfl_sync(~0u, m, 0);
                ok = __shfl_sync(~0u, ok, 0);
                __syncwarp();
                if (lane >= k && lane < k + m) {
                    const int slot = (i0 + lane) % TC_SLOTS, pos = sm.slot_pos[slot];
                    const uint32_t a = smem_u32(sm.ring + pos);
                    sm.slot_a[slot] = a;
                    sm.slot_b[slot] = a + ab;
                    sm.slot_meta[slot] = mine.meta;
                    mbar_arrive_expect_tx(&sm.full[slot], ab + bb);
                    bulk_g2s_first(sm.ring + pos, A + mine.a_off, ab, &sm.full[slot], pol);
                    const int nsub = ((mine.meta >> 10) & 3) + 1;
                    int boff = ab;
#pragma unroll
                    for (int j = 0; j < TC_MAXSUB; j++)
                        if (j < nsub) {
                            const int kb = (((mine.kss >> (4 * j)) & 15) + 1) * 2 * KB;
                            bulk_g2s(sm.ring + pos + boff, Bbuf + mine.b_off[j] * KB, kb, &sm.full[slot]);
                            boff += kb;
                        }
                }
                k += m;
            }
        }
        if (!ok) *fail = 1;
        // the last copy into every slot has landed before the CTA leaves (a no-op unless a wait failed)
        issued = __shfl_sync(~0u, issued, 0);
        if (lane == 0)
            for (int s = 0; s < TC_SLOTS && s < issued; s++)
                mbar_wait(&sm.full[s], ((issued - 1 - s) / TC_SLOTS) & 1, err, 12);
    } else if (warp == 5) {
        // ---- MMAs: lane 0 alone; each step's parameters come with its slot ----
        if (lane == 0) {
            int jc = 0;
            for (int i = 0; i < nsteps; i++) {
                const int slot = i % TC_SLOTS;
                if (*fail || !mbar_wait(&sm.full[slot], (i / TC_SLOTS) & 1, err, 14)) {
                    *fail = 1;
                    break;
                }
                const uint32_t a0 = sm.slot_a[slot], b0 = sm.slot_b[slot];
                const int meta = sm.slot_meta[slot], ks_all = (meta >> 16) & 0xff;
                const bool first = meta & 256, last = meta & 512;
                // split: every step has its own accumulator (drained by the epilogue, which
                // sums the steps of a job in FP32 on the CUDA cores), so that no accumulator
                // runs through more than one step's MMAs; otherwise one per job
                const int u = SPLIT ? i : jc, buf = u & 1;
                if ((SPLIT || first) && u >= 2) {  // the epilogue has read this buffer's previous use
                    if (!mbar_wait(&sm.acce[buf], ((u >> 1) - 1) & 1, err, 13)) {
                        *fail = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                }
                // The step's A chunks lie one after another, so do its B chunks: MMA q reads A
                // 2q K cores and B 2q K cores further on.  The descriptors advance by plain
                // adds to their start-address field (16-byte units; shared addresses stay
                // below 2^18, so the field never carries): this lane's issue rate bounds the pass.
                const uint32_t lbo = (uint32_t)(meta & 0xff) * 128u;
                const uint32_t d = tmem + (uint32_t)(buf * (SPLIT ? 2 * NV : NV));
                const uint64_t da = (2 * lbo) >> 4, db = (2 * KB) >> 4;
                uint64_t ad = smem_desc(a0, lbo, 128), bd = smem_desc(b0, KB, 128);
                // in each K core, part q of A (of B) lies q * alo (q * blo) 16-byte units
                // after part 0: the row cores of one part (the vector cores of one part)
                const uint64_t alo = (uint64_t)((meta & 0xff) / PARTS) * 8, blo = (uint64_t)NV;
                uint32_t acc = (SPLIT || first) ? 0u : 1u;
#pragma unroll 4
                for (int q = 0; q < ks_all; q++) {
                    if (SPLIT) {
                        // the correction terms in their own accumulator (added to hi*hi they
                        // would each be truncated at the scale of the 256x larger sum).  The
                        // parts of a B K core lie side by side along N, so one MMA of N = 2 NV
                        // gives hi = A0 B0 and the correction's A0 B1.
                        tc_mma(d, ad, bd, tc_idesc<2 * NV>(), acc);
                        tc_mma(d + NV, ad + alo, bd, tc_idesc<NV>(), 1u);
                        if (PARTS == 3) {
                            tc_mma(d + NV, ad, bd + 2 * blo, tc_idesc<NV>(), 1u);
                            tc_mma(d + NV, ad + 2 * alo, bd, tc_idesc<NV>(), 1u);
                            tc_mma(d + NV, ad + alo, bd + blo, tc_idesc<NV>(), 1u);
                        }
                    } else {
                        tc_mma(d, ad, bd, tc_idesc<NV>(), acc);
                    }
                    acc = 1u;
                    ad += da;
                    bd += db;
                }
                tc_commit(&sm.empty[slot]);
                if (SPLIT || last) tc_commit(&sm.accf[buf]);
                if (last) jc++;
            }
            tc_commit(&sm.fin);  // every MMA issued here has completed before tensor memory is freed
            mbar_wait(&sm.fin, 0, err, 15);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w owns accumulator rows 32w..32w+31 ----
        const int row = warp * 32 + lane;
        // a finished job's sums f (row `row`, vectors 0..NV-1) to their destination
        auto emit = [&](float (&f)[NV], int rows, int yrow, const int (&tdst)[4]) {
            if (MODE == 1) {
                if (row < rows) {
                    double* y = Y + yrow;
#pragma unroll
                    for (int q = 0; q < NV; q++)
                        if (q < nrhs) y[(size_t)q * ldy] = (add_y ? y[(size_t)q * ldy] : 0.0) + (double)f[q];
                }
            } else {
                // term row -> B cores of pass 2 (K = term): element (term m, vector q) at byte
                // ((m / 8) * NV / 8 + q / 8) * 128 + (q % 8) * 16 + (m % 8) * 2 of its block's
                // t_b; this warp's 32 stack rows fill the stack's K cores 4w..4w+3.  Lanes 2p,
                // 2p+1 pair their terms into 32-bit words (even lane: vector 2t, odd lane:
                // vector 2t+1); 16-byte row u of the staging (K core u / NV, vector u % NV) sits
                // at u ^ (2 (u / NV)), which spreads the four K cores over all banks.
                uint32_t* stg = reinterpret_cast<uint32_t*>(sm.stg[warp]);
                const bool odd = lane & 1;
#pragma unroll
                for (int part = 0; part < PARTS; part++) {
                    // part 0: BF16 of t; part p: BF16 of what parts 0..p-1 miss.  Each lane
                    // rounds its own pair once (one packed conversion), keeps the residual
                    // in f for the next part, and swaps halves with its neighbour: the even
                    // lane keeps the low halves (vector 2t), the odd lane the high ones.
#pragma unroll
                    for (int t = 0; t < NV / 2; t++) {
                        const uint32_t own = pack_bf16(f[2 * t], f[2 * t + 1]);
                        if (part + 1 < PARTS) {
                            f[2 * t] -= __uint_as_float(own << 16);
                            f[2 * t + 1] -= __uint_as_float(own & 0xffff0000u);
                        }
                        const uint32_t other = __shfl_xor_sync(~0u, own, 1);
                        const int q = odd ? 2 * t + 1 : 2 * t;
                        const uint32_t w = odd ? __byte_perm(own, other, 0x3276) : __byte_perm(own, other, 0x5410);
                        const int u = (lane >> 3) * NV + q;
                        stg[(u ^ ((lane >> 3) * 2)) * 4 + ((lane & 7) >> 1)] = w;
                    }
                    __syncwarp();
                    uint4* dst = reinterpret_cast<uint4*>(Bbuf);
                    const uint4* src = reinterpret_cast<const uint4*>(stg);
#pragma unroll
                    for (int it = 0; it < NV / 8; it++) {
                        const int u = it * 32 + lane, kcl = u / NV;
                        if (warp * 4 + kcl < (rows >> 3))
                            dst[((size_t)(tb_kc + tdst[kcl]) * PARTS + part) * NV + (u % NV)] = src[u ^ (kcl * 2)];
                    }
                    __syncwarp();
                }
            }
        };
        // where job (r0, rows)'s rows go, fetched before its accumulator is waited for
        auto dests = [&](int r0, int rows, int& yrow, int (&tdst)[4]) {
            yrow = (MODE == 1 && row < rows) ? map[r0 + row] : 0;
#pragma unroll
            for (int q = 0; q < 4; q++)
                tdst[q] = (MODE == 0 && warp * 4 + q < (rows >> 3)) ? map[r0 * 16 + warp * 4 + q] : 0;
        };
        // the next drain of accumulator buffer buf (use u of it) -> this thread's row
        auto drain = [&](int u, int buf, float (&f)[NV], bool fresh) -> bool {
            if (!__all_sync(~0u, !*fail && mbar_wait(&sm.accf[buf], (u >> 1) & 1, err, 16))) return false;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t taddr = tmem + (uint32_t)(buf * (SPLIT ? 2 * NV : NV)) + ((uint32_t)(warp * 32) << 16);
#pragma unroll
            for (int h = 0; h < NV / 32; h++) {
                uint32_t v[32], c[32];
                tc_ld32(taddr + 32 * h, v);
                if (SPLIT) tc_ld32(taddr + NV + 32 * h, c);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                // hi + c, then into the running sums: packed pairs, uniform branches
                if (SPLIT) {
#pragma unroll
                    for (int q = 0; q < 32; q += 2) add_f32x2(v[q], v[q + 1], c[q], c[q + 1]);
                }
                if (fresh) {
#pragma unroll
                    for (int q = 0; q < 32; q++) f[32 * h + q] = __uint_as_float(v[q]);
                } else {
#pragma unroll
                    for (int q = 0; q < 32; q += 2) add_f32x2(f[32 * h + q], f[32 * h + q + 1], v[q], v[q + 1]);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.acce[buf]);
            return true;
        };
        const int njobs = hi.x - lo.x;
        const int2* my_jobs = reinterpret_cast<const int2*>(jobs) + lo.x;
        bool ok = true;
        float f[NV];
        if (SPLIT) {
            // one drain per step; lane l holds the meta word of step i0 + l
            int jc = 0, rows = 0, yrow = 0, tdst[4] = {0, 0, 0, 0};
            for (int i0 = 0; i0 < nsteps && ok; i0 += 32) {
                const int mt = i0 + lane < nsteps ? my_steps[i0 + lane].meta : 0;
                const int cnt = min(32, nsteps - i0);
                for (int k = 0; k < cnt; k++) {
                    const int i = i0 + k, meta = __shfl_sync(~0u, mt, k);
                    const bool first = meta & 256, last = meta & 512;
                    if (first) {
                        const int2 jb = jc < njobs ? my_jobs[jc] : make_int2(0, 0);
                        rows = jb.y;
                        dests(jb.x, rows, yrow, tdst);
                    }
                    if (!(ok = drain(i, i & 1, f, first))) break;
                    if (last) {
                        emit(f, rows, yrow, tdst);
                        jc++;
                    }
                }
            }
        } else {
            // one drain per job; lane l holds job j0 + l
            int2 nxt = lane < njobs ? my_jobs[lane] : make_int2(0, 0);
            for (int j0 = 0; j0 < njobs && ok; j0 += 32) {
                const int2 mine = nxt;
                if (j0 + 32 + lane < njobs) nxt = my_jobs[j0 + 32 + lane];
                const int cnt = min(32, njobs - j0);
                for (int k = 0; k < cnt; k++) {
                    const int r0 = __shfl_sync(~0u, mine.x, k), rows = __shfl_sync(~0u, mine.y, k);
                    const int jc = j0 + k;
                    int yrow, tdst[4];
                    dests(r0, rows, yrow, tdst);
                    if (!(ok = drain(jc, jc & 1, f, true))) break;
                    emit(f, rows, yrow, tdst);
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
// host side
// ---------------------------------------------------------------------------

void free_tc(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    free_tcm(h);  // the on-chip variant's plan and buffers (tcm.cu)
    if (h->tc_u) cudaFree(h->tc_u);
    if (h->tc_v) cudaFree(h->tc_v);
    if (h->tc_bbuf) {
        cudaStreamSynchronize(s);  // a product in flight may still read it
        cudaFree(h->tc_bbuf);
    }
    h->tc_u = h->tc_v = h->tc_bbuf = nullptr;
    dfree(h->tc_kmap, s);
    for (int q = 0; q < 2; q++) {
        dfree(h->tc_steps[q], s);
        dfree(h->tc_jobs[q], s);
        dfree(h->tc_cta[q], s);
        h->tc_njobs[q] = 0;
    }
    h->tc_ready = false;
    h->tc_bytes = 0;
    h->tc_xkc = h->tc_tkc = 0;
    h->tc_grid = 0;
    h->tc_all_tiles = false;
    h->tc_near = false;
    h->tc_parts = 1;
}

namespace {

struct Chunk {
    long long a_off, b_kc;   // A arena byte, B buffer K core
    int ks, rc;              // MMAs; row cores of A
};

struct JobList {
    std::vector<Chunk> chunks;   // in job order
    std::vector<int> chunk0;     // per job: first chunk (then the end)
    std::vector<TcJob> info;
    std::vector<double> cost;
    std::vector<TcStep> steps;   // built by make_steps, in job order
    std::vector<int> step0;
    void begin(TcJob j)
    {
        chunk0.push_back((int)chunks.size());
        info.push_back(j);
        cost.push_back(0.0);
    }
    // K cores [0, kcores) of an A operand with rc row cores (B from K core b_kc on), in
    // chunks of at most kcc; cost in bytes with 64 vectors
    void add(long long a_off, long long b_kc, int rc, int kcores, int kcc, double b_weight)
    {
        for (int kc0 = 0; kc0 < kcores; kc0 += kcc) {
            const int nk = std::min(kcc, kcores - kc0);
            chunks.push_back(Chunk{a_off + (long long)kc0 * rc * 128, b_kc + kc0, nk / 2, rc});
            cost.back() += (double)nk * rc * 128 + b_weight * nk * 16 * TC_NMAX;
        }
    }
    // Steps of every job: consecutive chunks share a step (merge) while their A chunks
    // are adjacent and the step stays within TC_MAXSUB sub-steps, a_limit bytes of A and
    // ks_limit MMAs (B bytes).
    void make_steps(bool merge, long long a_limit, int ks_limit)
    {
        chunk0.push_back((int)chunks.size());
        for (size_t j = 0; j + 1 < chunk0.size(); j++) {
            step0.push_back((int)steps.size());
            TcStep cur{};
            int nsub = 0, ks_all = 0;
            long long ab = 0;
            auto flush = [&]() {
                if (!nsub) return;
                cur.meta |= (nsub - 1) << 10 | ks_all << 16;
                steps.push_back(cur);
                cur = TcStep{};
                nsub = ks_all = 0;
                ab = 0;
            };
            for (int c = chunk0[j]; c < chunk0[j + 1]; c++) {
                const Chunk& k = chunks[c];
                const long long kab = (long long)k.ks * 2 * k.rc * 128;
                if (!(merge && nsub > 0 && nsub < TC_MAXSUB && k.rc == (cur.meta & 0xff) && k.a_off == cur.a_off + ab &&
                      ab + kab <= a_limit && ks_all + k.ks <= ks_limit))
                    flush();
                if (!nsub) {
                    cur.a_off = k.a_off;
                    cur.meta = k.rc;
                }
                cur.b_off[nsub] = k.b_kc;
                cur.kss |= (k.ks - 1) << (4 * nsub);
                nsub++;
                ks_all += k.ks;
                ab += kab;
            }
            flush();
            steps[step0.back()].meta |= 256;
            steps.back().meta |= 512;
        }
        step0.push_back((int)steps.size());
    }
};

// Every copy a step issues stays inside its arena and its stage, and every job's
// output inside its buffer: checked here, on the host, before any launch.
bool steps_in_bounds(const JobList& L, long long abytes, long long bkcores, long long out_limit, int q, int parts)
{
    for (const TcStep& st : L.steps) {
        const int rc = st.meta & 0xff, nsub = ((st.meta >> 10) & 3) + 1, ks_all = (st.meta >> 16) & 0xff;
        // rc counts the row cores of all parts; a B K core holds every part
        const long long ab = (long long)ks_all * 2 * rc * 128, bb = (long long)ks_all * 2 * 16 * TC_NMAX * parts;
        int sum = 0;
        for (int j = 0; j < nsub; j++) {
            const int ks = ((st.kss >> (4 * j)) & 15) + 1;
            if (st.b_off[j] < 0 || st.b_off[j] + 2ll * ks > bkcores) return false;
            sum += ks;
        }
        if (sum != ks_all || rc < 1 || rc > 16 * parts || rc % parts || ab > TC_ABYTES || bb > TC_BBYTES ||
            st.a_off < 0 || st.a_off % 16 ||
            st.a_off + ab > abytes)
            return false;
    }
    for (const TcJob& j : L.info) {
        if (j.rows < 1 || j.rows > 128 || j.r0 < 0) return false;
        if (q == 1 ? (long long)j.r0 + j.rows > out_limit : j.r0 >= out_limit) return false;
    }
    return true;
}

// longest job first onto the least loaded CTA; emits steps and jobs CTA by CTA
hmg_status upload_jobs(hmg_matrix* h, int q, JobList& L, double job_cost, int grid)
{
    cudaStream_t s = h->stream;
    const int nj = (int)L.info.size();
    std::vector<int> order(nj);
    for (int j = 0; j < nj; j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return L.cost[a] > L.cost[b]; });
    using Load = std::pair<double, int>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int c = 0; c < grid; c++) heap.push({0.0, c});
    std::vector<std::vector<int>> mine(grid);
    for (int j : order) {
        Load l = heap.top();
        heap.pop();
        mine[l.second].push_back(j);
        heap.push({l.first + L.cost[j] + job_cost, l.second});
    }
    std::vector<TcStep> steps;
    std::vector<TcJob> jobs;
    std::vector<int2> cta(grid + 1);
    steps.reserve(L.steps.size());
    jobs.reserve(nj);
    for (int c = 0; c < grid; c++) {
        cta[c] = make_int2((int)jobs.size(), (int)steps.size());
        for (int j : mine[c]) {
            jobs.push_back(L.info[j]);
            const int a = L.step0[j], b = L.step0[j + 1];
            for (int i = a; i < b; i++) steps.push_back(L.steps[i]);
        }
    }
    cta[grid] = make_int2((int)jobs.size(), (int)steps.size());
    hmg_status st;
    if ((st = dalloc(&h->tc_steps[q], std::max(steps.size(), (size_t)1) * sizeof(TcStep), s)) ||
        (st = dalloc(&h->tc_jobs[q], std::max(jobs.size(), (size_t)1) * sizeof(TcJob), s)) ||
        (st = dalloc(&h->tc_cta[q], (size_t)(grid + 1) * sizeof(int2), s)))
        return st;
    if (!steps.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tc_steps[q], steps.data(), steps.size() * sizeof(TcStep), cudaMemcpyHostToDevice, s));
    if (!jobs.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tc_jobs[q], jobs.data(), jobs.size() * sizeof(TcJob), cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(h->tc_cta[q], cta.data(), cta.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));  // the host vectors go out of scope
    h->tc_njobs[q] = nj;
    return HMG_OK;
}

hmg_status alloc_arena(void** p, long long bytes, const char* what)
{
    cudaError_t ce = cudaMalloc(p, (size_t)std::max(bytes, 16ll));
    if (ce != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_error("hmg_build_bf16_factors: allocating %lld bytes for %s failed: %s", bytes, what, cudaGetErrorString(ce));
        return ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
    }
    return HMG_OK;
}

}  // namespace

hmg_status build_bf16_factors(hmg_matrix* h, bool near_tc, int parts)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    free_tc(h);
    if (h->far_prec != HMG_PREC_FP32) {
        set_error("hmg_build_bf16_factors: needs FP32 factors (hmg_precompute_aca with HMG_PREC_FP32)");
        return HMG_ERR_STATE;
    }
    if (h->ndense > 0 && !(h->near_mode == HMG_NEAR_STORED && h->near_prec == HMG_PREC_FP32)) {
        set_error("hmg_build_bf16_factors: needs an FP32 stored near field (hmg_precompute_dense with HMG_PREC_FP32)");
        return HMG_ERR_STATE;
    }
    if (h->group_count) {
        set_error("hmg_build_bf16_factors: not available on a group handle");
        return HMG_ERR_UNSUPPORTED;
    }
    for (int b = h->ndense; b < h->nblocks; b++)
        if (((h->h_rank[b] + 15) & ~15) > TC_MAXR16) {
            set_error("hmg_build_bf16_factors: block %d has rank %d (> %d)", b, h->h_rank[b], TC_MAXR16);
            return HMG_ERR_UNSUPPORTED;
        }
    if ((st = ensure_desc(h, 4))) return st;
    const int np = h->npairs, nt = h->ntiles, nb = h->nblocks, grid = h->nsm;
    std::vector<int> tps(nt + 1), pblock(np), ts(nt), tr0(nt);
    HMG_CUDA_TRY(cudaMemcpy(tps.data(), h->tile_pair_start, sizeof(int) * (nt + 1), cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(pblock.data(), h->pair_block, sizeof(int) * np, cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(ts.data(), h->tile_s, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(tr0.data(), h->tile_r0, sizeof(int) * nt, cudaMemcpyDeviceToHost));

    // B buffer of a product, in K cores: X (8 columns each), then t_b (16 terms = 2 K cores per group)
    const long long xkc = (h->n[1] + 7) / 8 + 4;
    // Split operands: the parts of a K core lie together (A: parts * rc row cores per K
    // core, B: parts * NV * 16 bytes per K core), so a chunk of K cores brings every part;
    // 1 / parts of the K cores and MMAs per step
    const long long a_half = TC_ABYTES / parts;
    const int ks_limit = TC_MAXSTEP / parts;
    std::vector<long long> toff(nb, -1);
    long long tgroups = 0;
    JobList k1, k2;
    // pass 1 jobs: stacks of the V^T of blocks with the same columns (one X chunk, one
    // MMA sequence for all of them), at most 128 terms, largest ranks first
    std::vector<int> vlist, vaux, kmap;
    std::vector<long long> voff;
    long long vbytes = 0;
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
            std::vector<std::vector<int>> stacks;
            std::vector<int> fill;
            for (size_t i = g0; i < g1; i++) {  // first fit, ranks decreasing
                const int b = far[i], r16 = (h->h_rank[b] + 15) & ~15;
                size_t k = 0;
                while (k < stacks.size() && fill[k] + r16 > 128) k++;
                if (k == stacks.size()) {
                    stacks.emplace_back();
                    fill.push_back(0);
                }
                stacks[k].push_back(b);
                fill[k] += r16;
            }
            const int c0 = h->h_c0[far[g0]], kw = ((c0 & 7) + h->h_m2[far[g0]] + 15) & ~15;
            for (size_t k = 0; k < stacks.size(); k++) {
                const int rows = fill[k], rc = rows / 8, job = (int)(kmap.size() / 16);
                kmap.resize(kmap.size() + 16, 0);
                int off8 = 0;
                for (int b : stacks[k]) {
                    const int r16 = (h->h_rank[b] + 15) & ~15;
                    toff[b] = tgroups;
                    for (int kc = 0; kc < r16 / 8; kc++) kmap[job * 16 + off8 + kc] = (int)(tgroups * 2 + kc);
                    tgroups += r16 / 16;
                    vlist.push_back(b);
                    voff.push_back(vbytes);
                    vaux.push_back(rc << 8 | off8);
                    off8 += r16 / 8;
                }
                k1.begin(TcJob{job, rows});
                k1.add(vbytes, c0 >> 3, rc * parts, kw / 8, std::min(2 * ks_limit, (int)(a_half / 128 / rc) & ~1),
                       0.25 * parts);
                vbytes += (long long)rows * kw * 2 * parts;
            }
            g0 = g1;
        }
    }
    // pass 2: per tile, its low-rank pairs (B = t_b) and near pairs (B = X)
    std::vector<int> ulist, nlist, utile, ntile;
    std::vector<long long> uoff, noff;
    long long ubytes = 0;
    bool all_tiles = true;
    for (int t = 0; t < nt; t++) {
        const int rc = ((ts[t] + 7) & ~7) / 8;
        bool started = false;
        for (int p = tps[t]; p < tps[t + 1]; p++) {
            const int b = pblock[p];
            const bool dense = b < h->ndense;
            if ((!dense && h->h_rank[b] == 0) || (dense && !near_tc)) continue;
            if (!started) {
                k2.begin(TcJob{tr0[t], ts[t]});
                started = true;
            }
            if (dense) {
                const int a = h->h_c0[b] & 7, kw = (a + h->h_m2[b] + 15) & ~15;
                nlist.push_back(p);
                ntile.push_back(t);
                noff.push_back(ubytes);
                k2.add(ubytes, h->h_c0[b] >> 3, rc * parts, kw / 8, (int)(a_half / 128 / 16), 0.25 * parts);
                ubytes += (long long)rc * 8 * kw * 2 * parts;
            } else {
                const int r16 = (h->h_rank[b] + 15) & ~15;
                ulist.push_back(p);
                utile.push_back(t);
                uoff.push_back(ubytes);
                k2.add(ubytes, xkc + toff[b] * 2, rc * parts, r16 / 8, (int)(a_half / 128 / 16), 1.0 * parts);
                ubytes += (long long)rc * 8 * r16 * 2 * parts;
            }
        }
        all_tiles = all_tiles && started;
    }

    k1.make_steps(false, TC_ABYTES, ks_limit);
    k2.make_steps(true, TC_ABYTES, ks_limit);
    if (!steps_in_bounds(k1, vbytes, xkc + tgroups * 2, (long long)kmap.size() / 16, 0, parts) ||
        !steps_in_bounds(k2, ubytes, xkc + tgroups * 2, h->n[0], 1, parts)) {
        set_error("hmg_build_bf16_factors: internal error: an operand step leaves its buffer");
        return HMG_ERR_UNSUPPORTED;
    }
    for (int v : kmap)
        if (v < 0 || v >= tgroups * 2) {
            set_error("hmg_build_bf16_factors: internal error: a t_b core lies outside its buffer");
            return HMG_ERR_UNSUPPORTED;
        }
    if ((st = alloc_arena(&h->tc_u, ubytes, "the tile operands"))) return st;
    if ((st = dalloc(&h->tc_kmap, std::max(kmap.size(), (size_t)1), s))) {
        free_tc(h);
        return st;
    }
    if (!kmap.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tc_kmap, kmap.data(), sizeof(int) * kmap.size(), cudaMemcpyHostToDevice, s));
    if ((st = alloc_arena(&h->tc_v, vbytes, "the V^T operands"))) {
        free_tc(h);
        return st;
    }
    int* dlist = nullptr;
    int* dtile = nullptr;
    long long* doff = nullptr;
    auto convert = [&](const std::vector<int>& list, const std::vector<int>& tiles, const std::vector<long long>& off,
                       int which) -> hmg_status {
        const int n = (int)list.size();
        if (n == 0) return HMG_OK;
        hmg_status e;
        if ((e = dalloc(&dlist, (size_t)n, s)) || (e = dalloc(&doff, (size_t)n, s)) ||
            (!tiles.empty() && (e = dalloc(&dtile, (size_t)n, s))))
            return e;
        HMG_CUDA_TRY(cudaMemcpyAsync(dlist, list.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(doff, off.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, s));
        if (!tiles.empty())
            HMG_CUDA_TRY(cudaMemcpyAsync(dtile, tiles.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
        const PairDesc* desc = static_cast<const PairDesc*>(h->pair_desc);
        __nv_bfloat16* up = static_cast<__nv_bfloat16*>(h->tc_u);
        __nv_bfloat16* vp = static_cast<__nv_bfloat16*>(h->tc_v);
        if (which == 0)
            k_tc_u<<<n, 256, 0, s>>>(desc, dlist, doff, dtile, h->tile_s, n, up, parts);
        else if (which == 1)
            k_tc_near<<<n, 256, 0, s>>>(desc, dlist, doff, dtile, h->tile_s, n, up, parts);
        else
            k_tc_v<<<n, 256, 0, s>>>(dlist, doff, dtile, n, h->ptrV, h->rank, h->blk_c0, h->blk_m2, vp, parts);
        HMG_LAUNCH_CHECK();
        HMG_CUDA_TRY(cudaStreamSynchronize(s));
        dfree(dlist, s);
        dfree(doff, s);
        dfree(dtile, s);
        dlist = dtile = nullptr;
        doff = nullptr;
        return HMG_OK;
    };
    if ((st = convert(ulist, utile, uoff, 0)) || (st = convert(nlist, ntile, noff, 1)) ||
        (st = convert(vlist, vaux, voff, 2)) || (st = upload_jobs(h, 0, k1, 1024.0, grid)) ||
        (st = upload_jobs(h, 1, k2, 4096.0, grid))) {
        dfree(dlist, s);
        dfree(doff, s);
        dfree(dtile, s);
        free_tc(h);
        return st;
    }
    h->tc_bytes = (ubytes + vbytes) / parts;
    h->tc_xkc = xkc;
    h->tc_tkc = tgroups * 2;
    h->tc_grid = grid;
    h->tc_all_tiles = all_tiles;
    h->tc_near = near_tc;
    h->tc_parts = parts;
    h->tc_ready = true;
    return HMG_OK;
}

template <int NV, int PARTS>
static hmg_status tc_product(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    char* bbuf = static_cast<char*>(h->tc_bbuf);
    const long long xkc = h->tc_xkc;
    k_tc_x<NV><<<(unsigned)((xkc * NV + 255) / 256), 256, 0, s>>>(X, ldx, nrhs, h->perm[1], h->n[1], xkc,
                                                                    reinterpret_cast<uint4*>(bbuf), PARTS);
    HMG_LAUNCH_CHECK();
    const size_t smem = sizeof(TcSmem);
    HMG_CUDA_TRY(cudaFuncSetAttribute(k_tc_pass<0, NV, PARTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HMG_CUDA_TRY(cudaFuncSetAttribute(k_tc_pass<1, NV, PARTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (h->tc_njobs[0] > 0) {
        k_tc_pass<0, NV, PARTS><<<h->tc_grid, TC_THREADS, smem, s>>>(
            reinterpret_cast<const TcStep*>(h->tc_steps[0]), reinterpret_cast<const TcJob*>(h->tc_jobs[0]),
            reinterpret_cast<const int2*>(h->tc_cta[0]), static_cast<const char*>(h->tc_v), bbuf, xkc, h->tc_kmap, 0,
            nullptr, 0, 0, h->dev_err);
        HMG_LAUNCH_CHECK();
    }
    if (!h->tc_near && h->ndense > 0) {
        // the near field in FP32 on the CUDA cores writes every row of Y first (32 vectors a pass)
        float* xm = nullptr;
        if ((st = dalloc(&xm, (size_t)h->n[1] * 32, s))) return st;
        for (int j0 = 0; j0 < nrhs && !st; j0 += 32) {
            launch_gather_multi32(h, X + (size_t)j0 * ldx, ldx, std::min(32, nrhs - j0), xm);
            st = launch_tile_multi32_dense(h, xm, std::min(32, nrhs - j0), Y + (size_t)j0 * ldy, ldy);
        }
        dfree(xm, s);
        if (st) return st;
    } else if (!h->tc_all_tiles) {
        // rows of tiles without products (all their blocks of rank 0) are zero
        HMG_CUDA_TRY(cudaMemset2DAsync(Y, sizeof(double) * ldy, 0, sizeof(double) * h->n[0], nrhs, s));
    }
    const int add_y = !h->tc_near && h->ndense > 0;
    if (h->tc_njobs[1] > 0) {
        k_tc_pass<1, NV, PARTS><<<h->tc_grid, TC_THREADS, smem, s>>>(
            reinterpret_cast<const TcStep*>(h->tc_steps[1]), reinterpret_cast<const TcJob*>(h->tc_jobs[1]),
            reinterpret_cast<const int2*>(h->tc_cta[1]), static_cast<const char*>(h->tc_u), bbuf, 0, h->perm[0], nrhs, Y,
            ldy, add_y, h->dev_err);
        HMG_LAUNCH_CHECK();
    }
    return HMG_OK;
}

template <int PARTS>
static hmg_status tc_product_parts(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    return nrhs > 32 ? tc_product<64, PARTS>(h, nrhs, X, ldx, Y, ldy) : tc_product<32, PARTS>(h, nrhs, X, ldx, Y, ldy);
}

// up to 64 vectors in one pass: MMAs of N = 32 for 2..32 vectors, N = 64 for 33..64
hmg_status matvec_multi_tc(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    // X and t_b cores (every part), kept with the handle, sized for 64 vectors
    if (!h->tc_bbuf) {
        const size_t bytes = (size_t)(h->tc_xkc + h->tc_tkc) * 16 * TC_NMAX * h->tc_parts;
        cudaError_t ce = cudaMalloc(&h->tc_bbuf, bytes);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            h->tc_bbuf = nullptr;
            set_error("hmg_matvec_multi: allocating %zu bytes of operand space failed: %s", bytes, cudaGetErrorString(ce));
            return ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
        }
    }
    if (h->tc_parts == 3) return tc_product_parts<3>(h, nrhs, X, ldx, Y, ldy);
    if (h->tc_parts == 2) return tc_product_parts<2>(h, nrhs, X, ldx, Y, ldy);
    return tc_product_parts<1>(h, nrhs, X, ldx, Y, ldy);
}

}  // namespace hmg
