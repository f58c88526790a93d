// tc.cu -- multi-vector products on the tensor cores (tcgen05), BF16 factors.
//
// hmg_build_bf16_factors converts the FP32 low-rank factors of a handle into a BF16
// copy laid out as tcgen05 operands; hmg_matvec_multi then multiplies 2..32 vectors
// per pass with it.  Per row tile (M = 128 rows) and admissible block of rank r the
// far-field product is D += U_slice (128 x r16, BF16) * T_b (r16 x 32, BF16) with
// r16 = r rounded up to 16, accumulated in FP32 in tensor memory across all of the
// tile's low-rank pairs (operands copied two stages deep with cp.async, so one pair's
// copy overlaps the previous pair's MMAs) and added to Y, which the CUDA-core
// multi-vector tile kernel has filled with the dense pairs' FP32 sums just before.  t_b = V_b^T X_b comes from the multi-vector K1 on the
// CUDA cores in FP32 and is rounded to BF16 for the MMA (the factors' own BF16 rounding, ~4e-3 per entry, dominates the
// error: products agree with FP32 factors to ~1e-3).
//
// Operand layout (no swizzle, K-major "core matrices" of 8 rows x 16 bytes):
//   U slice of a (tile, block) pair: core (mc, kc) = rows 8mc..8mc+7, terms 8kc..8kc+7,
//   stored core-by-core with mc fastest: ((kc * (s8 / 8)) + mc) * 128 bytes, s8 = tile
//   rows rounded to 8.  In shared memory the same cores sit at (kc * 16 + mc) * 128
//   bytes (16 row cores for M = 128; the rows past s8 stay zero).
//   T_b: core (nc, kc) = vectors 8nc..8nc+7, terms 8kc..8kc+7 at (kc * 4 + nc) * 128.
// Descriptors: leading byte offset = stride between K cores, stride byte offset =
// stride between row cores; instruction kind::f16 with BF16 A/B, FP32 D, M 128, N 32.
// Every wait on the MMA's mbarrier is bounded; on a time-out the kernel records an
// error flag (read by the host), skips the remaining work and frees its tensor memory.
#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "hmg_matrix.cuh"
#include "stream.cuh"

namespace hmg {

static constexpr int TC_N = 32;           // vectors per pass (MMA N)
static constexpr int TC_MAXR16 = 96;      // largest rank (rounded to 16) with room in shared memory
static constexpr long long TC_SPIN = 1ll << 26;

// ---------------------------------------------------------------------------
// conversion of the FP32 factors
// ---------------------------------------------------------------------------
// one CTA per pair: FP32 slice (s_pad x r, column-major) -> BF16 cores
__global__ void k_tc_u(const PairDesc* desc, const int* pair_tile, const long long* uoff, const int* tile_s,
                       int npairs, __nv_bfloat16* out)
{
    const int p = blockIdx.x;
    if (p >= npairs || uoff[p] < 0) return;
    const PairDesc d = desc[p];
    const int s = tile_s[pair_tile[p]], sp = (s + 3) & ~3, s8 = (s + 7) & ~7;
    const int r = d.ncol, r16 = (r + 15) & ~15;
    const float* src = static_cast<const float*>(d.data);
    __nv_bfloat16* dst = out + uoff[p] / 2;
    const int mcores = s8 / 8;
    for (int idx = threadIdx.x; idx < s8 * r16; idx += blockDim.x) {
        const int core = idx >> 6, e = idx & 63;
        const int kc = core / mcores, mc = core - kc * mcores;
        const int i = mc * 8 + (e >> 3), k = kc * 8 + (e & 7);
        const float v = (i < s && k < r) ? src[(size_t)k * sp + i] : 0.0f;
        dst[idx] = __float2bfloat16_rn(v);
    }
}

// ---------------------------------------------------------------------------
// t_b (FP32, [term][32] from the multi-vector K1) -> BF16 operand cores; terms
// r..r16-1 are zero
// ---------------------------------------------------------------------------
__global__ void k_tc_t(const int* far_blocks, int nfar, const int* rank, const long long* rank_off,
                       const long long* toff, const float* __restrict__ tm, __nv_bfloat16* tb)
{
    const int u = blockIdx.x;
    if (u >= nfar) return;
    const int b = far_blocks[u];
    const int r = rank[b], r16 = (r + 15) & ~15;
    const float* src = tm + (size_t)rank_off[b] * TC_N;
    __nv_bfloat16* out = tb + toff[b] * (16 * TC_N);
    for (int idx = threadIdx.x; idx < r16 * TC_N; idx += blockDim.x) {
        const int core = idx >> 6, e = idx & 63;
        const int kc = core >> 2, nc = core & 3;
        const int n = nc * 8 + (e >> 3), k = kc * 8 + (e & 7);
        out[idx] = __float2bfloat16_rn(k < r ? src[(size_t)k * TC_N + n] : 0.0f);
    }
}

// ---------------------------------------------------------------------------
// the tile kernel
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100; base offset 0, no swizzle
    return d;
}

// kind::f16, D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28
static constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                                     ((uint32_t)(128 >> 4) << 24);

struct TcSmem {
    __nv_bfloat16 A[2][TC_MAXR16 / 8][16][64];    // 2 stages x K cores x row cores x 8 rows x 8 terms
    __nv_bfloat16 B[2][TC_MAXR16 / 8][4][64];     // 2 stages x K cores x vector cores x 8 x 8
    unsigned long long mbar[2];
    uint32_t tmem;
    int fail;
};

__device__ __forceinline__ void tc_cp16(void* dst, const void* src)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t phase)
{
    uint32_t ok = 0;
    for (long long it = 0; it < TC_SPIN && !ok; it++)
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(mbar), "r"(phase)
            : "memory");
    return ok != 0;
}

// one CTA (4 warps) per row tile; the low-rank pairs' operands are copied two stages
// deep (cp.async), so the copy of one pair overlaps the MMAs of the previous one
__global__ void __launch_bounds__(128) k_tile_tc(const PairDesc* __restrict__ desc, const int* pair_block,
                                                 const long long* __restrict__ uoff, const char* __restrict__ tcu,
                                                 const __nv_bfloat16* __restrict__ tb, const long long* toff,
                                                 const int* tile_pair_start, const int* tile_r0, const int* tile_s,
                                                 const int* perm1, const float* __restrict__ xm, int nrhs, double* Y,
                                                 int ldy, int* err)
{
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem& sm = *reinterpret_cast<TcSmem*>(tc_raw);
    const int t = blockIdx.x, tid = threadIdx.x, warp = tid >> 5;
    const int s = tile_s[t], sp = (s + 3) & ~3, s8 = (s + 7) & ~7, tr0 = tile_r0[t];
    const int pbeg = tile_pair_start[t], pend = tile_pair_start[t + 1];
    const uint32_t mbar0 = static_cast<uint32_t>(__cvta_generic_to_shared(&sm.mbar[0]));
    const int mcores = s8 / 8;

    for (int i = tid; i < (int)(sizeof(sm.A) / 16); i += 128) reinterpret_cast<uint4*>(&sm.A[0][0][0][0])[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        sm.fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar0));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar0 + 8));
    }
    if (warp == 0) {
        const uint32_t slot = static_cast<uint32_t>(__cvta_generic_to_shared(&sm.tmem));
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(slot));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = sm.tmem;

    // the dense pairs ran before this kernel (CUDA cores, FP32); Y holds their sums
    float acc[TC_N];
#pragma unroll
    for (int j = 0; j < TC_N; j++) acc[j] = 0.0f;

    // low-rank pairs on the tensor cores
    auto next_far = [&](int p) {
        while (p < pend) {
            const PairDesc& d = desc[p];
            if (d.kind == PAIR_FAR && d.ncol > 0 && uoff[p] >= 0) break;
            p++;
        }
        return p;
    };
    auto copy = [&](int p, int b) {
        const int r16 = (desc[p].ncol + 15) & ~15, kcores = r16 / 8;
        const char* su = tcu + uoff[p];
        for (int i = tid; i < kcores * mcores * 8; i += 128) {
            const int core = i >> 3, part = i & 7;
            const int kc = core / mcores, mc = core - kc * mcores;
            tc_cp16(reinterpret_cast<uint4*>(&sm.A[b][kc][mc][0]) + part, su + (size_t)i * 16);
        }
        const char* st = reinterpret_cast<const char*>(tb + toff[pair_block[p]] * (16 * TC_N));
        for (int i = tid; i < kcores * 4 * 8; i += 128)
            tc_cp16(reinterpret_cast<uint4*>(&sm.B[b][0][0][0]) + i, st + (size_t)i * 16);
    };
    uint32_t phase[2] = {0u, 0u};
    bool busy[2] = {false, false};
    bool any = false;
    int cur = next_far(pbeg), b = 0;
    if (cur < pend) copy(cur, 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
    while (cur < pend) {
        const int nxt = next_far(cur + 1);
        if (nxt < pend) {
            if (busy[b ^ 1]) {  // the MMAs that read buffer b^1 must be done before it is refilled
                if (!tc_wait(mbar0 + 8 * (b ^ 1), phase[b ^ 1])) sm.fail = 1;
                phase[b ^ 1] ^= 1u;
                busy[b ^ 1] = false;
            }
            copy(nxt, b ^ 1);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (sm.fail) break;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int r16 = (desc[cur].ncol + 15) & ~15;
            const uint32_t a_base = static_cast<uint32_t>(__cvta_generic_to_shared(&sm.A[b][0][0][0]));
            const uint32_t b_base = static_cast<uint32_t>(__cvta_generic_to_shared(&sm.B[b][0][0][0]));
            for (int q = 0; q < r16 / 16; q++) {
                const uint64_t ad = smem_desc(a_base + q * 2 * (16 * 128), 16 * 128, 128);
                const uint64_t bd = smem_desc(b_base + q * 2 * (4 * 128), 4 * 128, 128);
                const uint32_t accumulate = (any || q > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred pd;\n setp.ne.b32 pd, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, pd;\n}" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar0 + 8 * b)
                         : "memory");
        }
        busy[b] = true;
        any = true;
        cur = nxt;
        b ^= 1;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    for (int q = 0; q < 2; q++)
        if (busy[q]) {
            if (!tc_wait(mbar0 + 8 * q, phase[q])) sm.fail = 1;
            busy[q] = false;
        }
    if (sm.fail && tid == 0) atomicExch(err, 1);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (any && !sm.fail) {
        uint32_t v[32];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
            "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
              "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
              "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
              "=r"(v[30]), "=r"(v[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < TC_N; j++) acc[j] += __uint_as_float(v[j]);
    }
    if (any && tid < s && !sm.fail) {
        const size_t row = (size_t)perm1[tr0 + tid];
#pragma unroll
        for (int j = 0; j < TC_N; j++)
            if (j < nrhs) Y[row + (size_t)j * ldy] += (double)acc[j];
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem));
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
void free_tc(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    if (h->tc_u) cudaFree(h->tc_u);
    h->tc_u = nullptr;
    dfree(h->tc_uoff, s);
    dfree(h->tc_toff, s);
    dfree(h->tc_pair_tile, s);
    dfree(h->tc_far_blocks, s);
    h->tc_ready = false;
    h->tc_bytes = 0;
    h->tc_tgroups = 0;
    h->tc_nfar = 0;
}

hmg_status build_bf16_factors(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    free_tc(h);
    if (h->far_prec != HMG_PREC_FP32) {
        set_error("hmg_build_bf16_factors: needs FP32 factors (hmg_precompute_aca with HMG_PREC_FP32)");
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
    const int np = h->npairs, nt = h->ntiles, nb = h->nblocks;
    std::vector<int> tps(nt + 1), pblock(np), ts(nt);
    HMG_CUDA_TRY(cudaMemcpy(tps.data(), h->tile_pair_start, sizeof(int) * (nt + 1), cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(pblock.data(), h->pair_block, sizeof(int) * np, cudaMemcpyDeviceToHost));
    HMG_CUDA_TRY(cudaMemcpy(ts.data(), h->tile_s, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    std::vector<long long> uoff(np, -1), toff(nb, 0);
    std::vector<int> ptile(np), farb;
    long long bytes = 0;
    for (int t = 0; t < nt; t++)
        for (int p = tps[t]; p < tps[t + 1]; p++) {
            ptile[p] = t;
            const int b = pblock[p];
            if (b < h->ndense || h->h_rank[b] == 0) continue;
            uoff[p] = bytes;
            bytes += (long long)((ts[t] + 7) & ~7) * ((h->h_rank[b] + 15) & ~15) * 2;
            bytes = (bytes + 15) & ~15ll;
        }
    long long groups = 0;
    for (int b = h->ndense; b < nb; b++) {
        if (h->h_rank[b] == 0) continue;
        toff[b] = groups;
        groups += (h->h_rank[b] + 15) / 16;
        farb.push_back(b);
    }
    cudaError_t ce = cudaMalloc(&h->tc_u, (size_t)std::max(bytes, 16ll));
    if (ce != cudaSuccess) {
        cudaGetLastError();
        h->tc_u = nullptr;
        set_error("hmg_build_bf16_factors: allocating %lld bytes failed: %s", bytes, cudaGetErrorString(ce));
        return ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
    }
    if ((st = dalloc(&h->tc_uoff, (size_t)std::max(np, 1), s)) || (st = dalloc(&h->tc_toff, (size_t)std::max(nb, 1), s)) ||
        (st = dalloc(&h->tc_pair_tile, (size_t)std::max(np, 1), s)) ||
        (st = dalloc(&h->tc_far_blocks, std::max(farb.size(), (size_t)1), s)))
        return st;
    if (np > 0) {
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tc_uoff, uoff.data(), sizeof(long long) * np, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tc_pair_tile, ptile.data(), sizeof(int) * np, cudaMemcpyHostToDevice, s));
    }
    HMG_CUDA_TRY(cudaMemcpyAsync(h->tc_toff, toff.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, s));
    if (!farb.empty())
        HMG_CUDA_TRY(cudaMemcpyAsync(h->tc_far_blocks, farb.data(), sizeof(int) * farb.size(), cudaMemcpyHostToDevice, s));
    if (np > 0) {
        k_tc_u<<<np, 256, 0, s>>>(static_cast<const PairDesc*>(h->pair_desc), h->tc_pair_tile, h->tc_uoff, h->tile_s,
                                  np, static_cast<__nv_bfloat16*>(h->tc_u));
        HMG_LAUNCH_CHECK();
    }
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    h->tc_bytes = bytes;
    h->tc_tgroups = groups;
    h->tc_nfar = (int)farb.size();
    h->tc_ready = true;
    return HMG_OK;
}

hmg_status matvec_multi_tc(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    if ((st = ensure_desc(h, 4))) return st;
    float* xm = nullptr;
    __nv_bfloat16* tb = nullptr;
    if ((st = dalloc(&xm, (size_t)h->n[1] * TC_N, s)) ||
        (st = dalloc(&tb, (size_t)std::max(h->tc_tgroups, 1ll) * 16 * TC_N, s))) {
        dfree(xm, s);
        return st;
    }
    launch_gather_multi32(h, X, ldx, nrhs, xm);
    if (h->tc_nfar > 0) {
        float* tm = nullptr;
        if ((st = dalloc(&tm, (size_t)(h->rank_total + 1) * TC_N, s))) {
            dfree(xm, s);
            dfree(tb, s);
            return st;
        }
        st = launch_vtx_multi32(h, xm, tm);
        if (!st) {
            k_tc_t<<<h->tc_nfar, 256, 0, s>>>(h->tc_far_blocks, h->tc_nfar, h->rank, h->rank_off, h->tc_toff, tm, tb);
            if (cudaGetLastError() != cudaSuccess) st = HMG_ERR_CUDA;
        }
        dfree(tm, s);
        if (st) {
            dfree(xm, s);
            dfree(tb, s);
            return st;
        }
    }
    if ((st = launch_tile_multi32_dense(h, xm, nrhs, Y, ldy))) {
        dfree(xm, s);
        dfree(tb, s);
        return st;
    }
    if (h->ntiles > 0 && h->tc_nfar > 0) {
        HMG_CUDA_TRY(cudaFuncSetAttribute(k_tile_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem)));
        k_tile_tc<<<h->ntiles, 128, sizeof(TcSmem), s>>>(static_cast<const PairDesc*>(h->pair_desc), h->pair_block, h->tc_uoff,
                                           static_cast<const char*>(h->tc_u), tb, h->tc_toff, h->tile_pair_start,
                                           h->tile_r0, h->tile_s, h->perm[0], xm, nrhs, Y, ldy, h->dev_err);
        HMG_LAUNCH_CHECK();
    }
    dfree(xm, s);
    dfree(tb, s);
    return HMG_OK;
}

}  // namespace hmg
