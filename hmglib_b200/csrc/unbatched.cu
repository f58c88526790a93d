// unbatched.cu -- the H-matvec one block at a time (hmg_matvec_unbatched).
//
// Replaces sequential_h_matrix_mvp_without_batching (linear_algebra.cu:4384-4443):
// y is cleared, then every dense block (in work-list order) and after them every
// admissible block is applied by its own kernel launch on the handle's stream.
//   * dense block: entries generated from the points in FP64 and multiplied at once
//     (the reference fills the block and calls cublasDgemv per block,
//     apply_dense_matrix_for_current_work_item);
//   * admissible block: t = V_b^T x, then y += U_b t, in FP64 arithmetic over the
//     stored factors (the reference recomputes the block's ACA in every call,
//     apply_aca_for_current_work_item; here the factors of hmg_precompute_aca are
//     read, so the result is the same operator as the batched product).
// It shares nothing with the batched product kernels but the storage layout: no
// descriptors, no row tiles of the product, no x gather, no per-tile reduction.
// Launches follow one another on one stream and each output row is written by one
// thread per launch, so the result is deterministic.  It is a checking path: one
// launch per block (1.66 million at N = 2^20) makes it launch-bound.
#include <algorithm>

#include "hmg_matrix.cuh"

namespace hmg {

static constexpr int UB_THREADS = 256;

__global__ void k_ub_clear(double* y, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = 0.0;
}

// y[perm1[r0 + i]] += sum_j K(r0 + i, c0 + j) x[perm2[c0 + j]]
__global__ void __launch_bounds__(UB_THREADS) k_ub_dense(int r0, int m1, int c0, int m2, KernelSpec K,
                                                          PointsView P, const int* perm1, const int* perm2,
                                                          const double* x, double* y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m1; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < m2; j++) acc = fma(kernel_entry(K, P, r0 + i, c0 + j), x[perm2[c0 + j]], acc);
        y[perm1[r0 + i]] += acc;
    }
}

// One CTA: t = V^T x (one warp per term), then y += U t over the block's tile
// slices (U slice of tile t: s_pad x r column-major at (pstart[t] - pstart[tf]) r).
template <typename T>
__global__ void __launch_bounds__(UB_THREADS) k_ub_lowrank(int r0, int c0, int m2, int r, const T* U, const T* V,
                                                            int tf, int tl, const int* tile_r0, const int* tile_s,
                                                            const int* tile_pstart, const int* perm1,
                                                            const int* perm2, const double* x, double* y)
{
    extern __shared__ double t[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int m2p = (m2 + 3) & ~3;
    for (int l = warp; l < r; l += nw) {
        double acc = 0.0;
        for (int j = lane; j < m2; j += 32) acc = fma((double)V[(size_t)l * m2p + j], x[perm2[c0 + j]], acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) t[l] = acc;
    }
    __syncthreads();
    const int p0 = tile_pstart[tf];
    for (int tt = tf; tt <= tl; tt++) {
        const int s = tile_s[tt], sp = (s + 3) & ~3;
        const T* base = U + (size_t)(tile_pstart[tt] - p0) * r;
        for (int i = threadIdx.x; i < s; i += blockDim.x) {
            double acc = 0.0;
            for (int l = 0; l < r; l++) acc = fma((double)base[(size_t)l * sp + i], t[l], acc);
            y[perm1[tile_r0[tt] + i]] += acc;
        }
    }
    (void)r0;
}

hmg_status matvec_unbatched(hmg_matrix* h, const double* x, double* y)
{
    if (h->group_count) {
        set_error("hmg_matvec_unbatched: not available on a group handle");
        return HMG_ERR_UNSUPPORTED;
    }
    if (h->naca > 0 && h->far_prec != HMG_PREC_FP64 && h->far_prec != HMG_PREC_FP32) {
        set_error("hmg_matvec_unbatched: needs FP64 or FP32 factors (hmg_precompute_aca)");
        return h->far_prec < 0 ? HMG_ERR_STATE : HMG_ERR_UNSUPPORTED;
    }
    cudaStream_t s = h->stream;
    PointsView P{};
    for (int d = 0; d < h->dim; d++) {
        P.c1[d] = h->zpts[0] + (size_t)d * h->n[0];
        P.c2[d] = h->zpts[1] + (size_t)d * h->n[1];
    }
    P.n1 = h->n[0];
    P.n2 = h->n[1];
    const int gclear = std::min(ceil_div(h->n[0], UB_THREADS), 1184);
    k_ub_clear<<<gclear, UB_THREADS, 0, s>>>(y, h->n[0]);
    HMG_LAUNCH_CHECK();
    for (int b = 0; b < h->ndense; b++) {
        const int m1 = h->h_m1[b];
        k_ub_dense<<<ceil_div(m1, UB_THREADS), UB_THREADS, 0, s>>>(h->h_r0[b], m1, h->h_c0[b], h->h_m2[b], h->kspec,
                                                                   P, h->perm[0], h->perm[1], x, y);
        HMG_LAUNCH_CHECK();
    }
    if (h->naca == 0) return HMG_OK;
    std::vector<void*> pu(h->nblocks), pv(h->nblocks);
    HMG_CUDA_TRY(cudaMemcpyAsync(pu.data(), h->ptrU, sizeof(void*) * h->nblocks, cudaMemcpyDeviceToHost, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(pv.data(), h->ptrV, sizeof(void*) * h->nblocks, cudaMemcpyDeviceToHost, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    for (int b = h->ndense; b < h->nblocks; b++) {
        const int r = h->h_rank[b];
        if (r == 0) continue;
        const size_t smem = sizeof(double) * (size_t)r;
        if (h->far_prec == HMG_PREC_FP64)
            k_ub_lowrank<double><<<1, UB_THREADS, smem, s>>>(
                h->h_r0[b], h->h_c0[b], h->h_m2[b], r, (const double*)pu[b], (const double*)pv[b],
                h->h_blk_tfirst[b], h->h_blk_tlast[b], h->tile_r0, h->tile_s, h->tile_pstart, h->perm[0],
                h->perm[1], x, y);
        else
            k_ub_lowrank<float><<<1, UB_THREADS, smem, s>>>(
                h->h_r0[b], h->h_c0[b], h->h_m2[b], r, (const float*)pu[b], (const float*)pv[b],
                h->h_blk_tfirst[b], h->h_blk_tlast[b], h->tile_r0, h->tile_s, h->tile_pstart, h->perm[0],
                h->perm[1], x, y);
        HMG_LAUNCH_CHECK();
    }
    return HMG_OK;
}

}  // namespace hmg
