// group.cu -- many independent H-matrices multiplied as one (hmg_group_create).
//
// The reference handles one H-matrix per call, each with its own MAGMA setup
// (hmglib.cu:119): a caller with hundreds of small point sets pays the per-call
// launches and synchronisations hundreds of times.  A group is the block-diagonal
// union of set-up handles: the points of set i occupy rows [off1_i, off1_i + n1_i)
// and columns [off2_i, off2_i + n2_i), every block of set i is shifted by those
// offsets, and each block carries its set's kernel parameter.  Compression
// (hmg_precompute_aca), the near field and every product then run over all sets in
// the same launches; x and y are the concatenations of the sets' vectors in set
// order.  Each set's tree is its own (bit-identical to the set alone), and so is each
// set's result: a tile never mixes sets and the pairs of a tile keep their order.
#include <algorithm>
#include <vector>

#include "hmg_matrix.cuh"

namespace hmg {

// out[d][off + i] = in[d][i] for d < din, 0 for din <= d < dout
__global__ void k_copy_points(const double* in, int n, int din, double* out, int nout, int off, int dout)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int d = 0; d < dout; d++) out[(size_t)d * nout + off + i] = d < din ? in[(size_t)d * n + i] : 0.0;
}

__global__ void k_offset_copy(const int* in, int n, int add, int* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i] + add;
}

hmg_status group_create(hmg_matrix** out, hmg_matrix* const* sets, int count, cudaStream_t s)
{
    hmg_status st;
    int n1 = 0, n2 = 0, dim = 2, bits = 0, levels = 0;
    long long nb = 0, nd = 0;
    const hmg_matrix* s0 = sets[0];
    for (int i = 0; i < count; i++) {
        const hmg_matrix* h = sets[i];
        if (!h || !h->setup_done || !h->kernel_set) {
            set_error("hmg_group_create: set %d is not set up with a kernel", i);
            return HMG_ERR_STATE;
        }
        if (h->group_count) {
            set_error("hmg_group_create: set %d is itself a group", i);
            return HMG_ERR_INVALID;
        }
        // (the reference Matern kernel's normalisation depends on the dimension)
        if (h->kspec.kind != s0->kspec.kind || h->kspec.reg != s0->kspec.reg ||
            (h->kspec.kind == HMG_KERNEL_MATERN_REF && h->kspec.matern_ref_denom != s0->kspec.matern_ref_denom)) {
            set_error("hmg_group_create: set %d has another kernel kind or regularization than set 0", i);
            return HMG_ERR_INVALID;
        }
        if ((long long)n1 + h->n[0] > 0x7fffffff || (long long)n2 + h->n[1] > 0x7fffffff) {
            set_error("hmg_group_create: more than 2^31 - 1 points in the group");
            return HMG_ERR_INVALID;
        }
        n1 += h->n[0];
        n2 += h->n[1];
        dim = std::max(dim, h->dim);
        bits = std::max(bits, h->bits);
        levels = std::max(levels, h->levels);
        nb += h->nblocks;
        nd += h->ndense;
    }
    if (nb > 0x7fffffff) {
        set_error("hmg_group_create: more than 2^31 - 1 blocks in the group");
        return HMG_ERR_INVALID;
    }
    hmg_matrix* g = nullptr;
    if ((st = hmg_create(&g, n1, n2, dim, dim == 2 ? 32 : 20, (void*)s))) return st;
    g->group_count = count;
    g->group_off[0].assign(1, 0);
    g->group_off[1].assign(1, 0);
    // points (SoA, a 2D set padded with zero third coordinates), permutations
    for (int i = 0; i < count; i++) {
        const hmg_matrix* h = sets[i];
        for (int w = 0; w < 2; w++) {
            const int off = g->group_off[w].back(), n = h->n[w];
            const int gn = g->n[w];
            if (n > 0) {
                k_copy_points<<<ceil_div(n, 256), 256, 0, s>>>(h->pts[w], n, h->dim, g->pts[w], gn, off, dim);
                k_copy_points<<<ceil_div(n, 256), 256, 0, s>>>(h->zpts[w], n, h->dim, g->zpts[w], gn, off, dim);
                k_offset_copy<<<ceil_div(n, 256), 256, 0, s>>>(h->perm[w], n, off, g->perm[w] + off);
                k_offset_copy<<<ceil_div(n, 256), 256, 0, s>>>(h->iperm[w], n, off, g->iperm[w] + off);
                HMG_LAUNCH_CHECK();
            }
            g->group_off[w].push_back(off + n);
        }
    }
    for (int w = 0; w < 2; w++)
        HMG_CUDA_TRY(cudaMemsetAsync(g->codes[w], 0, sizeof(uint64_t) * g->n[w], s));
    g->points_set[0] = g->points_set[1] = true;
    // blocks: every set's dense blocks, then every set's admissible blocks
    const int nbi = (int)nb;
    g->h_r0.resize(nbi); g->h_m1.resize(nbi); g->h_c0.resize(nbi); g->h_m2.resize(nbi); g->h_type.resize(nbi);
    std::vector<double> param(nbi);
    int q = 0;
    for (int pass = 0; pass < 2; pass++)
        for (int i = 0; i < count; i++) {
            const hmg_matrix* h = sets[i];
            const int b0 = pass == 0 ? 0 : h->ndense, b1 = pass == 0 ? h->ndense : h->nblocks;
            for (int b = b0; b < b1; b++, q++) {
                g->h_r0[q] = h->h_r0[b] + g->group_off[0][i];
                g->h_m1[q] = h->h_m1[b];
                g->h_c0[q] = h->h_c0[b] + g->group_off[1][i];
                g->h_m2[q] = h->h_m2[b];
                g->h_type[q] = h->h_type[b];
                param[q] = h->kspec.param;
            }
        }
    g->nblocks = nbi;
    g->ndense = (int)nd;
    g->naca = nbi - (int)nd;
    g->levels = levels;
    g->eta = s0->eta;
    g->c_leaf = s0->c_leaf;
    g->max_level = s0->max_level;
    g->rule = s0->rule;
    if ((st = dalloc(&g->blk_r0, (size_t)nbi, s)) || (st = dalloc(&g->blk_m1, (size_t)nbi, s)) ||
        (st = dalloc(&g->blk_c0, (size_t)nbi, s)) || (st = dalloc(&g->blk_m2, (size_t)nbi, s)) ||
        (st = dalloc(&g->blk_type, (size_t)nbi, s)) || (st = dalloc(&g->blk_param, (size_t)nbi, s))) {
        hmg_destroy(g);
        return st;
    }
    if (nbi > 0) {
        HMG_CUDA_TRY(cudaMemcpyAsync(g->blk_r0, g->h_r0.data(), sizeof(int) * nbi, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(g->blk_m1, g->h_m1.data(), sizeof(int) * nbi, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(g->blk_c0, g->h_c0.data(), sizeof(int) * nbi, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(g->blk_m2, g->h_m2.data(), sizeof(int) * nbi, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(g->blk_type, g->h_type.data(), sizeof(int) * nbi, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(g->blk_param, param.data(), sizeof(double) * nbi, cudaMemcpyHostToDevice, s));
    }
    if ((st = build_tiles(g))) {
        hmg_destroy(g);
        return st;
    }
    g->kspec = s0->kspec;
    g->kspec.dim = dim;
    g->kernel_set = true;
    g->setup_done = true;
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    *out = g;
    return HMG_OK;
}

// The sets' points and kernels, clustered together (hmg_group_setup): the union of
// their points is ordered and its block-cluster tree built in the same launches for
// every set (one Morton pass, one stable sort pair, one level loop from one root pair
// per set), instead of one hmg_setup per set followed by hmg_group_create.  The result
// is the handle hmg_group_create makes from the sets after hmg_setup with these
// parameters: the same permutation, blocks, block order and kernel parameters.
hmg_status group_setup(hmg_matrix** out, hmg_matrix* const* sets, int count, double eta, const int* c_leaf,
                       int max_level, int rule, cudaStream_t s)
{
    hmg_status st;
    int n1 = 0, n2 = 0, dim = 2;
    const hmg_matrix* s0 = sets[0];
    std::vector<int> sdim(count), sbits(count), sleaf(count);
    for (int i = 0; i < count; i++) {
        const hmg_matrix* h = sets[i];
        if (!h || !h->points_set[0] || !h->points_set[1] || !h->kernel_set) {
            set_error("hmg_group_setup: set %d needs its points (both sides) and a kernel", i);
            return HMG_ERR_STATE;
        }
        if (h->group_count) {
            set_error("hmg_group_setup: set %d is itself a group", i);
            return HMG_ERR_INVALID;
        }
        if (h->dim != 2 && h->dim != 3) {
            set_error("hmg_group_setup: set %d has dimension %d (2 or 3 are grouped)", i, h->dim);
            return HMG_ERR_UNSUPPORTED;
        }
        if (h->kspec.kind != s0->kspec.kind || h->kspec.reg != s0->kspec.reg ||
            (h->kspec.kind == HMG_KERNEL_MATERN_REF && h->kspec.matern_ref_denom != s0->kspec.matern_ref_denom)) {
            set_error("hmg_group_setup: set %d has another kernel kind or regularization than set 0", i);
            return HMG_ERR_INVALID;
        }
        if (c_leaf[i] < 1) {
            set_error("hmg_group_setup: c_leaf[%d] must be >= 1 (got %d)", i, c_leaf[i]);
            return HMG_ERR_INVALID;
        }
        if ((long long)n1 + h->n[0] > 0x7fffffff || (long long)n2 + h->n[1] > 0x7fffffff) {
            set_error("hmg_group_setup: more than 2^31 - 1 points in the group");
            return HMG_ERR_INVALID;
        }
        n1 += h->n[0];
        n2 += h->n[1];
        dim = std::max(dim, h->dim);
        sdim[i] = h->dim;
        // (dim, bits) pairs with Morton codes (morton.cu:65); others get code 0
        const bool coded = (h->dim == 2 && h->bits == 32) || (h->dim == 3 && h->bits == 20);
        sbits[i] = coded ? h->bits : 0;
        sleaf[i] = c_leaf[i];
    }
    hmg_matrix* g = nullptr;
    if ((st = hmg_create(&g, n1, n2, dim, dim == 2 ? 32 : 20, (void*)s))) return st;
    g->group_count = count;
    for (int w = 0; w < 2; w++) {
        g->group_off[w].assign(1, 0);
        for (int i = 0; i < count; i++) {
            const hmg_matrix* h = sets[i];
            const int off = g->group_off[w].back(), n = h->n[w];
            k_copy_points<<<ceil_div(n, 256), 256, 0, s>>>(h->pts[w], n, h->dim, g->pts[w], g->n[w], off, dim);
            HMG_LAUNCH_CHECK();
            g->group_off[w].push_back(off + n);
        }
    }
    g->points_set[0] = g->points_set[1] = true;
    g->eta = eta;
    g->c_leaf = *std::max_element(sleaf.begin(), sleaf.end());
    g->max_level = max_level;
    g->rule = rule;
    const int* offp[2] = {g->group_off[0].data(), g->group_off[1].data()};
    if ((st = group_setup_tree(g, count, offp, sdim.data(), sbits.data(), sleaf.data()))) {
        hmg_destroy(g);
        return st;
    }
    // each block's kernel parameter: that of the set holding its rows
    const int nb = g->nblocks;
    std::vector<double> param(nb);
    for (int q = 0; q < nb; q++) {
        const int set = (int)(std::upper_bound(g->group_off[0].begin(), g->group_off[0].end(), g->h_r0[q]) -
                              g->group_off[0].begin()) - 1;
        param[q] = sets[set]->kspec.param;
    }
    if ((st = dalloc(&g->blk_param, (size_t)(nb > 0 ? nb : 1), s))) {
        hmg_destroy(g);
        return st;
    }
    if (nb > 0) HMG_CUDA_TRY(cudaMemcpyAsync(g->blk_param, param.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    if ((st = build_tiles(g))) {
        hmg_destroy(g);
        return st;
    }
    g->kspec = s0->kspec;
    g->kspec.dim = dim;
    g->kernel_set = true;
    g->setup_done = true;
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    *out = g;
    return HMG_OK;
}

}  // namespace hmg
