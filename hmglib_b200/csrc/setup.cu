// setup.cu -- point ordering and block-cluster tree construction on the GPU.
//
// Replaces the reference's setup path (hmglib.cu:125-225):
//   * compute_minmax (helper.cu:108-138): one pass, order-preserving 64-bit keys
//     reduced with atomicMin/atomicMax (exact);
//   * get_morton_code (morton.cu:79-112): one thread per point;
//   * get_morton_ordering (helper.cu:140-167): the stable radix sort of util.cu;
//   * reorder_point_set (helper.cu:293-328): one gather of all dimensions;
//   * traverse_with_dynamic_arrays_dynamic_output (tree.cu:1429-1557): level-
//     synchronous, but the reference's per-level lookup-table construction for
//     bounding boxes (tree.cu:852-1245, ~30 Thrust calls per level) is replaced by
//     one CTA-per-cluster min/max reduction over the cluster's contiguous Z range,
//     written into a map indexed by the cluster's first point; children and leaves
//     are emitted at offsets from one packed (leaf, child) exclusive scan.
//   * organize_mat_vec_data (linear_algebra.cu:4037-4051): stable DENSE-first
//     partition by one scan.
#include <algorithm>
#include <vector>

#include "hmg_matrix.cuh"

namespace hmg {

// ---------------------------------------------------------------------------
// min / max and Morton codes
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long order_key(double x)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double order_key_inv(unsigned long long o)
{
    unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
    return __longlong_as_double((long long)b);
}

__global__ void k_minmax(const double* coords, int n, int dim, unsigned long long* mn,
                         unsigned long long* mx)
{
    for (int d = 0; d < dim; d++) {
        const double* c = coords + (size_t)d * n;
        unsigned long long lo = ~0ull, hi = 0ull;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
             i += (long long)gridDim.x * blockDim.x) {
            unsigned long long k = order_key(c[i]);
            lo = k < lo ? k : lo;
            hi = k > hi ? k : hi;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
            unsigned long long b = __shfl_xor_sync(0xffffffffu, hi, o);
            lo = a < lo ? a : lo;
            hi = b > hi ? b : hi;
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&mn[d], lo);
            atomicMax(&mx[d], hi);
        }
    }
}

// morton.cu:71-75: q = min(floor((c - min) / (max - min) * 2^bits), 2^bits - 1), then
// bit b of q goes to bit b*dim + d of the code (morton.cu:21-67, :93-103).
__global__ void k_morton(const double* coords, int n, int dim, int bits,
                         const unsigned long long* mn_key, const unsigned long long* mx_key,
                         uint64_t* codes)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t code = 0;
    const double scale = (double)(1ull << bits);
    const uint64_t cap = (1ull << bits) - 1ull;
    for (int d = 0; d < dim; d++) {
        double lo = order_key_inv(mn_key[d]);
        double hi = order_key_inv(mx_key[d]);
        double range = hi - lo;
        double t = (coords[(size_t)d * n + i] - lo) / range;
        // same conversion as the reference's device code: a NaN quotient (max == min)
        // converts to the top of the range and is capped below
        uint64_t q = (uint64_t)floor(t * scale);
        q = q < cap ? q : cap;
        for (int b = 0; b < bits; b++) code |= ((q >> b) & 1ull) << (b * dim + d);
    }
    codes[i] = code;
}

__global__ void k_iota(uint32_t* v, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (uint32_t)i;
}

__global__ void k_gather_points(const double* src, double* dst, const uint32_t* order, int n,
                                int dim, int* perm, int* iperm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t o = order[i];
    for (int d = 0; d < dim; d++) dst[(size_t)d * n + i] = src[(size_t)d * n + o];
    perm[i] = (int)o;
    iperm[o] = i;
}

__global__ void k_keys_to_double(const unsigned long long* mn_key, const unsigned long long* mx_key, int dim,
                                 double* mn, double* mx)
{
    int d = threadIdx.x;
    if (d < dim) {
        mn[d] = order_key_inv(mn_key[d]);
        mx[d] = order_key_inv(mx_key[d]);
    }
}

// Per-dimension minimum and maximum of n points (SoA coords[d*n+i]) into the device
// arrays mn[dim], mx[dim] (helper.cu:108-138, compute_minmax); exact.
hmg_status minmax_device(const double* coords, int n, int dim, double* mn, double* mx, cudaStream_t s)
{
    if (n <= 0 || dim <= 0) return HMG_OK;
    unsigned long long* mm = nullptr;
    hmg_status st = dalloc(&mm, (size_t)2 * dim, s);
    if (st) return st;
    HMG_CUDA_TRY(cudaMemsetAsync(mm, 0xff, sizeof(unsigned long long) * dim, s));
    HMG_CUDA_TRY(cudaMemsetAsync(mm + dim, 0, sizeof(unsigned long long) * dim, s));
    int g = ceil_div(n, 256);
    if (g > 1184) g = 1184;
    k_minmax<<<g, 256, 0, s>>>(coords, n, dim, mm, mm + dim);
    HMG_LAUNCH_CHECK();
    k_keys_to_double<<<1, 32, 0, s>>>(mm, mm + dim, dim, mn, mx);
    HMG_LAUNCH_CHECK();
    dfree(mm, s);
    return HMG_OK;
}

static bool morton_supported(int dim, int bits)
{
    return (dim == 2 && bits == 32) || (dim == 3 && bits == 20) || (dim == 10 && bits == 4);
}

hmg_status morton_codes(const double* coords, int n, int dim, int bits, uint64_t* codes,
                        cudaStream_t s)
{
    if (n <= 0) return HMG_OK;
    if (!morton_supported(dim, bits)) {
        // morton.cu:65 returns 0 for unsupported (dim, bits)
        HMG_CUDA_TRY(cudaMemsetAsync(codes, 0, sizeof(uint64_t) * n, s));
        return HMG_OK;
    }
    unsigned long long* mm = nullptr;
    hmg_status st = dalloc(&mm, (size_t)2 * dim, s);
    if (st) return st;
    HMG_CUDA_TRY(cudaMemsetAsync(mm, 0xff, sizeof(unsigned long long) * dim, s));
    HMG_CUDA_TRY(cudaMemsetAsync(mm + dim, 0, sizeof(unsigned long long) * dim, s));
    int g = ceil_div(n, 256);
    if (g > 1184) g = 1184;
    k_minmax<<<g, 256, 0, s>>>(coords, n, dim, mm, mm + dim);
    HMG_LAUNCH_CHECK();
    k_morton<<<ceil_div(n, 256), 256, 0, s>>>(coords, n, dim, bits, mm, mm + dim, codes);
    HMG_LAUNCH_CHECK();
    dfree(mm, s);
    return HMG_OK;
}

// ---------------------------------------------------------------------------
// block-cluster tree
// ---------------------------------------------------------------------------

// tree.cu:40-78 (findSplit): last index s in [first,last) whose code shares more than
// the common prefix of the end codes with codes[first]; midpoint for equal ends.
// The bit below the common prefix is 0 on a prefix of the sorted range, so the
// answer is found by bisection on that bit.
__device__ int split_index(const uint64_t* codes, int first, int last)
{
    uint64_t a = codes[first], b = codes[last];
    if (a == b) return (first + last) >> 1;
    int common = __clzll((long long)(a ^ b));
    int lo = first, hi = last;  // pred(lo) true, pred(hi) false
    while (hi - lo > 1) {
        int mid = lo + ((hi - lo) >> 1);
        if (__clzll((long long)(a ^ codes[mid])) > common)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// One CTA per cluster [l,u]: exact bounding box into the per-level maps (indexed by
// l), and the split point for clusters that may be subdivided.  leaf_at (grouped
// point sets, else null) gives the leaf size of the set that holds each point.
__global__ void k_cluster_bbox(const int* cl_l, const int* cl_u, int ncl, const double* z,
                               int n, int dim, const uint64_t* codes, int c_leaf, const int* leaf_at,
                               double* bb_lo, double* bb_hi, int* split_of)
{
    __shared__ double red[2][3][8];
    int c = blockIdx.x;
    if (c >= ncl) return;
    int l = cl_l[c], u = cl_u[c];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 0; d < dim; d++) {
        const double* zc = z + (size_t)d * n;
        double lo = zc[l], hi = zc[l];
        for (int i = l + threadIdx.x; i <= u; i += blockDim.x) {
            double v = zc[i];
            lo = fmin(lo, v);
            hi = fmax(hi, v);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            red[0][d][warp] = lo;
            red[1][d][warp] = hi;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int nw = blockDim.x >> 5;
        for (int d = 0; d < dim; d++) {
            double lo = red[0][d][0], hi = red[1][d][0];
            for (int w = 1; w < nw; w++) {
                lo = fmin(lo, red[0][d][w]);
                hi = fmax(hi, red[1][d][w]);
            }
            bb_lo[(size_t)d * n + l] = lo;
            bb_hi[(size_t)d * n + l] = hi;
        }
        if (u - l + 1 > (leaf_at ? leaf_at[l] : c_leaf)) split_of[l] = split_index(codes, l, u);
    }
}

// tree.cu:94-160 with the FMA contraction of the diameter sum made explicit.
__device__ __forceinline__ bool admissible(const double* lo1, const double* hi1,
                                           const double* lo2, const double* hi2, int dim,
                                           double eta, int rule)
{
    double s1 = 0.0, s2 = 0.0, s = 0.0;
    for (int d = 0; d < dim; d++) {
        double t1 = hi1[d] - lo1[d];
        double t2 = hi2[d] - lo2[d];
        s1 = __fma_rn(t1, t1, s1);
        s2 = __fma_rn(t2, t2, s2);
        double a = fmax(0.0, lo1[d] - hi2[d]);
        double b = fmax(0.0, lo2[d] - hi1[d]);
        s = __dadd_rn(s, __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
    }
    double d1 = sqrt(s1), d2 = sqrt(s2), dist = sqrt(s);
    double lhs = rule == HMG_ADMISSIBLE_MAX ? fmax(d1, d2) : fmin(d1, d2);
    return lhs <= __dmul_rn(eta, dist);
}

struct NodeArrays {
    int *l1, *u1, *l2, *u2;
};

// tree.cu:215-266 (count_for_new_level): per node 1 leaf or 4 children, packed as
// (leaf << 32) | children for a single scan.
__global__ void k_node_classify(NodeArrays nd, int nn, int n1, int n2, int dim,
                                const double* bb1_lo, const double* bb1_hi,
                                const double* bb2_lo, const double* bb2_hi, double eta,
                                int rule, int c_leaf, const int* leaf_at, int last_level, long long* packed,
                                signed char* leaf_type)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    int l1 = nd.l1[i], u1 = nd.u1[i], l2 = nd.l2[i], u2 = nd.u2[i];
    // both clusters of a node belong to one set: its leaf size
    if (leaf_at) c_leaf = leaf_at[l1];
    double lo1[3], hi1[3], lo2[3], hi2[3];
    for (int d = 0; d < dim; d++) {
        lo1[d] = bb1_lo[(size_t)d * n1 + l1];
        hi1[d] = bb1_hi[(size_t)d * n1 + l1];
        lo2[d] = bb2_lo[(size_t)d * n2 + l2];
        hi2[d] = bb2_hi[(size_t)d * n2 + l2];
    }
    bool adm = admissible(lo1, hi1, lo2, hi2, dim, eta, rule);
    int m1 = u1 - l1 + 1, m2 = u2 - l2 + 1;
    signed char t = 0;
    long long p;
    if (adm) {
        t = HMG_WT_ACA;
        p = 1ll << 32;
    } else if (m1 <= c_leaf || m2 <= c_leaf || last_level) {
        t = HMG_WT_DENSE;
        p = 1ll << 32;
    } else {
        p = 4;
    }
    packed[i] = p;
    leaf_type[i] = t;
}

struct LeafArrays {
    int *l1, *u1, *l2, *u2, *type;
};

// tree.cu:320-447 (generate_new_level): children 11, 12, 21, 22 and leaves at the
// scanned offsets.
__global__ void k_node_emit(NodeArrays nd, int nn, const long long* offs,
                            const signed char* leaf_type, const int* split1,
                            const int* split2, NodeArrays next, LeafArrays leaves,
                            int leaf_base)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    int l1 = nd.l1[i], u1 = nd.u1[i], l2 = nd.l2[i], u2 = nd.u2[i];
    long long o = offs[i];
    signed char t = leaf_type[i];
    if (t) {
        int k = leaf_base + (int)(o >> 32);
        leaves.l1[k] = l1; leaves.u1[k] = u1; leaves.l2[k] = l2; leaves.u2[k] = u2;
        leaves.type[k] = t;
    } else {
        int c = (int)(o & 0xffffffffll);
        int s1 = split1[l1], s2 = split2[l2];
        next.l1[c] = l1;     next.u1[c] = s1;  next.l2[c] = l2;     next.u2[c] = s2;
        next.l1[c + 1] = l1; next.u1[c + 1] = s1; next.l2[c + 1] = s2 + 1; next.u2[c + 1] = u2;
        next.l1[c + 2] = s1 + 1; next.u1[c + 2] = u1; next.l2[c + 2] = l2; next.u2[c + 2] = s2;
        next.l1[c + 3] = s1 + 1; next.u1[c + 3] = u1; next.l2[c + 3] = s2 + 1; next.u2[c + 3] = u2;
    }
}

// clusters of the next level: both children of every cluster larger than c_leaf
__global__ void k_cluster_count(const int* cl_l, const int* cl_u, int ncl, int c_leaf,
                                const int* leaf_at, int* cnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncl) return;
    cnt[i] = (cl_u[i] - cl_l[i] + 1 > (leaf_at ? leaf_at[cl_l[i]] : c_leaf)) ? 2 : 0;
}

__global__ void k_cluster_emit(const int* cl_l, const int* cl_u, int ncl, const int* off,
                               int c_leaf, const int* leaf_at, const int* split_of, int* nl, int* nu)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncl) return;
    int l = cl_l[i], u = cl_u[i];
    if (u - l + 1 <= (leaf_at ? leaf_at[l] : c_leaf)) return;
    int s = split_of[l];
    int o = off[i];
    nl[o] = l; nu[o] = s;
    nl[o + 1] = s + 1; nu[o + 1] = u;
}

// linear_algebra.cu:63-86: stable partition DENSE before ACA
__global__ void k_dense_flags(const int* type, int n, int* f)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = type[i] == HMG_WT_DENSE ? 1 : 0;
}

__global__ void k_partition(LeafArrays in, int n, const int* scanf, int ndense, int* r0,
                            int* m1, int* c0, int* m2, int* type)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int t = in.type[i];
    int dpos = scanf[i];
    int k = t == HMG_WT_DENSE ? dpos : ndense + (i - dpos);
    r0[k] = in.l1[i];
    m1[k] = in.u1[i] - in.l1[i] + 1;
    c0[k] = in.l2[i];
    m2[k] = in.u2[i] - in.l2[i] + 1;
    type[k] = t;
}

static void free_nodes(NodeArrays& a, cudaStream_t s)
{
    dfree(a.l1, s); dfree(a.u1, s); dfree(a.l2, s); dfree(a.u2, s);
}

static hmg_status alloc_nodes(NodeArrays& a, size_t n, cudaStream_t s)
{
    hmg_status st;
    a = {nullptr, nullptr, nullptr, nullptr};
    if ((st = dalloc(&a.l1, n, s)) || (st = dalloc(&a.u1, n, s)) || (st = dalloc(&a.l2, n, s)) ||
        (st = dalloc(&a.u2, n, s))) {
        free_nodes(a, s);
        return st;
    }
    return HMG_OK;
}

static void free_leaves(LeafArrays& a, cudaStream_t s)
{
    dfree(a.l1, s); dfree(a.u1, s); dfree(a.l2, s); dfree(a.u2, s); dfree(a.type, s);
}

static hmg_status alloc_leaves(LeafArrays& a, size_t n, cudaStream_t s)
{
    hmg_status st;
    a = {nullptr, nullptr, nullptr, nullptr, nullptr};
    if ((st = dalloc(&a.l1, n, s)) || (st = dalloc(&a.u1, n, s)) || (st = dalloc(&a.l2, n, s)) ||
        (st = dalloc(&a.u2, n, s)) || (st = dalloc(&a.type, n, s))) {
        free_leaves(a, s);
        return st;
    }
    return HMG_OK;
}

void free_tree(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    dfree(h->blk_r0, s); dfree(h->blk_m1, s); dfree(h->blk_c0, s); dfree(h->blk_m2, s);
    dfree(h->blk_type, s);
    dfree(h->tile_r0, s); dfree(h->tile_s, s); dfree(h->tile_pstart, s);
    dfree(h->blk_tfirst, s); dfree(h->blk_tlast, s);
    dfree(h->tile_pair_start, s); dfree(h->pair_block, s);
    dfree(h->blk_param, s);
    h->nblocks = h->ndense = h->naca = h->ntiles = h->npairs = h->levels = 0;
    h->setup_done = false;
}

// Per-set cluster state of the level-synchronous traversal.
struct ClusterSet {
    int n = 0;
    int ncl = 0;
    int* cl_l = nullptr;
    int* cl_u = nullptr;
    double* bb_lo = nullptr;  // [dim][n], valid at the current level's cluster starts
    double* bb_hi = nullptr;
    int* split_of = nullptr;  // [n]
};

static void free_cluster_set(ClusterSet& c, cudaStream_t s)
{
    dfree(c.cl_l, s); dfree(c.cl_u, s); dfree(c.bb_lo, s); dfree(c.bb_hi, s);
    dfree(c.split_of, s);
}

// Level-synchronous traversal (tree.cu:1429-1557) from nroots root pairs: root i pairs
// the row cluster [rl1[i], ru1[i]] with the column cluster [rl2[i], ru2[i]], and each
// side's cluster list starts from its roots' ranges.  Leaves are appended in the order
// the levels emit them; leaf_at[side] (grouped point sets, else null) gives the leaf
// size of the set that holds each point.
static hmg_status traverse(hmg_matrix* h, int nroots, const int* rl1, const int* ru1, const int* rl2,
                           const int* ru2, const int* const* leaf_at, LeafArrays& leaves, int& nleaves,
                           int& levels)
{
    cudaStream_t s = h->stream;
    hmg_status st = HMG_OK;
    const int dim = h->dim;
    ClusterSet cs[2];
    NodeArrays cur{}, nxt{};
    int leaf_cap = 0;
    long long* packed = nullptr;
    signed char* ltype = nullptr;
    int* ccnt = nullptr;
    long long* ptot = nullptr;
    int nn = nroots;
    nleaves = 0;
    levels = 0;
    leaves = LeafArrays{};

    for (int set = 0; set < 2; set++) {
        ClusterSet& c = cs[set];
        c.n = h->n[set];
        c.ncl = nroots;
        if ((st = dalloc(&c.cl_l, (size_t)nroots, s)) || (st = dalloc(&c.cl_u, (size_t)nroots, s)) ||
            (st = dalloc(&c.bb_lo, (size_t)dim * c.n, s)) ||
            (st = dalloc(&c.bb_hi, (size_t)dim * c.n, s)) ||
            (st = dalloc(&c.split_of, (size_t)c.n, s)))
            goto done;
        HMG_CUDA_TRY(cudaMemcpyAsync(c.cl_l, set ? rl2 : rl1, sizeof(int) * nroots, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(c.cl_u, set ? ru2 : ru1, sizeof(int) * nroots, cudaMemcpyHostToDevice, s));
    }
    if ((st = alloc_nodes(cur, (size_t)nroots, s))) goto done;
    HMG_CUDA_TRY(cudaMemcpyAsync(cur.l1, rl1, sizeof(int) * nroots, cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(cur.u1, ru1, sizeof(int) * nroots, cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(cur.l2, rl2, sizeof(int) * nroots, cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(cur.u2, ru2, sizeof(int) * nroots, cudaMemcpyHostToDevice, s));
    if ((st = dalloc(&ptot, 3, s))) goto done;

    for (int it = 0; it < h->max_level && nn > 0; it++) {
        levels = it + 1;
        bool last_level = it + 1 >= h->max_level;
        // bounding boxes and split points of this level's clusters
        for (int set = 0; set < 2; set++) {
            ClusterSet& c = cs[set];
            if (c.ncl > 0) {
                k_cluster_bbox<<<c.ncl, 256, 0, s>>>(c.cl_l, c.cl_u, c.ncl, h->zpts[set], c.n, dim,
                                                     h->codes[set], h->c_leaf, leaf_at[set], c.bb_lo,
                                                     c.bb_hi, c.split_of);
                HMG_LAUNCH_CHECK();
            }
        }
        if ((st = dalloc(&packed, (size_t)nn, s)) || (st = dalloc(&ltype, (size_t)nn, s)))
            goto done;
        k_node_classify<<<ceil_div(nn, 256), 256, 0, s>>>(
            cur, nn, h->n[0], h->n[1], dim, cs[0].bb_lo, cs[0].bb_hi, cs[1].bb_lo, cs[1].bb_hi,
            h->eta, h->rule, h->c_leaf, leaf_at[0], last_level ? 1 : 0, packed, ltype);
        HMG_LAUNCH_CHECK();
        if ((st = scan_exclusive<long long>(packed, packed, nn, ptot, s))) goto done;
        long long tot = 0;
        HMG_CUDA_TRY(cudaMemcpyAsync(&tot, ptot, sizeof(long long), cudaMemcpyDeviceToHost, s));
        HMG_CUDA_TRY(cudaStreamSynchronize(s));
        int new_leaves = (int)(tot >> 32);
        int new_children = (int)(tot & 0xffffffffll);
        if (nleaves + new_leaves > leaf_cap) {
            int ncap = leaf_cap ? leaf_cap : 4096;
            while (ncap < nleaves + new_leaves) ncap *= 2;
            LeafArrays nl{};
            if ((st = alloc_leaves(nl, (size_t)ncap, s))) goto done;
            if (nleaves) {
                HMG_CUDA_TRY(cudaMemcpyAsync(nl.l1, leaves.l1, sizeof(int) * nleaves, cudaMemcpyDeviceToDevice, s));
                HMG_CUDA_TRY(cudaMemcpyAsync(nl.u1, leaves.u1, sizeof(int) * nleaves, cudaMemcpyDeviceToDevice, s));
                HMG_CUDA_TRY(cudaMemcpyAsync(nl.l2, leaves.l2, sizeof(int) * nleaves, cudaMemcpyDeviceToDevice, s));
                HMG_CUDA_TRY(cudaMemcpyAsync(nl.u2, leaves.u2, sizeof(int) * nleaves, cudaMemcpyDeviceToDevice, s));
                HMG_CUDA_TRY(cudaMemcpyAsync(nl.type, leaves.type, sizeof(int) * nleaves, cudaMemcpyDeviceToDevice, s));
            }
            free_leaves(leaves, s);
            leaves = nl;
            leaf_cap = ncap;
        }
        if ((st = alloc_nodes(nxt, (size_t)(new_children > 0 ? new_children : 1), s))) goto done;
        k_node_emit<<<ceil_div(nn, 256), 256, 0, s>>>(cur, nn, packed, ltype, cs[0].split_of,
                                                      cs[1].split_of, nxt, leaves, nleaves);
        HMG_LAUNCH_CHECK();
        nleaves += new_leaves;
        free_nodes(cur, s);
        cur = nxt;
        nxt = NodeArrays{};
        nn = new_children;
        dfree(packed, s);
        dfree(ltype, s);

        // clusters of the next level
        if (nn > 0) {
            for (int set = 0; set < 2; set++) {
                ClusterSet& c = cs[set];
                int *nl = nullptr, *nu = nullptr;
                int ntot = 0;
                if ((st = dalloc(&ccnt, (size_t)c.ncl, s))) goto done;
                k_cluster_count<<<ceil_div(c.ncl, 256), 256, 0, s>>>(c.cl_l, c.cl_u, c.ncl,
                                                                     h->c_leaf, leaf_at[set], ccnt);
                HMG_LAUNCH_CHECK();
                if ((st = scan_exclusive<int>(ccnt, ccnt, c.ncl, (int*)ptot, s))) goto done;
                HMG_CUDA_TRY(cudaMemcpyAsync(&ntot, ptot, sizeof(int), cudaMemcpyDeviceToHost, s));
                HMG_CUDA_TRY(cudaStreamSynchronize(s));
                if ((st = dalloc(&nl, (size_t)(ntot > 0 ? ntot : 1), s)) ||
                    (st = dalloc(&nu, (size_t)(ntot > 0 ? ntot : 1), s)))
                    goto done;
                k_cluster_emit<<<ceil_div(c.ncl, 256), 256, 0, s>>>(c.cl_l, c.cl_u, c.ncl, ccnt,
                                                                    h->c_leaf, leaf_at[set], c.split_of,
                                                                    nl, nu);
                HMG_LAUNCH_CHECK();
                dfree(ccnt, s);
                dfree(c.cl_l, s);
                dfree(c.cl_u, s);
                c.cl_l = nl;
                c.cl_u = nu;
                c.ncl = ntot;
            }
        }
    }

done:
    free_nodes(cur, s);
    free_nodes(nxt, s);
    dfree(packed, s);
    dfree(ltype, s);
    dfree(ccnt, s);
    dfree(ptot, s);
    free_cluster_set(cs[0], s);
    free_cluster_set(cs[1], s);
    return st;
}

// sort key of a leaf for the grouped order: DENSE first, then the set of its rows
// (set_off: the first row of every set and the total, nsets + 1 entries)
__global__ void k_leaf_keys(LeafArrays in, int n, const int* set_off, int nsets, int set_bits,
                            uint64_t* keys, uint32_t* idx)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = in.l1[i];
    int lo = 0, hi = nsets;  // set_off[lo] <= r < set_off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (set_off[mid] <= r) lo = mid; else hi = mid;
    }
    keys[i] = ((uint64_t)(in.type[i] == HMG_WT_DENSE ? 0 : 1) << set_bits) | (uint64_t)lo;
    idx[i] = (uint32_t)i;
}

__global__ void k_gather_leaves(LeafArrays in, int n, const uint32_t* idx, int* r0, int* m1, int* c0,
                                int* m2, int* type)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = (int)idx[k];
    r0[k] = in.l1[i];
    m1[k] = in.u1[i] - in.l1[i] + 1;
    c0[k] = in.l2[i];
    m2[k] = in.u2[i] - in.l2[i] + 1;
    type[k] = in.type[i];
}

// The leaves as the handle's block arrays, DENSE first (linear_algebra.cu:63-86,
// a stable partition), and their host copies.  With set_off (grouped point sets: the
// first row of every set and the total, on the device) the order is DENSE first, then
// by set, each set's blocks in the order they were emitted.
static hmg_status partition_blocks(hmg_matrix* h, const LeafArrays& leaves, int nb, int levels,
                                   const int* set_off, int nsets)
{
    cudaStream_t s = h->stream;
    hmg_status st = HMG_OK;
    int* f = nullptr;
    int* tot = nullptr;
    uint64_t* keys = nullptr;
    uint32_t* idx = nullptr;
    int nd = 0;
    h->nblocks = nb;
    if ((st = dalloc(&h->blk_r0, (size_t)nb, s)) || (st = dalloc(&h->blk_m1, (size_t)nb, s)) ||
        (st = dalloc(&h->blk_c0, (size_t)nb, s)) || (st = dalloc(&h->blk_m2, (size_t)nb, s)) ||
        (st = dalloc(&h->blk_type, (size_t)nb, s)))
        goto done;
    if (nb > 0 && !set_off) {
        if ((st = dalloc(&f, (size_t)nb, s)) || (st = dalloc(&tot, 1, s))) goto done;
        k_dense_flags<<<ceil_div(nb, 256), 256, 0, s>>>(leaves.type, nb, f);
        HMG_LAUNCH_CHECK();
        if ((st = scan_exclusive<int>(f, f, nb, tot, s))) goto done;
        HMG_CUDA_TRY(cudaMemcpyAsync(&nd, tot, sizeof(int), cudaMemcpyDeviceToHost, s));
        HMG_CUDA_TRY(cudaStreamSynchronize(s));
        k_partition<<<ceil_div(nb, 256), 256, 0, s>>>(leaves, nb, f, nd, h->blk_r0, h->blk_m1,
                                                      h->blk_c0, h->blk_m2, h->blk_type);
        HMG_LAUNCH_CHECK();
    } else if (nb > 0) {
        int set_bits = 1;
        while ((1 << set_bits) < nsets) set_bits++;
        if ((st = dalloc(&keys, (size_t)nb, s)) || (st = dalloc(&idx, (size_t)nb, s))) goto done;
        k_leaf_keys<<<ceil_div(nb, 256), 256, 0, s>>>(leaves, nb, set_off, nsets, set_bits, keys, idx);
        HMG_LAUNCH_CHECK();
        if ((st = radix_sort_pairs(keys, idx, nb, set_bits + 1, s))) goto done;
        k_gather_leaves<<<ceil_div(nb, 256), 256, 0, s>>>(leaves, nb, idx, h->blk_r0, h->blk_m1, h->blk_c0,
                                                          h->blk_m2, h->blk_type);
        HMG_LAUNCH_CHECK();
    }
    h->levels = levels;
    h->h_r0.resize(nb); h->h_m1.resize(nb); h->h_c0.resize(nb); h->h_m2.resize(nb);
    h->h_type.resize(nb);
    if (nb > 0) {
        HMG_CUDA_TRY(cudaMemcpyAsync(h->h_r0.data(), h->blk_r0, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->h_m1.data(), h->blk_m1, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->h_c0.data(), h->blk_c0, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->h_m2.data(), h->blk_m2, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->h_type.data(), h->blk_type, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
    }
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    if (set_off) nd = (int)std::count(h->h_type.begin(), h->h_type.end(), (int)HMG_WT_DENSE);
    h->ndense = nd;
    h->naca = nb - nd;

done:
    dfree(f, s);
    dfree(tot, s);
    dfree(keys, s);
    dfree(idx, s);
    return st;
}

hmg_status setup_tree(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    hmg_status st = HMG_OK;
    const int dim = h->dim;

    // ---- Morton codes, sort, gather (hmglib.cu:128-162) ------------------------
    for (int set = 0; set < 2; set++) {
        int n = h->n[set];
        uint32_t* order = nullptr;
        if ((st = morton_codes(h->pts[set], n, dim, h->bits, h->codes[set], s))) return st;
        if ((st = dalloc(&order, (size_t)n, s))) return st;
        k_iota<<<ceil_div(n, 256), 256, 0, s>>>(order, n);
        HMG_LAUNCH_CHECK();
        int key_bits = dim * h->bits;
        if (key_bits > 64) key_bits = 64;
        if ((st = radix_sort_pairs(h->codes[set], order, n, key_bits, s))) {
            dfree(order, s);
            return st;
        }
        k_gather_points<<<ceil_div(n, 256), 256, 0, s>>>(h->pts[set], h->zpts[set], order, n,
                                                         dim, h->perm[set], h->iperm[set]);
        HMG_LAUNCH_CHECK();
        dfree(order, s);
    }

    // ---- block-cluster tree from the root pair, then the DENSE-first block list ----
    const int root[4] = {0, h->n[0] - 1, 0, h->n[1] - 1};
    const int* no_leaf_at[2] = {nullptr, nullptr};
    LeafArrays leaves{};
    int nleaves = 0, levels = 0;
    st = traverse(h, 1, &root[0], &root[1], &root[2], &root[3], no_leaf_at, leaves, nleaves, levels);
    if (!st) st = partition_blocks(h, leaves, nleaves, levels, nullptr, 0);
    free_leaves(leaves, s);
    return st;
}

// ---------------------------------------------------------------------------
// many point sets clustered in the same launches (hmg_group_setup)
// ---------------------------------------------------------------------------

// set of union index i: off[set] <= i < off[set + 1]
__device__ __forceinline__ int set_of_index(const int* off, int nsets, int i)
{
    int lo = 0, hi = nsets;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// One CTA per set: order keys of its per-dimension minimum and maximum into
// mm[(set * 3 + d) * 2 + {0, 1}] (exact, as k_minmax).
__global__ void k_minmax_sets(const double* coords, int n, const int* off, const int* sdim,
                              unsigned long long* mm)
{
    __shared__ unsigned long long red[2][32];
    const int set = blockIdx.x, a = off[set], b = off[set + 1], dim = sdim[set];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int d = 0; d < dim; d++) {
        const double* c = coords + (size_t)d * n;
        unsigned long long lo = ~0ull, hi = 0ull;
        for (int i = a + threadIdx.x; i < b; i += blockDim.x) {
            const unsigned long long k = order_key(c[i]);
            lo = k < lo ? k : lo;
            hi = k > hi ? k : hi;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, lo, o);
            const unsigned long long y = __shfl_xor_sync(0xffffffffu, hi, o);
            lo = x < lo ? x : lo;
            hi = y > hi ? y : hi;
        }
        if (lane == 0) {
            red[0][warp] = lo;
            red[1][warp] = hi;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < nw; w++) {
                lo = red[0][w] < lo ? red[0][w] : lo;
                hi = red[1][w] > hi ? red[1][w] : hi;
            }
            mm[((size_t)set * 3 + d) * 2] = lo;
            mm[((size_t)set * 3 + d) * 2 + 1] = hi;
        }
        __syncthreads();
    }
}

// k_morton for every set at once: point i of the union (stride n) takes its set's
// dimension, bits and extremes; sbits 0 marks a (dim, bits) without Morton codes
// (code 0, as morton.cu:65).  set_of[i] receives the point's set.
__global__ void k_morton_sets(const double* coords, int n, const int* off, int nsets, const int* sdim,
                              const int* sbits, const unsigned long long* mm, uint64_t* codes,
                              uint64_t* set_of)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int set = set_of_index(off, nsets, i);
    const int dim = sdim[set], bits = sbits[set];
    uint64_t code = 0;
    if (bits > 0) {
        const double scale = (double)(1ull << bits);
        const uint64_t cap = (1ull << bits) - 1ull;
        for (int d = 0; d < dim; d++) {
            double lo = order_key_inv(mm[((size_t)set * 3 + d) * 2]);
            double hi = order_key_inv(mm[((size_t)set * 3 + d) * 2 + 1]);
            double range = hi - lo;
            double t = (coords[(size_t)d * n + i] - lo) / range;
            uint64_t q = (uint64_t)floor(t * scale);
            q = q < cap ? q : cap;
            for (int b = 0; b < bits; b++) code |= ((q >> b) & 1ull) << (b * dim + d);
        }
    }
    codes[i] = code;
    set_of[i] = (uint64_t)set;
}

__global__ void k_gather_u64(const uint64_t* in, const uint32_t* idx, int n, uint64_t* out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[idx[i]];
}

__global__ void k_leaf_at(const int* off, int nsets, const int* sleaf, int n, int* leaf_at)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) leaf_at[i] = sleaf[set_of_index(off, nsets, i)];
}

// The tree of a group handle whose union points (g->pts, sets contiguous at off[w],
// 2D sets padded with a zero third coordinate) are in place: every set ordered by its
// own Morton codes, then one level-synchronous traversal from one root pair per set.
// Per set: sdim, sbits (0: no Morton codes), sleaf (leaf size).  Each set's
// permutation, tree and blocks are those hmg_setup gives the set alone; the blocks are
// ordered DENSE first, then by set.
hmg_status group_setup_tree(hmg_matrix* g, int nsets, const int* const* off, const int* sdim,
                            const int* sbits, const int* sleaf)
{
    cudaStream_t s = g->stream;
    hmg_status st = HMG_OK;
    int* doff[2] = {nullptr, nullptr};
    int *dsdim = nullptr, *dsbits = nullptr, *dsleaf = nullptr;
    int* leaf_at[2] = {nullptr, nullptr};
    unsigned long long* mm = nullptr;
    uint64_t *keys = nullptr, *set_of = nullptr;
    uint32_t* order = nullptr;
    LeafArrays leaves{};
    int nleaves = 0, levels = 0, code_bits = 1, set_bits = 1;
    std::vector<int> rl[2], ru[2];
    for (int i = 0; i < nsets; i++) code_bits = std::max(code_bits, std::min(64, sdim[i] * sbits[i]));
    while ((1 << set_bits) < nsets) set_bits++;
    if ((st = dalloc(&dsdim, (size_t)nsets, s)) || (st = dalloc(&dsbits, (size_t)nsets, s)) ||
        (st = dalloc(&dsleaf, (size_t)nsets, s)) || (st = dalloc(&mm, (size_t)nsets * 6, s)))
        goto done;
    HMG_CUDA_TRY(cudaMemcpyAsync(dsdim, sdim, sizeof(int) * nsets, cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(dsbits, sbits, sizeof(int) * nsets, cudaMemcpyHostToDevice, s));
    HMG_CUDA_TRY(cudaMemcpyAsync(dsleaf, sleaf, sizeof(int) * nsets, cudaMemcpyHostToDevice, s));
    for (int w = 0; w < 2; w++) {
        const int n = g->n[w];
        if ((st = dalloc(&doff[w], (size_t)nsets + 1, s)) || (st = dalloc(&leaf_at[w], (size_t)n, s)) ||
            (st = dalloc(&keys, (size_t)n, s)) || (st = dalloc(&set_of, (size_t)n, s)) ||
            (st = dalloc(&order, (size_t)n, s)))
            goto done;
        HMG_CUDA_TRY(cudaMemcpyAsync(doff[w], off[w], sizeof(int) * (nsets + 1), cudaMemcpyHostToDevice, s));
        // ---- every set's Morton codes, then its points in code order (hmglib.cu:128-162) ----
        k_minmax_sets<<<nsets, 256, 0, s>>>(g->pts[w], n, doff[w], dsdim, mm);
        HMG_LAUNCH_CHECK();
        k_morton_sets<<<ceil_div(n, 256), 256, 0, s>>>(g->pts[w], n, doff[w], nsets, dsdim, dsbits, mm,
                                                       g->codes[w], set_of);
        HMG_LAUNCH_CHECK();
        // stable by code, then stable by set: each set in its own stable code order
        HMG_CUDA_TRY(cudaMemcpyAsync(keys, g->codes[w], sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
        k_iota<<<ceil_div(n, 256), 256, 0, s>>>(order, n);
        HMG_LAUNCH_CHECK();
        if ((st = radix_sort_pairs(keys, order, n, code_bits, s))) goto done;
        k_gather_u64<<<ceil_div(n, 256), 256, 0, s>>>(set_of, order, n, keys);
        HMG_LAUNCH_CHECK();
        if ((st = radix_sort_pairs(keys, order, n, set_bits, s))) goto done;
        k_gather_u64<<<ceil_div(n, 256), 256, 0, s>>>(g->codes[w], order, n, keys);
        HMG_LAUNCH_CHECK();
        HMG_CUDA_TRY(cudaMemcpyAsync(g->codes[w], keys, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
        k_gather_points<<<ceil_div(n, 256), 256, 0, s>>>(g->pts[w], g->zpts[w], order, n, g->dim,
                                                         g->perm[w], g->iperm[w]);
        HMG_LAUNCH_CHECK();
        k_leaf_at<<<ceil_div(n, 256), 256, 0, s>>>(doff[w], nsets, dsleaf, n, leaf_at[w]);
        HMG_LAUNCH_CHECK();
        dfree(keys, s);
        dfree(set_of, s);
        dfree(order, s);
        rl[w].resize(nsets);
        ru[w].resize(nsets);
        for (int i = 0; i < nsets; i++) {
            rl[w][i] = off[w][i];
            ru[w][i] = off[w][i + 1] - 1;
        }
    }
    // ---- one traversal from every set's root pair, then the blocks -----------------
    {
        const int* la[2] = {leaf_at[0], leaf_at[1]};
        st = traverse(g, nsets, rl[0].data(), ru[0].data(), rl[1].data(), ru[1].data(), la, leaves, nleaves,
                      levels);
    }
    if (!st) st = partition_blocks(g, leaves, nleaves, levels, doff[0], nsets);

done:
    free_leaves(leaves, s);
    dfree(doff[0], s); dfree(doff[1], s);
    dfree(dsdim, s); dfree(dsbits, s); dfree(dsleaf, s);
    dfree(leaf_at[0], s); dfree(leaf_at[1], s);
    dfree(mm, s);
    dfree(keys, s); dfree(set_of, s); dfree(order, s);
    return st;
}

// ---------------------------------------------------------------------------
// row tiles and the (tile, block) pair lists of the matvec
// ---------------------------------------------------------------------------
__global__ void k_mark_bounds(const int* r0, const int* m1, int nb, int* mark)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    mark[r0[b]] = 1;
    mark[r0[b] + m1[b]] = 1;
}

__global__ void k_piece_starts(const int* mark, const int* scanned, int n, int* piece_start)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && mark[i]) piece_start[scanned[i]] = i;
}

__global__ void k_piece_tiles(const int* piece_start, int np, int n, int* cnt)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    int len = (k + 1 < np ? piece_start[k + 1] : n) - piece_start[k];
    cnt[k] = (len + HMG_TILE_ROWS - 1) / HMG_TILE_ROWS;
}

__global__ void k_emit_tiles(const int* piece_start, int np, int n, const int* toff,
                             int* tile_r0, int* tile_s, int* tile_spad)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    int st = piece_start[k];
    int len = (k + 1 < np ? piece_start[k + 1] : n) - st;
    int nt = (len + HMG_TILE_ROWS - 1) / HMG_TILE_ROWS;
    int base = len / nt, rem = len % nt;
    int r = st;
    for (int j = 0; j < nt; j++) {
        int sz = base + (j < rem ? 1 : 0);
        tile_r0[toff[k] + j] = r;
        tile_s[toff[k] + j] = sz;
        tile_spad[toff[k] + j] = (sz + 3) & ~3;
        r += sz;
    }
}

__global__ void k_tile_of_row(const int* tile_r0, const int* tile_s, int nt, int* tor)
{
    int t = blockIdx.x;
    if (t >= nt) return;
    for (int i = threadIdx.x; i < tile_s[t]; i += blockDim.x) tor[tile_r0[t] + i] = t;
}

__global__ void k_block_tiles(const int* r0, const int* m1, int nb, const int* tor, int* tf,
                              int* tl, int* cnt)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int a = tor[r0[b]], z = tor[r0[b] + m1[b] - 1];
    tf[b] = a;
    tl[b] = z;
    cnt[b] = z - a + 1;
}

__global__ void k_pair_keys(const int* tf, const int* tl, int nb, const int* off,
                            uint64_t* keys, uint32_t* vals, int* tile_cnt)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int o = off[b];
    for (int t = tf[b]; t <= tl[b]; t++, o++) {
        keys[o] = (uint64_t)t * (uint64_t)nb + (uint64_t)b;
        vals[o] = (uint32_t)b;
        atomicAdd(&tile_cnt[t], 1);
    }
}

hmg_status build_tiles(hmg_matrix* h)
{
    cudaStream_t s = h->stream;
    hmg_status st = HMG_OK;
    int n = h->n[0], nb = h->nblocks;
    int *mark = nullptr, *scanned = nullptr, *pstart = nullptr, *pcnt = nullptr, *tot = nullptr;
    int *tor = nullptr, *spad = nullptr, *bcnt = nullptr, *tcnt = nullptr;
    uint64_t* keys = nullptr;
    uint32_t* vals = nullptr;
    int np = 0, nt = 0, npairs = 0;
    if ((st = dalloc(&mark, (size_t)n + 1, s)) || (st = dalloc(&scanned, (size_t)n + 1, s)) ||
        (st = dalloc(&tot, 1, s)))
        goto done;
    HMG_CUDA_TRY(cudaMemsetAsync(mark, 0, sizeof(int) * (n + 1), s));
    k_mark_bounds<<<ceil_div(nb, 256), 256, 0, s>>>(h->blk_r0, h->blk_m1, nb, mark);
    HMG_LAUNCH_CHECK();
    if ((st = scan_exclusive<int>(mark, scanned, n, tot, s))) goto done;
    HMG_CUDA_TRY(cudaMemcpyAsync(&np, tot, sizeof(int), cudaMemcpyDeviceToHost, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    if ((st = dalloc(&pstart, (size_t)np, s)) || (st = dalloc(&pcnt, (size_t)np, s))) goto done;
    k_piece_starts<<<ceil_div(n, 256), 256, 0, s>>>(mark, scanned, n, pstart);
    HMG_LAUNCH_CHECK();
    k_piece_tiles<<<ceil_div(np, 256), 256, 0, s>>>(pstart, np, n, pcnt);
    HMG_LAUNCH_CHECK();
    if ((st = scan_exclusive<int>(pcnt, pcnt, np, tot, s))) goto done;
    HMG_CUDA_TRY(cudaMemcpyAsync(&nt, tot, sizeof(int), cudaMemcpyDeviceToHost, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    h->ntiles = nt;
    if ((st = dalloc(&h->tile_r0, (size_t)nt, s)) || (st = dalloc(&h->tile_s, (size_t)nt, s)) ||
        (st = dalloc(&h->tile_pstart, (size_t)nt + 1, s)) || (st = dalloc(&spad, (size_t)nt + 1, s)) ||
        (st = dalloc(&tor, (size_t)n, s)))
        goto done;
    k_emit_tiles<<<ceil_div(np, 256), 256, 0, s>>>(pstart, np, n, pcnt, h->tile_r0, h->tile_s, spad);
    HMG_LAUNCH_CHECK();
    HMG_CUDA_TRY(cudaMemsetAsync(spad + nt, 0, sizeof(int), s));
    if ((st = scan_exclusive<int>(spad, h->tile_pstart, nt + 1, nullptr, s))) goto done;
    k_tile_of_row<<<nt, 128, 0, s>>>(h->tile_r0, h->tile_s, nt, tor);
    HMG_LAUNCH_CHECK();

    if ((st = dalloc(&h->blk_tfirst, (size_t)nb, s)) || (st = dalloc(&h->blk_tlast, (size_t)nb, s)) ||
        (st = dalloc(&bcnt, (size_t)nb, s)) || (st = dalloc(&tcnt, (size_t)nt + 1, s)) ||
        (st = dalloc(&h->tile_pair_start, (size_t)nt + 1, s)))
        goto done;
    k_block_tiles<<<ceil_div(nb, 256), 256, 0, s>>>(h->blk_r0, h->blk_m1, nb, tor, h->blk_tfirst,
                                                    h->blk_tlast, bcnt);
    HMG_LAUNCH_CHECK();
    if ((st = scan_exclusive<int>(bcnt, bcnt, nb, tot, s))) goto done;
    HMG_CUDA_TRY(cudaMemcpyAsync(&npairs, tot, sizeof(int), cudaMemcpyDeviceToHost, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    h->npairs = npairs;
    if ((st = dalloc(&keys, (size_t)npairs, s)) || (st = dalloc(&vals, (size_t)npairs, s)))
        goto done;
    HMG_CUDA_TRY(cudaMemsetAsync(tcnt, 0, sizeof(int) * (nt + 1), s));
    k_pair_keys<<<ceil_div(nb, 256), 256, 0, s>>>(h->blk_tfirst, h->blk_tlast, nb, bcnt, keys,
                                                  vals, tcnt);
    HMG_LAUNCH_CHECK();
    {
        unsigned long long maxkey = (unsigned long long)nt * (unsigned long long)nb;
        int kb = 1;
        while (kb < 64 && (1ull << kb) <= maxkey) kb++;
        if ((st = radix_sort_pairs(keys, vals, npairs, kb, s))) goto done;
    }
    if ((st = scan_exclusive<int>(tcnt, h->tile_pair_start, nt + 1, nullptr, s))) goto done;
    h->pair_block = (int*)vals;
    vals = nullptr;
    h->h_tile_pstart.resize(nt + 1);
    h->h_blk_tfirst.resize(nb);
    h->h_blk_tlast.resize(nb);
    HMG_CUDA_TRY(cudaMemcpyAsync(h->h_tile_pstart.data(), h->tile_pstart, sizeof(int) * (nt + 1), cudaMemcpyDeviceToHost, s));
    if (nb) {
        HMG_CUDA_TRY(cudaMemcpyAsync(h->h_blk_tfirst.data(), h->blk_tfirst, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->h_blk_tlast.data(), h->blk_tlast, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
    }
    HMG_CUDA_TRY(cudaStreamSynchronize(s));

done:
    dfree(mark, s); dfree(scanned, s); dfree(pstart, s); dfree(pcnt, s); dfree(tot, s);
    dfree(tor, s); dfree(spad, s); dfree(bcnt, s); dfree(tcnt, s); dfree(keys, s); dfree(vals, s);
    return st;
}

}  // namespace hmg
