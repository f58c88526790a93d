// io.cu -- an H-matrix on disk (hmg_save / hmg_load).
//
// The reference has no serialisation; it can print the work-item tree for debugging
// (tree.cu:173-183).  Here a compressed H-matrix is written once and loaded by later
// runs without repeating the tree build and the compression: the points, the
// permutations, the block list, the ranks and storage tiers, the factor allocations
// byte for byte and the stored near field.  Row tiles and product descriptors are
// rebuilt on load (they are a deterministic function of the block list), so a loaded
// H-matrix multiplies bit-identically to the one saved.
//
// Format (little endian, native struct layouts of this library; version 1):
//   "HMGB200\0", u32 version, u32 header bytes, the Header struct, then sections in
//   order: points, blocks, [group parameters], [far field], [near field].  Each
//   array is written as its raw bytes; lengths follow from the header.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "hmg_matrix.cuh"

namespace hmg {

namespace {

struct Header {
    int n1, n2, dim, bits;
    double eta;
    int c_leaf, max_level, rule, levels;
    int nblocks, ndense;
    int kernel_set;
    KernelSpec kspec;
    int group_count;
    int far_prec;       // -1: not compressed
    int aca_k;
    double aca_eps;
    int near_prec;      // -1: not stored
    int near_mode;
    long long far_entries, far_rows, far_stored, far_alg_u, far_alg_v, rank_total;
    int max_rank;
    int nchunks;
    long long near_entries, near_stored;
};

constexpr char MAGIC[8] = {'H', 'M', 'G', 'B', '2', '0', '0', '\0'};
constexpr unsigned VERSION = 1;

struct File {
    FILE* f = nullptr;
    ~File()
    {
        if (f) fclose(f);
    }
};

bool put(FILE* f, const void* p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }
bool get(FILE* f, void* p, size_t n) { return n == 0 || fread(p, 1, n, f) == n; }

// device -> file through a bounded host buffer
hmg_status put_dev(FILE* f, const void* d, size_t n, cudaStream_t s)
{
    std::vector<char> buf(std::min(n, (size_t)(64u << 20)));
    for (size_t o = 0; o < n; o += buf.size()) {
        const size_t k = std::min(buf.size(), n - o);
        HMG_CUDA_TRY(cudaMemcpyAsync(buf.data(), static_cast<const char*>(d) + o, k, cudaMemcpyDeviceToHost, s));
        HMG_CUDA_TRY(cudaStreamSynchronize(s));
        if (!put(f, buf.data(), k)) {
            set_error("hmg_save: write failed");
            return HMG_ERR_INVALID;
        }
    }
    return HMG_OK;
}

hmg_status get_dev(FILE* f, void* d, size_t n, cudaStream_t s)
{
    std::vector<char> buf(std::min(n, (size_t)(64u << 20)));
    for (size_t o = 0; o < n; o += buf.size()) {
        const size_t k = std::min(buf.size(), n - o);
        if (!get(f, buf.data(), k)) {
            set_error("hmg_load: file truncated");
            return HMG_ERR_INVALID;
        }
        HMG_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(d) + o, buf.data(), k, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return HMG_OK;
}

}  // namespace

hmg_status save(hmg_matrix* h, const char* path)
{
    cudaStream_t s = h->stream;
    hmg_status st;
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    File fh;
    fh.f = fopen(path, "wb");
    if (!fh.f) {
        set_error("hmg_save: cannot open %s for writing", path);
        return HMG_ERR_INVALID;
    }
    FILE* f = fh.f;
    Header H{};
    H.n1 = h->n[0]; H.n2 = h->n[1]; H.dim = h->dim; H.bits = h->bits;
    H.eta = h->eta; H.c_leaf = h->c_leaf; H.max_level = h->max_level; H.rule = h->rule; H.levels = h->levels;
    H.nblocks = h->nblocks; H.ndense = h->ndense;
    H.kernel_set = h->kernel_set ? 1 : 0;
    H.kspec = h->kspec;
    H.group_count = h->group_count;
    H.far_prec = h->far_prec; H.aca_k = h->aca_k; H.aca_eps = h->aca_eps;
    H.near_prec = h->near_prec; H.near_mode = h->near_mode;
    H.far_entries = h->far_entries; H.far_rows = h->far_rows; H.far_stored = h->far_stored;
    H.far_alg_u = h->far_alg_u; H.far_alg_v = h->far_alg_v; H.rank_total = h->rank_total;
    H.max_rank = h->max_rank;
    H.nchunks = (int)h->far_chunks.size();
    H.near_entries = h->near_entries; H.near_stored = h->near_stored;
    const unsigned hb = sizeof(Header);
    if (!put(f, MAGIC, 8) || !put(f, &VERSION, 4) || !put(f, &hb, 4) || !put(f, &H, sizeof H)) {
        set_error("hmg_save: write failed");
        return HMG_ERR_INVALID;
    }
    // points
    for (int w = 0; w < 2; w++) {
        const size_t n = (size_t)h->n[w];
        if ((st = put_dev(f, h->pts[w], n * h->dim * 8, s)) || (st = put_dev(f, h->zpts[w], n * h->dim * 8, s)) ||
            (st = put_dev(f, h->codes[w], n * 8, s)) || (st = put_dev(f, h->perm[w], n * 4, s)) ||
            (st = put_dev(f, h->iperm[w], n * 4, s)))
            return st;
    }
    // blocks
    const size_t nb = (size_t)h->nblocks;
    if (!put(f, h->h_r0.data(), nb * 4) || !put(f, h->h_m1.data(), nb * 4) || !put(f, h->h_c0.data(), nb * 4) ||
        !put(f, h->h_m2.data(), nb * 4) || !put(f, h->h_type.data(), nb * 4)) {
        set_error("hmg_save: write failed");
        return HMG_ERR_INVALID;
    }
    if (h->group_count) {
        for (int w = 0; w < 2; w++)
            if (!put(f, h->group_off[w].data(), sizeof(int) * (h->group_count + 1))) {
                set_error("hmg_save: write failed");
                return HMG_ERR_INVALID;
            }
        if ((st = put_dev(f, h->blk_param, nb * 8, s))) return st;
    }
    // far field: ranks, tiers, the allocations and each block's place in them
    if (h->far_prec >= 0) {
        std::vector<void*> pu(nb, nullptr), pv(nb, nullptr);
        if (nb > 0) {
            HMG_CUDA_TRY(cudaMemcpy(pu.data(), h->ptrU, sizeof(void*) * nb, cudaMemcpyDeviceToHost));
            HMG_CUDA_TRY(cudaMemcpy(pv.data(), h->ptrV, sizeof(void*) * nb, cudaMemcpyDeviceToHost));
        }
        std::vector<long long> place(3 * nb, -1);  // chunk, offset of U, offset of V
        for (size_t b = (size_t)h->ndense; b < nb; b++) {
            if (h->h_rank[b] == 0) continue;
            for (size_t c = 0; c < h->far_chunks.size(); c++) {
                const char* base = static_cast<const char*>(h->far_chunks[c]);
                const char* u = static_cast<const char*>(pu[b]);
                if (u >= base && u < base + h->far_chunk_bytes[c]) {
                    place[3 * b] = (long long)c;
                    place[3 * b + 1] = u - base;
                    place[3 * b + 2] = static_cast<const char*>(pv[b]) - base;
                    break;
                }
            }
            if (place[3 * b] < 0) {
                set_error("hmg_save: block %zu's factors lie outside the factor allocations", b);
                return HMG_ERR_STATE;
            }
        }
        if (!put(f, h->h_rank.data(), nb * 4) || !put(f, h->h_r32.data(), nb * 4) ||
            !put(f, h->h_r16.data(), nb * 4) || !put(f, h->far_chunk_bytes.data(), 8 * h->far_chunk_bytes.size()) ||
            !put(f, place.data(), 8 * place.size())) {
            set_error("hmg_save: write failed");
            return HMG_ERR_INVALID;
        }
        for (size_t c = 0; c < h->far_chunks.size(); c++)
            if ((st = put_dev(f, h->far_chunks[c], h->far_chunk_bytes[c], s))) return st;
    }
    // near field
    if (h->near_prec >= 0) {
        const size_t esz = h->near_prec == HMG_PREC_FP64 ? 8 : 4;
        if ((st = put_dev(f, h->near_off, sizeof(long long) * (size_t)h->ndense, s)) ||
            (st = put_dev(f, h->near_data, (size_t)h->near_stored * esz, s)))
            return st;
    }
    if (fflush(f) != 0) {
        set_error("hmg_save: write failed");
        return HMG_ERR_INVALID;
    }
    return HMG_OK;
}

namespace {

// What hmg_load found in a file: the small arrays (checked on the host before any
// device work) and the file offsets of the large sections (copied to the device
// afterwards).
struct Plan {
    long long points_at[2] = {0, 0};  // pts, zpts, codes of each set (perm/iperm below)
    std::vector<int> perm[2], iperm[2];
    std::vector<int> r0, m1, c0, m2, type;
    std::vector<int> goff[2];
    long long param_at = -1;
    std::vector<int> rank, r32, r16;
    std::vector<size_t> cb;
    std::vector<long long> place;
    long long chunks_at = -1;
    std::vector<long long> near_off;
    long long near_at = -1;
    std::vector<long long> rows_p;  // padded tile rows of each block (the stored slice height)
};

struct Reader {
    FILE* f;
    long long size;
    long long pos() const { return ftello(f); }
    bool left(long long bytes) const { return bytes >= 0 && pos() >= 0 && bytes <= size - pos(); }
    bool skip(long long bytes) { return left(bytes) && fseeko(f, bytes, SEEK_CUR) == 0; }
    template <typename T>
    bool read(std::vector<T>& v, long long count)
    {
        if (count < 0 || !left(count * (long long)sizeof(T))) return false;
        v.resize((size_t)count);
        return get(f, v.data(), (size_t)count * sizeof(T));
    }
};

#define HMG_LOAD_CHECK(cond, ...)                     \
    do {                                              \
        if (!(cond)) {                                \
            set_error("hmg_load: " __VA_ARGS__);      \
            return HMG_ERR_INVALID;                   \
        }                                             \
    } while (0)

// Padded rows of every block's U / near slices, from the block list alone.  Row
// tiles are the pieces between consecutive block row bounds, each cut into
// ceil(len / HMG_TILE_ROWS) near-equal tiles whose rows are padded to 4; a block
// spans exactly the pieces inside its row range (the tiles build_tiles makes).
static void padded_rows(int n, const Plan& P, std::vector<long long>& rows_p)
{
    const size_t nb = P.r0.size();
    std::vector<char> mark((size_t)n + 1, 0);
    for (size_t b = 0; b < nb; b++) {
        mark[(size_t)P.r0[b]] = 1;
        mark[(size_t)P.r0[b] + P.m1[b]] = 1;
    }
    // acc[i] = padded rows of all tiles of the pieces that start before row i
    // (defined at piece bounds)
    std::vector<long long> acc((size_t)n + 1, 0);
    long long run = 0;
    int start = -1;
    for (int i = 0; i <= n; i++) {
        if (i == n || mark[(size_t)i]) {
            if (start >= 0) {
                const int len = i - start, nt = (len + HMG_TILE_ROWS - 1) / HMG_TILE_ROWS;
                const int base = len / nt, rem = len % nt;
                for (int j = 0; j < nt; j++) run += round_up4(base + (j < rem ? 1 : 0));
            }
            acc[(size_t)i] = run;
            start = i;
        }
    }
    rows_p.assign(nb, 0);
    for (size_t b = 0; b < nb; b++) rows_p[b] = acc[(size_t)P.r0[b] + P.m1[b]] - acc[(size_t)P.r0[b]];
}

// Reads every section's metadata and checks it before anything reaches the
// device: counts, the permutations, every block range, the group offsets, ranks
// and storage tiers, and each block's factor and near-field slices against their
// allocations.  Large sections are only skipped (their lengths must be present).
static hmg_status check_file(Reader& R, const Header& H, Plan& P)
{
    HMG_LOAD_CHECK(H.n1 >= 1 && H.n2 >= 1, "point counts %d, %d must be >= 1", H.n1, H.n2);
    HMG_LOAD_CHECK(H.dim == 2 || H.dim == 3, "dimension %d", H.dim);
    HMG_LOAD_CHECK(H.bits >= 1 && H.bits * H.dim <= 64, "Morton bits %d", H.bits);
    HMG_LOAD_CHECK(H.nblocks >= 0 && H.ndense >= 0 && H.ndense <= H.nblocks, "block counts %d / %d dense",
                   H.nblocks, H.ndense);
    HMG_LOAD_CHECK((long long)H.nblocks <= (long long)H.n1 * H.n2, "%d blocks for %d x %d points", H.nblocks, H.n1,
                   H.n2);
    HMG_LOAD_CHECK(H.c_leaf >= 1 && (H.rule == 0 || H.rule == 1) && std::isfinite(H.eta), "tree parameters");
    HMG_LOAD_CHECK(H.group_count >= 0 && H.group_count <= std::min(H.n1, H.n2), "group count %d", H.group_count);
    HMG_LOAD_CHECK(H.far_prec >= -1 && H.far_prec <= HMG_PREC_MIXED, "factor precision %d", H.far_prec);
    HMG_LOAD_CHECK(H.near_prec >= -1 && H.near_prec <= HMG_PREC_FP32, "near-field precision %d", H.near_prec);
    HMG_LOAD_CHECK(H.near_mode == HMG_NEAR_STORED || H.near_mode == HMG_NEAR_ONTHEFLY, "near-field mode %d",
                   H.near_mode);
    HMG_LOAD_CHECK(H.near_mode != HMG_NEAR_STORED || H.near_prec >= 0, "stored near-field mode without a near field");
    HMG_LOAD_CHECK(!H.kernel_set || (H.kspec.kind >= HMG_KERNEL_GAUSSIAN_REF && H.kspec.kind <= HMG_KERNEL_MATERN32 &&
                                     H.kspec.dim == H.dim),
                   "kernel kind %d / dimension %d", H.kspec.kind, H.kspec.dim);
    const int n[2] = {H.n1, H.n2};
    for (int w = 0; w < 2; w++) {
        P.points_at[w] = R.pos();
        HMG_LOAD_CHECK(R.skip((long long)n[w] * H.dim * 16 + (long long)n[w] * 8), "file truncated (points)");
        HMG_LOAD_CHECK(R.read(P.perm[w], n[w]) && R.read(P.iperm[w], n[w]), "file truncated (permutations)");
        for (int i = 0; i < n[w]; i++) {
            const int p = P.perm[w][(size_t)i];
            HMG_LOAD_CHECK(p >= 0 && p < n[w] && P.iperm[w][(size_t)p] == i,
                           "set %d: the permutation and its inverse disagree at point %d", w, i);
        }
    }
    const long long nb = H.nblocks;
    HMG_LOAD_CHECK(R.read(P.r0, nb) && R.read(P.m1, nb) && R.read(P.c0, nb) && R.read(P.m2, nb) &&
                       R.read(P.type, nb),
                   "file truncated (blocks)");
    for (long long b = 0; b < nb; b++) {
        const long long r0 = P.r0[b], m1 = P.m1[b], c0 = P.c0[b], m2 = P.m2[b];
        HMG_LOAD_CHECK(r0 >= 0 && m1 >= 1 && r0 + m1 <= H.n1 && c0 >= 0 && m2 >= 1 && c0 + m2 <= H.n2,
                       "block %lld: rows [%lld, %lld) / columns [%lld, %lld) outside the %d x %d matrix", b, r0,
                       r0 + m1, c0, c0 + m2, H.n1, H.n2);
        HMG_LOAD_CHECK(P.type[b] == (b < H.ndense ? HMG_WT_DENSE : HMG_WT_ACA),
                       "block %lld has type %d; dense blocks come first", b, P.type[b]);
    }
    if (H.group_count) {
        for (int w = 0; w < 2; w++) {
            HMG_LOAD_CHECK(R.read(P.goff[w], H.group_count + 1), "file truncated (group offsets)");
            HMG_LOAD_CHECK(P.goff[w][0] == 0 && P.goff[w][(size_t)H.group_count] == n[w], "group offsets of set %d",
                           w);
            for (int g = 0; g < H.group_count; g++)
                HMG_LOAD_CHECK(P.goff[w][(size_t)g] <= P.goff[w][(size_t)g + 1], "group offsets of set %d", w);
        }
        P.param_at = R.pos();
        HMG_LOAD_CHECK(R.skip(nb * 8), "file truncated (kernel parameters)");
    }
    padded_rows(H.n1, P, P.rows_p);
    if (H.far_prec >= 0) {
        HMG_LOAD_CHECK(H.nchunks >= 0 && H.nchunks <= H.nblocks, "%d factor allocations for %d blocks", H.nchunks,
                       H.nblocks);
        HMG_LOAD_CHECK(R.read(P.rank, nb) && R.read(P.r32, nb) && R.read(P.r16, nb) && R.read(P.cb, H.nchunks) &&
                           R.read(P.place, 3 * nb),
                       "file truncated (ranks)");
        long long total = 0;
        for (size_t c = 0; c < P.cb.size(); c++) {
            HMG_LOAD_CHECK(P.cb[c] > 0 && P.cb[c] <= ((size_t)1 << 42), "factor allocation %zu of %zu bytes", c, P.cb[c]);
            total += (long long)P.cb[c];
        }
        P.chunks_at = R.pos();
        HMG_LOAD_CHECK(R.skip(total), "file truncated (factors: %lld bytes)", total);
        const bool mixed = H.far_prec == HMG_PREC_MIXED;
        const long long esz = H.far_prec == HMG_PREC_FP64 ? 8 : 4;
        for (long long b = 0; b < nb; b++) {
            const int r = P.rank[b], r32 = P.r32[b], r16 = P.r16[b], r8 = r - r32 - r16;
            const long long m1 = P.m1[b], m2 = P.m2[b];
            HMG_LOAD_CHECK(r >= 0 && r <= 512 && r <= m1 && r <= m2 && (b >= H.ndense || r == 0),
                           "block %lld: rank %d", b, r);
            if (mixed)
                HMG_LOAD_CHECK(r32 >= 0 && r16 >= 0 && r8 >= 0 && r16 % 2 == 0 && r8 % 4 == 0,
                               "block %lld: storage tiers %d / %d / %d of rank %d", b, r32, r16, r8, r);
            else
                HMG_LOAD_CHECK(r32 == r && r16 == 0, "block %lld: storage tiers %d / %d of rank %d", b, r32, r16, r);
            if (r == 0) continue;
            const long long chunk = P.place[3 * b], ou = P.place[3 * b + 1], ov = P.place[3 * b + 2];
            HMG_LOAD_CHECK(chunk >= 0 && chunk < H.nchunks, "block %lld names factor allocation %lld of %d", b,
                           chunk, H.nchunks);
            const long long bpr = mixed ? 4ll * r32 + 2ll * r16 + r8 : r * esz;  // bytes per slice row
            const long long ub = P.rows_p[b] * bpr;
            const long long vb = ((m2 + 3) & ~3ll) * bpr + (mixed ? 4ll * r : 0);
            const long long cap = (long long)P.cb[(size_t)chunk];
            HMG_LOAD_CHECK(ou >= 0 && ov >= 0 && ou % 16 == 0 && ov % 16 == 0 && ou <= cap - ub && ov <= cap - vb,
                           "block %lld: factors at %lld (+%lld) and %lld (+%lld) outside their %lld-byte allocation",
                           b, ou, ub, ov, vb, cap);
        }
    }
    if (H.near_prec >= 0) {
        const long long esz = H.near_prec == HMG_PREC_FP64 ? 8 : 4;
        HMG_LOAD_CHECK(H.near_stored >= 0, "near field of %lld entries", H.near_stored);
        HMG_LOAD_CHECK(R.read(P.near_off, H.ndense), "file truncated (near-field offsets)");
        for (long long b = 0; b < H.ndense; b++) {
            const long long o = P.near_off[b], len = P.rows_p[b] * P.m2[b];
            HMG_LOAD_CHECK(o >= 0 && o % 4 == 0 && o <= H.near_stored - len,
                           "dense block %lld: slice at %lld (+%lld) outside the %lld-entry near field", b, o, len,
                           H.near_stored);
        }
        P.near_at = R.pos();
        HMG_LOAD_CHECK(H.near_stored <= (1ll << 42) && R.skip(H.near_stored * esz), "file truncated (near field)");
    }
    return HMG_OK;
}

// Copies a checked file into a new handle.  On failure the caller destroys `h`.
static hmg_status upload(hmg_matrix* h, Reader& R, const Header& H, const Plan& P, cudaStream_t s)
{
    hmg_status st;
    FILE* f = R.f;
    for (int w = 0; w < 2; w++) {
        const size_t n = (size_t)h->n[w];
        if (fseeko(f, P.points_at[w], SEEK_SET) != 0) {
            set_error("hmg_load: seek failed");
            return HMG_ERR_INVALID;
        }
        if ((st = get_dev(f, h->pts[w], n * h->dim * 8, s)) || (st = get_dev(f, h->zpts[w], n * h->dim * 8, s)) ||
            (st = get_dev(f, h->codes[w], n * 8, s)))
            return st;
        HMG_CUDA_TRY(cudaMemcpy(h->perm[w], P.perm[w].data(), n * 4, cudaMemcpyHostToDevice));
        HMG_CUDA_TRY(cudaMemcpy(h->iperm[w], P.iperm[w].data(), n * 4, cudaMemcpyHostToDevice));
        h->points_set[w] = true;
    }
    const size_t nb = (size_t)H.nblocks;
    h->h_r0 = P.r0; h->h_m1 = P.m1; h->h_c0 = P.c0; h->h_m2 = P.m2; h->h_type = P.type;
    h->eta = H.eta; h->c_leaf = H.c_leaf; h->max_level = H.max_level; h->rule = H.rule; h->levels = H.levels;
    h->nblocks = H.nblocks; h->ndense = H.ndense; h->naca = H.nblocks - H.ndense;
    if ((st = dalloc(&h->blk_r0, nb, s)) || (st = dalloc(&h->blk_m1, nb, s)) || (st = dalloc(&h->blk_c0, nb, s)) ||
        (st = dalloc(&h->blk_m2, nb, s)) || (st = dalloc(&h->blk_type, nb, s)))
        return st;
    if (nb > 0) {
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_r0, h->h_r0.data(), nb * 4, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_m1, h->h_m1.data(), nb * 4, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_c0, h->h_c0.data(), nb * 4, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_m2, h->h_m2.data(), nb * 4, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_type, h->h_type.data(), nb * 4, cudaMemcpyHostToDevice, s));
    }
    if (H.group_count) {
        h->group_count = H.group_count;
        h->group_off[0] = P.goff[0];
        h->group_off[1] = P.goff[1];
        if (fseeko(f, P.param_at, SEEK_SET) != 0) {
            set_error("hmg_load: seek failed");
            return HMG_ERR_INVALID;
        }
        if ((st = dalloc(&h->blk_param, nb, s)) || (st = get_dev(f, h->blk_param, nb * 8, s))) return st;
    }
    if ((st = build_tiles(h))) return st;
    // the slices were checked against the host's tile rows; the device's must agree
    for (size_t b = 0; b < nb; b++)
        if (h->h_tile_pstart[(size_t)h->h_blk_tlast[b] + 1] - h->h_tile_pstart[(size_t)h->h_blk_tfirst[b]] !=
            P.rows_p[b]) {
            set_error("hmg_load: block %zu's tile rows differ from the file's layout", b);
            return HMG_ERR_INVALID;
        }
    h->setup_done = true;
    h->kspec = H.kspec;
    h->kernel_set = H.kernel_set != 0;
    if (H.far_prec >= 0) {
        if (fseeko(f, P.chunks_at, SEEK_SET) != 0) {
            set_error("hmg_load: seek failed");
            return HMG_ERR_INVALID;
        }
        for (size_t c = 0; c < P.cb.size(); c++) {
            void* p = nullptr;
            cudaError_t ce = cudaMalloc(&p, P.cb[c]);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                set_error("hmg_load: allocating %zu bytes of factors failed: %s", P.cb[c], cudaGetErrorString(ce));
                return ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
            }
            h->far_chunks.push_back(p);
            h->far_chunk_bytes.push_back(P.cb[c]);
            if ((st = get_dev(f, p, P.cb[c], s))) return st;
        }
        const bool mixed = H.far_prec == HMG_PREC_MIXED;
        const long long esz = H.far_prec == HMG_PREC_FP64 ? 8 : 4;
        std::vector<void*> pu(nb, nullptr), pv(nb, nullptr);
        std::vector<long long> roff(nb + 1, 0);
        long long far_entries = 0, far_rows = 0, alg_u = 0, alg_v = 0, stored = 0;
        int max_rank = 0;
        for (size_t c = 0; c < P.cb.size(); c++) stored += (long long)P.cb[c];
        for (size_t b = 0; b < nb; b++) {
            const int r = P.rank[b];
            roff[b + 1] = roff[b] + r;
            if (b >= (size_t)H.ndense) {
                const long long m1 = P.m1[b], m2 = P.m2[b];
                const long long bpe = mixed ? 4ll * P.r32[b] + 2ll * P.r16[b] + (r - P.r32[b] - P.r16[b]) : r * esz;
                far_entries += (m1 + m2) * r;
                far_rows += m1 + m2;
                alg_u += m1 * bpe;
                alg_v += m2 * bpe;
                max_rank = std::max(max_rank, r);
            }
            if (r > 0) {
                char* base = static_cast<char*>(h->far_chunks[(size_t)P.place[3 * b]]);
                pu[b] = base + P.place[3 * b + 1];
                pv[b] = base + P.place[3 * b + 2];
            }
        }
        if ((st = dalloc(&h->rank, nb, s)) || (st = dalloc(&h->rank_off, nb + 1, s)) ||
            (st = dalloc(&h->ptrU, nb, s)) || (st = dalloc(&h->ptrV, nb, s)) || (st = dalloc(&h->tier32, nb, s)) ||
            (st = dalloc(&h->tier16, nb, s)))
            return st;
        if (nb > 0) {
            HMG_CUDA_TRY(cudaMemcpyAsync(h->rank, P.rank.data(), nb * 4, cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->tier32, P.r32.data(), nb * 4, cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->tier16, P.r16.data(), nb * 4, cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->ptrU, pu.data(), nb * sizeof(void*), cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->ptrV, pv.data(), nb * sizeof(void*), cudaMemcpyHostToDevice, s));
        }
        HMG_CUDA_TRY(cudaMemcpyAsync(h->rank_off, roff.data(), (nb + 1) * 8, cudaMemcpyHostToDevice, s));
        h->rank_total = roff[nb];
        if ((st = dalloc((char**)&h->tbuf, (size_t)(h->rank_total + 32) * 8, s))) return st;
        HMG_CUDA_TRY(cudaMemsetAsync(h->tbuf, 0, (size_t)(h->rank_total + 32) * 8, s));
        h->h_rank = P.rank;
        h->h_r32 = P.r32;
        h->h_r16 = P.r16;
        h->far_prec = H.far_prec; h->aca_k = H.aca_k; h->aca_eps = H.aca_eps;
        h->far_entries = far_entries; h->far_rows = far_rows; h->far_stored = stored;
        h->far_alg_u = alg_u; h->far_alg_v = alg_v; h->max_rank = max_rank;
    }
    if (H.near_prec >= 0 && H.ndense > 0) {
        const size_t esz = H.near_prec == HMG_PREC_FP64 ? 8 : 4;
        if ((st = dalloc(&h->near_off, (size_t)H.ndense, s))) return st;
        HMG_CUDA_TRY(cudaMemcpyAsync(h->near_off, P.near_off.data(), sizeof(long long) * (size_t)H.ndense,
                                     cudaMemcpyHostToDevice, s));
        cudaError_t ce = cudaMalloc(&h->near_data, (size_t)H.near_stored * esz);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            h->near_data = nullptr;
            set_error("hmg_load: allocating the near field failed: %s", cudaGetErrorString(ce));
            return ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
        }
        if (fseeko(f, P.near_at, SEEK_SET) != 0) {
            set_error("hmg_load: seek failed");
            return HMG_ERR_INVALID;
        }
        if ((st = get_dev(f, h->near_data, (size_t)H.near_stored * esz, s))) return st;
    }
    if (H.near_prec >= 0) {
        long long entries = 0;
        for (int b = 0; b < H.ndense; b++) entries += (long long)P.m1[(size_t)b] * P.m2[(size_t)b];
        h->near_prec = H.near_prec;
        h->near_entries = entries;
        h->near_stored = H.near_stored;
    }
    h->near_mode = H.near_mode;
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    return HMG_OK;
}

}  // namespace

hmg_status load(hmg_matrix** out, const char* path, cudaStream_t s)
{
    hmg_status st;
    File fh;
    fh.f = fopen(path, "rb");
    if (!fh.f) {
        set_error("hmg_load: cannot open %s", path);
        return HMG_ERR_INVALID;
    }
    FILE* f = fh.f;
    Reader R{f, 0};
    if (fseeko(f, 0, SEEK_END) != 0 || (R.size = ftello(f)) < 0 || fseeko(f, 0, SEEK_SET) != 0) {
        set_error("hmg_load: cannot size %s", path);
        return HMG_ERR_INVALID;
    }
    char magic[8];
    unsigned ver = 0, hb = 0;
    Header H{};
    if (!get(f, magic, 8) || memcmp(magic, MAGIC, 8) != 0 || !get(f, &ver, 4) || !get(f, &hb, 4)) {
        set_error("hmg_load: %s is not an H-matrix file", path);
        return HMG_ERR_INVALID;
    }
    if (ver != VERSION || hb != sizeof(Header) || !get(f, &H, sizeof H)) {
        set_error("hmg_load: %s has format version %u / header %u bytes; this library reads %u / %zu", path, ver, hb,
                  VERSION, sizeof(Header));
        return HMG_ERR_UNSUPPORTED;
    }
    Plan P;
    if ((st = check_file(R, H, P))) return st;
    hmg_matrix* h = nullptr;
    if ((st = hmg_create(&h, H.n1, H.n2, H.dim, H.bits, (void*)s))) return st;
    if ((st = upload(h, R, H, P, s))) {
        hmg_destroy(h);
        return st;
    }
    *out = h;
    return HMG_OK;
}

}  // namespace hmg
