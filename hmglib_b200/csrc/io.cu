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
    hmg_matrix* h = nullptr;
    if ((st = hmg_create(&h, H.n1, H.n2, H.dim, H.bits, (void*)s))) return st;
    auto fail = [&](hmg_status e) {
        hmg_destroy(h);
        return e;
    };
    for (int w = 0; w < 2; w++) {
        const size_t n = (size_t)h->n[w];
        if ((st = get_dev(f, h->pts[w], n * h->dim * 8, s)) || (st = get_dev(f, h->zpts[w], n * h->dim * 8, s)) ||
            (st = get_dev(f, h->codes[w], n * 8, s)) || (st = get_dev(f, h->perm[w], n * 4, s)) ||
            (st = get_dev(f, h->iperm[w], n * 4, s)))
            return fail(st);
        h->points_set[w] = true;
    }
    const size_t nb = (size_t)H.nblocks;
    h->h_r0.resize(nb); h->h_m1.resize(nb); h->h_c0.resize(nb); h->h_m2.resize(nb); h->h_type.resize(nb);
    if (!get(f, h->h_r0.data(), nb * 4) || !get(f, h->h_m1.data(), nb * 4) || !get(f, h->h_c0.data(), nb * 4) ||
        !get(f, h->h_m2.data(), nb * 4) || !get(f, h->h_type.data(), nb * 4)) {
        set_error("hmg_load: file truncated");
        return fail(HMG_ERR_INVALID);
    }
    h->eta = H.eta; h->c_leaf = H.c_leaf; h->max_level = H.max_level; h->rule = H.rule; h->levels = H.levels;
    h->nblocks = H.nblocks; h->ndense = H.ndense; h->naca = H.nblocks - H.ndense;
    if ((st = dalloc(&h->blk_r0, nb, s)) || (st = dalloc(&h->blk_m1, nb, s)) || (st = dalloc(&h->blk_c0, nb, s)) ||
        (st = dalloc(&h->blk_m2, nb, s)) || (st = dalloc(&h->blk_type, nb, s)))
        return fail(st);
    if (nb > 0) {
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_r0, h->h_r0.data(), nb * 4, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_m1, h->h_m1.data(), nb * 4, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_c0, h->h_c0.data(), nb * 4, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_m2, h->h_m2.data(), nb * 4, cudaMemcpyHostToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(h->blk_type, h->h_type.data(), nb * 4, cudaMemcpyHostToDevice, s));
    }
    if (H.group_count) {
        h->group_count = H.group_count;
        for (int w = 0; w < 2; w++) {
            h->group_off[w].resize(H.group_count + 1);
            if (!get(f, h->group_off[w].data(), sizeof(int) * (H.group_count + 1))) {
                set_error("hmg_load: file truncated");
                return fail(HMG_ERR_INVALID);
            }
        }
        if ((st = dalloc(&h->blk_param, nb, s)) || (st = get_dev(f, h->blk_param, nb * 8, s))) return fail(st);
    }
    if ((st = build_tiles(h))) return fail(st);
    h->setup_done = true;
    h->kspec = H.kspec;
    h->kernel_set = H.kernel_set != 0;
    if (H.far_prec >= 0) {
        std::vector<int> rank(nb), r32(nb), r16(nb);
        std::vector<size_t> cb((size_t)H.nchunks);
        std::vector<long long> place(3 * nb);
        if (!get(f, rank.data(), nb * 4) || !get(f, r32.data(), nb * 4) || !get(f, r16.data(), nb * 4) ||
            !get(f, cb.data(), 8 * cb.size()) || !get(f, place.data(), 8 * place.size())) {
            set_error("hmg_load: file truncated");
            return fail(HMG_ERR_INVALID);
        }
        for (size_t c = 0; c < cb.size(); c++) {
            void* p = nullptr;
            cudaError_t ce = cudaMalloc(&p, cb[c]);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                set_error("hmg_load: allocating %zu bytes of factors failed: %s", cb[c], cudaGetErrorString(ce));
                return fail(ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA);
            }
            h->far_chunks.push_back(p);
            h->far_chunk_bytes.push_back(cb[c]);
            if ((st = get_dev(f, p, cb[c], s))) return fail(st);
        }
        std::vector<void*> pu(nb, nullptr), pv(nb, nullptr);
        std::vector<long long> roff(nb + 1, 0);
        for (size_t b = 0; b < nb; b++) {
            roff[b + 1] = roff[b] + rank[b];
            if (place[3 * b] >= 0) {
                if (place[3 * b] >= (long long)cb.size()) {
                    set_error("hmg_load: block %zu names factor allocation %lld of %zu", b, place[3 * b], cb.size());
                    return fail(HMG_ERR_INVALID);
                }
                char* base = static_cast<char*>(h->far_chunks[(size_t)place[3 * b]]);
                pu[b] = base + place[3 * b + 1];
                pv[b] = base + place[3 * b + 2];
            }
        }
        if ((st = dalloc(&h->rank, nb, s)) || (st = dalloc(&h->rank_off, nb + 1, s)) ||
            (st = dalloc(&h->ptrU, nb, s)) || (st = dalloc(&h->ptrV, nb, s)) || (st = dalloc(&h->tier32, nb, s)) ||
            (st = dalloc(&h->tier16, nb, s)))
            return fail(st);
        if (nb > 0) {
            HMG_CUDA_TRY(cudaMemcpyAsync(h->rank, rank.data(), nb * 4, cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->tier32, r32.data(), nb * 4, cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->tier16, r16.data(), nb * 4, cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->ptrU, pu.data(), nb * sizeof(void*), cudaMemcpyHostToDevice, s));
            HMG_CUDA_TRY(cudaMemcpyAsync(h->ptrV, pv.data(), nb * sizeof(void*), cudaMemcpyHostToDevice, s));
        }
        HMG_CUDA_TRY(cudaMemcpyAsync(h->rank_off, roff.data(), (nb + 1) * 8, cudaMemcpyHostToDevice, s));
        h->rank_total = roff[nb];
        if ((st = dalloc((char**)&h->tbuf, (size_t)(h->rank_total + 32) * 8, s))) return fail(st);
        HMG_CUDA_TRY(cudaMemsetAsync(h->tbuf, 0, (size_t)(h->rank_total + 32) * 8, s));
        h->h_rank = rank;
        h->h_r32 = r32;
        h->h_r16 = r16;
        h->far_prec = H.far_prec; h->aca_k = H.aca_k; h->aca_eps = H.aca_eps;
        h->far_entries = H.far_entries; h->far_rows = H.far_rows; h->far_stored = H.far_stored;
        h->far_alg_u = H.far_alg_u; h->far_alg_v = H.far_alg_v; h->max_rank = H.max_rank;
    }
    if (H.near_prec >= 0 && H.ndense > 0) {
        const size_t esz = H.near_prec == HMG_PREC_FP64 ? 8 : 4;
        if ((st = dalloc(&h->near_off, (size_t)H.ndense, s)) ||
            (st = get_dev(f, h->near_off, sizeof(long long) * (size_t)H.ndense, s)))
            return fail(st);
        cudaError_t ce = cudaMalloc(&h->near_data, (size_t)H.near_stored * esz);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            h->near_data = nullptr;
            set_error("hmg_load: allocating the near field failed: %s", cudaGetErrorString(ce));
            return fail(ce == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA);
        }
        if ((st = get_dev(f, h->near_data, (size_t)H.near_stored * esz, s))) return fail(st);
    }
    if (H.near_prec >= 0) {
        h->near_prec = H.near_prec;
        h->near_entries = H.near_entries;
        h->near_stored = H.near_stored;
    }
    h->near_mode = H.near_mode;
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    *out = h;
    return HMG_OK;
}

}  // namespace hmg
