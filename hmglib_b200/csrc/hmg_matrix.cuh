// hmg_matrix.cuh -- the engine's handle (opaque `hmg_matrix` of include/hmg.h).
#pragma once

#include <vector>

#include "hmg_internal.cuh"
#include "util.cuh"

struct hmg_matrix {
    int n[2] = {0, 0};
    int dim = 0, bits = 0;
    int device = 0;
    int nsm = 0;          // SMs of the device (grid sizes)
    cudaStream_t stream = nullptr;

    // ---- points -------------------------------------------------------------
    bool points_set[2] = {false, false};
    double* pts[2] = {nullptr, nullptr};   // caller order, SoA dim x n
    double* zpts[2] = {nullptr, nullptr};  // Z order, SoA dim x n
    uint64_t* codes[2] = {nullptr, nullptr};  // Z-ordered (sorted) Morton codes
    int* perm[2] = {nullptr, nullptr};        // perm[i] = caller index of Z point i
    int* iperm[2] = {nullptr, nullptr};       // inverse: Z index of caller point i

    // ---- tree ---------------------------------------------------------------
    bool setup_done = false;
    double eta = 0.0;
    int c_leaf = 0, max_level = 0, rule = 0;
    int nblocks = 0, ndense = 0, naca = 0, levels = 0;
    int* blk_r0 = nullptr;  // device SoA, reference mat_vec_data order
    int* blk_m1 = nullptr;
    int* blk_c0 = nullptr;
    int* blk_m2 = nullptr;
    int* blk_type = nullptr;
    std::vector<int> h_r0, h_m1, h_c0, h_m2, h_type;

    // ---- row tiles ----------------------------------------------------------
    int ntiles = 0;
    int* tile_r0 = nullptr;     // first Z row of each tile
    int* tile_s = nullptr;      // rows in tile (<= HMG_TILE_ROWS)
    int* tile_pstart = nullptr; // padded row start (sum of round_up4(s) of earlier tiles)
    int* blk_tfirst = nullptr;  // first tile of each block's rows
    int* blk_tlast = nullptr;
    int npairs = 0;
    int* tile_pair_start = nullptr;  // CSR over tiles (ntiles+1)
    int* pair_block = nullptr;       // block index of each (tile, block) pair
    std::vector<int> h_tile_pstart, h_blk_tfirst, h_blk_tlast;

    // ---- kernel function ------------------------------------------------------
    bool kernel_set = false;
    hmg::KernelSpec kspec{};

    // ---- grouped H-matrices (hmg_group_create) ---------------------------------
    // The union of independent H-matrices: block-diagonal, each set's blocks shifted
    // by its point offsets; the kernel parameter is per block.
    int group_count = 0;              // 0: a single H-matrix
    double* blk_param = nullptr;      // per block kernel parameter (groups only)
    std::vector<int> group_off[2];    // first row / column of each set, then n

    // ---- near field -----------------------------------------------------------
    int near_mode = HMG_NEAR_ONTHEFLY;
    int near_prec = -1;               // -1: not stored
    void* near_data = nullptr;
    long long* near_off = nullptr;    // element offset of each block (dense blocks)
    long long near_entries = 0;       // sum m1*m2
    long long near_stored = 0;        // stored elements incl. padding

    // ---- far field ------------------------------------------------------------
    int far_prec = -1;                // -1: not computed
    int aca_k = 0;
    double aca_eps = 0.0;
    int* rank = nullptr;              // per block (0 for dense)
    long long* rank_off = nullptr;    // exclusive scan of ranks over blocks
    long long rank_total = 0;
    void** ptrU = nullptr;            // per block device pointer (ACA blocks)
    void** ptrV = nullptr;
    std::vector<void*> far_chunks;    // allocations holding the factors
    std::vector<size_t> far_chunk_bytes;
    std::vector<int> h_rank;
    int* tier32 = nullptr;            // mixed storage: per block terms in FP32
    int* tier16 = nullptr;            // ... in FP16 (the rest of the rank in FP8)
    std::vector<int> h_r32, h_r16;
    long long far_entries = 0, far_rows = 0, far_stored = 0;
    long long far_alg_u = 0;          // bytes of the stored U terms (without padding)
    long long far_alg_v = 0;          // bytes of the stored V terms
    int max_rank = 0;

    // ---- BF16 operands for tensor-core multi-vector products (tc.cu) -------------
    bool tc_ready = false;
    void* tc_u = nullptr;                     // pass 2 A operands: U slices, near slices
    void* tc_v = nullptr;                     // pass 1 A operands: V_b^T
    void* tc_bbuf = nullptr;                  // per product: X cores, then t_b cores
    int tc_parts = 1;                         // BF16 parts per operand (1, 2 or 3), interleaved by K core
    char* tc_steps[2] = {nullptr, nullptr};   // per pass: steps, CTA by CTA
    char* tc_jobs[2] = {nullptr, nullptr};    // per pass: jobs, CTA by CTA
    char* tc_cta[2] = {nullptr, nullptr};     // per CTA: first job and step (int2), then the ends
    int* tc_kmap = nullptr;                   // pass 1: per stack, t_b destination of its 16 K cores
    int tc_njobs[2] = {0, 0};
    int tc_grid = 0;
    bool tc_all_tiles = false;                // every row tile has a pass-2 job
    bool tc_near = false;                     // near field on the tensor cores (else FP32 CUDA cores)
    long long tc_xkc = 0, tc_tkc = 0;         // per product: K cores of X, of t_b (8 columns / terms each)
    long long tc_bytes = 0;                   // bytes of one part of the BF16 operands

    // ---- tensor-core products with operands converted on chip (tcm.cu) ------------
    bool tcm_ready = false;
    int tcm_min_nrhs = 17;    // on-chip tensor-core products from this many vectors a pass
    char* tcm_steps[2] = {nullptr, nullptr};  // per pass: steps, CTA by CTA
    char* tcm_jobs[2] = {nullptr, nullptr};   // per pass: jobs, CTA by CTA
    char* tcm_cta[2] = {nullptr, nullptr};    // per CTA: first job and step (int2), then the ends
    void* tcm_stacks = nullptr;               // pass 1: the stacks of V_b^T
    float* tcm_tscale = nullptr;              // pass 1: scale of every t_b term (FP16 / FP8 terms), else 1
    int tcm_njobs[2] = {0, 0};
    long long tcm_xkc = 0, tcm_tkc = 0;       // K cores of X, of t_b
    void* tcm_bbuf = nullptr;                 // per product: X cores, then t_b cores (3 parts, 64 vectors)
    bool tcm_all_tiles = false;               // every row tile has a pass-2 job

    // ---- matvec workspace -------------------------------------------------------
    double* xs64 = nullptr;   // Z-ordered x
    float* xs32 = nullptr;
    void* tbuf = nullptr;     // V^T x per block (rank_total entries)
    void* pair_desc = nullptr;     // per (tile, block) pair: slice pointer, vector, columns
    int desc_near_mode = -1, desc_near_prec = -2, desc_far_prec = -2, desc_elem = 0;
    void* k1_units = nullptr;      // K1 pieces of V^T (rows of one storage tier), grouped by tier
    int nk1 = 0;
    int k1_count[3] = {0, 0, 0};   // pieces per tier (FP32/FP64, FP16, FP8)
    int k1_piece_start[3][5] = {};  // per tier: first piece of each lane-group class, end
    int k1_task_start[3][5] = {};   // per tier: first warp task of each class, task count
    int* far_list = nullptr;       // admissible blocks with rank > 0 (streaming V^T x)
    int nfar_list = 0;
    int* dev_err = nullptr;        // pipeline wait time-out flag (0 = fine)
    int matvec_variant = 1;        // 0: streaming kernels where applicable, 1: plain-load kernels
    int k1_piece_bytes = 65536;    // K1 warp-task unit: V^T rows of one tier up to these bytes (hmg_autotune)
    int k1_ctas_per_sm = 8;        // K1 grid: CTAs per SM (hmg_autotune)
    bool use_graphs = false;       // replay products as a captured CUDA graph (hmg_set_graphs)
    void* graph_exec = nullptr;    // cudaGraphExec_t of the last product's launches
    void* graph_key = nullptr;     // what it was captured for (matvec.cu)
    void* capture_stream = nullptr;  // cudaStream_t the graph is captured on
    int arith_prec = HMG_PREC_FP32;  // products over FP32 / mixed storage: FP32 or FP64 arithmetic
    int last_variant_k1 = -1, last_variant_k2 = -1;
    double* dev_x = nullptr;
    double* dev_y = nullptr;
    int k1_grid = 0, k2_grid = 0;
    bool profiling = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t k1_aux[2] = {nullptr, nullptr};  // side streams of the FP16 / FP8 V^T x tiers (matvec.cu)
    cudaEvent_t k1_ev[3] = {nullptr, nullptr, nullptr};  // their fork and joins
};

namespace hmg {
hmg_status setup_tree(hmg_matrix* h);
hmg_status group_setup_tree(hmg_matrix* g, int nsets, const int* const* off, const int* sdim,
                            const int* sbits, const int* sleaf);
hmg_status build_tiles(hmg_matrix* h);
hmg_status group_create(hmg_matrix** out, hmg_matrix* const* sets, int count, cudaStream_t s);
hmg_status group_setup(hmg_matrix** out, hmg_matrix* const* sets, int count, double eta, const int* c_leaf,
                       int max_level, int rule, cudaStream_t s);
hmg_status save(hmg_matrix* h, const char* path);
hmg_status load(hmg_matrix** out, const char* path, cudaStream_t s);
hmg_status run_aca(hmg_matrix* h, int k, double eps, int precision);
hmg_status fill_near(hmg_matrix* h, int precision);
hmg_status matvec_device(hmg_matrix* h, const double* x, double* y, bool fp64_arith = false);
hmg_status matvec_unbatched(hmg_matrix* h, const double* x, double* y);
hmg_status matvec_multi(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy);
hmg_status matvec_multi_tc(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy);
hmg_status build_bf16_factors(hmg_matrix* h, bool near_on_tensor_cores, int parts);
hmg_status build_tcm(hmg_matrix* h);
hmg_status matvec_multi_tcm(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy);
void free_tcm(hmg_matrix* h);
hmg_status autotune(hmg_matrix* h, int reps, int* best_piece, int* best_ctas, double* best_ms);
void free_tc(hmg_matrix* h);
void free_product_graph(hmg_matrix* h);
void launch_gather_multi32(hmg_matrix* h, const double* X, int ldx, int nrhs, float* xm);
hmg_status launch_tile_multi32_dense(hmg_matrix* h, const float* xm, int nrhs, double* Y, int ldy);
hmg_status direct_matvec(hmg_matrix* h, const double* x, const int* rows, int nrows,
                         double* y);
hmg_status gaussian_rhs(hmg_matrix* h, double* b);
hmg_status cg_solve(hmg_matrix* h, double shift, const double* b, double* x, double tol, int maxit, int refine,
                    int* iters_out, double* relres_out);
hmg_status morton_codes(const double* coords, int n, int dim, int bits, uint64_t* codes,
                        cudaStream_t s);
hmg_status minmax_device(const double* coords, int n, int dim, double* mn, double* mx, cudaStream_t s);
void free_far(hmg_matrix* h);
void free_near(hmg_matrix* h);
void free_tree(hmg_matrix* h);
const char* last_error();
}  // namespace hmg
