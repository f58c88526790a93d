/*
 * hmg.h -- C ABI of the B200 H-matrix engine (libhmg.so).
 *
 * Plain C types only: an opaque handle, int/double/pointer arguments and a status
 * code.  Every function returns HMG_OK or an error status and never exits the
 * process; hmg_last_error() gives the message of the last failure on the calling
 * thread.  Device pointers are CUDA device (or managed) addresses on the device
 * that was current when the handle was created; work is ordered on the handle's
 * stream (hmg_create's `stream`, NULL = the legacy default stream) and the
 * functions documented as synchronous return after it finished.
 *
 * Each entry point names the kadircs/hmglib interface it replaces (path:line in
 * that project).  include/hmglib.h keeps the reference's own entry points on top
 * of these.
 */
#ifndef HMG_H
#define HMG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hmg_matrix hmg_matrix;

typedef enum {
    HMG_OK = 0,
    HMG_ERR_INVALID = 1,     /* bad argument */
    HMG_ERR_CUDA = 2,        /* a CUDA call failed (message in hmg_last_error) */
    HMG_ERR_NOMEM = 3,       /* device memory exhausted or over the handle's budget */
    HMG_ERR_STATE = 4,       /* call out of order (e.g. matvec before setup) */
    HMG_ERR_UNSUPPORTED = 5  /* configuration the engine does not implement */
} hmg_status;

/* kernel functions k(x, y) = f(r), r = |x - y| (kernel_system_assembler.h:26-102) */
#define HMG_KERNEL_GAUSSIAN_REF 1 /* exp(-r^2), the reference's gaussian assembler      */
#define HMG_KERNEL_MATERN_REF   2 /* Y1(r+1e-15) r / (2^{d/2} Gamma(1+d/2)), the ref's   */
#define HMG_KERNEL_GAUSSIAN     3 /* exp(-r^2 / param), param = length^2                 */
#define HMG_KERNEL_MATERN32     4 /* (1 + sqrt3 r/param) exp(-sqrt3 r/param), param=rho  */

/* admissibility rules (tree.cu:121-160) */
#define HMG_ADMISSIBLE_MAX 0 /* max(diam1, diam2) <= eta * dist  (the reference's rule) */
#define HMG_ADMISSIBLE_MIN 1 /* min(diam1, diam2) <= eta * dist                          */

/* storage precision of the near-field blocks and the low-rank factors */
#define HMG_PREC_FP64 0
#define HMG_PREC_FP32 1
/* Low-rank factors only (adaptive ACA): each block keeps its leading terms in FP32
 * and stores the terms whose tail sum of |u_l||v_l| is below 1e-4 of the block's
 * Frobenius norm in FP16 and below 1.5e-6 in FP8 e4m3, each scaled; the added error
 * is ~1e-7 of the block norm.  hmg_precompute_dense with this value stores FP32. */
#define HMG_PREC_MIXED 2
/* Tensor-core operands only (hmg_build_tensor_core_operands): BF16; BF16 pairs hi + lo
 * (16 significant bits, three MMAs per K step: hi*hi + hi*lo + lo*hi); BF16 triples
 * hi + lo + lo2 (24 significant bits, six MMAs per K step: hi*hi + hi*lo + lo*hi +
 * hi*lo2 + lo2*hi + lo*lo) */
#define HMG_PREC_BF16 3
#define HMG_PREC_BF16X3 4
#define HMG_PREC_BF16X6 5
/* Tensor-core operands converted on chip: no copy is stored.  The product kernels read
 * the handle's own FP32 near field and FP32 or mixed factors and split every value
 * into three BF16 parts in shared memory (FP16 and FP8 terms are exact in two and one
 * parts and run fewer MMAs); accuracy as HMG_PREC_BF16X6, memory only for the X and
 * t_b operands of a product (6 bytes x 64 vectors per column and per term). */
#define HMG_PREC_BF16X6_ONCHIP 6

/* near-field mode for hmg_matvec */
#define HMG_NEAR_STORED 0   /* read the blocks stored by hmg_precompute_dense          */
#define HMG_NEAR_ONTHEFLY 1 /* regenerate dense entries from the points in every call  */

typedef struct {
    int n1, n2, dim, bits;
    int block_count, dense_count, aca_count, levels;
    int tile_count;           /* row tiles of the matvec */
    int max_rank;             /* largest rank over admissible blocks (after ACA) */
    int64_t near_entries;     /* sum over dense blocks of m1*m2 */
    int64_t far_entries;      /* sum over admissible blocks of (m1+m2)*rank */
    int64_t far_rows;         /* sum over admissible blocks of m1+m2 */
    int64_t near_bytes;       /* bytes of stored near-field data (0 if not stored) */
    int64_t far_bytes;        /* bytes of stored factors */
    int64_t matvec_bytes;     /* bytes one hmg_matvec streams from HBM (algorithmic) */
    int near_precision, far_precision, near_mode;
    int64_t far_u_bytes;      /* bytes of the stored U terms (sum m1 * rank * size, no padding) */
    int64_t far_v_bytes;      /* bytes of the stored V terms */
    int matvec_launches;      /* kernels one hmg_matvec launches (plain-load kernels) */
    int group_count;          /* sets of a group handle (hmg_group_create), else 0 */
    int tc_parts;             /* BF16 parts per tensor-core operand (0: none built) */
    int64_t tc_bytes;         /* bytes of the stored tensor-core operands, all parts */
    int tc_onchip;            /* 1: tensor-core operands converted on chip (HMG_PREC_BF16X6_ONCHIP) */
} hmg_info;

/* message of the last failed call on this thread ("" if none) */
const char* hmg_last_error(void);
int hmg_version(void);

/* Allocate a handle for two point sets of n1 and n2 points in `dim` (2 or 3)
 * dimensions; `bits` is the Morton resolution per dimension (0 picks 32 for 2D,
 * 20 for 3D, the only pairs the reference supports, morton.cu:21-67).
 * `stream` is a cudaStream_t (NULL = default stream).
 * Replaces init_h_matrix_data (hmglib.cu:68-123). */
hmg_status hmg_create(hmg_matrix** out, int n1, int n2, int dim, int bits, void* stream);

/* Copy the coordinates of set 0 or 1: SoA, coords[d*n + i], n = n1 or n2.
 * on_device != 0: `coords` is a device pointer.  Replaces the caller writing
 * data.coords_d[set][d] (hmglib_test.cu:68-75).  Synchronous. */
hmg_status hmg_set_points(hmg_matrix* h, int set, const double* coords, int on_device);

/* Morton codes, Z-order permutation and block-cluster tree.  Replaces
 * setup_h_matrix (hmglib.cu:125-225).  root levels must be equal (the reference's
 * drivers set both to 0, paper_benchmark.cu:106-107).  Synchronous. */
hmg_status hmg_setup(hmg_matrix* h, double eta, int c_leaf, int max_level, int root_level1,
                     int root_level2, int rule);

/* Select the kernel function.  Replaces create_gaussian_kernel_system_assembler_object
 * / create_matern_kernel_system_assembler_object (kernel_system_assembler.cu:25-77). */
hmg_status hmg_set_kernel(hmg_matrix* h, int kind, double param, double regularization);

/* Batched ACA of all admissible blocks.  eps <= 0: the reference's fixed-rank ACA
 * (rank min(k,m1,m2), sequential row pivots; linear_algebra.cu:3684-4012);
 * eps > 0: adaptive ACA to relative accuracy eps with rank at most k.  Factors are
 * stored in `precision`.  Replaces precompute_aca (hmglib.cu:228-236).  Synchronous. */
hmg_status hmg_precompute_aca(hmg_matrix* h, int k, double eps, int precision);

/* Fill and store all dense blocks in `precision`.  Replaces precompute_dense
 * (hmglib.cu:239-268).  Synchronous. */
hmg_status hmg_precompute_dense(hmg_matrix* h, int precision);

/* near field source of hmg_matvec (HMG_NEAR_STORED needs hmg_precompute_dense) */
hmg_status hmg_set_near_mode(hmg_matrix* h, int mode);

/* y = H x on device vectors in the caller's point order; x is not modified.
 * Asynchronous on the handle's stream.  Replaces apply_h_matrix_mvp
 * (hmglib.cu:271-286). */
hmg_status hmg_matvec(hmg_matrix* h, const double* x, double* y);

/* y = H x one block at a time: every dense block (entries generated in FP64) and
 * then every admissible block (FP64 arithmetic over the stored FP64 or FP32
 * factors) is applied by its own kernel launch, in work-list order.  A second,
 * independent implementation of the product for checking, launch-bound by design.
 * Not on group handles or mixed storage.  Asynchronous on the handle's stream.
 * Replaces sequential_h_matrix_mvp_without_batching (linear_algebra.cu:4384-4443),
 * which apply_h_matrix_mvp_without_batching (hmglib.cu:288-301) calls. */
hmg_status hmg_matvec_unbatched(hmg_matrix* h, const double* x, double* y);

/* Same product with host vectors: copies x in, multiplies, copies y out, returns
 * when y is written.  x and y may be pageable or pinned memory; they are copied
 * directly between the caller's memory and the device (the driver stages pageable
 * memory itself). */
hmg_status hmg_matvec_host(hmg_matrix* h, const double* x_host, double* y_host);

/* y = K x in FP64 by direct summation on the GPU (no N^2 storage).  Replaces
 * apply_full_mvp (hmglib.cu:351-401).  Asynchronous on the handle's stream. */
hmg_status hmg_full_matvec(hmg_matrix* h, const double* x, double* y);

/* FP64 direct sum for a list of rows (caller order indices): y[t] = (K x)[rows[t]].
 * rows, x, y are device pointers.  Asynchronous. */
hmg_status hmg_full_matvec_rows(hmg_matrix* h, const double* x, const int* rows, int nrows,
                                double* y);

/* Tensor-core products (no reference counterpart): converts the handle's FP32 low-rank
 * factors (hmg_precompute_aca with HMG_PREC_FP32, ranks <= 128) into BF16 copies laid
 * out as tcgen05 operands, and with near_precision HMG_PREC_BF16 its FP32 stored near
 * field (hmg_precompute_dense with HMG_PREC_FP32) too.  Afterwards hmg_matvec_multi
 * with 2..64 vectors computes t_b = V_b^T X_b and U t_b on the tensor cores with BF16
 * operands (X and t_b rounded to BF16) and FP32 accumulation; the near field runs
 * there as well (HMG_PREC_BF16) or on the CUDA cores in FP32 (HMG_PREC_FP32).  Results
 * agree with the FP32 products to ~1e-3 (BF16 rounding).  HMG_PREC_BF16X3 keeps every
 * operand, the near field included, as a BF16 pair (hi and the rounding of what hi
 * misses) and multiplies hi*hi + hi*lo + lo*hi: ~7e-6, with twice the operand bytes
 * and three times the MMAs.  HMG_PREC_BF16X6 keeps three parts (24 bits, as FP32) and
 * adds the terms down to 2^-16 of hi*hi: ~4e-7, 1.5 times the bytes of X3.  With split
 * operands hi*hi and the correction terms accumulate apart and every accumulator is
 * drained after at most 128 K positions; the sums continue in FP32 on the CUDA cores.
 * The copies sit beside the FP32 storage (hmg_info.tc_bytes; one part holds ~0.6x its
 * bytes).  Single-vector products keep using the FP32 storage.  Recomputing the
 * factors or the near field drops the copies.
 * HMG_PREC_BF16X6_ONCHIP stores no copy: it plans the same two passes over the
 * handle's own storage -- FP32 or mixed (HMG_PREC_MIXED) factors and the FP32 near
 * field -- and the pass kernels split every value into three BF16 parts on chip while
 * they stream it (FP16 / FP8 terms into the parts that hold them exactly, with fewer
 * MMAs).  Products agree with FP64 to ~4e-7 like HMG_PREC_BF16X6, and the only memory
 * added is the X and t_b operand buffer (3 x 2 bytes x 64 vectors per column and per
 * term): this is the form that fits at N = 2^20.  Its products of fewer than 17
 * vectors a pass run on the CUDA cores (hmg_set_tensor_core_min_vectors).  The plan
 * is built on the host once, on several threads.
 * hmg_build_bf16_factors(h) is hmg_build_tensor_core_operands(h, HMG_PREC_BF16). */
hmg_status hmg_build_tensor_core_operands(hmg_matrix* h, int near_precision);
hmg_status hmg_build_bf16_factors(hmg_matrix* h);

/* Write a set-up H-matrix to `path` (points, permutations, block list, ranks and
 * storage tiers, factors, stored near field) and read it back into a new handle on
 * `stream`; the loaded H-matrix multiplies bit-identically to the saved one.  The
 * format is this library's own (versioned; other versions are refused with
 * HMG_ERR_UNSUPPORTED).  Synchronous.  No reference counterpart (the reference only
 * prints its tree for debugging, tree.cu:173-183). */
hmg_status hmg_save(hmg_matrix* h, const char* path);
hmg_status hmg_load(hmg_matrix** out, const char* path, void* stream);

/* Many independent H-matrices as one (no reference counterpart; the reference runs
 * one h_matrix_data per call with its own MAGMA setup, hmglib.cu:119).  `sets` are
 * handles after hmg_setup and hmg_set_kernel (same kernel kind and regularization,
 * any parameter, 2D and 3D mixed).  The new handle is their block-diagonal union: its
 * points are the sets' points in set order (rows of set i start at offset1_i, columns
 * at offset2_i), each block keeps its set's kernel parameter.  hmg_precompute_aca,
 * hmg_precompute_dense (required: the near field is stored), hmg_matvec,
 * hmg_matvec_multi and hmg_cg_solve then cover all sets in the same kernel launches;
 * vectors are the concatenation of the sets' vectors.  Each set's result equals its
 * own handle's bit for bit.  The set handles stay valid and independent. */
hmg_status hmg_group_create(hmg_matrix** out, hmg_matrix* const* sets, int count, void* stream);
/* The same group built without setting the sets up one by one: `sets` need only
 * hmg_set_points (both sides) and hmg_set_kernel (same kernel kind and regularization,
 * 2D and 3D mixed).  Every set's points are ordered by its own Morton codes and every
 * set's block-cluster tree is built in the same kernel launches (one level loop from
 * one root pair per set), with admissibility parameter eta, rule and max_level shared
 * and the leaf size c_leaf[i] of set i.  The result equals hmg_setup(sets[i], eta,
 * c_leaf[i], max_level, ..., rule) on every set followed by hmg_group_create, bit for
 * bit: the same permutations, blocks, block order and products.  The set handles are
 * not modified.  No reference counterpart (the reference builds one tree per call,
 * hmglib.cu:125-225). */
hmg_status hmg_group_setup(hmg_matrix** out, hmg_matrix* const* sets, int count, double eta, const int* c_leaf,
                           int max_level, int rule, void* stream);
/* offsets[0..count] of a group's rows (set 0) or columns (set 1); offsets[count] = n */
hmg_status hmg_group_offsets(hmg_matrix* h, int set, int64_t* offsets);

/* Y = H X for 1 <= nrhs <= 64 vectors: X (n2 x nrhs) and Y (n1 x nrhs) are device
 * FP64 column-major with leading dimensions ldx >= n2, ldy >= n1, caller order.  The
 * stored H-matrix is read once per 32 vectors (FP32 / FP64 storage with a stored near
 * field; otherwise one product per vector), once for all 64 with tensor-core operands
 * (hmg_build_tensor_core_operands).  Same arithmetic as hmg_matvec;
 * asynchronous on the handle's stream.  No reference counterpart (the reference
 * multiplies one vector per apply_h_matrix_mvp call, hmglib.cu:271-286). */
hmg_status hmg_matvec_multi(hmg_matrix* h, int nrhs, const double* X, int ldx, double* Y, int ldy);

/* Kernel-ridge solve (H + shift I) x = b by conjugate gradients with the handle's
 * H-matvec as operator (n1 == n2 and a symmetric positive definite kernel).  b and
 * x are device vectors in the caller's order; x holds the initial guess and
 * receives the solution.  FP64 vectors, inner products and stopping test.  refine
 * == 0: products in the handle's arithmetic (hmg_set_product_precision).  refine !=
 * 0: the residual is that of the stored operator applied in FP64 -- true residuals
 * use FP64-arithmetic products, CG steps use them until |r| <= 5e5 tol |b| and the
 * handle's arithmetic after (relaxed inexact Krylov), with restarts from the true
 * residual if the recurrence drifted.
 * Stops when |b - (H + shift I) x| <= tol |b| or after maxit products.  iters and
 * relres (may be NULL) receive the CG iterations and the final relative residual,
 * recomputed from x.  Synchronous.  No reference counterpart (hmglib has no solver;
 * its assemblers' `regularization` is the diagonal shift, kernel_system_assembler.h:47-48). */
hmg_status hmg_cg_solve(hmg_matrix* h, double shift, const double* b, double* x, double tol, int maxit,
                        int refine, int* iters, double* relres);

/* Kernel-ridge solves with several right-hand sides: (H + shift I) X = B for
 * 1 <= nrhs <= 64 columns (device FP64, column-major, leading dimensions ldb, ldx >=
 * n; X holds the initial guesses and receives the solutions).  Every column runs its
 * own conjugate-gradient recurrence; the columns share one hmg_matvec_multi product
 * per iteration, and vectors, inner products, step lengths and stopping tests are
 * FP64 on the device.  refine != 0 targets the stored operator applied in FP64 as
 * hmg_cg_solve does: true residuals with FP64-arithmetic products, inner CG with
 * FP64-arithmetic products until the largest relative residual is below
 * 5e5 tol and the handle's arithmetic after that, restarts from the true residual.
 * Stops when every column has |b_j - (H + shift I) x_j| <= tol |b_j| or after maxit
 * iterations; iters (may be NULL) receives the iterations, relres[nrhs] (may be
 * NULL) the final true relative residuals.  Synchronous.  No reference counterpart
 * (kernel_system_assembler.h:47-48 is the shift). */
hmg_status hmg_cg_solve_multi(hmg_matrix* h, int nrhs, double shift, const double* B, int ldb, double* X, int ldx,
                              double tol, int maxit, int refine, int* iters, double* relres);

/* The same solve driven step by step, for callers that interleave it with other
 * work (a serving loop): hmg_cg_multi_begin allocates the solve's work vectors;
 * each hmg_cg_multi_advance enqueues at most one piece of work on the handle's
 * stream (one CG iteration, or a true residual and restart) and never waits for the
 * GPU -- *enqueued (may be NULL) says whether it did; residual norms come back
 * through pinned buffers, at most two iterations behind; hmg_cg_multi_poll (non-
 * blocking) reports *done once the stopping test holds, with the iterations and the
 * latest true relative residuals; hmg_cg_multi_end waits for the stream and frees
 * the state.  B and X must stay valid until hmg_cg_multi_end. */
typedef struct hmg_cg_multi hmg_cg_multi;
hmg_status hmg_cg_multi_begin(hmg_cg_multi** out, hmg_matrix* h, int nrhs, double shift, const double* B, int ldb,
                              double* X, int ldx, double tol, int maxit, int refine);
hmg_status hmg_cg_multi_advance(hmg_cg_multi* s, int* enqueued);
hmg_status hmg_cg_multi_poll(hmg_cg_multi* s, int* done, int* iters, double* relres);
hmg_status hmg_cg_multi_end(hmg_cg_multi* s);

/* b_i = prod_d sqrt(pi)/2 (erf(1 - x_id) - erf(-x_id)) for set 0, caller order, device b.
 * Replaces set_gaussian_kernel_rhs (hmglib.cu:403-439). */
hmg_status hmg_gaussian_rhs(hmg_matrix* h, double* b);

hmg_status hmg_synchronize(hmg_matrix* h);

/* Per-phase device timing of hmg_matvec (no reference counterpart: the reference's
 * TIME_* macros are commented out, hmglib.cu:31-34).  on != 0 records CUDA events
 * between the product's kernels; hmg_get_profile returns the last product's
 * [gather x, V^T x, tile products, total] in milliseconds (synchronises). */
hmg_status hmg_set_profiling(hmg_matrix* h, int on);
hmg_status hmg_get_profile(hmg_matrix* h, double* ms4);

/* Product kernels (no reference counterpart): 1 (default) reads stored slices with
 * coalesced 16-byte loads straight into registers; 0 streams them through shared
 * memory with bulk asynchronous copies (not used for on-the-fly near fields or ranks
 * above 128).  Both give the same product to rounding (variant 0 sums in FP64,
 * variant 1 sums each slice in FP32 and the slices in FP64). */
hmg_status hmg_set_matvec_variant(hmg_matrix* h, int variant);

/* Autotuning (no reference counterpart): times the single-vector product of this
 * H-matrix for each V^T x task size (32, 64, 128 KB of V^T rows per warp task) and
 * grid (4, 8, 16 CTAs per SM), `reps` products each after an untimed one, and keeps
 * the fastest for later products.  Returns the choice and its ms per product (any
 * output pointer may be NULL).  Synchronous; results of products do not depend on it
 * beyond FP32 summation order within a piece. */
hmg_status hmg_autotune(hmg_matrix* h, int reps, int* piece_bytes, int* ctas_per_sm, double* ms);

/* Products as CUDA graphs (no reference counterpart): with on != 0, hmg_matvec and
 * hmg_matvec_host capture the launches of a product into a CUDA graph on the first call
 * and replay it (cudaGraphLaunch) while the arguments and the handle's storage stay the
 * same; any change (other x or y, other storage, modes or kernel) captures anew.
 * Results are bit-identical to direct launches.  Default off. */
hmg_status hmg_set_graphs(hmg_matrix* h, int on);

/* Multi-vector products on a handle with operands converted on chip
 * (hmg_build_tensor_core_operands with HMG_PREC_BF16X6_ONCHIP) run on the tensor
 * cores from nrhs vectors a pass (default 17); smaller batches run on the CUDA
 * cores, which are faster there: a tensor-core pass costs about the same for 2 to
 * 32 vectors.  nrhs >= 2; 2 sends every multi-vector product to the tensor cores.
 * No reference counterpart (the reference multiplies one vector per call). */
hmg_status hmg_set_tensor_core_min_vectors(hmg_matrix* h, int nrhs);

/* Arithmetic of the products over FP32 or mixed storage (no reference counterpart):
 * HMG_PREC_FP32 (default) multiplies each slice in FP32 and sums the slices in FP64;
 * HMG_PREC_FP64 converts every stored value and multiplies in FP64, so the stored
 * operator is applied exactly (to FP64 rounding).  FP64 storage always uses FP64.
 * hmg_cg_solve with refine chooses the arithmetic of its products itself. */
hmg_status hmg_set_product_precision(hmg_matrix* h, int precision);

/* Free the handle and all device memory it owns.  Replaces destroy_h_matrix_data
 * (hmglib.cu:305-348). */
hmg_status hmg_destroy(hmg_matrix* h);

/* ---- inspection (host copies, synchronous) ---------------------------------- */
hmg_status hmg_get_info(hmg_matrix* h, hmg_info* info);
/* Z-ordered (sorted) Morton codes of set 0/1 (the reference's code_d after setup) */
hmg_status hmg_get_codes(hmg_matrix* h, int set, uint64_t* codes);
/* order[i] = caller index of Z-ordered point i (the reference's order[set]) */
hmg_status hmg_get_order(hmg_matrix* h, int set, int64_t* order);
/* Z-ordered coordinates, SoA coords[d*n+i] (the reference permutes coords_d in place) */
hmg_status hmg_get_points(hmg_matrix* h, int set, double* coords);
/* the leaf list in the reference's mat_vec_data order (bounds inclusive, work_item
 * set1_l/set1_u/set2_l/set2_u/work_type, tree.h:38-55); arrays of block_count */
hmg_status hmg_get_blocks(hmg_matrix* h, int* s1l, int* s1u, int* s2l, int* s2u, int* type);
/* per block rank (0 for dense blocks) */
hmg_status hmg_get_ranks(hmg_matrix* h, int* ranks);
/* factors of block b as FP64 column-major U (m1 x r) and V (m2 x r) */
hmg_status hmg_get_factors(hmg_matrix* h, int block, double* U, double* V);

/* ---- primitives (device pointers, asynchronous on `stream`) ----------------- */
/* stable LSD radix sort of 64-bit keys carrying 32-bit values, in place;
 * `key_bits` = number of low key bits that can be nonzero (64 if unknown).  The
 * call reads the histogram of all digits back to the host to skip passes whose
 * digit is the same for every key, so it waits for `stream` once per call. */
hmg_status hmg_radix_sort_u64(uint64_t* keys, uint32_t* values, int n, int key_bits,
                              void* stream);
/* The same sort without any device allocation, for callers that must not have the
 * library call cudaMalloc (a program that owns all device memory through its own
 * pool, or a loop where an allocation's implicit synchronisation is not allowed).
 * No counterpart in the reference.  Scratch is a fixed array compiled into the
 * library (held on every GPU that loads it): n above 2^20 keys is rejected with
 * HMG_ERR_INVALID.  The first call on a device looks the array up (make it before
 * any stream capture) and keeps its address for the rest of the process (after a
 * cudaDeviceReset of that device the entry point cannot be used again).  The call
 * only enqueues work on `stream` and returns without waiting for it: the passes
 * whose digit is the same for every key are recognised on the device.  Calls share
 * the array, so calls that overlap on the GPU race -- keep them on one stream.
 * Result identical to hmg_radix_sort_u64. */
hmg_status hmg_radix_sort_u64_noalloc(uint64_t* keys, uint32_t* values, int n, int key_bits,
                                      void* stream);

/* Morton codes of n points (SoA coords[d*n+i]) with per-dimension min/max
 * computed on the device (helper.cu:108-138, morton.cu:79-112) */
hmg_status hmg_morton_codes(const double* coords, int n, int dim, int bits, uint64_t* codes,
                            void* stream);

#ifdef __cplusplus
}
#endif
#endif
