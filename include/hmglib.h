/*
 * hmglib.h -- drop-in replacement for kadircs/hmglib's src/hmglib.h (:29-121).
 *
 * Same struct h_matrix_data (same field names and types, in the same order) and
 * the same nine entry points, so the reference's drivers (hmglib_test.cu,
 * paper_benchmark.cu, paper_convergence_test.cu) compile against this header and
 * link against libhmg.so unchanged.  Differences a caller can observe:
 *
 *   * No MAGMA: magma_queue_t is an opaque pointer, and the field `magma_queue`
 *     holds the engine's handle (hmg_matrix*, include/hmg.h).
 *   * The entry points have C linkage (the reference's are C++-mangled) so that
 *     ctypes / cgo / JNI bindings can call them too.
 *   * Errors no longer exit the process (the reference calls exit() from
 *     checkCUDAError, helper.cu:31-37, and precompute_dense, hmglib.cu:243-247):
 *     a failing call leaves the structure unchanged where possible, prints the
 *     message to stderr and records it for hmg_last_error().
 *   * apply_h_matrix_mvp does not modify x (the reference permutes x in place and
 *     back, hmglib.cu:275,282).
 *   * root_level_set_1 and root_level_set_2 must be equal (the reference's drivers
 *     set both to 0; unequal levels take a tree branch the engine does not build).
 *
 * Like the reference, setup_h_matrix permutes data->coords_d[i][d] into Z order
 * and leaves the sorted Morton codes in code_d and the permutation in order.
 *
 * U, V and dA: as in the reference, they are NULL until precompute_aca /
 * precompute_dense and non-NULL afterwards (the reference tests them to decide
 * whether a compression exists, hmglib.cu:277-278).  They point into the engine's
 * own storage -- U and V both at the first factor allocation, whose blocks are laid
 * out as tile slices (hmg_internal.cuh), and dA at the near field in the same tile
 * layout -- not at the reference's rank-major concatenated U / V
 * (linear_algebra.cu:3808-3824) or column-major dense blocks (:3140-3342).  Read a
 * block's factors with hmg_get_factors; the library frees this storage in
 * destroy_h_matrix_data, so a caller must not.
 */
#ifndef HMGLIB_H
#define HMGLIB_H

#include <stdint.h>

#include "hmg.h"

#ifndef HMG_MAGMA_QUEUE_T_DEFINED
#define HMG_MAGMA_QUEUE_T_DEFINED
typedef void* magma_queue_t;
#endif

/* morton.h:23-41 */
struct point_set {
    double** coords;
    int dim;
    int size;
    double* max_per_dim;
    double* min_per_dim;
    unsigned int* point_ids;
};

struct morton_code {
    uint64_t* code;
    int size;
    int dim;
    int bits;
    double* max_values;
    double* min_values;
};

#define WT_ACA 1
#define WT_DENSE 2
#define MAX_POINT_DIMENSION 5

/* tree.h:38-55 */
struct work_item {
    int set1_l;
    int set1_u;
    int set2_l;
    int set2_u;
    int work_type;
    double max1[MAX_POINT_DIMENSION];
    double min1[MAX_POINT_DIMENSION];
    double max2[MAX_POINT_DIMENSION];
    double min2[MAX_POINT_DIMENSION];
    int dim;
    char level_1;
    char level_2;
};

/* linear_algebra.h:107-112 */
typedef struct mat_vec_data_info {
    int dense_count;
    int aca_count;
    int total_count;
} mat_vec_data_info;

/* system_assembler.h:23-32: the kernel function, now a plain descriptor living in
 * device memory (created by the functions of kernel_system_assembler.h) */
struct system_assembler {
    int kind;              /* HMG_KERNEL_* */
    double param;          /* length^2 or rho for the parameterised kinds */
    double regularization; /* added on the diagonal (kernel_system_assembler.h:47-48) */
};

struct h_matrix_data {
    double** coords_d[2];
    unsigned int* point_ids_d[2];
    double* max_per_dim_d[2];
    double* min_per_dim_d[2];
    double** coords_device[2];
    uint64_t* code_d[2];
    struct point_set* points_d[2];
    struct morton_code* morton_d[2];
    uint64_t* order[2];
    int bits;
    int dim;
    double eta;
    int max_level;
    int c_leaf;
    int mat_vec_data_count;
    int max_elements_in_array;
    int max_elements_in_mat_vec_data_array;
    struct work_item** mat_vec_data;
    int mat_vec_data_array_size;
    int k;
    double epsilon;
    mat_vec_data_info mat_vec_info;
    int point_count[2];
    struct system_assembler* assem;
    int max_batched_dense_size;
    int max_batched_aca_size;
    double dense_batching_ratio;
    double* U;
    double* V;
    double* dA;
    magma_queue_t magma_queue;
    int* dense_work_size;
    int* aca_work_size;
    int dense_batch_count;
    int aca_batch_count;
    char root_level_set_1;
    char root_level_set_2;
};

#ifdef __cplusplus
extern "C" {
#endif

/* hmglib.cu:68-123 */
void init_h_matrix_data(struct h_matrix_data* data, int point_count[2], int dim, int bits);
/* hmglib.cu:125-225 */
void setup_h_matrix(struct h_matrix_data* data);
/* hmglib.cu:271-286; x, y device vectors in the caller's order */
void apply_h_matrix_mvp(double* x, double* y, struct h_matrix_data* data);
/* hmglib.cu:288-301: one launch per block (hmg_matvec_unbatched), an independent
 * second product; FP64 factors */
void apply_h_matrix_mvp_without_batching(double* x, double* y, struct h_matrix_data* data);
/* hmglib.cu:305-348 */
void destroy_h_matrix_data(struct h_matrix_data* data);
/* hmglib.cu:228-236: fixed-rank ACA with rank data->k, FP64 factors */
void precompute_aca(struct h_matrix_data* data);
/* hmglib.cu:239-268: all dense blocks stored in FP64 */
void precompute_dense(struct h_matrix_data* data);
/* hmglib.cu:351-401: FP64 direct product (no N^2 matrix is formed) */
void apply_full_mvp(double* x, double* y, struct h_matrix_data* data);
/* hmglib.cu:420-439 */
void set_gaussian_kernel_rhs(double* b, struct h_matrix_data* data);

#ifdef __cplusplus
}
#endif

#endif
