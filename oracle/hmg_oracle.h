/*
 * hmg_oracle.h -- CPU restatement of the kadircs/hmglib H-matrix hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine
 * in hmglib_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may load it.  The product path never calls it.
 *
 * Each function names the reference code (path:line inside kadircs/hmglib)
 * whose behaviour it restates.  Integer work (Morton codes, the permutation,
 * the block-cluster tree) is bit-exact with the reference; floating-point work
 * follows the reference's operation order, with the FMA contractions nvcc
 * applies to the reference's device code written out as explicit fma() calls.
 *
 * Parity is pinned by tests/golden/ (known-answer Morton lattices from
 * src/helper.cu:261-291 and dumps of the reference's own GPU build).
 */
#ifndef HMG_ORACLE_H
#define HMG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* kernel kinds (same numbering as include/hmg.h) */
#define ORC_KERNEL_GAUSSIAN_REF 1 /* exp(-r*r)             kernel_system_assembler.h:33-36 */
#define ORC_KERNEL_MATERN_REF   2 /* yn(1,r+1e-15) r / ... kernel_system_assembler.h:77-80 */
#define ORC_KERNEL_GAUSSIAN     3 /* exp(-r^2 / l2)                                         */
#define ORC_KERNEL_MATERN32     4 /* (1 + sqrt3 r/rho) exp(-sqrt3 r/rho)                     */

#define ORC_WT_ACA 1
#define ORC_WT_DENSE 2

/* per-dimension min / max (helper.cu:108-138); coords are SoA: coords[d*n+i] */
void orc_minmax(const double* coords, int n, int dim, double* mn, double* mx);

/* Morton code per point (morton.cu:21-107) */
void orc_morton(const double* coords, int n, int dim, int bits, const double* mn,
                const double* mx, uint64_t* codes);

/* stable sort of codes, returning sorted codes and the permutation
 * (helper.cu:140-167: thrust::sort_by_key over (code, index)) */
void orc_sort(const uint64_t* codes, int n, uint64_t* sorted, int64_t* order);

/* gather coords into Z order (helper.cu:293-328) */
void orc_reorder(const double* coords, int n, int dim, const int64_t* order, double* out);

/* block-cluster tree traversal (tree.cu:40-160,215-447,1429-1557) followed by
 * the DENSE-first stable sort (linear_algebra.cu:63-86,4037-4051).
 * rule: 0 = max(diam1,diam2) <= eta*dist (tree.cu:159), 1 = min(...).
 * Returns an opaque list; free with orc_blocks_free. */
typedef struct orc_blocks orc_blocks;
orc_blocks* orc_tree(const double* coords1, const uint64_t* codes1, int n1,
                     const double* coords2, const uint64_t* codes2, int n2, int dim,
                     double eta, int c_leaf, int max_level, int root_level1,
                     int root_level2, int rule, int sort_dense_first);
int orc_blocks_count(const orc_blocks* b);
int orc_blocks_levels(const orc_blocks* b);
/* each output array has orc_blocks_count entries; bounds inclusive like work_item */
void orc_blocks_get(const orc_blocks* b, int* s1l, int* s1u, int* s2l, int* s2u,
                    int* type, int* level1, int* level2);
void orc_blocks_free(orc_blocks* b);

/* one kernel entry K(i,j) on Z-ordered coords (kernel_system_assembler.h:38-52,82-96) */
double orc_entry(int kind, double param, double reg, const double* c1, int n1,
                 const double* c2, int n2, int dim, int i, int j);

/* Fixed-rank batched ACA with the reference's pivot rules
 * (linear_algebra.cu:769-787,918-1147,2009-2222,3684-4012): rows in index order
 * skipping residual rows with norm < 1e-13, column pivot = last abs-argmax,
 * rank k_b = min(k, m1, m2).  For block b, U_b is m1 x k_b column-major at
 * U + uoff[b], V_b is m2 x k_b column-major at V + voff[b] (offsets are
 * sum_{c<b} m*k_c).  ranks[b] receives the number of nonzero terms. */
void orc_aca_fixed(int kind, double param, double reg, const double* c1, int n1,
                   const double* c2, int n2, int dim, int nb, const int* s1l,
                   const int* s1u, const int* s2l, const int* s2u, int k,
                   const int64_t* uoff, const int64_t* voff, double* U, double* V,
                   int* ranks);

/* Adaptive partially pivoted ACA (the engine's eps mode): next row = argmax |u_r|
 * over unused rows, column = first abs-argmax, stop when
 * |u_r||v_r| <= eps ||S_r||_F.  Storage like orc_aca_fixed with capacity kmax
 * per block (k_b = min(kmax,m1,m2)). */
void orc_aca_adaptive(int kind, double param, double reg, const double* c1, int n1,
                      const double* c2, int n2, int dim, int nb, const int* s1l,
                      const int* s1u, const int* s2l, const int* s2u, int kmax,
                      double eps, const int64_t* uoff, const int64_t* voff, double* U,
                      double* V, int* ranks);

/* H-matvec on Z-ordered vectors: dense blocks from kernel entries, low-rank blocks
 * from U,V (linear_algebra.cu:2817-3137,3345-3511,1429-1591). ys must hold n1. */
void orc_hmatvec(int kind, double param, double reg, const double* c1, int n1,
                 const double* c2, int n2, int dim, int nb, const int* s1l,
                 const int* s1u, const int* s2l, const int* s2u, const int* type,
                 const int64_t* uoff, const int64_t* voff, const double* U,
                 const double* V, const int* ranks, const double* xs, double* ys);

/* FP64 direct sum y_i = sum_j K(i,j) x_j over the Z-ordered sets for the listed
 * rows (rows==NULL: all n1 rows, in order; otherwise y[t] is row rows[t]).
 * This is apply_full_mvp (hmglib.cu:351-401) without the N^2 matrix. */
void orc_direct(int kind, double param, double reg, const double* c1, int n1,
                const double* c2, int n2, int dim, const double* xs, const int* rows,
                int nrows, double* y, int nthreads);

/* the right-hand side of set_gaussian_kernel_rhs (hmglib.cu:403-439) per point */
void orc_gaussian_rhs(const double* coords, int n, int dim, double* b);

#ifdef __cplusplus
}
#endif
#endif
