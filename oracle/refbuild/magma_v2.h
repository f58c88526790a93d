/*
 * Minimal stand-in for MAGMA's magma_v2.h, written for building kadircs/hmglib's
 * sources as a reference oracle (MAGMA is neither installed nor vendored).  It
 * declares only what the reference uses: init/finalize, a queue type, the
 * transpose flags and magmablas_dgemv_vbatched (implemented in magma_shim.cu).
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef HMG_REF_MAGMA_V2_SHIM_H
#define HMG_REF_MAGMA_V2_SHIM_H
#include <cuda_runtime.h>
typedef int magma_int_t;
typedef struct hmg_ref_magma_queue* magma_queue_t;
typedef enum { MagmaNoTrans = 111, MagmaTrans = 112 } magma_trans_t;
int magma_init(void);
int magma_finalize(void);
void magma_queue_create(magma_int_t dev, magma_queue_t* queue);
void magmablas_dgemv_vbatched(magma_trans_t trans, magma_int_t* m, magma_int_t* n, double alpha,
                              double const* const* dA_array, magma_int_t* ldda,
                              double const* const* dx_array, magma_int_t* incx, double beta,
                              double** dy_array, magma_int_t* incy, magma_int_t batchCount,
                              magma_queue_t queue);
#endif
