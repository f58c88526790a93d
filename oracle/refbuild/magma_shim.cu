// Variable-size batched FP64 GEMV with MAGMA's calling convention, so kadircs/hmglib's
// sources link without MAGMA.  One CTA per matrix, one thread per output entry,
// summing in index order.  TEST INFRASTRUCTURE ONLY (builds the reference oracle).
#include "magma_v2.h"

int magma_init(void) { return 0; }
int magma_finalize(void) { return 0; }
void magma_queue_create(magma_int_t, magma_queue_t* queue) { *queue = nullptr; }

__global__ void shim_dgemv_vbatched(int trans, const int* m, const int* n, double alpha,
                                    double const* const* A, const int* lda,
                                    double const* const* x, const int* incx, double beta,
                                    double** y, const int* incy)
{
    const int b = blockIdx.x;
    const int rows = m[b], cols = n[b], ld = lda[b], ix = incx[b], iy = incy[b];
    const double* a = A[b];
    const double* xv = x[b];
    double* yv = y[b];
    const int nout = trans ? cols : rows;
    for (int o = threadIdx.x; o < nout; o += blockDim.x) {
        double acc = 0.0;
        if (trans) {
            for (int i = 0; i < rows; i++) acc += a[i + (size_t)o * ld] * xv[(size_t)i * ix];
        } else {
            for (int j = 0; j < cols; j++) acc += a[o + (size_t)j * ld] * xv[(size_t)j * ix];
        }
        double prev = beta != 0.0 ? beta * yv[(size_t)o * iy] : 0.0;
        yv[(size_t)o * iy] = alpha * acc + prev;
    }
}

void magmablas_dgemv_vbatched(magma_trans_t trans, magma_int_t* m, magma_int_t* n, double alpha,
                              double const* const* dA_array, magma_int_t* ldda,
                              double const* const* dx_array, magma_int_t* incx, double beta,
                              double** dy_array, magma_int_t* incy, magma_int_t batchCount,
                              magma_queue_t)
{
    if (batchCount <= 0) return;
    shim_dgemv_vbatched<<<batchCount, 128>>>(trans == MagmaTrans ? 1 : 0, m, n, alpha, dA_array, ldda,
                                             dx_array, incx, beta, dy_array, incy);
    cudaDeviceSynchronize();
}
