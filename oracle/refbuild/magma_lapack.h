/* Empty stand-in for MAGMA's magma_lapack.h (nothing from it is used). */
#ifndef HMG_REF_MAGMA_LAPACK_SHIM_H
#define HMG_REF_MAGMA_LAPACK_SHIM_H
#endif
