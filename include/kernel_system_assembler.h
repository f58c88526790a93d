/*
 * kernel_system_assembler.h -- drop-in for kadircs/hmglib's
 * src/kernel_system_assembler.h (:26-102).
 *
 * The reference builds C++ objects with virtual get_matrix_entry() by device-side
 * `new` (kernel_system_assembler.cu:25-77).  Here an assembler is a plain
 * descriptor (struct system_assembler, include/hmglib.h) in device memory; the
 * engine reads it once and evaluates the kernel inline in its own kernels.
 *
 * Usage is unchanged (hmglib_test.cu:81-90): the caller cudaMallocs a device slot
 * for one pointer, `create_*` stores the device address of a new descriptor in
 * that slot, the caller copies it back and assigns it to data.assem, and
 * `destroy_*` frees the descriptor whose address is in the slot.
 */
#ifndef KERNEL_SYSTEM_ASSEMBLER_H
#define KERNEL_SYSTEM_ASSEMBLER_H

#include "hmglib.h"

#ifdef __cplusplus
struct gaussian_kernel_system_assembler : public system_assembler {};
struct matern_kernel_system_assembler : public system_assembler {};
struct gaussian_lengthscale_kernel_system_assembler : public system_assembler {};
struct matern32_kernel_system_assembler : public system_assembler {};
#else
struct gaussian_kernel_system_assembler { struct system_assembler base; };
struct matern_kernel_system_assembler { struct system_assembler base; };
struct gaussian_lengthscale_kernel_system_assembler { struct system_assembler base; };
struct matern32_kernel_system_assembler { struct system_assembler base; };
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* exp(-r^2) + regularization on the diagonal (kernel_system_assembler.h:26-52) */
void create_gaussian_kernel_system_assembler_object(struct gaussian_kernel_system_assembler** assem,
                                                    double regularization);
void destroy_gaussian_kernel_system_assembler_object(struct gaussian_kernel_system_assembler** assem);

/* Y1(r+1e-15) r / (2^{d/2} Gamma(1+d/2)) + regularization (kernel_system_assembler.h:70-96) */
void create_matern_kernel_system_assembler_object(struct matern_kernel_system_assembler** assem,
                                                  double regularization);
void destroy_matern_kernel_system_assembler_object(struct matern_kernel_system_assembler** assem);

/* extensions with no reference counterpart: exp(-r^2/length2), and
 * (1 + sqrt3 r/rho) exp(-sqrt3 r/rho) */
void create_gaussian_lengthscale_kernel_system_assembler_object(
    struct gaussian_lengthscale_kernel_system_assembler** assem, double length2, double regularization);
void create_matern32_kernel_system_assembler_object(struct matern32_kernel_system_assembler** assem,
                                                    double rho, double regularization);

#ifdef __cplusplus
}
#endif

#endif
