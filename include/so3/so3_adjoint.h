/*
 * so3_adjoint.h -- adjoint Wigner transforms, drop-in for the entry points of
 * the reference's include/so3/so3_adjoint.h.  They run on the GPU
 * (libso3gpu); f and flmn may be host or device pointers.  MW sampling and
 * non-steerable signals only (other parameters: status 3, exit(1) in the
 * default error mode), as the reference's direct adjoints assume MW.  As in
 * the reference, the entry point decides the layout: the _real variants use
 * the real layouts (n >= 0 coefficients, real samples) whatever the reality
 * flag says, the others the complex ones.
 */
#ifndef SO3_ADJOINT
#define SO3_ADJOINT

#include "so3_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* flmn = A^H f for the inverse transform A; reference src/c/so3_adjoint.c:34 */
void so3_adjoint_inverse_direct(SO3_COMPLEX(double) * flmn, const SO3_COMPLEX(double) * f,
                                const so3_parameters_t *parameters);
/* f = B^H flmn for the forward transform B; reference src/c/so3_adjoint.c:402 */
void so3_adjoint_forward_direct(SO3_COMPLEX(double) * f, const SO3_COMPLEX(double) * flmn,
                                const so3_parameters_t *parameters);
/* real signals: flmn (n >= 0) = A^H f for the real inverse transform; reference src/c/so3_adjoint.c:939 */
void so3_adjoint_inverse_direct_real(SO3_COMPLEX(double) * flmn, const double *f,
                                     const so3_parameters_t *parameters);
/* real signals: f = B^H flmn for the real forward transform; reference src/c/so3_adjoint.c:1313 */
void so3_adjoint_forward_direct_real(double *f, const SO3_COMPLEX(double) * flmn,
                                     const so3_parameters_t *parameters);

#ifdef __cplusplus
}
#endif
#endif
