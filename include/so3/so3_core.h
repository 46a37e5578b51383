/*
 * so3_core.h -- Wigner transforms on SO(3), drop-in for the reference's
 * include/so3/so3_core.h:15-46.  The four via-SSHT entry points run on the GPU
 * (libso3gpu); f and flmn may be host or device pointers (host buffers are
 * staged through device memory inside the call).  Sizes: f holds
 * so3_sampling_f_size(parameters) samples, flmn so3_sampling_flmn_size().
 * For the forward transforms with n_mode != SO3_N_MODE_ALL the caller zeroes
 * flmn beforehand, as in the reference.
 */
#ifndef SO3_CORE
#define SO3_CORE

#include "so3_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference src/c/so3_core.c:51 */
void so3_core_inverse_via_ssht(SO3_COMPLEX(double) * f, const SO3_COMPLEX(double) * flmn,
                               const so3_parameters_t *parameters);
/* reference src/c/so3_core.c:458 */
void so3_core_inverse_via_ssht_real(double *f, const SO3_COMPLEX(double) * flmn,
                                    const so3_parameters_t *parameters);
/* reference src/c/so3_core.c:246 */
void so3_core_forward_via_ssht(SO3_COMPLEX(double) * flmn, const SO3_COMPLEX(double) * f,
                               const so3_parameters_t *parameters);
/* reference src/c/so3_core.c:675 */
void so3_core_forward_via_ssht_real(SO3_COMPLEX(double) * flmn, const double *f,
                                    const so3_parameters_t *parameters);

/* reference src/c/so3_core.c:914, :1238, :1655, :1981.  The direct transforms
 * compute the same exact transform as the via-SSHT ones (the reference's own
 * tests hold them equal); here they run the same GPU path, MW sampling only,
 * as in the reference. */
void so3_core_inverse_direct(SO3_COMPLEX(double) * f, const SO3_COMPLEX(double) * flmn,
                             const so3_parameters_t *parameters);
void so3_core_inverse_direct_real(double *f, const SO3_COMPLEX(double) * flmn,
                                  const so3_parameters_t *parameters);
void so3_core_forward_direct(SO3_COMPLEX(double) * flmn, const SO3_COMPLEX(double) * f,
                             const so3_parameters_t *parameters);
void so3_core_forward_direct_real(SO3_COMPLEX(double) * flmn, const double *f,
                                  const so3_parameters_t *parameters);

#ifdef __cplusplus
}
#endif
#endif
