/*
 * so3_conv.h -- harmonic convolutions, drop-in for the reference's
 * include/so3/so3_conv.h:15-48.  Buffers may be host or device pointers.
 */
#ifndef SO3_CONV
#define SO3_CONV

#include "so3_types.h"

#ifdef __cplusplus
extern "C" {
#endif
/* reference src/c/so3_conv.c:154: forward(f), forward(g), harmonic
 * convolution, inverse -- all on the GPU path */
void so3_conv_convolution(SO3_COMPLEX(double) * h, const so3_parameters_t *h_parameter,
                          const SO3_COMPLEX(double) * f, const so3_parameters_t *f_parameter,
                          const SO3_COMPLEX(double) * g, const so3_parameters_t *g_parameter);
/* reference src/c/so3_conv.c:44 */
void so3_conv_harmonic_convolution(SO3_COMPLEX(double) * hlmn, const so3_parameters_t *h_parameters,
                                   const SO3_COMPLEX(double) * flmn,
                                   const so3_parameters_t *f_parameters,
                                   const SO3_COMPLEX(double) * glmn,
                                   const so3_parameters_t *g_parameters);
/* reference src/c/so3_conv.c:104 */
so3_parameters_t so3_conv_get_parameters_of_convolved_lmn(const so3_parameters_t *f_parameters,
                                                          const so3_parameters_t *g_parameters);
/* reference src/c/so3_conv.c:125 */
void so3_conv_get_parameters_of_convolved_lmn_void(so3_parameters_t *h_parameters,
                                                   const so3_parameters_t *f_parameters,
                                                   const so3_parameters_t *g_parameters);
/* reference src/c/so3_conv.c:186 */
void so3_conv_s2toso3_harmonic_convolution(SO3_COMPLEX(double) * hlmn,
                                           const so3_parameters_t *h_parameters,
                                           const SO3_COMPLEX(double) * flm,
                                           const SO3_COMPLEX(double) * glm);
#ifdef __cplusplus
}
#endif
#endif
