/*
 * ssht/ssht.h -- project-written stand-in for the subset of the SSHT library
 * (astro-informatics/ssht, conan range ssht/[>=1.3.7], not vendored by SO3)
 * that the SO3 reference sources call.  TEST INFRASTRUCTURE ONLY.
 *
 * Call sites in the reference: src/c/so3_core.c:100-111, :294-305, :509-520,
 * :728-739 (spin transforms), :983-1035 and :1496-1547 (Wigner Delta
 * recursions), src/c/so3_conv.c:205-206 (ssht_sampling_elm2ind).
 *
 * Conventions (SSHT's published ones, restated):
 *   sY_lm(theta, phi) = (-1)^s sqrt((2l+1)/(4 pi)) e^{i m phi} d^l_{m,-s}(theta)
 *   d^l_{mn}(beta) = i^{n-m} sum_{m'} Delta^l_{m'm} Delta^l_{m'n} e^{i m' beta},
 *   Delta^l_{m'm} = d^l_{m'm}(pi/2) in the standard (Condon-Shortley) phase.
 *   Quarter table: dl[m' * stride + m + offset] = Delta^l_{m'm}, 0 <= m', m <= l
 *   (offset 0, stride L).
 *   MW sampling: theta_t = pi (2t+1)/(2L-1), t < L; phi_p = 2 pi p/(2L-1).
 *   MWSS sampling: theta_t = pi t / L, t <= L; phi_p = pi p / L, p < 2L.
 *   Samples are stored f[t * nphi + p].
 */
#ifndef SO3_ORACLE_SSHT_STANDIN_H
#define SO3_ORACLE_SSHT_STANDIN_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SSHT_PI 3.141592653589793238462643383279502884197
#define SSHT_PION2 1.570796326794896619231321691639751442099
#define SSHT_SQRT2 1.41421356237309504880168872420969807856967

#ifndef SO3_SSHT_DL_METHOD_T_DEFINED
#define SO3_SSHT_DL_METHOD_T_DEFINED
typedef enum { SSHT_DL_RISBO = 0, SSHT_DL_TRAPANI = 1 } ssht_dl_method_t;
#endif

typedef enum {
  SSHT_DL_QUARTER = 0,
  SSHT_DL_QUARTER_EXTENDED,
  SSHT_DL_HALF,
  SSHT_DL_FULL
} ssht_dl_size_t;

double *ssht_dl_calloc(int L, ssht_dl_size_t dl_size);
int ssht_dl_get_offset(int L, ssht_dl_size_t dl_size);
int ssht_dl_get_stride(int L, ssht_dl_size_t dl_size);

void ssht_dl_beta_risbo_eighth_table(double *dl8, double beta, int L,
                                     ssht_dl_size_t dl_size, int el,
                                     double *sqrt_tbl, double *signs);
void ssht_dl_beta_risbo_fill_eighth2quarter_table(double *dl, double *dl8, int L,
                                                  ssht_dl_size_t dl_size,
                                                  ssht_dl_size_t dl8_size, int el,
                                                  double *signs);
void ssht_dl_halfpi_trapani_eighth_table(double *dl, int L, ssht_dl_size_t dl_size,
                                         int el, double *sqrt_tbl);
void ssht_dl_halfpi_trapani_fill_eighth2quarter_table(double *dl, int L,
                                                      ssht_dl_size_t dl_size, int el,
                                                      double *signs);

void ssht_core_mw_lb_inverse_sov_sym(double _Complex *f, const double _Complex *flm,
                                     int L0, int L, int spin,
                                     ssht_dl_method_t dl_method, int verbosity);
void ssht_core_mw_lb_inverse_sov_sym_ss(double _Complex *f,
                                        const double _Complex *flm, int L0, int L,
                                        int spin, ssht_dl_method_t dl_method,
                                        int verbosity);
void ssht_core_mw_lb_inverse_sov_sym_real(double *f, const double _Complex *flm,
                                          int L0, int L, ssht_dl_method_t dl_method,
                                          int verbosity);
void ssht_core_mw_lb_inverse_sov_sym_ss_real(double *f, const double _Complex *flm,
                                             int L0, int L,
                                             ssht_dl_method_t dl_method,
                                             int verbosity);
void ssht_core_mw_lb_forward_sov_conv_sym(double _Complex *flm,
                                          const double _Complex *f, int L0, int L,
                                          int spin, ssht_dl_method_t dl_method,
                                          int verbosity);
void ssht_core_mw_lb_forward_sov_conv_sym_ss(double _Complex *flm,
                                             const double _Complex *f, int L0, int L,
                                             int spin, ssht_dl_method_t dl_method,
                                             int verbosity);
void ssht_core_mw_lb_forward_sov_conv_sym_real(double _Complex *flm, const double *f,
                                               int L0, int L,
                                               ssht_dl_method_t dl_method,
                                               int verbosity);
void ssht_core_mw_lb_forward_sov_conv_sym_ss_real(double _Complex *flm,
                                                  const double *f, int L0, int L,
                                                  ssht_dl_method_t dl_method,
                                                  int verbosity);

void ssht_sampling_elm2ind(int *ind, int el, int m);

#ifdef __cplusplus
}
#endif
#endif
