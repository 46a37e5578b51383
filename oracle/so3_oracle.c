/*
 * so3_oracle.c -- CPU restatement of the SO3 reference's fast Wigner
 * transform path, used ONLY as the checker in tests, in the smoke check and
 * as the timed CPU baseline.  It is test infrastructure, not the product:
 * the GPU library never links or calls it.
 *
 * Every function names the reference lines it restates (paths relative to
 * the astro-informatics/so3 tree).  The per-spin transforms and Wigner Delta
 * recursions come from the project's SSHT stand-in (standin/ssht_standin.c),
 * the FFTs from the project's FFT engine (standin/fftw_standin.c).
 */
#include <complex.h>
#include <math.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "standin/fftw3.h"
#include "standin/ssht/ssht.h"
#include "so3/so3_types.h"

typedef double _Complex cplx;
#define SGN(k) (((k) & 1) ? -1.0 : 1.0)
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#define MIN(a, b) ((a) < (b) ? (a) : (b))

static void oracle_fail(const char *msg) {
  fprintf(stderr, "ORACLE ERROR: %s\n", msg);
  exit(1);
}

/* ------------------------------------------------ index helpers
 * restating src/c/so3_sampling.c:316-339 (flmn_size), :369-426 (elmn2ind),
 * :455-542 (ind2elmn), :571-650 (_real variants), :677-808 (loop values),
 * :835-882 (is_elmn_non_zero). */

int oracle_flmn_size(const so3_parameters_t *p) {
  int L = p->L, N = p->N;
  if (p->storage == SO3_STORAGE_PADDED)
    return p->reality ? N * L * L : (2 * N - 1) * L * L;
  return p->reality ? N * (6 * L * L - (N - 1) * (2 * N - 1)) / 6
                    : (2 * N - 1) * (3 * L * L - N * (N - 1)) / 3;
}

int oracle_elmn2ind(int el, int m, int n, const so3_parameters_t *p) {
  int L = p->L, N = p->N, an = abs(n), off;
  if (p->storage == SO3_STORAGE_PADDED) {
    off = p->n_order == SO3_N_ORDER_ZERO_FIRST ? (n < 0 ? -2 * n - 1 : 2 * n) * L * L
                                              : (N - 1 + n) * L * L;
    return off + el * el + el + m;
  }
  if (an > el)
    oracle_fail("compact storage has no entry with |n| > l");
  if (p->n_order == SO3_N_ORDER_ZERO_FIRST) {
    off = (2 * an - 1) * (3 * L * L - an * (an - 1)) / 3;
    if (n >= 0)
      off += L * L - n * n;
  } else {
    off = (N - 1 + n) * L * L - (2 * N - 1) * (N - 1) * N / 6;
    if (n <= 0)
      off += an * (2 * an + 1) * (an + 1) / 6;
    else
      off -= an * (2 * an - 1) * (an - 1) / 6;
  }
  return off + el * el - n * n + el + m;
}

int oracle_elmn2ind_real(int el, int m, int n, const so3_parameters_t *p) {
  so3_parameters_t q = *p;
  q.n_order = SO3_N_ORDER_NEGATIVE_FIRST;
  return oracle_elmn2ind(el, m, n, &q) - oracle_elmn2ind(0, 0, 0, &q);
}

void oracle_ind2elmn(int *el, int *m, int *n, int ind, const so3_parameters_t *p) {
  int L = p->L, N = p->N;
  if (p->storage == SO3_STORAGE_PADDED) {
    int blk = ind / (L * L);
    if (p->n_order == SO3_N_ORDER_ZERO_FIRST)
      *n = (blk % 2) ? -(blk + 1) / 2 : blk / 2;
    else
      *n = blk - (N - 1);
    ind %= L * L;
  } else {
    int off;
    if (p->n_order == SO3_N_ORDER_ZERO_FIRST) {
      *n = 0;
      off = 0;
      while (ind + off >= L * L) {
        ind -= L * L - off;
        if (*n >= 0) {
          *n = -(*n + 1);
          off = (*n) * (*n);
        } else {
          *n = -(*n);
        }
      }
    } else {
      *n = -N + 1;
      off = (*n) * (*n);
      while (ind + off >= L * L) {
        ind -= L * L - off;
        (*n)++;
        off = (*n) * (*n);
      }
    }
    ind += off;
  }
  *el = (int)sqrt((double)ind);
  *m = ind - (*el) * (*el) - *el;
}

void oracle_ind2elmn_real(int *el, int *m, int *n, int ind, const so3_parameters_t *p) {
  so3_parameters_t q = *p;
  q.n_order = SO3_N_ORDER_NEGATIVE_FIRST;
  oracle_ind2elmn(el, m, n, ind + oracle_elmn2ind(0, 0, 0, &q), &q);
}

void oracle_n_loop_values(int *s, int *e, int *inc, const so3_parameters_t *p) {
  int N = p->N;
  if (p->reality) {
    switch (p->n_mode) {
    case SO3_N_MODE_ALL:
    case SO3_N_MODE_L:
      *s = 0, *e = N - 1, *inc = 1;
      break;
    case SO3_N_MODE_EVEN:
      *s = 0, *e = ((N - 1) % 2 == 0) ? N - 1 : N - 2, *inc = 2;
      break;
    case SO3_N_MODE_ODD:
      *s = 1, *e = ((N - 1) % 2 != 0) ? N - 1 : N - 2, *inc = 2;
      break;
    case SO3_N_MODE_MAXIMUM:
      *s = N - 1, *e = N - 1, *inc = 1;
      break;
    default:
      oracle_fail("invalid n-mode");
    }
  } else {
    switch (p->n_mode) {
    case SO3_N_MODE_ALL:
    case SO3_N_MODE_L:
      *s = -N + 1, *e = N - 1, *inc = 1;
      break;
    case SO3_N_MODE_EVEN:
      *s = ((N - 1) % 2 == 0) ? -N + 1 : -N + 2;
      *e = ((N - 1) % 2 == 0) ? N - 1 : N - 2;
      *inc = 2;
      break;
    case SO3_N_MODE_ODD:
      *s = ((N - 1) % 2 != 0) ? -N + 1 : -N + 2;
      *e = ((N - 1) % 2 != 0) ? N - 1 : N - 2;
      *inc = 2;
      break;
    case SO3_N_MODE_MAXIMUM:
      *s = -N + 1, *e = N - 1, *inc = N > 1 ? 2 * N - 2 : 1;
      break;
    default:
      oracle_fail("invalid n-mode");
    }
  }
}

bool oracle_is_elmn_non_zero(int el, int m, int n, const so3_parameters_t *p) {
  int s, e, inc;
  oracle_n_loop_values(&s, &e, &inc, p);
  if (n < s || n > e || (n - s) % inc)
    return false;
  int es = MAX(p->L0, abs(n)), ee = p->n_mode == SO3_N_MODE_L ? abs(n) : p->L - 1;
  if (el < es || el > ee)
    return false;
  return m >= -el && m <= el;
}

/* n skipped by the via-SSHT loops (src/c/so3_core.c:166-170) */
static int skip_n(const so3_parameters_t *p, int n) {
  return (p->n_mode == SO3_N_MODE_EVEN && (n & 1)) ||
         (p->n_mode == SO3_N_MODE_ODD && !(n & 1)) ||
         (p->n_mode == SO3_N_MODE_MAXIMUM && abs(n) < p->N - 1);
}

static int plane_stride(const so3_parameters_t *p) {
  return p->sampling_scheme == SO3_SAMPLING_MW ? p->L * (2 * p->L - 1)
                                                : (p->L + 1) * 2 * p->L;
}

typedef void (*inv_c_fn)(cplx *, const cplx *, int, int, int, ssht_dl_method_t, int);
typedef void (*inv_r_fn)(double *, const cplx *, int, int, ssht_dl_method_t, int);
typedef void (*fwd_c_fn)(cplx *, const cplx *, int, int, int, ssht_dl_method_t, int);
typedef void (*fwd_r_fn)(cplx *, const double *, int, int, ssht_dl_method_t, int);

/* Block n of flmn copied into a full L*L array (src/c/so3_core.c:172-188). */
static void load_block(cplx *flm, const cplx *flmn, int n, const so3_parameters_t *p, int real) {
  int L = p->L;
  if (p->storage == SO3_STORAGE_PADDED) {
    int ind = real ? oracle_elmn2ind_real(0, 0, n, p) : oracle_elmn2ind(0, 0, n, p);
    memcpy(flm, flmn + ind, sizeof(cplx) * L * L);
  } else {
    int an = abs(n);
    int ind = real ? oracle_elmn2ind_real(an, -an, n, p) : oracle_elmn2ind(an, -an, n, p);
    for (int i = 0; i < n * n; i++)
      flm[i] = 0.0;
    memcpy(flm + n * n, flmn + ind, sizeof(cplx) * (L * L - n * n));
  }
}

/* src/c/so3_core.c:51-228 */
void oracle_inverse_via_ssht(cplx *f, const cplx *flmn, const so3_parameters_t *p) {
  int L0 = p->L0, L = p->L, N = p->N;
  int stride = plane_stride(p);
  inv_c_fn ssht = p->sampling_scheme == SO3_SAMPLING_MW ? ssht_core_mw_lb_inverse_sov_sym
                                                        : ssht_core_mw_lb_inverse_sov_sym_ss;
  int ng = p->steerable ? 2 * N : 2 * N - 1;
  cplx *fn = calloc((size_t)ng * stride, sizeof(cplx));
  cplx *flm = malloc(sizeof(cplx) * L * L);
  for (int n = -N + 1; n <= N - 1; n++) {
    if (skip_n(p, n))
      continue;
    int L0e = MAX(L0, abs(n));
    load_block(flm, flmn, n, p, 0);
    for (int el = L0e; el < L; el++) {
      double fac = sqrt((2.0 * el + 1.0) / (16.0 * pow(SO3_PI, 3.0)));
      for (int m = -el; m <= el; m++)
        flm[el * el + el + m] *= fac;
    }
    int plane = n < 0 ? n + ng : n;
    cplx *dst = fn + (size_t)plane * stride;
    ssht(dst, flm, L0e, L, -n, p->dl_method, 0);
    if (n & 1)
      for (int i = 0; i < stride; i++)
        dst[i] = -dst[i];
  }
  free(flm);
  so3o_fft1d *e = so3o_fft1d_create(ng);
  so3o_fft1d_exec_strided(e, fn, stride, stride, 1, +1);
  so3o_fft1d_destroy(e);
  int nout = p->steerable ? N : ng;
  memcpy(f, fn, sizeof(cplx) * (size_t)nout * stride);
  free(fn);
}

/* src/c/so3_core.c:246-441 */
void oracle_forward_via_ssht(cplx *flmn, const cplx *f, const so3_parameters_t *p) {
  int L0 = p->L0, L = p->L, N = p->N;
  int stride = plane_stride(p);
  fwd_c_fn ssht = p->sampling_scheme == SO3_SAMPLING_MW
                      ? ssht_core_mw_lb_forward_sov_conv_sym
                      : ssht_core_mw_lb_forward_sov_conv_sym_ss;
  int ng = 2 * N - 1;
  cplx *fn = calloc((size_t)ng * stride, sizeof(cplx));
  if (p->steerable) {
    for (int n = -N + 1; n < N; n += 2) {
      int plane = n < 0 ? n + 2 * N - 1 : n;
      for (int g = 0; g < N; g++) {
        double gamma = g * SO3_PI / N;
        cplx ph = cexp(-I * n * gamma);
        for (int i = 0; i < stride; i++)
          fn[(size_t)plane * stride + i] += (2 * SO3_PI / N) * f[(size_t)g * stride + i] * ph;
      }
    }
  } else {
    memcpy(fn, f, sizeof(cplx) * (size_t)ng * stride);
    so3o_fft1d *e = so3o_fft1d_create(ng);
    so3o_fft1d_exec_strided(e, fn, stride, stride, 1, -1);
    so3o_fft1d_destroy(e);
    double factor = 2 * SO3_PI / (double)ng;
    for (size_t i = 0; i < (size_t)ng * stride; i++)
      fn[i] *= factor;
  }
  cplx *flm = malloc(sizeof(cplx) * L * L);
  for (int n = -N + 1; n <= N - 1; n++) {
    if (skip_n(p, n))
      continue;
    int L0e = MAX(L0, abs(n));
    int plane = n < 0 ? n + ng : n;
    ssht(flm, fn + (size_t)plane * stride, L0e, L, -n, p->dl_method, 0);
    int ind, first;
    if (p->storage == SO3_STORAGE_PADDED) {
      ind = oracle_elmn2ind(0, 0, n, p);
      first = 0;
    } else {
      ind = oracle_elmn2ind(abs(n), -abs(n), n, p) - n * n;
      first = n * n;
    }
    for (int i = first; i < L * L; i++)
      flmn[ind + i] = flm[i];
    double sign = SGN(n);
    for (int el = L0e; el < L; el++) {
      double fac = sign * sqrt(4.0 * SO3_PI / (2.0 * el + 1.0));
      for (int m = -el; m <= el; m++)
        flmn[ind + el * el + el + m] *= fac;
    }
  }
  free(flm);
  free(fn);
}

/* src/c/so3_core.c:458-657 */
void oracle_inverse_via_ssht_real(double *f, const cplx *flmn, const so3_parameters_t *p) {
  int L0 = p->L0, L = p->L, N = p->N;
  int stride = plane_stride(p);
  int mw = p->sampling_scheme == SO3_SAMPLING_MW;
  inv_c_fn cssht = mw ? ssht_core_mw_lb_inverse_sov_sym : ssht_core_mw_lb_inverse_sov_sym_ss;
  inv_r_fn rssht =
      mw ? ssht_core_mw_lb_inverse_sov_sym_real : ssht_core_mw_lb_inverse_sov_sym_ss_real;
  int ng = 2 * N - 1;
  cplx *fn = calloc((size_t)N * stride, sizeof(cplx));
  cplx *flm = malloc(sizeof(cplx) * L * L);
  for (int n = 0; n <= N - 1; n++) {
    if (skip_n(p, n))
      continue;
    int L0e = MAX(L0, n);
    load_block(flm, flmn, n, p, 1);
    for (int el = L0e; el < L; el++) {
      double fac = sqrt((2.0 * el + 1.0) / (16.0 * pow(SO3_PI, 3.0)));
      for (int m = -el; m <= el; m++)
        flm[el * el + el + m] *= fac;
    }
    cplx *dst = fn + (size_t)n * stride;
    if (N > 1 || n) {
      cssht(dst, flm, L0e, L, -n, p->dl_method, 0);
    } else {
      double *fr = calloc(stride, sizeof(double));
      rssht(fr, flm, L0e, L, p->dl_method, 0);
      for (int i = 0; i < stride; i++)
        dst[i] = fr[i];
      free(fr);
    }
    if (n & 1)
      for (int i = 0; i < stride; i++)
        dst[i] = -dst[i];
  }
  free(flm);
  /* c2r over gamma: f[g] = Re sum_{k} X_k e^{+2 pi i k g/ng}, X Hermitian */
  so3o_fft1d *e = so3o_fft1d_create(ng);
  cplx *col = malloc(sizeof(cplx) * ng);
  for (int i = 0; i < stride; i++) {
    col[0] = creal(fn[i]);
    for (int k = 1; k < N; k++) {
      col[k] = fn[(size_t)k * stride + i];
      col[ng - k] = conj(col[k]);
    }
    so3o_fft1d_exec(e, col, +1);
    for (int g = 0; g < ng; g++)
      f[(size_t)g * stride + i] = creal(col[g]);
  }
  free(col);
  so3o_fft1d_destroy(e);
  free(fn);
}

/* src/c/so3_core.c:675-897 */
void oracle_forward_via_ssht_real(cplx *flmn, const double *f, const so3_parameters_t *p) {
  int L0 = p->L0, L = p->L, N = p->N;
  int stride = plane_stride(p);
  int mw = p->sampling_scheme == SO3_SAMPLING_MW;
  fwd_c_fn cssht =
      mw ? ssht_core_mw_lb_forward_sov_conv_sym : ssht_core_mw_lb_forward_sov_conv_sym_ss;
  fwd_r_fn rssht = mw ? ssht_core_mw_lb_forward_sov_conv_sym_real
                      : ssht_core_mw_lb_forward_sov_conv_sym_ss_real;
  int ng = 2 * N - 1;
  cplx *fn = malloc(sizeof(cplx) * (size_t)N * stride);
  so3o_fft1d *e = so3o_fft1d_create(ng);
  cplx *col = malloc(sizeof(cplx) * ng);
  double factor = 2 * SO3_PI / (double)ng;
  for (int i = 0; i < stride; i++) {
    for (int g = 0; g < ng; g++)
      col[g] = f[(size_t)g * stride + i];
    so3o_fft1d_exec(e, col, -1);
    for (int k = 0; k < N; k++)
      fn[(size_t)k * stride + i] = col[k] * factor;
  }
  free(col);
  so3o_fft1d_destroy(e);
  cplx *flm = malloc(sizeof(cplx) * L * L);
  for (int n = 0; n <= N - 1; n++) {
    if (skip_n(p, n))
      continue;
    int L0e = MAX(L0, n);
    if (N > 1) {
      cssht(flm, fn + (size_t)n * stride, L0e, L, -n, p->dl_method, 0);
    } else {
      double *fr = malloc(sizeof(double) * stride);
      for (int j = 0; j < stride; j++)
        fr[j] = creal(fn[j]);
      rssht(flm, fr, L0e, L, p->dl_method, 0);
      free(fr);
    }
    int ind, first;
    if (p->storage == SO3_STORAGE_PADDED) {
      ind = oracle_elmn2ind_real(0, 0, n, p);
      first = 0;
    } else {
      ind = oracle_elmn2ind_real(n, -n, n, p) - n * n;
      first = n * n;
    }
    for (int i = first; i < L * L; i++)
      flmn[ind + i] = flm[i];
    double sign = SGN(n);
    for (int el = L0e; el < L; el++) {
      double fac = sign * sqrt(4.0 * SO3_PI / (2.0 * el + 1.0));
      for (int m = -el; m <= el; m++)
        flmn[ind + el * el + el + m] *= fac;
    }
  }
  free(flm);
  free(fn);
}

/* ------------------------------------------------ convolutions
 * src/c/so3_conv.c:44-90 */
void oracle_harmonic_convolution(cplx *hlmn, const so3_parameters_t *hp, const cplx *flmn,
                                 const so3_parameters_t *fp, const cplx *glmn,
                                 const so3_parameters_t *gp) {
  int ns, ne, ni, ks, ke, ki;
  oracle_n_loop_values(&ns, &ne, &ni, hp);
  oracle_n_loop_values(&ks, &ke, &ki, fp);
  for (int n = ns; n <= ne; n += ni) {
    int es = MAX(hp->L0, abs(n)), ee = hp->n_mode == SO3_N_MODE_L ? abs(n) : hp->L - 1;
    for (int el = es; el <= ee; el++)
      for (int m = -el; m <= el; m++) {
        int ih = hp->reality ? oracle_elmn2ind_real(el, m, n, hp) : oracle_elmn2ind(el, m, n, hp);
        cplx acc = 0.0;
        for (int k = ks; k <= ke; k += ki) {
          if (!oracle_is_elmn_non_zero(el, n, k, gp))
            continue;
          int iff = fp->reality ? oracle_elmn2ind_real(el, m, k, fp) : oracle_elmn2ind(el, m, k, fp);
          int ig = gp->reality ? oracle_elmn2ind_real(el, n, k, gp) : oracle_elmn2ind(el, n, k, gp);
          acc += flmn[iff] * conj(glmn[ig]);
        }
        hlmn[ih] = acc;
      }
  }
}

/* src/c/so3_conv.c:104-122 */
so3_parameters_t oracle_convolved_parameters(const so3_parameters_t *fp,
                                             const so3_parameters_t *gp) {
  if (fp->sampling_scheme != gp->sampling_scheme || fp->n_order != gp->n_order ||
      fp->storage != gp->storage || fp->n_mode != gp->n_mode || fp->reality != gp->reality)
    oracle_fail("f and g parameters differ");
  so3_parameters_t h = *fp;
  h.L = MIN(fp->L, gp->L);
  h.N = h.L;
  h.L0 = MAX(fp->L0, gp->L0);
  return h;
}

/* src/c/so3_conv.c:186-215 */
void oracle_s2toso3_harmonic_convolution(cplx *hlmn, const so3_parameters_t *hp,
                                         const cplx *flm, const cplx *glm) {
  int len = oracle_flmn_size(hp);
  for (int i = 0; i < len; i++) {
    int el, m, n;
    if (hp->reality)
      oracle_ind2elmn_real(&el, &m, &n, i, hp);
    else
      oracle_ind2elmn(&el, &m, &n, i, hp);
    if (abs(m) <= el && abs(n) <= el)
      hlmn[i] = flm[el * el + el + m] * conj(glm[el * el + el + n]) *
                (8 * SO3_PI * SO3_PI / (2 * el + 1));
    else
      hlmn[i] = 0.0;
  }
}

/* quarter Delta plane of one degree, for recursion tests */
void so3o_dl_quarter_plane(double *out, int L, int el, int method);
void oracle_dl_plane(double *out, int L, int el, int method) {
  so3o_dl_quarter_plane(out, L, el, method);
}

/* plain complex DFT of a strided batch, for FFT tests */
void oracle_dft_strided(cplx *x, int n, int howmany, long stride, long dist, int sign) {
  so3o_fft1d *e = so3o_fft1d_create(n);
  so3o_fft1d_exec_strided(e, x, howmany, stride, dist, sign);
  so3o_fft1d_destroy(e);
}
