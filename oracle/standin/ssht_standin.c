/*
 * ssht_standin.c -- project-written restatement of the SSHT routines the SO3
 * reference calls (see ssht/ssht.h).  TEST INFRASTRUCTURE ONLY: it is the CPU
 * oracle's spin spherical-harmonic transform and the stand-in the reference C
 * is linked against; nothing in the GPU product links it.
 *
 * Sources of the algorithms restated here:
 *  - Wigner Delta(pi/2) by Risbo's half-step recursion (T. Risbo, J. Geodesy
 *    70 (1996) 383), derived from coupling spin j-1/2 with spin 1/2:
 *      d^J_{m'm} = [ sqrt((J+m')(J+m))  c d_{m'-1/2,m-1/2}
 *                  - sqrt((J+m')(J-m))  s d_{m'-1/2,m+1/2}
 *                  + sqrt((J-m')(J+m))  s d_{m'+1/2,m-1/2}
 *                  + sqrt((J-m')(J-m))  c d_{m'+1/2,m+1/2} ] / (2J),
 *    c = cos(beta/2), s = sin(beta/2); evaluated on the eighth m' >= m >= 0
 *    plus the margin its neighbours need, refilled at each integer level from
 *    Delta_{m,m'} = (-1)^{m-m'} Delta_{m'm}, Delta_{m',-m} = (-1)^{l+m'}
 *    Delta_{m'm} and Delta_{-m',m} = (-1)^{l+m} Delta_{m'm}.
 *  - Wigner Delta(pi/2) by Trapani & Navaza (Acta Cryst. A62 (2006) 262),
 *    eqs. 9-11: first row from the previous degree, then a three-term
 *    recursion down each column.
 *  - The MW/MWSS separation-of-variables transforms as stated in the SO3
 *    reference's in-tree direct path (src/c/so3_core.c:1001-1194 inverse,
 *    :1334-1618 forward) and prototypes/ssht/{inverse_sov_fft_phase,
 *    forward_sov_for_fft_phase}.m, specialised to one spin value.
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"
#include "ssht/ssht.h"

typedef double _Complex cplx;

#define SGN(k) (((k) & 1) ? -1.0 : 1.0)

/* ------------------------------------------------------------- dl tables */

#define EXT_OFF 3
#define EXT_STRIDE(L) ((L) + 6)

double *ssht_dl_calloc(int L, ssht_dl_size_t dl_size) {
  switch (dl_size) {
  case SSHT_DL_QUARTER:
    return calloc((size_t)L * L, sizeof(double));
  case SSHT_DL_QUARTER_EXTENDED:
    /* two layers: integer degree and half degree */
    return calloc(2 * (size_t)EXT_STRIDE(L) * EXT_STRIDE(L), sizeof(double));
  case SSHT_DL_HALF:
    return calloc((size_t)L * (2 * L - 1), sizeof(double));
  case SSHT_DL_FULL:
    return calloc((size_t)(2 * L - 1) * (2 * L - 1), sizeof(double));
  }
  return NULL;
}

int ssht_dl_get_offset(int L, ssht_dl_size_t dl_size) {
  switch (dl_size) {
  case SSHT_DL_QUARTER:
    return 0;
  case SSHT_DL_QUARTER_EXTENDED:
    return EXT_OFF;
  default:
    return L - 1;
  }
}

int ssht_dl_get_stride(int L, ssht_dl_size_t dl_size) {
  switch (dl_size) {
  case SSHT_DL_QUARTER:
    return L;
  case SSHT_DL_QUARTER_EXTENDED:
    return EXT_STRIDE(L);
  default:
    return 2 * L - 1;
  }
}

#define A8(u, v) A[((u) + EXT_OFF) * S + ((v) + EXT_OFF)]
#define H8(u, v) H[((u) + EXT_OFF) * S + ((v) + EXT_OFF)]

void ssht_dl_beta_risbo_eighth_table(double *dl8, double beta, int L,
                                     ssht_dl_size_t dl_size, int el,
                                     double *sqrt_tbl, double *signs) {
  (void)dl_size;
  (void)signs;
  int S = EXT_STRIDE(L);
  double *A = dl8, *H = dl8 + (size_t)S * S;
  if (el == 0) {
    A8(0, 0) = 1.0;
    return;
  }
  int l = el - 1; /* A holds degree l on entry */
  double c = cos(beta / 2.0), s = sin(beta / 2.0);

  /* margin of degree l from the eighth */
  for (int u = 0; u <= l; u++)
    for (int v = u + 1; v <= u + 2; v++)
      A8(u, v) = v <= l ? SGN(v - u) * A8(v, u) : 0.0;
  for (int u = 0; u <= l; u++)
    A8(u, -1) = SGN(l + u) * A8(u, 1);
  for (int u = 1; u <= 3; u++)
    for (int v = -1; v <= 2 - u; v++)
      A8(-u, v) = (u <= l) ? SGN(l + v) * A8(u, v) : 0.0;

  /* half degree J = l + 1/2 : H8(xp, yp) holds d_{xp-1/2, yp-1/2} */
  {
    int tJ = 2 * l + 1;
    double inv = 1.0 / tJ;
    for (int yp = 0; yp <= l + 1; yp++) {
      int b = l + yp;
      int x0 = yp - 1 > -l ? yp - 1 : -l;
      for (int xp = x0; xp <= l + 1; xp++) {
        int a = l + xp;
        double v = sqrt_tbl[a] * sqrt_tbl[b] * c * A8(xp - 1, yp - 1) -
                   sqrt_tbl[a] * sqrt_tbl[tJ - b] * s * A8(xp - 1, yp) +
                   sqrt_tbl[tJ - a] * sqrt_tbl[b] * s * A8(xp, yp - 1) +
                   sqrt_tbl[tJ - a] * sqrt_tbl[tJ - b] * c * A8(xp, yp);
        H8(xp, yp) = v * inv;
      }
    }
  }
  /* integer degree el on the eighth 0 <= v <= u <= el */
  {
    int tJ = 2 * el;
    double inv = 1.0 / tJ;
    for (int v = 0; v <= el; v++) {
      int b = el + v;
      for (int u = v; u <= el; u++) {
        int a = el + u;
        double val = sqrt_tbl[a] * sqrt_tbl[b] * c * H8(u, v) -
                     sqrt_tbl[a] * sqrt_tbl[tJ - b] * s * H8(u, v + 1) +
                     sqrt_tbl[tJ - a] * sqrt_tbl[b] * s * H8(u + 1, v) +
                     sqrt_tbl[tJ - a] * sqrt_tbl[tJ - b] * c * H8(u + 1, v + 1);
        A8(u, v) = val * inv;
      }
    }
  }
}

void ssht_dl_beta_risbo_fill_eighth2quarter_table(double *dl, double *dl8, int L,
                                                  ssht_dl_size_t dl_size,
                                                  ssht_dl_size_t dl8_size, int el,
                                                  double *signs) {
  (void)dl_size;
  (void)dl8_size;
  (void)signs;
  int S = EXT_STRIDE(L);
  const double *A = dl8;
  for (int u = 0; u <= el; u++)
    for (int v = 0; v <= el; v++)
      dl[u * L + v] = v <= u ? A8(u, v) : SGN(v - u) * A8(v, u);
}

void ssht_dl_halfpi_trapani_eighth_table(double *dl, int L, ssht_dl_size_t dl_size,
                                         int el, double *sqrt_tbl) {
  (void)dl_size;
  if (el == 0) {
    dl[0] = 1.0;
    return;
  }
  /* first row of degree el from row el-1 of degree el-1 (T&N eqs. 9, 10) */
  double *row = malloc(sizeof(double) * (el + 1));
  row[0] = -sqrt_tbl[2 * el - 1] / sqrt_tbl[2 * el] * dl[(el - 1) * L + 0];
  for (int m = 1; m <= el; m++)
    row[m] = sqrt_tbl[el] * sqrt_tbl[2 * el - 1] /
             (SSHT_SQRT2 * sqrt_tbl[el + m] * sqrt_tbl[el + m - 1]) *
             dl[(el - 1) * L + m - 1];
  for (int m = 0; m <= el; m++)
    dl[el * L + m] = row[m];
  free(row);
  /* down each column (T&N eq. 11) */
  for (int m = 0; m <= el; m++) {
    for (int mp = el - 1; mp >= m; mp--) {
      double t1 = sqrt_tbl[el - mp] * sqrt_tbl[el + mp + 1];
      double nxt2 = 0.0, t2 = 0.0;
      if (mp + 2 <= el) {
        t2 = sqrt_tbl[el - mp - 1] * sqrt_tbl[el + mp + 2];
        nxt2 = dl[(mp + 2) * L + m];
      }
      dl[mp * L + m] = (2.0 * m * dl[(mp + 1) * L + m] - t2 * nxt2) / t1;
    }
  }
}

void ssht_dl_halfpi_trapani_fill_eighth2quarter_table(double *dl, int L,
                                                      ssht_dl_size_t dl_size, int el,
                                                      double *signs) {
  (void)dl_size;
  (void)signs;
  for (int mp = 0; mp <= el; mp++)
    for (int m = mp + 1; m <= el; m++)
      dl[mp * L + m] = SGN(m - mp) * dl[m * L + mp];
}

void ssht_sampling_elm2ind(int *ind, int el, int m) { *ind = el * el + el + m; }

/* ------------------------------------------------- sequential Delta planes */

typedef struct {
  int L, method, cur;
  double *dl, *dl8, *sqrt_tbl, *signs;
} dl_iter;

static void dl_iter_init(dl_iter *it, int L, ssht_dl_method_t method) {
  it->L = L;
  it->method = method;
  it->cur = -1;
  it->dl = ssht_dl_calloc(L, SSHT_DL_QUARTER);
  it->dl8 = method == SSHT_DL_RISBO ? ssht_dl_calloc(L, SSHT_DL_QUARTER_EXTENDED) : NULL;
  it->sqrt_tbl = malloc(sizeof(double) * (2 * L + 2));
  for (int k = 0; k < 2 * L + 2; k++)
    it->sqrt_tbl[k] = sqrt((double)k);
  it->signs = malloc(sizeof(double) * (L + 2));
  for (int k = 0; k < L + 2; k++)
    it->signs[k] = SGN(k);
}

static void dl_iter_free(dl_iter *it) {
  free(it->dl);
  free(it->dl8);
  free(it->sqrt_tbl);
  free(it->signs);
}

/* Advance to degree el (el > cur); the quarter plane of el is left in it->dl. */
static void dl_iter_goto(dl_iter *it, int el) {
  for (int e = it->cur + 1; e <= el; e++) {
    if (it->method == SSHT_DL_RISBO)
      ssht_dl_beta_risbo_eighth_table(it->dl8, SSHT_PION2, it->L, SSHT_DL_QUARTER_EXTENDED, e,
                                      it->sqrt_tbl, it->signs);
    else
      ssht_dl_halfpi_trapani_eighth_table(it->dl, it->L, SSHT_DL_QUARTER, e, it->sqrt_tbl);
  }
  if (it->method == SSHT_DL_RISBO)
    ssht_dl_beta_risbo_fill_eighth2quarter_table(it->dl, it->dl8, it->L, SSHT_DL_QUARTER,
                                                 SSHT_DL_QUARTER_EXTENDED, el, it->signs);
  else
    ssht_dl_halfpi_trapani_fill_eighth2quarter_table(it->dl, it->L, SSHT_DL_QUARTER, el,
                                                     it->signs);
  it->cur = el;
}

/* i^k for integer k */
static cplx ipow(int k) {
  switch (((k % 4) + 4) % 4) {
  case 0:
    return 1.0;
  case 1:
    return I;
  case 2:
    return -1.0;
  default:
    return -I;
  }
}

/* ------------------------------------------------------- spin transforms */

/*
 * Inverse: f(theta_t, phi_p) = sum_{l >= max(L0,|s|)} sum_m flm sY_lm.
 * Fpos[m'][k] (m' >= 0, k = m mod P) = (-1)^s i^{-s-m} sum_l sqrt((2l+1)/4pi)
 *   Delta_{m'm} Delta_{m',-s} flm; m' < 0 from Fpos[-m'] (-1)^{m+s}.
 */
static void inverse_core(cplx *fc, double *fr, const cplx *flm, int L0, int L, int spin,
                         ssht_dl_method_t method, int ss) {
  int real = fr != NULL;
  int P = ss ? 2 * L : 2 * L - 1;
  int nt = ss ? L + 1 : L;
  int el_start = L0 > abs(spin) ? L0 : abs(spin);
  int mlo = real ? 0 : -(L - 1);
  cplx *Fpos = calloc((size_t)L * P, sizeof(cplx));
  cplx *fl = malloc(sizeof(cplx) * (2 * L - 1));
  dl_iter it;
  dl_iter_init(&it, L, method);
  for (int el = el_start; el < L; el++) {
    dl_iter_goto(&it, el);
    const double *dl = it.dl;
    double elfac = sqrt((2.0 * el + 1.0) / (4.0 * SSHT_PI));
    for (int m = -el; m <= el; m++)
      fl[m + L - 1] = SGN(spin) * ipow(-spin - m) * elfac * flm[el * el + el + m];
    int ms = -spin;
    for (int mp = 0; mp <= el; mp++) {
      double dsn = ms >= 0 ? dl[mp * L + ms] : SGN(el + mp) * dl[mp * L - ms];
      double sneg = SGN(el + mp);
      cplx *row = Fpos + (size_t)mp * P;
      const double *drow = dl + mp * L;
      row[0] += dsn * drow[0] * fl[L - 1];
      for (int m = 1; m <= el; m++) {
        row[m] += dsn * drow[m] * fl[L - 1 + m];
        if (!real)
          row[P - m] += dsn * sneg * drow[m] * fl[L - 1 - m];
      }
    }
  }
  dl_iter_free(&it);
  free(fl);

  /* theta synthesis per m column */
  cplx *Ft = calloc((size_t)nt * P, sizeof(cplx));
  cplx *col = malloc(sizeof(cplx) * P);
  so3o_fft1d *eP = so3o_fft1d_create(P);
  for (int m = mlo; m <= L - 1; m++) {
    int k = ((m % P) + P) % P;
    double sgn = SGN(m + spin);
    for (int j = 0; j < P; j++)
      col[j] = 0.0;
    for (int mp = -(L - 1); mp <= L - 1; mp++) {
      cplx v = mp >= 0 ? Fpos[(size_t)mp * P + k] : sgn * Fpos[(size_t)(-mp) * P + k];
      if (!ss)
        v *= cexp(I * mp * SSHT_PI / (2.0 * L - 1.0));
      col[((mp % P) + P) % P] = v;
    }
    so3o_fft1d_exec(eP, col, +1);
    for (int t = 0; t < nt; t++)
      Ft[(size_t)t * P + k] = col[t];
  }
  free(Fpos);
  /* phi synthesis per theta row */
  for (int t = 0; t < nt; t++) {
    cplx *r = Ft + (size_t)t * P;
    if (!real) {
      so3o_fft1d_exec(eP, r, +1);
      memcpy(fc + (size_t)t * P, r, sizeof(cplx) * P);
    } else {
      for (int k = 1; k <= L - 1; k++)
        r[P - k] = conj(r[k]);
      r[0] = creal(r[0]);
      if (ss)
        r[L] = 0.0;
      so3o_fft1d_exec(eP, r, +1);
      for (int p = 0; p < P; p++)
        fr[(size_t)t * P + p] = creal(r[p]);
    }
  }
  so3o_fft1d_destroy(eP);
  free(col);
  free(Ft);
}

/* quadrature weight w(p) = int_0^pi e^{-i p theta} sin(theta) dtheta */
static cplx qweight(int p) {
  if (p == 1)
    return -I * SSHT_PION2;
  if (p == -1)
    return I * SSHT_PION2;
  if (p % 2 == 0)
    return 2.0 / (1.0 - (double)p * p);
  return 0.0;
}

/*
 * Forward: flm = (-1)^s sqrt((2l+1)/4pi) i^{s+m} sum_{m'} Delta_{m'm}
 *   Delta_{m',-s} G[m'][m], G[m'] = 2 pi sum_{m''} Fmm[m''] w(m' - m''),
 * Fmm the 2-D Fourier coefficients of the theta-extended samples
 * (extension f(2pi - theta) = (-1)^{m+s} f(theta) per m column).
 */
static void forward_core(cplx *flm, const cplx *fc, const double *fr, int L0, int L,
                         int spin, ssht_dl_method_t method, int ss) {
  int real = fr != NULL;
  int P = ss ? 2 * L : 2 * L - 1;
  int nt = ss ? L + 1 : L;
  int el_start = L0 > abs(spin) ? L0 : abs(spin);
  int mlo = real ? 0 : -(L - 1);
  so3o_fft1d *eP = so3o_fft1d_create(P);

  /* phi analysis per theta row */
  cplx *Ft = malloc(sizeof(cplx) * (size_t)nt * P);
  for (int t = 0; t < nt; t++) {
    cplx *r = Ft + (size_t)t * P;
    for (int p = 0; p < P; p++)
      r[p] = real ? fr[(size_t)t * P + p] : fc[(size_t)t * P + p];
    so3o_fft1d_exec(eP, r, -1);
    for (int p = 0; p < P; p++)
      r[p] /= P;
  }

  /* convolution kernel in the oversampled domain */
  int Pc = 1;
  while (Pc < 4 * L - 3)
    Pc <<= 1;
  so3o_fft1d *eC = so3o_fft1d_create(Pc);
  cplx *wr = calloc(Pc, sizeof(cplx));
  for (int p = -2 * (L - 1); p <= 2 * (L - 1); p++)
    wr[((p % Pc) + Pc) % Pc] = qweight(p);
  so3o_fft1d_exec(eC, wr, +1);
  for (int r = 0; r < Pc; r++)
    wr[r] *= 2.0 * SSHT_PI / Pc;

  /* theta extension, analysis and weighting per m column */
  cplx *Gs = calloc((size_t)L * P, sizeof(cplx)); /* Gs[m'][k], m' >= 0 */
  cplx *col = malloc(sizeof(cplx) * P);
  cplx *cv = malloc(sizeof(cplx) * Pc);
  for (int m = mlo; m <= L - 1; m++) {
    int k = ((m % P) + P) % P;
    double sgn = SGN(m + spin);
    for (int t = 0; t < P; t++) {
      if (t < nt)
        col[t] = Ft[(size_t)t * P + k];
      else
        col[t] = sgn * Ft[(size_t)(ss ? 2 * L - t : 2 * L - 2 - t) * P + k];
    }
    so3o_fft1d_exec(eP, col, -1);
    for (int j = 0; j < Pc; j++)
      cv[j] = 0.0;
    for (int mpp = -(L - 1); mpp <= L - 1; mpp++) {
      cplx v = col[((mpp % P) + P) % P] / P;
      if (!ss)
        v *= cexp(-I * mpp * SSHT_PI / (2.0 * L - 1.0));
      cv[((mpp % Pc) + Pc) % Pc] = v;
    }
    so3o_fft1d_exec(eC, cv, +1);
    for (int r = 0; r < Pc; r++)
      cv[r] *= wr[r];
    so3o_fft1d_exec(eC, cv, -1);
    Gs[k] = cv[0];
    for (int mp = 1; mp <= L - 1; mp++)
      Gs[(size_t)mp * P + k] = cv[mp] + sgn * cv[Pc - mp];
  }
  free(cv);
  free(col);
  free(wr);
  free(Ft);
  so3o_fft1d_destroy(eC);
  so3o_fft1d_destroy(eP);

  /* Delta contraction */
  for (int i = 0; i < L * L; i++)
    flm[i] = 0.0;
  cplx *acc = malloc(sizeof(cplx) * (2 * L - 1));
  dl_iter it;
  dl_iter_init(&it, L, method);
  int ms = -spin;
  for (int el = el_start; el < L; el++) {
    dl_iter_goto(&it, el);
    const double *dl = it.dl;
    for (int m = -el; m <= el; m++)
      acc[m + L - 1] = 0.0;
    for (int mp = 0; mp <= el; mp++) {
      double dsn = ms >= 0 ? dl[mp * L + ms] : SGN(el + mp) * dl[mp * L - ms];
      double sneg = SGN(el + mp);
      const double *drow = dl + mp * L;
      const cplx *grow = Gs + (size_t)mp * P;
      acc[L - 1] += dsn * drow[0] * grow[0];
      for (int m = 1; m <= el; m++) {
        acc[L - 1 + m] += dsn * drow[m] * grow[m];
        if (!real)
          acc[L - 1 - m] += dsn * sneg * drow[m] * grow[P - m];
      }
    }
    double elfac = SGN(spin) * sqrt((2.0 * el + 1.0) / (4.0 * SSHT_PI));
    for (int m = real ? 0 : -el; m <= el; m++)
      flm[el * el + el + m] = elfac * ipow(spin + m) * acc[L - 1 + m];
    if (real)
      for (int m = 1; m <= el; m++)
        flm[el * el + el - m] = SGN(m) * conj(flm[el * el + el + m]);
  }
  dl_iter_free(&it);
  free(acc);
  free(Gs);
}

void ssht_core_mw_lb_inverse_sov_sym(cplx *f, const cplx *flm, int L0, int L, int spin,
                                     ssht_dl_method_t dl_method, int verbosity) {
  (void)verbosity;
  inverse_core(f, NULL, flm, L0, L, spin, dl_method, 0);
}
void ssht_core_mw_lb_inverse_sov_sym_ss(cplx *f, const cplx *flm, int L0, int L, int spin,
                                        ssht_dl_method_t dl_method, int verbosity) {
  (void)verbosity;
  inverse_core(f, NULL, flm, L0, L, spin, dl_method, 1);
}
void ssht_core_mw_lb_inverse_sov_sym_real(double *f, const cplx *flm, int L0, int L,
                                          ssht_dl_method_t dl_method, int verbosity) {
  (void)verbosity;
  inverse_core(NULL, f, flm, L0, L, 0, dl_method, 0);
}
void ssht_core_mw_lb_inverse_sov_sym_ss_real(double *f, const cplx *flm, int L0, int L,
                                             ssht_dl_method_t dl_method, int verbosity) {
  (void)verbosity;
  inverse_core(NULL, f, flm, L0, L, 0, dl_method, 1);
}
void ssht_core_mw_lb_forward_sov_conv_sym(cplx *flm, const cplx *f, int L0, int L, int spin,
                                          ssht_dl_method_t dl_method, int verbosity) {
  (void)verbosity;
  forward_core(flm, f, NULL, L0, L, spin, dl_method, 0);
}
void ssht_core_mw_lb_forward_sov_conv_sym_ss(cplx *flm, const cplx *f, int L0, int L,
                                             int spin, ssht_dl_method_t dl_method,
                                             int verbosity) {
  (void)verbosity;
  forward_core(flm, f, NULL, L0, L, spin, dl_method, 1);
}
void ssht_core_mw_lb_forward_sov_conv_sym_real(cplx *flm, const double *f, int L0, int L,
                                               ssht_dl_method_t dl_method, int verbosity) {
  (void)verbosity;
  forward_core(flm, NULL, f, L0, L, 0, dl_method, 0);
}
void ssht_core_mw_lb_forward_sov_conv_sym_ss_real(cplx *flm, const double *f, int L0, int L,
                                                  ssht_dl_method_t dl_method,
                                                  int verbosity) {
  (void)verbosity;
  forward_core(flm, NULL, f, L0, L, 0, dl_method, 1);
}

/* Exposed for tests: the quarter plane of degree el by either recursion. */
void so3o_dl_quarter_plane(double *out, int L, int el, int method) {
  dl_iter it;
  dl_iter_init(&it, L, (ssht_dl_method_t)method);
  dl_iter_goto(&it, el);
  for (int i = 0; i <= el; i++)
    for (int j = 0; j <= el; j++)
      out[i * (el + 1) + j] = it.dl[i * L + j];
  dl_iter_free(&it);
}
