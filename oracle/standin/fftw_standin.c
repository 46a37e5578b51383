/*
 * fftw_standin.c -- project-written implementation of the FFTW API subset
 * declared in fftw3.h.  TEST INFRASTRUCTURE ONLY (oracle and reference build).
 *
 * Engine: self-sorting (Stockham) mixed-radix DFT with radices 4, 2 and odd
 * primes up to 31 (odd radices use the sum/difference pairing of inputs
 * r and R-r), and Bluestein's chirp-z algorithm over a power-of-two length
 * for lengths with a prime factor above 31.  Twiddles are evaluated in long
 * double and rounded once.  FFTW itself is not present in this tree; the
 * semantics implemented are FFTW's documented ones.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

typedef double _Complex cplx;
#define MAXRAD 31

struct so3o_fft1d {
  int n;
  int nrad;
  int rad[64];
  cplx *roots; /* e^{-2 pi i k / n}, k in [0, n) */
  cplx *buf;   /* Stockham ping-pong scratch, length n (or m for Bluestein) */
  int blue;
  int m;
  struct so3o_fft1d *sub;
  cplx *chirp; /* e^{-i pi k^2 / n}, k in [0, n) */
  cplx *kern;  /* FFT_m of the conjugate chirp kernel, scaled by 1/m */
  cplx *bwork; /* Bluestein work array of length m */
};

static cplx unit_root(long num, long den) {
  /* e^{-2 pi i num / den} evaluated in long double */
  long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)num / (long double)den;
  return (double)cosl(a) - I * (double)sinl(a);
}

static int factorize(int n, int *rad) {
  int nr = 0;
  while (n % 4 == 0) {
    rad[nr++] = 4;
    n /= 4;
  }
  while (n % 2 == 0) {
    rad[nr++] = 2;
    n /= 2;
  }
  for (int p = 3; p <= MAXRAD && n > 1; p += 2)
    while (n % p == 0) {
      rad[nr++] = p;
      n /= p;
    }
  return n > 1 ? -1 : nr;
}

so3o_fft1d *so3o_fft1d_create(int n) {
  so3o_fft1d *p = calloc(1, sizeof *p);
  p->n = n;
  int nr = factorize(n, p->rad);
  if (nr >= 0) {
    p->nrad = nr;
    p->roots = malloc(sizeof(cplx) * n);
    for (int k = 0; k < n; k++)
      p->roots[k] = unit_root(k, n);
    p->buf = malloc(sizeof(cplx) * n);
  } else {
    int m = 1;
    while (m < 2 * n - 1)
      m <<= 1;
    p->blue = 1;
    p->m = m;
    p->sub = so3o_fft1d_create(m);
    p->chirp = malloc(sizeof(cplx) * n);
    p->kern = calloc(m, sizeof(cplx));
    p->bwork = malloc(sizeof(cplx) * m);
    for (int k = 0; k < n; k++) {
      long kk = ((long)k * k) % (2L * n);
      p->chirp[k] = unit_root(kk, 2L * n); /* e^{-i pi k^2/n} */
    }
    p->kern[0] = conj(p->chirp[0]);
    for (int k = 1; k < n; k++)
      p->kern[k] = p->kern[m - k] = conj(p->chirp[k]);
    so3o_fft1d_exec(p->sub, p->kern, -1);
    for (int k = 0; k < m; k++)
      p->kern[k] /= m;
  }
  return p;
}

void so3o_fft1d_destroy(so3o_fft1d *p) {
  if (!p)
    return;
  free(p->roots);
  free(p->buf);
  if (p->blue) {
    so3o_fft1d_destroy(p->sub);
    free(p->chirp);
    free(p->kern);
    free(p->bwork);
  }
  free(p);
}

int so3o_fft1d_len(const so3o_fft1d *p) { return p->n; }

/* In-register radix-R forward butterfly; roots step for e^{-2 pi i / R} is rstep. */
static inline void butterfly(cplx *v, int R, const cplx *roots, int rstep) {
  if (R == 2) {
    cplx a = v[0] + v[1], b = v[0] - v[1];
    v[0] = a;
    v[1] = b;
    return;
  }
  if (R == 4) {
    cplx t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3];
    cplx d = v[1] - v[3];
    cplx t3 = cimag(d) - I * creal(d); /* -i * d */
    v[0] = t0 + t2;
    v[2] = t0 - t2;
    v[1] = t1 + t3;
    v[3] = t1 - t3;
    return;
  }
  int h = (R - 1) / 2;
  cplx s[MAXRAD / 2 + 1], d[MAXRAD / 2 + 1];
  cplx v0 = v[0], tot = v[0];
  for (int r = 1; r <= h; r++) {
    s[r] = v[r] + v[R - r];
    d[r] = v[r] - v[R - r];
    tot += s[r];
  }
  cplx out[MAXRAD];
  out[0] = tot;
  for (int q = 1; q <= h; q++) {
    double ar = creal(v0), ai = cimag(v0), br = 0.0, bi = 0.0;
    for (int r = 1; r <= h; r++) {
      cplx w = roots[((r * q) % R) * rstep];
      double c = creal(w), sn = -cimag(w); /* cos, sin of 2 pi r q / R */
      ar += c * creal(s[r]);
      ai += c * cimag(s[r]);
      br += sn * creal(d[r]);
      bi += sn * cimag(d[r]);
    }
    /* V_q = A - iB, V_{R-q} = A + iB */
    out[q] = (ar + bi) + I * (ai - br);
    out[R - q] = (ar - bi) + I * (ai + br);
  }
  for (int q = 0; q < R; q++)
    v[q] = out[q];
}

static void stockham_forward(const so3o_fft1d *p, cplx *x) {
  int n = p->n, Ns = 1;
  cplx *src = x, *dst = p->buf;
  for (int ip = 0; ip < p->nrad; ip++) {
    int R = p->rad[ip];
    int m = n / R;
    int tstep = n / (Ns * R);
    int rstep = n / R;
    for (int j = 0; j < m; j++) {
      int k = j % Ns;
      cplx v[MAXRAD];
      v[0] = src[j];
      for (int r = 1; r < R; r++) {
        cplx a = src[j + r * m];
        if (k)
          a *= p->roots[(long)r * k * tstep];
        v[r] = a;
      }
      butterfly(v, R, p->roots, rstep);
      int idxD = (j / Ns) * Ns * R + k;
      for (int q = 0; q < R; q++)
        dst[idxD + q * Ns] = v[q];
    }
    cplx *t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  if (src != x)
    memcpy(x, src, sizeof(cplx) * n);
}

static void exec_forward(const so3o_fft1d *p, cplx *x) {
  if (p->n == 1)
    return;
  if (!p->blue) {
    stockham_forward(p, x);
    return;
  }
  int n = p->n, m = p->m;
  cplx *a = p->bwork;
  for (int k = 0; k < n; k++)
    a[k] = x[k] * p->chirp[k];
  for (int k = n; k < m; k++)
    a[k] = 0.0;
  exec_forward(p->sub, a);
  for (int k = 0; k < m; k++)
    a[k] = conj(a[k] * p->kern[k]);
  exec_forward(p->sub, a); /* inverse via conjugation */
  for (int k = 0; k < n; k++)
    x[k] = p->chirp[k] * conj(a[k]);
}

void so3o_fft1d_exec(const so3o_fft1d *p, cplx *x, int sign) {
  if (sign < 0) {
    exec_forward(p, x);
    return;
  }
  for (int k = 0; k < p->n; k++)
    x[k] = conj(x[k]);
  exec_forward(p, x);
  for (int k = 0; k < p->n; k++)
    x[k] = conj(x[k]);
}

void so3o_fft1d_exec_strided(const so3o_fft1d *p, cplx *x, int howmany, long stride,
                             long dist, int sign) {
  int n = p->n;
  if (stride == 1) {
    for (int b = 0; b < howmany; b++)
      so3o_fft1d_exec(p, x + b * dist, sign);
    return;
  }
  enum { BLK = 16 };
  cplx *tmp = malloc(sizeof(cplx) * (size_t)n * BLK);
  for (int b0 = 0; b0 < howmany; b0 += BLK) {
    int nb = howmany - b0 < BLK ? howmany - b0 : BLK;
    for (int j = 0; j < n; j++)
      for (int b = 0; b < nb; b++)
        tmp[(size_t)b * n + j] = x[(b0 + b) * dist + j * stride];
    for (int b = 0; b < nb; b++)
      so3o_fft1d_exec(p, tmp + (size_t)b * n, sign);
    for (int j = 0; j < n; j++)
      for (int b = 0; b < nb; b++)
        x[(b0 + b) * dist + j * stride] = tmp[(size_t)b * n + j];
  }
  free(tmp);
}

/* ------------------------------------------------------------------ plans */

enum { K_MANY_C2C, K_MANY_C2R, K_MANY_R2C, K_ND_C2C, K_R2C_2D, K_C2R_ND };

struct so3o_fftw_plan_s {
  int kind, sign, rank;
  int n[3];
  int howmany, istride, idist, ostride, odist;
  void *in, *out;
};

static fftw_plan new_plan(int kind) {
  fftw_plan p = calloc(1, sizeof *p);
  p->kind = kind;
  return p;
}

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in,
                             const int *inembed, int istride, int idist,
                             fftw_complex *out, const int *onembed, int ostride,
                             int odist, int sign, unsigned flags) {
  (void)inembed;
  (void)onembed;
  (void)flags;
  fftw_plan p = new_plan(K_MANY_C2C);
  p->rank = rank;
  p->n[0] = n[0];
  p->howmany = howmany;
  p->istride = istride;
  p->idist = idist;
  p->ostride = ostride;
  p->odist = odist;
  p->sign = sign;
  p->in = in;
  p->out = out;
  return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride,
                                 int idist, double *out, const int *onembed,
                                 int ostride, int odist, unsigned flags) {
  fftw_plan p = fftw_plan_many_dft(rank, n, howmany, in, inembed, istride, idist,
                                   NULL, onembed, ostride, odist, FFTW_BACKWARD, flags);
  p->kind = K_MANY_C2R;
  p->out = out;
  return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in,
                                 const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed,
                                 int ostride, int odist, unsigned flags) {
  fftw_plan p = fftw_plan_many_dft(rank, n, howmany, NULL, inembed, istride, idist,
                                   out, onembed, ostride, odist, FFTW_FORWARD, flags);
  p->kind = K_MANY_R2C;
  p->in = in;
  return p;
}

static fftw_plan nd_plan(int kind, int rank, int n0, int n1, int n2, void *in, void *out,
                         int sign) {
  fftw_plan p = new_plan(kind);
  p->rank = rank;
  p->n[0] = n0;
  p->n[1] = n1;
  p->n[2] = n2;
  p->in = in;
  p->out = out;
  p->sign = sign;
  return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags) {
  (void)flags;
  return nd_plan(K_ND_C2C, 1, n, 1, 1, in, out, sign);
}
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags) {
  (void)flags;
  return nd_plan(K_ND_C2C, 2, n0, n1, 1, in, out, sign);
}
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  return nd_plan(K_ND_C2C, 3, n0, n1, n2, in, out, sign);
}
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out,
                               unsigned flags) {
  (void)flags;
  return nd_plan(K_R2C_2D, 2, n0, n1, 1, in, out, FFTW_FORWARD);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out,
                               unsigned flags) {
  (void)flags;
  return nd_plan(K_C2R_ND, 2, n0, n1, 1, in, out, FFTW_BACKWARD);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags) {
  (void)flags;
  return nd_plan(K_C2R_ND, 3, n0, n1, n2, in, out, FFTW_BACKWARD);
}

/* Transform every line along `axis` of a row-major complex array. */
static void along_axis(cplx *x, int rank, const int *dims, int axis, int sign) {
  long inner = 1, outer = 1;
  for (int d = axis + 1; d < rank; d++)
    inner *= dims[d];
  for (int d = 0; d < axis; d++)
    outer *= dims[d];
  int n = dims[axis];
  if (n == 1)
    return;
  so3o_fft1d *e = so3o_fft1d_create(n);
  for (long o = 0; o < outer; o++)
    so3o_fft1d_exec_strided(e, x + o * inner * n, (int)inner, inner, 1, sign);
  so3o_fft1d_destroy(e);
}

static void c2r_line(const so3o_fft1d *e, const cplx *in, long istride, double *out,
                     long ostride, cplx *tmp) {
  int n = so3o_fft1d_len(e);
  int h = n / 2;
  for (int k = 0; k <= h; k++)
    tmp[k] = in[k * istride];
  for (int k = 1; k < n - h; k++)
    tmp[n - k] = conj(tmp[k]);
  tmp[0] = creal(tmp[0]);
  if (n % 2 == 0)
    tmp[h] = creal(tmp[h]);
  so3o_fft1d_exec(e, tmp, +1);
  for (int j = 0; j < n; j++)
    out[j * ostride] = creal(tmp[j]);
}

static void r2c_line(const so3o_fft1d *e, const double *in, long istride, cplx *out,
                     long ostride, cplx *tmp) {
  int n = so3o_fft1d_len(e);
  for (int j = 0; j < n; j++)
    tmp[j] = in[j * istride];
  so3o_fft1d_exec(e, tmp, -1);
  for (int k = 0; k <= n / 2; k++)
    out[k * ostride] = tmp[k];
}

static void run_plan(const struct so3o_fftw_plan_s *p, void *in, void *out) {
  switch (p->kind) {
  case K_MANY_C2C: {
    int n = p->n[0];
    cplx *ci = in, *co = out;
    if (ci != co)
      for (int b = 0; b < p->howmany; b++)
        for (int j = 0; j < n; j++)
          co[(long)b * p->odist + (long)j * p->ostride] =
              ci[(long)b * p->idist + (long)j * p->istride];
    so3o_fft1d *e = so3o_fft1d_create(n);
    so3o_fft1d_exec_strided(e, co, p->howmany, p->ostride, p->odist, p->sign);
    so3o_fft1d_destroy(e);
    break;
  }
  case K_MANY_C2R: {
    int n = p->n[0];
    so3o_fft1d *e = so3o_fft1d_create(n);
    cplx *tmp = malloc(sizeof(cplx) * n);
    for (int b = 0; b < p->howmany; b++)
      c2r_line(e, (cplx *)in + (long)b * p->idist, p->istride,
               (double *)out + (long)b * p->odist, p->ostride, tmp);
    free(tmp);
    so3o_fft1d_destroy(e);
    break;
  }
  case K_MANY_R2C: {
    int n = p->n[0];
    so3o_fft1d *e = so3o_fft1d_create(n);
    cplx *tmp = malloc(sizeof(cplx) * n);
    for (int b = 0; b < p->howmany; b++)
      r2c_line(e, (double *)in + (long)b * p->idist, p->istride,
               (cplx *)out + (long)b * p->odist, p->ostride, tmp);
    free(tmp);
    so3o_fft1d_destroy(e);
    break;
  }
  case K_ND_C2C: {
    long tot = (long)p->n[0] * p->n[1] * p->n[2];
    if (in != out)
      memmove(out, in, sizeof(cplx) * tot);
    for (int ax = 0; ax < p->rank; ax++)
      along_axis(out, p->rank, p->n, ax, p->sign);
    break;
  }
  case K_R2C_2D: {
    int n0 = p->n[0], n1 = p->n[1], h = n1 / 2 + 1;
    so3o_fft1d *e = so3o_fft1d_create(n1);
    cplx *tmp = malloc(sizeof(cplx) * n1);
    cplx *co = out;
    double *ri = in;
    for (int i = 0; i < n0; i++)
      r2c_line(e, ri + (long)i * n1, 1, co + (long)i * h, 1, tmp);
    free(tmp);
    so3o_fft1d_destroy(e);
    int dims[2] = {n0, h};
    along_axis(co, 2, dims, 0, -1);
    break;
  }
  case K_C2R_ND: {
    int rank = p->rank;
    int last = p->n[rank - 1], h = last / 2 + 1;
    int dims[3] = {p->n[0], p->n[1], p->n[2]};
    dims[rank - 1] = h;
    long lines = 1;
    for (int d = 0; d < rank - 1; d++)
      lines *= p->n[d];
    cplx *t = malloc(sizeof(cplx) * lines * h);
    memcpy(t, in, sizeof(cplx) * lines * h);
    for (int ax = 0; ax < rank - 1; ax++)
      along_axis(t, rank, dims, ax, +1);
    so3o_fft1d *e = so3o_fft1d_create(last);
    cplx *tmp = malloc(sizeof(cplx) * last);
    for (long i = 0; i < lines; i++)
      c2r_line(e, t + i * h, 1, (double *)out + i * last, 1, tmp);
    free(tmp);
    free(t);
    so3o_fft1d_destroy(e);
    break;
  }
  }
}

void fftw_execute(const fftw_plan p) { run_plan(p, p->in, p->out); }

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
  run_plan(p, in, out);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }
