/*
 * fftw3.h -- project-written stand-in for the subset of the FFTW 3.3 API that
 * the SO3 reference sources call (src/c/so3_core.c:145-158, :348-363,
 * :564-576, :791-805, :1172-1194, :1339-1352, :1381-1388, :1419-1484,
 * :1913-1934, :2085-2244).  TEST INFRASTRUCTURE ONLY: it lets the oracle and
 * the reference C be compiled without FFTW.  The transforms follow FFTW's
 * published definitions: FFTW_FORWARD computes X_k = sum_j x_j e^{-2 pi i jk/n},
 * FFTW_BACKWARD the same with +i, both unnormalised; multi-dimensional arrays
 * are row-major; r2c writes n/2+1 outputs along the last dimension and c2r
 * reads them, treating the input as Hermitian.
 *
 * As in FFTW, when <complex.h> is included first fftw_complex is the C99
 * double complex type, so reference code can pass `complex double *`.
 */
#ifndef SO3_ORACLE_FFTW3_STANDIN_H
#define SO3_ORACLE_FFTW3_STANDIN_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex fftw_complex;
typedef struct so3o_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in,
                             const int *inembed, int istride, int idist,
                             fftw_complex *out, const int *onembed, int ostride,
                             int odist, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride,
                                 int idist, double *out, const int *onembed,
                                 int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in,
                                 const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed,
                                 int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);

/* Project engine used directly by the oracle restatement and the SSHT
 * stand-in: a contiguous in-place 1-D DFT of length n.  sign = -1 forward,
 * +1 backward, unnormalised. */
typedef struct so3o_fft1d so3o_fft1d;
so3o_fft1d *so3o_fft1d_create(int n);
void so3o_fft1d_destroy(so3o_fft1d *p);
void so3o_fft1d_exec(const so3o_fft1d *p, double _Complex *x, int sign);
int so3o_fft1d_len(const so3o_fft1d *p);
/* Strided batch: `howmany` sequences, element j of sequence b at
 * x[b*dist + j*stride], transformed in place. */
void so3o_fft1d_exec_strided(const so3o_fft1d *p, double _Complex *x, int howmany,
                             long stride, long dist, int sign);

#ifdef __cplusplus
}
#endif
#endif
