// FFT stages of the transforms.  Each CTA stages T sequences in shared
// memory, runs the FP64 engine of fft_core.cuh and writes the results back;
// backward (synthesis) DFTs run the forward engine on conjugated data.
//
// Inverse (reference src/c/so3_core.c:202-216 with SSHT's synthesis, in-tree
// equivalent :1148-1194):
//   beta : per (n, m) column, expand m' >= 0 to -(L-1)..L-1 with
//          F[-m'] = (-1)^{m+n} F[m'], MW half-sample phase e^{i m' pi/(2L-1)},
//          inverse DFT over the extended circle, keep the nb beta rows.
//   alpha: per (n, beta) row, inverse DFT over m.
//   gamma: per (beta, alpha) sample, inverse DFT over n (c2r for real signals).
// Forward (reference :329-371 with SSHT's analysis, in-tree :1334-1490):
//   gamma: DFT over the gamma samples, times 2 pi/(2N-1) (r2c for real).
//   alpha: DFT over alpha, divided by nalpha.
//   beta : extend beta to the full circle with (-1)^{m+n}, DFT, divide,
//          phase e^{-i m'' pi/(2L-1)} (MW), convolve with the quadrature
//          weights through a power-of-two oversampled product, and fold
//          G[m'] + (-1)^{m+n} G[-m'] onto m' >= 0.
#include "so3gpu_internal.h"

namespace so3g {

namespace {
constexpr int kThreads = 256;
constexpr size_t kSmemCap = 200 * 1024;

int pick_T(int ld, int buffers_per_seq, int Tmax) {
  int T = Tmax;
  while (T > 1 && (size_t)buffers_per_seq * T * ld * sizeof(double2) > kSmemCap) T >>= 1;
  return T;
}

// Sequences per CTA and dynamic shared memory for a plan of engine length ld:
// large-radix instances may use up to kSmemCap (one CTA per SM), the others
// stay within half of an SM's shared memory (two CTAs per SM).
struct Sizing {
  int T;
  size_t smem;
};
Sizing size_for(bool big, int ld, int Tmax) {
  Sizing z;
  const size_t cap = big ? kSmemCap : kSmemCap / 2 + 10 * 1024;
  int T = Tmax;
  while (T > 1 && 2 * (size_t)T * ld * sizeof(double2) > cap) T >>= 1;
  z.T = T;
  z.smem = 2 * (size_t)T * ld * sizeof(double2);
  return z;
}

template <typename K>
int set_smem(K kernel, size_t bytes) {
  SO3G_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return kOk;
}

// Instances for plans with a radix above 8 carry the large odd-radix
// butterflies (high register use, one CTA per SM); the others stay below 128
// registers and run two CTAs per SM.
template <bool BIG>
__device__ __forceinline__ double2* run_fft(double2* a, double2* b, int T, int ld, const FftPlan& P) {
  return fft_fwd_smem<BIG>(a, b, T, ld, P);
}

__device__ __forceinline__ int wrapi(int k, int P) {
  k %= P;
  return k < 0 ? k + P : k;
}
__device__ __forceinline__ double2 phase(int k, int den, double sign) {  // e^{sign i pi k/den}
  double s, c;
  sincospi((double)k / (double)den, &s, &c);
  return make_double2(c, sign * s);
}
}  // namespace

// ------------------------------------------------------------------ inverse
template <bool BIG>
__global__ void __launch_bounds__(kThreads, BIG ? 1 : 2) inv_beta_kernel(Geometry g, FftPlan P, double2* __restrict__ W,
                                                             int T, int ld) {
  extern __shared__ double2 sm[];
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int plane = blockIdx.y, n = plane - g.plane0;
  const int c0 = blockIdx.x * T, ncols = 2 * g.L - 1, L = g.L, Pn = g.P;
  double2* base = W + (long long)plane * g.PS;
  if (!g.mw)
    for (int t = threadIdx.x; t < T; t += blockDim.x) a[t * ld + L] = make_double2(0.0, 0.0);
  for (int idx = threadIdx.x; idx < L * T; idx += blockDim.x) {
    const int t = idx % T, mp = idx / T, c = c0 + t;
    double2 v = c < ncols ? base[(long long)mp * g.RS + c] : make_double2(0.0, 0.0);
    const int m = c - (L - 1);
    const double sg = ((m + n) & 1) ? -1.0 : 1.0;
    double2 xp = v, xn = make_double2(sg * v.x, sg * v.y);
    if (g.mw) {
      const double2 e = phase(mp, 2 * L - 1, 1.0);
      xp = cmul(xp, e);
      xn = cmul(xn, cconj(e));
    }
    a[t * ld + mp] = cconj(xp);
    if (mp > 0) a[t * ld + Pn - mp] = cconj(xn);
  }
  __syncthreads();
  double2* r = run_fft<BIG>(a, b, T, ld, P);
  for (int idx = threadIdx.x; idx < g.nb * T; idx += blockDim.x) {
    const int t = idx % T, row = idx / T, c = c0 + t;
    if (c < ncols) base[(long long)row * g.RS + c] = cconj(r[t * ld + row]);
  }
}

template <bool BIG>
__global__ void __launch_bounds__(kThreads, BIG ? 1 : 2) inv_alpha_kernel(Geometry g, FftPlan P, double2* __restrict__ W,
                                                              int T, int ld) {
  extern __shared__ double2 sm[];
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int L = g.L, Pn = g.P, nrows = g.nplanes * g.nb;
  const int r0 = blockIdx.x * T;
  for (int idx = threadIdx.x; idx < T * Pn; idx += blockDim.x) {
    const int j = idx / Pn, k = idx - j * Pn, row = r0 + j;
    double2 v = make_double2(0.0, 0.0);
    if (row < nrows) {
      const int m = k <= L - 1 ? k : k - Pn;
      if (m >= -(L - 1)) {  // MWSS Nyquist index k = L stays zero
        const long long off = (long long)(row / g.nb) * g.PS + (long long)(row % g.nb) * g.RS;
        v = W[off + m + L - 1];
      }
    }
    a[j * ld + k] = cconj(v);
  }
  __syncthreads();
  double2* r = run_fft<BIG>(a, b, T, ld, P);
  for (int idx = threadIdx.x; idx < T * g.na; idx += blockDim.x) {
    const int j = idx / g.na, k = idx - j * g.na, row = r0 + j;
    if (row < nrows) {
      const long long off = (long long)(row / g.nb) * g.PS + (long long)(row % g.nb) * g.RS;
      W[off + k] = cconj(r[j * ld + k]);
    }
  }
}

template <bool REAL, bool BIG>
__global__ void __launch_bounds__(kThreads, BIG ? 1 : 2) inv_gamma_kernel(Geometry g, FftPlan P, const double2* __restrict__ W,
                                                              void* __restrict__ fout, int T, int ld) {
  extern __shared__ double2 sm[];
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int row = blockIdx.y, a0 = blockIdx.x * T, ng = g.ng;
  for (int idx = threadIdx.x; idx < g.nplanes * T; idx += blockDim.x) {
    const int t = idx % T, p = idx / T, al = a0 + t;
    double2 v = al < g.na ? W[(long long)p * g.PS + (long long)row * g.RS + al] : make_double2(0.0, 0.0);
    if (!REAL) {
      const int k = wrapi(p - g.plane0, ng);
      a[t * ld + k] = cconj(v);
    } else {
      // Hermitian completion of planes n = 0..N-1, Im of n = 0 ignored
      if (p == 0) {
        a[t * ld] = make_double2(v.x, 0.0);
      } else {
        a[t * ld + p] = cconj(v);
        a[t * ld + ng - p] = v;
      }
    }
  }
  __syncthreads();
  double2* r = run_fft<BIG>(a, b, T, ld, P);
  const long long plane_sz = (long long)g.nb * g.na;
  for (int idx = threadIdx.x; idx < ng * T; idx += blockDim.x) {
    const int t = idx % T, gi = idx / T, al = a0 + t;
    if (al >= g.na) continue;
    const long long o = (long long)gi * plane_sz + (long long)row * g.na + al;
    const double2 y = r[t * ld + gi];
    if (REAL)
      static_cast<double*>(fout)[o] = y.x;
    else
      static_cast<double2*>(fout)[o] = cconj(y);
  }
}

// ------------------------------------------------------------------ forward
template <bool REAL, bool BIG>
__global__ void __launch_bounds__(kThreads, BIG ? 1 : 2) fwd_gamma_kernel(Geometry g, FftPlan P, const void* __restrict__ fin,
                                                              double2* __restrict__ W, int T, int ld) {
  extern __shared__ double2 sm[];
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int row = blockIdx.y, a0 = blockIdx.x * T, ng = g.ng;
  const long long plane_sz = (long long)g.nb * g.na;
  for (int idx = threadIdx.x; idx < ng * T; idx += blockDim.x) {
    const int t = idx % T, gi = idx / T, al = a0 + t;
    double2 v = make_double2(0.0, 0.0);
    if (al < g.na) {
      const long long o = (long long)gi * plane_sz + (long long)row * g.na + al;
      if (REAL)
        v = make_double2(static_cast<const double*>(fin)[o], 0.0);
      else
        v = static_cast<const double2*>(fin)[o];
    }
    a[t * ld + gi] = v;
  }
  __syncthreads();
  double2* r = run_fft<BIG>(a, b, T, ld, P);
  const double scale = 2.0 * 3.141592653589793238462643383279502884 / ng;
  for (int idx = threadIdx.x; idx < g.nplanes * T; idx += blockDim.x) {
    const int t = idx % T, p = idx / T, al = a0 + t;
    if (al >= g.na) continue;
    const int k = REAL ? p : wrapi(p - g.plane0, ng);
    W[(long long)p * g.PS + (long long)row * g.RS + al] = cscale(r[t * ld + k], scale);
  }
}

template <bool BIG>
__global__ void __launch_bounds__(kThreads, BIG ? 1 : 2) fwd_alpha_kernel(Geometry g, FftPlan P, double2* __restrict__ W,
                                                              int T, int ld) {
  extern __shared__ double2 sm[];
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int L = g.L, Pn = g.P, nrows = g.nplanes * g.nb, ncols = 2 * L - 1;
  const int r0 = blockIdx.x * T;
  for (int idx = threadIdx.x; idx < T * Pn; idx += blockDim.x) {
    const int j = idx / Pn, k = idx - j * Pn, row = r0 + j;
    double2 v = make_double2(0.0, 0.0);
    if (row < nrows) v = W[(long long)(row / g.nb) * g.PS + (long long)(row % g.nb) * g.RS + k];
    a[j * ld + k] = v;
  }
  __syncthreads();
  double2* r = run_fft<BIG>(a, b, T, ld, P);
  const double inv = 1.0 / Pn;
  for (int idx = threadIdx.x; idx < T * ncols; idx += blockDim.x) {
    const int j = idx / ncols, c = idx - j * ncols, row = r0 + j;
    if (row < nrows) {
      const int k = wrapi(c - (L - 1), Pn);
      W[(long long)(row / g.nb) * g.PS + (long long)(row % g.nb) * g.RS + c] = cscale(r[j * ld + k], inv);
    }
  }
}

template <bool BIG>
__global__ void __launch_bounds__(kThreads, BIG ? 1 : 2) fwd_beta_conv_kernel(Geometry g, FftPlan P, FftPlan Pc,
                                                                  const double2* __restrict__ wr,
                                                                  double2* __restrict__ W, int T, int ld) {
  extern __shared__ double2 sm[];
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int plane = blockIdx.y, n = plane - g.plane0;
  const int c0 = blockIdx.x * T, L = g.L, ncols = 2 * L - 1, Pn = g.P, pc = g.Pc;
  double2* base = W + (long long)plane * g.PS;
  for (int idx = threadIdx.x; idx < g.nb * T; idx += blockDim.x) {
    const int t = idx % T, row = idx / T, c = c0 + t;
    a[t * ld + row] = c < ncols ? base[(long long)row * g.RS + c] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < (Pn - g.nb) * T; idx += blockDim.x) {
    const int t = idx % T, row = g.nb + idx / T, c = c0 + t;
    const int m = c - (L - 1);
    const double sg = ((m + n) & 1) ? -1.0 : 1.0;
    const int src = g.mw ? 2 * L - 2 - row : 2 * L - row;
    a[t * ld + row] = cscale(a[t * ld + src], sg);
  }
  __syncthreads();
  double2* r = run_fft<BIG>(a, b, T, ld, P);
  // conv input: F[m''] / P with the MW phase, at m'' mod Pc, zero elsewhere
  const double invP = 1.0 / Pn;
  double2* o = (r == a) ? b : a;
  for (int idx = threadIdx.x; idx < T * pc; idx += blockDim.x) {
    const int t = idx / pc, k = idx - t * pc;
    o[t * ld + k] = make_double2(0.0, 0.0);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < T * (2 * L - 1); idx += blockDim.x) {
    const int t = idx / (2 * L - 1), mpp = idx - t * (2 * L - 1) - (L - 1);
    double2 v = cscale(r[t * ld + wrapi(mpp, Pn)], invP);
    if (g.mw) v = cmul(v, phase(mpp, 2 * L - 1, -1.0));
    o[t * ld + wrapi(mpp, pc)] = cconj(v);
  }
  __syncthreads();
  double2* o2 = (o == a) ? b : a;
  double2* q = run_fft<BIG>(o, o2, T, ld, Pc);  // conj of the inverse DFT
  for (int idx = threadIdx.x; idx < T * pc; idx += blockDim.x) {
    const int t = idx / pc, k = idx - t * pc;
    q[t * ld + k] = cmul(cconj(q[t * ld + k]), __ldg(wr + k));
  }
  __syncthreads();
  double2* q2 = (q == a) ? b : a;
  double2* G = run_fft<BIG>(q, q2, T, ld, Pc);
  for (int idx = threadIdx.x; idx < L * T; idx += blockDim.x) {
    const int t = idx % T, mp = idx / T, c = c0 + t;
    if (c >= ncols) continue;
    const int m = c - (L - 1);
    const double sg = ((m + n) & 1) ? -1.0 : 1.0;
    double2 v = G[t * ld + mp];
    if (mp > 0) {
      const double2 u = G[t * ld + pc - mp];
      v = make_double2(v.x + sg * u.x, v.y + sg * u.y);
    }
    base[(long long)mp * g.RS + c] = v;
  }
}

// ------------------------------------------------------------------ launchers
int launch_inv_beta(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const int ld = p.ld();
  const Sizing z = size_for(p.big(), ld, 16);
  const int T = z.T;
  const size_t sm = z.smem;
  dim3 grid((2 * g.L - 1 + T - 1) / T, g.nplanes);
  if (p.big()) {
    if (int rc = set_smem(inv_beta_kernel<true>, sm)) return rc;
    inv_beta_kernel<true><<<grid, kThreads, sm, s>>>(g, p, W, T, ld);
  } else {
    if (int rc = set_smem(inv_beta_kernel<false>, sm)) return rc;
    inv_beta_kernel<false><<<grid, kThreads, sm, s>>>(g, p, W, T, ld);
  }
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

int launch_inv_alpha(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const int ld = p.ld();
  const Sizing z = size_for(p.big(), ld, 16);
  const int T = z.T;
  const size_t sm = z.smem;
  const int nrows = g.nplanes * g.nb;
  if (p.big()) {
    if (int rc = set_smem(inv_alpha_kernel<true>, sm)) return rc;
    inv_alpha_kernel<true><<<(nrows + T - 1) / T, kThreads, sm, s>>>(g, p, W, T, ld);
  } else {
    if (int rc = set_smem(inv_alpha_kernel<false>, sm)) return rc;
    inv_alpha_kernel<false><<<(nrows + T - 1) / T, kThreads, sm, s>>>(g, p, W, T, ld);
  }
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

int launch_inv_gamma(const Geometry& g, const FftPlan& p, const double2* W, void* f, cudaStream_t s) {
  const int ld = p.ld() > g.nplanes ? p.ld() : g.nplanes;
  const Sizing z = size_for(p.big(), ld, 16);
  const int T = z.T;
  const size_t sm = z.smem;
  dim3 grid((g.na + T - 1) / T, g.nb);
#define SO3G_GAMMA_INV(R, B)                                                  \
  do {                                                                        \
    if (int rc = set_smem(inv_gamma_kernel<R, B>, sm)) return rc;             \
    inv_gamma_kernel<R, B><<<grid, kThreads, sm, s>>>(g, p, W, f, T, ld);     \
  } while (0)
  if (g.real) {
    if (p.big()) SO3G_GAMMA_INV(true, true); else SO3G_GAMMA_INV(true, false);
  } else {
    if (p.big()) SO3G_GAMMA_INV(false, true); else SO3G_GAMMA_INV(false, false);
  }
#undef SO3G_GAMMA_INV
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

int launch_fwd_gamma(const Geometry& g, const FftPlan& p, const void* f, double2* W, cudaStream_t s) {
  const int ld = p.ld();
  const Sizing z = size_for(p.big(), ld, 16);
  const int T = z.T;
  const size_t sm = z.smem;
  dim3 grid((g.na + T - 1) / T, g.nb);
#define SO3G_GAMMA_FWD(R, B)                                                  \
  do {                                                                        \
    if (int rc = set_smem(fwd_gamma_kernel<R, B>, sm)) return rc;             \
    fwd_gamma_kernel<R, B><<<grid, kThreads, sm, s>>>(g, p, f, W, T, ld);     \
  } while (0)
  if (g.real) {
    if (p.big()) SO3G_GAMMA_FWD(true, true); else SO3G_GAMMA_FWD(true, false);
  } else {
    if (p.big()) SO3G_GAMMA_FWD(false, true); else SO3G_GAMMA_FWD(false, false);
  }
#undef SO3G_GAMMA_FWD
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

int launch_fwd_alpha(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const int ld = p.ld();
  const Sizing z = size_for(p.big(), ld, 16);
  const int T = z.T;
  const size_t sm = z.smem;
  const int nrows = g.nplanes * g.nb;
  if (p.big()) {
    if (int rc = set_smem(fwd_alpha_kernel<true>, sm)) return rc;
    fwd_alpha_kernel<true><<<(nrows + T - 1) / T, kThreads, sm, s>>>(g, p, W, T, ld);
  } else {
    if (int rc = set_smem(fwd_alpha_kernel<false>, sm)) return rc;
    fwd_alpha_kernel<false><<<(nrows + T - 1) / T, kThreads, sm, s>>>(g, p, W, T, ld);
  }
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

int launch_fwd_beta_conv(const Geometry& g, const FftPlan& p, const FftPlan& pc, const double2* wr, double2* W,
                         cudaStream_t s) {
  int ld = p.ld() > pc.ld() ? p.ld() : pc.ld();
  const Sizing z = size_for(p.big() || pc.big(), ld, 8);
  const int T = z.T;
  const size_t sm = z.smem;
  dim3 grid((2 * g.L - 1 + T - 1) / T, g.nplanes);
  if (p.big() || pc.big()) {
    if (int rc = set_smem(fwd_beta_conv_kernel<true>, sm)) return rc;
    fwd_beta_conv_kernel<true><<<grid, kThreads, sm, s>>>(g, p, pc, wr, W, T, ld);
  } else {
    if (int rc = set_smem(fwd_beta_conv_kernel<false>, sm)) return rc;
    fwd_beta_conv_kernel<false><<<grid, kThreads, sm, s>>>(g, p, pc, wr, W, T, ld);
  }
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace so3g
