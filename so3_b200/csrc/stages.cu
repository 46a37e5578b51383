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
#include <algorithm>

#include "fft_fixed.cuh"
#include "so3gpu_internal.h"

namespace so3g {

namespace {
constexpr int kThreads = 256;
constexpr size_t kSmemCap = 200 * 1024;

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

// DFT engines the stage kernels are instantiated with.  Gen<BIG> runs any
// plan from its runtime description (fft_core.cuh): instances for plans with
// a radix above 8 carry the large odd-radix butterflies (high register use,
// one CTA per SM), the others stay below 128 registers and run two CTAs per
// SM.  Fix<...> runs a compile-time plan (fft_fixed.cuh) with T sequences of
// pitch LD per CTA of NT threads; T and LD of the kernel arguments are then
// ignored.  runP / runC are the two DFT lengths of the forward beta kernel
// (extended beta circle, weight convolution); single-length stages use runP.
template <bool BIG>
struct Gen {
  static constexpr bool fixed = false;
  static constexpr int NT = kThreads, MINB = BIG ? 1 : 2, T = 0, LD = 0, nP = 0;
  static constexpr bool io = false, has_out = false;
  template <class In, class Out>
  static __device__ __forceinline__ void runIO(const In&, const Out&, double2*, double2*, const FftPlan&) {}
  template <class Out>
  static __device__ __forceinline__ void runPOut(double2*, double2*, const FftPlan&, const Out&) {}
  static __device__ __forceinline__ int at(int k) { return k; }
  static __device__ __forceinline__ int atC(int k) { return k; }
  static __device__ __forceinline__ double2* runP(double2* a, double2* b, int T_, int ld, const FftPlan& P) {
    return fft_fwd_smem<BIG>(a, b, T_, ld, P);
  }
  static __device__ __forceinline__ double2* runC(double2* a, double2* b, int T_, int ld, const FftPlan& P) {
    return fft_fwd_smem<BIG>(a, b, T_, ld, P);
  }
};

template <template <int, int, int> class PP, template <int, int, int> class PC, int T_, int NT_, int MINB_>
struct Fix {
  static constexpr bool fixed = true;
  static constexpr int NT = NT_, MINB = MINB_, T = T_;
  static constexpr int ldP = PP<1, 1, 1>::ld, ldC = PC<1, 1, 1>::ld;
  static constexpr int nP = PP<1, 1, 1>::n;  // runP length
  // the runP plan reads its input and writes its output through callables
  static constexpr bool io = PP<1, 1, 1>::io;
  template <class In, class Out>
  static __device__ __forceinline__ void runIO(const In& in, const Out& out, double2* a, double2* b,
                                               const FftPlan& P) {
    PP<T_, LD, NT_>::run_io(in, out, a, b, P);
  }
  // the runP plan's last pass can store through a callable (1023 = 31*11*3)
  static constexpr bool has_out = nP == 1023;
  template <class Out>
  static __device__ __forceinline__ void runPOut(double2* a, double2* b, const FftPlan& P, const Out& out) {
    if constexpr (has_out) PP<T_, LD, NT_>::run_out(a, b, P, out);
  }
  static constexpr int ldmax = ldP > ldC ? ldP : ldC;
  // pitch = 8/T (mod 8) 16-byte slots: the T sequences of one index, which
  // consecutive threads handle, fall into distinct banks
  static constexpr int LDMOD = T_ >= 8 ? 1 : T_ == 4 ? 2 : T_ == 2 ? 4 : 0;
  static constexpr int LD = T_ > 1 ? ldmax + ((LDMOD - ldmax % 8 + 8) % 8) : ldmax;
  // element k of a sequence in the buffers of the runP / runC lengths
  static __device__ __forceinline__ int at(int k) { return fx::phys<PP<1, 1, 1>::sk>(k); }
  static __device__ __forceinline__ int atC(int k) { return fx::phys<PC<1, 1, 1>::sk>(k); }
  static __device__ __forceinline__ double2* runP(double2* a, double2* b, int, int, const FftPlan& P) {
    return PP<T_, LD, NT_>::run(a, b, P);
  }
  static __device__ __forceinline__ double2* runC(double2* a, double2* b, int, int, const FftPlan& P) {
    return PC<T_, LD, NT_>::run(a, b, P);
  }
  static constexpr size_t smem() { return 2 * (size_t)T_ * LD * sizeof(double2); }
};

// Variants the autotuner chooses from (sequences per CTA, CTA size, minimum
// CTAs per SM): alpha / extended-beta length 1023 (L = 512), gamma length 127
// (N = 64), and the forward beta pair 1023 / 2048.  Variant 0 is the default.
using E1023a = Fix<fx::P1023, fx::P1023, 1, 128, 4>;
using E1023b = Fix<fx::P1023, fx::P1023, 1, 64, 8>;
using E1023c = Fix<fx::P1023, fx::P1023, 2, 128, 3>;
using E1023p = Fix<fx::P1023, fx::P1023, 1, 128, 3>;  // persistent inverse alpha (prefetch registers)
using E1023c2 = Fix<fx::P1023n2, fx::P1023n2, 2, 128, 3>;  // radix-31 butterflies in two output groups
using E127a = Fix<fx::P127, fx::P127, 4, 128, 4>;
using E127b = Fix<fx::P127, fx::P127, 8, 128, 3>;
using E127c = Fix<fx::P127, fx::P127, 2, 64, 8>;
using E127ra = Fix<fx::P127R, fx::P127R, 8, 128, 4>;
using E127rb = Fix<fx::P127R, fx::P127R, 16, 256, 2>;
using E127rc = Fix<fx::P127R, fx::P127R, 4, 64, 8>;
using EConv1023a = Fix<fx::P1023, fx::P2048, 1, 128, 3>;
using EConv1023b = Fix<fx::P1023, fx::P2048, 1, 256, 2>;

__device__ __forceinline__ int wrapi(int k, int P) {
  k %= P;
  return k < 0 ? k + P : k;
}
// k mod P for -P < k < P (a signed plane or frequency index)
__device__ __forceinline__ int wrap1(int k, int P) { return k < 0 ? k + P : k; }

// Offset of row `row` (plane-major over the nb beta rows) of the row-major
// part of the scratch.
__device__ __forceinline__ long long row_off(const Geometry& g, int row) {
  return (long long)(row / g.nb) * g.PS + (long long)(row % g.nb) * g.RS;
}
}  // namespace

// ------------------------------------------------------------------ inverse
// Inverse beta stage, two columns per DFT.  Column m of plane n is the
// mirror-symmetric sequence x(m') = e^{i m' theta} F(m'), x(-m') = s e^{-i m'
// theta} F(m') with s = (-1)^{m+n} (theta = pi/P for MW, 0 for MWSS), so its
// synthesis y(k) = F(0) + sum_{m'>0} F(m') (e^{i m' b_k} + s e^{-i m' b_k}),
// b_k = (2k+1) pi / P (MW) or 2 k pi / P (MWSS), is a cosine (s = +1) or sine
// (s = -1) transform.  Adjacent columns have opposite s: with A the s = +1
// and B the s = -1 column of a pair, one DFT of
//   z(m') = e^{i m' theta} (A + B)(m'),  z(-m') = e^{-i m' theta} (A - B)(m'),
//   z(0) = A(0) + B(0)
// gives y_z = y_A + y_B, and since b at the mirrored row k' (P-1-k for MW,
// P-k mod P for MWSS) is 2 pi - b_k,
//   y_A(k) = (y_z(k) + y_z(k')) / 2 - B(0),  y_B(k) = (y_z(k) - y_z(k')) / 2 + B(0).
// Sequence t of a CTA is column pair q = blockIdx.x * T + t (columns 2q,
// 2q + 1; the last pair of the 2L - 1 columns has one).
template <class E>
__global__ void __launch_bounds__(E::NT, E::MINB) inv_beta_kernel(Geometry g, FftPlan P, double2* __restrict__ W,
                                                             int T_, int ld_) {
  extern __shared__ double2 sm[];
  __shared__ double2 b0s[E::fixed ? E::T : 16];  // B(0) of each pair
  const int T = E::fixed ? E::T : T_, ld = E::fixed ? E::LD : ld_;
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int plane = blockIdx.y, n = plane - g.plane0;
  const int q0 = blockIdx.x * T, ncols = 2 * g.L - 1, L = g.L, Pn = g.P;
  double2* base = W + (long long)plane * g.PS;                        // row-major output
  const double2* cbase = W + g.QOFF + (long long)plane * g.QS;        // column-major input
  if (!g.mw)
    for (int t = threadIdx.x; t < T; t += E::NT) a[t * ld + E::at(L)] = make_double2(0.0, 0.0);
  // column 2q has s = +1 when (2q - (L-1) + n) is even
  const bool first_is_a = ((L - 1 + n) & 1) == 0;
  // m' fastest: whole columns read contiguously
  auto fetch = [&](int t, int mp, double2& v0, double2& v1) {
    const int c = 2 * (q0 + t);
    v0 = c < ncols ? cbase[(long long)c * g.CS + mp] : make_double2(0.0, 0.0);
    v1 = c + 1 < ncols ? cbase[(long long)(c + 1) * g.CS + mp] : make_double2(0.0, 0.0);
  };
  auto put = [&](int t, int mp, double2 v0, double2 v1) {
    const double2 A = first_is_a ? v0 : v1, B = first_is_a ? v1 : v0;
    if (mp == 0) {
      b0s[t] = B;
      a[t * ld + E::at(0)] = cconj(cadd(A, B));
      return;
    }
    double2 xp = cadd(A, B), xn = csub(A, B);
    if (g.mw) {
      const double2 e = cconj(__ldg(P.half + mp));  // e^{i pi m'/(2L-1)}
      xp = cmul(xp, e);
      xn = cmul(xn, cconj(e));
    }
    a[t * ld + E::at(mp)] = cconj(xp);
    a[t * ld + E::at(Pn - mp)] = cconj(xn);
  };
  auto load = [&](int t, int mp) {
    double2 v0, v1;
    fetch(t, mp, v0, v1);
    put(t, mp, v0, v1);
  };
  if constexpr (E::fixed) {  // no index division per element
    // an odd fixed plan of length nP is the MW circle of L = (nP + 1) / 2: all
    // loads of a sequence are issued before its first shared-memory store
    constexpr int LC = (E::nP + 1) / 2, NI = (LC + E::NT - 1) / E::NT;
    if (L == LC) {
      for (int t = 0; t < E::T; t++) {
        double2 v0[NI], v1[NI];
#pragma unroll
        for (int i = 0; i < NI; i++) {
          const int mp = threadIdx.x + i * E::NT;
          if (mp < LC) fetch(t, mp, v0[i], v1[i]);
        }
#pragma unroll
        for (int i = 0; i < NI; i++) {
          const int mp = threadIdx.x + i * E::NT;
          if (mp < LC) put(t, mp, v0[i], v1[i]);
        }
      }
    } else {
      for (int t = 0; t < E::T; t++)
        for (int mp = threadIdx.x; mp < L; mp += E::NT) load(t, mp);
    }
  } else {
    for (int idx = threadIdx.x; idx < L * T; idx += E::NT) load(idx / L, idx % L);
  }
  __syncthreads();
  double2* r = E::runP(a, b, T, ld, P);
  // y_z(k) = conj(r[k]); rows k < nb of both columns, written pairwise
  for (int idx = threadIdx.x; idx < g.nb * T; idx += E::NT) {
    const int t = idx % T, row = idx / T, c = 2 * (q0 + t);
    if (c >= ncols) continue;
    int mrow = g.mw ? Pn - 1 - row : Pn - row;
    if (mrow >= Pn) mrow -= Pn;
    const double2 y0 = cconj(r[t * ld + E::at(row)]), y1 = cconj(r[t * ld + E::at(mrow)]);
    const double2 B0 = b0s[t];
    const double2 yA = make_double2(0.5 * (y0.x + y1.x) - B0.x, 0.5 * (y0.y + y1.y) - B0.y);
    const double2 yB = make_double2(0.5 * (y0.x - y1.x) + B0.x, 0.5 * (y0.y - y1.y) + B0.y);
    double2* dst = base + (long long)row * g.RS + c;
    if (c + 1 < ncols) {
      dst[0] = first_is_a ? yA : yB;
      dst[1] = first_is_a ? yB : yA;
    } else {
      dst[0] = first_is_a ? yA : yB;
    }
  }
}

template <class E>
__global__ void __launch_bounds__(E::NT, E::MINB) inv_alpha_kernel(Geometry g, FftPlan P, double2* __restrict__ W,
                                                              int T_, int ld_) {
  extern __shared__ double2 sm[];
  const int T = E::fixed ? E::T : T_, ld = E::fixed ? E::LD : ld_;
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int L = g.L, Pn = g.P, nrows = g.nplanes * g.nb;
  const int r0 = blockIdx.x * T;
  auto load = [&](int j, int k, long long off, bool ok) {
    double2 v = make_double2(0.0, 0.0);
    const int m = k <= L - 1 ? k : k - Pn;
    if (ok && m >= -(L - 1)) v = W[off + m + L - 1];  // MWSS Nyquist index k = L stays zero
    a[j * ld + E::at(k)] = cconj(v);
  };
  if constexpr (E::fixed) {  // row offsets once per sequence, no index division per element
    for (int j = 0; j < E::T; j++) {
      const int row = r0 + j;
      const bool ok = row < nrows;
      const long long off = ok ? row_off(g, row) : 0;
      for (int k = threadIdx.x; k < E::nP; k += E::NT) load(j, k, off, ok);
    }
  } else {
    for (int idx = threadIdx.x; idx < T * Pn; idx += E::NT) {
      const int j = idx / Pn, row = r0 + j;
      load(j, idx - j * Pn, row < nrows ? row_off(g, row) : 0, row < nrows);
    }
  }
  __syncthreads();
  double2* r = E::runP(a, b, T, ld, P);
  if constexpr (E::fixed) {
    for (int j = 0; j < E::T; j++) {
      const int row = r0 + j;
      if (row >= nrows) break;
      double2* dst = W + row_off(g, row);
      for (int k = threadIdx.x; k < g.na; k += E::NT) dst[k] = cconj(r[j * ld + E::at(k)]);
    }
  } else {
    for (int idx = threadIdx.x; idx < T * g.na; idx += E::NT) {
      const int j = idx / g.na, k = idx - j * g.na, row = r0 + j;
      if (row < nrows) W[row_off(g, row) + k] = cconj(r[j * ld + E::at(k)]);
    }
  }
}

template <bool REAL, class E>
__global__ void __launch_bounds__(E::NT, E::MINB) inv_gamma_kernel(Geometry g, FftPlan P, const double2* __restrict__ W,
                                                              void* __restrict__ fout, int T_, int ld_, int row0) {
  extern __shared__ double2 sm[];
  const int T = E::fixed ? E::T : T_, ld = E::fixed ? E::LD : ld_;
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int row = row0 + blockIdx.y, a0 = blockIdx.x * T, ng = g.ng;
  if constexpr (!REAL && E::io) {
    // the plan reads plane (k + plane0) mod ng and writes gamma sample k
    // straight from / to global memory (complex: nplanes == ng)
    const long long plane_sz = (long long)g.nb * g.na;
    double2* f = static_cast<double2*>(fout);
    auto in = [&](int t, int k) {
      const int al = a0 + t;
      int p = k + g.plane0;
      if (p >= ng) p -= ng;
      return al < g.na ? cconj(W[(long long)p * g.PS + (long long)row * g.RS + al]) : make_double2(0.0, 0.0);
    };
    auto out = [&](int t, int k, double2 y) {
      const int al = a0 + t;
      if (al < g.na) f[(long long)k * plane_sz + (long long)row * g.na + al] = cconj(y);
    };
    E::runIO(in, out, a, b, P);
    return;
  }
  if (!REAL && g.steer)  // the 2N-point circle of a steerable signal has no plane n = N
    for (int t = threadIdx.x; t < T; t += E::NT) a[t * ld + E::at(g.N)] = make_double2(0.0, 0.0);
  for (int idx = threadIdx.x; idx < g.nplanes * T; idx += E::NT) {
    const int t = idx % T, p = idx / T, al = a0 + t;
    double2 v = al < g.na ? W[(long long)p * g.PS + (long long)row * g.RS + al] : make_double2(0.0, 0.0);
    if (!REAL) {
      const int k = wrap1(p - g.plane0, ng);
      a[t * ld + E::at(k)] = cconj(v);
    } else {
      // Hermitian completion of planes n = 0..N-1, Im of n = 0 ignored
      if (p == 0) {
        a[t * ld] = make_double2(v.x, 0.0);
      } else {
        a[t * ld + E::at(p)] = cconj(v);
        a[t * ld + E::at(ng - p)] = v;
      }
    }
  }
  __syncthreads();
  double2* r = E::runP(a, b, T, ld, P);
  const long long plane_sz = (long long)g.nb * g.na;
  for (int idx = threadIdx.x; idx < g.nf * T; idx += E::NT) {  // steerable: the first N of 2N samples
    const int t = idx % T, gi = idx / T, al = a0 + t;
    if (al >= g.na) continue;
    const long long o = (long long)gi * plane_sz + (long long)row * g.na + al;
    const double2 y = r[t * ld + E::at(gi)];
    if (REAL)
      static_cast<double*>(fout)[o] = y.x;
    else
      static_cast<double2*>(fout)[o] = cconj(y);
  }
}

// Persistent variants of the alpha stages: a CTA walks its sequences
// blockIdx.x, + gridDim.x, ... and issues the next sequence's global loads
// into registers before the current sequence's passes, so the load latency
// hides behind the DFT.  Same element arithmetic as inv_alpha_kernel /
// fwd_alpha_kernel.
template <class E>
__global__ void __launch_bounds__(E::NT, E::MINB) inv_alpha_pf_kernel(Geometry g, FftPlan P, double2* __restrict__ W) {
  static_assert(E::fixed && E::T == 1, "one sequence per CTA");
  extern __shared__ double2 sm[];
  constexpr int NT = E::NT, Pn = E::nP, NPT = (Pn + NT - 1) / NT;
  double2* a = sm;
  double2* b = sm + E::LD;
  const int L = g.L, nrows = g.nplanes * g.nb;
  double2 pre[NPT];
  auto fetch = [&](int row) {
    const double2* src = W + row_off(g, row) + (L - 1);
#pragma unroll
    for (int i = 0; i < NPT; i++) {
      const int k = threadIdx.x + i * NT;
      const int m = k <= L - 1 ? k : k - Pn;
      pre[i] = (k < Pn && m >= -(L - 1)) ? src[m] : make_double2(0.0, 0.0);  // MWSS Nyquist k = L stays zero
    }
  };
  int row = blockIdx.x;
  if (row < nrows) fetch(row);
  for (; row < nrows; row += gridDim.x) {
#pragma unroll
    for (int i = 0; i < NPT; i++) {
      const int k = threadIdx.x + i * NT;
      if (k < Pn) a[E::at(k)] = cconj(pre[i]);
    }
    __syncthreads();
    if (row + gridDim.x < nrows) fetch(row + gridDim.x);
    double2* dst = W + row_off(g, row);
    E::runPOut(a, b, P, [&](int, int k, double2 v) {
      if (k < g.na) dst[k] = cconj(v);
    });
  }
}

// ------------------------------------------------------------------ forward
template <bool REAL, class E>
__global__ void __launch_bounds__(E::NT, E::MINB) fwd_gamma_kernel(Geometry g, FftPlan P, const void* __restrict__ fin,
                                                              double2* __restrict__ W, int T_, int ld_, int row0) {
  extern __shared__ double2 sm[];
  const int T = E::fixed ? E::T : T_, ld = E::fixed ? E::LD : ld_;
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int row = row0 + blockIdx.y, a0 = blockIdx.x * T, ng = g.ng;
  const long long plane_sz = (long long)g.nb * g.na;
  // 2 pi / (2N-1); steerable (so3_core.c:309-328): 2 pi / N over the N samples
  const double scale = 2.0 * 3.141592653589793238462643383279502884 / g.nf;
  if constexpr (!REAL && E::io) {
    // the plan reads gamma sample k and writes plane (k + plane0) mod ng
    // straight from / to global memory (complex: nplanes == ng)
    const double2* f = static_cast<const double2*>(fin);
    auto in = [&](int t, int k) {
      const int al = a0 + t;
      return al < g.na ? f[(long long)k * plane_sz + (long long)row * g.na + al] : make_double2(0.0, 0.0);
    };
    auto out = [&](int t, int k, double2 y) {
      const int al = a0 + t;
      int p = k + g.plane0;
      if (p >= ng) p -= ng;
      if (al < g.na) W[(long long)p * g.PS + (long long)row * g.RS + al] = cscale(y, scale);
    };
    E::runIO(in, out, a, b, P);
    return;
  }
  for (int idx = threadIdx.x; idx < ng * T; idx += E::NT) {
    const int t = idx % T, gi = idx / T, al = a0 + t;
    double2 v = make_double2(0.0, 0.0);
    if (al < g.na && gi < g.nf) {  // steerable: samples N..2N-1 of the circle are zero
      const long long o = (long long)gi * plane_sz + (long long)row * g.na + al;
      if (REAL)
        v = make_double2(static_cast<const double*>(fin)[o], 0.0);
      else
        v = static_cast<const double2*>(fin)[o];
    }
    a[t * ld + E::at(gi)] = v;
  }
  __syncthreads();
  double2* r = E::runP(a, b, T, ld, P);
  for (int idx = threadIdx.x; idx < g.nplanes * T; idx += E::NT) {
    const int t = idx % T, p = idx / T, al = a0 + t;
    if (al >= g.na) continue;
    const int k = REAL ? p : wrap1(p - g.plane0, ng);
    // steerable: only n = N-1 (mod 2) is analysed (so3_core.c:315); the other planes are zero
    const bool keep = !g.steer || (((p - g.plane0) - (g.N - 1)) & 1) == 0;
    W[(long long)p * g.PS + (long long)row * g.RS + al] =
        keep ? cscale(r[t * ld + E::at(k)], scale) : make_double2(0.0, 0.0);
  }
}

template <class E>
__global__ void __launch_bounds__(E::NT, E::MINB) fwd_alpha_kernel(Geometry g, FftPlan P, double2* __restrict__ W,
                                                              int T_, int ld_) {
  extern __shared__ double2 sm[];
  const int T = E::fixed ? E::T : T_, ld = E::fixed ? E::LD : ld_;
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int L = g.L, Pn = g.P, nrows = g.nplanes * g.nb, ncols = 2 * L - 1;
  const int r0 = blockIdx.x * T;
  if constexpr (E::fixed) {  // row offsets once per sequence, no index division per element
    for (int j = 0; j < E::T; j++) {
      const int row = r0 + j;
      const double2* src = W + (row < nrows ? row_off(g, row) : 0);
      for (int k = threadIdx.x; k < E::nP; k += E::NT)
        a[j * ld + E::at(k)] = row < nrows ? src[k] : make_double2(0.0, 0.0);
    }
  } else {
    for (int idx = threadIdx.x; idx < T * Pn; idx += E::NT) {
      const int j = idx / Pn, k = idx - j * Pn, row = r0 + j;
      a[j * ld + E::at(k)] = row < nrows ? W[row_off(g, row) + k] : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
  double2* r = E::runP(a, b, T, ld, P);
  const double inv = 1.0 / Pn;
  if constexpr (E::fixed) {
    for (int j = 0; j < E::T; j++) {
      const int row = r0 + j;
      if (row >= nrows) break;
      double2* dst = W + row_off(g, row);
      for (int c = threadIdx.x; c < ncols; c += E::NT)
        dst[c] = cscale(r[j * ld + E::at(wrap1(c - (L - 1), Pn))], inv);
    }
  } else {
    for (int idx = threadIdx.x; idx < T * ncols; idx += E::NT) {
      const int j = idx / ncols, c = idx - j * ncols, row = r0 + j;
      if (row < nrows) W[row_off(g, row) + c] = cscale(r[j * ld + E::at(wrap1(c - (L - 1), Pn))], inv);
    }
  }
}

template <class E>
__global__ void __launch_bounds__(E::NT, E::MINB) fwd_alpha_pf_kernel(Geometry g, FftPlan P, double2* __restrict__ W) {
  static_assert(E::fixed && E::T == 1, "one sequence per CTA");
  extern __shared__ double2 sm[];
  constexpr int NT = E::NT, Pn = E::nP, NPT = (Pn + NT - 1) / NT;
  double2* a = sm;
  double2* b = sm + E::LD;
  const int L = g.L, nrows = g.nplanes * g.nb, ncols = 2 * L - 1;
  const double inv = 1.0 / Pn;
  double2 pre[NPT];
  auto fetch = [&](int row) {
    const double2* src = W + row_off(g, row);
#pragma unroll
    for (int i = 0; i < NPT; i++) {
      const int k = threadIdx.x + i * NT;
      pre[i] = k < Pn ? src[k] : make_double2(0.0, 0.0);
    }
  };
  int row = blockIdx.x;
  if (row < nrows) fetch(row);
  for (; row < nrows; row += gridDim.x) {
#pragma unroll
    for (int i = 0; i < NPT; i++) {
      const int k = threadIdx.x + i * NT;
      if (k < Pn) a[E::at(k)] = pre[i];
    }
    __syncthreads();
    if (row + gridDim.x < nrows) fetch(row + gridDim.x);
    double2* dst = W + row_off(g, row);
    E::runPOut(a, b, P, [&](int, int k, double2 v) {  // frequency k -> column m + L - 1
      const int c = k <= L - 1 ? k + L - 1 : k - Pn + L - 1;
      if (c >= 0 && c < ncols) dst[c] = cscale(v, inv);
    });
  }
}

// Forward beta stage, two columns per pipeline.  Per column (plane n,
// order m, s = (-1)^{m+n}): extend the beta samples onto the circle with
// x(mirror(b)) = s x(b) (mirror(b) = 2L-2-b for MW, 2L-b for MWSS), DFT,
// divide by P, MW phase e^{-i m'' pi/P}, convolve with the quadrature weights
// w (so3_sampling.c:32-51) through a power-of-two oversampled product and
// fold G(m') + s G(-m') onto m' >= 0.  The spectrum v of an s = +1 column is
// even in m'', that of an s = -1 column odd, and w = w_e + w_o with w_e the
// even weights and w_o nonzero at p = +-1 only; so for a pair A (s = +1), B
// (s = -1) pushed through ONE extension, DFT and convolution with w_e:
//   out_A(m') = G(m') + G(-m')   (m' >= 1),   out_A(0) = G(0)
//   out_B(m') = G(m') - G(-m')   (m' >= 1),   out_B(0) = i pi^2 (v(1) - v(-1))
// (the terms of w_o cancel in both folds except in out_B(0)).  This holds for
// the antisymmetric part of B; B's samples at its self-mirror rows (MW: row
// L-1; MWSS: rows 0 and L), which the unpaired extension keeps as they are,
// are taken out of the pipeline and added back through the stage's response
// to a unit sample there (the vectors h of the weight table).  Sequence t of
// a CTA is column pair q = blockIdx.x * T + t (columns 2q, 2q+1).
template <class E>
__global__ void __launch_bounds__(E::NT, E::MINB) fwd_beta_conv_kernel(Geometry g, FftPlan P, FftPlan Pc,
                                                                  const double2* __restrict__ wr,
                                                                  double2* __restrict__ W, int T_, int ld_) {
  extern __shared__ double2 sm[];
  constexpr int TS = E::fixed ? E::T : 8;
  __shared__ double2 selfB[TS][2];  // B's samples at its self-mirror rows
  __shared__ double2 b0[TS];        // out_B(0)
  const int T = E::fixed ? E::T : T_, ld = E::fixed ? E::LD : ld_;
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int plane = blockIdx.y, n = plane - g.plane0;
  const int q0 = blockIdx.x * T, L = g.L, ncols = 2 * L - 1, Pn = g.P, pc = g.Pc;
  const bool first_is_a = ((L - 1 + n) & 1) == 0;  // column 2q has m + n even
  const int sm0 = g.mw ? L - 1 : 0, sm1 = g.mw ? -1 : L;
  const double2* base = W + (long long)plane * g.PS;
  auto fetch = [&](int t, int row, double2& v0, double2& v1) {
    const int c = 2 * (q0 + t);
    v0 = c < ncols ? base[(long long)row * g.RS + c] : make_double2(0.0, 0.0);
    v1 = c + 1 < ncols ? base[(long long)row * g.RS + c + 1] : make_double2(0.0, 0.0);
  };
  auto put = [&](int t, int row, double2 v0, double2 v1) {
    const double2 A = first_is_a ? v0 : v1;
    double2 B = first_is_a ? v1 : v0;
    if (row == sm0 || row == sm1) {
      selfB[t][row == sm0 ? 0 : 1] = B;
      B = make_double2(0.0, 0.0);
    }
    a[t * ld + E::at(row)] = cadd(A, B);
    const int mr = g.mw ? 2 * L - 2 - row : 2 * L - row;  // mirror row on the extended circle
    if (mr >= g.nb && mr < Pn) a[t * ld + E::at(mr)] = csub(A, B);
  };
  constexpr int LC = E::fixed ? (E::nP + 1) / 2 : 0;  // nb of the MW circle of an odd fixed plan
  if (E::fixed && g.nb == LC) {  // all loads of a sequence before its first shared-memory store
    constexpr int NI = E::fixed ? (LC + E::NT - 1) / E::NT : 1;
    for (int t = 0; t < T; t++) {
      double2 v0[NI], v1[NI];
#pragma unroll
      for (int i = 0; i < NI; i++) {
        const int row = threadIdx.x + i * E::NT;
        if (row < LC) fetch(t, row, v0[i], v1[i]);
      }
#pragma unroll
      for (int i = 0; i < NI; i++) {
        const int row = threadIdx.x + i * E::NT;
        if (row < LC) put(t, row, v0[i], v1[i]);
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < g.nb * T; idx += E::NT) {
      const int t = idx % T, row = idx / T;
      double2 v0, v1;
      fetch(t, row, v0, v1);
      put(t, row, v0, v1);
    }
  }
  __syncthreads();
  double2* r = E::runP(a, b, T, ld, P);
  // conv input: F[m''] / P with the MW phase, at m'' mod Pc, zero elsewhere
  const double invP = 1.0 / Pn;
  double2* o = (r == a) ? b : a;
  for (int idx = threadIdx.x; idx < T * pc; idx += E::NT) {
    const int t = idx / pc, k = idx - t * pc;
    o[t * ld + E::atC(k)] = make_double2(0.0, 0.0);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < T * (2 * L - 1); idx += E::NT) {
    const int t = idx / (2 * L - 1), mpp = idx - t * (2 * L - 1) - (L - 1);
    double2 v = cscale(r[t * ld + E::at(wrapi(mpp, Pn))], invP);
    if (g.mw) {  // e^{-i pi m''/(2L-1)}
      const double2 e = __ldg(P.half + (mpp < 0 ? -mpp : mpp));
      v = cmul(v, mpp < 0 ? cconj(e) : e);
    }
    o[t * ld + E::atC(wrapi(mpp, pc))] = cconj(v);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < T; t += E::NT) {
    // i pi^2 (v(1) - v(-1)); o holds conj(v).  Read before the first pass of
    // the convolution below overwrites o (after its first barrier).
    double2 d = make_double2(0.0, 0.0);
    if (L > 1) d = cconj(csub(o[t * ld + E::atC(1)], o[t * ld + E::atC(pc - 1)]));
    const double pi2 = 9.8696044010893586188344909998761511;
    b0[t] = make_double2(-pi2 * d.y, pi2 * d.x);
  }
  double2* o2 = (o == a) ? b : a;
  double2* q = E::runC(o, o2, T, ld, Pc);  // conj of the inverse DFT
  for (int idx = threadIdx.x; idx < T * pc; idx += E::NT) {
    const int t = idx / pc, k = idx - t * pc;
    q[t * ld + E::atC(k)] = cscale(cconj(q[t * ld + E::atC(k)]), __ldg(&wr[k].x));  // real spectrum of w_e
  }
  __syncthreads();
  double2* q2 = (q == a) ? b : a;
  double2* G = E::runC(q, q2, T, ld, Pc);
  double2* cbase = W + g.QOFF + (long long)plane * g.QS;  // column-major output
  const double2* h0 = wr + pc;
  const double2* h1 = wr + pc + L;
  for (int idx = threadIdx.x; idx < L * T; idx += E::NT) {
    const int mp = idx % L, t = idx / L, c = 2 * (q0 + t);  // m' fastest: whole columns written contiguously
    if (c >= ncols) continue;
    const double2 gp = G[t * ld + E::atC(mp)];
    double2 oa = gp, ob = b0[t];
    if (mp > 0) {
      const double2 gm = G[t * ld + E::atC(pc - mp)];
      oa = cadd(gp, gm);
      ob = csub(gp, gm);
    }
    ob = cadd(ob, cmul(selfB[t][0], __ldg(h0 + mp)));
    if (!g.mw) ob = cadd(ob, cmul(selfB[t][1], __ldg(h1 + mp)));
    const int ca = first_is_a ? c : c + 1, cb = first_is_a ? c + 1 : c;
    if (ca < ncols) cbase[(long long)ca * g.CS + mp] = oa;
    if (cb < ncols) cbase[(long long)cb * g.CS + mp] = ob;
  }
}

// ------------------------------------------------------------------ adjoint
// Beta stages of the adjoint transforms (reference src/c/so3_adjoint.c, MW;
// complex planes n = -(N-1)..N-1 or real planes n >= 0).  Generic engines
// only (any length); one column (plane n, order m, s = (-1)^{m+n}) per
// sequence.
//
// Inverse adjoint (so3_adjoint.c:190-231): the nb beta samples zero-extended
// onto the 2L-1 circle, forward DFT, phase e^{-i m' pi/(2L-1)}, folded
// F(m') + s F(-m') onto m' >= 0 (the contraction's sum over -l <= m' <= l).
template <class E>
__global__ void __launch_bounds__(E::NT, E::MINB) adj_inv_beta_kernel(Geometry g, FftPlan P, double2* __restrict__ W,
                                                                 int T_, int ld_) {
  static_assert(!E::fixed, "generic engines");
  extern __shared__ double2 sm[];
  const int T = T_, ld = ld_;
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int plane = blockIdx.y, n = plane - g.plane0;
  const int c0 = blockIdx.x * T, L = g.L, ncols = 2 * L - 1, Pn = g.P;
  const double2* base = W + (long long)plane * g.PS;
  for (int idx = threadIdx.x; idx < Pn * T; idx += E::NT) {
    const int t = idx % T, row = idx / T, c = c0 + t;  // columns fastest: rows read contiguously
    a[t * ld + row] = (row < g.nb && c < ncols) ? base[(long long)row * g.RS + c] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const double2* r = E::runP(a, b, T, ld, P);
  double2* cbase = W + g.QOFF + (long long)plane * g.QS;
  for (int idx = threadIdx.x; idx < L * T; idx += E::NT) {
    const int mp = idx % L, t = idx / L, c = c0 + t;
    if (c >= ncols) continue;
    const int m = c - (L - 1);
    const double sg = ((m + n) & 1) ? -1.0 : 1.0;
    const double2 e = __ldg(P.half + mp);  // e^{-i pi m'/(2L-1)}
    double2 v = cmul(r[t * ld + mp], e);
    if (mp > 0) v = cadd(v, cscale(cmul(r[t * ld + Pn - mp], cconj(e)), sg));
    cbase[(long long)c * g.CS + mp] = v;
  }
}

// Forward adjoint (so3_adjoint.c:718-896): G(-m') = s G(m') extended from
// the contraction's m' >= 0, convolved with the quadrature weights (F(m'') =
// 4 pi^2 sum_{m'} G(m') w(m'' - m'), through the Pc-point product with the
// table's full-weight spectrum), phase e^{+i m'' pi/(2L-1)}, inverse DFT over
// the 2L-1 circle divided by 2L-1, and the adjoint of the periodic
// extension: out(b) = y(b) + s y(2L-2-b) for b < L-1, out(L-1) = y(L-1).
template <class E>
__global__ void __launch_bounds__(E::NT, E::MINB) adj_fwd_beta_kernel(Geometry g, FftPlan P, FftPlan Pc,
                                                                 const double2* __restrict__ wr,
                                                                 double2* __restrict__ W, int T_, int ld_) {
  static_assert(!E::fixed, "generic engines");
  extern __shared__ double2 sm[];
  const int T = T_, ld = ld_;
  double2* a = sm;
  double2* b = sm + (size_t)T * ld;
  const int plane = blockIdx.y, n = plane - g.plane0;
  const int c0 = blockIdx.x * T, L = g.L, ncols = 2 * L - 1, Pn = g.P, pc = g.Pc;
  const double2* cbase = W + g.QOFF + (long long)plane * g.QS;
  for (int idx = threadIdx.x; idx < pc * T; idx += E::NT) {
    const int k = idx % pc, t = idx / pc, c = c0 + t;  // m' fastest: columns read contiguously
    double2 v = make_double2(0.0, 0.0);
    if (c < ncols) {
      const int m = c - (L - 1);
      const double sg = ((m + n) & 1) ? -1.0 : 1.0;
      if (k < L) v = cbase[(long long)c * g.CS + k];
      else if (k > pc - L) v = cscale(cbase[(long long)c * g.CS + (pc - k)], sg);
    }
    a[t * ld + k] = v;
  }
  __syncthreads();
  double2* y = E::runC(a, b, T, ld, Pc);  // forward DFT
  const double2* wf = wr + 2 * (size_t)L + pc;
  for (int idx = threadIdx.x; idx < pc * T; idx += E::NT) {
    const int k = idx % pc, t = idx / pc;
    y[t * ld + k] = cconj(cmul(y[t * ld + k], __ldg(wf + k)));
  }
  __syncthreads();
  double2* o = (y == a) ? b : a;
  double2* cv = E::runC(y, o, T, ld, Pc);  // conj: 4 pi^2 (G * w)
  double2* d = (cv == a) ? b : a;
  for (int idx = threadIdx.x; idx < Pn * T; idx += E::NT) {
    const int k = idx % Pn, t = idx / Pn;
    const int mpp = k <= L - 1 ? k : k - Pn;  // m'' in [-(L-1), L-1]
    const double2 F = cconj(cv[t * ld + (mpp < 0 ? mpp + pc : mpp)]);
    const double2 e = __ldg(P.half + (mpp < 0 ? -mpp : mpp));  // e^{-i pi |m''|/(2L-1)}
    const double2 ph = mpp < 0 ? e : cconj(e);                   // e^{+i pi m''/(2L-1)}
    d[t * ld + k] = cconj(cmul(F, ph));
  }
  __syncthreads();
  double2* other = (d == a) ? b : a;
  const double2* yb = E::runP(d, other, T, ld, P);  // conj: (2L-1) y(b)
  const double invP = 1.0 / Pn;
  double2* base = W + (long long)plane * g.PS;
  for (int idx = threadIdx.x; idx < g.nb * T; idx += E::NT) {
    const int t = idx % T, row = idx / T, c = c0 + t;  // columns fastest: rows written contiguously
    if (c >= ncols) continue;
    const int m = c - (L - 1);
    const double sg = ((m + n) & 1) ? -1.0 : 1.0;
    double2 v = cscale(cconj(yb[t * ld + row]), invP);
    if (row < L - 1) v = cadd(v, cscale(cconj(yb[t * ld + (Pn - 1 - row)]), sg * invP));
    base[(long long)row * g.RS + c] = v;
  }
}

// ------------------------------------------------------------------ launchers
namespace {

enum class Eng { kGenSmall, kGenBig, k1023, k127, k127r };
Eng pick(const FftPlan& p) {
  if (!p.blue && p.n == 1023) return Eng::k1023;
  if (p.blue && p.n == 127 && p.rkern) return Eng::k127r;
  if (p.blue && p.n == 127 && p.m == 256) return Eng::k127;
  return p.big() ? Eng::kGenBig : Eng::kGenSmall;
}

// Launch geometry of one engine: sequences per CTA and shared memory.
template <class E>
Sizing sizing(int ld, int Tmax) {
  if constexpr (E::fixed) return Sizing{E::T, E::smem()};
  return size_for(E::MINB == 1, ld, Tmax);
}

template <class E>
int inv_beta(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const Sizing z = sizing<E>(p.ld(), 16);
  dim3 grid((g.L + z.T - 1) / z.T, g.nplanes);  // L column pairs per plane
  if (int rc = set_smem(inv_beta_kernel<E>, z.smem)) return rc;
  inv_beta_kernel<E><<<grid, E::NT, z.smem, s>>>(g, p, W, z.T, p.ld());
  return kOk;
}
// Grid of a persistent kernel: as many CTAs as fit on the device at once.
template <typename K>
int persistent_grid(K kernel, int nt, size_t smem, int ntiles, int* grid) {
  int dev = 0, sms = 0, per_sm = 0;
  SO3G_CUDA(cudaGetDevice(&dev));
  SO3G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  SO3G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, nt, smem));
  *grid = std::max(1, std::min(ntiles, sms * std::max(per_sm, 1)));
  return kOk;
}

template <class E>
int inv_alpha_pf(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const size_t smem = 2 * (size_t)E::LD * sizeof(double2);
  if (int rc = set_smem(inv_alpha_pf_kernel<E>, smem)) return rc;
  int grid = 0;
  if (int rc = persistent_grid(inv_alpha_pf_kernel<E>, E::NT, smem, g.nplanes * g.nb, &grid)) return rc;
  inv_alpha_pf_kernel<E><<<grid, E::NT, smem, s>>>(g, p, W);
  return kOk;
}

template <class E>
int fwd_alpha_pf(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const size_t smem = 2 * (size_t)E::LD * sizeof(double2);
  if (int rc = set_smem(fwd_alpha_pf_kernel<E>, smem)) return rc;
  int grid = 0;
  if (int rc = persistent_grid(fwd_alpha_pf_kernel<E>, E::NT, smem, g.nplanes * g.nb, &grid)) return rc;
  fwd_alpha_pf_kernel<E><<<grid, E::NT, smem, s>>>(g, p, W);
  return kOk;
}

template <class E>
int inv_alpha(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const Sizing z = sizing<E>(p.ld(), 16);
  const int nrows = g.nplanes * g.nb;
  if (int rc = set_smem(inv_alpha_kernel<E>, z.smem)) return rc;
  inv_alpha_kernel<E><<<(nrows + z.T - 1) / z.T, E::NT, z.smem, s>>>(g, p, W, z.T, p.ld());
  return kOk;
}
template <bool REAL, class E>
int inv_gamma(const Geometry& g, const FftPlan& p, const double2* W, void* f, cudaStream_t s, int row_lo,
              int row_hi) {
  const int ld = p.ld() > g.nplanes ? p.ld() : g.nplanes;
  const Sizing z = sizing<E>(ld, 16);
  dim3 grid((g.na + z.T - 1) / z.T, row_hi - row_lo);
  if (int rc = set_smem(inv_gamma_kernel<REAL, E>, z.smem)) return rc;
  inv_gamma_kernel<REAL, E><<<grid, E::NT, z.smem, s>>>(g, p, W, f, z.T, ld, row_lo);
  return kOk;
}
template <bool REAL, class E>
int fwd_gamma(const Geometry& g, const FftPlan& p, const void* f, double2* W, cudaStream_t s, int row_lo,
              int row_hi) {
  const Sizing z = sizing<E>(p.ld(), 16);
  dim3 grid((g.na + z.T - 1) / z.T, row_hi - row_lo);
  if (int rc = set_smem(fwd_gamma_kernel<REAL, E>, z.smem)) return rc;
  fwd_gamma_kernel<REAL, E><<<grid, E::NT, z.smem, s>>>(g, p, f, W, z.T, p.ld(), row_lo);
  return kOk;
}
template <class E>
int fwd_alpha(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const Sizing z = sizing<E>(p.ld(), 16);
  const int nrows = g.nplanes * g.nb;
  if (int rc = set_smem(fwd_alpha_kernel<E>, z.smem)) return rc;
  fwd_alpha_kernel<E><<<(nrows + z.T - 1) / z.T, E::NT, z.smem, s>>>(g, p, W, z.T, p.ld());
  return kOk;
}
template <class E>
int fwd_beta_conv(const Geometry& g, const FftPlan& p, const FftPlan& pc, const double2* wr, double2* W,
                  cudaStream_t s) {
  const int ld = p.ld() > pc.ld() ? p.ld() : pc.ld();
  const Sizing z = sizing<E>(ld, 8);
  dim3 grid((g.L + z.T - 1) / z.T, g.nplanes);  // L column pairs per plane
  if (int rc = set_smem(fwd_beta_conv_kernel<E>, z.smem)) return rc;
  fwd_beta_conv_kernel<E><<<grid, E::NT, z.smem, s>>>(g, p, pc, wr, W, z.T, ld);
  return kOk;
}

int launched() {
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace

int launch_inv_beta(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  int rc;
  const int v = g.var[kStInvBeta];
  switch (pick(p)) {
    case Eng::k1023:
      rc = v == 1   ? inv_beta<E1023b>(g, p, W, s)
           : v == 2 ? inv_beta<E1023c>(g, p, W, s)
           : v == 3 ? inv_beta<E1023c2>(g, p, W, s)
                    : inv_beta<E1023a>(g, p, W, s);
      break;
    case Eng::k127:
      rc = v == 1 ? inv_beta<E127b>(g, p, W, s) : v == 2 ? inv_beta<E127c>(g, p, W, s) : inv_beta<E127a>(g, p, W, s);
      break;
    case Eng::k127r:
      rc = v == 1 ? inv_beta<E127rb>(g, p, W, s) : v == 2 ? inv_beta<E127rc>(g, p, W, s) : inv_beta<E127ra>(g, p, W, s);
      break;
    case Eng::kGenBig: rc = inv_beta<Gen<true>>(g, p, W, s); break;
    default: rc = inv_beta<Gen<false>>(g, p, W, s); break;
  }
  return rc ? rc : launched();
}

int launch_inv_alpha(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  int rc;
  const int v = g.var[kStInvAlpha];
  switch (pick(p)) {
    case Eng::k1023:
      rc = v == 1   ? inv_alpha<E1023b>(g, p, W, s)
           : v == 2 ? inv_alpha<E1023c>(g, p, W, s)
           : v == 3 ? inv_alpha_pf<E1023p>(g, p, W, s)
                    : inv_alpha<E1023a>(g, p, W, s);
      break;
    case Eng::k127:
      rc = v == 1 ? inv_alpha<E127b>(g, p, W, s) : v == 2 ? inv_alpha<E127c>(g, p, W, s) : inv_alpha<E127a>(g, p, W, s);
      break;
    case Eng::k127r:
      rc = v == 1 ? inv_alpha<E127rb>(g, p, W, s) : v == 2 ? inv_alpha<E127rc>(g, p, W, s)
                                                             : inv_alpha<E127ra>(g, p, W, s);
      break;
    case Eng::kGenBig: rc = inv_alpha<Gen<true>>(g, p, W, s); break;
    default: rc = inv_alpha<Gen<false>>(g, p, W, s); break;
  }
  return rc ? rc : launched();
}

int launch_inv_gamma(const Geometry& g, const FftPlan& p, const double2* W, void* f, cudaStream_t s, int row_lo,
                     int row_hi) {
  if (row_hi < 0 || row_hi > g.nb) row_hi = g.nb;
  if (row_lo >= row_hi) return kOk;
  int rc;
  const Eng e = pick(p);
  const int v = g.var[kStInvGamma];
  if (g.real) {
    rc = e == Eng::kGenBig ? inv_gamma<true, Gen<true>>(g, p, W, f, s, row_lo, row_hi)
                           : inv_gamma<true, Gen<false>>(g, p, W, f, s, row_lo, row_hi);
  } else if (e == Eng::k127) {
    rc = v == 1   ? inv_gamma<false, E127b>(g, p, W, f, s, row_lo, row_hi)
         : v == 2 ? inv_gamma<false, E127c>(g, p, W, f, s, row_lo, row_hi)
                  : inv_gamma<false, E127a>(g, p, W, f, s, row_lo, row_hi);
  } else if (e == Eng::k127r) {
    rc = v == 1   ? inv_gamma<false, E127rb>(g, p, W, f, s, row_lo, row_hi)
         : v == 2 ? inv_gamma<false, E127rc>(g, p, W, f, s, row_lo, row_hi)
                  : inv_gamma<false, E127ra>(g, p, W, f, s, row_lo, row_hi);
  } else {
    rc = e == Eng::kGenBig ? inv_gamma<false, Gen<true>>(g, p, W, f, s, row_lo, row_hi)
                           : inv_gamma<false, Gen<false>>(g, p, W, f, s, row_lo, row_hi);
  }
  return rc ? rc : launched();
}

int launch_fwd_gamma(const Geometry& g, const FftPlan& p, const void* f, double2* W, cudaStream_t s, int row_lo,
                     int row_hi) {
  if (row_hi < 0 || row_hi > g.nb) row_hi = g.nb;
  if (row_lo >= row_hi) return kOk;
  int rc;
  const Eng e = pick(p);
  const int v = g.var[kStFwdGamma];
  if (g.real) {
    rc = e == Eng::kGenBig ? fwd_gamma<true, Gen<true>>(g, p, f, W, s, row_lo, row_hi)
                           : fwd_gamma<true, Gen<false>>(g, p, f, W, s, row_lo, row_hi);
  } else if (e == Eng::k127) {
    rc = v == 1   ? fwd_gamma<false, E127b>(g, p, f, W, s, row_lo, row_hi)
         : v == 2 ? fwd_gamma<false, E127c>(g, p, f, W, s, row_lo, row_hi)
                  : fwd_gamma<false, E127a>(g, p, f, W, s, row_lo, row_hi);
  } else if (e == Eng::k127r) {
    rc = v == 1   ? fwd_gamma<false, E127rb>(g, p, f, W, s, row_lo, row_hi)
         : v == 2 ? fwd_gamma<false, E127rc>(g, p, f, W, s, row_lo, row_hi)
                  : fwd_gamma<false, E127ra>(g, p, f, W, s, row_lo, row_hi);
  } else {
    rc = e == Eng::kGenBig ? fwd_gamma<false, Gen<true>>(g, p, f, W, s, row_lo, row_hi)
                           : fwd_gamma<false, Gen<false>>(g, p, f, W, s, row_lo, row_hi);
  }
  return rc ? rc : launched();
}

int launch_fwd_alpha(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  int rc;
  const int v = g.var[kStFwdAlpha];
  switch (pick(p)) {
    case Eng::k1023:
      rc = v == 1   ? fwd_alpha<E1023b>(g, p, W, s)
           : v == 2 ? fwd_alpha<E1023c>(g, p, W, s)
           : v == 3 ? fwd_alpha_pf<E1023a>(g, p, W, s)
                    : fwd_alpha<E1023a>(g, p, W, s);
      break;
    case Eng::k127:
      rc = v == 1 ? fwd_alpha<E127b>(g, p, W, s) : v == 2 ? fwd_alpha<E127c>(g, p, W, s) : fwd_alpha<E127a>(g, p, W, s);
      break;
    case Eng::k127r:
      rc = v == 1 ? fwd_alpha<E127rb>(g, p, W, s) : v == 2 ? fwd_alpha<E127rc>(g, p, W, s)
                                                             : fwd_alpha<E127ra>(g, p, W, s);
      break;
    case Eng::kGenBig: rc = fwd_alpha<Gen<true>>(g, p, W, s); break;
    default: rc = fwd_alpha<Gen<false>>(g, p, W, s); break;
  }
  return rc ? rc : launched();
}

namespace {
bool conv_fixed(const FftPlan& p, const FftPlan& pc) { return pick(p) == Eng::k1023 && !pc.blue && pc.n == 2048; }
}  // namespace

int launch_fwd_beta_conv(const Geometry& g, const FftPlan& p, const FftPlan& pc, const double2* wr, double2* W,
                         cudaStream_t s) {
  int rc;
  if (conv_fixed(p, pc))
    rc = g.var[kStFwdBetaConv] == 1 ? fwd_beta_conv<EConv1023b>(g, p, pc, wr, W, s)
                                    : fwd_beta_conv<EConv1023a>(g, p, pc, wr, W, s);
  else if (p.big() || pc.big())
    rc = fwd_beta_conv<Gen<true>>(g, p, pc, wr, W, s);
  else
    rc = fwd_beta_conv<Gen<false>>(g, p, pc, wr, W, s);
  return rc ? rc : launched();
}

namespace {
template <class E>
int adj_inv_beta(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  const Sizing z = sizing<E>(p.ld(), 16);
  dim3 grid((2 * g.L - 1 + z.T - 1) / z.T, g.nplanes);
  if (int rc = set_smem(adj_inv_beta_kernel<E>, z.smem)) return rc;
  adj_inv_beta_kernel<E><<<grid, E::NT, z.smem, s>>>(g, p, W, z.T, p.ld());
  return kOk;
}
template <class E>
int adj_fwd_beta(const Geometry& g, const FftPlan& p, const FftPlan& pc, const double2* wr, double2* W,
                 cudaStream_t s) {
  const int ld = p.ld() > pc.ld() ? p.ld() : pc.ld();
  const Sizing z = sizing<E>(ld, 8);
  dim3 grid((2 * g.L - 1 + z.T - 1) / z.T, g.nplanes);
  if (int rc = set_smem(adj_fwd_beta_kernel<E>, z.smem)) return rc;
  adj_fwd_beta_kernel<E><<<grid, E::NT, z.smem, s>>>(g, p, pc, wr, W, z.T, ld);
  return kOk;
}
}  // namespace

int launch_adj_inv_beta(const Geometry& g, const FftPlan& p, double2* W, cudaStream_t s) {
  if (!g.mw) return fail(kUnsupported, "adjoint transforms: MW sampling only");
  const int rc = p.big() ? adj_inv_beta<Gen<true>>(g, p, W, s) : adj_inv_beta<Gen<false>>(g, p, W, s);
  return rc ? rc : launched();
}

int launch_adj_fwd_beta(const Geometry& g, const FftPlan& p, const FftPlan& pc, const double2* wr, double2* W,
                        cudaStream_t s) {
  if (!g.mw) return fail(kUnsupported, "adjoint transforms: MW sampling only");
  const int rc = (p.big() || pc.big()) ? adj_fwd_beta<Gen<true>>(g, p, pc, wr, W, s)
                                       : adj_fwd_beta<Gen<false>>(g, p, pc, wr, W, s);
  return rc ? rc : launched();
}

// ------------------------------------------------------------------ autotuner
int stage_variants(const Geometry& g, const FftPlan& pP, const FftPlan& pg, const FftPlan& pc, int stage) {
  switch (stage) {
    case kStInvBeta:
    case kStInvAlpha:
    case kStFwdAlpha:
      return pick(pP) == Eng::k1023 ? 4 : (pick(pP) == Eng::k127 || pick(pP) == Eng::k127r) ? 3 : 1;
    case kStInvGamma:
    case kStFwdGamma: return (!g.real && (pick(pg) == Eng::k127 || pick(pg) == Eng::k127r)) ? 3 : 1;
    case kStFwdBetaConv: return conv_fixed(pP, pc) ? 2 : 1;
    default: return 1;
  }
}

int autotune_stages(Geometry* g, const FftPlan& pP, const FftPlan& pg, const FftPlan& pc, const double2* wr,
                    double2* W, cudaStream_t s, int reps) {
  const int stages[] = {kStInvBeta, kStInvAlpha, kStInvGamma, kStFwdGamma, kStFwdAlpha, kStFwdBetaConv};
  cudaEvent_t e0, e1;
  SO3G_CUDA(cudaEventCreate(&e0));
  SO3G_CUDA(cudaEventCreate(&e1));
  int rc = kOk;
  for (int st : stages) {
    const int nv = stage_variants(*g, pP, pg, pc, st);
    if (nv <= 1) {
      g->var[st] = 0;
      continue;
    }
    float best = 1e30f;
    int best_v = 0;
    for (int v = 0; v < nv && rc == kOk; v++) {
      g->var[st] = (signed char)v;
      auto run = [&]() -> int {
        switch (st) {
          case kStInvBeta: return launch_inv_beta(*g, pP, W, s);
          case kStInvAlpha: return launch_inv_alpha(*g, pP, W, s);
          case kStInvGamma: return launch_inv_gamma(*g, pg, W, W, s);  // samples written over the scratch
          case kStFwdGamma: return launch_fwd_gamma(*g, pg, W, W, s);
          case kStFwdAlpha: return launch_fwd_alpha(*g, pP, W, s);
          default: return launch_fwd_beta_conv(*g, pP, pc, wr, W, s);
        }
      };
      if ((rc = run())) break;
      if (cudaEventRecord(e0, s) != cudaSuccess) rc = fail(kCudaError, "autotune event");
      for (int i = 0; i < reps && rc == kOk; i++) rc = run();
      if (rc == kOk && cudaEventRecord(e1, s) != cudaSuccess) rc = fail(kCudaError, "autotune event");
      if (rc == kOk && cudaEventSynchronize(e1) != cudaSuccess) rc = fail(kCudaError, "autotune sync");
      float ms = 0.f;
      if (rc == kOk) cudaEventElapsedTime(&ms, e0, e1);
      if (rc == kOk && ms < best) {
        best = ms;
        best_v = v;
      }
    }
    g->var[st] = (signed char)best_v;
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

}  // namespace so3g
