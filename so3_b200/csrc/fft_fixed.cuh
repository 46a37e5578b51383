// Compile-time DFT plans for the lengths that dominate the transform stages.
//
// Same self-sorting (Stockham, decimation in time) passes as fft_core.cuh,
// but with the length, the radix order, the number of sequences per CTA (T),
// their shared-memory pitch (LD) and the CTA size (NT) fixed at compile time:
// every index division becomes a multiply-shift, loop bounds are constants,
// and the odd-radix butterfly constants come from a constant-memory table
// (fft_trig.h) at compile-time offsets, i.e. as constant-bank operands
// instead of registers.  Large odd
// radices run as NG "units" per butterfly, each streaming over the R inputs
// and accumulating one group of output pairs (q, R-q); that keeps register
// use low enough for several CTAs per SM.  Twiddles e^{-2 pi i k/n} come
// from the plan's root table (long double on the host, read through L1).
#pragma once
#include "fft_core.cuh"
#include "fft_trig.h"

namespace so3g {
namespace fx {

// Shared-memory position of element i of a sequence.  Plans with a first
// radix-8 pass (SK = true) leave one pad slot after every 8 elements, so that
// its stride-8 stores (and the T-interleaved staging loops) fall into
// distinct banks; odd-radix plans store densely (SK = false).
template <bool SK>
__host__ __device__ constexpr int phys(int i) { return SK ? i + (i >> 3) : i; }
template <bool SK>
__host__ __device__ constexpr int extent(int n) { return phys<SK>(n - 1) + 1; }

// Odd prime radix, whole butterfly in registers.
template <int R>
__device__ __forceinline__ void bfly_odd(double2* v) {
  constexpr int H = (R - 1) / 2;
  double2 s[H + 1], d[H + 1];
  double2 tot = v[0];
#pragma unroll
  for (int r = 1; r <= H; r++) {
    s[r] = cadd(v[r], v[R - r]);
    d[r] = csub(v[r], v[R - r]);
    tot = cadd(tot, s[r]);
  }
  const double2 v0 = v[0];
  v[0] = tot;
#pragma unroll
  for (int q = 1; q <= H; q++) {
    double ar = v0.x, ai = v0.y, br = 0.0, bi = 0.0;
#pragma unroll
    for (int r = 1; r <= H; r++) {
      const int k = (r * q) % R;
      const double c = k <= H ? kTrigCos[TrigOff<R>::v + k] : kTrigCos[TrigOff<R>::v + R - k];
      const double sn = k <= H ? kTrigSin[TrigOff<R>::v + k] : -kTrigSin[TrigOff<R>::v + R - k];
      ar = fma(c, s[r].x, ar);
      ai = fma(c, s[r].y, ai);
      br = fma(sn, d[r].x, br);
      bi = fma(sn, d[r].y, bi);
    }
    v[q] = make_double2(ar + bi, ai - br);
    v[R - q] = make_double2(ar - bi, ai + br);
  }
}

template <int R>
__device__ __forceinline__ void bfly_any(double2* v) {
  if constexpr (R == 2 || R == 4 || R == 8)
    bfly<R>(v, nullptr);
  else
    bfly_odd<R>(v);
}

// One output group of an odd-radix butterfly: pairs q = QA..QB (and q = 0
// when ZERO), streaming over the inputs x_r = in[phys<SK>(j + r * M)] (times
// tw^r when TW).  Output q goes to d[phys<SK>(o + q * NS)].
template <int R, int QA, int QB, bool ZERO, int M, int NS, bool TW, bool SK>
__device__ __forceinline__ void odd_group(const double2* __restrict__ in, int j, double2* __restrict__ d, int o,
                                          const double2* __restrict__ roots, int tw_step) {
  constexpr int H = (R - 1) / 2;
  constexpr int G = QB - QA + 1;
  double2 a[G], b[G];
#pragma unroll
  for (int i = 0; i < G; i++) a[i] = b[i] = make_double2(0.0, 0.0);
  const double2 v0 = in[phys<SK>(j)];
  double2 tot = v0;
#pragma unroll
  for (int r = 1; r <= H; r++) {
    double2 xp = in[phys<SK>(j + r * M)], xn = in[phys<SK>(j + (R - r) * M)];
    if constexpr (TW) {
      xp = cmul(xp, __ldg(roots + r * tw_step));
      xn = cmul(xn, __ldg(roots + (R - r) * tw_step));
    }
    const double2 s = cadd(xp, xn), dd = csub(xp, xn);
    if constexpr (ZERO) tot = cadd(tot, s);
#pragma unroll
    for (int i = 0; i < G; i++) {
      const int q = QA + i;
      const int k = (r * q) % R;
      const double c = k <= H ? kTrigCos[TrigOff<R>::v + k] : kTrigCos[TrigOff<R>::v + R - k];
      const double sn = k <= H ? kTrigSin[TrigOff<R>::v + k] : -kTrigSin[TrigOff<R>::v + R - k];
      a[i].x = fma(c, s.x, a[i].x);
      a[i].y = fma(c, s.y, a[i].y);
      b[i].x = fma(sn, dd.x, b[i].x);
      b[i].y = fma(sn, dd.y, b[i].y);
    }
  }
  if constexpr (ZERO) d[phys<SK>(o)] = tot;
#pragma unroll
  for (int i = 0; i < G; i++) {
    const int q = QA + i;
    const double ar = v0.x + a[i].x, ai = v0.y + a[i].y;
    d[phys<SK>(o + q * NS)] = make_double2(ar + b[i].y, ai - b[i].x);
    d[phys<SK>(o + (R - q) * NS)] = make_double2(ar - b[i].y, ai + b[i].x);
  }
}

// One Stockham pass of radix R at stride NS over T sequences of length N
// (sequence t at src[t * LD]).  NG > 1 splits each butterfly into NG output
// groups handled by different threads (odd R only).  The sequence index runs
// fastest over the threads, so the lanes of a warp that work on the same
// butterfly of different sequences read the same twiddles (one cache sector
// for up to T lanes) and, with the pitch LD = 8/T (mod 8) slots, hit
// distinct shared-memory banks.
template <int N, int R, int NS, int T, int LD, int NT, int NG, bool SK>
__device__ __forceinline__ void pass(const double2* __restrict__ src, double2* __restrict__ dst,
                                     const double2* __restrict__ roots) {
  constexpr int M = N / R;
  constexpr int TSTEP = N / (NS * R);
  constexpr int UNITS = M * NG;
  constexpr bool TW = NS > 1;
  for (int u = threadIdx.x; u < T * UNITS; u += NT) {
    const int t = u % T;
    const int rem = u / T;
    const int g = NG == 1 ? 0 : rem / M;
    const int j = NG == 1 ? rem : rem - g * M;
    const int k = j % NS;
    const double2* s = src + t * LD;
    double2* d = dst + t * LD;
    const int o = (j / NS) * NS * R + k;
    if constexpr (NG == 1) {
      double2 v[R];
      v[0] = s[phys<SK>(j)];
#pragma unroll
      for (int r = 1; r < R; r++) {
        double2 x = s[phys<SK>(j + r * M)];
        if constexpr (TW) x = cmul(x, __ldg(roots + r * k * TSTEP));
        v[r] = x;
      }
      bfly_any<R>(v);
#pragma unroll
      for (int q = 0; q < R; q++) d[phys<SK>(o + q * NS)] = v[q];
    } else {
      static_assert(R % 2 == 1 && NG <= 3, "output groups need an odd radix");
      constexpr int H = (R - 1) / 2;
      constexpr int QS = (H + NG - 1) / NG;
      const int tws = k * TSTEP;
      if (g == 0) {
        odd_group<R, 1, QS, true, M, NS, TW, SK>(s, j, d, o, roots, tws);
      } else if constexpr (NG == 2) {
        odd_group<R, QS + 1, H, false, M, NS, TW, SK>(s, j, d, o, roots, tws);
      } else if (g == 1) {
        odd_group<R, QS + 1, 2 * QS, false, M, NS, TW, SK>(s, j, d, o, roots, tws);
      } else {
        odd_group<R, 2 * QS + 1, H, false, M, NS, TW, SK>(s, j, d, o, roots, tws);
      }
    }
  }
}

// A whole-butterfly pass (NG = 1) of the same structure as pass(), with the
// load and the store of each element given as functors: in(t, i) returns
// element i of sequence t of the source, out(t, i, v) stores output i.  Lets
// a permutation or a pointwise factor ride on a pass instead of costing a
// shared-memory round trip of its own.
template <int N, int R, int NS, int T, int NT, class In, class Out>
__device__ __forceinline__ void pass_io(const In& in, const Out& out, const double2* __restrict__ roots) {
  constexpr int M = N / R;
  constexpr int TSTEP = N / (NS * R);
  constexpr bool TW = NS > 1;
  for (int u = threadIdx.x; u < T * M; u += NT) {
    const int t = u % T;
    const int j = u / T;
    const int k = j % NS;
    const int o = (j / NS) * NS * R + k;
    double2 v[R];
    v[0] = in(t, j);
#pragma unroll
    for (int r = 1; r < R; r++) {
      double2 x = in(t, j + r * M);
      if constexpr (TW) x = cmul(x, __ldg(roots + r * k * TSTEP));
      v[r] = x;
    }
    bfly_any<R>(v);
#pragma unroll
    for (int q = 0; q < R; q++) out(t, o + q * NS, v[q]);
  }
}

// ---------------------------------------------------------------- plans
// Each plan: static constexpr n (length), ld (buffer extent per sequence,
// padded by phys), and run(a, b, P) -> buffer holding the result (a and b:
// T * LD entries; element i of sequence t at t * LD + phys<sk>(i)).

// 1023 = 31 * 11 * 3 (the MW alpha / extended-beta length at L = 512).  The
// radix-31 butterflies run as NG output groups (each group reads all 31
// inputs; fewer groups read shared memory less and need more registers);
// every output is accumulated in the same order for any NG.
template <int NG, int T, int LD, int NT>
struct P1023G {
  static constexpr bool sk = false;
  static constexpr bool io = false;  // no run_io form
  static constexpr int n = 1023, ld = extent<sk>(1023);
  static __device__ __forceinline__ double2* run(double2* a, double2* b, const FftPlan& P) {
    pass<1023, 31, 1, T, LD, NT, NG, sk>(a, b, P.roots);
    __syncthreads();
    pass<1023, 11, 31, T, LD, NT, 1, sk>(b, a, P.roots);
    __syncthreads();
    pass<1023, 3, 341, T, LD, NT, 1, sk>(a, b, P.roots);
    __syncthreads();
    return b;
  }
  // Same passes; the last one hands output k of sequence t to out(t, k, X)
  // (straight to global memory) instead of a shared buffer.  Barrier at the
  // end: the last pass reads a.
  struct Seq {
    const double2* p;
    __device__ double2 operator()(int t, int i) const { return p[t * LD + i]; }
  };
  static constexpr bool has_out = true;
  template <class Out>
  static __device__ __forceinline__ void run_out(double2* a, double2* b, const FftPlan& P, const Out& out) {
    pass<1023, 31, 1, T, LD, NT, NG, sk>(a, b, P.roots);
    __syncthreads();
    pass<1023, 11, 31, T, LD, NT, 1, sk>(b, a, P.roots);
    __syncthreads();
    pass_io<1023, 3, 341, T, NT>(Seq{a}, out, P.roots);
    __syncthreads();
  }
};
template <int T, int LD, int NT>
using P1023 = P1023G<3, T, LD, NT>;
template <int T, int LD, int NT>
using P1023n2 = P1023G<2, T, LD, NT>;

// 2048 = 8 * 8 * 8 * 4 (the quadrature-weight convolution length at L = 512).
template <int T, int LD, int NT>
struct P2048 {
  static constexpr bool sk = true;
  static constexpr bool io = false;  // no run_io form
  static constexpr int n = 2048, ld = extent<sk>(2048);
  static __device__ __forceinline__ double2* run(double2* a, double2* b, const FftPlan& P) {
    pass<2048, 8, 1, T, LD, NT, 1, sk>(a, b, P.roots);
    __syncthreads();
    pass<2048, 8, 8, T, LD, NT, 1, sk>(b, a, P.roots);
    __syncthreads();
    pass<2048, 8, 64, T, LD, NT, 1, sk>(a, b, P.roots);
    __syncthreads();
    pass<2048, 4, 512, T, LD, NT, 1, sk>(b, a, P.roots);
    __syncthreads();
    return a;
  }
};

// 256 = 8 * 8 * 4 with an explicit root table (Bluestein inner length).
template <int T, int LD, int NT>
__device__ __forceinline__ double2* fft256(double2* a, double2* b, const double2* roots) {
  pass<256, 8, 1, T, LD, NT, 1, true>(a, b, roots);
  __syncthreads();
  pass<256, 8, 8, T, LD, NT, 1, true>(b, a, roots);
  __syncthreads();
  pass<256, 4, 64, T, LD, NT, 1, true>(a, b, roots);
  __syncthreads();
  return b;
}

// 127 (prime; the gamma length at N = 64) by Bluestein's algorithm over 256.
template <int T, int LD, int NT>
struct P127 {
  static constexpr bool sk = true;
  static constexpr bool io = false;  // no run_io form
  static constexpr int n = 127, ld = extent<sk>(256);
  static __device__ __forceinline__ double2* run(double2* a, double2* b, const FftPlan& P) {
    for (int w = threadIdx.x; w < T * 256; w += NT) {
      const int t = w % T, k = w / T;  // t fastest: lanes of one k share the chirp load
      double2* s = a + t * LD;
      s[phys<true>(k)] = k < 127 ? cmul(s[phys<true>(k)], __ldg(P.chirp + k)) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2* r = fft256<T, LD, NT>(a, b, P.mroots);
    for (int w = threadIdx.x; w < T * 256; w += NT) {
      const int t = w % T, k = w / T;
      double2* s = r + t * LD;
      s[phys<true>(k)] = cconj(cmul(s[phys<true>(k)], __ldg(P.kern + k)));
    }
    __syncthreads();
    double2* o = r == a ? b : a;
    r = fft256<T, LD, NT>(r, o, P.mroots);
    for (int w = threadIdx.x; w < T * 127; w += NT) {
      const int t = w % T, k = w / T;
      double2* s = r + t * LD;
      s[phys<true>(k)] = cmul(__ldg(P.chirp + k), cconj(s[phys<true>(k)]));
    }
    __syncthreads();
    return r;
  }
};

// 127 (prime) by Rader's algorithm: with the primitive root 3,
//   X[3^{-b}] = x[0] + sum_{a < 126} x[3^a] w^{3^{a-b}},   X[0] = sum_n x[n],
// a cyclic convolution of length 126 = 7 * 9 * 2 evaluated as
// conj(FFT(conj(FFT(u) * V))) with V = FFT(v) / 126 precomputed.  About half
// the arithmetic of Bluestein over 256 and half its shared memory.  The
// gather x[3^a] rides on the first pass of the first FFT, the product with V
// (and the conjugation) on its last pass, the scatter to X[3^{-b}] on the
// last pass of the second FFT: six passes, no separate shared-memory sweeps
// (the stage is bound by shared-memory traffic).  Input x in a (entries
// 0..126); returns the buffer holding X.
template <int T, int LD, int NT>
struct P127R {
  static constexpr bool sk = false;
  static constexpr int n = 127, ld = extent<sk>(127);
  struct Plain {
    double2* p;
    __device__ double2 operator()(int t, int i) const { return p[t * LD + i]; }
    __device__ void operator()(int t, int i, double2 v) const { p[t * LD + i] = v; }
  };
  template <class In>
  struct Gather {  // element a of the convolution input: x[3^a]
    const In& in;
    const int* perm;
    __device__ double2 operator()(int t, int i) const { return in(t, __ldg(perm + i)); }
  };
  struct Kernel {  // conj(U[k] V[k]); X[0] = x[0] + U[0]
    double2* p;
    const double2* kern;
    const double2* x0;
    double2* X0;
    __device__ void operator()(int t, int k, double2 u) const {
      if (k == 0) X0[t] = cadd(x0[t], u);
      p[t * LD + k] = cconj(cmul(u, __ldg(kern + k)));
    }
  };
  template <class Out>
  struct Scatter {  // X[3^{-b}] = x[0] + conj(second FFT)[b]
    const Out& out;
    const int* perm;
    const double2* x0;
    __device__ void operator()(int t, int b, double2 v) const { out(t, __ldg(perm + b), cadd(x0[t], cconj(v))); }
  };
  // 126 = 7 * 9 * 2 in three passes: source -> t1 -> t2 -> out (the radix-9
  // butterfly direct, which needs no twiddles between two radix-3 passes)
  template <class In, class Out>
  static __device__ __forceinline__ void fft126(const In& in, double2* t1, double2* t2, const Out& out,
                                                const double2* roots) {
    pass_io<126, 7, 1, T, NT>(in, Plain{t1}, roots);
    __syncthreads();
    pass_io<126, 9, 7, T, NT>(Plain{t1}, Plain{t2}, roots);
    __syncthreads();
    pass_io<126, 2, 63, T, NT>(Plain{t2}, out, roots);
  }
  // Element k of input sequence t is in(t, k); output k goes to out(t, k, X).
  // in -> b -> a -> conj(U V) in b -> a -> b -> out: in may read a (x[0] is
  // read before the second pass overwrites a, behind the first pass's
  // barrier) and out may write a.  No barrier after the last stores.
  template <class In, class Out>
  static __device__ __forceinline__ void run_io(const In& in, const Out& out, double2* a, double2* b,
                                                const FftPlan& P) {
    __shared__ double2 x0[T], X0[T];
    for (int t = threadIdx.x; t < T; t += NT) x0[t] = in(t, 0);
    fft126(Gather<In>{in, P.rperm}, b, a, Kernel{b, P.rkern, x0, X0}, P.rroots);
    __syncthreads();
    fft126(Plain{b}, a, b, Scatter<Out>{out, P.rperm + 126, x0}, P.rroots);
    for (int t = threadIdx.x; t < T; t += NT) out(t, 0, X0[t]);
  }
  static constexpr bool io = true;
  static __device__ __forceinline__ double2* run(double2* a, double2* b, const FftPlan& P) {
    const Plain pa{a};
    run_io(pa, pa, a, b, P);
    __syncthreads();
    return a;
  }
};

}  // namespace fx
}  // namespace so3g
