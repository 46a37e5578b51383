// Shared-memory FP64 DFT engine used by every transform stage.
//
// A CTA transforms T sequences that it has staged in shared memory.  Lengths
// whose prime factors are all <= 31 run as a self-sorting (Stockham)
// mixed-radix DFT -- radix 8/4/2 for the power-of-two part and odd prime
// radices with the r / R-r input pairing; any other length runs Bluestein's
// chirp-z algorithm over a power-of-two length m >= 2n-1.  Twiddles and chirp
// tables are evaluated on the host in long double (state.cpp) and read
// through the read-only cache; the odd-radix butterfly constants
// cos/sin(2 pi k/R) are the roots k*n/R of the same table, loaded once per
// pass into registers (every lane reads the same address).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace so3g {

constexpr int kMaxPasses = 16;

struct FftPlan {
  int n;                     // transform length
  int npass;                 // Stockham passes for length n (0 if Bluestein)
  int rad[kMaxPasses];
  int blue;                  // 1 -> Bluestein
  int m;                     // Bluestein length
  int mpass;
  int mrad[kMaxPasses];
  const double2* roots;      // e^{-2 pi i k/n}, k < n     (not Bluestein)
  const double2* mroots;     // e^{-2 pi i k/m}, k < m     (Bluestein)
  const double2* chirp;      // e^{-i pi k^2/n}, k < n     (Bluestein)
  const double2* kern;       // FFT_m(conj chirp) / m      (Bluestein)
  const double2* half;       // e^{-i pi k/n}, k < n       (half-step roots: the MW beta phases)
  // Rader tables (n = 127 only, else null): the prime-length DFT as a cyclic
  // convolution of length n-1 with primitive root 3
  const double2* rroots;     // e^{-2 pi i k/(n-1)}, k < n-1
  const double2* rkern;      // FFT_{n-1}(e^{-2 pi i 3^{-m}/n}) / (n-1)
  const int* rperm;          // [0, n-1): 3^a mod n (gather); [n-1, 2n-2): 3^{-b} mod n (scatter)
  int ld() const { return blue ? m : n; }
  // any radix above 8 (needs the large-radix kernel instances)
  bool big() const {
    for (int i = 0; i < npass; i++)
      if (rad[i] > 8) return true;
    for (int i = 0; i < mpass; i++)
      if (mrad[i] > 8) return true;
    return false;
  }
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by -i
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }

// cs[k] = (cos, sin)(2 pi k / R), k = 1 .. (R-1)/2, used by odd radices only.
template <int R>
__device__ __forceinline__ void bfly(double2* v, const double2* cs) {
  if constexpr (R == 2) {
    double2 a = cadd(v[0], v[1]), b = csub(v[0], v[1]);
    v[0] = a;
    v[1] = b;
  } else if constexpr (R == 4) {
    double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    double2 t2 = cadd(v[1], v[3]), t3 = mul_mi(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  } else if constexpr (R == 8) {
    // two radix-4 on even/odd, then twiddle by e^{-2 pi i k/8} and radix-2
    double2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    bfly<4>(e, nullptr);
    bfly<4>(o, nullptr);
    const double h = 0.70710678118654752440084436210484903928;
    // o1 *= (1 - i)/sqrt2, o2 *= -i, o3 *= (-1 - i)/sqrt2
    double2 o1 = make_double2((o[1].x + o[1].y) * h, (o[1].y - o[1].x) * h);
    double2 o2 = mul_mi(o[2]);
    double2 o3 = make_double2((o[3].y - o[3].x) * h, -(o[3].x + o[3].y) * h);
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  } else {
    constexpr int H = (R - 1) / 2;
    double2 s[H + 1], d[H + 1];
    double2 tot = v[0];
#pragma unroll
    for (int r = 1; r <= H; r++) {
      s[r] = cadd(v[r], v[R - r]);
      d[r] = csub(v[r], v[R - r]);
      tot = cadd(tot, s[r]);
    }
    double2 v0 = v[0];
    v[0] = tot;
#pragma unroll
    for (int q = 1; q <= H; q++) {
      double ar = v0.x, ai = v0.y, br = 0.0, bi = 0.0;
#pragma unroll
      for (int r = 1; r <= H; r++) {
        const int k = (r * q) % R;  // compile-time after unrolling
        const double c = k <= H ? cs[k].x : cs[R - k].x;
        const double sn = k <= H ? cs[k].y : -cs[R - k].y;
        ar = fma(c, s[r].x, ar);
        ai = fma(c, s[r].y, ai);
        br = fma(sn, d[r].x, br);
        bi = fma(sn, d[r].y, bi);
      }
      v[q] = make_double2(ar + bi, ai - br);
      v[R - q] = make_double2(ar - bi, ai + br);
    }
  }
}

// One Stockham pass: T sequences of length n, sequence t at src[t*ld].
template <int R>
__device__ __forceinline__ void stockham_pass(const double2* __restrict__ src, double2* __restrict__ dst,
                                              int n, int Ns, int T, int ld, const double2* __restrict__ roots) {
  const int m = n / R;
  const int tstep = n / (Ns * R);
  const int total = T * m;
  double2 cs[R / 2 + 1];
  if constexpr (R % 2 == 1) {
#pragma unroll
    for (int k = 1; k <= R / 2; k++) {
      const double2 w = __ldg(roots + k * m);  // e^{-2 pi i k/R}
      cs[k] = make_double2(w.x, -w.y);
    }
  }
  for (int w = threadIdx.x; w < total; w += blockDim.x) {
    const int t = w / m;
    const int j = w - t * m;
    const int k = j % Ns;
    const double2* s = src + t * ld;
    double2 v[R];
    v[0] = s[j];
#pragma unroll
    for (int r = 1; r < R; r++) {
      double2 a = s[j + r * m];
      if (k) a = cmul(a, __ldg(roots + r * k * tstep));
      v[r] = a;
    }
    bfly<R>(v, cs);
    double2* d = dst + t * ld + (j / Ns) * Ns * R + k;
#pragma unroll
    for (int q = 0; q < R; q++) d[q * Ns] = v[q];
  }
}

static __device__ __noinline__ void dispatch_big(int R, const double2* src, double2* dst, int n, int Ns, int T, int ld,
                                          const double2* roots) {
  switch (R) {
    case 11: stockham_pass<11>(src, dst, n, Ns, T, ld, roots); break;
    case 13: stockham_pass<13>(src, dst, n, Ns, T, ld, roots); break;
    case 17: stockham_pass<17>(src, dst, n, Ns, T, ld, roots); break;
    case 19: stockham_pass<19>(src, dst, n, Ns, T, ld, roots); break;
    case 23: stockham_pass<23>(src, dst, n, Ns, T, ld, roots); break;
    case 29: stockham_pass<29>(src, dst, n, Ns, T, ld, roots); break;
    case 31: stockham_pass<31>(src, dst, n, Ns, T, ld, roots); break;
    default: break;
  }
}

// BIG selects the radix set: false -> {2,3,4,5,7,8} only (low register use,
// two CTAs per SM), true -> also the odd primes 11..31.
template <bool BIG>
__device__ __forceinline__ void dispatch_pass(int R, const double2* src, double2* dst, int n, int Ns, int T,
                                              int ld, const double2* roots) {
  switch (R) {
    case 2: stockham_pass<2>(src, dst, n, Ns, T, ld, roots); break;
    case 3: stockham_pass<3>(src, dst, n, Ns, T, ld, roots); break;
    case 4: stockham_pass<4>(src, dst, n, Ns, T, ld, roots); break;
    case 5: stockham_pass<5>(src, dst, n, Ns, T, ld, roots); break;
    case 7: stockham_pass<7>(src, dst, n, Ns, T, ld, roots); break;
    case 8: stockham_pass<8>(src, dst, n, Ns, T, ld, roots); break;
    default: if constexpr (BIG) dispatch_big(R, src, dst, n, Ns, T, ld, roots); break;
  }
}
// Runs the passes; data starts in a, returns the buffer holding the result.
template <bool BIG>
__device__ __forceinline__ double2* run_passes(double2* a, double2* b, int n, const int* rad, int npass, int T,
                                               int ld, const double2* roots) {
  int Ns = 1;
  for (int p = 0; p < npass; p++) {
    dispatch_pass<BIG>(rad[p], a, b, n, Ns, T, ld, roots);
    __syncthreads();
    double2* t = a;
    a = b;
    b = t;
    Ns *= rad[p];
  }
  return a;
}

// Forward DFT (e^{-2 pi i jk/n}, unnormalised) of T sequences held in a[t*ld + j],
// j < n; b is scratch of the same size.  Both buffers need ld >= plan.ld().
// Caller must __syncthreads() after staging the input.  Returns the buffer
// holding the n outputs of each sequence.
template <bool BIG>
__device__ __forceinline__ double2* fft_fwd_smem(double2* a, double2* b, int T, int ld, const FftPlan& P) {
  if (P.n == 1) return a;
  if (!P.blue) return run_passes<BIG>(a, b, P.n, P.rad, P.npass, T, ld, P.roots);
  const int n = P.n, m = P.m;
  for (int w = threadIdx.x; w < T * m; w += blockDim.x) {
    const int t = w / m, k = w - t * m;
    double2* s = a + t * ld;
    s[k] = k < n ? cmul(s[k], __ldg(P.chirp + k)) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* r = run_passes<BIG>(a, b, m, P.mrad, P.mpass, T, ld, P.mroots);
  for (int w = threadIdx.x; w < T * m; w += blockDim.x) {
    const int t = w / m, k = w - t * m;
    double2* s = r + t * ld;
    s[k] = cconj(cmul(s[k], __ldg(P.kern + k)));
  }
  __syncthreads();
  double2* o = (r == a) ? b : a;
  r = run_passes<BIG>(r, o, m, P.mrad, P.mpass, T, ld, P.mroots);
  for (int w = threadIdx.x; w < T * n; w += blockDim.x) {
    const int t = w / n, k = w - t * n;
    double2* s = r + t * ld;
    s[k] = cmul(__ldg(P.chirp + k), cconj(s[k]));
  }
  __syncthreads();
  return r;
}

}  // namespace so3g
