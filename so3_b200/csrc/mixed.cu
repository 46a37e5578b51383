// Split-precision Wigner contractions on the int8 tensor cores (Ozaki
// scheme), for batches of complex signals.
//
// For fixed |m| = mu, |n| = nu the FP64 contractions of contract.cu are
// matrix products shared by every signal of a batch:
//   inverse  Y[m', c] = sum_l  A[m', l] X[l, c]     (rows m', reduction l)
//   forward  Y[l, c]  = sum_m' A[m', l] X'[m', c]   (rows l,  reduction m')
// with A[m', l] = Delta^l_{m' mu} Delta^l_{m' nu} (zero for m' > l) and one
// column c per signal, sign combination (+-mu, +-nu) and real / imaginary
// part (8 per signal).  The (-1)^{l+m'} of the combinations with one negative
// index is split as in contract.cu: the factor carrying the reduction index
// goes into X, the other is applied to the output.
//
// Each operand is scaled by a power of two (A: 2, every column of X: the
// smallest power of two above twice its largest magnitude) and split into 7
// int8 slices, r = sum_i q_i 2^{-7i}: the balanced base-128 digits of the
// 49-bit fixed-point value (q_2..q_7 in [-64, 63], q_1 in [-65, 65]), so that
// the dropped low-order products carry no common sign.  The 28
// slice products with i + j <= 8 are accumulated exactly in int32 on
// mma.sync m16n8k32 (one accumulator per diagonal i + j) and combined in FP64.
// The dropped products and the 49-bit rounding leave a normwise error near
// 1e-12 of the contraction, far inside the 1e-10 budget of the split path;
// Delta, the quadrature weights, the DFT stages and the final combination
// stay FP64.
//
// A is generated per CTA from the FP64 Delta table (rows of the quarter
// planes read contiguously through the transpose symmetry
// Delta^l_{m' k} = (-1)^{m'-k} Delta^l_{k m'}), split in registers and staged
// in shared memory; X is split once per batch by a slicing kernel.
#include <cstdint>

#include "so3gpu_internal.h"

namespace so3g {

namespace {

constexpr int kS = 7;            // slices per operand
constexpr int kND = kS;          // diagonals i + j = 2 .. kS + 1
constexpr int kGrp = 8;          // signals per CTA column group
constexpr int kCol = 8;          // columns per signal
constexpr int kRowsB = kGrp * kCol;  // 64 B-operand rows per group
constexpr int kTile = 32;        // CTA rows and K per step
constexpr int kThreads = 256;
constexpr double kInv8Pi2 = 0.012665147955292221430803304553147533;  // 1/(8 pi^2)

struct MixSmem {
  uint8_t A[2][kS][kTile][32];    // [buffer][slice][row][k bytes], 16-byte chunks swizzled
  uint8_t B[2][kS][kRowsB][32];   // [buffer][slice][signal * 8 + column][k bytes]
};

__device__ __forceinline__ int swz(int row, int chunk) { return chunk ^ ((row >> 2) & 1); }

// Splits r in [-1/2, 1/2] into 7 balanced digits (see the file comment);
// q[0] is the most significant.
__device__ __forceinline__ void split7(double r, int (&q)[kS]) {
  const double shifter = 6755399441055744.0;                 // 1.5 * 2^52
  const double y = fma(r, 562949953421312.0, shifter);       // rint(r * 2^49) + shifter
  const long long v = __double_as_longlong(y) - __double_as_longlong(shifter);
  const unsigned lo = (unsigned)v;
  const int hi = (int)(v >> 32);
  q[6] = lo & 127;
  q[5] = (lo >> 7) & 127;
  q[4] = (lo >> 14) & 127;
  q[3] = (lo >> 21) & 127;
  q[2] = ((lo >> 28) | ((unsigned)hi << 4)) & 127;
  q[1] = (hi >> 3) & 127;
  q[0] = hi >> 10;
  // balanced digits in [-64, 63] (carry upwards): the dropped low-order
  // products then have no common sign, so their sum does not grow with K
#pragma unroll
  for (int i = kS - 1; i > 0; i--) {
    const int c = q[i] >= 64;
    q[i] -= c << 7;
    q[i - 1] += c;
  }
}

__device__ __forceinline__ void cp16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ void mma_s8(int (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ double2 ipow(double2 v, int k) {  // v * i^k
  switch (k & 3) {
    case 0: return v;
    case 1: return make_double2(-v.y, v.x);
    case 2: return make_double2(-v.x, -v.y);
    default: return make_double2(v.y, -v.x);
  }
}

// Stores the 7 slice words of 4 consecutive K entries of A row `row`.
__device__ __forceinline__ void store_a(MixSmem& S, int buf, int row, int word, const double (&x)[4]) {
  unsigned w[kS];
#pragma unroll
  for (int i = 0; i < kS; i++) w[i] = 0u;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    int q[kS];
    split7(0.5 * x[e], q);  // A scale 2
#pragma unroll
    for (int i = 0; i < kS; i++) w[i] |= (unsigned)(q[i] & 255) << (8 * e);
  }
  const int off = row * 32 + swz(row, word >> 2) * 16 + (word & 3) * 4;
#pragma unroll
  for (int i = 0; i < kS; i++) *reinterpret_cast<unsigned*>(&S.A[buf][i][0][0] + off) = w[i];
}

// B tile of one K step: 7 slices x 64 rows x 32 bytes from the sliced
// operand (layout [slice][row][Lp]).
__device__ __forceinline__ void load_b(MixSmem& S, int buf, const uint8_t* __restrict__ xs, int Lp, int k0) {
  for (int idx = threadIdx.x; idx < kS * kRowsB * 2; idx += kThreads) {
    const int i = idx / (kRowsB * 2), rem = idx - i * kRowsB * 2, row = rem >> 1, chunk = rem & 1;
    const uint8_t* src = xs + ((size_t)i * kRowsB + row) * Lp + k0 + chunk * 16;
    cp16(&S.B[buf][i][row][swz(row, chunk) * 16], src);
  }
}

// 28 slice products of one K step for a warp tile of 16 rows x 2 signals.
// B slices 0..3 first, then 4..6 (only A slices 0..2 pair with those), so at
// most four B fragments are live.
__device__ __forceinline__ void mma_step(const MixSmem& S, int buf, int msub, int npair, int lane,
                                         int (&acc)[kND][2][4]) {
  const int r8 = lane & 7, which = lane >> 3;
  // B: matrices (sig0, chunk0) (sig0, chunk1) (sig1, chunk0) (sig1, chunk1)
  const int brow = npair * 16 + (which >> 1) * 8 + r8, bchunk = which & 1;
  // A: matrices (rows 0-7, chunk0) (rows 8-15, chunk0) (rows 0-7, chunk1) (rows 8-15, chunk1)
  const int arow = msub * 16 + (which & 1) * 8 + r8, achunk = which >> 1;
  unsigned b[4][4];
#pragma unroll
  for (int j = 0; j < 4; j++) ldsm_x4(b[j], &S.B[buf][j][brow][swz(brow, bchunk) * 16]);
#pragma unroll
  for (int i = 0; i < kS; i++) {
    unsigned a[4];
    ldsm_x4(a, &S.A[buf][i][arow][swz(arow, achunk) * 16]);
#pragma unroll
    for (int j = 0; j < 4 && j < kS - i; j++) {
      mma_s8(acc[i + j][0], a, b[j][0], b[j][1]);
      mma_s8(acc[i + j][1], a, b[j][2], b[j][3]);
    }
  }
#pragma unroll
  for (int j = 4; j < kS; j++) ldsm_x4(b[j - 4], &S.B[buf][j][brow][swz(brow, bchunk) * 16]);
#pragma unroll
  for (int i = 0; i < kS - 4; i++) {
    unsigned a[4];
    ldsm_x4(a, &S.A[buf][i][arow][swz(arow, achunk) * 16]);
#pragma unroll
    for (int j = 4; j < kS - i; j++) {
      mma_s8(acc[i + j][0], a, b[j - 4][0], b[j - 4][1]);
      mma_s8(acc[i + j][1], a, b[j - 4][2], b[j - 4][3]);
    }
  }
}

// FP64 value of one accumulator element (A scale 2 folded in).
__device__ __forceinline__ double combine(const int (&acc)[kND][2][4], int nt, int e) {
  double v = 0.0, w = 2.0 * 0.000061035156250000000;  // 2 * 2^{-14} (diagonal i + j = 2)
#pragma unroll
  for (int d = 0; d < kND; d++) {
    v = fma((double)acc[d][nt][e], w, v);
    w *= 0.0078125;  // 2^{-7}
  }
  return v;
}

struct MixArgs {
  const uint8_t* xs;       // [grp][mu * N + nu][7][64][Lp]
  const double* xscale;    // [grp][mu * N + nu][64]
  const double* dl;        // Delta quarter planes
  const long long* base;   // block bases per plane
  double2* W;              // inverse: per-signal scratch, signal b at W + b * wstride
  double2* const* flmn;    // forward: per-signal coefficient arrays
  long long wstride;
  int L, N, L0, Lp, MT, plane0, n_mode, nsig, compact;
  long long RS, PS;
};

__device__ __forceinline__ void decode(const MixArgs& a, int bx, int* mu, int* nu, int* t) {
  *nu = bx % a.N;
  const int rest = bx / a.N;
  *t = rest % a.MT;
  *mu = rest / a.MT;
}

// ---------------------------------------------------------------- inverse
__global__ void __launch_bounds__(kThreads, 2) mixed_inverse_kernel(MixArgs a) {
  extern __shared__ __align__(128) unsigned char smraw[];
  MixSmem& S = *reinterpret_cast<MixSmem*>(smraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int mu, nu, mt;
  decode(a, blockIdx.x, &mu, &nu, &mt);
  const int grp = blockIdx.y, L = a.L;
  const int m0 = mt * kTile;
  const int lmin = max(max(mu, nu), a.L0);
  const int kfirst = max(lmin, m0) & ~(kTile - 1);
  const int nk = kfirst < L ? (L - kfirst + kTile - 1) / kTile : 0;
  const size_t gp = (size_t)grp * a.L * a.N + (size_t)mu * a.N + nu;  // slicing-kernel order
  const uint8_t* xs = a.xs + gp * kS * kRowsB * (size_t)a.Lp;

  int acc[kND][2][4];
#pragma unroll
  for (int d = 0; d < kND; d++)
#pragma unroll
    for (int n = 0; n < 2; n++)
#pragma unroll
      for (int e = 0; e < 4; e++) acc[d][n][e] = 0;

  // A generation: thread -> row m' = m0 + 8*(warp%4) + lane%8 and K entries
  // l = k0 + 4*word .. +3 with word = 4*(warp/4) + lane/8: the Delta loads of a
  // warp read 8 consecutive m' per plane, and its 32 slice-word stores hit 32
  // distinct banks.
  const int grow = 8 * (warp & 3) + (lane & 7), gword = 4 * (warp >> 2) + (lane >> 3), mp = m0 + grow;
  auto fetch = [&](int k0, double (&x)[4]) {
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int l = k0 + 4 * gword + e;
      double v = 0.0;
      if (l < L && l >= lmin && mp <= l) {
        const double* P = a.dl + dl_plane_offset(l);
        v = P[(long long)mu * (l + 1) + mp] * P[(long long)nu * (l + 1) + mp];
      }
      x[e] = v;
    }
  };

  const int msub = warp & 1, npair = warp >> 1;
  if (nk > 0) {
    double x[4];
    fetch(kfirst, x);
    load_b(S, 0, xs, a.Lp, kfirst);
    cp_commit();
    store_a(S, 0, grow, gword, x);
    for (int k = 0; k < nk; k++) {
      const int buf = k & 1;
      cp_wait_all();
      __syncthreads();
      const bool more = k + 1 < nk;
      if (more) {
        fetch(kfirst + (k + 1) * kTile, x);
        load_b(S, buf ^ 1, xs, a.Lp, kfirst + (k + 1) * kTile);
        cp_commit();
      }
      mma_step(S, buf, msub, npair, lane, acc);
      if (more) store_a(S, buf ^ 1, grow, gword, x);
    }
  }

  // epilogue: thread holds rows g, g+8 of its 16-row sub-tile, columns 2t
  // (re) and 2t+1 (im) of sign combination t, for two signals
  const int g = lane >> 2, t = lane & 3;
  const int ms = (t & 1) ? -1 : 1, ns = (t & 2) ? -1 : 1;
  if ((ms < 0 && mu == 0) || (ns < 0 && nu == 0)) return;
  const int m = ms * mu, n = ns * nu;
  const bool one_neg = ms * ns < 0;
  const double sgn_mn = ((mu + nu) & 1) ? -1.0 : 1.0;
  const double* sc = a.xscale + gp * kRowsB;
#pragma unroll
  for (int nt = 0; nt < 2; nt++) {
    const int b = npair * 2 + nt, sig = grp * kGrp + b;
    if (sig >= a.nsig) continue;
    const double sre = sc[b * kCol + 2 * t], sim = sc[b * kCol + 2 * t + 1];
    double2* W = a.W + (long long)sig * a.wstride + (long long)(a.plane0 + n) * a.PS + (m + L - 1);
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int row = m0 + msub * 16 + g + 8 * h;
      if (row >= L) continue;
      double2 v = make_double2(combine(acc, nt, 2 * h) * sre, combine(acc, nt, 2 * h + 1) * sim);
      const double s = (one_neg && (row & 1)) ? -sgn_mn : sgn_mn;
      v = make_double2(v.x * s, v.y * s);
      W[(long long)row * a.RS] = ipow(v, n - m + 4 * L);
    }
  }
}

// ---------------------------------------------------------------- forward
__global__ void __launch_bounds__(kThreads, 2) mixed_forward_kernel(MixArgs a) {
  extern __shared__ __align__(128) unsigned char smraw[];
  MixSmem& S = *reinterpret_cast<MixSmem*>(smraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int mu, nu, lt;
  decode(a, blockIdx.x, &mu, &nu, &lt);
  const int grp = blockIdx.y, L = a.L;
  const int l0 = lt * kTile;
  const int lmin = max(max(mu, nu), a.L0);
  const bool any_row = l0 + kTile > lmin && l0 < L;
  const int kend = min(L, l0 + kTile);  // m' < kend (A[m', l] = 0 for m' > l)
  const int nk = any_row ? (kend + kTile - 1) / kTile : 0;
  const size_t gp = (size_t)grp * a.L * a.N + (size_t)mu * a.N + nu;
  const uint8_t* xs = a.xs + gp * kS * kRowsB * (size_t)a.Lp;

  int acc[kND][2][4];
#pragma unroll
  for (int d = 0; d < kND; d++)
#pragma unroll
    for (int n = 0; n < 2; n++)
#pragma unroll
      for (int e = 0; e < 4; e++) acc[d][n][e] = 0;

  // A generation: thread -> row l = l0 + tid/8, K entries m' = k0 + 4*(tid%8) .. +3
  const int grow = tid >> 3, gword = tid & 7, l = l0 + grow;
  const bool lrow = l < L && l >= lmin;
  auto fetch = [&](int k0, double (&x)[4]) {
    const double* P = a.dl + (lrow ? dl_plane_offset(l) : 0);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int mp = k0 + 4 * gword + e;
      x[e] = (lrow && mp <= l) ? P[(long long)mu * (l + 1) + mp] * P[(long long)nu * (l + 1) + mp] : 0.0;
    }
  };

  const int msub = warp & 1, npair = warp >> 1;
  if (nk > 0) {
    double x[4];
    fetch(0, x);
    load_b(S, 0, xs, a.Lp, 0);
    cp_commit();
    store_a(S, 0, grow, gword, x);
    for (int k = 0; k < nk; k++) {
      const int buf = k & 1;
      cp_wait_all();
      __syncthreads();
      const bool more = k + 1 < nk;
      if (more) {
        fetch((k + 1) * kTile, x);
        load_b(S, buf ^ 1, xs, a.Lp, (k + 1) * kTile);
        cp_commit();
      }
      mma_step(S, buf, msub, npair, lane, acc);
      if (more) store_a(S, buf ^ 1, grow, gword, x);
    }
  }

  const int g = lane >> 2, t = lane & 3;
  const int ms = (t & 1) ? -1 : 1, ns = (t & 2) ? -1 : 1;
  if ((ms < 0 && mu == 0) || (ns < 0 && nu == 0)) return;
  const int m = ms * mu, n = ns * nu;
  if (plane_skipped(a.n_mode, a.N, n)) return;  // caller-zeroed blocks stay untouched
  const bool one_neg = ms * ns < 0;
  const double sgn_mn = ((mu + nu) & 1) ? -1.0 : 1.0;
  const double* sc = a.xscale + gp * kRowsB;
  const long long blk = a.base[a.plane0 + n];
#pragma unroll
  for (int nt = 0; nt < 2; nt++) {
    const int b = npair * 2 + nt, sig = grp * kGrp + b;
    if (sig >= a.nsig) continue;
    const double sre = sc[b * kCol + 2 * t], sim = sc[b * kCol + 2 * t + 1];
    double2* F = a.flmn[sig];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int lr = l0 + msub * 16 + g + 8 * h;
      if (lr >= L || mu > lr) continue;
      if (a.compact && lr < nu) continue;  // not stored
      double2 v = make_double2(0.0, 0.0);
      if (lr >= lmin) {
        v = make_double2(combine(acc, nt, 2 * h) * sre, combine(acc, nt, 2 * h + 1) * sim);
        const double s = (one_neg && (lr & 1)) ? -sgn_mn : sgn_mn;
        v = ipow(make_double2(v.x * s, v.y * s), m - n + 4 * L);
      }
      F[blk + (long long)lr * lr + lr + m] = v;
    }
  }
}

// ---------------------------------------------------------------- slicing
// One warp per (pair mu * N + nu, signal): column scales over the reduction index, then
// the 7 slices of the 8 columns.  Inverse: X[l, c] from the coefficients;
// forward: X'[m', c] from the scratch planes.
struct SliceArgs {
  uint8_t* xs;
  double* xscale;
  const double2* const* flmn;  // inverse input, per signal
  const double2* W;            // forward input, signal b at W + b * wstride
  const long long* base;
  long long wstride;
  int L, N, L0, Lp, MT, plane0, n_mode, nsig, npairs;
  long long RS, PS;
};

template <bool FWD>
__device__ __forceinline__ void column_values(const SliceArgs& a, int sig, int mu, int nu, int k, double (&v)[kCol]) {
  const int lmin = max(max(mu, nu), a.L0);
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const int ms = (s & 1) ? -1 : 1, ns = (s & 2) ? -1 : 1;
    double2 x = make_double2(0.0, 0.0);
    const bool combo = !(ms < 0 && mu == 0) && !(ns < 0 && nu == 0);
    const int m = ms * mu, n = ns * nu;
    if (sig < a.nsig && combo && k < a.L && !plane_skipped(a.n_mode, a.N, n)) {
      const bool one_neg = ms * ns < 0;
      if (!FWD) {
        if (k >= lmin) {
          x = a.flmn[sig][a.base[a.plane0 + n] + (long long)k * k + k + m];
          double f = (2.0 * k + 1.0) * kInv8Pi2;
          if (one_neg && (k & 1)) f = -f;
          x = make_double2(x.x * f, x.y * f);
        }
      } else {
        x = a.W[(long long)sig * a.wstride + (long long)(a.plane0 + n) * a.PS + (long long)k * a.RS + (m + a.L - 1)];
        if (one_neg && (k & 1)) x = make_double2(-x.x, -x.y);
      }
    }
    v[2 * s] = x.x;
    v[2 * s + 1] = x.y;
  }
}

template <bool FWD>
__global__ void __launch_bounds__(256) slice_kernel(SliceArgs a) {
  const int lane = threadIdx.x & 31, b = threadIdx.x >> 5;  // 8 warps = 8 signals of the group
  const int pair = blockIdx.x, grp = blockIdx.y, sig = grp * kGrp + b;
  const int nu = pair % a.N, mu = pair / a.N;
  const size_t gp = (size_t)grp * a.npairs + pair;
  double mx[kCol];
#pragma unroll
  for (int c = 0; c < kCol; c++) mx[c] = 0.0;
  for (int k = lane; k < a.Lp; k += 32) {
    double v[kCol];
    column_values<FWD>(a, sig, mu, nu, k, v);
#pragma unroll
    for (int c = 0; c < kCol; c++) mx[c] = fmax(mx[c], fabs(v[c]));
  }
  double scale[kCol];
#pragma unroll
  for (int c = 0; c < kCol; c++) {
    double m = mx[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    int e = 0;
    frexp(m, &e);
    scale[c] = m > 0.0 ? ldexp(1.0, e + 1) : 1.0;  // |x / scale| < 1/2
    if (lane == 0) a.xscale[gp * kRowsB + b * kCol + c] = scale[c];
  }
  uint8_t* out = a.xs + gp * kS * kRowsB * (size_t)a.Lp;
  for (int k = lane; k < a.Lp; k += 32) {
    double v[kCol];
    column_values<FWD>(a, sig, mu, nu, k, v);
#pragma unroll
    for (int c = 0; c < kCol; c++) {
      int q[kS];
      split7(v[c] / scale[c], q);
#pragma unroll
      for (int i = 0; i < kS; i++) out[((size_t)i * kRowsB + b * kCol + c) * a.Lp + k] = (uint8_t)(q[i] & 255);
    }
  }
}

}  // namespace

// ---------------------------------------------------------------- host side
size_t mixed_scratch_bytes(const Geometry& g, int nsig) {
  const int Lp = (g.L + kTile - 1) / kTile * kTile;
  const size_t groups = (nsig + kGrp - 1) / kGrp, pairs = (size_t)g.L * g.N;
  return groups * pairs * (kS * kRowsB * (size_t)Lp + kRowsB * sizeof(double)) + 256;
}

static int mixed_args(const Geometry& g, int n_mode, int nsig, void* scratch, MixArgs* m, SliceArgs* s) {
  const int Lp = (g.L + kTile - 1) / kTile * kTile, MT = Lp / kTile;
  const size_t groups = (nsig + kGrp - 1) / kGrp, pairs = (size_t)g.L * g.N;
  if (pairs * MT > 0x7fffffffu) return fail(kUnsupported, "split-precision grid too large");
  uint8_t* xs = static_cast<uint8_t*>(scratch);
  double* xscale = reinterpret_cast<double*>(xs + ((groups * pairs * kS * kRowsB * (size_t)Lp + 255) & ~size_t(255)));
  *m = MixArgs{};
  m->xs = xs;
  m->xscale = xscale;
  m->L = g.L, m->N = g.N, m->L0 = g.L0, m->Lp = Lp, m->MT = MT, m->plane0 = g.plane0, m->n_mode = n_mode;
  m->nsig = nsig, m->RS = g.RS, m->PS = g.PS;
  *s = SliceArgs{};
  s->xs = xs;
  s->xscale = xscale;
  s->L = g.L, s->N = g.N, s->L0 = g.L0, s->Lp = Lp, s->MT = MT, s->plane0 = g.plane0, s->n_mode = n_mode;
  s->nsig = nsig, s->npairs = (int)pairs, s->RS = g.RS, s->PS = g.PS;
  return kOk;
}

int launch_mixed_inverse(const Geometry& g, int n_mode, const double2* const* flmn_dev, int nsig,
                         const long long* bases, const double* dl, double2* W, long long wstride, void* scratch,
                         cudaStream_t s) {
  if (g.real) return fail(kUnsupported, "split-precision contractions take complex signals");
  MixArgs m;
  SliceArgs sa;
  if (int rc = mixed_args(g, n_mode, nsig, scratch, &m, &sa)) return rc;
  sa.flmn = flmn_dev;
  sa.base = bases;
  const dim3 sgrid((unsigned)sa.npairs, (nsig + kGrp - 1) / kGrp);
  const dim3 grid((unsigned)(sa.npairs * sa.MT), (nsig + kGrp - 1) / kGrp);
  slice_kernel<false><<<sgrid, 256, 0, s>>>(sa);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  m.dl = dl;
  m.base = bases;
  m.W = W;
  m.wstride = wstride;
  SO3G_CUDA(cudaFuncSetAttribute(mixed_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MixSmem)));
  mixed_inverse_kernel<<<grid, kThreads, sizeof(MixSmem), s>>>(m);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

int launch_mixed_forward(const Geometry& g, int n_mode, const double2* W, long long wstride, int nsig,
                         const long long* bases, const double* dl, double2* const* flmn_dev, int storage_compact,
                         void* scratch, cudaStream_t s) {
  if (g.real) return fail(kUnsupported, "split-precision contractions take complex signals");
  MixArgs m;
  SliceArgs sa;
  if (int rc = mixed_args(g, n_mode, nsig, scratch, &m, &sa)) return rc;
  sa.W = W;
  sa.wstride = wstride;
  sa.base = bases;
  const dim3 sgrid((unsigned)sa.npairs, (nsig + kGrp - 1) / kGrp);
  const dim3 grid((unsigned)(sa.npairs * sa.MT), (nsig + kGrp - 1) / kGrp);
  slice_kernel<true><<<sgrid, 256, 0, s>>>(sa);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  m.dl = dl;
  m.base = bases;
  m.flmn = flmn_dev;
  m.compact = storage_compact;
  SO3G_CUDA(cudaFuncSetAttribute(mixed_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MixSmem)));
  mixed_forward_kernel<<<grid, kThreads, sizeof(MixSmem), s>>>(m);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace so3g
