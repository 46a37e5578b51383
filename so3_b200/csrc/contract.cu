// FP64 Wigner contractions: the O(N L^3) core of the transform.
//
// Inverse (replaces SSHT's per-spin Fmm accumulation called at the
// reference's src/c/so3_core.c:204 and the in-tree src/c/so3_core.c:1081-1165):
//   F[n][m'][m] = i^{n-m} sum_{l >= max(L0,|n|,|m|,m')} (2l+1)/(8 pi^2)
//                 Delta^l_{m'm} Delta^l_{m'n} f_lmn ,   m' >= 0.
// Forward (replaces SSHT's forward Delta sum, src/c/so3_core.c:408-428 and
// in-tree :1589-1617):
//   f_lmn = i^{m-n} sum_{m'=0}^{l} Delta^l_{m'm} Delta^l_{m'n} G[n][m'][m].
//
// Both are three-operand contractions (every pair of the free indices shares
// an operand), so no plain GEMM exists for one signal; the kernels are built
// for the FP64 pipe:
//  * Negative m, n use Delta^l_{m',-k} = (-1)^{l+m'} Delta^l_{m'k}: one product
//    w = Delta_{m'|m|} Delta_{m'|n|} feeds the four sign combinations (+m,+n),
//    (-m,+n), (+m,-n), (-m,-n) (9 FP64 instructions per 4 complex MACs).  The
//    (-1)^{l+m'} of combinations with one negative index is split between the
//    operand that carries l and the one that carries m'.
//  * CTA tile: 32 output rows (m' for the inverse, l for the forward) x 32 |m|
//    x 2 |n|.  The reduction index (l, resp. m') is walked in chunks of 4,
//    staged in shared memory with cp.async, double buffered.
//  * Lanes form an 8 (rows) x 4 (|m|) grid, warps step |m| by 4: a warp reads
//    32 distinct Delta_{m'|m|} (2 wavefronts with the 36-double row pitch),
//    8 distinct Delta_{m'|n|} pairs and 4 distinct coefficient quadruples
//    (1 wavefront each), for 72 FP64 instructions per lane.
//  * Grid order |n|-pair fastest, then rows, then |m|: CTAs resident at the
//    same time share one Delta tile column and one coefficient slice in L2.
#include <cstdlib>

#include "so3gpu_internal.h"

namespace so3g {

namespace {
constexpr int kThreads = 256;
constexpr int kRows = 32;    // output rows per CTA (m' or l)
constexpr int kCols = 32;    // |m| per CTA
constexpr int kNG = 2;       // |n| per CTA
constexpr int kChunk = 4;    // reduction steps per shared-memory stage
constexpr int kPitch = 36;   // doubles per staged Delta row (32 + 4: conflict-free)
constexpr int kPer = kRows / 8;  // rows per lane
constexpr double kInv8Pi2 = 0.012665147955292221430803304553147533;  // 1/(8 pi^2)

struct Slab {
  double B[kChunk][kRows][kPitch];  // Delta^l_{row, |m|}
  double A[kChunk][kRows][kNG];     // Delta^l_{row, |n|}  (times (2l+1)/(8 pi^2) in the inverse)
  double2 H[kChunk][kCols][kNG][4]; // coefficients / spectra, sign-folded
};
constexpr size_t kSmem = 2 * sizeof(Slab);

__device__ __forceinline__ double2 ipow_mul(double2 v, int k) {  // v * i^k
  switch (k & 3) {
    case 0: return v;
    case 1: return make_double2(-v.y, v.x);
    case 2: return make_double2(-v.x, -v.y);
    default: return make_double2(v.y, -v.x);
  }
}
__device__ __forceinline__ double2 sc(double2 v, double s) { return make_double2(v.x * s, v.y * s); }

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// 4 sign combinations s: bit0 -> m negative, bit1 -> n negative.  scale
// multiplies every product (the (2l+1)/(8 pi^2) of the inverse, 1 in the
// forward); oddneg flips the sign of the combinations with one negative index
// ((-1)^l in the inverse, (-1)^{m'} in the forward); symmu != 0 rebuilds the
// -m coefficient of a real signal with N == 1 from the +m one.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0));
}

template <int NSIGN, bool SYM>
__device__ __forceinline__ void mac_chunk(const Slab& S, int lc, int warp, int lm, int lu, double scale, bool oddneg,
                                          int mu, double2 (&acc)[kPer][kNG][4]) {
  const int col = 4 * warp + lu;
  double2 h[kNG][4];
#pragma unroll
  for (int j = 0; j < kNG; j++) {
#pragma unroll
    for (int s = 0; s < NSIGN; s++) h[j][s] = S.H[lc][col][j][s];
    if (SYM) h[j][1] = (mu & 1) ? make_double2(-h[j][0].x, h[j][0].y) : make_double2(h[j][0].x, -h[j][0].y);
  }
  const double sneg = oddneg ? -scale : scale;
#pragma unroll
  for (int i = 0; i < kPer; i++) {
    const int row = lm + 8 * i;
    const double b = S.B[lc][row][col];
    const double2 a = *reinterpret_cast<const double2*>(&S.A[lc][row][0]);
    const double p0 = b * a.x, p1 = b * a.y;
    const double w0 = p0 * scale, w1 = p1 * scale, v0 = p0 * sneg, v1 = p1 * sneg;
#pragma unroll
    for (int s = 0; s < NSIGN; s++) {
      const bool one_neg = (s == 1) || (s == 2);
      const double x0 = one_neg ? v0 : w0, x1 = one_neg ? v1 : w1;
      acc[i][0][s].x = fma(x0, h[0][s].x, acc[i][0][s].x);
      acc[i][0][s].y = fma(x0, h[0][s].y, acc[i][0][s].y);
      acc[i][1][s].x = fma(x1, h[1][s].x, acc[i][1][s].x);
      acc[i][1][s].y = fma(x1, h[1][s].y, acc[i][1][s].y);
    }
  }
}
}  // namespace

// FP64 contraction engine for complex signals: the FP64 tensor cores
// (mma.sync f64; measured 1.3-1.6x faster at L=512, N=64), unless the
// environment sets SO3GPU_FP64_MMA=0 (the FP64 FMA kernels, which real
// signals always use).
static bool fp64_tensor_cores() {
  const char* e = getenv("SO3GPU_FP64_MMA");
  return !(e && e[0] == '0');
}

struct InvArgs {
  const double2* flmn;
  const long long* base;  // per plane
  const double* dl;
  double2* W;
  int L, N, L0, plane0, n_mode, real, sym_n0;
  int nu_lo, nu_hi;  // |n| range [nu_lo, nu_hi) of this launch
  long long CS, QS;  // column-major scratch strides
  double wconst;     // > 0: this weight for every l instead of (2l+1)/(8 pi^2) (adjoint forward)
};

// ------------------------------------------------------------------ inverse
template <int NSIGN>
__global__ void __launch_bounds__(kThreads, 1) inverse_contract_kernel(InvArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Slab* st = reinterpret_cast<Slab*>(smraw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, lm = lane & 7, lu = lane >> 3;
  const int nu0 = a.nu_lo + blockIdx.x * kNG, mp0 = blockIdx.y * kRows, mu0 = blockIdx.z * kCols;
  const int L = a.L;
  bool act[kNG];
#pragma unroll
  for (int j = 0; j < kNG; j++) act[j] = (nu0 + j < a.nu_hi) && !plane_skipped(a.n_mode, a.N, nu0 + j);

  double2 acc[kPer][kNG][4];
#pragma unroll
  for (int i = 0; i < kPer; i++)
#pragma unroll
    for (int j = 0; j < kNG; j++)
#pragma unroll
      for (int s = 0; s < 4; s++) acc[i][j][s] = make_double2(0.0, 0.0);

  const int lstart = max(max(a.L0, nu0), max(mp0, mu0));
  const int mu_own = mu0 + 4 * warp + lu;
  long long bsel[kNG][2];  // flmn block bases of +|n| and -|n|
#pragma unroll
  for (int j = 0; j < kNG; j++) {
    const int nu = min(nu0 + j, a.N - 1);
    bsel[j][0] = a.base[a.plane0 + nu];
    bsel[j][1] = NSIGN == 4 ? a.base[a.plane0 - nu] : 0;
  }
  const int nchunk = lstart < L ? (L - lstart + kChunk - 1) / kChunk : 0;

  auto stage = [&](int c, Slab& S) {
    const int lbase = lstart + c * kChunk;
    for (int idx = tid; idx < kChunk * kRows * kCols; idx += kThreads) {
      const int lc = idx / (kRows * kCols), rem = idx - lc * kRows * kCols, r = rem / kCols, col = rem - r * kCols;
      const int l = lbase + lc;
      const bool ok = l < L && mp0 + r <= l && mu0 + col <= l;
      const double* src = ok ? a.dl + dl_plane_offset(l) + (long long)(mp0 + r) * (l + 1) + mu0 + col : a.dl;
      cp_async8(&S.B[lc][r][col], src, ok);
    }
    for (int idx = tid; idx < kChunk * kRows * kNG; idx += kThreads) {
      const int lc = idx / (kRows * kNG), rem = idx - lc * kRows * kNG, r = rem / kNG, j = rem - r * kNG;
      const int l = lbase + lc, nu = nu0 + j;
      const bool ok = l < L && act[j] && mp0 + r <= l && nu <= l;
      const double* src = ok ? a.dl + dl_plane_offset(l) + (long long)(mp0 + r) * (l + 1) + nu : a.dl;
      cp_async8(&S.A[lc][r][j], src, ok);
    }
    for (int idx = tid; idx < kChunk * kCols * kNG * NSIGN; idx += kThreads) {
      const int lc = idx / (kCols * kNG * NSIGN), rem = idx - lc * kCols * kNG * NSIGN;
      const int col = rem / (kNG * NSIGN), rem2 = rem - col * kNG * NSIGN, j = rem2 / NSIGN, sg = rem2 - j * NSIGN;
      const int l = lbase + lc, nu = nu0 + j, mu = mu0 + col;
      const bool ok = l < L && act[j] && mu <= l && nu <= l;
      const int m = (sg & 1) ? -mu : mu;
      const double2* src = ok ? a.flmn + bsel[j][sg >> 1] + (long long)l * l + l + m : a.flmn;
      cp_async16(&S.H[lc][col][j][sg], src, ok);
    }
  };

  if (nchunk > 0) {
    stage(0, st[0]);
    cp_commit();
    for (int c = 0; c < nchunk; c++) {
      if (c + 1 < nchunk) {
        stage(c + 1, st[(c + 1) & 1]);
        cp_commit();
        cp_wait<1>();
      } else {
        cp_wait<0>();
      }
      __syncthreads();
      const Slab& S = st[c & 1];
      const int lbase = lstart + c * kChunk;
#pragma unroll
      for (int lc = 0; lc < kChunk; lc++) {
        const int l = lbase + lc;
        const double cl = a.wconst > 0.0 ? a.wconst : (2.0 * l + 1.0) * kInv8Pi2;
        if (a.sym_n0)
          mac_chunk<NSIGN, true>(S, lc, warp, lm, lu, cl, l & 1, mu_own, acc);
        else
          mac_chunk<NSIGN, false>(S, lc, warp, lm, lu, cl, l & 1, mu_own, acc);
      }
      __syncthreads();
    }
  }

  const int mu = mu0 + 4 * warp + lu;
  if (mu >= L) return;
#pragma unroll
  for (int i = 0; i < kPer; i++) {
    const int mp = mp0 + lm + 8 * i;
    if (mp >= L) continue;
    const double odd_mp = (mp & 1) ? -1.0 : 1.0;
#pragma unroll
    for (int j = 0; j < kNG; j++) {
      const int nu = nu0 + j;
      if (nu >= a.nu_hi) continue;
#pragma unroll
      for (int s = 0; s < NSIGN; s++) {
        const int ms = (s & 1) ? -1 : 1, ns = (s & 2) ? -1 : 1;
        if (ms < 0 && mu == 0) continue;
        if (ns < 0 && nu == 0) continue;
        const int m = ms * mu, n = ns * nu;
        double2 v = acc[i][j][s];
        if (ms * ns < 0) v = sc(v, odd_mp);
        v = ipow_mul(v, n - m + 4 * L);
        a.W[(long long)(a.plane0 + n) * a.QS + (long long)(m + L - 1) * a.CS + mp] = v;
      }
    }
  }
}

// ------------------------------------------------------------------ inverse, FP64 tensor cores
// The same contraction as inverse_contract_kernel on the FP64 tensor cores
// (mma.sync.aligned.m8n8k4 f64): for a pair (mu, nu) = (|m|, |n|) it is the
// product Y[m', c] = sum_l W[m', l] X[l, c] with W[m', l] = Delta^l_{m' mu}
// Delta^l_{m' nu} and one column c = 2 s + part per sign combination s
// (bit 0: m = -mu, bit 1: n = -nu) and real / imaginary part; X carries
// (2l+1)/(8 pi^2), and (-1)^l on combinations with one negative index (the
// output carries the (-1)^{m'} of those).  One MMA: 8 rows m' x 8 columns x
// 4 reduction steps l (256 multiply-adds).  CTA tile: 32 m' x 16 mu x 2 nu;
// warp w: rows 8 (w & 3) .. +7, mu block 8 (w >> 2) .. +7, both nu: 16 MMAs
// (32 accumulators per lane) per 4-step chunk.  Delta tiles staged with
// cp.async (double buffered); X built from the coefficients with the weights
// applied while staging (its loads are issued one chunk ahead).
namespace {
constexpr int kDT = 256;       // threads
constexpr int kDR = 32;        // m' per CTA
constexpr int kDM = 16;        // mu per CTA
constexpr int kDN = 2;         // nu per CTA
constexpr int kDK = 4;         // l per chunk (MMA K)
constexpr int kBP = 17;        // Bm pitch (doubles): lanes (g, q) hit distinct bank pairs
constexpr int kAP = 3;         // An pitch
// X block of one (mu, nu): 8 columns c x 4 steps l, element c * 4 + l.  Block
// pitches 36 (nu) and 81 (mu) doubles put the staging stores of a warp on 16
// distinct bank pairs (inverse lanes: sign, nu, 4 mu; forward lanes: l, sign,
// nu); a fragment read is 32 consecutive doubles either way.
constexpr int kXJ = 36, kXM = 81;
struct DSlab {
  double Bm[kDR][kDK][kBP];           // Delta^l_{m', mu0 + j}
  double An[kDR][kDK][kAP];           // Delta^l_{m', nu0 + j}
  double X[kDM * kXM];                // [mu][nu][c][l], weighted and sign-folded
};
__device__ __forceinline__ double& xat(DSlab& S, int jm, int j, int c, int l) {
  return S.X[jm * kXM + j * kXJ + c * kDK + l];
}

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}
}  // namespace

template <int NSIGN>
__global__ void __launch_bounds__(kDT, 2) inverse_contract_dmma_kernel(InvArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  DSlab* st = reinterpret_cast<DSlab*>(smraw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, q = lane & 3;
  const int nu0 = a.nu_lo + blockIdx.x * kDN, mp0 = blockIdx.y * kDR, mu0 = blockIdx.z * kDM;
  const int L = a.L;
  bool act[kDN];
#pragma unroll
  for (int j = 0; j < kDN; j++) act[j] = (nu0 + j < a.nu_hi) && !plane_skipped(a.n_mode, a.N, nu0 + j);
  const int mb = warp & 3, jm0 = 8 * (warp >> 2);  // rows 8 mb .., mu block jm0 ..
  double acc[8][kDN][2];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < kDN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

  // reduction range, aligned to the chunk: l in [l_lo, L), l_lo = 4 floor(max(...)/4)
  const int lstart = max(max(a.L0, nu0), max(mp0, mu0));
  const int l_lo = lstart & ~(kDK - 1);
  const int nchunk = l_lo < L ? (L - l_lo + kDK - 1) / kDK : 0;
  long long bsel[kDN][2];
#pragma unroll
  for (int j = 0; j < kDN; j++) {
    const int nu = min(nu0 + j, a.N - 1);
    bsel[j][0] = a.base[a.plane0 + nu];
    bsel[j][1] = NSIGN == 4 ? a.base[a.plane0 - nu] : 0;
  }

  auto stage_delta = [&](int c, DSlab& S) {
    const int lb = l_lo + c * kDK;
    for (int idx = tid; idx < kDR * kDK * kDM; idx += kDT) {  // mu fastest: a row segment of a plane
      const int j = idx % kDM, rest = idx / kDM, lc = rest % kDK, r = rest / kDK;
      const int l = lb + lc, mp = mp0 + r, mu = mu0 + j;
      const bool ok = l < L && l >= lstart && mp <= l && mu <= l;
      const double* src = ok ? a.dl + dl_plane_offset(l) + (long long)mp * (l + 1) + mu : a.dl;
      cp_async8(&S.Bm[r][lc][j], src, ok);
    }
    for (int idx = tid; idx < kDR * kDK * kDN; idx += kDT) {
      const int j = idx % kDN, rest = idx / kDN, lc = rest % kDK, r = rest / kDK;
      const int l = lb + lc, mp = mp0 + r, nu = nu0 + j;
      const bool ok = l < L && l >= lstart && act[j] && mp <= l && nu <= l;
      const double* src = ok ? a.dl + dl_plane_offset(l) + (long long)mp * (l + 1) + nu : a.dl;
      cp_async8(&S.An[r][lc][j], src, ok);
    }
  };
  // coefficient loads of a chunk: 4 l x 16 mu x 2 nu x NSIGN complex values, 2 per thread
  constexpr int kXN = kDK * kDM * kDN * 4;  // 512 (NSIGN 4) slots, 2 per thread
  double2 xv[2];
  auto load_x = [&](int c) {
    const int lb = l_lo + c * kDK;
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int idx = tid + u * kDT;  // sg fastest, then nu, mu, l
      const int sg = idx & 3, j = (idx >> 2) & 1, jm = (idx >> 3) & 15, lc = idx >> 7;
      const int l = lb + lc, mu = mu0 + jm, nu = nu0 + j;
      const bool ok = sg < NSIGN && l < L && l >= lstart && act[j] && mu <= l && nu <= l &&
                      !((sg & 1) && mu == 0) && !((sg & 2) && nu == 0);
      const int m = (sg & 1) ? -mu : mu;
      xv[u] = ok ? __ldg(a.flmn + bsel[j][sg >> 1] + (long long)l * l + l + m) : make_double2(0.0, 0.0);
    }
  };
  auto store_x = [&](int c, DSlab& S) {
    const int lb = l_lo + c * kDK;
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int idx = tid + u * kDT;
      const int sg = idx & 3, j = (idx >> 2) & 1, jm = (idx >> 3) & 15, lc = idx >> 7;
      const int l = lb + lc;
      double w = a.wconst > 0.0 ? a.wconst : (2.0 * l + 1.0) * kInv8Pi2;
      if ((sg == 1 || sg == 2) && (l & 1)) w = -w;  // one negative index: (-1)^l here
      xat(S, jm, j, 2 * sg, lc) = xv[u].x * w;
      xat(S, jm, j, 2 * sg + 1, lc) = xv[u].y * w;
    }
  };
  static_assert(kXN == 2 * kDT, "two coefficient slots per thread");

  if (nchunk > 0) {
    stage_delta(0, st[0]);
    cp_commit();
    load_x(0);
    for (int c = 0; c < nchunk; c++) {
      DSlab& S = st[c & 1];
      store_x(c, S);
      if (c + 1 < nchunk) {
        stage_delta(c + 1, st[(c + 1) & 1]);
        cp_commit();
        load_x(c + 1);
        cp_wait<1>();
      } else {
        cp_wait<0>();
      }
      __syncthreads();
      // fragments: A (W) row g = m' 8 mb + g, column q = l; B (X) row q = l, column g = c
      const double an0 = S.An[8 * mb + g][q][0], an1 = S.An[8 * mb + g][q][1];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const double bm = S.Bm[8 * mb + g][q][jm0 + i];
        dmma(acc[i][0], bm * an0, xat(S, jm0 + i, 0, g, q));
        dmma(acc[i][1], bm * an1, xat(S, jm0 + i, 1, g, q));
      }
      __syncthreads();
    }
  }

  // accumulator (row g, columns 2q, 2q+1) = sign combination q, real / imaginary part
  const int mp = mp0 + 8 * mb + g;
  const int s = q;
  if (mp >= L || s >= NSIGN) return;
  const int ms = (s & 1) ? -1 : 1, ns = (s & 2) ? -1 : 1;
  const double odd_mp = (mp & 1) ? -1.0 : 1.0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int mu = mu0 + jm0 + i;
    if (mu >= L || (ms < 0 && mu == 0)) continue;
#pragma unroll
    for (int j = 0; j < kDN; j++) {
      const int nu = nu0 + j;
      if (nu >= a.nu_hi || (ns < 0 && nu == 0)) continue;
      const int m = ms * mu, n = ns * nu;
      double2 v = make_double2(acc[i][j][0], acc[i][j][1]);
      if (ms * ns < 0) v = sc(v, odd_mp);
      v = ipow_mul(v, n - m + 4 * L);
      a.W[(long long)(a.plane0 + n) * a.QS + (long long)(m + L - 1) * a.CS + mp] = v;
    }
  }
}

int launch_inverse_contract(const Geometry& g, int n_mode, const double2* flmn, const long long* bases,
                            const double* dl, double2* W, int sym_n0, cudaStream_t s, int nu_lo, int nu_hi,
                            double wconst) {
  if (nu_hi < 0 || nu_hi > g.N) nu_hi = g.N;
  if (nu_lo >= nu_hi) return kOk;
  InvArgs a{flmn, bases, dl, W + g.QOFF, g.L, g.N, g.L0, g.plane0, n_mode, g.real, sym_n0, nu_lo, nu_hi, g.CS, g.QS,
            wconst};
  if (!g.real && !sym_n0 && fp64_tensor_cores()) {
    dim3 gd((nu_hi - nu_lo + kDN - 1) / kDN, (g.L + kDR - 1) / kDR, (g.L + kDM - 1) / kDM);
    const int smem = (int)(2 * sizeof(DSlab));
    SO3G_CUDA(cudaFuncSetAttribute(inverse_contract_dmma_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    inverse_contract_dmma_kernel<4><<<gd, kDT, smem, s>>>(a);
    SO3G_LAUNCHED();
    SO3G_CUDA(cudaGetLastError());
    return kOk;
  }
  dim3 grid((nu_hi - nu_lo + kNG - 1) / kNG, (g.L + kRows - 1) / kRows, (g.L + kCols - 1) / kCols);
  if (g.real) {
    SO3G_CUDA(cudaFuncSetAttribute(inverse_contract_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    inverse_contract_kernel<2><<<grid, kThreads, kSmem, s>>>(a);
  } else {
    SO3G_CUDA(cudaFuncSetAttribute(inverse_contract_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    inverse_contract_kernel<4><<<grid, kThreads, kSmem, s>>>(a);
  }
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

// ------------------------------------------------------------------ forward
struct FwdArgs {
  const double2* W;
  const long long* base;
  const double* dl;
  double2* flmn;
  int L, N, L0, plane0, n_mode, real, compact;
  int nu_lo, nu_hi;  // |n| range [nu_lo, nu_hi) of this launch
  long long CS, QS;  // column-major scratch strides
  double lw;         // > 0: outputs times lw (2l+1) (adjoint inverse)
};

template <int NSIGN>
__global__ void __launch_bounds__(kThreads, 1) forward_contract_kernel(FwdArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Slab* st = reinterpret_cast<Slab*>(smraw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, lm = lane & 7, lu = lane >> 3;
  const int nu0 = a.nu_lo + blockIdx.x * kNG, l0 = blockIdx.y * kRows, mu0 = blockIdx.z * kCols;
  const int L = a.L;
  bool act[kNG];
#pragma unroll
  for (int j = 0; j < kNG; j++) act[j] = (nu0 + j < a.nu_hi) && !plane_skipped(a.n_mode, a.N, nu0 + j);
  if (!act[0] && !act[1]) return;  // caller-zeroed blocks stay untouched

  double2 acc[kPer][kNG][4];
#pragma unroll
  for (int i = 0; i < kPer; i++)
#pragma unroll
    for (int j = 0; j < kNG; j++)
#pragma unroll
      for (int s = 0; s < 4; s++) acc[i][j][s] = make_double2(0.0, 0.0);

  const int ltop = min(L - 1, l0 + kRows - 1);
  const bool any = ltop >= max(max(a.L0, nu0), mu0);
  const int nchunk = any ? (ltop + 1 + kChunk - 1) / kChunk : 0;

  auto stage = [&](int c, Slab& S) {
    const int mbase = c * kChunk;
    for (int idx = tid; idx < kChunk * kRows * kCols; idx += kThreads) {
      const int mc = idx / (kRows * kCols), rem = idx - mc * kRows * kCols, r = rem / kCols, col = rem - r * kCols;
      const int mp = mbase + mc, l = l0 + r;
      const bool ok = l < L && mp <= l && mu0 + col <= l;
      const double* src = ok ? a.dl + dl_plane_offset(l) + (long long)mp * (l + 1) + mu0 + col : a.dl;
      cp_async8(&S.B[mc][r][col], src, ok);
    }
    for (int idx = tid; idx < kChunk * kRows * kNG; idx += kThreads) {
      const int mc = idx / (kRows * kNG), rem = idx - mc * kRows * kNG, r = rem / kNG, j = rem - r * kNG;
      const int mp = mbase + mc, l = l0 + r, nu = nu0 + j;
      const bool ok = l < L && act[j] && mp <= l && nu <= l;
      const double* src = ok ? a.dl + dl_plane_offset(l) + (long long)mp * (l + 1) + nu : a.dl;
      cp_async8(&S.A[mc][r][j], src, ok);
    }
    for (int idx = tid; idx < kChunk * kCols * kNG * NSIGN; idx += kThreads) {
      // m' fastest: consecutive threads read consecutive entries of a column
      const int mc = idx % kChunk, rem = idx / kChunk;
      const int col = rem / (kNG * NSIGN), rem2 = rem - col * kNG * NSIGN, j = rem2 / NSIGN, sg = rem2 - j * NSIGN;
      const int mp = mbase + mc, nu = nu0 + j, mu = mu0 + col;
      const bool ok = mp < L && act[j] && mu < L;
      const int n = (sg & 2) ? -nu : nu, m = (sg & 1) ? -mu : mu;
      const double2* src =
          ok ? a.W + (long long)(a.plane0 + n) * a.QS + (long long)(L - 1 + m) * a.CS + mp : a.W;
      cp_async16(&S.H[mc][col][j][sg], src, ok);
    }
  };

  if (nchunk > 0) {
    stage(0, st[0]);
    cp_commit();
    for (int c = 0; c < nchunk; c++) {
      if (c + 1 < nchunk) {
        stage(c + 1, st[(c + 1) & 1]);
        cp_commit();
        cp_wait<1>();
      } else {
        cp_wait<0>();
      }
      __syncthreads();
      const Slab& S = st[c & 1];
#pragma unroll
      for (int mc = 0; mc < kChunk; mc++) mac_chunk<NSIGN, false>(S, mc, warp, lm, lu, 1.0, (c * kChunk + mc) & 1, 0, acc);
      __syncthreads();
    }
  }

  const int mu = mu0 + 4 * warp + lu;
  if (mu >= L) return;
#pragma unroll
  for (int i = 0; i < kPer; i++) {
    const int l = l0 + lm + 8 * i;
    if (l >= L || mu > l) continue;
    const double odd_l = (l & 1) ? -1.0 : 1.0;
#pragma unroll
    for (int j = 0; j < kNG; j++) {
      const int nu = nu0 + j;
      if (!act[j]) continue;
      if (a.compact && l < nu) continue;  // not stored
#pragma unroll
      for (int s = 0; s < NSIGN; s++) {
        const int ms = (s & 1) ? -1 : 1, ns = (s & 2) ? -1 : 1;
        if (ms < 0 && mu == 0) continue;
        if (ns < 0 && nu == 0) continue;
        const int m = ms * mu, n = ns * nu;
        double2 v = make_double2(0.0, 0.0);
        if (l >= max(a.L0, nu)) {
          v = acc[i][j][s];
          if (ms * ns < 0) v = sc(v, odd_l);
          v = ipow_mul(v, m - n + 4 * L);
          if (a.lw > 0.0) v = sc(v, a.lw * (2.0 * l + 1.0));
        }
        a.flmn[a.base[a.plane0 + n] + (long long)l * l + l + m] = v;
      }
    }
  }
}

// ------------------------------------------------------------------ forward, FP64 tensor cores
// The forward contraction on the FP64 tensor cores: for a pair (mu, nu),
// Y[l, c] = sum_{m'} W[l, m'] X[m', c] with W[l, m'] = Delta^l_{m' mu}
// Delta^l_{m' nu} (m' <= l) and X the spectra G(n, m, m') of the column-major
// scratch, (-1)^{m'} folded in for combinations with one negative index (the
// output carries their (-1)^l).  CTA tile 32 l x 16 mu x 2 nu, warps and
// staging as in inverse_contract_dmma_kernel.
template <int NSIGN>
__global__ void __launch_bounds__(kDT, 2) forward_contract_dmma_kernel(FwdArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  DSlab* st = reinterpret_cast<DSlab*>(smraw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, q = lane & 3;
  const int nu0 = a.nu_lo + blockIdx.x * kDN, l0 = blockIdx.y * kDR, mu0 = blockIdx.z * kDM;
  const int L = a.L;
  bool act[kDN];
#pragma unroll
  for (int j = 0; j < kDN; j++) act[j] = (nu0 + j < a.nu_hi) && !plane_skipped(a.n_mode, a.N, nu0 + j);
  if (!act[0] && !act[1]) return;  // caller-zeroed blocks stay untouched
  const int mb = warp & 3, jm0 = 8 * (warp >> 2);
  double acc[8][kDN][2];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < kDN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int ltop = min(L - 1, l0 + kDR - 1);
  const bool any = ltop >= max(max(a.L0, nu0), mu0);
  const int nchunk = any ? (ltop + 1 + kDK - 1) / kDK : 0;  // m' = 0 .. ltop

  auto stage_delta = [&](int c, DSlab& S) {
    const int mb0 = c * kDK;
    for (int idx = tid; idx < kDR * kDK * kDM; idx += kDT) {
      const int j = idx % kDM, rest = idx / kDM, mc = rest % kDK, r = rest / kDK;
      const int mp = mb0 + mc, l = l0 + r, mu = mu0 + j;
      const bool ok = l < L && mp <= l && mu <= l;
      const double* src = ok ? a.dl + dl_plane_offset(l) + (long long)mp * (l + 1) + mu : a.dl;
      cp_async8(&S.Bm[r][mc][j], src, ok);
    }
    for (int idx = tid; idx < kDR * kDK * kDN; idx += kDT) {
      const int j = idx % kDN, rest = idx / kDN, mc = rest % kDK, r = rest / kDK;
      const int mp = mb0 + mc, l = l0 + r, nu = nu0 + j;
      const bool ok = l < L && act[j] && mp <= l && nu <= l;
      const double* src = ok ? a.dl + dl_plane_offset(l) + (long long)mp * (l + 1) + nu : a.dl;
      cp_async8(&S.An[r][mc][j], src, ok);
    }
  };
  double2 xv[2];
  auto load_x = [&](int c) {
    const int mb0 = c * kDK;
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int idx = tid + u * kDT;  // m' fastest (contiguous in a column), then sign, nu, mu
      const int mc = idx & 3, sg = (idx >> 2) & 3, j = (idx >> 4) & 1, jm = idx >> 5;
      const int mp = mb0 + mc, mu = mu0 + jm, nu = nu0 + j;
      const bool ok = sg < NSIGN && mp < L && act[j] && mu < L && !((sg & 1) && mu == 0) && !((sg & 2) && nu == 0);
      const int n = (sg & 2) ? -nu : nu, m = (sg & 1) ? -mu : mu;
      xv[u] = ok ? __ldg(a.W + (long long)(a.plane0 + n) * a.QS + (long long)(L - 1 + m) * a.CS + mp)
                 : make_double2(0.0, 0.0);
    }
  };
  auto store_x = [&](int c, DSlab& S) {
    const int mb0 = c * kDK;
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int idx = tid + u * kDT;
      const int mc = idx & 3, sg = (idx >> 2) & 3, j = (idx >> 4) & 1, jm = idx >> 5;
      const double w = ((sg == 1 || sg == 2) && ((mb0 + mc) & 1)) ? -1.0 : 1.0;  // (-1)^{m'}
      xat(S, jm, j, 2 * sg, mc) = xv[u].x * w;
      xat(S, jm, j, 2 * sg + 1, mc) = xv[u].y * w;
    }
  };

  if (nchunk > 0) {
    stage_delta(0, st[0]);
    cp_commit();
    load_x(0);
    for (int c = 0; c < nchunk; c++) {
      DSlab& S = st[c & 1];
      store_x(c, S);
      if (c + 1 < nchunk) {
        stage_delta(c + 1, st[(c + 1) & 1]);
        cp_commit();
        load_x(c + 1);
        cp_wait<1>();
      } else {
        cp_wait<0>();
      }
      __syncthreads();
      const double an0 = S.An[8 * mb + g][q][0], an1 = S.An[8 * mb + g][q][1];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const double bm = S.Bm[8 * mb + g][q][jm0 + i];
        dmma(acc[i][0], bm * an0, xat(S, jm0 + i, 0, g, q));
        dmma(acc[i][1], bm * an1, xat(S, jm0 + i, 1, g, q));
      }
      __syncthreads();
    }
  }

  const int l = l0 + 8 * mb + g;
  const int s = q;
  if (l >= L || s >= NSIGN) return;
  const int ms = (s & 1) ? -1 : 1, ns = (s & 2) ? -1 : 1;
  const double odd_l = (l & 1) ? -1.0 : 1.0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int mu = mu0 + jm0 + i;
    if (mu >= L || mu > l || (ms < 0 && mu == 0)) continue;
#pragma unroll
    for (int j = 0; j < kDN; j++) {
      const int nu = nu0 + j;
      if (!act[j] || (ns < 0 && nu == 0)) continue;
      if (a.compact && l < nu) continue;  // not stored
      const int m = ms * mu, n = ns * nu;
      double2 v = make_double2(0.0, 0.0);
      if (l >= max(a.L0, nu)) {
        v = make_double2(acc[i][j][0], acc[i][j][1]);
        if (ms * ns < 0) v = sc(v, odd_l);
        v = ipow_mul(v, m - n + 4 * L);
        if (a.lw > 0.0) v = sc(v, a.lw * (2.0 * l + 1.0));
      }
      a.flmn[a.base[a.plane0 + n] + (long long)l * l + l + m] = v;
    }
  }
}

int launch_forward_contract(const Geometry& g, int n_mode, const double2* W, const long long* bases,
                            const double* dl, double2* flmn, int storage_compact, cudaStream_t s, int nu_lo,
                            int nu_hi, double lw) {
  if (nu_hi < 0 || nu_hi > g.N) nu_hi = g.N;
  if (nu_lo >= nu_hi) return kOk;
  FwdArgs a{W + g.QOFF, bases, dl, flmn, g.L, g.N, g.L0, g.plane0, n_mode, g.real, storage_compact, nu_lo, nu_hi,
            g.CS, g.QS, lw};
  if (!g.real && fp64_tensor_cores()) {
    dim3 gd((nu_hi - nu_lo + kDN - 1) / kDN, (g.L + kDR - 1) / kDR, (g.L + kDM - 1) / kDM);
    const int smem = (int)(2 * sizeof(DSlab));
    SO3G_CUDA(cudaFuncSetAttribute(forward_contract_dmma_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    forward_contract_dmma_kernel<4><<<gd, kDT, smem, s>>>(a);
    SO3G_LAUNCHED();
    SO3G_CUDA(cudaGetLastError());
    return kOk;
  }
  dim3 grid((nu_hi - nu_lo + kNG - 1) / kNG, (g.L + kRows - 1) / kRows, (g.L + kCols - 1) / kCols);
  if (g.real) {
    SO3G_CUDA(cudaFuncSetAttribute(forward_contract_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    forward_contract_kernel<2><<<grid, kThreads, kSmem, s>>>(a);
  } else {
    SO3G_CUDA(cudaFuncSetAttribute(forward_contract_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    forward_contract_kernel<4><<<grid, kThreads, kSmem, s>>>(a);
  }
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace so3g
