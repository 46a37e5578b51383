// Split-precision Wigner contractions on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, Ozaki scheme), for batches of complex signals.
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
// smallest power of two above twice its largest magnitude), rounded to 49-bit
// fixed point and cut into 7 balanced base-128 digits q_i in [-64, 64]
// (offset-binary extraction: the digits of v + sum_i 64*128^i, minus 64), so
// r = sum_i q_i 2^{-7(i+1)} exactly and the dropped low-order products carry
// no common sign.  The 28 digit products with i + j <= 6 are accumulated
// exactly in int32, one accumulator per diagonal d = i + j, and combined in
// FP64 with weights 2^{-7(d+2)}.  Delta, the quadrature weights, the DFT
// stages and the final combination stay FP64.
//
// Kernel: one CTA per (pair (mu, nu), 64-row tile of the output index, group
// of 16 signals).  Tensor-core product D_d[c, r] += Xs_i[c, k] As_j[r, k]
// with M = 128 signal columns c, N = 64 output rows r, K = the reduction
// index in chunks of 64 through a 2-stage shared-memory ring.  The 7
// accumulators live in tensor memory (7 x 64 int32 columns of 128 lanes).
// Warp roles: warp 0 allocates tensor memory and one of its threads issues
// the MMAs; warp 1 streams the pre-sliced X chunk of each stage with one bulk
// copy; warps 2-9 generate the A digits of each stage from the FP64 Delta
// table and, after the last chunk, read the accumulators back, combine the
// diagonals in FP64 and store.  X is sliced once per batch (slice_inv_kernel,
// slice_fwd_kernel)
// into the exact shared-memory image of a stage.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <memory>
#include <vector>

#include "so3gpu_internal.h"
#include "tc_sm100.cuh"

namespace so3g {

namespace {

constexpr int kS = 7;                  // digits per operand
constexpr int kND = kS;                // diagonals d = i + j = 0 .. 6
constexpr int kSig = 16;               // signals per group
constexpr int kCol = 8;                // columns per signal
constexpr int kM = kSig * kCol;        // 128 MMA rows (signal columns)
constexpr int kN = 64;                 // MMA columns (output rows of the Wigner index)
constexpr int kKC = 64;                // reduction entries per stage
constexpr int kStages = 2;
constexpr int kXStage = kS * kM * kKC;  // 57344 bytes
constexpr int kAStage = kS * kN * kKC;  // 28672 bytes
constexpr int kThreads = 320;           // 10 warps
constexpr int kGen = 256;               // generator / epilogue threads (warps 2-9)
constexpr int kTmemCols = 512;
constexpr double kInv8Pi2 = 0.012665147955292221430803304553147533;  // 1/(8 pi^2)
constexpr long long kDigitOffset = 283691315109952LL;                 // sum_{i<7} 64 * 128^i

// Byte offset of (row, k) inside one digit plane of an operand tile with
// `rows` rows and kKC reduction bytes: core matrices of 8 rows x 16 bytes,
// row groups 128 bytes apart, 16-byte k groups rows*16 bytes apart.
__host__ __device__ constexpr int tile_off(int rows, int row, int k) {
  return (k >> 4) * (rows * 16) + (row >> 3) * 128 + (row & 7) * 16 + (k & 15);
}

// Byte offset of (row r, reduction entry k) inside one digit plane of a
// 64-row operand tile of the tables (Delta products, beta matrix): core
// matrices of 8 rows x 16 bytes, the 4 k groups of a row group 128 bytes
// apart, row groups 512 bytes apart.  The 7 digit planes of a tile are 4096
// bytes apart, so the row groups of consecutive digit planes are uniformly
// 512 bytes apart: digits j .. j+3 of a K-major tile form one operand of
// 64 x (number of digits) rows.
__host__ __device__ constexpr int atile_off(int r, int k) {
  return (r >> 3) * 512 + (k >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

struct __align__(16) TcSmem {
  uint8_t X[kStages][kXStage];   // [stage][digit][tile_off(kM, c, k)]
  uint8_t A[kStages][kAStage];   // [stage][digit][atile_off(r, k)]
  unsigned long long full[kStages];
  unsigned long long empty[kStages];
  unsigned long long accum;
  uint32_t tmem_base;
};

__device__ int g_tc_error;  // bit 1: a wait gave up (see tc::mbar_wait)

// 7 digits of 4 values r in [-1/2, 1/2], packed: byte e of w[i] = digit i of
// value e (digit 0 most significant).
__device__ __forceinline__ void split_pack4(const double (&r)[4], uint32_t (&w)[kS]) {
#pragma unroll
  for (int i = 0; i < kS; i++) w[i] = 0u;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const double shifter = 6755399441055744.0;                  // 1.5 * 2^52
    const double y = fma(r[e], 562949953421312.0, shifter);     // rint(r * 2^49) + shifter
    const long long v = __double_as_longlong(y) - __double_as_longlong(shifter);
    const unsigned long long u = (unsigned long long)(v + kDigitOffset);
    const uint32_t lo = (uint32_t)u, hi = (uint32_t)(u >> 32);
    uint32_t d[kS];
    d[6] = lo & 127u;
    d[5] = (lo >> 7) & 127u;
    d[4] = (lo >> 14) & 127u;
    d[3] = (lo >> 21) & 127u;
    d[2] = ((lo >> 28) | (hi << 4)) & 127u;
    d[1] = (hi >> 3) & 127u;
    d[0] = hi >> 10;  // up to 128
#pragma unroll
    for (int i = 0; i < kS; i++) w[i] |= ((d[i] - 64u) & 255u) << (8 * e);
  }
}

// Exact int32 -> FP64 on the FP64 pipe: the bits 0x43300000:(x + 2^31) are
// the double 2^52 + 2^31 + x; one subtraction leaves x.  (The conversion
// instruction runs on a narrow unit that would otherwise bound the epilogue.)
__device__ __forceinline__ double int_to_double(int x) {
  return __hiloint2double(0x43300000, x ^ (int)0x80000000) - 4503601774854144.0;
}

// Exact int64 -> FP64 for |x| < 2^51 on the FP64 pipe: adding x to the bits
// of 1.5 * 2^52 gives the double 1.5 * 2^52 + x; one subtraction leaves x.
__device__ __forceinline__ double ll_to_double(long long x) {
  return __longlong_as_double(0x4338000000000000LL + x) - 6755399441055744.0;
}

__device__ __forceinline__ double2 ipow(double2 v, int k) {  // v * i^k
  switch (k & 3) {
    case 0: return v;
    case 1: return make_double2(-v.y, v.x);
    case 2: return make_double2(-v.x, -v.y);
    default: return make_double2(v.y, -v.x);
  }
}

struct MixArgs {
  const uint8_t* xs;       // [grp][pair][chunk][kXStage]
  const double* xscale;    // [grp][pair][kM]
  const double* dl;        // Delta quarter planes
  const long long* base;   // block bases per plane
  double2* W;              // inverse: column-major scratch part of signal 0; signal b at W + b * wstride
  double2* const* flmn;    // forward: per-signal coefficient arrays
  const uint8_t* tab;      // resident A-digit blocks (null: generate from Delta)
  const long long* pair_off;  // first block of each pair in tab
  long long wstride;
  int L, N, L0, nchunk, MT, plane0, n_mode, nsig, compact;
  int real;          // real signals: planes n >= 0 only, combinations with n = -nu are empty
  long long CS, QS;  // column-major scratch strides
};

// Resident A digits: for every pair (mu, nu) and every block (row tile t of
// m', chunk kc of l) with kc >= max(t, q), q = max(mu, nu) / 64 (all other
// blocks are zero: A[m', l] needs l >= m' and l >= max(mu, nu)), the 7 x 64
// x 64 digits in the inverse kernel's stage image (rows m', reduction l).
// Blocks of a pair are stored row tile by row tile.
__host__ __device__ inline long long digit_blocks(int q, int nc) {
  return (long long)q * (nc - q) + (long long)(nc - q) * (nc - q + 1) / 2;
}
__host__ __device__ inline long long digit_block(int t, int kc, int q, int nc) {
  if (t <= q) return (long long)t * (nc - q) + (kc - q);
  return (long long)q * (nc - q) + (long long)(t - q) * nc - (long long)(t - q) * (t + q - 1) / 2 + (kc - t);
}

// A digits of one stage.  Thread task (row rho = 8*w + lane%8, quad q =
// 4*it + lane/8, it = 0..3): the 4 reduction entries k0 + 4q .. +3 of row
// rho; the 32 lanes of a warp store 32 distinct banks.
//   inverse: row = m' (r0 + rho), reduction = l;  A^T[l, m'] = Delta_{mu m'} Delta_{nu m'} (l >= m', l >= lmin)
//   forward: row = l  (r0 + rho), reduction = m'; same product
// Delta_{mu m'} is read as row mu of the quarter plane (the transpose
// symmetry's sign (-1)^{mu+nu} is applied in the epilogue).
template <bool FWD>
__device__ __forceinline__ void gen_load(const MixArgs& a, int mu, int nu, int lmin, int r0, int k0, int gw, int lane,
                                         double (&x)[4][4]) {
  const int rho = 8 * gw + (lane & 7);
#pragma unroll
  for (int it = 0; it < 4; it++) {
    const int q = 4 * it + (lane >> 3);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int kk = k0 + 4 * q + e;
      int l, mp;
      if (FWD) {
        l = r0 + rho;
        mp = kk;
      } else {
        l = kk;
        mp = r0 + rho;
      }
      double v = 0.0;
      if (l < a.L && l >= lmin && mp <= l) {
        const double* P = a.dl + dl_plane_offset(l);
        v = P[(long long)mu * (l + 1) + mp] * P[(long long)nu * (l + 1) + mp];
      }
      x[it][e] = 0.5 * v;  // A scale 2
    }
  }
}

__device__ __forceinline__ void gen_store(uint8_t* As, int gw, int lane, const double (&x)[4][4]) {
  const int rho = 8 * gw + (lane & 7);
#pragma unroll
  for (int it = 0; it < 4; it++) {
    const int q = 4 * it + (lane >> 3);
    uint32_t w[kS];
    split_pack4(x[it], w);
    const int off = atile_off(rho, 4 * q);
#pragma unroll
    for (int i = 0; i < kS; i++) *reinterpret_cast<uint32_t*>(As + i * (kN * kKC) + off) = w[i];
  }
}

template <bool FWD, bool TAB>
__global__ void __launch_bounds__(kThreads, 1) mixed_tc_kernel(MixArgs a) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(smraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nu = blockIdx.x % a.N;
  const int rest = blockIdx.x / a.N;
  const int t = rest % a.MT, mu = rest / a.MT;  // consecutive CTAs: same mu and tile, all nu
  const int grp = blockIdx.y, L = a.L;
  const int r0 = t * kN;
  const int lmin = max(max(mu, nu), a.L0);
  int kc0, nk;
  if (FWD) {
    const bool any_row = r0 + kN > lmin && r0 < L;
    const int kend = min(L, r0 + kN);  // m' <= l < r0 + 64
    kc0 = 0;
    nk = any_row ? (kend + kKC - 1) / kKC : 0;
  } else {
    const int kstart = max(lmin, r0) & ~(kKC - 1);
    kc0 = kstart / kKC;
    nk = kstart < L ? (L - kstart + kKC - 1) / kKC : 0;
  }
  const size_t gp = (size_t)grp * a.L * a.N + (size_t)mu * a.N + nu;  // slicing-kernel order
  const uint8_t* xs = a.xs + gp * (size_t)a.nchunk * kXStage;
  // a wait of an earlier CTA gave up: skip the work (the host reports the flag)
  if (*reinterpret_cast<volatile int*>(&g_tc_error)) return;

  const uint32_t full0 = tc::smem_u32(&S.full[0]), empty0 = tc::smem_u32(&S.empty[0]);
  const uint32_t accum = tc::smem_u32(&S.accum);
  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      tc::mbar_init(full0 + 8 * s, TAB ? 1 : kGen + 1);
      tc::mbar_init(empty0 + 8 * s, 1);
    }
    tc::mbar_init(accum, 1);
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&S.tmem_base), kTmemCols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tbase = S.tmem_base;

  if (warp == 0) {
    // ------------------------------------------------ MMA issue (one thread)
    if (lane == 0 && nk > 0) {
      // resident blocks are stored rows m', reduction l; the forward reads them
      // transposed as an MN-major operand (16-l units 1024 B apart, 8-m' groups 128 B apart)
      constexpr uint32_t idesc = tc::idesc_s8(kM, kN) | ((FWD && TAB) ? (1u << 16) : 0u);
      for (int k = 0; k < nk; k++) {
        const int s = k & 1;
        tc::mbar_wait(full0 + 8 * s, (k >> 1) & 1, &g_tc_error, 2);
        tc::tc_fence_after();
        const uint32_t xb = tc::smem_u32(&S.X[s][0]), ab = tc::smem_u32(&S.A[s][0]);
#pragma unroll
        for (int ks = 0; ks < kKC / 32; ks++) {
#pragma unroll
          for (int i = 0; i < kS; i++) {
            // X digit i: LBO = 16-byte k groups (kM*16 bytes apart), SBO = 8-row groups (128 bytes)
            const uint64_t ad = tc::smem_desc(xb + i * (kM * kKC) + ks * 2 * (kM * 16), kM * 16, 128);
            if constexpr (FWD && TAB) {
#pragma unroll
              for (int j = 0; j + i < kND; j++) {
                const uint64_t bd = tc::smem_desc(ab + j * (kN * kKC) + ks * 2048, 512, 128);
                tc::mma_i8(tbase + (uint32_t)(kN * (i + j)), ad, bd, idesc, (k | ks | i) != 0);
              }
            } else {
              // K-major A operand: digits j0 .. j0+3 stacked along N (see issue_item)
#pragma unroll
              for (int j0 = 0; j0 + i < kND; j0 += 4) {
                const int nj = (kND - i - j0) < 4 ? (kND - i - j0) : 4;
                const uint64_t bd = tc::smem_desc(ab + j0 * (kN * kKC) + ks * 256, 128, 512);
                tc::mma_i8(tbase + (uint32_t)(kN * (i + j0)), ad, bd, tc::idesc_s8(kM, kN * nj), (k | ks | i) != 0);
              }
            }
          }
        }
        tc::mma_commit(empty0 + 8 * s);  // stage free once these products have read it
      }
      tc::mma_commit(accum);
    }
  } else if (warp == 1) {
    // ------------------------------------------------ X stream (one thread)
    if (lane == 0) {
      const int q = max(mu, nu) / kKC, ncap = a.nchunk;
      const uint8_t* tb = TAB ? a.tab + (size_t)a.pair_off[(size_t)mu * a.N + nu] * kAStage : nullptr;
      for (int k = 0; k < nk; k++) {
        const int s = k & 1;
        if (k >= kStages) tc::mbar_wait(empty0 + 8 * s, ((k >> 1) - 1) & 1, &g_tc_error, 2);
        tc::mbar_arrive_expect_tx(full0 + 8 * s, TAB ? kXStage + kAStage : kXStage);
        tc::bulk_g2s(tc::smem_u32(&S.X[s][0]), xs + (size_t)(kc0 + k) * kXStage, kXStage, full0 + 8 * s);
        if (TAB) {
          const long long blk = FWD ? digit_block(k, t, q, ncap) : digit_block(t, kc0 + k, q, ncap);
          tc::bulk_g2s(tc::smem_u32(&S.A[s][0]), tb + blk * kAStage, kAStage, full0 + 8 * s);
        }
      }
    }
  } else {
    // ------------------------------------------------ A digits, then epilogue
    const int gw = warp - 2;
    // the Delta loads of chunk k+1 are in flight while chunk k is split
    double xa[4][4], xb[4][4];
    if (!TAB && nk > 0) gen_load<FWD>(a, mu, nu, lmin, r0, kc0 * kKC, gw, lane, xa);
    for (int k = 0; k < (TAB ? 0 : nk); k += 2) {
      if (k + 1 < nk) gen_load<FWD>(a, mu, nu, lmin, r0, (kc0 + k + 1) * kKC, gw, lane, xb);
      if (k >= kStages) tc::mbar_wait(empty0, ((k >> 1) - 1) & 1, &g_tc_error, 2);
      gen_store(&S.A[0][0], gw, lane, xa);
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(full0);
      if (k + 1 >= nk) break;
      if (k + 2 < nk) gen_load<FWD>(a, mu, nu, lmin, r0, (kc0 + k + 2) * kKC, gw, lane, xa);
      if (k + 1 >= kStages) tc::mbar_wait(empty0 + 8, (((k + 1) >> 1) - 1) & 1, &g_tc_error, 2);
      gen_store(&S.A[1][0], gw, lane, xb);
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(full0 + 8);
    }

    // epilogue: thread <-> TMEM lane c (signal column), 32 output rows
    const int lq = warp & 3, ch = gw >> 2;
    const int c = 32 * lq + lane;
    const int b = c >> 3, combo = (c >> 1) & 3, part = c & 1;
    const int ms = (combo & 1) ? -1 : 1, ns = (combo & 2) ? -1 : 1;
    const bool valid_combo = !((ms < 0 && mu == 0) || (ns < 0 && nu == 0) || (a.real && ns < 0));
    const int m = ms * mu, n = ns * nu;
    const int sig = grp * kSig + b;
    const bool one_neg = ms * ns < 0;
    const double sgn_mn = ((mu + nu) & 1) ? -1.0 : 1.0;
    const double scale = a.xscale[gp * kM + c];
    const bool skipped = FWD && plane_skipped(a.n_mode, a.N, n);
    if (nk > 0) {
      tc::mbar_wait(accum, 0, &g_tc_error, 2);
      tc::tc_fence_after();
    }
    double2* Wout = nullptr;
    double2* F = nullptr;
    long long blk = 0;
    // empty combinations (real signals: n = -nu) have no plane: nothing is read or written for them
    if (!FWD) {
      if (valid_combo)
        Wout = a.W + (long long)sig * a.wstride + (long long)(a.plane0 + n) * a.QS + (long long)(m + L - 1) * a.CS;
    } else if (sig < a.nsig && valid_combo) {
      F = a.flmn[sig];
      blk = a.base[a.plane0 + n];
    }
#pragma unroll 1
    for (int g = 0; g < 4; g++) {
      __syncwarp();  // the tensor-memory loads below are warp-collective
      const int col = 32 * ch + 8 * g;  // first of the 8 output rows of this group
      double v[8];
#pragma unroll
      for (int e = 0; e < 8; e++) v[e] = 0.0;
      if (nk > 0) {
        int acc[kND][8];
#pragma unroll
        for (int d = 0; d < kND; d++)
          tc::tmem_ld8(tbase + ((uint32_t)(32 * lq) << 16) + (uint32_t)(kN * d + col), acc[d]);
        tc::tmem_wait_ld();
        double wd = 2.0 * 0.000061035156250000000;  // 2 * 2^{-14}: A scale, diagonal 0
#pragma unroll
        for (int d = 0; d < kND; d++) {
#pragma unroll
          for (int e = 0; e < 8; e++) v[e] = fma(int_to_double(acc[d][e]), wd, v[e]);
          wd *= 0.0078125;  // 2^{-7}
        }
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] *= scale;
      }
      // lanes c (re) and c^1 (im): the re lane writes rows col..col+3, the im lane col+4..col+7
      double re[4], im[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const double send = part ? v[q] : v[4 + q];
        const double recv = __shfl_xor_sync(0xffffffffu, send, 1);
        re[q] = part ? recv : v[q];
        im[q] = part ? v[4 + q] : recv;
      }
      if (!valid_combo || sig >= a.nsig || skipped) continue;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int row = r0 + col + 4 * part + q;
        if (row >= L) continue;
        const double s = (one_neg && (row & 1)) ? -sgn_mn : sgn_mn;
        double2 val = make_double2(re[q] * s, im[q] * s);
        if (!FWD) {
          Wout[row] = ipow(val, n - m + 4 * L);
        } else {
          const int lr = row;
          if (mu > lr) continue;
          if (a.compact && lr < nu) continue;  // not stored
          if (lr < lmin) val = make_double2(0.0, 0.0);
          else val = ipow(val, m - n + 4 * L);
          F[blk + (long long)lr * lr + lr + m] = val;
        }
      }
    }
  }

  // the products have completed before tensor memory is released (immediate
  // in the normal case: the epilogue waited for the same commit)
  if (warp == 0 && lane == 0 && nk > 0) tc::mbar_wait(accum, 0, &g_tc_error, 2);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc::tc_fence_after();
    tc::tmem_dealloc(tbase, kTmemCols);
  }
}

// ---------------------------------------------------------------- slicing
// The X operand of a pair (mu, nu): column c = 8 * signal + 2 * combo + part
// (combo bit 0: m = -mu, bit 1: n = -nu; part: real / imaginary), reduction
// entries k < 64 * nchunk, cut into the 7 digit planes of every stage image
// with the column's power-of-two scale.
//   inverse: X[l, c]   = (2l+1)/(8 pi^2) f_{l m n} (times (-1)^l for one negative index)
//   forward: X'[m', c] = Wc[n][m][m']             (times (-1)^{m'} for one negative index)
struct SliceArgs {
  uint8_t* xs;
  double* xscale;
  const double2* const* flmn;  // inverse input, per signal
  // directional convolution (inverse only): the coefficients are h_lmn =
  // flm_lm conj(glm_ln) 8 pi^2 / (2l+1) of so3_conv.c:186-215, computed on
  // load (never stored); flm shared, glm per signal
  const double2* flm;
  const double2* const* glm;
  const double2* W;            // forward input: column-major scratch part of signal 0, signal b at W + b * wstride
  const long long* base;
  long long wstride;
  int L, N, L0, nchunk, plane0, n_mode, nsig, npairs;
  int real;  // real signals: planes n >= 0 only
  long long CS, QS;
};

__device__ __forceinline__ double scale_of(double mx) {  // power of two with |x / scale| < 1/2
  int ex = 0;
  frexp(mx, &ex);
  return mx > 0.0 ? ldexp(1.0, ex + 1) : 1.0;
}

// Slicing: each CTA reads its columns twice (scales, then digits; the second
// read is served mostly by L2) and writes 16-entry digit slots of the stage
// images; nothing is staged in shared memory.
constexpr int kSliceCols = 8;  // complex columns per forward slicing CTA (4 sign combinations x 2 signals)

// Inverse.  One CTA per (nu, block of kMuPer mu, signal): its complex
// columns (kMuPer mu x combos (+-m, +-nu)) are the rows 8 * (signal % 16)
// .. +7 of the stage images of its pairs.  Entries l < max(mu, nu, L0) are
// zero.  Two passes over the CTA's flmn entries (runs of kMuPer consecutive
// m per (n, l)): the first finds the column scales, the second (served
// mostly by L2, a CTA's entries being a few hundred KB) writes the digits.
// Nothing is staged in shared memory, so several CTAs per SM keep loads in
// flight.
constexpr int kMuPer = 4;  // 64-byte runs of m per (n, l)

struct InvColumn {
  const double2* src;   // entry l at src[l * l + l] (the signal's flmn, or flm of a convolution)
  const double2* gsrc;  // convolution: entry l of the kernel glm at gsrc[l * l + l] (order n)
  int lmin;
  bool act, flip;
};
__device__ __forceinline__ InvColumn inv_column(const SliceArgs& a, int sig, int mu, int nu, int combo) {
  const int ms = (combo & 1) ? -1 : 1, ns = (combo & 2) ? -1 : 1;
  const int m = ms * mu, n = ns * nu;
  InvColumn c;
  c.act = mu < a.L && sig < a.nsig && !(ms < 0 && mu == 0) && !(ns < 0 && nu == 0) && !(a.real && ns < 0) &&
          !plane_skipped(a.n_mode, a.N, n);
  c.lmin = max(max(mu, nu), a.L0);
  c.flip = ms * ns < 0;
  c.src = c.act ? (a.flm ? a.flm + m : a.flmn[sig] + a.base[a.plane0 + n] + m) : nullptr;
  c.gsrc = (c.act && a.flm) ? a.glm[sig] + n : nullptr;
  return c;
}
// Weighted entry l of the column (both parts), times (-1)^l on flipped
// columns: (2l+1)/(8 pi^2) f_lmn, or for a convolution (2l+1)/(8 pi^2) h_lmn
// = flm_lm conj(glm_ln).
__device__ __forceinline__ double2 inv_value(const InvColumn& c, int L, int l) {
  if (!(c.act && l < L && l >= c.lmin)) return make_double2(0.0, 0.0);
  const double2 x = __ldg(c.src + (long long)l * l + l);
  double2 v;
  if (c.gsrc) {
    const double2 gk = __ldg(c.gsrc + (long long)l * l + l);
    v = make_double2(fma(x.x, gk.x, x.y * gk.y), fma(x.y, gk.x, -x.x * gk.y));
  } else {
    const double f = (2.0 * l + 1.0) * kInv8Pi2;
    v = make_double2(x.x * f, x.y * f);
  }
  if (c.flip && (l & 1)) v = make_double2(-v.x, -v.y);
  return v;
}
__device__ __forceinline__ double inv_entry(const InvColumn& c, int L, int l, int part) {
  const double2 v = inv_value(c, L, l);
  return part ? v.y : v.x;
}

__global__ void __launch_bounds__(256, 3) slice_inv_kernel(SliceArgs a) {
  __shared__ double wmax[8][2 * 4 * kMuPer];  // [warp][2 (4 j + combo) + part]
  __shared__ double scl[kMuPer][2 * 4];
  const int Lp = a.nchunk * kKC, L = a.L;
  const int nu = blockIdx.x % a.N, mu0 = (blockIdx.x / a.N) * kMuPer, sig = blockIdx.y;
  const int grp = sig / kSig, b = sig % kSig;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  {
    // thread <-> (j, combo) fixed (m fastest across lanes), l = l0 + 16 i;
    // 8 loads in flight per thread
    const int j = threadIdx.x % kMuPer, combo = (threadIdx.x / kMuPer) & 3, l0 = threadIdx.x / (4 * kMuPer);
    constexpr int LSTEP = 256 / (4 * kMuPer);  // l-lanes
    const InvColumn col = inv_column(a, sig, mu0 + j, nu, combo);
    double mr = 0.0, mi = 0.0;
    if (col.act) {
      for (int l1 = l0; l1 < L; l1 += LSTEP * 8) {
        double2 x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) x[u] = inv_value(col, L, l1 + LSTEP * u);
#pragma unroll
        for (int u = 0; u < 8; u++) {
          mr = fmax(mr, fabs(x[u].x));
          mi = fmax(mi, fabs(x[u].y));
        }
      }
    }
    // lanes l and l + 16 of a warp hold the same column
    mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, 16));
    mi = fmax(mi, __shfl_xor_sync(0xffffffffu, mi, 16));
    if (lane < 16) {
      wmax[warp][2 * (j * 4 + combo)] = mr;
      wmax[warp][2 * (j * 4 + combo) + 1] = mi;
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * 4 * kMuPer) {
    double mx = 0.0;
#pragma unroll
    for (int w = 0; w < 8; w++) mx = fmax(mx, wmax[w][threadIdx.x]);
    const int jc = threadIdx.x >> 1, part = threadIdx.x & 1;
    scl[jc >> 2][2 * (jc & 3) + part] = scale_of(mx);
  }
  __syncthreads();
  for (int j = 0; j < kMuPer; j++) {
    const int mu = mu0 + j;
    if (mu >= L) break;
    const size_t gp = (size_t)grp * a.npairs + (size_t)mu * a.N + nu;
    if (threadIdx.x < 8) a.xscale[gp * kM + 8 * b + threadIdx.x] = scl[j][threadIdx.x];
  }
  // digits: 8 real columns per pair, 16 entries per work item
  for (int w = threadIdx.x; w < kMuPer * 8 * (Lp / 16); w += blockDim.x) {
    const int c = w & 7, j = (w >> 3) % kMuPer, kb = w / (8 * kMuPer);
    const int mu = mu0 + j;
    if (mu >= L) continue;
    // chunks below the one holding l = max(mu, nu, L0) are never read: the
    // inverse items start at that chunk (decode_item), so they are not written
    if (16 * kb / kKC < max(max(mu, nu), a.L0) / kKC) continue;
    const int combo = c >> 1, part = c & 1;
    const double inv = 1.0 / scl[j][c];
    const InvColumn col = inv_column(a, sig, mu, nu, combo);
    uint32_t d[4][kS];
#pragma unroll
    for (int qd = 0; qd < 4; qd++) {
      double r[4];
#pragma unroll
      for (int e = 0; e < 4; e++) r[e] = inv_entry(col, L, 16 * kb + 4 * qd + e, part) * inv;
      split_pack4(r, d[qd]);
    }
    const size_t gp = (size_t)grp * a.npairs + (size_t)mu * a.N + nu;
    uint8_t* dst = a.xs + gp * (size_t)a.nchunk * kXStage + (size_t)(kb >> 2) * kXStage +
                   tile_off(kM, 8 * b + c, (kb & 3) * 16);
#pragma unroll
    for (int i = 0; i < kS; i++)
      *reinterpret_cast<uint4*>(dst + i * (kM * kKC)) = make_uint4(d[0][i], d[1][i], d[2][i], d[3][i]);
  }
}

// Streaming form of the inverse slicing (uniform batches of plain
// coefficients, L <= 1024): the caller's flmn is read in storage order, where
// the entries l^2 + l + m of a row l are contiguous in m, so consecutive
// threads read consecutive addresses and a CTA reads whole rows of one plane.
// Pass 1 (inv_colscale_kernel) finds the scale of every column (n, m, part);
// pass 2 (inv_digit_kernel) cuts one 16-entry reduction slot of every column
// of a plane into digits.  Both give the same scales and digits as
// slice_inv_kernel (same arithmetic per entry).  Column (n, m) is row
// 8 (signal % 16) + 2 combo (+ part) of pair (|m|, |n|), combo bit 0: m < 0,
// bit 1: n < 0; the (-1)^l of combinations with one negative index is applied
// on the entry.
constexpr int kStreamThreads = 256;

// Pass 1: one CTA per (plane, signal); thread t owns the columns m = t - (L-1)
// + 256 k (k < OWN) and walks the rows l >= max(|n|, L0) four at a time.
// Skipped planes are left to pass 2 (zero digits, scale 1).
template <int OWN>
__global__ void __launch_bounds__(kStreamThreads) inv_colscale_kernel(SliceArgs a, double* colscl, int nplanes) {
  const int p = blockIdx.x, sig = blockIdx.y, L = a.L, n = p - a.plane0, t = threadIdx.x;
  const int ncol = 2 * L - 1;
  if (plane_skipped(a.n_mode, a.N, n)) return;
  const double2* src = a.flmn[sig] + a.base[p];
  double mr[OWN], mi[OWN];
  int mm[OWN];
#pragma unroll
  for (int k = 0; k < OWN; k++) mr[k] = mi[k] = 0.0, mm[k] = t + kStreamThreads * k - (L - 1);
  for (int l = max(abs(n), a.L0); l < L; l += 4) {
    double2 x[4][OWN];
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int k = 0; k < OWN; k++) {
        const int ll = l + u, m = mm[k];
        x[u][k] = (ll < L && m <= L - 1 && abs(m) <= ll) ? __ldg(src + (long long)ll * ll + ll + m)
                                                          : make_double2(0.0, 0.0);
      }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const double w = (2.0 * (l + u) + 1.0) * kInv8Pi2;
#pragma unroll
      for (int k = 0; k < OWN; k++) {
        mr[k] = fmax(mr[k], fabs(x[u][k].x * w));
        mi[k] = fmax(mi[k], fabs(x[u][k].y * w));
      }
    }
  }
  double* out = colscl + ((size_t)sig * nplanes + p) * (size_t)ncol * 2;
#pragma unroll
  for (int k = 0; k < OWN; k++) {
    const int m = mm[k];
    if (m <= L - 1) {
      out[2 * (m + L - 1)] = scale_of(mr[k]);
      out[2 * (m + L - 1) + 1] = scale_of(mi[k]);
    }
  }
}

// Pass 2: one CTA per (reduction slot kb of 16 entries, nu = |n|, signal);
// thread t takes the sign combination t % 4 of the columns mu = t / 4 + 64 k:
// the four lanes of a mu write the 4 x 32 contiguous bytes of the signal's 8
// rows of the pair's image per digit plane (rows c, c+1: both parts), and the
// 8 mu of a warp read 128-byte runs of each row l of the planes +-nu.
// Slots of chunks below the one holding l = max(mu, nu, L0) are never read by
// the products and are not written; the column scales are written by the
// first written slot.
__global__ void __launch_bounds__(kStreamThreads, 2) inv_digit_kernel(SliceArgs a, const double* colscl, int nplanes) {
  const int kb = blockIdx.x, nu = blockIdx.y, sig = blockIdx.z, combo = threadIdx.x & 3;
  const int L = a.L, ncol = 2 * L - 1;
  const int ms = (combo & 1) ? -1 : 1, ns = (combo & 2) ? -1 : 1, n = ns * nu, p = a.plane0 + n;
  if ((ns < 0 && nu == 0) || (a.real && ns < 0)) return;  // no such plane (whole warps: combo is lane % 4)
  const bool skipped = plane_skipped(a.n_mode, a.N, n);
  const bool flip = ms * ns < 0;
  const int grp = sig / kSig, b = sig % kSig, c = 8 * b + 2 * combo;
  const double2* src = a.flmn[sig] + a.base[p];
  const double* scl = colscl + ((size_t)sig * nplanes + p) * (size_t)ncol * 2;
  for (int mu = (int)threadIdx.x / 4; mu < L; mu += kStreamThreads / 4) {
    const int m = ms * mu, lmin = max(max(mu, nu), a.L0);
    if ((ms < 0 && mu == 0) || 16 * kb / kKC < lmin / kKC) continue;
    const double sr = skipped ? 1.0 : scl[2 * (m + L - 1)];
    const double si = skipped ? 1.0 : scl[2 * (m + L - 1) + 1];
    const size_t gp = (size_t)grp * a.npairs + (size_t)mu * a.N + nu;
    if (kb == 4 * (lmin / kKC)) {
      a.xscale[gp * kM + c] = sr;
      a.xscale[gp * kM + c + 1] = si;
    }
    double2 x[16];
#pragma unroll
    for (int e = 0; e < 16; e++) {
      const int l = 16 * kb + e;
      x[e] = (!skipped && l < L && l >= lmin) ? __ldg(src + (long long)l * l + l + m) : make_double2(0.0, 0.0);
    }
    uint8_t* dst = a.xs + gp * (size_t)a.nchunk * kXStage + (size_t)(kb >> 2) * kXStage + tile_off(kM, c, (kb & 3) * 16);
#pragma unroll
    for (int part = 0; part < 2; part++) {
      const double inv = 1.0 / (part ? si : sr);
      uint32_t d[4][kS];
#pragma unroll
      for (int qd = 0; qd < 4; qd++) {
        double r[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int l = 16 * kb + 4 * qd + e;
          const double f = (2.0 * l + 1.0) * kInv8Pi2;
          double v = (part ? x[4 * qd + e].y : x[4 * qd + e].x) * f;
          if (flip && (l & 1)) v = -v;
          r[e] = v * inv;
        }
        split_pack4(r, d[qd]);
      }
#pragma unroll
      for (int i = 0; i < kS; i++)
        *reinterpret_cast<uint4*>(dst + 16 * part + i * (kM * kKC)) = make_uint4(d[0][i], d[1][i], d[2][i], d[3][i]);
    }
  }
}

// Forward.  One CTA per (pair, kSigPer signals): complex columns cc = 4 *
// signal + combo (rows 8 kSigPer q .. of the pair's stage image for the
// q-th set of kSigPer signals of the group); warp <-> column, lanes along m'
// (512-byte runs).
constexpr int kSigPer = kSliceCols / 4;
struct FwdColumn {
  const double2* src;  // entry k (m') at src[k]
  bool act, flip;
};
__device__ __forceinline__ FwdColumn fwd_column(const SliceArgs& a, int sig, int mu, int nu, int combo) {
  const int ms = (combo & 1) ? -1 : 1, ns = (combo & 2) ? -1 : 1;
  const int m = ms * mu, n = ns * nu;
  FwdColumn c;
  c.act = sig < a.nsig && !(ms < 0 && mu == 0) && !(ns < 0 && nu == 0) && !(a.real && ns < 0) &&
          !plane_skipped(a.n_mode, a.N, n);
  c.flip = ms * ns < 0;
  c.src = c.act ? a.W + (long long)sig * a.wstride + (long long)(a.plane0 + n) * a.QS + (long long)(m + a.L - 1) * a.CS
                : nullptr;
  return c;
}

// Two passes over the CTA's columns (contiguous runs of m'): warp cc finds
// the scales of column cc, then every thread writes 16-entry digit slots
// from a second read (served mostly by L2).  No staging in shared memory.
__global__ void __launch_bounds__(256) slice_fwd_kernel(SliceArgs a) {
  __shared__ double scl[2 * kSliceCols];
  const int Lp = a.nchunk * kKC, L = a.L;
  const int pair = blockIdx.x, q4 = blockIdx.y;  // q4: set of kSigPer signals
  const int nu = pair % a.N, mu = pair / a.N;
  const int grp = (kSigPer * q4) / kSig, qin = q4 % (kSig / kSigPer);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int cc = warp; cc < kSliceCols; cc += 8) {
    const FwdColumn col = fwd_column(a, kSigPer * q4 + (cc >> 2), mu, nu, cc & 3);
    double mr = 0.0, mi = 0.0;
    if (col.act) {
      for (int k1 = lane; k1 < L; k1 += 32 * 8) {  // 8 loads in flight per lane
        double2 x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int k = k1 + 32 * u;
          x[u] = k < L ? __ldg(col.src + k) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          mr = fmax(mr, fabs(x[u].x));
          mi = fmax(mi, fabs(x[u].y));
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
      mi = fmax(mi, __shfl_xor_sync(0xffffffffu, mi, o));
    }
    if (lane == 0) scl[2 * cc] = scale_of(mr), scl[2 * cc + 1] = scale_of(mi);
  }
  __syncthreads();
  const size_t gp = (size_t)grp * a.npairs + pair;
  if (threadIdx.x < 2 * kSliceCols) a.xscale[gp * kM + 2 * kSliceCols * qin + threadIdx.x] = scl[threadIdx.x];
  uint8_t* pb = a.xs + gp * (size_t)a.nchunk * kXStage;
  const int c_base = 2 * kSliceCols * qin, nblk = Lp / 16;
  for (int w = threadIdx.x; w < 2 * kSliceCols * nblk; w += blockDim.x) {
    const int c = w % (2 * kSliceCols), kb = w / (2 * kSliceCols), cc = c >> 1, part = c & 1;
    const FwdColumn col = fwd_column(a, kSigPer * q4 + (cc >> 2), mu, nu, cc & 3);
    const double inv = 1.0 / scl[c];
    const double* src = reinterpret_cast<const double*>(col.src) + part;
    uint32_t d[4][kS];
#pragma unroll
    for (int qd = 0; qd < 4; qd++) {
      double r[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int k = 16 * kb + 4 * qd + e;
        double x = (col.act && k < L) ? __ldg(src + 2 * k) : 0.0;
        if (col.flip && (k & 1)) x = -x;
        r[e] = x * inv;
      }
      split_pack4(r, d[qd]);
    }
    uint8_t* dst = pb + (size_t)(kb >> 2) * kXStage + tile_off(kM, c_base + c, (kb & 3) * 16);
#pragma unroll
    for (int i = 0; i < kS; i++)
      *reinterpret_cast<uint4*>(dst + i * (kM * kKC)) = make_uint4(d[0][i], d[1][i], d[2][i], d[3][i]);
  }
}

// ---------------------------------------------------------------- persistent form
// With the resident digit table, the products run as a persistent kernel:
// one CTA per SM walks the work items (pair, output tile, signal group) with
// a stride of the grid size.  The bulk-copy thread runs ahead across item
// boundaries through the 2-stage ring; the MMA thread starts an item as soon
// as the epilogue has drained the accumulators of the previous one (mbarrier
// acce, 256 arrivals), so the epilogue's FP64 combination and global stores
// overlap the next item's products.
struct __align__(16) TcpSmem {
  uint8_t X[kStages][kXStage];
  uint8_t A[kStages][kAStage];
  unsigned long long full[kStages];
  unsigned long long empty[kStages];
  unsigned long long accf;  // accumulators complete (tcgen05.commit)
  unsigned long long acce;  // accumulators drained (epilogue threads)
  uint32_t tmem_base;
};

struct ItemC {  // one contraction work item
  int mu, nu, t, grp, kc0, nk, lmin;
  bool valid;  // false: padding item past the band limit (no products, no output)
};

// Item order.  Inverse: (group, mu, tile, nu), nu fastest (the CTAs in
// flight share mu rows of the digit table and one mu's operands).  Forward:
// (group, nu, block of 16 mu, tile, mu), mu fastest: the coefficients
// (l, +-mu) and (l, +-(mu+1)) share 32-byte sectors of the caller's flmn, and
// CTAs that run at the same time write both halves; one block's operands
// (16 pairs) stay in L2 across its tiles.
constexpr int kMuBlock = 16;
__host__ __device__ inline long long mixed_items(int L, int N, int MT, int groups, bool fwd) {
  return fwd ? (long long)kMuBlock * MT * ((L + kMuBlock - 1) / kMuBlock) * N * groups : (long long)L * N * MT * groups;
}

template <bool FWD>
__device__ __forceinline__ ItemC decode_item(const MixArgs& a, int item) {
  ItemC it;
  if (FWD) {
    const int mi = item % kMuBlock;
    int r = item / kMuBlock;
    it.t = r % a.MT;
    r /= a.MT;
    const int nmb = (a.L + kMuBlock - 1) / kMuBlock;
    const int mb = r % nmb;
    r /= nmb;
    it.nu = r % a.N;
    it.grp = r / a.N;
    it.mu = mb * kMuBlock + mi;
    if (it.mu >= a.L) {  // past the band limit: no work
      it.mu = a.L - 1, it.kc0 = 0, it.nk = 0, it.lmin = a.L, it.valid = false;
      return it;
    }
  } else {
    const int per = a.L * a.N * a.MT;
    const int bx = item % per;
    it.grp = item / per;
    it.nu = bx % a.N;
    const int rest = bx / a.N;
    it.t = rest % a.MT;
    it.mu = rest / a.MT;
  }
  it.valid = true;
  const int r0 = it.t * kN;
  it.lmin = max(max(it.mu, it.nu), a.L0);
  if (FWD) {
    const bool any_row = r0 + kN > it.lmin && r0 < a.L;
    it.kc0 = 0;
    it.nk = any_row ? (min(a.L, r0 + kN) + kKC - 1) / kKC : 0;
  } else {
    const int kstart = max(it.lmin, r0) & ~(kKC - 1);
    it.kc0 = kstart / kKC;
    it.nk = kstart < a.L ? (a.L - kstart + kKC - 1) / kKC : 0;
  }
  return it;
}

// Sum of the 7 diagonals of 8 accumulator columns, as FP64 (weight w0 on
// diagonal 0, then / 128 per diagonal).  PAIRED (reductions of at most 512
// entries): diagonals (1,2), (3,4), (5,6) are first folded exactly in int32
// as 128 acc_d + acc_{d+1} (|digit products| <= 64 * 64, so the largest
// folded sum, 64 * 64 * 512 * (6 * 128 + 7), stays below 2^31), leaving 4
// conversions and 4 FMAs per value instead of 7 and 7.
template <bool PAIRED>
__device__ __forceinline__ void drain8(uint32_t taddr, double w0, double (&v)[8]) {
  int acc[kND][8];
#pragma unroll
  for (int d = 0; d < kND; d++) tc::tmem_ld8(taddr + (uint32_t)(kN * d), acc[d]);
  tc::tmem_wait_ld();
#pragma unroll
  for (int e = 0; e < 8; e++) v[e] = 0.0;
  if (PAIRED) {
    // exact integer sums: hi = acc0 2^14 + (128 acc1 + acc2) (|hi| < 2^39),
    // lo = (128 acc3 + acc4) 2^14 + (128 acc5 + acc6) (|lo| < 2^46); value =
    // w0 (hi 2^{-14} + lo 2^{-42}): two conversions and two FP64 operations
    const double whi = w0 * 0.00006103515625, wlo = w0 * 2.2737367544323206e-13;  // 2^{-14}, 2^{-42}
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const long long hi = (long long)acc[0][e] * 16384 + (acc[1][e] * 128 + acc[2][e]);
      const long long lo = (long long)(acc[3][e] * 128 + acc[4][e]) * 16384 + (acc[5][e] * 128 + acc[6][e]);
      v[e] = fma(ll_to_double(hi), whi, ll_to_double(lo) * wlo);
    }
  } else {
    double wd = w0;
#pragma unroll
    for (int d = 0; d < kND; d++) {
#pragma unroll
      for (int e = 0; e < 8; e++) v[e] = fma(int_to_double(acc[d][e]), wd, v[e]);
      wd *= 0.0078125;
    }
  }
}

// Issue of one item's products from the ring (G: running chunk counter).
// K-major table operand (inverse contraction, beta stage): for digit i of X
// the digits j = 0 .. 6-i of the table are consecutive in shared memory with
// uniformly spaced row groups (atile_off), and the accumulators of diagonals
// i .. 6 are consecutive tensor-memory columns, so the products X_i A_j of up
// to 4 digits j run as ONE MMA with N = 64 x (number of digits) <= 256: 10
// instructions per 32 reduction entries instead of 28, and X_i is read from
// shared memory 10 times instead of 28 (at N = 64 the operand reads, not the
// multiply-adds, bound the instruction rate).  MN-major table operand (forward
// contraction): the column groups of consecutive digits are not uniformly
// spaced, so each product is its own N = 64 MMA.
template <bool MNB>
__device__ __forceinline__ void issue_item(TcpSmem& S, uint32_t tbase, int nk, int& G) {
  const uint32_t full0 = tc::smem_u32(&S.full[0]), empty0 = tc::smem_u32(&S.empty[0]);
  for (int k = 0; k < nk; k++, G++) {
    const int st = G & 1;
    tc::mbar_wait(full0 + 8 * st, (G >> 1) & 1, &g_tc_error, 2);
    tc::tc_fence_after();
    const uint32_t xb = tc::smem_u32(&S.X[st][0]), ab = tc::smem_u32(&S.A[st][0]);
#pragma unroll
    for (int ks = 0; ks < kKC / 32; ks++) {
#pragma unroll
      for (int i = 0; i < kS; i++) {
        const uint64_t ad = tc::smem_desc(xb + i * (kM * kKC) + ks * 2 * (kM * 16), kM * 16, 128);
        if constexpr (MNB) {
#pragma unroll
          for (int j = 0; j + i < kND; j++) {
            const uint64_t bd = tc::smem_desc(ab + j * (kN * kKC) + ks * 2048, 512, 128);
            tc::mma_i8(tbase + (uint32_t)(kN * (i + j)), ad, bd, tc::idesc_s8(kM, kN) | (1u << 16), (k | ks | i) != 0);
          }
        } else {
#pragma unroll
          for (int j0 = 0; j0 + i < kND; j0 += 4) {
            const int nj = (kND - i - j0) < 4 ? (kND - i - j0) : 4;
            const uint64_t bd = tc::smem_desc(ab + j0 * (kN * kKC) + ks * 256, 128, 512);
            tc::mma_i8(tbase + (uint32_t)(kN * (i + j0)), ad, bd, tc::idesc_s8(kM, kN * nj), (k | ks | i) != 0);
          }
        }
      }
    }
    tc::mma_commit(empty0 + 8 * st);
  }
}

__device__ __forceinline__ void load_chunk(TcpSmem& S, int& G, const uint8_t* xsrc, const uint8_t* asrc) {
  const uint32_t full0 = tc::smem_u32(&S.full[0]), empty0 = tc::smem_u32(&S.empty[0]);
  const int st = G & 1;
  if (G >= kStages) tc::mbar_wait(empty0 + 8 * st, ((G >> 1) - 1) & 1, &g_tc_error, 2);
  tc::mbar_arrive_expect_tx(full0 + 8 * st, kXStage + kAStage);
  tc::bulk_g2s(tc::smem_u32(&S.X[st][0]), xsrc, kXStage, full0 + 8 * st);
  tc::bulk_g2s(tc::smem_u32(&S.A[st][0]), asrc, kAStage, full0 + 8 * st);
  G++;
}

__device__ __forceinline__ void tcp_setup(TcpSmem& S, int tid, int warp) {
  if (tid == 0) {
    for (int st = 0; st < kStages; st++) {
      tc::mbar_init(tc::smem_u32(&S.full[st]), 1);
      tc::mbar_init(tc::smem_u32(&S.empty[st]), 1);
    }
    tc::mbar_init(tc::smem_u32(&S.accf), 1);
    tc::mbar_init(tc::smem_u32(&S.acce), kGen);
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&S.tmem_base), kTmemCols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
}

__device__ __forceinline__ void tcp_teardown(TcpSmem& S, int warp) {
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc::tc_fence_after();
    tc::tmem_dealloc(S.tmem_base, kTmemCols);
  }
}

// Epilogue drain of one item: the thread's 32 output rows (4 groups of 8)
// combined into v, then the accumulators are released.
__device__ __forceinline__ void drain_item(TcpSmem& S, int lq, int ch, double w0, bool paired, int& ia,
                                           double (&v)[4][8]) {
  tc::mbar_wait(tc::smem_u32(&S.accf), ia & 1, &g_tc_error, 2);
  tc::tc_fence_after();
#pragma unroll
  for (int g = 0; g < 4; g++) {
    __syncwarp();
    const uint32_t ta = S.tmem_base + ((uint32_t)(32 * lq) << 16) + (uint32_t)(32 * ch + 8 * g);
    if (paired)
      drain8<true>(ta, w0, v[g]);
    else
      drain8<false>(ta, w0, v[g]);
  }
  tc::tc_fence_before();
  tc::mbar_arrive(tc::smem_u32(&S.acce));
  ia++;
}

template <bool FWD>
__global__ void __launch_bounds__(kThreads, 1) mixed_tcp_kernel(MixArgs a, int nitems) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  TcpSmem& S = *reinterpret_cast<TcpSmem*>(smraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (*reinterpret_cast<volatile int*>(&g_tc_error)) return;
  tcp_setup(S, tid, warp);
  if (warp == 0) {
    if (lane == 0) {
      int G = 0, ia = 0;
      for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const ItemC it = decode_item<FWD>(a, item);
        if (it.nk == 0) continue;
        if (ia > 0) tc::mbar_wait(tc::smem_u32(&S.acce), (ia - 1) & 1, &g_tc_error, 2);
        tc::tc_fence_after();
        issue_item<FWD>(S, S.tmem_base, it.nk, G);
        tc::mma_commit(tc::smem_u32(&S.accf));
        ia++;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int G = 0;
      for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const ItemC it = decode_item<FWD>(a, item);
        if (it.nk == 0) continue;
        const size_t gp = (size_t)it.grp * a.L * a.N + (size_t)it.mu * a.N + it.nu;
        const uint8_t* xs = a.xs + gp * (size_t)a.nchunk * kXStage;
        const int q = max(it.mu, it.nu) / kKC;
        const uint8_t* tb = a.tab + (size_t)a.pair_off[(size_t)it.mu * a.N + it.nu] * kAStage;
        for (int k = 0; k < it.nk; k++) {
          const long long blk = FWD ? digit_block(k, it.t, q, a.nchunk) : digit_block(it.t, it.kc0 + k, q, a.nchunk);
          load_chunk(S, G, xs + (size_t)(it.kc0 + k) * kXStage, tb + blk * kAStage);
        }
      }
    }
  } else {
    const int gw = warp - 2, lq = warp & 3, ch = gw >> 2;
    const int c = 32 * lq + lane;
    const int b = c >> 3, combo = (c >> 1) & 3, part = c & 1;
    const int ms = (combo & 1) ? -1 : 1, ns = (combo & 2) ? -1 : 1;
    const bool paired = a.nchunk * kKC <= 512;
    int ia = 0;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      const ItemC it = decode_item<FWD>(a, item);
      if (!it.valid) continue;
      // per-item metadata first: these loads overlap the wait for the products
      const int mu = it.mu, nu = it.nu, L = a.L, r0 = it.t * kN;
      const bool valid_combo = !((ms < 0 && mu == 0) || (ns < 0 && nu == 0) || (a.real && ns < 0));
      const int m = ms * mu, n = ns * nu;
      const int sig = it.grp * kSig + b;
      const bool one_neg = ms * ns < 0;
      const double sgn_mn = ((mu + nu) & 1) ? -1.0 : 1.0;
      const size_t gp = (size_t)it.grp * a.L * a.N + (size_t)mu * a.N + nu;
      const double scale = a.xscale[gp * kM + c];
      const bool skipped = FWD && plane_skipped(a.n_mode, a.N, n);
      double2* Wout = nullptr;
      double2* F = nullptr;
      long long blk = 0;
      // empty combinations (real signals: n = -nu) have no plane: nothing is read or written for them
      if (!FWD) {
        if (valid_combo)
          Wout = a.W + (long long)sig * a.wstride + (long long)(a.plane0 + n) * a.QS + (long long)(m + L - 1) * a.CS;
      } else if (sig < a.nsig && valid_combo) {
        F = a.flmn[sig];
        blk = a.base[a.plane0 + n];
      }
      double v[4][8];
      if (it.nk > 0) {
        drain_item(S, lq, ch, 2.0 * 0.000061035156250000000, paired, ia, v);  // A scale 2, 2^{-14}
      } else {
#pragma unroll
        for (int g = 0; g < 4; g++)
#pragma unroll
          for (int e = 0; e < 8; e++) v[g][e] = 0.0;
      }
#pragma unroll
      for (int g = 0; g < 4; g++) {
        const int col = 32 * ch + 8 * g;
        double re[4], im[4];
#pragma unroll
        for (int qq = 0; qq < 4; qq++) {
          const double send = (part ? v[g][qq] : v[g][4 + qq]) * scale;
          const double recv = __shfl_xor_sync(0xffffffffu, send, 1);
          re[qq] = part ? recv : v[g][qq] * scale;
          im[qq] = part ? v[g][4 + qq] * scale : recv;
        }
        if (!valid_combo || sig >= a.nsig || skipped) continue;
#pragma unroll
        for (int qq = 0; qq < 4; qq++) {
          const int row = r0 + col + 4 * part + qq;
          if (row >= L) continue;
          const double sgn = (one_neg && (row & 1)) ? -sgn_mn : sgn_mn;
          double2 val = make_double2(re[qq] * sgn, im[qq] * sgn);
          if (!FWD) {
            Wout[row] = ipow(val, n - m + 4 * L);
          } else {
            const int lr = row;
            if (mu > lr) continue;
            if (a.compact && lr < nu) continue;
            if (lr < it.lmin) val = make_double2(0.0, 0.0);
            else val = ipow(val, m - n + 4 * L);
            F[blk + (long long)lr * lr + lr + m] = val;
          }
        }
      }
    }
  }
  tcp_teardown(S, warp);
}

// One CTA per pair: every stored block of the pair, generated exactly as the
// inverse kernel's producer warps generate a stage (8 warps of 32 lanes).
__global__ void __launch_bounds__(256) digit_table_kernel(MixArgs a, uint8_t* tab) {
  const int pair = blockIdx.x, mu = pair / a.N, nu = pair % a.N;
  const int gw = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = max(mu, nu) / kKC, nc = a.nchunk, lmin = max(mu, nu);
  uint8_t* out = tab + (size_t)a.pair_off[pair] * kAStage;
  for (int t = 0; t < nc; t++)
    for (int kc = max(t, q); kc < nc; kc++) {
      double x[4][4];
      gen_load<false>(a, mu, nu, lmin, t * kN, kc * kKC, gw, lane, x);
      gen_store(out + digit_block(t, kc, q, nc) * kAStage, gw, lane, x);
    }
}

// ---------------------------------------------------------------- forward beta stage
// The forward beta stage of one (n, m) column (extension onto the circle,
// DFT, MW phase, quadrature-weight convolution, fold; stages.cu) is a fixed
// linear map of the L beta samples g_b onto the L outputs m' >= 0 that
// depends only on L and on s = (-1)^{m+n}:
//   out(m') = sum_b R_s(m', b) g_b                   (s = +1, and m' = 0)
//   out(m') = i sum_b R_s(m', b) g_b                 (s = -1, m' >= 1)
// with R_s real:  R_s(m', b) = sum_{m''} c_b(m'') W_s(m'', m'),
//   c_b(m'') = (e^{-i m'' beta_b} + s e^{i m'' beta_b}) / (2L-1)  (b < L-1),
//   c_{L-1}(m'') = (-1)^{m''} / (2L-1)     (beta_b = pi (2b+1)/(2L-1), MW),
//   W_s(m'', m') = 2 pi (w(m'-m'') + s w(-m'-m'')) for m' >= 1, 2 pi w(-m'') for m' = 0,
// w the quadrature weights of so3_sampling.c:32-51.  For the split-precision
// batch path the stage runs as one more int8 Ozaki product on the tensor
// cores: the columns of a parity class form the 128-row operand (64 columns
// x re/im), R_s (FP64, sliced once per L) the resident 64-row operand.
__device__ __forceinline__ double2 quad_weight(int p, int L) {
  if (p > 2 * (L - 1) || p < -2 * (L - 1)) return make_double2(0.0, 0.0);
  if (p == 1) return make_double2(0.0, -1.5707963267948966192313216916397514);
  if (p == -1) return make_double2(0.0, 1.5707963267948966192313216916397514);
  if (p & 1) return make_double2(0.0, 0.0);
  return make_double2(2.0 / (1.0 - (double)p * (double)p), 0.0);
}

// R_s in FP64: out[(sc * L + m') * L + b], sc = 0 (s = +1) or 1 (s = -1).
__global__ void beta_matrix_kernel(int L, double* out) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= 2LL * L * L) return;
  const int b = (int)(id % L), mp = (int)((id / L) % L), sc = (int)(id / ((long long)L * L));
  const double s = sc ? -1.0 : 1.0;
  const int P = 2 * L - 1;
  double2 acc = make_double2(0.0, 0.0);
  for (int mpp = -(L - 1); mpp <= L - 1; mpp++) {
    double2 c;
    if (b < L - 1) {
      // e^{-i pi m'' (2b+1) / P}: angle reduced exactly modulo 2P
      long long k = ((long long)mpp * (2 * b + 1)) % (2LL * P);
      if (k < 0) k += 2LL * P;
      double sn, cs;
      sincospi((double)k / (double)P, &sn, &cs);
      c = make_double2((1.0 + s) * cs / P, (-1.0 + s) * sn / P);  // e^{-ix} + s e^{ix}
    } else {
      c = make_double2(((mpp & 1) ? -1.0 : 1.0) / P, 0.0);
    }
    double2 Wv;
    if (mp >= 1) {
      const double2 w1 = quad_weight(mp - mpp, L), w2 = quad_weight(-mp - mpp, L);
      Wv = make_double2(w1.x + s * w2.x, w1.y + s * w2.y);
    } else {
      Wv = quad_weight(-mpp, L);
    }
    acc.x = fma(c.x, Wv.x, fma(-c.y, Wv.y, acc.x));
    acc.y = fma(c.x, Wv.y, fma(c.y, Wv.x, acc.y));
  }
  acc.x *= 6.283185307179586476925286766559005768;
  acc.y *= 6.283185307179586476925286766559005768;
  out[id] = (sc == 1 && mp >= 1) ? acc.y : acc.x;  // the real factor (see above)
}

struct BetaArgs {
  uint8_t* xs;           // [sig][tile][chunk][kXStage]
  double* xscale;        // [sig][tile][kM]
  const double2* W;      // row-major scratch part of signal 0, signal b at W + b * wstride (slicing input)
  double2* Wc;           // column-major scratch part of signal 0 (products' output)
  const uint8_t* tab;    // R digits: [sc][tile t][chunk kc][kAStage]
  double rscale;         // R = rscale * (digit value)
  long long wstride;
  int L, nplanes, plane0, ct, nchunk, MT, nsig;
  long long RS, PS, CS, QS;
};

// Column tile (p, sc, ct): the columns m = m_first + 2 (64 ct + j), j < 64, of
// plane p whose parity class (m + n) mod 2 is sc.
__device__ __forceinline__ int beta_first_m(int L, int n, int sc) {
  const int m = -(L - 1);
  return (((m + n) & 1) == sc) ? m : m + 1;
}

// One CTA per (signal, column tile): 128 rows c = 2 j + part (column j of the
// tile, real / imaginary part), reduction b < L; scales, then 7 digit planes
// in the stage image of beta_tc_kernel.
__global__ void __launch_bounds__(256) beta_slice_kernel(BetaArgs a) {
  __shared__ double colmax[2][kM];
  const int c = threadIdx.x & (kM - 1), half = threadIdx.x >> 7;
  const int tile = blockIdx.x, sig = blockIdx.y;
  const int ct = tile % a.ct, sc = (tile / a.ct) & 1, p = tile / (2 * a.ct);
  const int n = p - a.plane0, L = a.L, j = c >> 1, part = c & 1;
  const int m = beta_first_m(L, n, sc) + 2 * (64 * ct + j);
  const bool active = m <= L - 1 && sig < a.nsig;
  const double* src = reinterpret_cast<const double*>(a.W + (long long)sig * a.wstride + (long long)p * a.PS +
                                                      (active ? m + L - 1 : 0)) + part;
  const int nblk = a.nchunk * (kKC / 16);
  double mx = 0.0;
  for (int kb = half; kb < nblk; kb += 2)
#pragma unroll
    for (int e = 0; e < 16; e++) {
      const int bb = 16 * kb + e;
      if (active && bb < L) mx = fmax(mx, fabs(__ldg(src + 2LL * bb * a.RS)));
    }
  colmax[half][c] = mx;
  __syncthreads();
  mx = fmax(colmax[0][c], colmax[1][c]);
  int ex = 0;
  frexp(mx, &ex);
  const double scale = mx > 0.0 ? ldexp(1.0, ex + 1) : 1.0;
  const double inv = 1.0 / scale;
  const size_t gt = (size_t)sig * gridDim.x + tile;
  if (half == 0) a.xscale[gt * kM + c] = scale;
  uint8_t* out = a.xs + gt * (size_t)a.nchunk * kXStage;
  for (int kb = half; kb < nblk; kb += 2) {
    double v[16];
#pragma unroll
    for (int e = 0; e < 16; e++) {
      const int bb = 16 * kb + e;
      v[e] = (active && bb < L) ? __ldg(src + 2LL * bb * a.RS) * inv : 0.0;
    }
    uint32_t w[4][kS];
#pragma unroll
    for (int qd = 0; qd < 4; qd++) {
      double r[4];
#pragma unroll
      for (int e = 0; e < 4; e++) r[e] = v[4 * qd + e];
      split_pack4(r, w[qd]);
    }
    uint8_t* dst = out + (size_t)(kb >> 2) * kXStage + tile_off(kM, c, (kb & 3) * 16);
#pragma unroll
    for (int i = 0; i < kS; i++)
      *reinterpret_cast<uint4*>(dst + i * (kM * kKC)) = make_uint4(w[0][i], w[1][i], w[2][i], w[3][i]);
  }
}

// Single-read form (at most 512 reduction rows): one CTA per (group of 8
// consecutive columns m0 .. m0+7 of a plane, signal), i.e. 4 columns of each
// parity class, rows c = 8 (q mod 16) .. +7 of column tile q / 16 of both
// classes.  The CTA's beta samples (128-byte row segments) are read from HBM
// once into shared memory; the 16 column scales and the digits come from
// there.  Same scales and digits as beta_slice_kernel.
constexpr int kBsCols = 8;
__global__ void __launch_bounds__(256, 3) beta_slice1_kernel(BetaArgs a, int ntiles) {
  extern __shared__ __align__(16) unsigned char bsraw[];
  const int L = a.L, rows = a.nchunk * kKC, tot = rows * kBsCols;
  double2* st = reinterpret_cast<double2*>(bsraw);               // [row][kBsCols]
  double* red = reinterpret_cast<double*>(bsraw + (size_t)tot * sizeof(double2));  // [8 warps][16]
  double* scl = red + 8 * 16;                                      // [16]
  const int qpp = 16 * a.ct, q = blockIdx.x % qpp, p = blockIdx.x / qpp, sig = blockIdx.y;
  const int n = p - a.plane0, m0 = -(L - 1) + kBsCols * q;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double2* src = a.W + (long long)sig * a.wstride + (long long)p * a.PS + (m0 + L - 1);
  for (int base = 0; base < tot; base += 256 * 16) {
    double2 v[16];
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int idx = base + 256 * u + tid, r = idx >> 3, col = idx & 7;
      v[u] = (idx < tot && r < L && m0 + col <= L - 1) ? __ldg(src + (long long)r * a.RS + col) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int idx = base + 256 * u + tid;
      if (idx < tot) st[idx] = v[u];
    }
  }
  __syncthreads();
  {
    // (column, part) cp = tid % 16; rows tid / 16 + 16 i
    const int cp = tid & 15;
    const double* sd = reinterpret_cast<const double*>(st);
    double mx = 0.0;
    for (int r = tid >> 4; r < rows; r += 16) mx = fmax(mx, fabs(sd[2 * (r * kBsCols + (cp >> 1)) + (cp & 1)]));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
    if (lane < 16) red[warp * 16 + cp] = mx;
  }
  __syncthreads();
  if (tid < 16) {
    double mx = 0.0;
#pragma unroll
    for (int w = 0; w < 8; w++) mx = fmax(mx, red[w * 16 + tid]);
    int ex = 0;
    frexp(mx, &ex);
    scl[tid] = mx > 0.0 ? ldexp(1.0, ex + 1) : 1.0;
  }
  __syncthreads();
  const int nslot = rows / 16;
  for (int w = tid; w < 16 * nslot; w += 256) {
    const int cp = w & 15, kb = w >> 4, col = cp >> 1, part = cp & 1;
    const int m = m0 + col, sc = (m + n) & 1;
    const int jj = 4 * (q & 15) + (col >> 1), c = 2 * jj + part;
    const int tile = q / 16 + a.ct * (sc + 2 * p);
    const size_t gt = (size_t)sig * ntiles + tile;
    const double scale = scl[cp], inv = 1.0 / scale;
    if (kb == 0) a.xscale[gt * kM + c] = scale;
    const double* sd = reinterpret_cast<const double*>(st) + part;
    uint32_t d[4][kS];
#pragma unroll
    for (int qd = 0; qd < 4; qd++) {
      double r[4];
#pragma unroll
      for (int e = 0; e < 4; e++) r[e] = sd[2 * ((16 * kb + 4 * qd + e) * kBsCols + col)] * inv;
      split_pack4(r, d[qd]);
    }
    uint8_t* dst = a.xs + gt * (size_t)a.nchunk * kXStage + (size_t)(kb >> 2) * kXStage + tile_off(kM, c, (kb & 3) * 16);
#pragma unroll
    for (int i = 0; i < kS; i++)
      *reinterpret_cast<uint4*>(dst + i * (kM * kKC)) = make_uint4(d[0][i], d[1][i], d[2][i], d[3][i]);
  }
}

// Persistent: one CTA per SM walks the items (64-row tile t of m', column
// tile, signal), t fastest: the MT items of one column tile run on
// neighbouring CTAs at the same time, so its digits come from HBM once and
// from L2 for the other output tiles.  D_d[c, m'] over the L beta samples in
// chunks of 64, both operands streamed by bulk copies.
__global__ void __launch_bounds__(kThreads, 1) beta_tc_kernel(BetaArgs a, int ntiles, int nitems) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  TcpSmem& S = *reinterpret_cast<TcpSmem*>(smraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nk = a.nchunk, L = a.L;
  if (*reinterpret_cast<volatile int*>(&g_tc_error)) return;
  tcp_setup(S, tid, warp);
  if (warp == 0) {
    if (lane == 0) {
      int G = 0, ia = 0;
      for (int item = blockIdx.x; item < nitems; item += gridDim.x, ia++) {
        if (ia > 0) tc::mbar_wait(tc::smem_u32(&S.acce), (ia - 1) & 1, &g_tc_error, 2);
        tc::tc_fence_after();
        issue_item<false>(S, S.tmem_base, nk, G);
        tc::mma_commit(tc::smem_u32(&S.accf));
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int G = 0;
      for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int t = item % a.MT, rest = item / a.MT, tile = rest % ntiles, sig = rest / ntiles;
        const int sc = (tile / a.ct) & 1;
        const size_t gt = (size_t)sig * ntiles + tile;
        const uint8_t* xs = a.xs + gt * (size_t)nk * kXStage;
        const uint8_t* tb = a.tab + (size_t)(sc * a.MT + t) * nk * kAStage;
        for (int k = 0; k < nk; k++) load_chunk(S, G, xs + (size_t)k * kXStage, tb + (size_t)k * kAStage);
      }
    }
  } else {
    const int gw = warp - 2, lq = warp & 3, ch = gw >> 2;
    const int c = 32 * lq + lane, j = c >> 1, part = c & 1;
    int ia = 0;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      const int t = item % a.MT, rest = item / a.MT, tile = rest % ntiles, sig = rest / ntiles;
      const int ct = tile % a.ct, sc = (tile / a.ct) & 1, p = tile / (2 * a.ct);
      const int n = p - a.plane0, r0 = t * kN;
      const int m = beta_first_m(L, n, sc) + 2 * (64 * ct + j);
      const bool active = m <= L - 1 && sig < a.nsig;
      const size_t gt = (size_t)sig * ntiles + tile;
      const double scale = a.xscale[gt * kM + c];
      double v[4][8];
      drain_item(S, lq, ch, a.rscale * 0.000061035156250000000, a.nchunk * kKC <= 512, ia, v);  // R scale x 2^{-14}
      double2* out = a.Wc + (long long)sig * a.wstride + (long long)p * a.QS + (long long)(m + L - 1) * a.CS;
#pragma unroll
      for (int g = 0; g < 4; g++) {
        const int col = 32 * ch + 8 * g;
        double re[4], im[4];
#pragma unroll
        for (int qq = 0; qq < 4; qq++) {
          const double send = (part ? v[g][qq] : v[g][4 + qq]) * scale;
          const double recv = __shfl_xor_sync(0xffffffffu, send, 1);
          re[qq] = part ? recv : v[g][qq] * scale;
          im[qq] = part ? v[g][4 + qq] * scale : recv;
        }
        if (!active) continue;
#pragma unroll
        for (int qq = 0; qq < 4; qq++) {
          const int row = r0 + col + 4 * part + qq;
          if (row >= L) continue;
          double2 val = make_double2(re[qq], im[qq]);
          if (sc == 1 && row >= 1) val = make_double2(-val.y, val.x);  // times i
          out[row] = val;
        }
      }
    }
  }
  tcp_teardown(S, warp);
}

// ---------------------------------------------------------------- ragged batches
// Split-precision contractions of signals with different parameters (L, N,
// L0, storage, n-order, n-mode) in one launch.  The Delta products A[m', l] =
// Delta^l_{m' mu} Delta^l_{m' nu} do not depend on L or N, so signals of
// different geometry share the tensor-core tiles: the host sorts the signals
// by (recursion, L, N) and cuts them into groups of 16 (one M = 128 operand);
// a group runs at its largest L and N, each signal's columns are zero past its
// own L, N (and below its L0) and its outputs are written in its own layout.
// Work items of all groups form one 1-D grid; A comes from a resident digit
// table when one covers the groups' band limits (the digits do not depend on
// L or N), else the producer warps generate it from the FP64 Delta table.
struct SigDesc {
  const double2* flmn;    // inverse: coefficients in; forward: coefficients out
  double2* Wc;            // column-major scratch part: inverse output, forward input
  const long long* base;  // block bases of the signal's parameters
  long long CS, QS;       // its column-major strides
  int L, N, L0, plane0, n_mode, compact;
};
struct GroupDesc {
  long long xs_off;  // byte offset of the group's stage images [pair][chunk][kXStage]
  long long sc_off;  // offset (doubles) of its column scales [pair][kM]
  int Lg, Ng, nc;    // largest L and N of the group, reduction chunks
  int sig0, nsig;    // first signal (index into the descriptors) and count (<= 16)
  int item0, slice0;  // first tensor-core item and first slicing block of the group
};
struct RagArgs {
  uint8_t* xs;
  double* xscale;
  const SigDesc* sigs;
  const GroupDesc* groups;
  const double* dl;
  int ngroups;
  // resident digit table (null: generate A from dl): blocks of pair (mu, nu)
  // from pair_off[mu * tab_N + nu], tab_nc chunks (every group has L <= tab_L
  // and N <= tab_N, so its blocks are the table's)
  const uint8_t* tab;
  const long long* pair_off;
  int tab_N, tab_nc;
};

// Group of a 1-D block index (prefix offsets item0 or slice0, ascending).
template <bool ITEMS>
__device__ __forceinline__ int ragged_group(const RagArgs& a, int x) {
  int g = 0;
  while (g + 1 < a.ngroups && (ITEMS ? a.groups[g + 1].item0 : a.groups[g + 1].slice0) <= x) g++;
  return g;
}

// Inverse slicing of a ragged group: block (slot b, nu, block of kMuPer mu),
// the same two passes as slice_inv_kernel, columns read in the signal's own
// layout and written into the group's stage images.
__global__ void __launch_bounds__(256, 3) ragged_slice_inv_kernel(RagArgs a) {
  __shared__ double wmax[8][2 * 4 * kMuPer];
  __shared__ double scl[kMuPer][2 * 4];
  const int gi = ragged_group<false>(a, blockIdx.x);
  const GroupDesc G = a.groups[gi];
  const int local = blockIdx.x - G.slice0;
  const int b = local % kSig, rest = local / kSig;
  const int nu = rest % G.Ng, mu0 = (rest / G.Ng) * kMuPer;
  const int Lp = G.nc * kKC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  SigDesc sd{};
  const bool has = b < G.nsig;
  if (has) sd = a.sigs[G.sig0 + b];
  // column of slot b for (mu, nu, combo), in the signal's own layout
  auto column = [&](int mu, int combo) {
    InvColumn c;
    const int ms = (combo & 1) ? -1 : 1, ns = (combo & 2) ? -1 : 1;
    const int m = ms * mu, n = ns * nu;
    c.act = has && mu < sd.L && nu < sd.N && !(ms < 0 && mu == 0) && !(ns < 0 && nu == 0) &&
            !plane_skipped(sd.n_mode, sd.N, n);
    c.lmin = max(max(mu, nu), sd.L0);
    c.flip = ms * ns < 0;
    c.src = c.act ? sd.flmn + sd.base[sd.plane0 + n] + m : nullptr;
    c.gsrc = nullptr;
    return c;
  };
  const int Ls = has ? sd.L : 0;
  {
    const int j = threadIdx.x % kMuPer, combo = (threadIdx.x / kMuPer) & 3, l0 = threadIdx.x / (4 * kMuPer);
    constexpr int LSTEP = 256 / (4 * kMuPer);
    const InvColumn col = column(mu0 + j, combo);
    double mr = 0.0, mi = 0.0;
    if (col.act) {
      for (int l1 = l0; l1 < Ls; l1 += LSTEP * 8) {
        double2 x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) x[u] = inv_value(col, Ls, l1 + LSTEP * u);
#pragma unroll
        for (int u = 0; u < 8; u++) {
          mr = fmax(mr, fabs(x[u].x));
          mi = fmax(mi, fabs(x[u].y));
        }
      }
    }
    mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, 16));
    mi = fmax(mi, __shfl_xor_sync(0xffffffffu, mi, 16));
    if (lane < 16) {
      wmax[warp][2 * (j * 4 + combo)] = mr;
      wmax[warp][2 * (j * 4 + combo) + 1] = mi;
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * 4 * kMuPer) {
    double mx = 0.0;
#pragma unroll
    for (int w = 0; w < 8; w++) mx = fmax(mx, wmax[w][threadIdx.x]);
    const int jc = threadIdx.x >> 1, part = threadIdx.x & 1;
    scl[jc >> 2][2 * (jc & 3) + part] = scale_of(mx);
  }
  __syncthreads();
  for (int j = 0; j < kMuPer; j++) {
    const int mu = mu0 + j;
    if (mu >= G.Lg) break;
    const long long gp = (long long)mu * G.Ng + nu;
    if (threadIdx.x < 8) a.xscale[G.sc_off + gp * kM + 8 * b + threadIdx.x] = scl[j][threadIdx.x];
  }
  for (int w = threadIdx.x; w < kMuPer * 8 * (Lp / 16); w += blockDim.x) {
    const int c = w & 7, j = (w >> 3) % kMuPer, kb = w / (8 * kMuPer);
    const int mu = mu0 + j;
    if (mu >= G.Lg) continue;
    // chunks below the one holding l = max(mu, nu) are never read (ragged_tc_kernel)
    if (16 * kb / kKC < max(mu, nu) / kKC) continue;
    const int combo = c >> 1, part = c & 1;
    const double inv = 1.0 / scl[j][c];
    const InvColumn col = column(mu, combo);
    uint32_t d[4][kS];
#pragma unroll
    for (int qd = 0; qd < 4; qd++) {
      double r[4];
#pragma unroll
      for (int e = 0; e < 4; e++) r[e] = inv_entry(col, Ls, 16 * kb + 4 * qd + e, part) * inv;
      split_pack4(r, d[qd]);
    }
    const long long gp = (long long)mu * G.Ng + nu;
    uint8_t* dst = a.xs + G.xs_off + gp * (long long)G.nc * kXStage + (long long)(kb >> 2) * kXStage +
                   tile_off(kM, 8 * b + c, (kb & 3) * 16);
#pragma unroll
    for (int i = 0; i < kS; i++)
      *reinterpret_cast<uint4*>(dst + i * (kM * kKC)) = make_uint4(d[0][i], d[1][i], d[2][i], d[3][i]);
  }
}

// Forward slicing of a ragged group: block (pair, set q4 of kSigPer slots),
// as slice_fwd_kernel, columns read from each signal's own column-major part.
__global__ void __launch_bounds__(256) ragged_slice_fwd_kernel(RagArgs a) {
  __shared__ double scl[2 * kSliceCols];
  const int gi = ragged_group<false>(a, blockIdx.x);
  const GroupDesc G = a.groups[gi];
  const int local = blockIdx.x - G.slice0;
  const int npairs = G.Lg * G.Ng;
  const int pair = local % npairs, q4 = local / npairs;  // q4 < kSig / kSigPer
  const int nu = pair % G.Ng, mu = pair / G.Ng;
  const int Lp = G.nc * kKC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // complex column cc (slot kSigPer q4 + cc / 4, combo cc % 4)
  auto column = [&](int cc, int* Ls) {
    FwdColumn c;
    const int b = kSigPer * q4 + (cc >> 2), combo = cc & 3;
    const int ms = (combo & 1) ? -1 : 1, ns = (combo & 2) ? -1 : 1;
    const int m = ms * mu, n = ns * nu;
    c.act = false;
    c.flip = ms * ns < 0;
    c.src = nullptr;
    *Ls = 0;
    if (b < G.nsig) {
      const SigDesc& sd = a.sigs[G.sig0 + b];
      c.act = mu < sd.L && nu < sd.N && !(ms < 0 && mu == 0) && !(ns < 0 && nu == 0) &&
              !plane_skipped(sd.n_mode, sd.N, n);
      if (c.act) c.src = sd.Wc + (long long)(sd.plane0 + n) * sd.QS + (long long)(m + sd.L - 1) * sd.CS;
      *Ls = sd.L;
    }
    return c;
  };
  for (int cc = warp; cc < kSliceCols; cc += 8) {
    int Ls;
    const FwdColumn col = column(cc, &Ls);
    double mr = 0.0, mi = 0.0;
    if (col.act) {
      for (int k1 = lane; k1 < Ls; k1 += 32 * 8) {
        double2 x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int k = k1 + 32 * u;
          x[u] = k < Ls ? __ldg(col.src + k) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          mr = fmax(mr, fabs(x[u].x));
          mi = fmax(mi, fabs(x[u].y));
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
      mi = fmax(mi, __shfl_xor_sync(0xffffffffu, mi, o));
    }
    if (lane == 0) scl[2 * cc] = scale_of(mr), scl[2 * cc + 1] = scale_of(mi);
  }
  __syncthreads();
  if (threadIdx.x < 2 * kSliceCols)
    a.xscale[G.sc_off + (long long)pair * kM + 2 * kSliceCols * q4 + threadIdx.x] = scl[threadIdx.x];
  uint8_t* pb = a.xs + G.xs_off + (long long)pair * G.nc * kXStage;
  const int c_base = 2 * kSliceCols * q4, nblk = Lp / 16;
  for (int w = threadIdx.x; w < 2 * kSliceCols * nblk; w += blockDim.x) {
    const int c = w % (2 * kSliceCols), kb = w / (2 * kSliceCols), cc = c >> 1, part = c & 1;
    int Ls;
    const FwdColumn col = column(cc, &Ls);
    const double inv = 1.0 / scl[c];
    const double* src = reinterpret_cast<const double*>(col.src) + part;
    uint32_t d[4][kS];
#pragma unroll
    for (int qd = 0; qd < 4; qd++) {
      double r[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int k = 16 * kb + 4 * qd + e;
        double x = (col.act && k < Ls) ? __ldg(src + 2 * k) : 0.0;
        if (col.flip && (k & 1)) x = -x;
        r[e] = x * inv;
      }
      split_pack4(r, d[qd]);
    }
    uint8_t* dst = pb + (long long)(kb >> 2) * kXStage + tile_off(kM, c_base + c, (kb & 3) * 16);
#pragma unroll
    for (int i = 0; i < kS; i++)
      *reinterpret_cast<uint4*>(dst + i * (kM * kKC)) = make_uint4(d[0][i], d[1][i], d[2][i], d[3][i]);
  }
}

// Tensor-core products of a ragged batch: one CTA per item (group, mu, tile,
// nu); A streamed from the covering digit table (TAB) or generated from Delta
// by the producer warps as mixed_tc_kernel does; outputs in each signal's own
// layout.
template <bool FWD, bool TAB>
__global__ void __launch_bounds__(kThreads, 1) ragged_tc_kernel(RagArgs ra) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(smraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gi = ragged_group<true>(ra, blockIdx.x);
  const GroupDesc G = ra.groups[gi];
  const int MT = G.nc;
  const int local = blockIdx.x - G.item0;
  const int nu = local % G.Ng, rest = local / G.Ng;
  const int t = rest % MT, mu = rest / MT;
  const int L = G.Lg, r0 = t * kN;
  const int lmin = max(mu, nu);  // the signals' own L0 zero their columns / outputs
  MixArgs a{};
  a.dl = ra.dl;
  a.L = L;
  a.N = G.Ng;
  int kc0, nk;
  if (FWD) {
    const bool any_row = r0 + kN > lmin && r0 < L;
    kc0 = 0;
    nk = any_row ? (min(L, r0 + kN) + kKC - 1) / kKC : 0;
  } else {
    const int kstart = max(lmin, r0) & ~(kKC - 1);
    kc0 = kstart / kKC;
    nk = kstart < L ? (L - kstart + kKC - 1) / kKC : 0;
  }
  const long long gp = (long long)mu * G.Ng + nu;
  const uint8_t* xs = ra.xs + G.xs_off + gp * (long long)G.nc * kXStage;
  if (*reinterpret_cast<volatile int*>(&g_tc_error)) return;

  const uint32_t full0 = tc::smem_u32(&S.full[0]), empty0 = tc::smem_u32(&S.empty[0]);
  const uint32_t accum = tc::smem_u32(&S.accum);
  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      tc::mbar_init(full0 + 8 * s, TAB ? 1 : kGen + 1);
      tc::mbar_init(empty0 + 8 * s, 1);
    }
    tc::mbar_init(accum, 1);
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&S.tmem_base), kTmemCols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tbase = S.tmem_base;

  if (warp == 0) {
    if (lane == 0 && nk > 0) {
      // table blocks are stored rows m', reduction l; the forward reads them
      // transposed as an MN-major operand
      constexpr uint32_t idesc = tc::idesc_s8(kM, kN) | ((FWD && TAB) ? (1u << 16) : 0u);
      for (int k = 0; k < nk; k++) {
        const int s = k & 1;
        tc::mbar_wait(full0 + 8 * s, (k >> 1) & 1, &g_tc_error, 2);
        tc::tc_fence_after();
        const uint32_t xb = tc::smem_u32(&S.X[s][0]), ab = tc::smem_u32(&S.A[s][0]);
#pragma unroll
        for (int ks = 0; ks < kKC / 32; ks++) {
#pragma unroll
          for (int i = 0; i < kS; i++) {
            const uint64_t ad = tc::smem_desc(xb + i * (kM * kKC) + ks * 2 * (kM * 16), kM * 16, 128);
            if constexpr (FWD && TAB) {
#pragma unroll
              for (int j = 0; j + i < kND; j++) {
                const uint64_t bd = tc::smem_desc(ab + j * (kN * kKC) + ks * 2048, 512, 128);
                tc::mma_i8(tbase + (uint32_t)(kN * (i + j)), ad, bd, idesc, (k | ks | i) != 0);
              }
            } else {
              // K-major A operand: digits j0 .. j0+3 stacked along N (see issue_item)
#pragma unroll
              for (int j0 = 0; j0 + i < kND; j0 += 4) {
                const int nj = (kND - i - j0) < 4 ? (kND - i - j0) : 4;
                const uint64_t bd = tc::smem_desc(ab + j0 * (kN * kKC) + ks * 256, 128, 512);
                tc::mma_i8(tbase + (uint32_t)(kN * (i + j0)), ad, bd, tc::idesc_s8(kM, kN * nj), (k | ks | i) != 0);
              }
            }
          }
        }
        tc::mma_commit(empty0 + 8 * s);
      }
      tc::mma_commit(accum);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const int q = max(mu, nu) / kKC;
      const uint8_t* tb = TAB ? ra.tab + (long long)ra.pair_off[(long long)mu * ra.tab_N + nu] * kAStage : nullptr;
      for (int k = 0; k < nk; k++) {
        const int s = k & 1;
        if (k >= kStages) tc::mbar_wait(empty0 + 8 * s, ((k >> 1) - 1) & 1, &g_tc_error, 2);
        tc::mbar_arrive_expect_tx(full0 + 8 * s, TAB ? kXStage + kAStage : kXStage);
        tc::bulk_g2s(tc::smem_u32(&S.X[s][0]), xs + (long long)(kc0 + k) * kXStage, kXStage, full0 + 8 * s);
        if (TAB) {
          const long long blk = FWD ? digit_block(k, t, q, ra.tab_nc) : digit_block(t, kc0 + k, q, ra.tab_nc);
          tc::bulk_g2s(tc::smem_u32(&S.A[s][0]), tb + blk * kAStage, kAStage, full0 + 8 * s);
        }
      }
    }
  } else {
    const int gw = warp - 2;
    double xa[4][4], xb[4][4];
    if (!TAB && nk > 0) gen_load<FWD>(a, mu, nu, lmin, r0, kc0 * kKC, gw, lane, xa);
    for (int k = 0; k < (TAB ? 0 : nk); k += 2) {
      if (k + 1 < nk) gen_load<FWD>(a, mu, nu, lmin, r0, (kc0 + k + 1) * kKC, gw, lane, xb);
      if (k >= kStages) tc::mbar_wait(empty0, ((k >> 1) - 1) & 1, &g_tc_error, 2);
      gen_store(&S.A[0][0], gw, lane, xa);
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(full0);
      if (k + 1 >= nk) break;
      if (k + 2 < nk) gen_load<FWD>(a, mu, nu, lmin, r0, (kc0 + k + 2) * kKC, gw, lane, xa);
      if (k + 1 >= kStages) tc::mbar_wait(empty0 + 8, (((k + 1) >> 1) - 1) & 1, &g_tc_error, 2);
      gen_store(&S.A[1][0], gw, lane, xb);
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(full0 + 8);
    }

    // epilogue: thread <-> TMEM lane c (signal column), 32 output rows
    const int lq = warp & 3, ch = gw >> 2;
    const int c = 32 * lq + lane;
    const int b = c >> 3, combo = (c >> 1) & 3, part = c & 1;
    const int ms = (combo & 1) ? -1 : 1, ns = (combo & 2) ? -1 : 1;
    const int m = ms * mu, n = ns * nu;
    const bool one_neg = ms * ns < 0;
    const double sgn_mn = ((mu + nu) & 1) ? -1.0 : 1.0;
    const double scale = ra.xscale[G.sc_off + gp * kM + c];
    bool live = b < G.nsig && !((ms < 0 && mu == 0) || (ns < 0 && nu == 0));
    SigDesc sd{};
    if (live) {
      sd = ra.sigs[G.sig0 + b];
      live = mu < sd.L && nu < sd.N && !(FWD && plane_skipped(sd.n_mode, sd.N, n));
    }
    if (nk > 0) {
      tc::mbar_wait(accum, 0, &g_tc_error, 2);
      tc::tc_fence_after();
    }
    double2* Wout = nullptr;
    double2* F = nullptr;
    long long blk = 0;
    if (live) {
      if (!FWD) {
        Wout = sd.Wc + (long long)(sd.plane0 + n) * sd.QS + (long long)(m + sd.L - 1) * sd.CS;
      } else {
        F = const_cast<double2*>(sd.flmn);
        blk = sd.base[sd.plane0 + n];
      }
    }
    const int lmin_s = max(lmin, sd.L0);
#pragma unroll 1
    for (int g = 0; g < 4; g++) {
      __syncwarp();
      const int col = 32 * ch + 8 * g;
      double v[8];
#pragma unroll
      for (int e = 0; e < 8; e++) v[e] = 0.0;
      if (nk > 0) {
        int acc[kND][8];
#pragma unroll
        for (int d = 0; d < kND; d++)
          tc::tmem_ld8(tbase + ((uint32_t)(32 * lq) << 16) + (uint32_t)(kN * d + col), acc[d]);
        tc::tmem_wait_ld();
        double wd = 2.0 * 0.000061035156250000000;  // A scale 2, diagonal 0: 2^{-14}
#pragma unroll
        for (int d = 0; d < kND; d++) {
#pragma unroll
          for (int e = 0; e < 8; e++) v[e] = fma(int_to_double(acc[d][e]), wd, v[e]);
          wd *= 0.0078125;
        }
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] *= scale;
      }
      double re[4], im[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const double send = part ? v[q] : v[4 + q];
        const double recv = __shfl_xor_sync(0xffffffffu, send, 1);
        re[q] = part ? recv : v[q];
        im[q] = part ? v[4 + q] : recv;
      }
      if (!live) continue;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int row = r0 + col + 4 * part + q;
        if (row >= sd.L) continue;
        const double s = (one_neg && (row & 1)) ? -sgn_mn : sgn_mn;
        double2 val = make_double2(re[q] * s, im[q] * s);
        if (!FWD) {
          Wout[row] = ipow(val, n - m + 4 * sd.L);
        } else {
          const int lr = row;
          if (mu > lr) continue;
          if (sd.compact && lr < nu) continue;  // not stored
          if (lr < lmin_s) val = make_double2(0.0, 0.0);
          else val = ipow(val, m - n + 4 * sd.L);
          F[blk + (long long)lr * lr + lr + m] = val;
        }
      }
    }
  }

  if (warp == 0 && lane == 0 && nk > 0) tc::mbar_wait(accum, 0, &g_tc_error, 2);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc::tc_fence_after();
    tc::tmem_dealloc(tbase, kTmemCols);
  }
}

}  // namespace

// ---------------------------------------------------------------- host side
static int nchunks(const Geometry& g) { return (g.L + kKC - 1) / kKC; }

static size_t beta_scratch_bytes(const Geometry& g, int nsig);
bool mixed_beta_supported(const Geometry& g);

// Sliced operands of the contractions and of the forward beta products (the
// two never live at the same time, so they share one region).
// The single-read slicing kernels (inv_colscale + inv_digit, beta_slice1) are
// the default; SO3GPU_STREAM_SLICE=0 selects the per-pair kernels
// (slice_inv_kernel, beta_slice_kernel), which write the same digits.
static bool stream_slicing() {
  const char* e = getenv("SO3GPU_STREAM_SLICE");
  return !(e && e[0] == '0');
}

// Column scales of the streaming inverse slicing: [signal][plane][2L-1][part].
static size_t colscale_bytes(const Geometry& g, int nsig) {
  return (size_t)nsig * (g.real ? g.N : 2 * g.N - 1) * (2 * (size_t)g.L - 1) * 2 * sizeof(double);
}

size_t mixed_scratch_bytes(const Geometry& g, int nsig) {
  const size_t groups = (nsig + kSig - 1) / kSig, pairs = (size_t)g.L * g.N;
  const size_t contr = ((groups * pairs * nchunks(g) * (size_t)kXStage + 255) & ~size_t(255)) +
                       ((groups * pairs * kM * sizeof(double) + 255) & ~size_t(255)) + colscale_bytes(g, nsig) + 256;
  return mixed_beta_supported(g) ? std::max(contr, beta_scratch_bytes(g, nsig)) : contr;
}

static int mixed_args(const Geometry& g, int n_mode, int nsig, void* scratch, MixArgs* m, SliceArgs* s) {
  const int nc = nchunks(g), MT = nc;  // output tiles of 64 rows = reduction chunks of 64
  const size_t groups = (nsig + kSig - 1) / kSig, pairs = (size_t)g.L * g.N;
  if (pairs * MT > 0x7fffffffu || groups > 65535) return fail(kUnsupported, "split-precision grid too large");
  uint8_t* xs = static_cast<uint8_t*>(scratch);
  double* xscale = reinterpret_cast<double*>(xs + ((groups * pairs * nc * (size_t)kXStage + 255) & ~size_t(255)));
  *m = MixArgs{};
  m->xs = xs;
  m->xscale = xscale;
  m->L = g.L, m->N = g.N, m->L0 = g.L0, m->nchunk = nc, m->MT = MT, m->plane0 = g.plane0, m->n_mode = n_mode;
  m->nsig = nsig, m->CS = g.CS, m->QS = g.QS, m->real = g.real;
  *s = SliceArgs{};
  s->xs = xs;
  s->xscale = xscale;
  s->L = g.L, s->N = g.N, s->L0 = g.L0, s->nchunk = nc, s->plane0 = g.plane0, s->n_mode = n_mode;
  s->nsig = nsig, s->npairs = (int)pairs, s->CS = g.CS, s->QS = g.QS, s->real = g.real;
  return kOk;
}

size_t digit_table_bytes(int L, int N) {
  const int nc = (L + kKC - 1) / kKC;
  size_t blocks = 0;
  for (int mu = 0; mu < L; mu++)
    for (int nu = 0; nu < N; nu++) blocks += (size_t)digit_blocks(std::max(mu, nu) / kKC, nc);
  return blocks * kAStage;
}

// Resident digit tables, one per (L, N, Delta recursion), built on the
// second split-precision call of that geometry (a geometry seen once, as in a
// request trace of varied band limits, never pays for a table) when it fits:
// at most a quarter of the device memory in total and 4 GiB of free memory
// left after it (SO3GPU_DIGIT_TABLE=0 disables them, =1 builds on first
// use).  Tables are kept until the process exits, so streams that use one
// never see it change.  Without a table the kernels generate the digits from
// Delta.
int ensure_digit_table(Device* D, const Geometry& g, int method, const double* dl, cudaStream_t s,
                       const DigitTable** out, bool force) {
  *out = nullptr;
  const char* env = getenv("SO3GPU_DIGIT_TABLE");
  if (env && env[0] == '0') return kOk;
  std::lock_guard<std::mutex> lk(D->mu);
  for (const auto& t : D->digit_tables)
    if (t->L == g.L && t->N == g.N && t->method == method) {
      *out = t.get();
      return kOk;
    }
  // the build reads the Delta planes l < g.L: only from the device's current
  // table of this recursion, and only if it holds them (else generate)
  if (D->dl[method].d != dl || D->dl[method].Lcap < g.L) return kOk;
  const long long key = ((long long)g.L << 20) ^ ((long long)g.N << 2) ^ method;
  if (++D->digit_uses[key] < 2 && !(env && env[0] == '1') && !force) return kOk;
  const size_t bytes = digit_table_bytes(g.L, g.N);
  size_t used = 0;
  for (const auto& t : D->digit_tables) used += t->bytes;
  size_t freeb = 0, total = 0;
  SO3G_CUDA(cudaMemGetInfo(&freeb, &total));
  if (used + bytes > total / 4 || freeb < bytes + (size_t(4) << 30)) return kOk;  // generate instead
  const int nc = (g.L + kKC - 1) / kKC;
  std::vector<long long> off((size_t)g.L * g.N);
  long long acc = 0;
  for (int mu = 0; mu < g.L; mu++)
    for (int nu = 0; nu < g.N; nu++) {
      off[(size_t)mu * g.N + nu] = acc;
      acc += digit_blocks(std::max(mu, nu) / kKC, nc);
    }
  auto t = std::make_unique<DigitTable>();
  t->L = g.L, t->N = g.N, t->method = method, t->bytes = bytes;
  SO3G_CUDA(cudaMalloc(&t->d, bytes));
  if (cudaMalloc(&t->pair_off, off.size() * sizeof(long long)) != cudaSuccess) {
    cudaFree(t->d);
    return fail(kCudaError, "digit table offsets: cudaMalloc failed");
  }
  SO3G_CUDA(cudaMemcpyAsync(t->pair_off, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice, s));
  MixArgs a{};
  a.dl = dl, a.pair_off = t->pair_off, a.L = g.L, a.N = g.N, a.nchunk = nc;
  digit_table_kernel<<<(unsigned)(g.L * g.N), 256, 0, s>>>(a, t->d);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  SO3G_CUDA(cudaStreamSynchronize(s));  // offsets upload complete before the host vector goes
  *out = t.get();
  D->digit_tables.push_back(std::move(t));
  return kOk;
}

// A resident digit table whose (L, N) cover (L, N) for this recursion, for
// the ragged contractions (digits do not depend on the band limits); with
// build, the L = 512, N = 64 table is built when none covers and (L, N) fit
// it (same memory rule as ensure_digit_table).  Null: generate from Delta.
const DigitTable* covering_digit_table(Device* D, int L, int N, int method, const double* dl, bool build,
                                       cudaStream_t s) {
  {
    std::lock_guard<std::mutex> lk(D->mu);
    for (const auto& t : D->digit_tables)
      if (t->method == method && t->L >= L && t->N >= N) return t.get();
  }
  const char* env = getenv("SO3GPU_DIGIT_TABLE");
  if (!build || L > 512 || N > 64 || (env && env[0] == '0')) return nullptr;
  Geometry g{};
  g.L = 512, g.N = 64;
  const DigitTable* t = nullptr;
  // built now, not on a geometry's second request as ensure_digit_table
  // would: the ragged path has no per-geometry history.  The build needs the
  // Delta planes up to l = 511; with a smaller resident Delta table
  // (ensure_digit_table checks) the products generate A from Delta instead.
  const int rc = ensure_digit_table(D, g, method, dl, s, &t, true);
  return rc == kOk ? t : nullptr;
}

// Streaming multiprocessors of the current device (persistent grids).
static int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      n <= 0)
    return 148;
  return n;
}

template <bool FWD>
static int launch_tc(const MixArgs& m, int nsig, cudaStream_t s) {
  const dim3 grid((unsigned)(m.L * m.N * m.MT), (nsig + kSig - 1) / kSig);
  const int smem = (int)sizeof(TcSmem);
  if (m.tab) {
    const int psmem = (int)sizeof(TcpSmem);
    const long long items = mixed_items(m.L, m.N, m.MT, (int)grid.y, FWD);
    if (items > 0x7fffffffLL) return fail(kUnsupported, "split-precision contraction: too many work items");
    SO3G_CUDA(cudaFuncSetAttribute(mixed_tcp_kernel<FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem));
    mixed_tcp_kernel<FWD><<<(int)std::min<long long>(items, sm_count()), kThreads, psmem, s>>>(m, (int)items);
  } else {
    SO3G_CUDA(cudaFuncSetAttribute(mixed_tc_kernel<FWD, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    mixed_tc_kernel<FWD, false><<<grid, kThreads, smem, s>>>(m);
  }
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

int launch_mixed_inverse(const Geometry& g, int n_mode, const double2* const* flmn_dev, int nsig,
                         const long long* bases, const double* dl, const DigitTable* tab, double2* W,
                         long long wstride, void* scratch, cudaStream_t s, const double2* conv_flm,
                         const double2* const* conv_glm) {
  if (g.real && conv_flm) return fail(kUnsupported, "split-precision convolution: complex signals only");
  MixArgs m;
  SliceArgs sa;
  if (int rc = mixed_args(g, n_mode, nsig, scratch, &m, &sa)) return rc;
  sa.flmn = flmn_dev;
  sa.base = bases;
  sa.flm = conv_flm;
  sa.glm = conv_glm;
  if (!conv_flm && g.L <= 1024 && nsig <= 65535 && stream_slicing()) {
    // streaming slicing: column scales, then digits, reading the coefficients in storage order
    const int nplanes = g.real ? g.N : 2 * g.N - 1, ncol = 2 * g.L - 1;
    const size_t groups = (nsig + kSig - 1) / kSig;
    double* colscl = reinterpret_cast<double*>(
        reinterpret_cast<char*>(sa.xscale) + ((groups * (size_t)sa.npairs * kM * sizeof(double) + 255) & ~size_t(255)));
    const dim3 g1((unsigned)nplanes, (unsigned)nsig);
    if (ncol <= kStreamThreads)
      inv_colscale_kernel<1><<<g1, kStreamThreads, 0, s>>>(sa, colscl, nplanes);
    else if (ncol <= 2 * kStreamThreads)
      inv_colscale_kernel<2><<<g1, kStreamThreads, 0, s>>>(sa, colscl, nplanes);
    else if (ncol <= 4 * kStreamThreads)
      inv_colscale_kernel<4><<<g1, kStreamThreads, 0, s>>>(sa, colscl, nplanes);
    else
      inv_colscale_kernel<8><<<g1, kStreamThreads, 0, s>>>(sa, colscl, nplanes);
    SO3G_LAUNCHED();
    SO3G_CUDA(cudaGetLastError());
    inv_digit_kernel<<<dim3((unsigned)(4 * sa.nchunk), (unsigned)g.N, (unsigned)nsig), kStreamThreads, 0, s>>>(
        sa, colscl, nplanes);
    SO3G_LAUNCHED();
    SO3G_CUDA(cudaGetLastError());
  } else {
    // every signal of the last group (zeros past nsig), so the group's stage images are complete
    slice_inv_kernel<<<dim3((unsigned)(g.N * ((g.L + kMuPer - 1) / kMuPer)),
                        (unsigned)(((nsig + kSig - 1) / kSig) * kSig)),
                       256, 0, s>>>(sa);
    SO3G_LAUNCHED();
    SO3G_CUDA(cudaGetLastError());
  }
  m.dl = dl;
  m.base = bases;
  m.W = W + g.QOFF;
  m.wstride = wstride;
  if (tab) m.tab = tab->d, m.pair_off = tab->pair_off;
  return launch_tc<false>(m, nsig, s);
}

int launch_mixed_forward(const Geometry& g, int n_mode, const double2* W, long long wstride, int nsig,
                         const long long* bases, const double* dl, const DigitTable* tab, double2* const* flmn_dev,
                         int storage_compact, void* scratch, cudaStream_t s) {
  MixArgs m;
  SliceArgs sa;
  if (int rc = mixed_args(g, n_mode, nsig, scratch, &m, &sa)) return rc;
  sa.W = W + g.QOFF;
  sa.wstride = wstride;
  sa.base = bases;
  slice_fwd_kernel<<<dim3((unsigned)sa.npairs, (unsigned)(((nsig + kSig - 1) / kSig) * (kSig / kSigPer))), 256, 0,
                     s>>>(sa);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  m.dl = dl;
  m.base = bases;
  m.flmn = flmn_dev;
  m.compact = storage_compact;
  if (tab) m.tab = tab->d, m.pair_off = tab->pair_off;
  return launch_tc<true>(m, nsig, s);
}

// ---------------------------------------------------------------- forward beta (host)
static int beta_tiles(const Geometry& g, int* ct) {
  *ct = (g.L + 63) / 64;  // column tiles per parity class (a class holds at most L columns)
  return g.nplanes * 2 * *ct;
}

static size_t beta_scratch_bytes(const Geometry& g, int nsig) {
  int ct = 0;
  const size_t tiles = beta_tiles(g, &ct);
  return (size_t)nsig * tiles * ((size_t)nchunks(g) * kXStage + kM * sizeof(double)) + 256;
}

bool mixed_beta_supported(const Geometry& g) { return g.mw && !g.real && g.nb == g.L; }

// The 7 digits of r in [-1/2, 1/2] (host copy of split_pack4's rule).
static void split_host(double r, uint8_t* q) {
  const long long v = (long long)std::nearbyint(r * 562949953421312.0);
  const unsigned long long u = (unsigned long long)(v + kDigitOffset);
  for (int i = 0; i < kS; i++) {
    const int d = (int)((u >> (7 * (kS - 1 - i))) & (i == 0 ? 255u : 127u));
    q[i] = (uint8_t)((d - 64) & 255);
  }
}

// Resident digits of R_s for this L (MW), one table per device and L, built
// on the second split-precision forward call of that L (the first runs the
// FP64 beta stage, so a band limit seen once never pays for the build);
// SO3GPU_DIGIT_TABLE=1 builds on first use.
int ensure_beta_table(Device* D, const Geometry& g, cudaStream_t s, const BetaTable** out) {
  *out = nullptr;
  std::lock_guard<std::mutex> lk(D->mu);
  for (const auto& t : D->beta_tables)
    if (t->L == g.L) {
      *out = t.get();
      return kOk;
    }
  const char* env = getenv("SO3GPU_DIGIT_TABLE");
  if (++D->beta_uses[g.L] < 2 && !(env && env[0] == '1')) return kOk;
  const int L = g.L, nc = nchunks(g), MT = nc;
  double* dR = nullptr;
  SO3G_CUDA(cudaMalloc(&dR, 2 * (size_t)L * L * sizeof(double)));
  beta_matrix_kernel<<<(unsigned)((2LL * L * L + 255) / 256), 256, 0, s>>>(L, dR);
  SO3G_LAUNCHED();
  std::vector<double> R(2 * (size_t)L * L);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(R.data(), dR, R.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dR);
  if (e != cudaSuccess) return fail(kCudaError, std::string("beta matrix: ") + cudaGetErrorString(e));
  double mx = 0.0;
  for (double v : R) mx = std::max(mx, std::fabs(v));
  int ex = 0;
  std::frexp(mx, &ex);
  const double rscale = mx > 0.0 ? std::ldexp(1.0, ex + 1) : 1.0;  // |R / rscale| < 1/2
  const size_t bytes = (size_t)2 * MT * nc * kAStage;
  std::vector<uint8_t> host(bytes, 0);
  uint8_t q[kS];
  for (int sc = 0; sc < 2; sc++)
    for (int mp = 0; mp < L; mp++)
      for (int b = 0; b < L; b++) {
        split_host(R[((size_t)sc * L + mp) * L + b] / rscale, q);
        uint8_t* blk = host.data() + ((size_t)(sc * MT + mp / kN) * nc + b / kKC) * kAStage;
        const int off = atile_off(mp % kN, b % kKC);
        for (int i = 0; i < kS; i++) blk[i * (kN * kKC) + off] = q[i];
      }
  auto t = std::make_unique<BetaTable>();
  t->L = L, t->rscale = rscale, t->bytes = bytes;
  SO3G_CUDA(cudaMalloc(&t->d, bytes));
  SO3G_CUDA(cudaMemcpyAsync(t->d, host.data(), bytes, cudaMemcpyHostToDevice, s));
  SO3G_CUDA(cudaStreamSynchronize(s));  // the host image goes out of scope
  *out = t.get();
  D->beta_tables.push_back(std::move(t));
  return kOk;
}

int launch_mixed_fwd_beta(const Geometry& g, double2* W, long long wstride, int nsig, const BetaTable* tab,
                          void* scratch, cudaStream_t s) {
  if (!mixed_beta_supported(g)) return fail(kUnsupported, "split-precision beta stage: complex MW signals only");
  BetaArgs a{};
  int ct = 0;
  const int tiles = beta_tiles(g, &ct);
  if (nsig > 65535) return fail(kUnsupported, "split-precision beta stage: batch too large");
  a.xs = static_cast<uint8_t*>(scratch);
  a.xscale = reinterpret_cast<double*>(a.xs + (((size_t)nsig * tiles * nchunks(g) * kXStage + 255) & ~size_t(255)));
  a.W = W, a.Wc = W + g.QOFF, a.tab = tab->d, a.rscale = tab->rscale, a.wstride = wstride;
  a.L = g.L, a.nplanes = g.nplanes, a.plane0 = g.plane0, a.ct = ct, a.nchunk = nchunks(g), a.MT = nchunks(g);
  a.nsig = nsig, a.RS = g.RS, a.PS = g.PS, a.CS = g.CS, a.QS = g.QS;
  if (a.nchunk * kKC <= 512 && stream_slicing()) {
    // single read of the beta samples through shared memory
    const int bsmem = a.nchunk * kKC * kBsCols * (int)sizeof(double2) + (8 * 16 + 16) * (int)sizeof(double);
    SO3G_CUDA(cudaFuncSetAttribute(beta_slice1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bsmem));
    beta_slice1_kernel<<<dim3((unsigned)(16 * ct * g.nplanes), (unsigned)nsig), 256, bsmem, s>>>(a, tiles);
  } else {
    beta_slice_kernel<<<dim3((unsigned)tiles, (unsigned)nsig), 256, 0, s>>>(a);
  }
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  const int smem = (int)sizeof(TcpSmem);
  const long long items = (long long)tiles * a.MT * nsig;
  if (items > 0x7fffffffLL) return fail(kUnsupported, "split-precision beta stage: too many work items");
  SO3G_CUDA(cudaFuncSetAttribute(beta_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int grid = (int)std::min<long long>(items, sm_count());
  beta_tc_kernel<<<grid, kThreads, smem, s>>>(a, tiles, (int)items);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------- ragged batches (host)
namespace {
struct RaggedPlan {
  std::vector<SigDesc> sigs;
  std::vector<GroupDesc> groups;
  size_t xs_bytes = 0, sc_count = 0;
  long long items = 0, slices = 0;
  size_t sc_off = 0, sig_off = 0, grp_off = 0, total = 0;
};

RaggedPlan ragged_plan(const std::vector<RaggedSig>& in, bool fwd) {
  RaggedPlan P;
  std::vector<int> order(in.size());
  for (size_t i = 0; i < in.size(); i++) order[i] = (int)i;
  // similar geometries share a group: the group runs at its largest L and N
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return in[x].g.L != in[y].g.L ? in[x].g.L > in[y].g.L : in[x].g.N > in[y].g.N;
  });
  for (int i : order) {
    const RaggedSig& r = in[i];
    SigDesc d{};
    d.flmn = static_cast<const double2*>(r.flmn);
    d.Wc = r.Wc;
    d.base = r.base;
    d.CS = r.g.CS, d.QS = r.g.QS;
    d.L = r.g.L, d.N = r.g.N, d.L0 = r.g.L0, d.plane0 = r.g.plane0, d.n_mode = r.n_mode, d.compact = r.compact;
    P.sigs.push_back(d);
  }
  for (size_t s0 = 0; s0 < P.sigs.size(); s0 += kSig) {
    GroupDesc G{};
    G.sig0 = (int)s0;
    G.nsig = (int)std::min<size_t>(kSig, P.sigs.size() - s0);
    for (int b = 0; b < G.nsig; b++) {
      G.Lg = std::max(G.Lg, P.sigs[s0 + b].L);
      G.Ng = std::max(G.Ng, P.sigs[s0 + b].N);
    }
    G.nc = (G.Lg + kKC - 1) / kKC;
    const size_t pairs = (size_t)G.Lg * G.Ng;
    G.xs_off = (long long)P.xs_bytes;
    G.sc_off = (long long)P.sc_count;
    G.item0 = (int)P.items;
    G.slice0 = (int)P.slices;
    P.xs_bytes += pairs * G.nc * (size_t)kXStage;
    P.sc_count += pairs * kM;
    P.items += (long long)pairs * G.nc;
    P.slices += fwd ? (long long)pairs * (kSig / kSigPer) : (long long)G.Ng * ((G.Lg + kMuPer - 1) / kMuPer) * kSig;
    P.groups.push_back(G);
  }
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  P.sc_off = al(P.xs_bytes);
  P.sig_off = al(P.sc_off + P.sc_count * sizeof(double));
  P.grp_off = al(P.sig_off + P.sigs.size() * sizeof(SigDesc));
  P.total = al(P.grp_off + P.groups.size() * sizeof(GroupDesc));
  return P;
}
}  // namespace

size_t ragged_scratch_bytes(const std::vector<RaggedSig>& sigs, bool fwd) {
  return sigs.empty() ? 0 : ragged_plan(sigs, fwd).total;
}

int launch_mixed_ragged(bool fwd, const std::vector<RaggedSig>& sigs, const double* dl, const DigitTable* tab,
                        void* scratch, cudaStream_t s) {
  if (sigs.empty()) return kOk;
  for (const auto& r : sigs)
    if (r.g.real) return fail(kUnsupported, "split-precision contractions take complex signals");
  const RaggedPlan P = ragged_plan(sigs, fwd);
  if (P.items > 0x7fffffffLL || P.slices > 0x7fffffffLL)
    return fail(kUnsupported, "split-precision ragged batch: too many work items");
  char* base = static_cast<char*>(scratch);
  // pageable copies: the bytes are staged by the time cudaMemcpyAsync returns
  SO3G_CUDA(cudaMemcpyAsync(base + P.sig_off, P.sigs.data(), P.sigs.size() * sizeof(SigDesc),
                            cudaMemcpyHostToDevice, s));
  SO3G_CUDA(cudaMemcpyAsync(base + P.grp_off, P.groups.data(), P.groups.size() * sizeof(GroupDesc),
                            cudaMemcpyHostToDevice, s));
  RagArgs a{};
  a.xs = reinterpret_cast<uint8_t*>(base);
  a.xscale = reinterpret_cast<double*>(base + P.sc_off);
  a.sigs = reinterpret_cast<const SigDesc*>(base + P.sig_off);
  a.groups = reinterpret_cast<const GroupDesc*>(base + P.grp_off);
  a.dl = dl;
  a.ngroups = (int)P.groups.size();
  bool use_tab = tab != nullptr;
  for (const GroupDesc& G : P.groups) use_tab = use_tab && G.Lg <= tab->L && G.Ng <= tab->N;
  if (use_tab) {
    a.tab = tab->d;
    a.pair_off = tab->pair_off;
    a.tab_N = tab->N;
    a.tab_nc = (tab->L + kKC - 1) / kKC;
  }
  if (fwd)
    ragged_slice_fwd_kernel<<<(unsigned)P.slices, 256, 0, s>>>(a);
  else
    ragged_slice_inv_kernel<<<(unsigned)P.slices, 256, 0, s>>>(a);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  if (P.items == 0) return kOk;
  const int smem = (int)sizeof(TcSmem);
  auto run = [&](auto kernel) -> int {
    SO3G_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kernel<<<(unsigned)P.items, kThreads, smem, s>>>(a);
    return kOk;
  };
  int rc;
  if (fwd)
    rc = use_tab ? run(ragged_tc_kernel<true, true>) : run(ragged_tc_kernel<true, false>);
  else
    rc = use_tab ? run(ragged_tc_kernel<false, true>) : run(ragged_tc_kernel<false, false>);
  if (rc) return rc;
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

// Reads and clears the tensor-core kernels' wait-timeout flag (0: none).
int mixed_take_error() {
  int v = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)) != cudaSuccess) return -1;
  if (v) cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int));
  return v;
}

}  // namespace so3g
