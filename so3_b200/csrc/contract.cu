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
// Negative m, n use Delta^l_{m',-k} = (-1)^{l+m'} Delta^l_{m'k}: one product
// w = Delta_{m'|m|} Delta_{m'|n|} feeds the four sign combinations
// (+m,+n), (-m,+n), (+m,-n), (-m,-n); combinations with exactly one negative
// index carry (-1)^{l+m'}, split as (-1)^l folded into the operand that
// depends on l and (-1)^{m'} into the one that depends on m'.
//
// CTA = 4 warps.  Lanes span 32 consecutive |m| (coalesced loads of Delta rows
// and of coefficient/spectral rows); each warp owns 8 values of the output
// index (m' for the inverse, l for the forward); blockIdx.z = |n|.
#include "so3gpu_internal.h"

namespace so3g {

namespace {
constexpr int kWarps = 4;
constexpr int kPer = 8;                  // output rows per warp
constexpr int kTile = kWarps * kPer;     // 32 output rows per CTA
constexpr double kInv8Pi2 = 0.012665147955292221430803304553147533;  // 1/(8 pi^2)

__device__ __forceinline__ double2 ipow_mul(double2 v, int k) {  // v * i^k
  switch (k & 3) {
    case 0: return v;
    case 1: return make_double2(-v.y, v.x);
    case 2: return make_double2(-v.x, -v.y);
    default: return make_double2(v.y, -v.x);
  }
}
}  // namespace

struct InvArgs {
  const double2* flmn;
  const long long* base;  // per plane
  const double* dl;
  double2* W;
  int L, N, L0, plane0, n_mode, real, sym_n0;
  long long RS, PS;
};

__global__ void __launch_bounds__(128) inverse_contract_kernel(InvArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int mu = blockIdx.x * 32 + lane;
  const int mp0 = blockIdx.y * kTile + warp * kPer;
  const int nu = blockIdx.z;
  const int L = a.L;
  const bool neg_n = !a.real && nu > 0;  // a distinct -nu plane exists
  const bool skipped = plane_skipped(a.n_mode, a.N, nu);  // +nu and -nu share parity and |n|

  double2 acc[kPer][4];
#pragma unroll
  for (int i = 0; i < kPer; i++)
#pragma unroll
    for (int s = 0; s < 4; s++) acc[i][s] = make_double2(0.0, 0.0);

  if (!skipped) {
    const long long bp = a.base[a.plane0 + nu];
    const long long bn = neg_n ? a.base[a.plane0 - nu] : 0;
    int lstart = max(max(a.L0, nu), max((int)(blockIdx.y * kTile), (int)(blockIdx.x * 32)));
    for (int l = lstart; l < L; l++) {
      const bool mu_ok = mu <= l;
      const double c = (2.0 * l + 1.0) * kInv8Pi2;
      const double sl = (l & 1) ? -c : c;
      const long long row = (long long)l * l + l;
      double2 h[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
      if (mu_ok) {
        double2 pp = __ldg(a.flmn + bp + row + mu);
        double2 mp_ = __ldg(a.flmn + bp + row - mu);
        if (a.sym_n0) {  // real signal, N == 1: f_{l,-m,0} = (-1)^m conj f_{l,m,0}
          mp_ = (mu & 1) ? make_double2(-pp.x, pp.y) : make_double2(pp.x, -pp.y);
        }
        h[0] = make_double2(c * pp.x, c * pp.y);
        h[1] = make_double2(sl * mp_.x, sl * mp_.y);
        if (neg_n) {
          double2 pm = __ldg(a.flmn + bn + row + mu);
          double2 mm = __ldg(a.flmn + bn + row - mu);
          h[2] = make_double2(sl * pm.x, sl * pm.y);
          h[3] = make_double2(c * mm.x, c * mm.y);
        }
      }
      const double* P = a.dl + dl_plane_offset(l);
      const int ld = l + 1;
#pragma unroll
      for (int i = 0; i < kPer; i++) {
        const int mp = mp0 + i;
        if (mp <= l && mu_ok) {
          const double w = __ldg(P + (long long)mp * ld + mu) * __ldg(P + (long long)mp * ld + nu);
#pragma unroll
          for (int s = 0; s < 4; s++) {
            acc[i][s].x = fma(w, h[s].x, acc[i][s].x);
            acc[i][s].y = fma(w, h[s].y, acc[i][s].y);
          }
        }
      }
    }
  }
  if (mu >= L) return;
  const int nplanes_sign = neg_n ? 2 : 1;
#pragma unroll
  for (int i = 0; i < kPer; i++) {
    const int mp = mp0 + i;
    if (mp >= L) continue;
    const double odd_mp = (mp & 1) ? -1.0 : 1.0;
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const int ms = (s & 1) ? -1 : 1, ns = (s & 2) ? -1 : 1;
      if (ms < 0 && mu == 0) continue;
      if (ns < 0 && nplanes_sign == 1) continue;
      const int m = ms * mu, n = ns * nu;
      double2 v = acc[i][s];
      if (ms * ns < 0) v = make_double2(v.x * odd_mp, v.y * odd_mp);
      v = ipow_mul(v, n - m + 4 * L);
      a.W[(long long)(a.plane0 + n) * a.PS + (long long)mp * a.RS + (m + L - 1)] = v;
    }
  }
}

int launch_inverse_contract(const Geometry& g, int n_mode, const double2* flmn, const long long* bases,
                            const double* dl, double2* W, int sym_n0, cudaStream_t s) {
  InvArgs a{flmn, bases, dl, W, g.L, g.N, g.L0, g.plane0, n_mode, g.real, sym_n0, g.RS, g.PS};
  dim3 grid((g.L + 31) / 32, (g.L + kTile - 1) / kTile, g.N);
  inverse_contract_kernel<<<grid, 128, 0, s>>>(a);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

struct FwdArgs {
  const double2* W;
  const long long* base;
  const double* dl;
  double2* flmn;
  int L, N, L0, plane0, n_mode, real, compact;
  long long RS, PS;
};

__global__ void __launch_bounds__(128) forward_contract_kernel(FwdArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int mu = blockIdx.x * 32 + lane;
  const int l0 = blockIdx.y * kTile + warp * kPer;
  const int nu = blockIdx.z;
  const int L = a.L;
  const bool neg_n = !a.real && nu > 0;
  if (plane_skipped(a.n_mode, a.N, nu)) return;  // caller-zeroed blocks stay untouched

  double2 acc[kPer][4];
#pragma unroll
  for (int i = 0; i < kPer; i++)
#pragma unroll
    for (int s = 0; s < 4; s++) acc[i][s] = make_double2(0.0, 0.0);

  const int ltop = min(L - 1, (int)(blockIdx.y * kTile) + kTile - 1);
  const int lmin_needed = max(max(a.L0, nu), (int)(blockIdx.x * 32));
  if (ltop >= lmin_needed) {
    const double2* Gp = a.W + (long long)(a.plane0 + nu) * a.PS + (L - 1);
    const double2* Gn = a.W + (long long)(a.plane0 - nu) * a.PS + (L - 1);
    const bool mu_ok = mu < L;
    for (int mp = 0; mp <= ltop; mp++) {
      double2 g[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
      if (mu_ok) {
        const double sm = (mp & 1) ? -1.0 : 1.0;
        const long long r = (long long)mp * a.RS;
        double2 pp = __ldg(Gp + r + mu), mp_ = __ldg(Gp + r - mu);
        g[0] = pp;
        g[1] = make_double2(sm * mp_.x, sm * mp_.y);
        if (neg_n) {
          double2 pm = __ldg(Gn + r + mu), mm = __ldg(Gn + r - mu);
          g[2] = make_double2(sm * pm.x, sm * pm.y);
          g[3] = mm;
        }
      }
#pragma unroll
      for (int i = 0; i < kPer; i++) {
        const int l = l0 + i;
        if (l < L && mp <= l && mu <= l && l >= nu) {
          const double* P = a.dl + dl_plane_offset(l) + (long long)mp * (l + 1);
          const double w = __ldg(P + mu) * __ldg(P + nu);
#pragma unroll
          for (int s = 0; s < 4; s++) {
            acc[i][s].x = fma(w, g[s].x, acc[i][s].x);
            acc[i][s].y = fma(w, g[s].y, acc[i][s].y);
          }
        }
      }
    }
  }
  if (mu >= L) return;
#pragma unroll
  for (int i = 0; i < kPer; i++) {
    const int l = l0 + i;
    if (l >= L || mu > l) continue;
    const double odd_l = (l & 1) ? -1.0 : 1.0;
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const int ms = (s & 1) ? -1 : 1, ns = (s & 2) ? -1 : 1;
      if (ms < 0 && mu == 0) continue;
      if (ns < 0 && !neg_n) continue;
      const int m = ms * mu, n = ns * nu;
      if (a.compact && l < nu) continue;  // not stored
      double2 v = make_double2(0.0, 0.0);
      if (l >= max(a.L0, nu)) {
        v = acc[i][s];
        if (ms * ns < 0) v = make_double2(v.x * odd_l, v.y * odd_l);
        v = ipow_mul(v, m - n + 4 * L);
      }
      a.flmn[a.base[a.plane0 + n] + (long long)l * l + l + m] = v;
    }
  }
}

int launch_forward_contract(const Geometry& g, int n_mode, const double2* W, const long long* bases,
                            const double* dl, double2* flmn, int storage_compact, cudaStream_t s) {
  FwdArgs a{W, bases, dl, flmn, g.L, g.N, g.L0, g.plane0, n_mode, g.real, storage_compact, g.RS, g.PS};
  dim3 grid((g.L + 31) / 32, (g.L + kTile - 1) / kTile, g.N);
  forward_contract_kernel<<<grid, 128, 0, s>>>(a);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace so3g
