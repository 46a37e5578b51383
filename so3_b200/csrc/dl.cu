// Resident Wigner Delta(pi/2) table: quarter planes 0 <= m', m <= l for every
// degree l < Lcap, plane l at dl_plane_offset(l), row-major (m' rows).
//
// Replaces the per-call, per-n recomputation inside SSHT (called from the
// reference's src/c/so3_core.c:204, :408) and the in-tree recursions at
// src/c/so3_core.c:1001-1035.  Both recursions the reference offers are built:
//
//  * Trapani & Navaza (2006): the first row of degree l follows from the first
//    row of degree l-1 (eqs. 9-10; one sweep over l), after which every column
//    m of every degree is an independent three-term recursion down m' (eq. 11):
//    one GPU thread per (l, m), no inter-thread dependence.
//  * Risbo (1996): half-step recursion over the eighth m' >= m >= 0 plus the
//    margin its neighbours need; degree l needs all of degree l-1, so one CTA
//    sweeps the degrees with barriers between the half steps.
//
// Upper-triangle entries (m' < m) are filled from Delta_{m'm} =
// (-1)^{m-m'} Delta_{mm'}.
#include "so3gpu_internal.h"

namespace so3g {

__device__ __forceinline__ double sgn(int k) { return (k & 1) ? -1.0 : 1.0; }

// Row m' = l of every plane: Delta^l_{l,0} = -sqrt((2l-1)/(2l)) Delta^{l-1}_{l-1,0},
// Delta^l_{l,m} = sqrt(l(2l-1) / (2(l+m)(l+m-1))) Delta^{l-1}_{l-1,m-1}.
__global__ void dl_trapani_top_rows(double* __restrict__ T, int Lcap) {
  if (threadIdx.x == 0) T[0] = 1.0;
  __syncthreads();
  for (int l = 1; l < Lcap; l++) {
    const double* prev = T + dl_plane_offset(l - 1) + (long long)(l - 1) * l;  // row l-1 of plane l-1
    double* row = T + dl_plane_offset(l) + (long long)l * (l + 1);            // row l of plane l
    for (int m = threadIdx.x; m <= l; m += blockDim.x) {
      double v;
      if (m == 0)
        v = -sqrt((2.0 * l - 1.0) / (2.0 * l)) * prev[0];
      else
        v = sqrt((double)l * (2.0 * l - 1.0) / (2.0 * (l + m) * (l + m - 1.0))) * prev[m - 1];
      row[m] = v;
    }
    __syncthreads();
  }
}

// Column m of plane l, rows m' = l-1 .. m:
// sqrt((l-m')(l+m'+1)) D_{m'} = 2m D_{m'+1} - sqrt((l-m'-1)(l+m'+2)) D_{m'+2}.
__global__ void dl_trapani_columns(double* __restrict__ T) {
  const int l = blockIdx.x;
  double* P = T + dl_plane_offset(l);
  const int ld = l + 1;
  for (int m = threadIdx.x; m <= l; m += blockDim.x) {
    double d1 = P[(long long)l * ld + m], d2 = 0.0;  // D_{m'+1}, D_{m'+2}
    for (int mp = l - 1; mp >= m; mp--) {
      const double t1 = sqrt((double)(l - mp) * (double)(l + mp + 1));
      const double t2 = (mp + 2 <= l) ? sqrt((double)(l - mp - 1) * (double)(l + mp + 2)) : 0.0;
      const double d0 = (2.0 * m * d1 - t2 * d2) / t1;
      P[(long long)mp * ld + m] = d0;
      d2 = d1;
      d1 = d0;
    }
  }
}

__global__ void dl_fill_upper(double* __restrict__ T) {
  const int l = blockIdx.x;
  double* P = T + dl_plane_offset(l);
  const int ld = l + 1;
  for (int i = threadIdx.x; i < ld * ld; i += blockDim.x) {
    const int mp = i / ld, m = i - mp * ld;
    if (mp < m) P[i] = sgn(m - mp) * P[(long long)m * ld + mp];
  }
}

int launch_build_dl_trapani(double* table, int L0cap, int Lcap, cudaStream_t s) {
  (void)L0cap;
  dl_trapani_top_rows<<<1, 1024, 0, s>>>(table, Lcap);
  SO3G_LAUNCHED();
  dl_trapani_columns<<<Lcap, 256, 0, s>>>(table);
  SO3G_LAUNCHED();
  dl_fill_upper<<<Lcap, 256, 0, s>>>(table);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------- Risbo
// Work layout: two (Lcap+6)^2 layers, index (u+3)*S + (v+3) for u, v >= -3.
// Layer A holds integer degree l on the eighth plus margin; layer H holds the
// half degree l+1/2 with H(xp, yp) = d_{xp-1/2, yp-1/2}.
__global__ void __launch_bounds__(1024) dl_risbo_sweep(double* __restrict__ T, int Lcap, double* __restrict__ work) {
  const int S = Lcap + 6;
  double* A = work;
  double* H = work + (size_t)S * S;
#define RA(u, v) A[((u) + 3) * S + ((v) + 3)]
#define RH(u, v) H[((u) + 3) * S + ((v) + 3)]
  const int tid = threadIdx.x, nt = blockDim.x;
  const double c = 0.70710678118654752440084436210484903928;  // cos(pi/4) = sin(pi/4)
  for (int i = tid; i < 2 * S * S; i += nt) work[i] = 0.0;
  __syncthreads();
  if (tid == 0) {
    RA(0, 0) = 1.0;
    T[0] = 1.0;
  }
  __syncthreads();
  for (int el = 1; el < Lcap; el++) {
    const int l = el - 1;
    // margin of degree l
    for (int i = tid; i < 2 * (l + 1); i += nt) {
      const int u = i >> 1, v = u + 1 + (i & 1);
      RA(u, v) = v <= l ? sgn(v - u) * RA(v, u) : 0.0;
    }
    __syncthreads();
    for (int u = tid; u <= l; u += nt) RA(u, -1) = sgn(l + u) * RA(u, 1);
    __syncthreads();
    if (tid < 6) {
      // (u, v) pairs: (1,-1),(1,0),(1,1),(2,-1),(2,0),(3,-1)
      const int us[6] = {1, 1, 1, 2, 2, 3}, vs[6] = {-1, 0, 1, -1, 0, -1};
      const int u = us[tid], v = vs[tid];
      RA(-u, v) = (u <= l) ? sgn(l + v) * RA(u, v) : 0.0;
    }
    __syncthreads();
    // half degree J = l + 1/2
    {
      const int tJ = 2 * l + 1;
      const double inv = 1.0 / tJ;
      const int W = l + 3, Hh = l + 2;  // xp in [-1, l+1], yp in [0, l+1]
      for (int i = tid; i < W * Hh; i += nt) {
        const int yp = i / W, xp = i - yp * W - 1;
        const int x0 = yp - 1 > -l ? yp - 1 : -l;
        if (xp < x0) continue;
        const int a = l + xp, b = l + yp;
        const double sa = sqrt((double)a), sb = sqrt((double)b);
        const double sA = sqrt((double)(tJ - a)), sB = sqrt((double)(tJ - b));
        const double v = sa * sb * c * RA(xp - 1, yp - 1) - sa * sB * c * RA(xp - 1, yp) +
                         sA * sb * c * RA(xp, yp - 1) + sA * sB * c * RA(xp, yp);
        RH(xp, yp) = v * inv;
      }
    }
    __syncthreads();
    // integer degree el on the eighth
    {
      const int tJ = 2 * el;
      const double inv = 1.0 / tJ;
      const int W = el + 1;
      for (int i = tid; i < W * W; i += nt) {
        const int v = i / W, u = i - v * W;
        if (u < v) continue;
        const int a = el + u, b = el + v;
        const double sa = sqrt((double)a), sb = sqrt((double)b);
        const double sA = sqrt((double)(tJ - a)), sB = sqrt((double)(tJ - b));
        const double val = sa * sb * c * RH(u, v) - sa * sB * c * RH(u, v + 1) + sA * sb * c * RH(u + 1, v) +
                           sA * sB * c * RH(u + 1, v + 1);
        RA(u, v) = val * inv;
      }
    }
    __syncthreads();
    // quarter plane el into the table
    {
      double* P = T + dl_plane_offset(el);
      const int ld = el + 1;
      for (int i = tid; i < ld * ld; i += nt) {
        const int u = i / ld, v = i - u * ld;
        P[i] = v <= u ? RA(u, v) : sgn(v - u) * RA(v, u);
      }
    }
    __syncthreads();
  }
#undef RA
#undef RH
}

int launch_build_dl_risbo(double* table, int Lcap, double* work, cudaStream_t s) {
  dl_risbo_sweep<<<1, 1024, 0, s>>>(table, Lcap, work);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace so3g
