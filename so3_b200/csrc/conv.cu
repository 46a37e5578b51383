// Harmonic-space convolutions (reference src/c/so3_conv.c).
//
//  s2toso3 (so3_conv.c:186-215): h_lmn = f_lm conj(g_ln) 8 pi^2/(2l+1) for
//    |n| <= l, 0 otherwise, over every stored entry of hlmn.  One thread per
//    (n-block, l*l+l+m) element; the block base table replaces the per-index
//    ind2elmn inversion of the reference.
//  SO(3) x SO(3) (so3_conv.c:44-90): h_lmn = sum_k f_lmk conj(g_lnk) over k
//    in f's n-loop where g_lnk is a non-zero slot; one thread per output.
#include "so3gpu_internal.h"

namespace so3g {

namespace {
constexpr double k8Pi2 = 78.956835208714863096923300678716626;  // 8 pi^2

__device__ __forceinline__ int isqrt_floor(int e) {
  int l = (int)sqrt((double)e);
  while (l * l > e) l--;
  while ((l + 1) * (l + 1) <= e) l++;
  return l;
}
__device__ __forceinline__ double2 cmulconj(double2 a, double2 b) {  // a * conj(b)
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}

struct LoopN {
  int start, stop, inc;
};
__device__ __forceinline__ bool in_loop(int i, LoopN r) {
  return i >= r.start && i <= r.stop && (i - r.start) % r.inc == 0;
}
}  // namespace

__global__ void s2toso3_kernel(const double2* __restrict__ flm, const double2* __restrict__ glm,
                               const long long* __restrict__ base, double2* __restrict__ h, int L, int N, int real,
                               int compact) {
  const int plane = blockIdx.y;
  const int n = real ? plane : plane - (N - 1);
  const int an = n < 0 ? -n : n;
  const long long b = base[plane];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < L * L; e += gridDim.x * blockDim.x) {
    const int l = isqrt_floor(e);
    const int m = e - l * l - l;
    if (compact && l < an) continue;
    double2 v = make_double2(0.0, 0.0);
    if (an <= l) {
      const double2 p = cmulconj(flm[e], glm[l * l + l + n]);
      const double s = k8Pi2 / (2 * l + 1);
      v = make_double2(p.x * s, p.y * s);
    }
    h[b + e] = v;
    (void)m;
  }
}

int launch_s2toso3(const so3_parameters_t& hp, const long long* bases, const double2* flm, const double2* glm,
                   double2* hlmn, cudaStream_t s) {
  const int real = hp.reality != 0;
  const int planes = real ? hp.N : 2 * hp.N - 1;
  const int per = hp.L * hp.L;
  dim3 grid((per + 255) / 256 < 1024 ? (per + 255) / 256 : 1024, planes);
  s2toso3_kernel<<<grid, 256, 0, s>>>(flm, glm, bases, hlmn, hp.L, hp.N, real, hp.storage == SO3_STORAGE_COMPACT);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

struct ConvSide {
  const long long* base;
  int L0, L, N, mode, real;
  LoopN loop;
};

static LoopN n_loop(const so3_parameters_t& p) {
  const int N = p.N;
  LoopN r{};
  if (p.reality) {
    switch (p.n_mode) {
      case SO3_N_MODE_EVEN: r = {0, ((N - 1) % 2 == 0) ? N - 1 : N - 2, 2}; break;
      case SO3_N_MODE_ODD: r = {1, ((N - 1) % 2 != 0) ? N - 1 : N - 2, 2}; break;
      case SO3_N_MODE_MAXIMUM: r = {N - 1, N - 1, 1}; break;
      default: r = {0, N - 1, 1}; break;
    }
  } else {
    switch (p.n_mode) {
      case SO3_N_MODE_EVEN:
        r = {((N - 1) % 2 == 0) ? -N + 1 : -N + 2, ((N - 1) % 2 == 0) ? N - 1 : N - 2, 2};
        break;
      case SO3_N_MODE_ODD:
        r = {((N - 1) % 2 != 0) ? -N + 1 : -N + 2, ((N - 1) % 2 != 0) ? N - 1 : N - 2, 2};
        break;
      case SO3_N_MODE_MAXIMUM: r = {-N + 1, N - 1, N > 1 ? 2 * N - 2 : 1}; break;
      default: r = {-N + 1, N - 1, 1}; break;
    }
  }
  return r;
}

__global__ void harmonic_conv_kernel(ConvSide H, ConvSide F, ConvSide G, const double2* __restrict__ f,
                                     const double2* __restrict__ g, double2* __restrict__ h) {
  const int hplane = blockIdx.y;
  const int n = H.real ? hplane : hplane - (H.N - 1);
  if (!in_loop(n, H.loop)) return;
  const int an = n < 0 ? -n : n;
  const int el_lo = max(H.L0, an), el_hi = H.mode == SO3_N_MODE_L ? an : H.L - 1;
  const int fplane0 = F.real ? 0 : F.N - 1, gplane0 = G.real ? 0 : G.N - 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < H.L * H.L; e += gridDim.x * blockDim.x) {
    const int l = isqrt_floor(e);
    if (l < el_lo || l > el_hi) continue;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = F.loop.start; k <= F.loop.stop; k += F.loop.inc) {
      // g_{l, n, k} non-zero slot?
      if (!in_loop(k, G.loop)) continue;
      const int ak = k < 0 ? -k : k;
      const int gl_lo = max(G.L0, ak), gl_hi = G.mode == SO3_N_MODE_L ? ak : G.L - 1;
      if (l < gl_lo || l > gl_hi || an > l) continue;
      const double2 fv = f[F.base[fplane0 + k] + e];
      const double2 gv = g[G.base[gplane0 + k] + (long long)l * l + l + n];
      acc = make_double2(acc.x + fma(fv.x, gv.x, fv.y * gv.y), acc.y + fma(fv.y, gv.x, -fv.x * gv.y));
    }
    h[H.base[hplane] + e] = acc;
  }
}

int launch_harmonic_convolution(const so3_parameters_t& hp, const so3_parameters_t& fp, const so3_parameters_t& gp,
                                const long long* hb, const long long* fb, const long long* gb, const double2* flmn,
                                const double2* glmn, double2* hlmn, cudaStream_t s) {
  ConvSide H{hb, hp.L0, hp.L, hp.N, (int)hp.n_mode, hp.reality != 0, n_loop(hp)};
  ConvSide F{fb, fp.L0, fp.L, fp.N, (int)fp.n_mode, fp.reality != 0, n_loop(fp)};
  ConvSide G{gb, gp.L0, gp.L, gp.N, (int)gp.n_mode, gp.reality != 0, n_loop(gp)};
  const int planes = hp.reality ? hp.N : 2 * hp.N - 1;
  const int per = hp.L * hp.L;
  dim3 grid((per + 255) / 256 < 1024 ? (per + 255) / 256 : 1024, planes);
  harmonic_conv_kernel<<<grid, 256, 0, s>>>(H, F, G, flmn, glmn, hlmn);
  SO3G_LAUNCHED();
  SO3G_CUDA(cudaGetLastError());
  return kOk;
}

}  // namespace so3g
