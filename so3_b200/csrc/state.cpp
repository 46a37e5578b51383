// Per-device state of libso3gpu: error reporting, resident Wigner tables, FFT
// plans, block-offset tables and grow-only scratch.  Host code only.
#include <cmath>
#include <cstdlib>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>

#include "so3gpu_internal.h"

namespace so3g {

std::atomic<long long> g_launches{0};

static thread_local std::string t_last_error;
void set_error(const std::string& msg) { t_last_error = msg; }
const std::string& last_error() { return t_last_error; }
int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

// ------------------------------------------------------------------ geometry
Geometry make_geometry(const so3_parameters_t& p, int real) {
  Geometry g{};
  g.L = p.L;
  g.N = p.N;
  g.L0 = p.L0;
  g.mw = p.sampling_scheme == SO3_SAMPLING_MW;
  g.real = real;
  g.na = g.mw ? 2 * p.L - 1 : 2 * p.L;
  g.nb = g.mw ? p.L : p.L + 1;
  g.P = g.na;
  g.steer = p.steerable != 0;
  g.ng = g.steer ? 2 * p.N : 2 * p.N - 1;
  g.nf = g.steer ? p.N : 2 * p.N - 1;
  g.nplanes = real ? p.N : 2 * p.N - 1;
  g.plane0 = real ? 0 : p.N - 1;
  g.RS = ((2L * p.L + 7) / 8) * 8;
  g.PS = g.RS * g.nb;
  g.CS = ((long)p.L + 7) / 8 * 8;
  g.QS = g.CS * (2L * p.L - 1);
  g.QOFF = (long)g.nplanes * g.PS;
  int pc = 1;
  while (pc < 4 * p.L - 3) pc <<= 1;
  g.Pc = pc;
  return g;
}

size_t workspace_bytes(const so3_parameters_t& p, int real) {
  Geometry g = make_geometry(p, real);
  return (size_t)g.nplanes * (size_t)(g.PS + g.QS) * sizeof(double2);
}

static long long base_negfirst(long long n, long long L, long long N, int compact) {
  if (!compact) return (N - 1 + n) * L * L;
  long long an = n < 0 ? -n : n;
  long long off = (N - 1 + n) * L * L - (2 * N - 1) * (N - 1) * N / 6;
  if (n <= 0)
    off += an * (2 * an + 1) * (an + 1) / 6;
  else
    off -= an * (2 * an - 1) * (an - 1) / 6;
  return off - n * n;
}

static long long base_zerofirst(long long n, long long L, int compact) {
  if (!compact) return (n < 0 ? -2 * n - 1 : 2 * n) * L * L;
  long long an = n < 0 ? -n : n;
  long long off = (2 * an - 1) * (3 * L * L - an * (an - 1)) / 3;
  if (n >= 0) off += L * L - n * n;
  return off - n * n;
}

std::vector<long long> block_bases(const so3_parameters_t& p, int real) {
  const long long L = p.L, N = p.N;
  const int compact = p.storage == SO3_STORAGE_COMPACT;
  std::vector<long long> b;
  if (real) {
    long long b0 = base_negfirst(0, L, N, compact);
    for (long long n = 0; n < N; n++) b.push_back(base_negfirst(n, L, N, compact) - b0);
  } else {
    for (long long n = -(N - 1); n <= N - 1; n++)
      b.push_back(p.n_order == SO3_N_ORDER_ZERO_FIRST ? base_zerofirst(n, L, compact)
                                                      : base_negfirst(n, L, N, compact));
  }
  return b;
}

int validate(const so3_parameters_t& p, int real) {
  (void)real;
  if (p.L < 1) return fail(kInvalidParameter, "L must be >= 1");
  if (p.N < 1) return fail(kInvalidParameter, "N must be >= 1");
  if (p.L0 < 0 || p.L0 > p.L) return fail(kInvalidParameter, "L0 must lie in [0, L]");
  if (p.sampling_scheme != SO3_SAMPLING_MW && p.sampling_scheme != SO3_SAMPLING_MW_SS)
    return fail(kInvalidParameter, "Invalid sampling scheme.");
  if (p.storage != SO3_STORAGE_PADDED && p.storage != SO3_STORAGE_COMPACT)
    return fail(kInvalidParameter, "Invalid storage method.");
  if (p.n_order != SO3_N_ORDER_ZERO_FIRST && p.n_order != SO3_N_ORDER_NEGATIVE_FIRST)
    return fail(kInvalidParameter, "Invalid n-order.");
  if (p.n_mode < SO3_N_MODE_ALL || p.n_mode >= SO3_N_MODE_SIZE) return fail(kInvalidParameter, "Invalid n-mode.");
  if (p.dl_method != SSHT_DL_RISBO && p.dl_method != SSHT_DL_TRAPANI)
    return fail(kInvalidParameter, "Invalid dl method");
  if (p.storage == SO3_STORAGE_COMPACT && p.N > p.L)
    return fail(kInvalidParameter, "compact storage needs N <= L");
  // the reference's real transforms ignore the flag (so3_core.c:526-547) and
  // write 2N-1 gamma planes into a buffer sized for the N of a steerable signal
  if (p.steerable && (p.reality || real))
    return fail(kUnsupported, "steerable signals are supported for complex transforms only");
  if (p.L > 4096) return fail(kUnsupported, "L > 4096 is not supported");
  if (p.N > 2048) return fail(kUnsupported, "N > 2048 is not supported");
  double fsz = (double)(2 * p.L) * (p.L + 1) * (2 * p.N - 1);
  if (fsz > 2147483647.0) return fail(kUnsupported, "sample count exceeds the int range of the C ABI");
  return kOk;
}

// ------------------------------------------------------------------ devices
size_t resident_bytes(Device* D) {
  std::lock_guard<std::mutex> lk(D->mu);
  size_t b = 0;
  for (const DlTable& t : D->dl)
    if (t.d) b += (size_t)dl_plane_offset(t.Lcap) * sizeof(double);
  for (const auto& t : D->digit_tables) b += t->bytes + (size_t)t->L * t->N * sizeof(long long);
  for (const auto& t : D->beta_tables) b += t->bytes;
  for (const auto& kv : D->conv_kernels) b += (size_t)(16 * (kv.first / 2) + 2 * (kv.first / 2)) * sizeof(double2);  // 2 Pc <= 16L, plus 2L
  for (const auto& kv : D->ffts) b += (size_t)4 * (kv.first + 256) * sizeof(double2);
  for (const auto& kv : D->bases) b += 4096 * sizeof(long long);
  return b;
}

static std::mutex g_dev_mu;
static std::map<int, std::unique_ptr<Device>> g_devs;

Device* device_state(int device) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  auto it = g_devs.find(device);
  if (it != g_devs.end()) return it->second.get();
  auto d = std::make_unique<Device>();
  d->device = device;
  Device* raw = d.get();
  g_devs[device] = std::move(d);
  return raw;
}

static cudaEvent_t take_event(StageTimer* t) {
  if (!t->pool.empty()) {
    cudaEvent_t e = t->pool.back();
    t->pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void timer_begin(StageTimer* t, cudaStream_t s, cudaEvent_t* ev) {
  *ev = nullptr;
  if (!t || !t->on) return;
  *ev = take_event(t);
  cudaEventRecord(*ev, s);
}

void timer_end(StageTimer* t, cudaStream_t s, int stage, cudaEvent_t start) {
  if (!t || !t->on || !start) return;
  cudaEvent_t e = take_event(t);
  cudaEventRecord(e, s);
  t->pending.push_back({stage, {start, e}});
}

int timer_collect(StageTimer* t) {
  for (auto& pe : t->pending) {
    SO3G_CUDA(cudaEventSynchronize(pe.second.second));
    float ms = 0.f;
    SO3G_CUDA(cudaEventElapsedTime(&ms, pe.second.first, pe.second.second));
    t->total_ms[pe.first] += ms;
    t->count[pe.first] += 1;
    t->pool.push_back(pe.second.first);
    t->pool.push_back(pe.second.second);
  }
  t->pending.clear();
  return kOk;
}

int ensure_ws(Workspace* W, size_t bytes, void** out) {
  if (bytes > W->ws_bytes && W->borrowed)
    return fail(kOutOfMemory, "borrowed workspace too small for this call");
  if (bytes > W->ws_bytes) {
    if (W->ws) cudaFree(W->ws);
    W->ws = nullptr;
    W->ws_bytes = 0;
    cudaError_t e = cudaMalloc(&W->ws, bytes);
    if (e != cudaSuccess) return fail(kOutOfMemory, std::string("workspace allocation failed: ") + cudaGetErrorString(e));
    W->ws_bytes = bytes;
  }
  *out = W->ws;
  return kOk;
}

// ------------------------------------------------------------------ tables
int ensure_dl(Device* D, int L, int method, cudaStream_t s, const double** out) {
  DlTable& T = D->dl[method];
  if (T.Lcap >= L) {
    *out = T.d;
    return kOk;
  }
  int Lcap = 1;
  while (Lcap < L) Lcap <<= 1;  // power-of-two capacity: a few rebuilds at most
  if (Lcap < 64) Lcap = 64;
  size_t bytes = (size_t)dl_plane_offset(Lcap) * sizeof(double);
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, bytes);
  if (e != cudaSuccess) return fail(kOutOfMemory, std::string("Delta table allocation failed: ") + cudaGetErrorString(e));
  int rc;
  if (method == SSHT_DL_TRAPANI) {
    rc = launch_build_dl_trapani(d, 0, Lcap, s);
  } else {
    double* work = nullptr;
    size_t wb = 2 * (size_t)(Lcap + 6) * (Lcap + 6) * sizeof(double);
    e = cudaMalloc(&work, wb);
    if (e != cudaSuccess) {
      cudaFree(d);
      return fail(kOutOfMemory, "Risbo work allocation failed");
    }
    rc = launch_build_dl_risbo(d, Lcap, work, s);
    cudaStreamSynchronize(s);
    cudaFree(work);
  }
  if (rc != kOk) {
    cudaFree(d);
    return rc;
  }
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaFree(d);
    return fail(kCudaError, std::string("Delta table build failed: ") + cudaGetErrorString(e));
  }
  if (T.d) cudaFree(T.d);
  T.d = d;
  T.Lcap = Lcap;
  *out = d;
  return kOk;
}

// ------------------------------------------------------------------ FFT plans
typedef std::complex<long double> cld;
static const long double kPiL = 3.141592653589793238462643383279502884L;

static cld root_l(long long num, long long den) {  // e^{-2 pi i num/den}
  long double a = 2.0L * kPiL * (long double)num / (long double)den;
  return cld(cosl(a), -sinl(a));
}

static int factor_stockham(int n, int* rad) {
  int np = 0;
  while (n % 8 == 0) rad[np++] = 8, n /= 8;
  while (n % 4 == 0) rad[np++] = 4, n /= 4;
  while (n % 2 == 0) rad[np++] = 2, n /= 2;
  const int primes[] = {3, 5, 7, 11, 13, 17, 19, 23, 29, 31};
  for (int p : primes)
    while (n % p == 0) {
      if (np >= kMaxPasses) return -1;
      rad[np++] = p, n /= p;
    }
  return n == 1 ? np : -1;
}

// in-place radix-2 FFT in long double (host-side table preparation only)
static void fft_ld(std::vector<cld>& x, int sign) {
  const size_t n = x.size();
  for (size_t i = 1, j = 0; i < n; i++) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(x[i], x[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; k++) {
        cld w = root_l((long long)k, (long long)len);
        if (sign > 0) w = std::conj(w);
        cld u = x[i + k], v = x[i + k + len / 2] * w;
        x[i + k] = u + v;
        x[i + k + len / 2] = u - v;
      }
  }
}

int ensure_fft(Device* D, int n, FftPlan* out) {
  const int key = n;
  auto it = D->ffts.find(key);
  if (it != D->ffts.end()) {
    *out = it->second->plan;
    return kOk;
  }
  auto dp = std::make_unique<DevPlan>();
  FftPlan& P = dp->plan;
  P.n = n;
  int np = factor_stockham(n, P.rad);
  std::vector<double2> host;
  if (np >= 0) {
    P.npass = np;
    P.blue = 0;
    host.resize(n);
    for (int k = 0; k < n; k++) {
      cld r = root_l(k, n);
      host[k] = make_double2((double)r.real(), (double)r.imag());
    }
  } else {
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    P.blue = 1;
    P.m = m;
    P.npass = 0;
    P.mpass = factor_stockham(m, P.mrad);
    host.resize((size_t)m + n + m);
    for (int k = 0; k < m; k++) {
      cld r = root_l(k, m);
      host[k] = make_double2((double)r.real(), (double)r.imag());
    }
    std::vector<cld> ch(n);
    for (int k = 0; k < n; k++) {
      long long kk = ((long long)k * k) % (2LL * n);
      ch[k] = root_l(kk, 2LL * n);  // e^{-i pi k^2/n}
      host[m + k] = make_double2((double)ch[k].real(), (double)ch[k].imag());
    }
    std::vector<cld> ker(m, cld(0, 0));
    ker[0] = std::conj(ch[0]);
    for (int k = 1; k < n; k++) ker[k] = ker[m - k] = std::conj(ch[k]);
    fft_ld(ker, -1);
    for (int k = 0; k < m; k++) {
      cld v = ker[k] / (long double)m;
      host[(size_t)m + n + k] = make_double2((double)v.real(), (double)v.imag());
    }
  }
  const size_t half_at = host.size();
  host.resize(half_at + n);
  for (int k = 0; k < n; k++) {
    cld r = root_l(k, 2LL * n);  // e^{-i pi k/n}
    host[half_at + k] = make_double2((double)r.real(), (double)r.imag());
  }
  // Rader's algorithm for the prime 127 (gamma length at N = 64): X[3^{-b}] =
  // x[0] + sum_a x[3^a] w^{3^{a-b}}, a cyclic convolution of length 126
  const bool rader = n == 127;
  size_t rader_at = host.size();
  std::vector<int> perm;
  if (rader) {
    const int q = n - 1;
    host.resize(rader_at + 2 * (size_t)q);
    for (int k = 0; k < q; k++) {
      cld r = root_l(k, q);
      host[rader_at + k] = make_double2((double)r.real(), (double)r.imag());
    }
    perm.resize(2 * (size_t)q);
    std::vector<int> pw(q);  // 3^a mod n
    long long v = 1;
    for (int a = 0; a < q; a++) {
      pw[a] = (int)v;
      v = v * 3 % n;
    }
    for (int a = 0; a < q; a++) {
      perm[a] = pw[a];
      perm[q + a] = pw[(q - a) % q];  // 3^{-a} = 3^{q-a}
    }
    // kernel: FFT_q of v[m] = w^{3^{-m}}, divided by q (direct long-double DFT)
    for (int k = 0; k < q; k++) {
      cld acc(0, 0);
      for (int m = 0; m < q; m++) acc += root_l(perm[q + m], n) * root_l((long long)m * k % q, q);
      acc /= (long double)q;
      host[rader_at + q + k] = make_double2((double)acc.real(), (double)acc.imag());
    }
  }
  cudaError_t e = cudaMalloc(&dp->mem, host.size() * sizeof(double2));
  if (e != cudaSuccess) return fail(kOutOfMemory, "FFT table allocation failed");
  e = cudaMemcpy(dp->mem, host.data(), host.size() * sizeof(double2), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(kCudaError, std::string("FFT table upload: ") + cudaGetErrorString(e));
  P.half = dp->mem + half_at;
  if (rader) {
    P.rroots = dp->mem + rader_at;
    P.rkern = dp->mem + rader_at + (n - 1);
    e = cudaMalloc(&dp->imem, perm.size() * sizeof(int));
    if (e != cudaSuccess) return fail(kOutOfMemory, "FFT table allocation failed");
    e = cudaMemcpy(dp->imem, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(kCudaError, std::string("FFT table upload: ") + cudaGetErrorString(e));
    P.rperm = dp->imem;
  }
  if (!P.blue) {
    P.roots = dp->mem;
  } else {
    P.mroots = dp->mem;
    P.chirp = dp->mem + P.m;
    P.kern = dp->mem + P.m + n;
  }
  *out = P;
  D->ffts[key] = std::move(dp);
  return kOk;
}

// Weight-convolution kernel: wr[r] = (2 pi / Pc) sum_p w(p) e^{+2 pi i p r / Pc},
// w(p) = int_0^pi e^{-i p theta} sin(theta) d theta (reference
// src/c/so3_sampling.c:32-51), |p| <= 2(L-1).
// Tables of the forward beta stage (stages.cu), per (L, sampling), Pc + 2L
// complex entries:
//  [0, Pc)        2 pi / Pc * DFT(w_e): the spectrum of the even part of the
//                 quadrature weights w_e(p) = 2 / (1 - p^2) (even p, |p| <=
//                 2(L-1)) that the paired columns are convolved with (real);
//  [Pc, Pc + L)   h_0(m'): the stage's output for the odd (s = -1) column of
//                 a unit sample at its first self-mirror beta row (MW: row
//                 L-1 at beta = pi; MWSS: row 0 at beta = 0), with the full
//                 weights w (so3_sampling.c:32-51);
//  [Pc + L, Pc + 2L) h_1(m'): the same for MWSS row L (beta = pi); zero for MW;
//  [Pc + 2L, 2 Pc + 2L) 4 pi^2 / Pc * DFT(w) of the full weights (the
//                 convolution of the adjoint forward transform).
// h(m') = G(m') - G(-m') (m' >= 1), G(0), with G = 2 pi v * w and v(m'') =
// e^{-i m'' beta} / P, m'' in [-(L-1), L-1].
int ensure_conv_kernel(Device* D, const Geometry& g, const double2** out) {
  const int key = 2 * g.L + (g.mw ? 1 : 0);
  auto it = D->conv_kernels.find(key);
  if (it != D->conv_kernels.end()) {
    *out = it->second;
    return kOk;
  }
  const int Pc = g.Pc, L = g.L, P = g.P;
  auto weight = [&](long long p) -> cld {
    if (p > 2LL * (L - 1) || p < -2LL * (L - 1)) return cld(0, 0);
    if (p == 1) return cld(0, -kPiL / 2);
    if (p == -1) return cld(0, kPiL / 2);
    if (p % 2 != 0) return cld(0, 0);
    return cld(2.0L / (1.0L - (long double)p * p), 0);
  };
  std::vector<cld> w(Pc, cld(0, 0));
  for (int p = -2 * (L - 1); p <= 2 * (L - 1); p += 2) w[((p % Pc) + Pc) % Pc] += weight(p);
  fft_ld(w, +1);
  std::vector<double2> host(2 * (size_t)Pc + 2 * (size_t)L, make_double2(0.0, 0.0));
  {
    std::vector<cld> wf(Pc, cld(0, 0));
    for (int p = -2 * (L - 1); p <= 2 * (L - 1); p++) wf[((p % Pc) + Pc) % Pc] += weight(p);
    fft_ld(wf, -1);  // forward DFT
    for (int r = 0; r < Pc; r++) {
      const cld v = wf[r] * (4.0L * kPiL * kPiL / (long double)Pc);
      host[(size_t)Pc + 2 * (size_t)L + r] = make_double2((double)v.real(), (double)v.imag());
    }
  }
  for (int r = 0; r < Pc; r++) {
    // w_e is real and even: its spectrum is real
    const long double v = w[r].real() * (2.0L * kPiL / (long double)Pc);
    host[r] = make_double2((double)v, 0.0);
  }
  // correction vectors: v(m'') = (+1 or (-1)^{m''}) / P
  for (int which = 0; which < (g.mw ? 1 : 2); which++) {
    const bool alternating = g.mw || which == 1;  // beta = pi
    std::vector<cld> G(2 * (size_t)L - 1);
    for (int mp = -(L - 1); mp <= L - 1; mp++) {
      cld acc(0, 0);
      for (int mpp = -(L - 1); mpp <= L - 1; mpp++) {
        const long double v = ((alternating && (mpp & 1)) ? -1.0L : 1.0L) / (long double)P;
        acc += v * weight((long long)mp - mpp);
      }
      G[mp + L - 1] = acc * (2.0L * kPiL);
    }
    for (int mp = 0; mp < L; mp++) {
      const cld h = mp == 0 ? G[L - 1] : G[mp + L - 1] - G[L - 1 - mp];
      host[(size_t)Pc + (size_t)which * L + mp] = make_double2((double)h.real(), (double)h.imag());
    }
  }
  double2* d = nullptr;
  if (cudaMalloc(&d, host.size() * sizeof(double2)) != cudaSuccess)
    return fail(kOutOfMemory, "beta-stage weight table allocation failed");
  SO3G_CUDA(cudaMemcpy(d, host.data(), host.size() * sizeof(double2), cudaMemcpyHostToDevice));
  D->conv_kernels[key] = d;
  *out = d;
  return kOk;
}

int ensure_bases(Device* D, const so3_parameters_t& p, int real, const long long** out) {
  char key[128];
  snprintf(key, sizeof key, "%d/%d/%d/%d/%d", p.L, p.N, (int)p.storage, (int)p.n_order, real);
  auto it = D->bases.find(key);
  if (it != D->bases.end()) {
    *out = it->second;
    return kOk;
  }
  std::vector<long long> b = block_bases(p, real);
  long long* d = nullptr;
  if (cudaMalloc(&d, b.size() * sizeof(long long)) != cudaSuccess) return fail(kOutOfMemory, "base table allocation failed");
  SO3G_CUDA(cudaMemcpy(d, b.data(), b.size() * sizeof(long long), cudaMemcpyHostToDevice));
  D->bases[key] = d;
  *out = d;
  return kOk;
}

}  // namespace so3g
