// so3gpu_inverse_noalloc: the complex inverse Wigner transform for callers
// that cannot allocate device memory -- code that runs where cudaMalloc is
// not allowed (inside a stream-ordered section that must not synchronise the
// device, under an allocator or memory cap owned by someone else, or in a
// real-time loop that forbids allocation after start-up).  It never calls
// cudaMalloc, cudaFree or any allocating routine: the transform scratch, the
// Wigner Delta(pi/2) tables, the FFT tables and the block-offset table live
// in the file-scope device arrays below, which every GPU that loads the
// library holds until the process exits: kStaticBytes = 35,089,464 bytes
// (33.5 MiB), of which 32 MiB are scratch.
//
// Limits: complex, non-steerable signals only (reality != 0 or steerable !=
// 0: status 3, before any device work -- a real signal's buffers are sized
// for the real layout, which this entry point does not handle); transform
// scratch of at most kScratchBytes (32 MiB; MW or MWSS sampling with L <= 64
// and N <= 64 always fits), L <= kMaxL, N <= kMaxN.  Larger requests are
// rejected with status 3 and a message.
//
// Set-up: the first call in a CUDA context (the device's primary context, as
// the runtime API uses it) resolves the arrays' device addresses with
// cudaGetSymbolAddress and builds the Delta tables on the call's stream, then
// waits for them; make that first call before any stream capture.  The set-up
// is keyed by the context's unique id, so a call from a new context (after
// cudaDeviceReset, or a context made with the driver API) sets up again.  A
// later call whose band limits, storage or n-order differ from the previous
// call's uploads new FFT and offset tables from host memory with
// cudaMemcpyAsync; make such calls outside capture too (a captured region may
// only repeat the configuration of the call before it).
//
// Every call shares the arrays and leaves the last call's contents behind;
// each call writes every scratch entry before it reads it, so nothing needs
// clearing.  Calls whose GPU work overlaps (different streams, or different
// host threads) race on the shared arrays: serialise them.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda.h>

#include "so3gpu.h"
#include "so3gpu_internal.h"

namespace so3g {
namespace {

constexpr size_t kScratchBytes = 32u << 20;
constexpr int kMaxL = 64;
constexpr int kMaxN = 64;
constexpr int kDlEntries = kMaxL * (kMaxL + 1) * (2 * kMaxL + 1) / 6;
constexpr int kRisboWork = 2 * (kMaxL + 6) * (kMaxL + 6);
constexpr int kFftSlot = 2 * 256 + 2 * 128;  // Bluestein m + n + m, then n half-step roots, for n <= 128
constexpr int kMaxPlanes = 2 * kMaxN - 1;

static __device__ __align__(256) double2 g_scratch[kScratchBytes / sizeof(double2)];
static __device__ __align__(256) double g_dl[2][kDlEntries];
static __device__ __align__(256) double g_risbo_work[kRisboWork];
static __device__ __align__(256) double2 g_fft[2][kFftSlot];
static __device__ __align__(256) long long g_bases[kMaxPlanes];
constexpr size_t kStaticBytes = kScratchBytes + sizeof(double) * (2 * (size_t)kDlEntries + kRisboWork) +
                                sizeof(double2) * 2 * kFftSlot + sizeof(long long) * kMaxPlanes;
static_assert(kStaticBytes == 35089464, "the documented size of the static arrays");

struct NoAllocDevice {
  bool ready = false;
  unsigned long long ctx_id = 0;  // context the set-up ran in
  double2* scratch = nullptr;
  double* dl[2] = {nullptr, nullptr};
  double* risbo_work = nullptr;
  double2* fft = nullptr;
  long long* bases = nullptr;
  FftPlan plan[2]{};
  int plan_n[2] = {0, 0};
  char bases_key[64] = {0};
  // host images of the uploaded tables (no heap use per call)
  double2 host_fft[2][kFftSlot];
  long long host_bases[kMaxPlanes];
};

std::mutex g_mu;
NoAllocDevice g_state[64];

typedef std::complex<long double> cld;
const long double kPiL = 3.141592653589793238462643383279502884L;

cld root_l(long long num, long long den) {  // e^{-2 pi i num/den}
  const long double a = 2.0L * kPiL * (long double)num / (long double)den;
  return cld(cosl(a), -sinl(a));
}

int factor_small(int n, int* rad) {  // same radix order as the allocating planner
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

// radix-2 FFT in long double on a fixed-size host array (m <= 256)
void fft_ld_fixed(cld* x, int n, int sign) {
  for (int i = 1, j = 0; i < n; i++) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(x[i], x[j]);
  }
  for (int len = 2; len <= n; len <<= 1)
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < len / 2; k++) {
        cld w = root_l(k, len);
        if (sign > 0) w = std::conj(w);
        const cld u = x[i + k], v = x[i + k + len / 2] * w;
        x[i + k] = u + v;
        x[i + k + len / 2] = u - v;
      }
}

// Half-step roots e^{-i pi k/n} of a plan, at slot offset `at`.
void half_table(int n, FftPlan* P, double2* h, const double2* dev, int at) {
  for (int k = 0; k < n; k++) {
    const cld r = root_l(k, 2LL * n);
    h[at + k] = make_double2((double)r.real(), (double)r.imag());
  }
  P->half = dev + at;
}

// Fills plan tables for length n into host slot h; device pointers point at dev.
void plan_tables(int n, FftPlan* P, double2* h, const double2* dev) {
  *P = FftPlan{};
  P->n = n;
  const int np = factor_small(n, P->rad);
  if (np >= 0) {
    P->npass = np;
    for (int k = 0; k < n; k++) {
      const cld r = root_l(k, n);
      h[k] = make_double2((double)r.real(), (double)r.imag());
    }
    P->roots = dev;
    half_table(n, P, h, dev, n);
    return;
  }
  int m = 1;
  while (m < 2 * n - 1) m <<= 1;
  P->blue = 1;
  P->m = m;
  P->mpass = factor_small(m, P->mrad);
  for (int k = 0; k < m; k++) {
    const cld r = root_l(k, m);
    h[k] = make_double2((double)r.real(), (double)r.imag());
  }
  cld ch[128];
  cld ker[256];
  for (int k = 0; k < n; k++) {
    ch[k] = root_l(((long long)k * k) % (2LL * n), 2LL * n);
    h[m + k] = make_double2((double)ch[k].real(), (double)ch[k].imag());
  }
  for (int k = 0; k < m; k++) ker[k] = cld(0, 0);
  ker[0] = std::conj(ch[0]);
  for (int k = 1; k < n; k++) ker[k] = ker[m - k] = std::conj(ch[k]);
  fft_ld_fixed(ker, m, -1);
  for (int k = 0; k < m; k++) {
    const cld v = ker[k] / (long double)m;
    h[m + n + k] = make_double2((double)v.real(), (double)v.imag());
  }
  P->mroots = dev;
  P->chirp = dev + m;
  P->kern = dev + m + n;
  half_table(n, P, h, dev, 2 * m + n);
}

// Unique id of the calling thread's current CUDA context, through the driver
// entry points the runtime exposes (the library does not link libcuda).
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
int current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0, q1;
    SO3G_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0));
    SO3G_CUDA(cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1));
    if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
      return fail(kCudaError, "so3gpu_inverse_noalloc: driver entry points cuCtxGetCurrent / cuCtxGetId missing");
    get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
    get_id = reinterpret_cast<CtxGetIdFn>(f1);
  }
  CUcontext c = nullptr;
  if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, id) != CUDA_SUCCESS)
    return fail(kCudaError, "so3gpu_inverse_noalloc: no current CUDA context");
  return kOk;
}

int setup_device(NoAllocDevice& S, cudaStream_t s) {
  // resolving a symbol makes the runtime's context current if no call has yet
  void* probe = nullptr;
  SO3G_CUDA(cudaGetSymbolAddress(&probe, g_scratch));
  unsigned long long id = 0;
  if (int rc = current_context_id(&id)) return rc;
  if (S.ready && S.ctx_id == id) return kOk;
  // first call in this context: nothing cached from another context is valid
  S.ready = false;
  S.plan_n[0] = S.plan_n[1] = 0;
  S.bases_key[0] = 0;
  SO3G_CUDA(cudaGetSymbolAddress((void**)&S.scratch, g_scratch));
  SO3G_CUDA(cudaGetSymbolAddress((void**)&S.dl[0], g_dl));
  S.dl[1] = S.dl[0] + kDlEntries;
  SO3G_CUDA(cudaGetSymbolAddress((void**)&S.risbo_work, g_risbo_work));
  SO3G_CUDA(cudaGetSymbolAddress((void**)&S.fft, g_fft));
  SO3G_CUDA(cudaGetSymbolAddress((void**)&S.bases, g_bases));
  if (int rc = launch_build_dl_risbo(S.dl[SSHT_DL_RISBO], kMaxL, S.risbo_work, s)) return rc;
  if (int rc = launch_build_dl_trapani(S.dl[SSHT_DL_TRAPANI], 0, kMaxL, s)) return rc;
  SO3G_CUDA(cudaStreamSynchronize(s));
  S.ctx_id = id;
  S.ready = true;
  return kOk;
}

int run(void* f, const void* flmn, const so3_parameters_t* p, cudaStream_t s) {
  if (!p || !f || !flmn) return fail(kInvalidParameter, "null argument");
  // checked before anything else: the buffers of a real signal are sized for
  // the real layout, which this entry point does not handle
  if (p->reality != 0) return fail(kUnsupported, "so3gpu_inverse_noalloc: complex signals only (reality = 0)");
  if (p->steerable != 0) return fail(kUnsupported, "so3gpu_inverse_noalloc: steerable signals are not supported");
  if (int rc = validate(*p, 0)) return rc;
  if (p->L > kMaxL || p->N > kMaxN)
    return fail(kUnsupported, "so3gpu_inverse_noalloc: L <= 64 and N <= 64 only");
  if (workspace_bytes(*p, 0) > kScratchBytes)
    return fail(kUnsupported, "so3gpu_inverse_noalloc: transform scratch exceeds the 32 MiB static array");
  int dev = 0;
  SO3G_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(kUnsupported, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  NoAllocDevice& S = g_state[dev];
  if (int rc = setup_device(S, s)) return rc;
  const Geometry g = make_geometry(*p, 0);
  const int lens[2] = {g.P, g.ng};
  for (int i = 0; i < 2; i++) {
    if (S.plan_n[i] != lens[i]) {
      double2* dev_slot = S.fft + (size_t)i * kFftSlot;
      plan_tables(lens[i], &S.plan[i], S.host_fft[i], dev_slot);
      SO3G_CUDA(cudaMemcpyAsync(dev_slot, S.host_fft[i], sizeof(double2) * kFftSlot, cudaMemcpyHostToDevice, s));
      S.plan_n[i] = lens[i];
    }
  }
  char key[64];
  snprintf(key, sizeof key, "%d/%d/%d/%d", p->L, p->N, (int)p->storage, (int)p->n_order);
  if (strcmp(key, S.bases_key) != 0) {
    const std::vector<long long> b = block_bases(*p, 0);
    for (size_t i = 0; i < b.size(); i++) S.host_bases[i] = b[i];
    SO3G_CUDA(cudaMemcpyAsync(S.bases, S.host_bases, sizeof(long long) * b.size(), cudaMemcpyHostToDevice, s));
    strcpy(S.bases_key, key);
  }
  double2* W = S.scratch;
  const double* dl = S.dl[p->dl_method];
  if (int rc = launch_inverse_contract(g, p->n_mode, static_cast<const double2*>(flmn), S.bases, dl, W, 0, s))
    return rc;
  if (int rc = launch_inv_beta(g, S.plan[0], W, s)) return rc;
  if (int rc = launch_inv_alpha(g, S.plan[0], W, s)) return rc;
  return launch_inv_gamma(g, S.plan[1], W, f, s);
}

}  // namespace
}  // namespace so3g

extern "C" int so3gpu_inverse_noalloc(void* f, const void* flmn, const so3_parameters_t* parameters,
                                      void* stream) {
  const int rc = so3g::run(f, flmn, parameters, (cudaStream_t)stream);
  so3g_record_status(rc);
  return rc;
}
