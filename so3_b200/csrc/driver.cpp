// Transform drivers: stage order of the inverse and forward Wigner transforms
// on device pointers.  Host code only; every kernel runs on stream s.
#include <algorithm>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "so3/so3_sampling.h"
#include "so3gpu_internal.h"

namespace so3g {

struct Resources {
  Geometry g;
  const double* dl = nullptr;
  FftPlan pP{}, pg{}, pc{};
  const long long* bases = nullptr;
  const double2* wr = nullptr;
};

static int acquire(Device* D, const so3_parameters_t& p, int real, cudaStream_t s, Resources* r, bool conv) {
  if (int rc = validate(p, real)) return rc;
  r->g = make_geometry(p, real);
  std::lock_guard<std::mutex> lk(D->mu);
  if (int rc = ensure_dl(D, p.L, p.dl_method, s, &r->dl)) return rc;
  if (int rc = ensure_fft(D, r->g.P, &r->pP)) return rc;
  if (int rc = ensure_fft(D, r->g.ng, &r->pg)) return rc;
  if (int rc = ensure_bases(D, p, real, &r->bases)) return rc;
  if (conv) {
    if (int rc = ensure_fft(D, r->g.Pc, &r->pc)) return rc;
    if (int rc = ensure_conv_kernel(D, r->g, &r->wr)) return rc;
  }
  return kOk;
}

static std::string tune_key(const so3_parameters_t& p, int real) {
  return std::to_string(p.L) + "/" + std::to_string(p.N) + "/" + std::to_string((int)p.sampling_scheme) + "/" +
         std::to_string(real) + "/" + std::to_string(p.steerable ? 1 : 0);
}

// Threads that must not stop for tuning (the request server's worker) use
// the default stage variants for geometries nobody has tuned yet.
static thread_local bool t_no_autotune = false;
void set_thread_autotune(bool on) { t_no_autotune = !on; }

// Stage variants for this geometry: cached per device, else measured on the
// workspace (skipped while s is being captured, on threads that disabled it,
// and when the environment sets SO3GPU_AUTOTUNE=0; defaults are used then).
static int ensure_tuned(Device* D, const so3_parameters_t& p, int real, Resources* r, double2* W, cudaStream_t s) {
  const std::string key = tune_key(p, real);
  {
    std::lock_guard<std::mutex> lk(D->mu);
    auto it = D->tuned.find(key);
    if (it != D->tuned.end()) {
      for (int i = 0; i < 8; i++) r->g.var[i] = it->second[i];
      return kOk;
    }
  }
  if (t_no_autotune) return kOk;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  SO3G_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) return kOk;
  const char* env = getenv("SO3GPU_AUTOTUNE");
  Geometry g = r->g;
  if (!(env && env[0] == '0')) {
    FftPlan pc{};
    const double2* wr = nullptr;
    {
      std::lock_guard<std::mutex> lk(D->mu);
      if (int rc = ensure_fft(D, g.Pc, &pc)) return rc;
      if (int rc = ensure_conv_kernel(D, g, &wr)) return rc;
    }
    if (int rc = autotune_stages(&g, r->pP, r->pg, pc, wr, W, s, 3)) return rc;
  }
  std::lock_guard<std::mutex> lk(D->mu);
  D->tuned[key] = std::vector<signed char>(g.var, g.var + 8);
  for (int i = 0; i < 8; i++) r->g.var[i] = g.var[i];
  return kOk;
}

int get_stage_variants(Device* D, const so3_parameters_t& p, int real, int* var) {
  std::lock_guard<std::mutex> lk(D->mu);
  auto it = D->tuned.find(tune_key(p, real));
  if (it == D->tuned.end()) return 0;
  for (int i = 0; i < 8; i++) var[i] = it->second[i];
  return 1;
}

int set_stage_variants(Device* D, const so3_parameters_t& p, int real, const int* var) {
  std::vector<signed char> v(8);
  for (int i = 0; i < 8; i++) {
    if (var[i] < 0 || var[i] > 7) return fail(kInvalidParameter, "stage variant out of range");
    v[i] = (signed char)var[i];
  }
  std::lock_guard<std::mutex> lk(D->mu);
  D->tuned[tune_key(p, real)] = v;
  return kOk;
}

int prepare(Device* D, const so3_parameters_t& p, int real, cudaStream_t s, Workspace* wk) {
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, true)) return rc;
  if (!wk) return kOk;
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, workspace_bytes(p, real), &ws)) return rc;
  return ensure_tuned(D, p, real, &r, static_cast<double2*>(ws), s);
}

int run_inverse(Device* D, Workspace* wk, const so3_parameters_t& p, const void* flmn_d, void* f_d, int real,
                cudaStream_t s) {
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, false)) return rc;
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, workspace_bytes(p, real), &ws)) return rc;
  double2* W = static_cast<double2*>(ws);
  if (int rc = ensure_tuned(D, p, real, &r, W, s)) return rc;
  const int sym_n0 = real && p.N == 1;
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  int rc;
  timer_begin(T, s, &ev);
  rc = launch_inverse_contract(r.g, p.n_mode, static_cast<const double2*>(flmn_d), r.bases, r.dl, W, sym_n0, s);
  if (rc) return rc;
  timer_end(T, s, kStInvContract, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_inv_beta(r.g, r.pP, W, s))) return rc;
  timer_end(T, s, kStInvBeta, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_inv_alpha(r.g, r.pP, W, s))) return rc;
  timer_end(T, s, kStInvAlpha, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_inv_gamma(r.g, r.pg, W, f_d, s))) return rc;
  timer_end(T, s, kStInvGamma, ev);
  return kOk;
}

int run_forward(Device* D, Workspace* wk, const so3_parameters_t& p, const void* f_d, void* flmn_d, int real,
                cudaStream_t s) {
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, true)) return rc;
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, workspace_bytes(p, real), &ws)) return rc;
  double2* W = static_cast<double2*>(ws);
  if (int rc = ensure_tuned(D, p, real, &r, W, s)) return rc;
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  int rc;
  timer_begin(T, s, &ev);
  if ((rc = launch_fwd_gamma(r.g, r.pg, f_d, W, s))) return rc;
  timer_end(T, s, kStFwdGamma, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_fwd_alpha(r.g, r.pP, W, s))) return rc;
  timer_end(T, s, kStFwdAlpha, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_fwd_beta_conv(r.g, r.pP, r.pc, r.wr, W, s))) return rc;
  timer_end(T, s, kStFwdBetaConv, ev);
  timer_begin(T, s, &ev);
  rc = launch_forward_contract(r.g, p.n_mode, W, r.bases, r.dl, static_cast<double2*>(flmn_d),
                               p.storage == SO3_STORAGE_COMPACT, s);
  if (rc) return rc;
  timer_end(T, s, kStFwdContract, ev);
  return kOk;
}

// ------------------------------------------------------------ staged drop-in
namespace {

typedef std::vector<std::pair<long long, long long>> Ranges;

// Element ranges [begin, end) of the coefficient blocks of the planes with |n|
// in [nu_lo, nu_hi), merged where adjacent.  Block n holds l >= |n| (compact)
// or l >= 0 (padded) up to L-1, element (l, m) at base[n] + l*l + l + m.
Ranges block_ranges(const std::vector<long long>& base, const Geometry& g, int compact, int n_mode, int nu_lo,
                    int nu_hi, bool skip_inactive) {
  Ranges r;
  const long long L2 = (long long)g.L * g.L;
  for (int nu = nu_lo; nu < nu_hi; nu++)
    for (int neg = 0; neg < (g.real ? 1 : 2); neg++) {
      if (neg && nu == 0) continue;
      const int n = neg ? -nu : nu;
      if (skip_inactive && plane_skipped(n_mode, g.N, n)) continue;
      const long long b = base[g.plane0 + n];
      r.push_back({b + (compact ? (long long)nu * nu : 0), b + L2});
    }
  std::sort(r.begin(), r.end());
  Ranges m;
  for (const auto& x : r) {
    if (!m.empty() && m.back().second == x.first)
      m.back().second = x.second;
    else
      m.push_back(x);
  }
  return m;
}

// Size from which a staged side is split into chunks (64 MiB; the
// environment variable SO3GPU_STAGE_CHUNK_BYTES overrides it, which the tests
// use to exercise the chunked path at small sizes).
size_t chunk_threshold() {
  const char* e = getenv("SO3GPU_STAGE_CHUNK_BYTES");
  if (e && *e) return (size_t)strtoull(e, nullptr, 10);
  return size_t(64) << 20;
}

// Chunk boundaries b[0] = 0 < ... < b[k] = total, interior ones multiples of
// align; returns k (1 when the data are too small for overlap to pay).
int split(int total, size_t bytes, int align, int* b) {
  int k = bytes > 0 && bytes >= chunk_threshold() ? kMaxChunks : 1;
  int nb = 0;
  b[nb++] = 0;
  for (int i = 1; i < k; i++) {
    int v = (int)((long long)total * i / k);
    v -= v % align;
    if (v > b[nb - 1] && v < total) b[nb++] = v;
  }
  b[nb] = total;
  return nb;
}

int copy_blocks(void* dst, const void* src, const Ranges& r, cudaMemcpyKind kind, cudaStream_t s) {
  for (const auto& x : r)
    SO3G_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + x.first * 16, static_cast<const char*>(src) + x.first * 16,
                              (size_t)(x.second - x.first) * 16, kind, s));
  return kOk;
}

// beta rows [r0, r1) of every gamma plane of a sample array f[g][b][a]
int copy_rows(void* dst, const void* src, const Geometry& g, int r0, int r1, cudaMemcpyKind kind, cudaStream_t s) {
  const size_t es = g.real ? sizeof(double) : sizeof(double2);
  const size_t pitch = (size_t)g.nb * g.na * es, off = (size_t)r0 * g.na * es;
  SO3G_CUDA(cudaMemcpy2DAsync(static_cast<char*>(dst) + off, pitch, static_cast<const char*>(src) + off, pitch,
                              (size_t)(r1 - r0) * g.na * es, g.nf, kind, s));
  return kOk;
}

}  // namespace

int run_inverse_staged(Device* D, Workspace* wk, const so3_parameters_t& p, int real, const StagedIo& io,
                       cudaStream_t s) {
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, false)) return rc;
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, workspace_bytes(p, real), &ws)) return rc;
  double2* W = static_cast<double2*>(ws);
  if (int rc = ensure_tuned(D, p, real, &r, W, s)) return rc;
  const Geometry& g = r.g;
  const int sym_n0 = real && p.N == 1;
  const int compact = p.storage == SO3_STORAGE_COMPACT;
  const std::vector<long long> base = block_bases(p, real);
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  int rc;
  int nb[kMaxChunks + 1], rb[kMaxChunks + 1];
  const size_t in_bytes = (size_t)g.nplanes * g.L * g.L * 16;
  const int kn = split(g.N, io.host_in ? in_bytes : 0, 2, nb);
  timer_begin(T, s, &ev);
  for (int k = 0; k < kn; k++) {
    if (io.host_in) {
      const Ranges cr = block_ranges(base, g, compact, p.n_mode, nb[k], nb[k + 1], true);
      if ((rc = copy_blocks(const_cast<void*>(io.dev_in), io.host_in, cr, cudaMemcpyHostToDevice, io.cin))) return rc;
      SO3G_CUDA(cudaEventRecord(io.ev[k], io.cin));
      SO3G_CUDA(cudaStreamWaitEvent(s, io.ev[k], 0));
    }
    rc = launch_inverse_contract(g, p.n_mode, static_cast<const double2*>(io.dev_in), r.bases, r.dl, W, sym_n0, s,
                                 nb[k], nb[k + 1]);
    if (rc) return rc;
  }
  timer_end(T, s, kStInvContract, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_inv_beta(g, r.pP, W, s))) return rc;
  timer_end(T, s, kStInvBeta, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_inv_alpha(g, r.pP, W, s))) return rc;
  timer_end(T, s, kStInvAlpha, ev);
  const size_t out_bytes = (size_t)g.nf * g.nb * g.na * (g.real ? 8 : 16);
  const int kr = split(g.nb, io.host_out ? out_bytes : 0, 1, rb);
  timer_begin(T, s, &ev);
  for (int k = 0; k < kr; k++) {
    if ((rc = launch_inv_gamma(g, r.pg, W, io.dev_out, s, rb[k], rb[k + 1]))) return rc;
    if (io.host_out) SO3G_CUDA(cudaEventRecord(io.ev[kMaxChunks + k], s));
  }
  timer_end(T, s, kStInvGamma, ev);
  if (io.host_out)
    for (int k = 0; k < kr; k++) {
      SO3G_CUDA(cudaStreamWaitEvent(io.cout, io.ev[kMaxChunks + k], 0));
      if ((rc = copy_rows(io.host_out, io.dev_out, g, rb[k], rb[k + 1], cudaMemcpyDeviceToHost, io.cout))) return rc;
    }
  return kOk;
}

int run_forward_staged(Device* D, Workspace* wk, const so3_parameters_t& p, int real, bool zero_first,
                       const StagedIo& io, cudaStream_t s) {
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, true)) return rc;
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, workspace_bytes(p, real), &ws)) return rc;
  double2* W = static_cast<double2*>(ws);
  if (int rc = ensure_tuned(D, p, real, &r, W, s)) return rc;
  const Geometry& g = r.g;
  const int compact = p.storage == SO3_STORAGE_COMPACT;
  const std::vector<long long> base = block_bases(p, real);
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  int rc;
  int nb[kMaxChunks + 1], rb[kMaxChunks + 1];
  const size_t in_bytes = (size_t)g.nf * g.nb * g.na * (g.real ? 8 : 16);
  const int kr = split(g.nb, io.host_in ? in_bytes : 0, 1, rb);
  timer_begin(T, s, &ev);
  for (int k = 0; k < kr; k++) {
    if (io.host_in) {
      if ((rc = copy_rows(const_cast<void*>(io.dev_in), io.host_in, g, rb[k], rb[k + 1], cudaMemcpyHostToDevice,
                          io.cin)))
        return rc;
      SO3G_CUDA(cudaEventRecord(io.ev[k], io.cin));
      SO3G_CUDA(cudaStreamWaitEvent(s, io.ev[k], 0));
    }
    if ((rc = launch_fwd_gamma(g, r.pg, io.dev_in, W, s, rb[k], rb[k + 1]))) return rc;
  }
  timer_end(T, s, kStFwdGamma, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_fwd_alpha(g, r.pP, W, s))) return rc;
  timer_end(T, s, kStFwdAlpha, ev);
  timer_begin(T, s, &ev);
  if ((rc = launch_fwd_beta_conv(g, r.pP, r.pc, r.wr, W, s))) return rc;
  timer_end(T, s, kStFwdBetaConv, ev);
  if (zero_first) {
    const Ranges all = block_ranges(base, g, compact, p.n_mode, 0, g.N, false);
    long long hi = 0;
    for (const auto& x : all) hi = std::max(hi, x.second);
    SO3G_CUDA(cudaMemsetAsync(io.dev_out, 0, (size_t)hi * 16, s));
  }
  const size_t out_bytes = (size_t)g.nplanes * g.L * g.L * 16;
  const int kn = split(g.N, io.host_out ? out_bytes : 0, 2, nb);
  timer_begin(T, s, &ev);
  for (int k = 0; k < kn; k++) {
    rc = launch_forward_contract(g, p.n_mode, W, r.bases, r.dl, static_cast<double2*>(io.dev_out), compact, s,
                                 nb[k], nb[k + 1]);
    if (rc) return rc;
    if (io.host_out) SO3G_CUDA(cudaEventRecord(io.ev[kMaxChunks + k], s));
  }
  timer_end(T, s, kStFwdContract, ev);
  if (io.host_out)
    for (int k = 0; k < kn; k++) {
      SO3G_CUDA(cudaStreamWaitEvent(io.cout, io.ev[kMaxChunks + k], 0));
      const Ranges cr = block_ranges(base, g, compact, p.n_mode, nb[k], nb[k + 1], !zero_first);
      if ((rc = copy_blocks(io.host_out, io.dev_out, cr, cudaMemcpyDeviceToHost, io.cout))) return rc;
    }
  return kOk;
}

// ------------------------------------------------------------ batches
namespace {

// Workspace layout of a split-precision batch: nsig scratch plane sets, the
// sliced operand, and the table of per-signal coefficient pointers.
struct BatchLayout {
  size_t wbytes, scratch_off, table_off, total;
};
BatchLayout batch_layout(const Geometry& g, const so3_parameters_t& p, int real, int nsig) {
  BatchLayout b;
  b.wbytes = (workspace_bytes(p, real) + 255) & ~size_t(255);
  b.scratch_off = b.wbytes * nsig;
  b.table_off = b.scratch_off + ((mixed_scratch_bytes(g, nsig) + 255) & ~size_t(255));
  b.total = b.table_off + sizeof(void*) * (size_t)nsig;
  return b;
}

// The pointer table is copied from pageable host memory: cudaMemcpyAsync has
// staged the bytes by the time it returns (the DMA itself stays ordered on s),
// so the host vector may go and the host does not wait for earlier work on s.
int upload_table(void* dst, const void* const* ptrs, int nsig, cudaStream_t s) {
  std::vector<const void*> host(ptrs, ptrs + nsig);
  SO3G_CUDA(cudaMemcpyAsync(dst, host.data(), sizeof(void*) * (size_t)nsig, cudaMemcpyHostToDevice, s));
  return kOk;
}

}  // namespace

// Real signals take the split contractions too (planes n >= 0, the tensor-core
// columns of the combinations with n = -nu stay empty), except N = 1, whose
// FP64 inverse symmetrises the single plane (the reference's real spin
// transform for n = 0).
static bool split_real_ok(const so3_parameters_t& p, int real) { return !real || p.N > 1; }

size_t batch_workspace_bytes(const so3_parameters_t& p, int real, int nsig, int precision) {
  if (precision == kPrecFp64 || !split_real_ok(p, real) || nsig <= 0) return workspace_bytes(p, real);
  return batch_layout(make_geometry(p, real), p, real, nsig).total;
}

int run_inverse_batch(Device* D, Workspace* wk, const so3_parameters_t& p, int real, int nsig,
                      const void* const* flmn_d, void* const* f_d, int precision, cudaStream_t s) {
  if (nsig < 0) return fail(kInvalidParameter, "negative batch size");
  if (precision != kPrecFp64 && precision != kPrecMixedInt8) return fail(kInvalidParameter, "unknown precision");
  if (precision == kPrecFp64 || !split_real_ok(p, real)) {
    for (int b = 0; b < nsig; b++)
      if (int rc = run_inverse(D, wk, p, flmn_d[b], f_d[b], real, s)) return rc;
    return kOk;
  }
  if (nsig == 0) return kOk;
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, false)) return rc;
  const BatchLayout bl = batch_layout(r.g, p, real, nsig);
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, bl.total, &ws)) return rc;
  char* base = static_cast<char*>(ws);
  double2* W = reinterpret_cast<double2*>(base);
  if (int rc = ensure_tuned(D, p, real, &r, W, s)) return rc;
  if (int rc = upload_table(base + bl.table_off, flmn_d, nsig, s)) return rc;
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  int rc;
  const long long wstride = (long long)(bl.wbytes / sizeof(double2));
  const DigitTable* tab = nullptr;
  if ((rc = ensure_digit_table(D, r.g, p.dl_method, r.dl, s, &tab))) return rc;
  timer_begin(T, s, &ev);
  rc = launch_mixed_inverse(r.g, p.n_mode, reinterpret_cast<const double2* const*>(base + bl.table_off), nsig, r.bases,
                            r.dl, tab, W, wstride, base + bl.scratch_off, s);
  if (rc) return rc;
  timer_end(T, s, kStMixInv, ev);
  for (int b = 0; b < nsig; b++) {
    double2* Wb = W + (size_t)b * wstride;
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_beta(r.g, r.pP, Wb, s))) return rc;
    timer_end(T, s, kStInvBeta, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_alpha(r.g, r.pP, Wb, s))) return rc;
    timer_end(T, s, kStInvAlpha, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_gamma(r.g, r.pg, Wb, f_d[b], s))) return rc;
    timer_end(T, s, kStInvGamma, ev);
  }
  return kOk;
}

int run_forward_batch(Device* D, Workspace* wk, const so3_parameters_t& p, int real, int nsig, const void* const* f_d,
                      void* const* flmn_d, int precision, cudaStream_t s) {
  if (nsig < 0) return fail(kInvalidParameter, "negative batch size");
  if (precision != kPrecFp64 && precision != kPrecMixedInt8) return fail(kInvalidParameter, "unknown precision");
  if (precision == kPrecFp64 || !split_real_ok(p, real)) {
    for (int b = 0; b < nsig; b++)
      if (int rc = run_forward(D, wk, p, f_d[b], flmn_d[b], real, s)) return rc;
    return kOk;
  }
  if (nsig == 0) return kOk;
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, true)) return rc;
  const BatchLayout bl = batch_layout(r.g, p, real, nsig);
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, bl.total, &ws)) return rc;
  char* base = static_cast<char*>(ws);
  double2* W = reinterpret_cast<double2*>(base);
  if (int rc = ensure_tuned(D, p, real, &r, W, s)) return rc;
  if (int rc = upload_table(base + bl.table_off, flmn_d, nsig, s)) return rc;
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  int rc;
  const long long wstride = (long long)(bl.wbytes / sizeof(double2));
  // forward beta stage: one tensor-core product over the whole batch where
  // supported (complex MW) and its matrix table is resident, else the FP64
  // DFT + weight convolution per signal
  const BetaTable* bt = nullptr;
  if (mixed_beta_supported(r.g) && (rc = ensure_beta_table(D, r.g, s, &bt))) return rc;
  for (int b = 0; b < nsig; b++) {
    double2* Wb = W + (size_t)b * wstride;
    timer_begin(T, s, &ev);
    if ((rc = launch_fwd_gamma(r.g, r.pg, f_d[b], Wb, s))) return rc;
    timer_end(T, s, kStFwdGamma, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_fwd_alpha(r.g, r.pP, Wb, s))) return rc;
    timer_end(T, s, kStFwdAlpha, ev);
    if (bt) continue;
    timer_begin(T, s, &ev);
    if ((rc = launch_fwd_beta_conv(r.g, r.pP, r.pc, r.wr, Wb, s))) return rc;
    timer_end(T, s, kStFwdBetaConv, ev);
  }
  if (bt) {
    timer_begin(T, s, &ev);
    if ((rc = launch_mixed_fwd_beta(r.g, W, wstride, nsig, bt, base + bl.scratch_off, s))) return rc;
    timer_end(T, s, kStMixFwdBeta, ev);
  }
  const DigitTable* tab = nullptr;
  if ((rc = ensure_digit_table(D, r.g, p.dl_method, r.dl, s, &tab))) return rc;
  timer_begin(T, s, &ev);
  rc = launch_mixed_forward(r.g, p.n_mode, W, wstride, nsig, r.bases, r.dl, tab,
                            reinterpret_cast<double2* const*>(base + bl.table_off), p.storage == SO3_STORAGE_COMPACT,
                            base + bl.scratch_off, s);
  if (rc) return rc;
  timer_end(T, s, kStMixFwd, ev);
  return kOk;
}

int run_conv_inverse_batch(Device* D, Workspace* wk, const so3_parameters_t& p, int nsig, const void* flm_d,
                           const void* const* glm_d, void* const* f_d, int precision, cudaStream_t s) {
  if (nsig < 0) return fail(kInvalidParameter, "negative batch size");
  if (precision != kPrecFp64 && precision != kPrecMixedInt8) return fail(kInvalidParameter, "unknown precision");
  if (p.reality) return fail(kUnsupported, "directional convolutions produce complex signals");
  if (nsig == 0) return kOk;
  Resources r;
  if (int rc = acquire(D, p, 0, s, &r, false)) return rc;
  int rc;
  if (precision == kPrecFp64) {
    // hlmn of each kernel after the transform's scratch; run_inverse keeps the (larger) workspace
    const size_t wb = (workspace_bytes(p, 0) + 255) & ~size_t(255);
    void* ws = nullptr;
    if ((rc = ensure_ws(wk, wb + (size_t)so3_sampling_flmn_size(&p) * sizeof(double2), &ws))) return rc;
    double2* h = reinterpret_cast<double2*>(static_cast<char*>(ws) + wb);
    for (int b = 0; b < nsig; b++) {
      if ((rc = launch_s2toso3(p, r.bases, static_cast<const double2*>(flm_d), static_cast<const double2*>(glm_d[b]),
                               h, s)))
        return rc;
      if ((rc = run_inverse(D, wk, p, h, f_d[b], 0, s))) return rc;
    }
    return kOk;
  }
  const BatchLayout bl = batch_layout(r.g, p, 0, nsig);
  void* ws = nullptr;
  if ((rc = ensure_ws(wk, bl.total, &ws))) return rc;
  char* base = static_cast<char*>(ws);
  double2* W = reinterpret_cast<double2*>(base);
  if ((rc = ensure_tuned(D, p, 0, &r, W, s))) return rc;
  if ((rc = upload_table(base + bl.table_off, glm_d, nsig, s))) return rc;
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  const long long wstride = (long long)(bl.wbytes / sizeof(double2));
  const DigitTable* tab = nullptr;
  if ((rc = ensure_digit_table(D, r.g, p.dl_method, r.dl, s, &tab))) return rc;
  timer_begin(T, s, &ev);
  rc = launch_mixed_inverse(r.g, p.n_mode, nullptr, nsig, r.bases, r.dl, tab, W, wstride, base + bl.scratch_off, s,
                            static_cast<const double2*>(flm_d),
                            reinterpret_cast<const double2* const*>(base + bl.table_off));
  if (rc) return rc;
  timer_end(T, s, kStMixInv, ev);
  for (int b = 0; b < nsig; b++) {
    double2* Wb = W + (size_t)b * wstride;
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_beta(r.g, r.pP, Wb, s))) return rc;
    timer_end(T, s, kStInvBeta, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_alpha(r.g, r.pP, Wb, s))) return rc;
    timer_end(T, s, kStInvAlpha, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_gamma(r.g, r.pg, Wb, f_d[b], s))) return rc;
    timer_end(T, s, kStInvGamma, ev);
  }
  return kOk;
}

// ------------------------------------------------------------ ragged batches
namespace {

// Per-signal state of a ragged batch.
struct RagItem {
  int idx;  // position in the caller's arrays
  Resources r;
  size_t ws_off;
};

// Signals of a ragged split-precision batch: complex ones go to the
// tensor-core contraction (per Delta recursion), real ones to the FP64 path.
int ragged_prepare(Device* D, const so3_parameters_t* ps, int nsig, bool conv_tables, cudaStream_t s,
                   std::vector<RagItem>* items, std::vector<int>* fp64) {
  int Lmax[2] = {0, 0};
  for (int i = 0; i < nsig; i++) {
    if (int rc = validate(ps[i], ps[i].reality != 0)) return rc;
    if (!ps[i].reality) Lmax[ps[i].dl_method] = std::max(Lmax[ps[i].dl_method], ps[i].L);
  }
  {
    // Delta tables to the largest L first, so no later call regrows them
    std::lock_guard<std::mutex> lk(D->mu);
    const double* t;
    for (int m = 0; m < 2; m++)
      if (Lmax[m] > 0)
        if (int rc = ensure_dl(D, Lmax[m], m, s, &t)) return rc;
  }
  size_t off = 0;
  for (int i = 0; i < nsig; i++) {
    if (ps[i].reality) {
      fp64->push_back(i);
      continue;
    }
    RagItem it;
    it.idx = i;
    if (int rc = acquire(D, ps[i], 0, s, &it.r, conv_tables)) return rc;
    it.ws_off = off;
    off += (workspace_bytes(ps[i], 0) + 255) & ~size_t(255);
    items->push_back(it);
  }
  return kOk;
}

size_t ragged_ws_end(const std::vector<RagItem>& items, const so3_parameters_t* ps) {
  return items.empty() ? 0 : items.back().ws_off + ((workspace_bytes(ps[items.back().idx], 0) + 255) & ~size_t(255));
}

}  // namespace

size_t ragged_workspace_bytes(const so3_parameters_t* ps, int nsig, bool fwd) {
  size_t sig = 0;
  std::vector<RaggedSig> rs[2];
  for (int i = 0; i < nsig; i++) {
    if (ps[i].reality) continue;
    sig += (workspace_bytes(ps[i], 0) + 255) & ~size_t(255);
    RaggedSig r{};
    r.g = make_geometry(ps[i], 0);
    rs[ps[i].dl_method & 1].push_back(r);
  }
  return sig + std::max(ragged_scratch_bytes(rs[0], fwd), ragged_scratch_bytes(rs[1], fwd));
}

int run_inverse_ragged(Device* D, Workspace* wk, const so3_parameters_t* ps, int nsig, const void* const* flmn_d,
                       void* const* f_d, int precision, cudaStream_t s) {
  if (nsig < 0) return fail(kInvalidParameter, "negative batch size");
  if (precision != kPrecFp64 && precision != kPrecMixedInt8) return fail(kInvalidParameter, "unknown precision");
  if (precision == kPrecFp64) {
    for (int b = 0; b < nsig; b++)
      if (int rc = run_inverse(D, wk, ps[b], flmn_d[b], f_d[b], ps[b].reality != 0, s)) return rc;
    return kOk;
  }
  std::vector<RagItem> items;
  std::vector<int> fp64;
  if (int rc = ragged_prepare(D, ps, nsig, false, s, &items, &fp64)) return rc;
  for (int i : fp64)  // real signals: the FP64 path, before the batch workspace is laid out
    if (int rc = run_inverse(D, wk, ps[i], flmn_d[i], f_d[i], 1, s)) return rc;
  if (items.empty()) return kOk;
  const size_t sig_end = ragged_ws_end(items, ps);
  std::vector<RaggedSig> rs[2];
  for (const RagItem& it : items) {
    RaggedSig r;
    r.flmn = flmn_d[it.idx];
    r.Wc = nullptr;  // set once the workspace exists
    r.base = it.r.bases;
    r.g = it.r.g;
    r.n_mode = ps[it.idx].n_mode;
    r.compact = ps[it.idx].storage == SO3_STORAGE_COMPACT;
    rs[ps[it.idx].dl_method].push_back(r);
  }
  const size_t rag = std::max(ragged_scratch_bytes(rs[0], false), ragged_scratch_bytes(rs[1], false));
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, sig_end + rag, &ws)) return rc;
  char* wsb = static_cast<char*>(ws);
  int rc;
  {
    int k[2] = {0, 0};
    for (RagItem& it : items) {
      double2* W = reinterpret_cast<double2*>(wsb + it.ws_off);
      if ((rc = ensure_tuned(D, ps[it.idx], 0, &it.r, W, s))) return rc;
      rs[ps[it.idx].dl_method][k[ps[it.idx].dl_method]++].Wc = W + it.r.g.QOFF;
    }
  }
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  for (int m = 0; m < 2; m++) {
    if (rs[m].empty()) continue;
    const double* dl = nullptr;
    {
      std::lock_guard<std::mutex> lk(D->mu);
      if ((rc = ensure_dl(D, 1, m, s, &dl))) return rc;  // current table (already large enough)
    }
    int Lm = 0, Nm = 0;
    for (const RaggedSig& r : rs[m]) Lm = std::max(Lm, r.g.L), Nm = std::max(Nm, r.g.N);
    const DigitTable* tab = covering_digit_table(D, Lm, Nm, m, dl, true, s);
    timer_begin(T, s, &ev);
    if ((rc = launch_mixed_ragged(false, rs[m], dl, tab, wsb + sig_end, s))) return rc;
    timer_end(T, s, kStMixInv, ev);
  }
  for (const RagItem& it : items) {
    double2* W = reinterpret_cast<double2*>(wsb + it.ws_off);
    const Resources& r = it.r;
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_beta(r.g, r.pP, W, s))) return rc;
    timer_end(T, s, kStInvBeta, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_alpha(r.g, r.pP, W, s))) return rc;
    timer_end(T, s, kStInvAlpha, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_inv_gamma(r.g, r.pg, W, f_d[it.idx], s))) return rc;
    timer_end(T, s, kStInvGamma, ev);
  }
  return kOk;
}

int run_forward_ragged(Device* D, Workspace* wk, const so3_parameters_t* ps, int nsig, const void* const* f_d,
                       void* const* flmn_d, int precision, cudaStream_t s) {
  if (nsig < 0) return fail(kInvalidParameter, "negative batch size");
  if (precision != kPrecFp64 && precision != kPrecMixedInt8) return fail(kInvalidParameter, "unknown precision");
  if (precision == kPrecFp64) {
    for (int b = 0; b < nsig; b++)
      if (int rc = run_forward(D, wk, ps[b], f_d[b], flmn_d[b], ps[b].reality != 0, s)) return rc;
    return kOk;
  }
  std::vector<RagItem> items;
  std::vector<int> fp64;
  if (int rc = ragged_prepare(D, ps, nsig, true, s, &items, &fp64)) return rc;
  for (int i : fp64)
    if (int rc = run_forward(D, wk, ps[i], f_d[i], flmn_d[i], 1, s)) return rc;
  if (items.empty()) return kOk;
  const size_t sig_end = ragged_ws_end(items, ps);
  std::vector<RaggedSig> rs[2];
  for (const RagItem& it : items) {
    RaggedSig r;
    r.flmn = flmn_d[it.idx];
    r.Wc = nullptr;
    r.base = it.r.bases;
    r.g = it.r.g;
    r.n_mode = ps[it.idx].n_mode;
    r.compact = ps[it.idx].storage == SO3_STORAGE_COMPACT;
    rs[ps[it.idx].dl_method].push_back(r);
  }
  const size_t rag = std::max(ragged_scratch_bytes(rs[0], true), ragged_scratch_bytes(rs[1], true));
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, sig_end + rag, &ws)) return rc;
  char* wsb = static_cast<char*>(ws);
  int rc;
  StageTimer* T = &wk->timer;
  cudaEvent_t ev;
  int k[2] = {0, 0};
  for (RagItem& it : items) {
    double2* W = reinterpret_cast<double2*>(wsb + it.ws_off);
    if ((rc = ensure_tuned(D, ps[it.idx], 0, &it.r, W, s))) return rc;
    const Resources& r = it.r;
    rs[ps[it.idx].dl_method][k[ps[it.idx].dl_method]++].Wc = W + r.g.QOFF;
    timer_begin(T, s, &ev);
    if ((rc = launch_fwd_gamma(r.g, r.pg, f_d[it.idx], W, s))) return rc;
    timer_end(T, s, kStFwdGamma, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_fwd_alpha(r.g, r.pP, W, s))) return rc;
    timer_end(T, s, kStFwdAlpha, ev);
    timer_begin(T, s, &ev);
    if ((rc = launch_fwd_beta_conv(r.g, r.pP, r.pc, r.wr, W, s))) return rc;
    timer_end(T, s, kStFwdBetaConv, ev);
  }
  for (int m = 0; m < 2; m++) {
    if (rs[m].empty()) continue;
    const double* dl = nullptr;
    {
      std::lock_guard<std::mutex> lk(D->mu);
      if ((rc = ensure_dl(D, 1, m, s, &dl))) return rc;
    }
    int Lm = 0, Nm = 0;
    for (const RaggedSig& r : rs[m]) Lm = std::max(Lm, r.g.L), Nm = std::max(Nm, r.g.N);
    const DigitTable* tab = covering_digit_table(D, Lm, Nm, m, dl, true, s);
    timer_begin(T, s, &ev);
    if ((rc = launch_mixed_ragged(true, rs[m], dl, tab, wsb + sig_end, s))) return rc;
    timer_end(T, s, kStMixFwd, ev);
  }
  return kOk;
}

// ------------------------------------------------------------ adjoint transforms
// Adjoints of the inverse and forward transforms (reference
// src/c/so3_adjoint.c:34-400, :402-938 complex; :939-1312, :1313-1841 real,
// MW).  The reference's FFT normalisations are folded into one contraction
// weight: the adjoint inverse's analysis DFTs over gamma and alpha carry
// 2 pi/(2N-1) and 1/(2L-1) (the forward stages'), undone in the forward
// contraction's (2l+1)/(8 pi^2) weight; the adjoint forward's
// 1/((2L-1)(2N-1)) rides on the inverse contraction.  Real signals: planes
// n >= 0, r2c over gamma in the adjoint inverse (the reference's 2-D r2c over
// alpha and gamma), c2r in the adjoint forward (its 2-D c2r: the inverse DFT
// over alpha, then c2r over gamma with the imaginary part of n = 0 dropped).
static int adjoint_check(const so3_parameters_t& p) {
  if (int rc = validate(p, p.reality ? 1 : 0)) return rc;
  if (p.sampling_scheme != SO3_SAMPLING_MW) return fail(kUnsupported, "adjoint transforms: MW sampling only");
  if (p.steerable) return fail(kUnsupported, "adjoint transforms: steerable signals are not supported");
  return kOk;
}

int run_adjoint_inverse(Device* D, Workspace* wk, const so3_parameters_t& p, const void* f_d, void* flmn_d,
                        cudaStream_t s) {
  if (int rc = adjoint_check(p)) return rc;
  const int real = p.reality ? 1 : 0;
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, false)) return rc;
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, workspace_bytes(p, real), &ws)) return rc;
  double2* W = static_cast<double2*>(ws);
  if (int rc = ensure_tuned(D, p, real, &r, W, s)) return rc;
  // every coefficient starts at zero (so3_adjoint.c:234-243): skipped n-blocks and l < L0 stay zero
  SO3G_CUDA(cudaMemsetAsync(flmn_d, 0, (size_t)so3_sampling_flmn_size(&p) * sizeof(double2), s));
  int rc;
  if ((rc = launch_fwd_gamma(r.g, r.pg, f_d, W, s))) return rc;
  if ((rc = launch_fwd_alpha(r.g, r.pP, W, s))) return rc;
  if ((rc = launch_adj_inv_beta(r.g, r.pP, W, s))) return rc;
  const double kPi = 3.141592653589793238462643383279502884;
  const double lw = (double)(2 * p.N - 1) * (2 * p.L - 1) / (16.0 * kPi * kPi * kPi);  // (2l+1)/(8pi^2) (2N-1)(2L-1)/(2pi)
  return launch_forward_contract(r.g, p.n_mode, W, r.bases, r.dl, static_cast<double2*>(flmn_d),
                                 p.storage == SO3_STORAGE_COMPACT, s, 0, -1, lw);
}

int run_adjoint_forward(Device* D, Workspace* wk, const so3_parameters_t& p, const void* flmn_d, void* f_d,
                        cudaStream_t s) {
  if (int rc = adjoint_check(p)) return rc;
  const int real = p.reality ? 1 : 0;
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, true)) return rc;
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, workspace_bytes(p, real), &ws)) return rc;
  double2* W = static_cast<double2*>(ws);
  if (int rc = ensure_tuned(D, p, real, &r, W, s)) return rc;
  int rc;
  const double wconst = 1.0 / ((double)(2 * p.L - 1) * (2 * p.N - 1));
  if ((rc = launch_inverse_contract(r.g, p.n_mode, static_cast<const double2*>(flmn_d), r.bases, r.dl, W, 0, s, 0,
                                    -1, wconst)))
    return rc;
  if ((rc = launch_adj_fwd_beta(r.g, r.pP, r.pc, r.wr, W, s))) return rc;
  if ((rc = launch_inv_alpha(r.g, r.pP, W, s))) return rc;
  return launch_inv_gamma(r.g, r.pg, W, f_d, s);
}

}  // namespace so3g
