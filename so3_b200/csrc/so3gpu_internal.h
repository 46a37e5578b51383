// Internal declarations shared by the CUDA translation units of libso3gpu.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "fft_core.cuh"
#include "so3/so3_types.h"

namespace so3g {

// ---------------------------------------------------------------- errors
// Status codes returned by every internal entry point.
enum Status : int {
  kOk = 0,
  kInvalidParameter = 1,
  kCudaError = 2,
  kUnsupported = 3,
  kOutOfMemory = 4,
};
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);  // records msg, returns code
#define SO3G_CUDA(call)                                                               \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return ::so3g::fail(::so3g::kCudaError, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Counter of kernel launches issued by this library (all devices).
extern std::atomic<long long> g_launches;
#define SO3G_LAUNCHED() (::so3g::g_launches.fetch_add(1, std::memory_order_relaxed))

// ---------------------------------------------------------------- geometry
// Scratch of one transform, two parts, complex FP64.  Plane index = n +
// plane0 (plane0 = N-1 for complex signals, 0 for real ones, which keep
// n >= 0 only); column index c = m + L - 1.
//  * row-major part W[plane][row][col] at the workspace start: col stride 1,
//    row stride RS (>= 2L, multiple of 8 so every row starts on a 128-byte
//    boundary), plane stride PS = RS * nb.  Rows are beta samples (after the
//    beta stage) and the alpha / gamma stages work on it.
//  * column-major part Wc[plane][col][m'] at offset QOFF = nplanes * PS:
//    m' stride 1, column stride CS (>= L, multiple of 8), plane stride QS =
//    CS * (2L - 1).  It holds the beta-Fourier spectra F(n, m', m) between a
//    contraction and a beta stage, so that both read and write whole columns
//    contiguously; the beta stages transpose between the two parts.
struct Geometry {
  int L, N, L0;
  int mw;       // 1 MW, 0 MWSS
  int real;     // reality flag of the transform being run
  int na, nb;   // alpha / beta samples
  int P;        // DFT length over alpha and over the extended beta circle (= na)
  int ng;       // gamma DFT length: 2N-1, or 2N for steerable signals
  int nf;       // gamma samples of the caller's f: 2N-1, or N for steerable signals
  int steer;    // steerable signal (complex only): supersampled gamma axis
  int nplanes;  // 2N-1 (complex) or N (real)
  int plane0;
  long RS, PS;
  long CS, QS, QOFF;  // column-major part (see above)
  int Pc;       // weight-convolution length (power of two >= 4L-3)
  // Kernel variant of each DFT stage (index = Stage below; 0 = default),
  // chosen by the autotuner for this geometry.
  signed char var[8];
};
Geometry make_geometry(const so3_parameters_t& p, int real);

// Plane index -> "virtual base" offset into the caller's flmn array, such that
// element (l, m, n) sits at base[n] + l*l + l + m (entries with l < |n| are
// absent in compact storage).  Encodes storage and n-order.
std::vector<long long> block_bases(const so3_parameters_t& p, int real);

// ---------------------------------------------------------------- tables
// Quarter Delta(pi/2) planes of every degree l < Lcap, plane l at offset
// l(l+1)(2l+1)/6, row-major (m' rows, m columns, both 0..l).  Planes do not
// depend on the band limit, so one table serves every L <= Lcap.
struct DlTable {
  int Lcap = 0;
  double* d = nullptr;
};
__host__ __device__ inline long long dl_plane_offset(int l) {
  return (long long)l * (l + 1) * (2 * l + 1) / 6;
}

struct DevPlan {
  FftPlan plan{};
  double2* mem = nullptr;  // owns roots/mroots/chirp/kern/half/rroots/rkern
  int* imem = nullptr;     // owns rperm
};

// Resident int8 digits of the split-precision contractions' Delta products
// for one (L, N, Delta recursion); see mixed.cu.
struct DigitTable {
  int L = 0, N = 0, method = -1;
  uint8_t* d = nullptr;
  long long* pair_off = nullptr;
  size_t bytes = 0;
};

// Resident int8 digits of the forward beta stage's real matrices R_s for one
// L (MW sampling); see mixed.cu.
struct BetaTable {
  int L = 0;
  uint8_t* d = nullptr;
  double rscale = 1.0;
  size_t bytes = 0;
};

struct Device {
  int device = 0;
  std::mutex mu;
  std::map<std::string, std::vector<signed char>> tuned;  // stage variants by geometry key
  DlTable dl[2];                                 // per dl_method
  std::map<int, std::unique_ptr<DevPlan>> ffts;  // by length
  std::map<int, double2*> conv_kernels;          // forward-beta weight tables by 2L + (MW)
  std::map<std::string, long long*> bases;       // block bases by parameter key
  std::vector<std::unique_ptr<DigitTable>> digit_tables;
  std::map<long long, int> digit_uses;  // split-precision calls per (L, N, recursion) without a table
  std::vector<std::unique_ptr<BetaTable>> beta_tables;
  std::map<int, int> beta_uses;  // split-precision forward calls per L without a beta table
};

// Per-stage CUDA-event timing (optional, per caller context).
enum Stage : int {
  kStInvContract = 0,
  kStInvBeta,
  kStInvAlpha,
  kStInvGamma,
  kStFwdGamma,
  kStFwdAlpha,
  kStFwdBetaConv,
  kStFwdContract,
  kStMixInv,  // split-precision contraction (slicing + tensor-core products), inverse
  kStMixFwd,  // split-precision contraction, forward
  kStMixFwdBeta,  // split-precision forward beta stage (slicing + tensor-core products)
  kStCount = 16
};
struct StageTimer {
  bool on = false;
  std::vector<cudaEvent_t> pool;  // free events
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  double total_ms[kStCount] = {};
  long long count[kStCount] = {};
};
// Marks the start of `stage` on stream s; call mark_end after the launch.
void timer_begin(StageTimer* t, cudaStream_t s, cudaEvent_t* ev);
void timer_end(StageTimer* t, cudaStream_t s, int stage, cudaEvent_t start);
int timer_collect(StageTimer* t);  // synchronises on the recorded events

// Grow-only device scratch owned by one caller context (never shared between
// contexts, so contexts on different streams do not race).
struct Workspace {
  void* ws = nullptr;
  size_t ws_bytes = 0;
  bool borrowed = false;  // ws is owned by the caller (never reallocated or freed here)
  StageTimer timer;
};
Device* device_state(int device);  // lazily created per CUDA device

int ensure_dl(Device* D, int L, int method, cudaStream_t s, const double** out);
int ensure_fft(Device* D, int n, FftPlan* out);
int ensure_conv_kernel(Device* D, const Geometry& g, const double2** out);
int ensure_bases(Device* D, const so3_parameters_t& p, int real, const long long** out);
int ensure_ws(Workspace* W, size_t bytes, void** out);
size_t workspace_bytes(const so3_parameters_t& p, int real);
// Device bytes of the resident per-device tables (Delta tables, digit and
// beta tables, weight tables, DFT plans, block bases).
size_t resident_bytes(Device* D);

// ---------------------------------------------------------------- launches
int launch_build_dl_trapani(double* table, int L0cap, int Lcap, cudaStream_t s);
int launch_build_dl_risbo(double* table, int Lcap, double* work, cudaStream_t s);

struct ModeInfo {
  int n_mode;  // so3_n_mode_t
  int N;
};
__host__ __device__ inline bool plane_skipped(int mode, int N, int n) {
  if (mode == SO3_N_MODE_EVEN) return (n & 1) != 0;
  if (mode == SO3_N_MODE_ODD) return (n & 1) == 0;
  if (mode == SO3_N_MODE_MAXIMUM) return (n < 0 ? -n : n) < N - 1;
  return false;
}

// nu_lo/nu_hi restrict a launch to the planes with |n| in [nu_lo, nu_hi)
// (nu_hi < 0: up to N); ranges split at even |n| so CTAs never straddle.
// wconst > 0 replaces the inverse's per-degree weight (2l+1)/(8 pi^2) by a
// constant; lw > 0 multiplies the forward's outputs by lw (2l+1) (the
// adjoint transforms).
int launch_inverse_contract(const Geometry& g, int n_mode, const double2* flmn, const long long* bases,
                            const double* dl, double2* W, int sym_n0, cudaStream_t s, int nu_lo = 0,
                            int nu_hi = -1, double wconst = 0.0);
int launch_forward_contract(const Geometry& g, int n_mode, const double2* W, const long long* bases,
                            const double* dl, double2* flmn, int storage_compact, cudaStream_t s, int nu_lo = 0,
                            int nu_hi = -1, double lw = 0.0);

int launch_inv_beta(const Geometry& g, const FftPlan& pP, double2* W, cudaStream_t s);
int launch_inv_alpha(const Geometry& g, const FftPlan& pP, double2* W, cudaStream_t s);
// row_lo/row_hi restrict the gamma stages to the beta rows [row_lo, row_hi)
// (row_hi < 0: up to nb).
int launch_inv_gamma(const Geometry& g, const FftPlan& pg, const double2* W, void* f, cudaStream_t s,
                     int row_lo = 0, int row_hi = -1);
int launch_fwd_gamma(const Geometry& g, const FftPlan& pg, const void* f, double2* W, cudaStream_t s,
                     int row_lo = 0, int row_hi = -1);
int launch_fwd_alpha(const Geometry& g, const FftPlan& pP, double2* W, cudaStream_t s);
int launch_fwd_beta_conv(const Geometry& g, const FftPlan& pP, const FftPlan& pc, const double2* wr,
                         double2* W, cudaStream_t s);

// Beta stages of the adjoint transforms (MW, complex; stages.cu).  Inverse
// adjoint: per column of the row-major part, zero-extend the nb beta samples
// onto the 2L-1 circle, DFT, phase e^{-i m' pi/(2L-1)}, fold F(m') +
// (-1)^{m+n} F(-m') onto m' >= 0 into the column-major part.  Forward
// adjoint: per column of the column-major part, extend G(-m') = (-1)^{m+n}
// G(m'), convolve with 4 pi^2 w (table wr), phase e^{+i m'' pi/(2L-1)},
// inverse DFT / (2L-1), fold the periodic extension back onto the L beta
// samples into the row-major part.
int launch_adj_inv_beta(const Geometry& g, const FftPlan& pP, double2* W, cudaStream_t s);
int launch_adj_fwd_beta(const Geometry& g, const FftPlan& pP, const FftPlan& pc, const double2* wr, double2* W,
                        cudaStream_t s);
int launch_s2toso3(const so3_parameters_t& hp, const long long* bases, const double2* flm, const double2* glm,
                   double2* hlmn, cudaStream_t s);
int launch_harmonic_convolution(const so3_parameters_t& hp, const so3_parameters_t& fp,
                                const so3_parameters_t& gp, const long long* hb, const long long* fb,
                                const long long* gb, const double2* flmn, const double2* glmn, double2* hlmn,
                                cudaStream_t s);
int launch_zero(void* p, size_t bytes, cudaStream_t s);

// Autotuner of the DFT stages: times every kernel variant of each stage on
// the workspace W (its contents are scratch; results are discarded) and
// writes the fastest into g->var.  Synchronises stream s: never call it while
// s is being captured.  reps timed launches per variant after one warm-up.
int autotune_stages(Geometry* g, const FftPlan& pP, const FftPlan& pg, const FftPlan& pc, const double2* wr,
                    double2* W, cudaStream_t s, int reps);
// Number of kernel variants the tuner can choose from for a stage.
int stage_variants(const Geometry& g, const FftPlan& pP, const FftPlan& pg, const FftPlan& pc, int stage);

// Split-precision (int8 tensor-core) contractions of a batch of complex
// signals sharing one parameter set.  flmn_dev / W: per-signal coefficient
// pointers (a device array of nsig pointers) and scratch planes (signal b at
// W + b * wstride); scratch: mixed_scratch_bytes(g, nsig) bytes.
size_t mixed_scratch_bytes(const Geometry& g, int nsig);
// force: build now instead of on the geometry's second call.
int ensure_digit_table(Device* D, const Geometry& g, int method, const double* dl, cudaStream_t s,
                       const DigitTable** out, bool force = false);
size_t digit_table_bytes(int L, int N);
// Forward beta stage of a split-precision batch as an int8 tensor-core
// product (complex MW signals; W: row-major scratch of signal 0, output into
// the column-major parts).
bool mixed_beta_supported(const Geometry& g);
int ensure_beta_table(Device* D, const Geometry& g, cudaStream_t s, const BetaTable** out);
int launch_mixed_fwd_beta(const Geometry& g, double2* W, long long wstride, int nsig, const BetaTable* tab,
                          void* scratch, cudaStream_t s);
// tab: resident digits of (g.L, g.N) or null (digits generated from dl).
// conv_flm / conv_glm (device array of nsig kernel pointers): when set, the
// coefficients of signal b are the directional convolution h_lmn = flm_lm
// conj(glm_b,ln) 8 pi^2/(2l+1), computed on load (flmn_dev unused).
int launch_mixed_inverse(const Geometry& g, int n_mode, const double2* const* flmn_dev, int nsig,
                         const long long* bases, const double* dl, const DigitTable* tab, double2* W,
                         long long wstride, void* scratch, cudaStream_t s, const double2* conv_flm = nullptr,
                         const double2* const* conv_glm = nullptr);
int launch_mixed_forward(const Geometry& g, int n_mode, const double2* W, long long wstride, int nsig,
                         const long long* bases, const double* dl, const DigitTable* tab, double2* const* flmn_dev,
                         int storage_compact, void* scratch, cudaStream_t s);
// One signal of a ragged split-precision batch (complex; any L, N, L0,
// storage, n-order, n-mode; one Delta recursion per launch).
struct RaggedSig {
  const void* flmn;        // inverse: coefficients in; forward: coefficients out (device)
  double2* Wc;             // column-major part of the signal's scratch (inverse out, forward in)
  const long long* base;   // block bases of its parameters (device)
  Geometry g;
  int n_mode, compact;
};
// Scratch of a ragged contraction (stage images of the groups of 16 similar
// signals, their column scales and the descriptor tables).
size_t ragged_scratch_bytes(const std::vector<RaggedSig>& sigs, bool fwd);
// Slicing and tensor-core products of every signal in two launches; dl: the
// Delta table of the batch's recursion, covering the largest L.
int launch_mixed_ragged(bool fwd, const std::vector<RaggedSig>& sigs, const double* dl, const DigitTable* tab,
                        void* scratch, cudaStream_t s);
// Resident digit table covering (L, N) for a recursion (see mixed.cu), built
// at L = 512, N = 64 when `build` and none covers; null: digits generated.
const DigitTable* covering_digit_table(Device* D, int L, int N, int method, const double* dl, bool build,
                                       cudaStream_t s);
// Reads and clears the flag the tensor-core kernels set when a bounded wait
// gave up (0: none; synchronous).
int mixed_take_error();

// ---------------------------------------------------------------- drivers
// Per-thread switch of the stage autotuner (default on).
void set_thread_autotune(bool on);
// Contraction arithmetic of a batch: FP64 (the reference-exact path) or the
// int8 split (complex signals only; real signals always use FP64).
enum Precision : int { kPrecFp64 = 0, kPrecMixedInt8 = 1 };
// Lock-protected creation of the per-device read-only resources a transform
// with parameters p needs; safe to call before stream capture.
// Tuned / pinned stage variants of a geometry (get: 1 if known, else 0).
// Variants beyond a stage's count fall back to its default kernel.
int get_stage_variants(Device* D, const so3_parameters_t& p, int real, int* var);
int set_stage_variants(Device* D, const so3_parameters_t& p, int real, const int* var);
// With a workspace it also sizes the workspace and tunes the stage kernels
// for this geometry (both synchronise s, so prepare before stream capture).
int prepare(Device* D, const so3_parameters_t& p, int real, cudaStream_t s, Workspace* wk = nullptr);
int run_inverse(Device* D, Workspace* wk, const so3_parameters_t& p, const void* flmn_d, void* f_d, int real,
                cudaStream_t s);
int run_forward(Device* D, Workspace* wk, const so3_parameters_t& p, const void* f_d, void* flmn_d, int real,
                cudaStream_t s);
// Workspace bytes a batch of nsig signals needs (run_*_batch).
size_t batch_workspace_bytes(const so3_parameters_t& p, int real, int nsig, int precision);
// Batches: f_d / flmn_d are host arrays of nsig device pointers.
int run_inverse_batch(Device* D, Workspace* wk, const so3_parameters_t& p, int real, int nsig,
                      const void* const* flmn_d, void* const* f_d, int precision, cudaStream_t s);
int run_forward_batch(Device* D, Workspace* wk, const so3_parameters_t& p, int real, int nsig, const void* const* f_d,
                      void* const* flmn_d, int precision, cudaStream_t s);
// Batches of signals with one parameter set each (ps[b]; any L, N, L0,
// sampling, storage, n-order, n-mode, recursion).  Split precision: every
// complex signal's contraction runs in one ragged tensor-core launch per
// Delta recursion; real signals and precision FP64 run the FP64 path per
// signal.
int run_inverse_ragged(Device* D, Workspace* wk, const so3_parameters_t* ps, int nsig, const void* const* flmn_d,
                       void* const* f_d, int precision, cudaStream_t s);
int run_forward_ragged(Device* D, Workspace* wk, const so3_parameters_t* ps, int nsig, const void* const* f_d,
                       void* const* flmn_d, int precision, cudaStream_t s);
// Adjoint transforms (complex MW): flmn <- A_inverse^H f and f <- A_forward^H
// flmn, device pointers, on stream s.
int run_adjoint_inverse(Device* D, Workspace* wk, const so3_parameters_t& p, const void* f_d, void* flmn_d,
                        cudaStream_t s);
int run_adjoint_forward(Device* D, Workspace* wk, const so3_parameters_t& p, const void* flmn_d, void* f_d,
                        cudaStream_t s);
// Workspace bytes of a split-precision ragged call (complex signals).
size_t ragged_workspace_bytes(const so3_parameters_t* ps, int nsig, bool fwd);
// Directional convolutions of one S^2 signal flm with nsig kernels glm_d[b]
// (so3_conv_s2toso3_harmonic_convolution with h parameters p) followed by the
// inverse transform into f_d[b] (complex signals).  FP64: hlmn of each kernel
// in the workspace, then the FP64 inverse.  Split precision: h is computed in
// the contraction's operand load and never stored.
int run_conv_inverse_batch(Device* D, Workspace* wk, const so3_parameters_t& p, int nsig, const void* flm_d,
                           const void* const* glm_d, void* const* f_d, int precision, cudaStream_t s);

// Drop-in calls on caller buffers that may live in host memory: the
// transform runs in chunks (|n| ranges for the contractions, beta-row ranges
// for the gamma stages) so that the host<->device copies of one chunk overlap
// the kernels of the others.  host_in / host_out are the caller's host
// buffers (nullptr when that side is already device memory); dev_in / dev_out
// are the device buffers the kernels use.  Copies run on cin / cout, ordered
// against the compute stream s by events; the caller synchronises cout and s.
constexpr int kMaxChunks = 8;
struct StagedIo {
  const void* host_in = nullptr;
  void* host_out = nullptr;
  const void* dev_in = nullptr;
  void* dev_out = nullptr;
  cudaStream_t cin = nullptr, cout = nullptr;
  cudaEvent_t ev[2 * kMaxChunks] = {};
};
int run_inverse_staged(Device* D, Workspace* wk, const so3_parameters_t& p, int real, const StagedIo& io,
                       cudaStream_t s);
// zero_first: clear the whole coefficient array first (skipped n-blocks read
// back as zero); otherwise skipped blocks of a host output keep the caller's
// contents, as in the reference.
int run_forward_staged(Device* D, Workspace* wk, const so3_parameters_t& p, int real, bool zero_first,
                       const StagedIo& io, cudaStream_t s);

const std::string& last_error();
int validate(const so3_parameters_t& p, int real);

}  // namespace so3g

// Records the status of the calling thread's last call (so3gpu_last_status).
void so3g_record_status(int rc);
