// Transform drivers: stage order of the inverse and forward Wigner transforms
// on device pointers.  Host code only; every kernel runs on stream s.
#include <cstdlib>

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

int prepare(Device* D, const so3_parameters_t& p, int real, cudaStream_t s) {
  Resources r;
  return acquire(D, p, real, s, &r, true);
}

int run_inverse(Device* D, Workspace* wk, const so3_parameters_t& p, const void* flmn_d, void* f_d, int real,
                cudaStream_t s) {
  Resources r;
  if (int rc = acquire(D, p, real, s, &r, false)) return rc;
  void* ws = nullptr;
  if (int rc = ensure_ws(wk, workspace_bytes(p, real), &ws)) return rc;
  double2* W = static_cast<double2*>(ws);
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

}  // namespace so3g
