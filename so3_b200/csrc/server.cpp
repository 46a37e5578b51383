// Request-serving loop: inverse, forward and directional-convolution requests
// of mixed (L, N) submitted from any host thread, run on one GPU with
// continuous batching.
//
//  * Slots: up to max_inflight requests (or batches) are on the device at
//    once, each on its own CUDA stream with its own scratch, so their kernels
//    overlap.  A request that arrives while others run is admitted as soon as
//    a slot and memory free up; it never waits for the running ones to end.
//  * Memory admission: the budget covers the device's resident tables (Delta,
//    digit, beta and weight tables, plans), the scratch of the units in flight
//    and the callers' input and output buffers of those units.  Scratch comes
//    from the stream-ordered allocator (cudaMallocAsync / cudaFreeAsync on
//    the slot's stream), so admitting and retiring work never synchronises
//    the device.  A request that cannot fit beside the resident tables
//    fails with status 4.
//  * Batching: queued complex split-precision requests of one direction are
//    admitted together (up to max_batch) whatever their parameters: the unit
//    runs the ragged tensor-core contraction, where signals of different
//    (L, N) share the operand tiles at the tiles' largest L and N (identical
//    parameters take the uniform batch path and its resident digit tables).
//    Companions are picked from the queue by geometry so that the padded
//    work stays at least half useful.  A split-precision unit of fewer than 4
//    signals runs on the FP64 path (the fallback: the tensor-core operands
//    hold 16 signals, so small batches would waste most of the products).
//    A result depends on its companions only through that choice: within a
//    split-precision batch the split is per signal and the int32
//    accumulation exact, and the FP64 path is within the split tolerance.
//  * Resident state: Wigner tables, DFT plans, index tables and tuned kernel
//    variants are the per-device ones of the library, shared by all slots;
//    the Delta tables are built up to max_L at creation so they never grow
//    (a growing table would be reallocated under running work).
//  * Completion: a host callback enqueued after each unit stamps its finish
//    time and wakes the worker thread, which retires the slot and admits more.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "so3/so3_sampling.h"
#include "so3gpu.h"
#include "so3gpu_internal.h"

namespace so3g {
namespace {

double now_us() {
  return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Req {
  long long id = 0;
  int kind = 0;  // 0 inverse, 1 forward, 2 directional convolution + inverse
  so3_parameters_t p{};
  const void* in = nullptr;
  const void* in2 = nullptr;
  void* out = nullptr;
  int precision = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  int status = 0;
  bool done = false;
  int batch = 1;
};

struct Slot {
  cudaStream_t s = nullptr;
  Workspace wk;
  std::vector<Req*> reqs;
  size_t bytes = 0;
  bool busy = false;
  int status = 0;
  std::atomic<bool> finished{false};
  std::atomic<double> t_finish{0.0};
  void* owner = nullptr;
};

bool same_params(const Req& a, const Req& b) {
  return a.kind == b.kind && a.precision == b.precision && a.p.L == b.p.L && a.p.N == b.p.N &&
         a.p.L0 == b.p.L0 && a.p.sampling_scheme == b.p.sampling_scheme && a.p.n_order == b.p.n_order &&
         a.p.storage == b.p.storage && a.p.n_mode == b.p.n_mode && a.p.dl_method == b.p.dl_method &&
         a.p.reality == b.p.reality && a.p.steerable == b.p.steerable;
}
// Requests that may share a ragged split-precision unit.
bool ragged_mates(const Req& a, const Req& b) {
  return a.kind == b.kind && a.kind != 2 && a.precision == kPrecMixedInt8 && b.precision == kPrecMixedInt8 &&
         !a.p.reality && !b.p.reality;
}
// Contraction work of a request, and of a tile padded to the largest L, N.
double work_of(const so3_parameters_t& p) { return (double)p.L * p.L * p.L * p.N; }

size_t buffer_bytes(const Req& r) {
  const size_t fl = (size_t)so3_sampling_flmn_size(&r.p) * sizeof(double2);
  const size_t f = (size_t)so3_sampling_f_size(&r.p) * (r.p.reality ? sizeof(double) : sizeof(double2));
  if (r.kind == 2) return 2 * (size_t)r.p.L * r.p.L * sizeof(double2) + f;
  return fl + f;
}

}  // namespace

class Server {
 public:
  Server(int device, size_t budget, int slots, int max_batch, int max_L)
      : device_(device), budget_(budget), max_batch_(max_batch < 1 ? 1 : (max_batch > 64 ? 64 : max_batch)) {
    nslots_ = slots < 1 ? 1 : slots;
    max_L_ = max_L;
  }

  int start() {
    SO3G_CUDA(cudaSetDevice(device_));
    D_ = device_state(device_);
    slots_.reserve(nslots_);
    for (int i = 0; i < nslots_; i++) {
      auto sl = std::make_unique<Slot>();
      SO3G_CUDA(cudaStreamCreateWithFlags(&sl->s, cudaStreamNonBlocking));
      sl->owner = this;
      slots_.push_back(std::move(sl));
    }
    // keep freed scratch in the pool up to the budget (no release to the OS
    // between requests)
    cudaMemPool_t pool;
    SO3G_CUDA(cudaDeviceGetDefaultMemPool(&pool, device_));
    unsigned long long thr = budget_;
    SO3G_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    if (max_L_ > 0) {
      const double* t;
      std::lock_guard<std::mutex> lk(D_->mu);
      for (int m = 0; m < 2; m++)
        if (int rc = ensure_dl(D_, max_L_, m, slots_[0]->s, &t)) return rc;
    }
    // tables resident before the server existed belong to other users of the
    // device; the budget is charged for the Delta tables the server reads
    // (to max_L) and for every table built after this point
    base_resident_ = resident_bytes(D_);
    dl_charge_ = 0;
    if (max_L_ > 0) {
      int cap = 1;
      while (cap < max_L_) cap <<= 1;
      if (cap < 64) cap = 64;
      dl_charge_ = 2 * (size_t)dl_plane_offset(cap) * sizeof(double);
    }
    worker_ = std::thread([this] {
      set_thread_autotune(false);  // never stall admission on tuning a new geometry
      loop();
    });
    return kOk;
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    if (worker_.joinable()) worker_.join();
    for (auto& sl : slots_)
      if (sl->s) {
        cudaStreamSynchronize(sl->s);
        cudaStreamDestroy(sl->s);
      }
    for (auto& kv : reqs_) delete kv.second;
  }

  long long submit(int kind, const so3_parameters_t& p, const void* in, const void* in2, void* out, int precision) {
    if (kind < 0 || kind > 2 || !in || !out || (kind == 2 && !in2))
      return -fail(kInvalidParameter, "server request: bad kind or null buffer");
    if (precision != kPrecFp64 && precision != kPrecMixedInt8) return -fail(kInvalidParameter, "unknown precision");
    if (int rc = validate(p, p.reality != 0)) return -rc;
    if (kind == 2 && p.reality) return -fail(kUnsupported, "convolution requests produce complex samples");
    if (max_L_ > 0 && p.L > max_L_) return -fail(kUnsupported, "request band limit above the server's max_L");
    Req* r = new Req();
    r->kind = kind;
    r->p = p;
    r->in = in;
    r->in2 = in2;
    r->out = out;
    // split precision where the contractions can read the resident digit table
    // (L <= 512, N <= 64); larger geometries take the FP64 path, for which
    // generating the digits per tile costs more than the split saves
    r->precision = (kind == 2 || p.reality || p.L > 512 || p.N > 64) ? kPrecFp64 : precision;
    r->t_submit = now_us();
    {
      std::lock_guard<std::mutex> lk(mu_);
      r->id = next_id_++;
      reqs_[r->id] = r;
      queue_.push_back(r);
    }
    cv_.notify_all();
    return r->id;
  }

  // 1 done (fills outputs and forgets the request), 0 pending, <0 unknown id
  int query(long long id, bool wait, double* queue_us, double* total_us, int* batch, int* status) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return -1;
    Req* r = it->second;
    if (wait) done_cv_.wait(lk, [&] { return r->done; });
    if (!r->done) return 0;
    if (queue_us) *queue_us = r->t_admit - r->t_submit;
    if (total_us) *total_us = r->t_done - r->t_submit;
    if (batch) *batch = r->batch;
    if (status) *status = r->status;
    reqs_.erase(it);
    delete r;
    return 1;
  }

  void drain() {
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return queue_.empty() && busy_ == 0; });
  }

  void stats(long long* submitted, long long* completed, long long* batches, size_t* peak_bytes) {
    std::lock_guard<std::mutex> lk(mu_);
    if (submitted) *submitted = next_id_;
    if (completed) *completed = completed_;
    if (batches) *batches = units_;
    if (peak_bytes) *peak_bytes = peak_bytes_;
  }

 private:
  static void CUDART_CB on_done(void* arg) {
    Slot* sl = static_cast<Slot*>(arg);
    sl->t_finish.store(now_us());
    sl->finished.store(true);
    Server* sv = static_cast<Server*>(sl->owner);
    { std::lock_guard<std::mutex> lk(sv->mu_); }
    sv->cv_.notify_all();
  }

  // Precision a unit runs in: split precision pays only for batches of at
  // least kMinSplitBatch signals (the tensor-core operand holds 16 signals and
  // its scratch is sized per group of 16); smaller split-precision units run
  // on the FP64 path, the fallback (more accurate, so still within the split
  // tolerance).
  static constexpr int kMinSplitBatch = 4;
  static int unit_precision(const std::vector<Req*>& b) {
    return (b[0]->precision == kPrecMixedInt8 && (int)b.size() >= kMinSplitBatch) ? kPrecMixedInt8 : kPrecFp64;
  }
  // A unit whose requests differ in parameters: the ragged drivers, which run
  // each signal with its own parameters (in split precision, one shared
  // tensor-core contraction; in FP64, one transform after the other).
  static bool unit_ragged(const std::vector<Req*>& b) {
    for (const Req* r : b)
      if (!same_params(*r, *b[0])) return true;
    return false;
  }

  size_t unit_bytes(const std::vector<Req*>& b) const {
    const Req& r = *b[0];
    const int real = r.p.reality != 0;
    size_t need;
    if (unit_ragged(b) && unit_precision(b) == kPrecMixedInt8) {
      std::vector<so3_parameters_t> ps;
      for (const Req* q : b) ps.push_back(q->p);
      need = ragged_workspace_bytes(ps.data(), (int)ps.size(), r.kind == 1);
    } else if (unit_ragged(b)) {  // FP64, one signal at a time in one workspace
      need = 0;
      for (const Req* q : b) need = std::max(need, workspace_bytes(q->p, q->p.reality != 0));
    } else {
      need = batch_workspace_bytes(r.p, real, (int)b.size(), unit_precision(b));
    }
    if (r.kind == 2) need = ((need + 255) & ~size_t(255)) + (size_t)so3_sampling_flmn_size(&r.p) * sizeof(double2);
    for (const Req* q : b) need += buffer_bytes(*q);  // the callers' buffers count against the budget
    return need;
  }

  // Companions of the oldest queued request r0 for a split-precision unit:
  // queued requests that may share its tiles, taken in order of geometric
  // closeness while the unit's useful work stays at least half of its padded
  // work (sum of L^3 N over count * Lmax^3 Nmax).
  std::vector<Req*> pick_unit() const {
    Req* r0 = queue_.front();
    std::vector<Req*> unit{r0};
    if (!(r0->precision == kPrecMixedInt8 && r0->kind != 2 && !r0->p.reality)) return unit;
    std::vector<std::pair<double, Req*>> cand;
    const double w0 = std::log(work_of(r0->p));
    const size_t scan = std::min<size_t>(queue_.size(), 512);
    for (size_t i = 1; i < scan; i++)
      if (ragged_mates(*queue_[i], *r0)) cand.push_back({std::fabs(std::log(work_of(queue_[i]->p)) - w0), queue_[i]});
    std::stable_sort(cand.begin(), cand.end(),
                     [](const std::pair<double, Req*>& x, const std::pair<double, Req*>& y) { return x.first < y.first; });
    double sum = work_of(r0->p);
    int Lm = r0->p.L, Nm = r0->p.N;
    for (const auto& c : cand) {
      if ((int)unit.size() >= max_batch_) break;
      const so3_parameters_t& q = c.second->p;
      const int L2 = std::max(Lm, q.L), N2 = std::max(Nm, q.N);
      const double eff = (sum + work_of(q)) / ((double)(unit.size() + 1) * (double)L2 * L2 * L2 * N2);
      if (eff < 0.5) continue;
      unit.push_back(c.second);
      sum += work_of(q);
      Lm = L2, Nm = N2;
    }
    return unit;
  }

  // Enqueues the unit's work, the release of its scratch and the completion
  // callback on the slot's stream (worker thread, no lock held).
  void launch(Slot* sl) {
    const Req& r = *sl->reqs[0];
    const int real = r.p.reality != 0;
    const int n = (int)sl->reqs.size();
    int rc = kOk;
    void* ws = nullptr;
    if (cudaMallocAsync(&ws, sl->bytes, sl->s) != cudaSuccess) {
      cudaGetLastError();
      rc = fail(kOutOfMemory, "server scratch allocation failed");
    }
    if (rc == kOk) {
      sl->wk.ws = ws;
      sl->wk.ws_bytes = sl->bytes;
      sl->wk.borrowed = true;  // a size mismatch fails the unit instead of reallocating
      if (r.kind == 2) {
        const size_t wb = (workspace_bytes(r.p, 0) + 255) & ~size_t(255);
        double2* hlmn = reinterpret_cast<double2*>(static_cast<char*>(ws) + wb);
        const long long* hb = nullptr;
        {
          std::lock_guard<std::mutex> lk(D_->mu);
          rc = ensure_bases(D_, r.p, 0, &hb);
        }
        if (rc == kOk)
          rc = launch_s2toso3(r.p, hb, static_cast<const double2*>(r.in), static_cast<const double2*>(r.in2), hlmn,
                              sl->s);
        if (rc == kOk) rc = run_inverse(D_, &sl->wk, r.p, hlmn, r.out, 0, sl->s);
      } else {
        std::vector<const void*> ins(n);
        std::vector<void*> outs(n);
        std::vector<so3_parameters_t> ps(n);
        for (int i = 0; i < n; i++) {
          ins[i] = sl->reqs[i]->in;
          outs[i] = sl->reqs[i]->out;
          ps[i] = sl->reqs[i]->p;
        }
        const int prec = unit_precision(sl->reqs);
        if (unit_ragged(sl->reqs))
          rc = r.kind == 0 ? run_inverse_ragged(D_, &sl->wk, ps.data(), n, ins.data(), outs.data(), prec, sl->s)
                           : run_forward_ragged(D_, &sl->wk, ps.data(), n, ins.data(), outs.data(), prec, sl->s);
        else
          rc = r.kind == 0 ? run_inverse_batch(D_, &sl->wk, r.p, real, n, ins.data(), outs.data(), prec, sl->s)
                           : run_forward_batch(D_, &sl->wk, r.p, real, n, ins.data(), outs.data(), prec, sl->s);
      }
      cudaFreeAsync(ws, sl->s);
      sl->wk.ws = nullptr;
      sl->wk.ws_bytes = 0;
    }
    sl->status = rc;
    if (cudaLaunchHostFunc(sl->s, on_done, sl) != cudaSuccess) {
      cudaGetLastError();
      cudaStreamSynchronize(sl->s);
      sl->status = sl->status ? sl->status : fail(kCudaError, "server completion callback");
      on_done(sl);
    }
  }

  void retire_locked() {
    for (auto& sl : slots_) {
      if (!sl->busy || !sl->finished.load()) continue;
      const double t = sl->t_finish.load();
      for (Req* r : sl->reqs) {
        r->t_done = t;
        r->status = sl->status;
        r->done = true;
        completed_++;
      }
      sl->reqs.clear();
      sl->busy = false;
      sl->finished.store(false);
      inflight_bytes_ -= sl->bytes;
      sl->bytes = 0;
      busy_--;
    }
  }

  void loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      retire_locked();
      done_cv_.notify_all();
      if (stop_ && queue_.empty() && busy_ == 0) break;
      // admission: first-come first-served, as long as a slot and the budget allow
      bool launched = false;
      while (!queue_.empty()) {
        Slot* free_slot = nullptr;
        for (auto& sl : slots_)
          if (!sl->busy) {
            free_slot = sl.get();
            break;
          }
        if (!free_slot) break;
        std::vector<Req*> unit = pick_unit();
        const size_t now_res = resident_bytes(D_);
        const size_t resident = dl_charge_ + (now_res > base_resident_ ? now_res - base_resident_ : 0);
        const size_t room = budget_ > resident ? budget_ - resident : 0;
        size_t need = unit_bytes(unit);
        while (need > room && unit.size() > 1) {  // shrink the batch to fit
          unit.pop_back();
          need = unit_bytes(unit);
        }
        if (need > room) {  // can never run beside the resident tables
          Req* r = unit[0];
          queue_.pop_front();
          r->status = fail(kOutOfMemory, "request scratch exceeds the server memory budget");
          r->t_admit = r->t_done = now_us();
          r->done = true;
          completed_++;
          continue;
        }
        if (inflight_bytes_ + need > room) break;  // wait for memory
        for (Req* r : unit) {
          for (auto it = queue_.begin(); it != queue_.end(); ++it)
            if (*it == r) {
              queue_.erase(it);
              break;
            }
          r->t_admit = now_us();
          r->batch = (int)unit.size();
        }
        free_slot->reqs = unit;
        free_slot->bytes = need;
        free_slot->busy = true;
        free_slot->finished.store(false);
        inflight_bytes_ += need;
        if (inflight_bytes_ + resident > peak_bytes_) peak_bytes_ = inflight_bytes_ + resident;
        busy_++;
        units_++;
        lk.unlock();
        launch(free_slot);
        lk.lock();
        launched = true;
      }
      if (!launched)
        cv_.wait_for(lk, std::chrono::microseconds(200), [&] {
          if (stop_) return true;
          for (auto& sl : slots_)
            if (sl->busy && sl->finished.load()) return true;
          if (queue_.empty()) return false;
          for (auto& sl : slots_)
            if (!sl->busy) return true;
          return false;
        });
    }
    done_cv_.notify_all();
  }

  int device_;
  size_t budget_;
  int nslots_ = 1, max_batch_ = 8, max_L_ = 0;
  Device* D_ = nullptr;
  std::vector<std::unique_ptr<Slot>> slots_;
  std::thread worker_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::deque<Req*> queue_;
  std::unordered_map<long long, Req*> reqs_;
  long long next_id_ = 0, completed_ = 0, units_ = 0;
  size_t inflight_bytes_ = 0, peak_bytes_ = 0;
  size_t base_resident_ = 0, dl_charge_ = 0;  // see start()
  int busy_ = 0;
  bool stop_ = false;
};

}  // namespace so3g

struct so3gpu_server {
  std::unique_ptr<so3g::Server> impl;
};

extern "C" {

so3gpu_server* so3gpu_server_create(int device, size_t memory_budget, int max_inflight, int max_batch, int max_L) {
  auto* s = new so3gpu_server();
  s->impl = std::make_unique<so3g::Server>(device, memory_budget, max_inflight, max_batch, max_L);
  const int rc = s->impl->start();
  so3g_record_status(rc);
  if (rc) {
    delete s;
    return nullptr;
  }
  return s;
}

void so3gpu_server_destroy(so3gpu_server* s) { delete s; }

long long so3gpu_server_submit(so3gpu_server* s, int kind, const so3_parameters_t* p, const void* in, const void* in2,
                               void* out, int precision) {
  if (!s || !p) {
    so3g_record_status(so3g::fail(so3g::kInvalidParameter, "null server or parameters"));
    return -so3g::kInvalidParameter;
  }
  const long long id = s->impl->submit(kind, *p, in, in2, out, precision);
  so3g_record_status(id < 0 ? (int)-id : 0);
  return id;
}

int so3gpu_server_poll(so3gpu_server* s, long long id, double* queue_us, double* total_us, int* batch,
                       int* status) {
  return s ? s->impl->query(id, false, queue_us, total_us, batch, status) : -1;
}

int so3gpu_server_wait(so3gpu_server* s, long long id, double* queue_us, double* total_us, int* batch,
                       int* status) {
  return s ? s->impl->query(id, true, queue_us, total_us, batch, status) : -1;
}

void so3gpu_server_drain(so3gpu_server* s) {
  if (s) s->impl->drain();
}

void so3gpu_server_stats(so3gpu_server* s, long long* submitted, long long* completed, long long* units,
                         size_t* peak_bytes) {
  if (s) s->impl->stats(submitted, completed, units, peak_bytes);
}

}  // extern "C"
