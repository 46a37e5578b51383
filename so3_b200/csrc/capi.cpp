// The C ABI of libso3gpu: the reference's transform and convolution entry
// points (include/so3/so3_core.h, so3_conv.h) plus the device-pointer
// extension API (include/so3gpu.h).
//
// Drop-in calls accept host or device pointers: host buffers are staged
// through per-device scratch, the work runs on a library-owned stream and the
// call returns once the result is in the caller's buffer.  Calls on one device
// are serialised by a mutex (the reference is single-threaded; this makes the
// drop-in thread-safe).  Errors follow the reference (message, exit(1)) unless
// so3gpu_set_error_mode(1) was called; the status of the last call is always
// available from so3gpu_last_status().
#include <cuda_runtime.h>

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "so3/so3_adjoint.h"
#include "so3/so3_conv.h"
#include "so3/so3_core.h"
#include "so3/so3_sampling.h"
#include "so3gpu.h"
#include "so3gpu_internal.h"

using so3g::Device;
using so3g::Workspace;
typedef std::complex<double> cd;

namespace {

std::atomic<int> g_error_mode{0};
thread_local int t_status = 0;

int finish(int rc) {
  t_status = rc;
  if (rc != so3g::kOk && g_error_mode.load() == 0) {
    printf("ERROR: %s.\n", so3g::last_error().c_str());
    fflush(stdout);
    exit(1);
  }
  return rc;
}

struct Staging {
  void* buf = nullptr;
  size_t bytes = 0;
  int get(size_t need, void** out) {
    if (need > bytes) {
      if (buf) cudaFree(buf);
      buf = nullptr;
      bytes = 0;
      cudaError_t e = cudaMalloc(&buf, need);
      if (e != cudaSuccess) return so3g::fail(so3g::kOutOfMemory, "staging allocation failed");
      bytes = need;
    }
    *out = buf;
    return so3g::kOk;
  }
};

struct DropIn {
  std::mutex mu;
  Workspace wk;
  Staging io[4];
  cudaStream_t stream = nullptr;              // kernels
  cudaStream_t cin = nullptr, cout = nullptr;  // host->device / device->host copies
  cudaEvent_t ev[2 * so3g::kMaxChunks] = {};
};

std::mutex g_dropin_mu;
std::map<int, std::unique_ptr<DropIn>> g_dropin;

int current_device(int* dev) {
  cudaError_t e = cudaGetDevice(dev);
  if (e != cudaSuccess) return so3g::fail(so3g::kCudaError, std::string("no CUDA device: ") + cudaGetErrorString(e));
  return so3g::kOk;
}

DropIn* dropin(int dev) {
  std::lock_guard<std::mutex> lk(g_dropin_mu);
  auto& slot = g_dropin[dev];
  if (!slot) {
    slot = std::make_unique<DropIn>();
    cudaStreamCreateWithFlags(&slot->stream, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&slot->cin, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&slot->cout, cudaStreamNonBlocking);
    for (cudaEvent_t& e : slot->ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  }
  return slot.get();
}

bool device_accessible(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device view of a caller buffer: the buffer itself if the GPU can address it,
// else a staging buffer (filled from the host when `upload`).
int device_view(DropIn* X, int slot, const void* host, size_t bytes, bool upload, void** dev, bool* staged) {
  if (device_accessible(host)) {
    *dev = const_cast<void*>(host);
    *staged = false;
    return so3g::kOk;
  }
  if (int rc = X->io[slot].get(bytes ? bytes : 16, dev)) return rc;
  *staged = true;
  if (upload && bytes) SO3G_CUDA(cudaMemcpyAsync(*dev, host, bytes, cudaMemcpyHostToDevice, X->stream));
  return so3g::kOk;
}

int download(DropIn* X, void* host, const void* dev, size_t bytes, bool staged) {
  if (staged && bytes) SO3G_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, X->stream));
  SO3G_CUDA(cudaStreamSynchronize(X->stream));
  return so3g::kOk;
}

size_t f_bytes(const so3_parameters_t* p, int real) {
  return (size_t)so3_sampling_f_size(p) * (real ? sizeof(double) : sizeof(cd));
}
size_t flmn_bytes(const so3_parameters_t* p, int real) {
  so3_parameters_t q = *p;
  q.reality = real;
  return (size_t)so3_sampling_flmn_size(&q) * sizeof(cd);
}

// Device buffer for one side of a staged call: the caller's own buffer when
// the GPU can address it (no copies), else a staging buffer.
int stage_side(DropIn* X, int slot, const void* user, size_t bytes, void** dev, bool* host) {
  *host = !device_accessible(user);
  if (!*host) {
    *dev = const_cast<void*>(user);
    return so3g::kOk;
  }
  return X->io[slot].get(bytes ? bytes : 16, dev);
}

// Waits for the copies and kernels of a staged call (also after a failure,
// so nothing still reads or writes the caller's buffers on return).
int drain(DropIn* X, int rc) {
  const cudaError_t a = cudaStreamSynchronize(X->cin);
  const cudaError_t b = cudaStreamSynchronize(X->stream);
  const cudaError_t c = cudaStreamSynchronize(X->cout);
  if (rc) return rc;
  const cudaError_t e = a != cudaSuccess ? a : (b != cudaSuccess ? b : c);
  if (e != cudaSuccess) return so3g::fail(so3g::kCudaError, std::string("staged transform: ") + cudaGetErrorString(e));
  return so3g::kOk;
}

so3g::StagedIo staged_io(DropIn* X, const void* in_user, void* din, bool in_host, void* out_user, void* dout,
                         bool out_host) {
  so3g::StagedIo io;
  io.host_in = in_host ? in_user : nullptr;
  io.host_out = out_host ? out_user : nullptr;
  io.dev_in = din;
  io.dev_out = dout;
  io.cin = X->cin;
  io.cout = X->cout;
  for (int i = 0; i < 2 * so3g::kMaxChunks; i++) io.ev[i] = X->ev[i];
  return io;
}

int dropin_inverse(void* f, const void* flmn, const so3_parameters_t* p, int real) {
  if (!p) return so3g::fail(so3g::kInvalidParameter, "null parameters");
  if (int rc = so3g::validate(*p, real)) return rc;
  int dev;
  if (int rc = current_device(&dev)) return rc;
  DropIn* X = dropin(dev);
  std::lock_guard<std::mutex> lk(X->mu);
  void *din, *dout;
  bool hin, hout;
  if (int rc = stage_side(X, 0, flmn, flmn_bytes(p, real), &din, &hin)) return rc;
  if (int rc = stage_side(X, 1, f, f_bytes(p, real), &dout, &hout)) return rc;
  const so3g::StagedIo io = staged_io(X, flmn, din, hin, f, dout, hout);
  return drain(X, so3g::run_inverse_staged(so3g::device_state(dev), &X->wk, *p, real, io, X->stream));
}

int dropin_forward(void* flmn, const void* f, const so3_parameters_t* p, int real, bool zero_first) {
  if (!p) return so3g::fail(so3g::kInvalidParameter, "null parameters");
  if (int rc = so3g::validate(*p, real)) return rc;
  int dev;
  if (int rc = current_device(&dev)) return rc;
  DropIn* X = dropin(dev);
  std::lock_guard<std::mutex> lk(X->mu);
  void *din, *dout;
  bool hin, hout;
  // Skipped n-blocks of a host output are never copied back, so they keep the
  // caller's contents (reference semantics); a device output is written only
  // where the transform computes.
  if (int rc = stage_side(X, 0, f, f_bytes(p, real), &din, &hin)) return rc;
  if (int rc = stage_side(X, 1, flmn, flmn_bytes(p, real), &dout, &hout)) return rc;
  const so3g::StagedIo io = staged_io(X, f, din, hin, flmn, dout, hout);
  return drain(X, so3g::run_forward_staged(so3g::device_state(dev), &X->wk, *p, real, zero_first, io, X->stream));
}

// Adjoint transforms on host or device buffers (whole arrays staged; the
// adjoint inverse writes every coefficient, the adjoint forward every sample).
int dropin_adjoint(void* out, const void* in, const so3_parameters_t* p, bool inverse, int real) {
  if (!p) return so3g::fail(so3g::kInvalidParameter, "null parameters");
  int dev;
  if (int rc = current_device(&dev)) return rc;
  DropIn* X = dropin(dev);
  std::lock_guard<std::mutex> lk(X->mu);
  so3_parameters_t q = *p;  // the entry point decides the layout, as the reference's do
  q.reality = real;
  p = &q;
  const size_t fb = f_bytes(p, real), lb = flmn_bytes(p, real);
  void *din = nullptr, *dout = nullptr;
  bool sin = false, sout = false;
  if (int rc = device_view(X, 0, in, inverse ? fb : lb, true, &din, &sin)) return rc;
  if (int rc = device_view(X, 1, out, inverse ? lb : fb, false, &dout, &sout)) return rc;
  Device* D = so3g::device_state(dev);
  const int rc = inverse ? so3g::run_adjoint_inverse(D, &X->wk, *p, din, dout, X->stream)
                         : so3g::run_adjoint_forward(D, &X->wk, *p, din, dout, X->stream);
  if (rc) {
    cudaStreamSynchronize(X->stream);
    return rc;
  }
  return download(X, out, dout, inverse ? lb : fb, sout);
}

int require_mw(const so3_parameters_t* p) {
  if (p && p->sampling_scheme != SO3_SAMPLING_MW)
    return so3g::fail(so3g::kUnsupported, "the direct transforms support MW sampling only");
  return so3g::kOk;
}

}  // namespace

void so3g_record_status(int rc) { t_status = rc; }

struct so3gpu_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  Workspace wk;
  std::mutex mu;
};

extern "C" {

// ------------------------------------------------------------ drop-in core
void so3_core_inverse_via_ssht(cd* f, const cd* flmn, const so3_parameters_t* p) {
  finish(dropin_inverse(f, flmn, p, 0));
}
void so3_core_inverse_via_ssht_real(double* f, const cd* flmn, const so3_parameters_t* p) {
  finish(dropin_inverse(f, flmn, p, 1));
}
void so3_core_forward_via_ssht(cd* flmn, const cd* f, const so3_parameters_t* p) {
  finish(dropin_forward(flmn, f, p, 0, false));
}
void so3_core_forward_via_ssht_real(cd* flmn, const double* f, const so3_parameters_t* p) {
  finish(dropin_forward(flmn, f, p, 1, false));
}
void so3_core_inverse_direct(cd* f, const cd* flmn, const so3_parameters_t* p) {
  int rc = require_mw(p);
  finish(rc ? rc : dropin_inverse(f, flmn, p, 0));
}
void so3_core_inverse_direct_real(double* f, const cd* flmn, const so3_parameters_t* p) {
  int rc = require_mw(p);
  finish(rc ? rc : dropin_inverse(f, flmn, p, 1));
}
void so3_core_forward_direct(cd* flmn, const cd* f, const so3_parameters_t* p) {
  int rc = require_mw(p);
  finish(rc ? rc : dropin_forward(flmn, f, p, 0, true));
}
void so3_core_forward_direct_real(cd* flmn, const double* f, const so3_parameters_t* p) {
  int rc = require_mw(p);
  finish(rc ? rc : dropin_forward(flmn, f, p, 1, true));
}

// ------------------------------------------------------------ drop-in adjoint
void so3_adjoint_inverse_direct(cd* flmn, const cd* f, const so3_parameters_t* p) {
  finish(dropin_adjoint(flmn, f, p, true, 0));
}
void so3_adjoint_forward_direct(cd* f, const cd* flmn, const so3_parameters_t* p) {
  finish(dropin_adjoint(f, flmn, p, false, 0));
}
void so3_adjoint_inverse_direct_real(cd* flmn, const double* f, const so3_parameters_t* p) {
  finish(dropin_adjoint(flmn, f, p, true, 1));
}
void so3_adjoint_forward_direct_real(double* f, const cd* flmn, const so3_parameters_t* p) {
  finish(dropin_adjoint(f, flmn, p, false, 1));
}

// ------------------------------------------------------------ drop-in conv
so3_parameters_t so3_conv_get_parameters_of_convolved_lmn(const so3_parameters_t* fp, const so3_parameters_t* gp) {
  const char* err = nullptr;
  if (fp->sampling_scheme != gp->sampling_scheme) err = "f and g must have the same sampling_scheme";
  else if (fp->n_order != gp->n_order) err = "f and g must have the same n_order";
  else if (fp->storage != gp->storage) err = "f and g must have the same storage";
  else if (fp->n_mode != gp->n_mode) err = "f and g must have the same n_mode";
  else if (fp->reality != gp->reality) err = "f and g must have the same reality";
  so3_parameters_t h = *fp;
  if (err) {
    so3g::set_error(err);
    finish(so3g::kInvalidParameter);
    return h;
  }
  h.L = fp->L < gp->L ? fp->L : gp->L;
  h.N = h.L;
  h.L0 = fp->L0 > gp->L0 ? fp->L0 : gp->L0;
  t_status = 0;
  return h;
}

void so3_conv_get_parameters_of_convolved_lmn_void(so3_parameters_t* hp, const so3_parameters_t* fp,
                                                   const so3_parameters_t* gp) {
  *hp = so3_conv_get_parameters_of_convolved_lmn(fp, gp);
}

void so3_conv_harmonic_convolution(cd* hlmn, const so3_parameters_t* hp, const cd* flmn, const so3_parameters_t* fp,
                                   const cd* glmn, const so3_parameters_t* gp) {
  int rc = so3g::kOk, dev = 0;
  if (!hp || !fp || !gp) rc = so3g::fail(so3g::kInvalidParameter, "null parameters");
  if (!rc) rc = current_device(&dev);
  if (rc) {
    finish(rc);
    return;
  }
  DropIn* X = dropin(dev);
  Device* D = so3g::device_state(dev);
  std::lock_guard<std::mutex> lk(X->mu);
  const long long *hb, *fb, *gb;
  {
    std::lock_guard<std::mutex> dl(D->mu);
    if (!rc) rc = so3g::ensure_bases(D, *hp, hp->reality != 0, &hb);
    if (!rc) rc = so3g::ensure_bases(D, *fp, fp->reality != 0, &fb);
    if (!rc) rc = so3g::ensure_bases(D, *gp, gp->reality != 0, &gb);
  }
  void *dh = nullptr, *df = nullptr, *dg = nullptr;
  bool sh = false, sf = false, sg = false;
  const size_t hbytes = (size_t)so3_sampling_flmn_size(hp) * sizeof(cd);
  if (!rc) rc = device_view(X, 0, flmn, (size_t)so3_sampling_flmn_size(fp) * sizeof(cd), true, &df, &sf);
  if (!rc) rc = device_view(X, 1, glmn, (size_t)so3_sampling_flmn_size(gp) * sizeof(cd), true, &dg, &sg);
  if (!rc) rc = device_view(X, 2, hlmn, hbytes, true, &dh, &sh);
  if (!rc)
    rc = so3g::launch_harmonic_convolution(*hp, *fp, *gp, hb, fb, gb, (const double2*)df, (const double2*)dg,
                                           (double2*)dh, X->stream);
  if (!rc) rc = download(X, hlmn, dh, hbytes, sh);
  finish(rc);
}

void so3_conv_s2toso3_harmonic_convolution(cd* hlmn, const so3_parameters_t* hp, const cd* flm, const cd* glm) {
  int rc = so3g::kOk, dev = 0;
  if (!hp) rc = so3g::fail(so3g::kInvalidParameter, "null parameters");
  if (!rc) rc = current_device(&dev);
  if (rc) {
    finish(rc);
    return;
  }
  DropIn* X = dropin(dev);
  Device* D = so3g::device_state(dev);
  std::lock_guard<std::mutex> lk(X->mu);
  const long long* hb = nullptr;
  {
    std::lock_guard<std::mutex> dl(D->mu);
    rc = so3g::ensure_bases(D, *hp, hp->reality != 0, &hb);
  }
  void *dh = nullptr, *df = nullptr, *dg = nullptr;
  bool sh = false, sf = false, sg = false;
  const size_t lm = (size_t)hp->L * hp->L * sizeof(cd);
  const size_t hbytes = (size_t)so3_sampling_flmn_size(hp) * sizeof(cd);
  if (!rc) rc = device_view(X, 0, flm, lm, true, &df, &sf);
  if (!rc) rc = device_view(X, 1, glm, lm, true, &dg, &sg);
  if (!rc) rc = device_view(X, 2, hlmn, hbytes, false, &dh, &sh);
  if (!rc) rc = so3g::launch_s2toso3(*hp, hb, (const double2*)df, (const double2*)dg, (double2*)dh, X->stream);
  if (!rc) rc = download(X, hlmn, dh, hbytes, sh);
  finish(rc);
}

void so3_conv_convolution(cd* h, const so3_parameters_t* hp, const cd* f, const so3_parameters_t* fp, const cd* g,
                          const so3_parameters_t* gp) {
  // forward(f), forward(g), harmonic convolution, inverse (reference
  // src/c/so3_conv.c:154-184), with host round trips kept out of the middle.
  int rc = so3g::kOk;
  if (!hp || !fp || !gp) {
    finish(so3g::fail(so3g::kInvalidParameter, "null parameters"));
    return;
  }
  const size_t fl = (size_t)so3_sampling_flmn_size(fp) * sizeof(cd);
  const size_t gl = (size_t)so3_sampling_flmn_size(gp) * sizeof(cd);
  const size_t hl = (size_t)so3_sampling_flmn_size(hp) * sizeof(cd);
  void *dfl = nullptr, *dgl = nullptr, *dhl = nullptr;
  if (cudaMalloc(&dfl, fl) != cudaSuccess || cudaMalloc(&dgl, gl) != cudaSuccess || cudaMalloc(&dhl, hl) != cudaSuccess)
    rc = so3g::fail(so3g::kOutOfMemory, "convolution buffers");
  if (!rc) rc = dropin_forward(dfl, f, fp, 0, true);
  if (!rc) rc = dropin_forward(dgl, g, gp, 0, true);
  if (!rc) {
    so3_conv_harmonic_convolution((cd*)dhl, hp, (const cd*)dfl, fp, (const cd*)dgl, gp);
    rc = t_status;
  }
  if (!rc) rc = dropin_inverse(h, dhl, hp, 0);
  cudaFree(dfl);
  cudaFree(dgl);
  cudaFree(dhl);
  finish(rc);
}

// ------------------------------------------------------------ extension API
so3gpu_context* so3gpu_context_create(int device, void* stream) {
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    so3g::set_error("invalid device");
    t_status = so3g::kCudaError;
    return nullptr;
  }
  cudaSetDevice(prev);
  auto* c = new so3gpu_context();
  c->device = device;
  c->stream = (cudaStream_t)stream;
  t_status = 0;
  return c;
}

void so3gpu_context_destroy(so3gpu_context* c) {
  if (!c) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  if (c->wk.ws) cudaFree(c->wk.ws);
  cudaSetDevice(prev);
  delete c;
}

int so3gpu_context_set_stream(so3gpu_context* c, void* stream) {
  if (!c) return t_status = so3g::fail(so3g::kInvalidParameter, "null context");
  c->stream = (cudaStream_t)stream;
  return t_status = 0;
}

size_t so3gpu_workspace_size(const so3_parameters_t* p) { return p ? so3g::workspace_bytes(*p, p->reality != 0) : 0; }

namespace {
struct DeviceScope {
  int prev = 0;
  explicit DeviceScope(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DeviceScope() { cudaSetDevice(prev); }
};
}  // namespace

int so3gpu_prepare(so3gpu_context* c, const so3_parameters_t* p) {
  if (!c || !p) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  DeviceScope ds(c->device);
  std::lock_guard<std::mutex> lk(c->mu);
  int rc = so3g::prepare(so3g::device_state(c->device), *p, p->reality != 0, c->stream, &c->wk);
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = so3g::fail(so3g::kCudaError, "prepare sync");
  return t_status = rc;
}

static int ctx_transform(so3gpu_context* c, void* out, const void* in, const so3_parameters_t* p, int real,
                         bool inverse) {
  if (!c || !p || !out || !in) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  DeviceScope ds(c->device);
  std::lock_guard<std::mutex> lk(c->mu);
  Device* D = so3g::device_state(c->device);
  int rc = inverse ? so3g::run_inverse(D, &c->wk, *p, in, out, real, c->stream)
                   : so3g::run_forward(D, &c->wk, *p, in, out, real, c->stream);
  return t_status = rc;
}

int so3gpu_inverse(so3gpu_context* c, void* f, const void* flmn, const so3_parameters_t* p) {
  return ctx_transform(c, f, flmn, p, 0, true);
}
int so3gpu_forward(so3gpu_context* c, void* flmn, const void* f, const so3_parameters_t* p) {
  return ctx_transform(c, flmn, f, p, 0, false);
}
int so3gpu_inverse_real(so3gpu_context* c, double* f, const void* flmn, const so3_parameters_t* p) {
  return ctx_transform(c, f, flmn, p, 1, true);
}
int so3gpu_forward_real(so3gpu_context* c, void* flmn, const double* f, const so3_parameters_t* p) {
  return ctx_transform(c, flmn, f, p, 1, false);
}

static int ctx_batch(so3gpu_context* c, void* const* out, const void* const* in, int count, const so3_parameters_t* p,
                     int precision, bool inverse) {
  if (!c || !p || (count > 0 && (!out || !in))) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  for (int i = 0; i < count; i++)
    if (!out[i] || !in[i]) return t_status = so3g::fail(so3g::kInvalidParameter, "null signal pointer");
  DeviceScope ds(c->device);
  std::lock_guard<std::mutex> lk(c->mu);
  Device* D = so3g::device_state(c->device);
  const int real = p->reality != 0;
  int rc = inverse ? so3g::run_inverse_batch(D, &c->wk, *p, real, count, in, out, precision, c->stream)
                   : so3g::run_forward_batch(D, &c->wk, *p, real, count, in, out, precision, c->stream);
  return t_status = rc;
}

int so3gpu_inverse_batch(so3gpu_context* c, void* const* f, const void* const* flmn, int count,
                         const so3_parameters_t* p, int precision) {
  return ctx_batch(c, f, flmn, count, p, precision, true);
}
int so3gpu_forward_batch(so3gpu_context* c, void* const* flmn, const void* const* f, int count,
                         const so3_parameters_t* p, int precision) {
  return ctx_batch(c, flmn, f, count, p, precision, false);
}

static int ctx_ragged(so3gpu_context* c, void* const* out, const void* const* in, const so3_parameters_t* ps,
                      int count, int precision, bool inverse) {
  if (!c || (count > 0 && (!out || !in || !ps))) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  for (int i = 0; i < count; i++)
    if (!out[i] || !in[i]) return t_status = so3g::fail(so3g::kInvalidParameter, "null signal pointer");
  DeviceScope ds(c->device);
  std::lock_guard<std::mutex> lk(c->mu);
  Device* D = so3g::device_state(c->device);
  int rc = inverse ? so3g::run_inverse_ragged(D, &c->wk, ps, count, in, out, precision, c->stream)
                   : so3g::run_forward_ragged(D, &c->wk, ps, count, in, out, precision, c->stream);
  return t_status = rc;
}

int so3gpu_inverse_ragged(so3gpu_context* c, void* const* f, const void* const* flmn, const so3_parameters_t* ps,
                          int count, int precision) {
  return ctx_ragged(c, f, flmn, ps, count, precision, true);
}
int so3gpu_forward_ragged(so3gpu_context* c, void* const* flmn, const void* const* f, const so3_parameters_t* ps,
                          int count, int precision) {
  return ctx_ragged(c, flmn, f, ps, count, precision, false);
}

int so3gpu_s2toso3_inverse_batch(so3gpu_context* c, void* const* f, const void* flm, const void* const* glm, int count,
                                 const so3_parameters_t* hp, int precision) {
  if (!c || !hp || !flm || (count > 0 && (!f || !glm)))
    return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  for (int i = 0; i < count; i++)
    if (!f[i] || !glm[i]) return t_status = so3g::fail(so3g::kInvalidParameter, "null signal pointer");
  DeviceScope ds(c->device);
  std::lock_guard<std::mutex> lk(c->mu);
  Device* D = so3g::device_state(c->device);
  return t_status = so3g::run_conv_inverse_batch(D, &c->wk, *hp, count, flm, glm, f, precision, c->stream);
}

int so3gpu_s2toso3_harmonic_convolution(so3gpu_context* c, void* hlmn, const so3_parameters_t* hp, const void* flm,
                                        const void* glm) {
  if (!c || !hp) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  DeviceScope ds(c->device);
  Device* D = so3g::device_state(c->device);
  const long long* hb = nullptr;
  int rc;
  {
    std::lock_guard<std::mutex> lk(D->mu);
    rc = so3g::ensure_bases(D, *hp, hp->reality != 0, &hb);
  }
  if (!rc) rc = so3g::launch_s2toso3(*hp, hb, (const double2*)flm, (const double2*)glm, (double2*)hlmn, c->stream);
  return t_status = rc;
}

int so3gpu_harmonic_convolution(so3gpu_context* c, void* hlmn, const so3_parameters_t* hp, const void* flmn,
                                const so3_parameters_t* fp, const void* glmn, const so3_parameters_t* gp) {
  if (!c || !hp || !fp || !gp) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  DeviceScope ds(c->device);
  Device* D = so3g::device_state(c->device);
  const long long *hb = nullptr, *fb = nullptr, *gb = nullptr;
  int rc;
  {
    std::lock_guard<std::mutex> lk(D->mu);
    rc = so3g::ensure_bases(D, *hp, hp->reality != 0, &hb);
    if (!rc) rc = so3g::ensure_bases(D, *fp, fp->reality != 0, &fb);
    if (!rc) rc = so3g::ensure_bases(D, *gp, gp->reality != 0, &gb);
  }
  if (!rc)
    rc = so3g::launch_harmonic_convolution(*hp, *fp, *gp, hb, fb, gb, (const double2*)flmn, (const double2*)glmn,
                                           (double2*)hlmn, c->stream);
  return t_status = rc;
}

int so3gpu_stage_timing(so3gpu_context* c, int enable) {
  if (!c) return t_status = so3g::fail(so3g::kInvalidParameter, "null context");
  c->wk.timer.on = enable != 0;
  return t_status = 0;
}

int so3gpu_stage_times(so3gpu_context* c, double* total_ms, long long* counts, int n) {
  if (!c || !total_ms || !counts) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  DeviceScope ds(c->device);
  if (int rc = so3g::timer_collect(&c->wk.timer)) return t_status = rc;
  for (int i = 0; i < n && i < so3g::kStCount; i++) {
    total_ms[i] = c->wk.timer.total_ms[i];
    counts[i] = c->wk.timer.count[i];
    c->wk.timer.total_ms[i] = 0.0;
    c->wk.timer.count[i] = 0;
  }
  return t_status = 0;
}

int so3gpu_get_stage_variants(int device, const so3_parameters_t* p, int* var) {
  if (!p || !var) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument"), 0;
  t_status = 0;
  return so3g::get_stage_variants(so3g::device_state(device), *p, p->reality != 0, var);
}

int so3gpu_set_stage_variants(int device, const so3_parameters_t* p, const int* var) {
  if (!p || !var) return t_status = so3g::fail(so3g::kInvalidParameter, "null argument");
  return t_status = so3g::set_stage_variants(so3g::device_state(device), *p, p->reality != 0, var);
}

int so3gpu_last_status(void) { return t_status; }
const char* so3gpu_last_error(void) { return so3g::last_error().c_str(); }
void so3gpu_set_error_mode(int mode) { g_error_mode.store(mode ? 1 : 0); }
long long so3gpu_launch_count(void) { return so3g::g_launches.load(); }
int so3gpu_take_kernel_error(void) { return so3g::mixed_take_error(); }

}  // extern "C"
