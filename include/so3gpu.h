/*
 * so3gpu.h -- device-pointer extension API of libso3gpu (B200, sm_100a).
 *
 * The drop-in entry points of so3_core.h / so3_conv.h accept host or device
 * pointers and block until the result is in the caller's buffer.  This API
 * is the asynchronous form: device pointers only, work enqueued on the
 * context's CUDA stream, no host synchronisation.  Resident per-device
 * resources (Wigner Delta(pi/2) tables, FFT plans, index tables) are shared
 * by all contexts of a device; each context owns its own scratch, so contexts
 * on different streams may run concurrently.
 *
 * Status codes: 0 success, 1 invalid parameter, 2 CUDA error, 3 unsupported
 * configuration, 4 out of device memory.  The message of the last failure on
 * the calling thread is so3gpu_last_error().
 */
#ifndef SO3GPU_H
#define SO3GPU_H

#include <stddef.h>

#include "so3/so3_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct so3gpu_context so3gpu_context;

/* stream: a cudaStream_t (NULL = legacy default stream). */
so3gpu_context *so3gpu_context_create(int device, void *stream);
void so3gpu_context_destroy(so3gpu_context *ctx);
int so3gpu_context_set_stream(so3gpu_context *ctx, void *stream);

/* Builds the resident tables and plans the transform with these parameters
 * needs (blocking).  Call it before capturing transforms in a CUDA graph. */
int so3gpu_prepare(so3gpu_context *ctx, const so3_parameters_t *parameters);
/* Device scratch (bytes) one transform with these parameters uses. */
size_t so3gpu_workspace_size(const so3_parameters_t *parameters);

/* Same transforms as so3_core_*_via_ssht, on device pointers. */
int so3gpu_inverse(so3gpu_context *ctx, void *f, const void *flmn, const so3_parameters_t *parameters);
int so3gpu_forward(so3gpu_context *ctx, void *flmn, const void *f, const so3_parameters_t *parameters);
int so3gpu_inverse_real(so3gpu_context *ctx, double *f, const void *flmn,
                        const so3_parameters_t *parameters);
int so3gpu_forward_real(so3gpu_context *ctx, void *flmn, const double *f,
                        const so3_parameters_t *parameters);

/* Batches of `count` signals sharing one parameter set (no counterpart in the
 * reference).  f and flmn are host arrays of `count` device pointers.
 * precision SO3GPU_PRECISION_FP64: the FP64 path signal by signal (results
 * identical to so3gpu_inverse / so3gpu_forward).  SO3GPU_PRECISION_MIXED_INT8:
 * the Wigner contractions of all signals run as int8 tensor-core products
 * (7-slice Ozaki split, exact int32 accumulation, FP64 recombination) while
 * Delta, the quadrature weights and every DFT stay FP64; normwise relative
 * error against the FP64 path below 1e-10 (about 1e-12 measured).  Real
 * signals (parameters->reality) take the split contractions over their planes
 * n >= 0 and the FP64 forward beta stage; real signals with N = 1 use the
 * FP64 path.  The batch workspace holds `count` scratch plane sets (2.13 GB
 * each at L = 512, N = 64) plus the sliced operands (15.0 GB per group of 16
 * signals at L = 512, N = 64) and the column scales. */
#define SO3GPU_PRECISION_FP64 0
#define SO3GPU_PRECISION_MIXED_INT8 1
int so3gpu_inverse_batch(so3gpu_context *ctx, void *const *f, const void *const *flmn, int count,
                         const so3_parameters_t *parameters, int precision);
int so3gpu_forward_batch(so3gpu_context *ctx, void *const *flmn, const void *const *f, int count,
                         const so3_parameters_t *parameters, int precision);

/* Batches of signals of different parameters (no counterpart in the
 * reference): signal k has its own parameters[k] (any L, N, L0, sampling,
 * storage, n-order, n-mode, recursion).  SO3GPU_PRECISION_MIXED_INT8: the
 * Wigner contractions of all complex signals run in one int8 tensor-core
 * launch per Delta recursion -- signals sorted by (L, N) share 16-signal
 * operand tiles at the tile's largest L and N -- while every DFT stage runs
 * per signal in FP64; real signals, and precision FP64, take the FP64 path
 * per signal.  Same error contract as so3gpu_inverse_batch. */
int so3gpu_inverse_ragged(so3gpu_context *ctx, void *const *f, const void *const *flmn,
                          const so3_parameters_t *parameters, int count, int precision);
int so3gpu_forward_ragged(so3gpu_context *ctx, void *const *flmn, const void *const *f,
                          const so3_parameters_t *parameters, int count, int precision);

/* Directional convolutions of one S^2 signal with `count` kernels, then the
 * inverse transform (no counterpart in the reference; the composition of
 * so3_conv_s2toso3_harmonic_convolution, src/c/so3_conv.c:186-215, with
 * so3_core_inverse_via_ssht): f[k] = inverse(h_k), h_k,lmn = flm_lm
 * conj(glm[k]_ln) 8 pi^2 / (2l+1), h parameters `h_parameters` (complex).
 * flm and glm[k] hold L*L coefficients.  SO3GPU_PRECISION_FP64 materialises
 * each h_k in the workspace and runs the FP64 inverse; MIXED_INT8 computes h
 * inside the split-precision contraction's operand load (never stored). */
int so3gpu_s2toso3_inverse_batch(so3gpu_context *ctx, void *const *f, const void *flm, const void *const *glm,
                                 int count, const so3_parameters_t *h_parameters, int precision);

/* Same as so3_conv_s2toso3_harmonic_convolution / so3_conv_harmonic_convolution. */
int so3gpu_s2toso3_harmonic_convolution(so3gpu_context *ctx, void *hlmn, const so3_parameters_t *h_parameters,
                                        const void *flm, const void *glm);
int so3gpu_harmonic_convolution(so3gpu_context *ctx, void *hlmn, const so3_parameters_t *h_parameters,
                                const void *flmn, const so3_parameters_t *f_parameters, const void *glmn,
                                const so3_parameters_t *g_parameters);

/* Per-stage timing with CUDA events on the context's stream (off by
 * default).  so3gpu_stage_times waits for the recorded events, returns the
 * accumulated milliseconds and launch counts per stage since the previous
 * call (stages: 0 inverse contraction, 1 inverse beta, 2 inverse alpha,
 * 3 inverse gamma, 4 forward gamma, 5 forward alpha, 6 forward beta and
 * quadrature convolution, 7 forward contraction, 8 / 9 split-precision
 * inverse / forward contraction of a batch) and resets them. */
int so3gpu_stage_timing(so3gpu_context *ctx, int enable);
int so3gpu_stage_times(so3gpu_context *ctx, double *total_ms, long long *counts, int n);
/* Kernel variants of the DFT stages for the geometry of p (L, N, sampling,
 * reality) on a device: 8 entries indexed like so3gpu_stage_times (only the
 * FFT stages have more than one variant).  The autotuner fills them on the
 * first transform of a geometry (or in so3gpu_prepare); setting them pins a
 * choice and skips tuning.  get returns 1 if the geometry has been tuned or
 * pinned, 0 if not (var untouched). */
int so3gpu_get_stage_variants(int device, const so3_parameters_t *p, int *var);
int so3gpu_set_stage_variants(int device, const so3_parameters_t *p, const int *var);

/* Complex inverse transform (same result as so3gpu_inverse) that allocates
 * no device memory; no counterpart in the reference.  For callers that cannot
 * call cudaMalloc: code running under an allocator or memory cap owned by
 * someone else, or loops that must not allocate (and so must not risk an
 * implicit device synchronisation) after start-up.  f and flmn are device
 * pointers; stream is a cudaStream_t (NULL: legacy default stream).  Its
 * scratch, Wigner tables and FFT tables are file-scope device arrays of
 * 35,089,464 bytes in total (32 MiB of them scratch), held by every GPU that
 * loads the library until exit.  Complex, non-steerable signals only:
 * reality != 0 or steerable != 0 return status 3 before any device work.
 * L > 64, N > 64 or more than 32 MiB of scratch return status 3 (MW and MWSS
 * with L <= 64, N <= 64 always fit).  The first call in a CUDA context (the
 * runtime's primary context; again after cudaDeviceReset) builds the tables
 * and waits for them: make it before any stream capture.  A call whose L, N,
 * sampling, storage or n-order differ from the previous call's uploads new
 * FFT and offset tables from host memory: make such calls outside stream
 * capture as well.  Calls share the arrays, so calls whose GPU work overlaps
 * race: serialise them. */
int so3gpu_inverse_noalloc(void *f, const void *flmn, const so3_parameters_t *parameters, void *stream);

/* Request server (no counterpart in the reference): inverse (kind 0),
 * forward (kind 1) and directional-convolution (kind 2: in = flm, in2 = glm,
 * both L*L complex; out = samples of the inverse transform of the
 * so3_conv_s2toso3_harmonic_convolution result) requests of any parameters,
 * submitted from any host thread, run on one device with continuous
 * batching.  Up to max_inflight units run at once on separate streams;
 * queued complex split-precision (SO3GPU_PRECISION_MIXED_INT8) requests of
 * one direction are admitted together, up to max_batch per unit, whatever
 * their parameters (companions chosen by geometry; the unit's contractions
 * share the ragged tensor-core launch of so3gpu_inverse_ragged).  The
 * memory_budget covers the device's resident tables, the scratch of the
 * units in flight and the callers' buffers of those units; a unit is
 * admitted when a slot and the budget allow, first come first served, and a
 * request that cannot fit beside the resident tables completes with status
 * 4.  max_L (> 0) builds the Wigner tables up to that band limit at creation
 * and rejects larger requests; 0 lets the tables grow, which synchronises
 * the device when it happens.  Buffers are device pointers owned by the
 * caller until the request completes.  submit returns the request id (>= 0)
 * or minus a status code.  poll / wait return 1 once the request is done
 * (filling queueing and total latency in microseconds, the size of the unit
 * it ran in, and its status; the request is then forgotten), poll returns 0
 * while it is pending, -1 for unknown ids.  stats' peak_bytes is the largest
 * resident + in-flight total seen.  destroy waits for every submitted
 * request. */
typedef struct so3gpu_server so3gpu_server;
so3gpu_server *so3gpu_server_create(int device, size_t memory_budget, int max_inflight, int max_batch, int max_L);
void so3gpu_server_destroy(so3gpu_server *server);
long long so3gpu_server_submit(so3gpu_server *server, int kind, const so3_parameters_t *parameters,
                               const void *in, const void *in2, void *out, int precision);
int so3gpu_server_poll(so3gpu_server *server, long long id, double *queue_us, double *total_us, int *batch,
                       int *status);
int so3gpu_server_wait(so3gpu_server *server, long long id, double *queue_us, double *total_us, int *batch,
                       int *status);
void so3gpu_server_drain(so3gpu_server *server);
void so3gpu_server_stats(so3gpu_server *server, long long *submitted, long long *completed, long long *units,
                         size_t *peak_bytes);

/* Diagnostics. */
int so3gpu_last_status(void);
const char *so3gpu_last_error(void);
/* mode 0 (default): errors in the drop-in entry points print and exit(1) like
 * the reference; mode 1: they record the status and return. */
void so3gpu_set_error_mode(int mode);
/* Number of kernels this library has launched since load (all devices). */
long long so3gpu_launch_count(void);
/* Reads and clears the current device's flag that the tensor-core kernels set
 * when one of their bounded waits gave up (0: none; a nonzero value means the
 * results of the split-precision calls since the last read are invalid).
 * Synchronous. */
int so3gpu_take_kernel_error(void);

#ifdef __cplusplus
}
#endif
#endif
