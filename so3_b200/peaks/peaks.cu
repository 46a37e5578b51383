// Throughput probes of the benchmark (not part of libso3gpu): the
// denominators the contraction kernels are reported against, built into
// so3_b200/lib/libso3peaks.so and loaded by bench.py only.  FP64: each
// thread runs 8 independent FMA chains in registers.  int8 tensor cores:
// back-to-back tcgen05.mma kind::i8 products from shared memory into tensor
// memory (the instruction the split-precision contractions issue).  HBM: a
// device-to-device copy of a buffer far larger than L2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "tc_sm100.cuh"

namespace {
using namespace so3g;

#define PK_CUDA(call)                            \
  do {                                           \
    if ((call) != cudaSuccess) return -1.0;      \
  } while (0)

__global__ void fp64_fma_chain(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int i = 0; i < 8; i++) x[i] = threadIdx.x * 1e-9 + i;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = fma(x[i], a, b);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += x[i];
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

// One CTA per SM; one thread issues tcgen05.mma kind::i8 M=128 N=256 K=32
// products from shared memory into two tensor-memory accumulators, 64 per
// batch, with at most two batches in flight (commit to alternating
// mbarriers).  Operand contents do not matter (zeros).
__global__ void __launch_bounds__(128, 1) int8_tc_chain(int iters, int* flag) {
  __shared__ __align__(1024) uint8_t sa[128 * 32];
  __shared__ __align__(1024) uint8_t sb[256 * 32];
  __shared__ unsigned long long bar[2];
  __shared__ uint32_t slot;
  for (int i = threadIdx.x; i < 128 * 32 / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(sa)[i] = 0u;
  for (int i = threadIdx.x; i < 256 * 32 / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(sb)[i] = 0u;
  tc::fence_proxy_async_smem();
  const uint32_t b0 = tc::smem_u32(&bar[0]);
  if (threadIdx.x == 0) {
    tc::mbar_init(b0, 1);
    tc::mbar_init(b0 + 8, 1);
    tc::mbar_fence_init();
  }
  if (threadIdx.x < 32) tc::tmem_alloc(tc::smem_u32(&slot), 512);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tbase = slot;
  if (threadIdx.x == 0) {
    constexpr uint32_t idesc = tc::idesc_s8(128, 256);
    const uint64_t ad = tc::smem_desc(tc::smem_u32(sa), 128 * 16, 128);
    const uint64_t bd = tc::smem_desc(tc::smem_u32(sb), 256 * 16, 128);
    for (int it = 0; it < iters; it++) {
#pragma unroll 8
      for (int j = 0; j < 64; j++) tc::mma_i8(tbase + 256u * (j & 1), ad, bd, idesc, 1u);
      tc::mma_commit(b0 + 8 * (it & 1));
      if (it >= 1) tc::mbar_wait(b0 + 8 * ((it - 1) & 1), ((it - 1) >> 1) & 1, flag, 1);
    }
    tc::mbar_wait(b0 + 8 * ((iters - 1) & 1), ((iters - 1) >> 1) & 1, flag, 1);
  }
  tc::tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    __syncwarp();
    tc::tc_fence_after();
    tc::tmem_dealloc(tbase, 512);
  }
}

double int8_mma_tops() {
  int dev = 0, sms = 0;
  PK_CUDA(cudaGetDevice(&dev));
  PK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int* flag = nullptr;
  PK_CUDA(cudaMalloc(&flag, sizeof(int)));
  PK_CUDA(cudaMemset(flag, 0, sizeof(int)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms, iters = 256;
  int8_tc_chain<<<blocks, 128>>>(iters, flag);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(e0);
    int8_tc_chain<<<blocks, 128>>>(iters, flag);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  int h = 0;
  cudaMemcpy(&h, flag, sizeof(int), cudaMemcpyDeviceToHost);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(flag);
  PK_CUDA(cudaGetLastError());
  if (h) return -1.0;  // a bounded wait gave up
  const double ops = 2.0 * 128 * 256 * 32 * 64.0 * iters * (double)blocks;
  return ops / (best * 1e-3) / 1e12;
}

double fp64_tflops() {
  int dev = 0, sms = 0;
  PK_CUDA(cudaGetDevice(&dev));
  PK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double* out = nullptr;
  PK_CUDA(cudaMalloc(&out, sizeof(double)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  fp64_fma_chain<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(e0);
    fp64_fma_chain<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  PK_CUDA(cudaGetLastError());
  const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  return flops / (best * 1e-3) / 1e12;
}

// FP64 tensor-core throughput: each warp runs 8 independent chains of
// mma.sync.aligned.m8n8k4 f64 (8 x 8 x 4 = 256 multiply-adds per instruction).
__global__ void dmma_chain(double* out, int iters) {
  double a = 1.0 + 1e-9 * threadIdx.x, b = 0.999999;
  double c[8][2];
#pragma unroll
  for (int i = 0; i < 8; i++) c[i][0] = c[i][1] = 1e-3 * i;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                   : "+d"(c[i][0]), "+d"(c[i][1])
                   : "d"(a), "d"(b));
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += c[i][0] + c[i][1];
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

double dmma_tflops() {
  int dev = 0, sms = 0;
  PK_CUDA(cudaGetDevice(&dev));
  PK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double* out = nullptr;
  PK_CUDA(cudaMalloc(&out, sizeof(double)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 4, threads = 256;
  // a short launch first: the iteration count is sized for about 20 ms per launch
  int iters = 16;
  {
    cudaEventRecord(e0);
    dmma_chain<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double per_iter = ms > 0 ? ms / iters : 1e-3;
    iters = (int)std::min(4096.0, std::max(16.0, 20.0 / per_iter));
  }
  dmma_chain<<<blocks, threads>>>(out, iters);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(e0);
    dmma_chain<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  PK_CUDA(cudaGetLastError());
  const double flops = 2.0 * 256.0 * 8.0 * iters * (double)blocks * (threads / 32);
  return flops / (best * 1e-3) / 1e12;
}

// Device-to-device copy of 4 GiB (read + write counted), best of 5.
double hbm_copy_gbs() {
  const size_t bytes = size_t(4) << 30;
  void *a = nullptr, *b = nullptr;
  PK_CUDA(cudaMalloc(&a, bytes));
  if (cudaMalloc(&b, bytes) != cudaSuccess) {
    cudaFree(a);
    return -1.0;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaMemset(a, 1, bytes);
  cudaMemcpyAsync(b, a, bytes, cudaMemcpyDeviceToDevice, 0);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(e0);
    cudaMemcpyAsync(b, a, bytes, cudaMemcpyDeviceToDevice, 0);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(a);
  cudaFree(b);
  PK_CUDA(cudaGetLastError());
  return 2.0 * (double)bytes / (best * 1e-3) / 1e9;
}

}  // namespace

// Each returns the measured rate on `device`, or a negative value on a CUDA
// error.  FP64: TFLOP/s (2 flops per FMA); int8 tcgen05.mma M=128, N=256:
// TOP/s (2 ops per multiply-add); HBM: GB/s of a device-to-device copy.
extern "C" double so3peaks_fp64_tflops(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  return fp64_tflops();
}
extern "C" double so3peaks_int8_mma_tops(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  return int8_mma_tops();
}
extern "C" double so3peaks_dmma_tflops(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  return dmma_tflops();
}
extern "C" double so3peaks_hbm_copy_gbs(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  return hbm_copy_gbs();
}
