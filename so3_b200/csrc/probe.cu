// Throughput probes: the denominators the contraction kernels are reported
// against (the measured peaks file of this pool carries HBM and BF16 figures
// only).  FP64: each thread runs 8 independent FMA chains in registers.
// int8 tensor cores: each warp runs 8 independent mma.sync m16n8k32 s8
// accumulator chains on register operands (the instruction the split-precision
// contractions issue).
#include "so3gpu_internal.h"

namespace so3g {

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

__global__ void int8_mma_chain(int* out, int iters) {
  const unsigned a0 = threadIdx.x * 0x01010101u, a1 = a0 ^ 0x5a5a5a5au, a2 = a0 + 3u, a3 = a0 * 7u;
  const unsigned b0 = a0 ^ 0x33333333u, b1 = a0 + 11u;
  int c[8][4] = {};
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int j = 0; j < 8; j++)
      asm volatile(
          "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
          : "+r"(c[j][0]), "+r"(c[j][1]), "+r"(c[j][2]), "+r"(c[j][3])
          : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
  }
  int s = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) s += c[j][0] + c[j][1] + c[j][2] + c[j][3];
  if (s == 0x7fffffff) out[0] = s;  // keeps the chains live
}

int measure_int8_mma_rate(double* tops) {
  int dev = 0, sms = 0;
  SO3G_CUDA(cudaGetDevice(&dev));
  SO3G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int* out = nullptr;
  SO3G_CUDA(cudaMalloc(&out, sizeof(int)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 4, threads = 256, iters = 2048;
  int8_mma_chain<<<blocks, threads>>>(out, iters);  // warm-up
  SO3G_LAUNCHED();
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(e0);
    int8_mma_chain<<<blocks, threads>>>(out, iters);
    SO3G_LAUNCHED();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  SO3G_CUDA(cudaGetLastError());
  const double ops = 2.0 * 16 * 8 * 32 * 8.0 * iters * (double)blocks * (threads / 32);
  *tops = ops / (best * 1e-3) / 1e12;
  return kOk;
}

int measure_fp64_fma_rate(double* tflops) {
  int dev = 0, sms = 0;
  SO3G_CUDA(cudaGetDevice(&dev));
  SO3G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double* out = nullptr;
  SO3G_CUDA(cudaMalloc(&out, sizeof(double)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  fp64_fma_chain<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);  // warm-up
  SO3G_LAUNCHED();
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(e0);
    fp64_fma_chain<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    SO3G_LAUNCHED();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  SO3G_CUDA(cudaGetLastError());
  const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return kOk;
}

}  // namespace so3g
