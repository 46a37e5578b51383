// FP64 FMA throughput probe: the denominator the FP64 contraction kernels are
// reported against (the measured peaks file of this pool carries HBM and BF16
// figures only).  Each thread runs 8 independent FMA chains in registers.
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
