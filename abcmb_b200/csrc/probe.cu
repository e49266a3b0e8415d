// probe.cu -- FP64 FMA-rate probe: the denominator of the ODE kernel's roofline.
//
// Every thread runs 8 independent dependent-FMA chains (enough to cover the
// FP64 pipe latency) on a grid of 8 blocks of 256 threads per SM; the rate is
// 2 * FMAs / CUDA-event time.
#include <cuda_runtime.h>
#include "../../include/abcmb_b200.h"

namespace {
__global__ void fp64_fma_kernel(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
  double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 123.456) out[0] = s;   // keeps the chains live
}
}  // namespace

extern "C" int abcmb_probe_fp64_tflops(double* tflops, int iters, void* stream) {
  if (!tflops || iters <= 0) return ABCMB_ERR_ARG;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  double* scratch = nullptr;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = nsm * 8, threads = 256;
  fp64_fma_kernel<<<blocks, threads, 0, st>>>(scratch, 4, 0.999999, 1e-7);   // warm-up
  double best = 0.;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0, st);
    fp64_fma_kernel<<<blocks, threads, 0, st>>>(scratch, iters, 0.999999, 1e-7);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    double tf = flops / (ms * 1e-3) / 1e12;
    if (tf > best) best = tf;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return ABCMB_ERR_CUDA;
  *tflops = best;
  return ABCMB_OK;
}
