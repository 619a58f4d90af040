// Roofline calibration: the sustained FP32 FFMA throughput and the MUFU
// reciprocal-square-root throughput of this GPU, each measured with
// independent dependency chains (8 per thread, no memory traffic). The FP32
// far field needs 8 FMA-pipe operations and 1 MUFU.RSQ per quadrature pair,
// so both pipes bound it; its roofline fraction is reported against these
// measured figures rather than nominal spec-sheet numbers.
#include <cuda_runtime.h>

#include <string>

#include "common.h"

namespace eb {

__global__ void ffma_chain_kernel(float* out, int iters, float a, float b)
{
  float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
        x7 = x0 + 7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 1.2345f) out[blockIdx.x] = s;  // keeps the chains live
}

__device__ __forceinline__ float rsq_approx(float x)
{
  float y;
  asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__global__ void rsqrt_chain_kernel(float* out, int iters)
{
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = 1.0f + threadIdx.x + k;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = rsq_approx(x[k]) + 1.0f;
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == 1.2345f) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace eb

extern "C" int eb_measure_rsqrt_peak(double* tops, double* seconds)
{
  if (!tops) return eb::set_error(EB_ERR_INVALID, "null output");
  int dev = 0, nsm = 0;
  EB_CUDA(cudaGetDevice(&dev));
  EB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  float* out = nullptr;
  EB_CUDA(cudaMalloc(&out, sizeof(float) * 65536));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = nsm * 8, iters = 2048;
  eb::rsqrt_chain_kernel<<<blocks, threads>>>(out, 64);  // warm-up
  cudaEventRecord(e0);
  eb::rsqrt_chain_kernel<<<blocks, threads>>>(out, iters);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return eb::set_error(EB_ERR_CUDA, cudaGetErrorString(err));
  const double ops = 8.0 * iters * (double)threads * blocks;
  *tops = ops / (ms * 1e-3) / 1e12;
  if (seconds) *seconds = ms * 1e-3;
  return EB_OK;
}

extern "C" int eb_measure_fp32_peak(double* tflops, double* seconds)
{
  if (!tflops) return eb::set_error(EB_ERR_INVALID, "null output");
  int dev = 0, nsm = 0;
  EB_CUDA(cudaGetDevice(&dev));
  EB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  float* out = nullptr;
  EB_CUDA(cudaMalloc(&out, sizeof(float) * 65536));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = nsm * 8, iters = 4096;
  eb::ffma_chain_kernel<<<blocks, threads>>>(out, 64, 0.999f, 0.001f);  // warm-up
  cudaEventRecord(e0);
  eb::ffma_chain_kernel<<<blocks, threads>>>(out, iters, 0.999f, 0.001f);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return eb::set_error(EB_ERR_CUDA, cudaGetErrorString(err));
  const double flops = 2.0 * 8.0 * 16.0 * iters * (double)threads * blocks;
  *tflops = flops / (ms * 1e-3) / 1e12;
  if (seconds) *seconds = ms * 1e-3;
  return EB_OK;
}
