// peak_fp64.cu - FP64 throughput microbenchmark (libcsdpeak.so).
//
// Measures the FP64 rate of this GPU two ways: DMMA (mma.sync m8n8k4 f64 on
// the tensor cores) and DFMA (scalar fma.rn.f64), each as eight independent
// accumulator chains per thread / warp over a grid of 8 CTAs x 256 threads per
// SM.  bench.py uses the DMMA figure as the compute roofline of the FP64 FISTA
// kernel, since no FP64 figure is part of the driver-measured peaks.
#include <cuda_runtime.h>

#include <cstdio>

namespace {

__global__ void k_dmma(int iters, double seed, double* sink) {
  double d[8][2];
#pragma unroll
  for (int c = 0; c < 8; ++c) d[c][0] = d[c][1] = seed * (threadIdx.x + c);
  const double a = seed * 1.0000001, b = seed * 0.9999999;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 8; ++c)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(d[c][0]), "+d"(d[c][1])
                   : "d"(a), "d"(b));
  }
  double s = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) s += d[c][0] + d[c][1];
  if (s == 12345.678) sink[0] = s;
}

__global__ void k_dfma(int iters, double seed, double* sink) {
  double d[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) d[c] = seed * (threadIdx.x + c);
  const double a = 1.0000001, b = seed * 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 8; ++c) d[c] = fma(d[c], a, b);
  }
  double s = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) s += d[c];
  if (s == 12345.678) sink[0] = s;
}

}  // namespace

extern "C" int csd_peak_fp64(int device, double* dmma_tflops, double* dfma_tflops) {
  if (cudaSetDevice(device) != cudaSuccess) return 4;
  cudaDeviceProp p{};
  cudaGetDeviceProperties(&p, device);
  const int blocks = p.multiProcessorCount * 8, threads = 256;
  double* sink = nullptr;
  if (cudaMalloc(&sink, 64) != cudaSuccess) return 4;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 4096;
  float ms = 0.f;
  // DMMA: 256 FMA = 512 flop per instruction per warp
  k_dmma<<<blocks, threads>>>(64, 1.0, sink);
  cudaEventRecord(e0);
  k_dmma<<<blocks, threads>>>(iters, 1.0, sink);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  const double warps = static_cast<double>(blocks) * threads / 32.0;
  *dmma_tflops = warps * iters * 8.0 * 512.0 / (ms * 1e-3) / 1e12;
  k_dfma<<<blocks, threads>>>(64, 1.0, sink);
  cudaEventRecord(e0);
  k_dfma<<<blocks, threads>>>(iters, 1.0, sink);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  *dfma_tflops = static_cast<double>(blocks) * threads * iters * 8.0 * 2.0 / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}
