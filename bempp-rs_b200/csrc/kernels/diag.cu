// Fused multiply-add throughput probe: the CUDA-core FP64 / FP32 peak that the
// regular-quadrature kernels are measured against (no tensor cores on this path).
// Each thread runs kChains independent dependency chains of fma(x, a, b) so that the
// FMA pipes, not latency, bound the loop.
#include "launch.h"

namespace bempp_b200 {
namespace {

constexpr int kChains = 8;

template <typename T>
__global__ void fma_chain_kernel(T* out, int iters, T a, T b) {
  T x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = static_cast<T>(threadIdx.x + c) * static_cast<T>(1e-3);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == static_cast<T>(-12345.678)) out[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

// Returns the sustained FMA throughput in TFLOP/s (2 flops per FMA) over `reps` timed
// launches after one warm-up launch.
cudaError_t measure_fma_peak(int fp64, int iters, int reps, double* tflops) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int threads = 256, blocks = sms * 8;
  void* out = nullptr;
  e = cudaMalloc(&out, threads * sizeof(double));
  if (e != cudaSuccess) return e;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto launch = [&]() {
    if (fp64)
      fma_chain_kernel<double><<<blocks, threads>>>(static_cast<double*>(out), iters, 0.999999, 1e-7);
    else
      fma_chain_kernel<float><<<blocks, threads>>>(static_cast<float*>(out), iters, 0.999999f, 1e-7f);
  };
  launch();
  cudaEventRecord(t0);
  for (int r = 0; r < reps; ++r) launch();
  cudaEventRecord(t1);
  e = cudaEventSynchronize(t1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
  if (e == cudaSuccess) e = cudaGetLastError();
  const double flops = 2.0 * kChains * static_cast<double>(iters) * threads * blocks * reps;
  *tflops = ms > 0 ? flops / (ms * 1e-3) / 1e12 : 0.0;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(out);
  return e;
}

}  // namespace bempp_b200
