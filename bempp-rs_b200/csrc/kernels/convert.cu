// FP64 staging buffer -> single-precision output (F32 / interleaved C32 matrices).
#include "launch.h"

namespace bempp_b200 {

__global__ void convert_to_single_kernel(const double* __restrict__ src, float* __restrict__ dst,
                                         size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    dst[i] = static_cast<float>(src[i]);
}

cudaError_t launch_convert_to_single(const double* src, void* dst, size_t n_reals,
                                     cudaStream_t stream) {
  if (n_reals == 0) return cudaSuccess;
  int blocks = static_cast<int>(std::min<size_t>((n_reals + 255) / 256, 148 * 16));
  convert_to_single_kernel<<<blocks, 256, 0, stream>>>(src, static_cast<float*>(dst), n_reals);
  return cudaGetLastError();
}

}  // namespace bempp_b200
