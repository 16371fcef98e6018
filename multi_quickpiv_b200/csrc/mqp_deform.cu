// sm_100a kernels of the deforming multi-pass refinement (mqp_deform.cuh):
// one thread per pixel resamples both images around the dense predictor, one
// thread per fine IA adds the predictor back to its residual.
#include <cuda_runtime.h>

#include "mqp_internal.h"

namespace mqp {

namespace {

__global__ void __launch_bounds__(256) deform_kernel(DeformArgs a, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) deform_pixel(a, i);
}

__global__ void __launch_bounds__(128) deform_add_kernel(DeformArgs a, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) deform_add(a, i);
}

}  // namespace

cudaError_t launch_deform(const DeformArgs& a, cudaStream_t s) {
  const long long n = a.dims[0] * a.dims[1] * a.dims[2];
  if (n <= 0) return cudaSuccess;
  deform_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, n);
  return cudaGetLastError();
}

cudaError_t launch_deform_add(const DeformArgs& a, cudaStream_t s) {
  long long n = 1;
  for (int d = 0; d < a.nd; ++d) n *= a.vf_f[d];
  if (n <= 0) return cudaSuccess;
  deform_add_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a, n);
  return cudaGetLastError();
}

}  // namespace mqp
