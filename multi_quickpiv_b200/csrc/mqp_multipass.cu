// sm_100a kernel of the multi-pass refinement: the fine pass's whole-pixel
// predictor from the coarse pass's vectors (see mqp_multipass.cuh).
#include <cuda_runtime.h>

#include "mqp_internal.h"

namespace mqp {

__global__ void __launch_bounds__(256) predictor_kernel(PredArgs a, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) predictor_at(a, i);
}

cudaError_t launch_predictor(const PredArgs& a, cudaStream_t s) {
  long long n = 1;
  for (int d = 0; d < a.ndims; ++d) n *= a.vf_f[d];
  if (n < 1) return cudaSuccess;
  predictor_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, n);
  return cudaGetLastError();
}

}  // namespace mqp
