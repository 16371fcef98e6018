// sm_100a kernels of the vector-field post-processing (mqp_post.cuh): one
// thread per vector, plus the mean / standard deviation reduction of
// STD_masking.
#include <cuda_runtime.h>
#include <math.h>

#include "mqp_internal.h"

namespace mqp {

namespace {

constexpr int POST_THREADS = 128;
constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 256;

__global__ void __launch_bounds__(POST_THREADS) post_kernel(PostArgs a) {
  const long long i = (long long)blockIdx.x * POST_THREADS + threadIdx.x;
  if (i < a.n) post_at(a, i);
}

// Deterministic two-stage sums: block partials of sum(x) (mean == null) or
// of sum((x - *mean)^2), then one thread adds the partials in order.
__global__ void __launch_bounds__(RED_THREADS) post_sum_partials(const double* x, long long n, const double* mean,
                                                                 double* part) {
  __shared__ double sh[RED_THREADS];
  const double m = mean ? *mean : 0.0;
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (long long)gridDim.x * RED_THREADS)
    s += mean ? (x[i] - m) * (x[i] - m) : x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// out[0] = sum(part) / div
__global__ void post_sum_final(const double* part, int nparts, double div, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += part[b];
    *out = s / div;
  }
}

// stats = {mean, variance}: the mask |map - mean| > n * sqrt(variance)
__global__ void __launch_bounds__(POST_THREADS) post_std_mask_kernel(PostArgs a, const double* stats) {
  const long long i = (long long)blockIdx.x * POST_THREADS + threadIdx.x;
  if (i >= a.n) return;
  PostArgs b = a;
  b.p1 = stats[0];
  b.p2 = sqrt(stats[1]);
  post_std_mask_at(b, i);
}

}  // namespace

size_t post_scratch_bytes() { return (RED_BLOCKS + 2) * sizeof(double); }

cudaError_t launch_post(const PostArgs& a, double* scratch, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((a.n + POST_THREADS - 1) / POST_THREADS);
  if (a.op == POST_STD_MASK) {
    // Statistics.mean(map) and Statistics.std(map; mean) (n - 1 normalised)
    double* part = scratch;
    double* stats = scratch + RED_BLOCKS;
    post_sum_partials<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a.VF, a.n, nullptr, part);
    post_sum_final<<<1, 32, 0, s>>>(part, RED_BLOCKS, (double)a.n, stats + 0);
    post_sum_partials<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a.VF, a.n, stats + 0, part);
    post_sum_final<<<1, 32, 0, s>>>(part, RED_BLOCKS, (double)(a.n - 1), stats + 1);
    post_std_mask_kernel<<<blocks, POST_THREADS, 0, s>>>(a, stats);
    return cudaGetLastError();
  }
  post_kernel<<<blocks, POST_THREADS, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace mqp
