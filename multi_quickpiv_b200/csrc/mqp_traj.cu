// Pseudo-trajectories over a vector-field time series on the GPU:
// PIVtrajectories and PIVtrajectories_grid
// (src/postprocessing/postprocessing.jl:988-1120).  One thread follows one
// particle through the frames, exactly as the reference's per-particle loop:
// Float32 positions, the displacement sampled at the rounded (ties to even)
// position, and the rest of the trajectory frozen at the last position once
// that rounded position leaves the field.  Starting positions of the random
// variant come from a counter-based generator (splitmix64 of seed and
// particle/axis), since Julia's `rand` stream is not reproducible here; the
// grid variant is deterministic like the reference's.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>

#include "mqp_ctx.h"

namespace mqp {

struct TrajArgs {
  const void* comp[3];  // U, V, W: frames of the field, column-major (d1, d2[, d3], frames)
  int dtype;            // 0 float32, 1 float64
  int nd;               // 2 or 3 grid axes
  long long dims[3];    // grid extents (dims[2] = 1 for nd = 2)
  long long frames;
  int T0;               // 1-based first frame
  int numT;             // time points per trajectory (T1 - T0)
  long long lo[3], len[3], step[3];  // sampling range per axis: lo + step * k, k < len (1-based)
  double scale[3];
  int grid;
  long long np;         // particles
  unsigned long long seed;
  float* out[3];        // (numT, np) Float32 each, column-major
};

// splitmix64 finaliser of seed + (3 p + d + 1) * golden ratio: the random
// start of particle p along axis d is lo + step * (h % len)
__host__ __device__ inline unsigned long long traj_hash(unsigned long long seed, long long p, int d) {
  unsigned long long z = seed + (unsigned long long)(3 * p + d + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

namespace {

__device__ __forceinline__ double traj_load(const void* a, int dtype, long long i) {
  return dtype == 0 ? (double)__ldg((const float*)a + i) : __ldg((const double*)a + i);
}

__global__ void traj_kernel(TrajArgs a) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.np) return;
  long long s[3] = {1, 1, 1};
  long long rem = p;
  for (int d = 0; d < a.nd; ++d) {
    long long k;
    if (a.grid) {  // for z, for x, for y: y fastest (postprocessing.jl:1070)
      k = rem % a.len[d];
      rem /= a.len[d];
    } else {
      k = (long long)(traj_hash(a.seed, p, d) % (unsigned long long)a.len[d]);
    }
    s[d] = a.lo[d] + a.step[d] * k;
  }
  const long long plane = a.dims[0] * a.dims[1] * a.dims[2];
  auto at = [&](const long long (&q)[3], int frame0) {
    return (q[0] - 1) + a.dims[0] * ((q[1] - 1) + a.dims[1] * (q[2] - 1)) + plane * (long long)frame0;
  };
  float pos[3], dv[3] = {0.f, 0.f, 0.f};
  for (int d = 0; d < a.nd; ++d) {
    pos[d] = (float)s[d];
    a.out[d][(long long)a.numT * p] = pos[d];
  }
  long long q[3] = {s[0], s[1], s[2]};
  for (int d = 0; d < a.nd; ++d)
    dv[d] = (float)(a.scale[d] * traj_load(a.comp[d], a.dtype, at(q, a.T0 - 1)));
  for (int t = 1; t < a.numT; ++t) {
    bool out = false;
    for (int d = 0; d < a.nd; ++d) {
      const float prev = pos[d];
      pos[d] = prev + dv[d];
      a.out[d][t + (long long)a.numT * p] = pos[d];
      const float r = rintf(pos[d]);  // round(Int64, x): to nearest, ties to even
      if (!(r >= 1.f && r <= (float)a.dims[d])) out = true;  // NaN counts as outside
      else q[d] = (long long)r;
    }
    if (out) {
      // freeze the rest of the trajectory at the last position inside
      for (int d = 0; d < a.nd; ++d) {
        const float prev = a.out[d][(t - 1) + (long long)a.numT * p];
        for (int u = t; u < a.numT; ++u) a.out[d][u + (long long)a.numT * p] = prev;
      }
      return;
    }
    for (int d = 0; d < a.nd; ++d)
      dv[d] = (float)(a.scale[d] * traj_load(a.comp[d], a.dtype, at(q, a.T0 - 1 + t)));
  }
}

// The sampling ranges and counts of a request (or an error message).
std::string traj_resolve(const mqp_traj_params* p, TrajArgs& a) {
  if (!p) return "null parameters";
  if (p->ndims != 2 && p->ndims != 3) return "ndims must be 2 or 3";
  memset(&a, 0, sizeof(a));
  a.nd = p->ndims;
  for (int d = 0; d < 3; ++d) {
    a.dims[d] = d < a.nd ? p->dims[d] : 1;
    if (a.dims[d] < 1 || a.dims[d] > ((long long)1 << 24)) return "grid extents must be in [1, 2^24]";
  }
  a.frames = p->frames;
  a.T0 = p->T0;
  a.numT = p->T1 - p->T0;
  if (a.numT < 1) return "T1 must be above T0 (numT = T1 - T0 time points)";
  if (p->T0 < 1 || (long long)p->T1 - 1 > p->frames)
    return "frames T0 .. T1-1 (1-based) must exist: the last step samples frame T1-1";
  a.grid = p->grid != 0;
  a.np = 1;
  for (int d = 0; d < a.nd; ++d) {
    long long lo = p->sub_lo[d], hi = p->sub_hi[d];
    if (lo > hi) {  // an empty subregion samples 2:dims-1 (postprocessing.jl:1000, 1061)
      lo = 2;
      hi = a.dims[d] - 1;
    }
    const long long st = a.grid ? p->step[d] : 1;
    if (st < 1) return "step must be >= 1";
    if (hi < lo) return "empty sampling range (a field axis shorter than 3 with the default subregion)";
    if (lo < 1 || hi > a.dims[d]) return "subregion outside the field";
    a.lo[d] = lo;
    a.step[d] = st;
    a.len[d] = (hi - lo) / st + 1;
    a.np *= a.len[d];
    a.scale[d] = p->scale[d];
  }
  if (!a.grid) {
    if (p->numpoints < 0) return "numpoints must be >= 0";
    a.np = p->numpoints;
  }
  a.seed = p->seed;
  return "";
}

}  // namespace
}  // namespace mqp

using mqp_host::cuda_fail;
using mqp_host::fail;

namespace {

// Enqueue the kernel for a resolved request (the caller holds the context lock).
int traj_launch(mqp_ctx* ctx, mqp::TrajArgs a, int dtype, const void* const (&comp)[3], float* const (&out)[3],
                cudaStream_t s) {
  a.dtype = dtype;
  for (int d = 0; d < 3; ++d) {
    a.comp[d] = comp[d];
    a.out[d] = out[d];
  }
  const int threads = 128;
  const long long blocks = (a.np + threads - 1) / threads;
  if (blocks > 0x7fffffffLL) return fail(ctx, MQP_ERR_INVALID, "too many particles");
  mqp::traj_kernel<<<(unsigned)blocks, threads, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "trajectory kernel");
  return MQP_OK;
}

}  // namespace

extern "C" {

int mqp_traj_count(const mqp_traj_params* p, int64_t* numpoints_out) {
  mqp::TrajArgs a;
  const std::string msg = mqp::traj_resolve(p, a);
  if (!msg.empty()) return fail(nullptr, MQP_ERR_INVALID, msg);
  if (numpoints_out) *numpoints_out = a.np;
  return MQP_OK;
}

int mqp_trajectories_device(mqp_ctx* ctx, const mqp_traj_params* p, int dtype, const void* d_U, const void* d_V,
                            const void* d_W, float* d_TY, float* d_TX, float* d_TZ, void* stream) {
  mqp_host::NvtxRange nv("mqp_trajectories_device");
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  mqp::TrajArgs a;
  const std::string msg = mqp::traj_resolve(p, a);
  if (!msg.empty()) return fail(ctx, MQP_ERR_INVALID, msg);
  if (dtype != MQP_F32 && dtype != MQP_F64) return fail(ctx, MQP_ERR_INVALID, "dtype must be MQP_F32 or MQP_F64");
  if (a.np == 0) return MQP_OK;
  if (!d_U || !d_V || (a.nd == 3 && !d_W) || !d_TY || !d_TX || (a.nd == 3 && !d_TZ))
    return fail(ctx, MQP_ERR_INVALID, "null field component or trajectory array");
  const void* comp[3] = {d_U, d_V, d_W};
  float* out[3] = {d_TY, d_TX, d_TZ};
  return traj_launch(ctx, a, dtype, comp, out, stream ? (cudaStream_t)stream : cudaStreamLegacy);
}

int mqp_trajectories(mqp_ctx* ctx, const mqp_traj_params* p, int dtype, const void* U, const void* V, const void* W,
                     float* TY, float* TX, float* TZ) {
  mqp_host::NvtxRange nv("mqp_trajectories");
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  mqp::TrajArgs a;
  const std::string msg = mqp::traj_resolve(p, a);
  if (!msg.empty()) return fail(ctx, MQP_ERR_INVALID, msg);
  if (dtype != MQP_F32 && dtype != MQP_F64) return fail(ctx, MQP_ERR_INVALID, "dtype must be MQP_F32 or MQP_F64");
  if (a.np == 0) return MQP_OK;
  if (!U || !V || (a.nd == 3 && !W) || !TY || !TX || (a.nd == 3 && !TZ))
    return fail(ctx, MQP_ERR_INVALID, "null field component or trajectory array");
  // only frames T0 .. T1-1 are read: copy those, and present them as frames 1..numT
  const size_t es = dtype == MQP_F32 ? 4 : 8;
  const size_t plane = (size_t)(a.dims[0] * a.dims[1] * a.dims[2]);
  const size_t comp_b = plane * (size_t)a.numT * es;
  const size_t n = (size_t)a.numT * (size_t)a.np;
  cudaError_t e;
  if ((e = ctx->traj_in.ensure(comp_b * a.nd)) != cudaSuccess) return cuda_fail(ctx, e, "trajectory buffer");
  if ((e = ctx->traj_out.ensure(n * sizeof(float) * a.nd)) != cudaSuccess) return cuda_fail(ctx, e, "trajectory buffer");
  const void* host_in[3] = {U, V, W};
  float* host_out[3] = {TY, TX, TZ};
  const void* comp[3] = {nullptr, nullptr, nullptr};
  float* out[3] = {nullptr, nullptr, nullptr};
  for (int d = 0; d < a.nd; ++d) {
    char* dst = (char*)ctx->traj_in.ptr + d * comp_b;
    const char* src = (const char*)host_in[d] + plane * (size_t)(a.T0 - 1) * es;
    if ((e = cudaMemcpyAsync(dst, src, comp_b, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy in");
    comp[d] = dst;
    out[d] = (float*)ctx->traj_out.ptr + d * n;
  }
  a.frames = a.numT;
  a.T0 = 1;
  int rc = traj_launch(ctx, a, dtype, comp, out, ctx->stream);
  if (rc != MQP_OK) return rc;
  for (int d = 0; d < a.nd; ++d)
    if ((e = cudaMemcpyAsync(host_out[d], out[d], n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy out");
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "trajectories");
  return MQP_OK;
}

}  // extern "C"
