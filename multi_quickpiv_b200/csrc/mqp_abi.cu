// C ABI of the PIV hot path (include/mqp.h): contexts, parameter
// resolution with the reference's error behaviour, device buffers and the
// host<->device plumbing around the kernels.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "mqp.h"
#include "mqp_internal.h"

namespace {

thread_local std::string g_create_error;

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
};

}  // namespace

struct mqp_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  std::mutex mu;
  DevBuf img1, img2, mask, mask_skip, II1, IIg, IIg2, VF, SN, pred, planes, status, iscratch;
  // tracing
  bool profile = false;
  struct Span {
    cudaEvent_t a, b;
    int kind;  // 0 integral, 1 piv, 2 other
    int64_t ia;
  };
  std::vector<Span> spans;
  mqp_profile prof{};
};

namespace {

struct ProfileScope {
  mqp_ctx* ctx;
  cudaStream_t s;
  mqp_ctx::Span sp{};
  bool on;
  ProfileScope(mqp_ctx* c, cudaStream_t st, int kind, int64_t ia) : ctx(c), s(st), on(c->profile) {
    if (!on) return;
    sp.kind = kind;
    sp.ia = ia;
    cudaEventCreate(&sp.a);
    cudaEventCreate(&sp.b);
    cudaEventRecord(sp.a, s);
  }
  ~ProfileScope() {
    if (!on) return;
    cudaEventRecord(sp.b, s);
    ctx->spans.push_back(sp);
  }
};

}  // namespace

namespace {

// A resolved single-pass problem: per-axis sizes after toDims3 / _isize /
// _smarg / _step (src/piv_parameters.jl:83-87).
struct Problem {
  int ndims = 2;
  int64_t dims[3] = {1, 1, 1};
  int IS[3] = {0, 0, 0}, SM[3] = {0, 0, 0}, st[3] = {1, 1, 1};
  int64_t vf[3] = {1, 1, 1};
  int64_t n_ia = 0;
  int alg = 2;
};

int fail(mqp_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  else g_create_error = msg;
  return code;
}

int cuda_fail(mqp_ctx* ctx, cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? MQP_ERR_OOM : MQP_ERR_CUDA;
  return fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

// get_vectorfield_size (src/utils/piv_ops.jl:11-14)
int64_t vf_len(int64_t size, int IS, int st) {
  const int64_t stop = size - IS + 1;
  return stop < 1 ? 0 : (stop - 1) / st + 1;
}

int resolve(mqp_ctx* ctx, const mqp_params* p, int ndims, const int64_t dims[3], bool masked,
            int scale, Problem& pb) {
  if (!p || !dims) return fail(ctx, MQP_ERR_INVALID, "null parameter or dims pointer");
  if (ndims != 2 && ndims != 3) return fail(ctx, MQP_ERR_INVALID, "ndims must be 2 or 3");
  // gaussian_displacement's padded branch is a broken path in the reference
  // (src/utils/piv_ops.jl:261-266 prints ERROR and indexes out of range)
  if (!p->unpadded)
    return fail(ctx, MQP_ERR_UNSUPPORTED,
                "ERROR: all gaussian_displacement should be unpadded (stored unpadded must be true; "
                "setPIVParameters stores the good_pad argument there)");
  if (p->multipass < 1) return fail(ctx, MQP_ERR_INVALID, "multipass must be >= 1");
  pb.ndims = ndims;
  pb.alg = masked ? mqp::ALG_MASK_NSQECC : p->corr_alg;
  if (!masked && (p->corr_alg < 0 || p->corr_alg > 2))
    return fail(ctx, MQP_ERR_INVALID, "corr_alg must be MQP_FFTCC, MQP_ZNCC or MQP_NSQECC");
  pb.n_ia = 1;
  for (int d = 0; d < 3; ++d) {
    pb.dims[d] = d < ndims ? dims[d] : 1;
    if (d >= ndims) {
      pb.vf[d] = 1;
      continue;
    }
    if (dims[d] < 1) return fail(ctx, MQP_ERR_INVALID, "image extents must be >= 1");
    if (dims[d] > (int64_t)1 << 30) return fail(ctx, MQP_ERR_INVALID, "image extent too large");
    pb.IS[d] = p->interSize[d] * scale;
    pb.SM[d] = p->searchMargin[d] * scale;
    pb.st[d] = p->has_step ? p->step[d] * scale : pb.IS[d] - p->overlap[d] * scale;
    if (pb.IS[d] < 1) return fail(ctx, MQP_ERR_INVALID, "interSize must be >= 1 along every image axis");
    if (pb.SM[d] < 0) return fail(ctx, MQP_ERR_INVALID, "searchMargin must be >= 0");
    if (pb.st[d] < 1) return fail(ctx, MQP_ERR_INVALID, "step (or interSize - overlap) must be >= 1");
    pb.vf[d] = vf_len(dims[d], pb.IS[d], pb.st[d]);
    pb.n_ia *= pb.vf[d];
  }
  return MQP_OK;
}

}  // namespace

extern "C" {

int mqp_abi_version(void) { return MQP_ABI_VERSION; }

int mqp_create(mqp_ctx** out, int device) {
  if (!out) return fail(nullptr, MQP_ERR_INVALID, "null output pointer");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return fail(nullptr, MQP_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  if (device < 0 || device >= n) return fail(nullptr, MQP_ERR_CUDA, "no such CUDA device: " + std::to_string(device));
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(nullptr, MQP_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  mqp_ctx* c = new mqp_ctx();
  c->device = device;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(nullptr, MQP_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  *out = c;
  return MQP_OK;
}

int mqp_destroy(mqp_ctx* ctx) {
  if (!ctx) return MQP_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (DevBuf* b : {&ctx->img1, &ctx->img2, &ctx->mask, &ctx->mask_skip, &ctx->II1, &ctx->IIg, &ctx->IIg2,
                    &ctx->VF, &ctx->SN, &ctx->pred, &ctx->planes, &ctx->status, &ctx->iscratch})
    b->release();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return MQP_OK;
}

const char* mqp_last_error(const mqp_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : g_create_error.c_str();
}

int mqp_vf_dims(const mqp_params* p, int ndims, const int64_t dims[3], int64_t vf_dims_out[3]) {
  Problem pb;
  mqp_params q;
  if (!p) return fail(nullptr, MQP_ERR_INVALID, "null parameters");
  q = *p;
  q.unpadded = 1;  // shape only
  int rc = resolve(nullptr, &q, ndims, dims, false, 1, pb);
  if (rc != MQP_OK) return rc;
  for (int d = 0; d < 3; ++d) vf_dims_out[d] = pb.vf[d];
  return MQP_OK;
}

}  // extern "C"

namespace {

size_t elem_size(int dtype) { return dtype == MQP_F64 ? 8 : 4; }

// Enqueue one pass of the 2D path on device arrays.
int run_pass_2d(mqp_ctx* ctx, const Problem& pb, const mqp_params* p, const void* d1, const void* d2,
                const void* dmask, const void* dskip, int dtype, double* dVF, double* dSN,
                const int32_t* dpred, double* dplanes, int64_t ia_begin, int64_t ia_end, cudaStream_t s) {
  const int H = (int)pb.dims[0], W = (int)pb.dims[1];
  const int SS1 = pb.IS[0] + 2 * pb.SM[0], SS2 = pb.IS[1] + 2 * pb.SM[1];
  if (mqp::piv2d_fft_len(SS1, SS2) == 0)
    return fail(ctx, MQP_ERR_UNSUPPORTED, "2D search window (interSize + 2 searchMargin) above 64 is not supported yet");
  if (pb.IS[0] > H || pb.IS[1] > W) return MQP_OK;  // empty vector field
  const size_t ii_bytes = (size_t)(H + 1) * (size_t)(W + 1) * sizeof(double);
  cudaError_t e;
  mqp::Piv2dArgs a;
  memset(&a, 0, sizeof(a));
  a.img1 = d1;
  a.img2 = d2;
  a.mask = dmask;
  a.mask_skip = dskip;
  a.mask_threshold = p->mask_threshold;
  a.dtype = dtype;
  if (pb.alg == mqp::ALG_NSQECC || pb.alg == mqp::ALG_ZNCC) {
    if ((e = ctx->iscratch.ensure(mqp::integral2d_scratch_bytes(H, W))) != cudaSuccess)
      return cuda_fail(ctx, e, "integral scratch");
  }
  double* isc = (double*)ctx->iscratch.ptr;
  if (pb.alg == mqp::ALG_NSQECC || pb.alg == mqp::ALG_ZNCC) {
    ProfileScope ps(ctx, s, 0, 0);
    if ((e = ctx->IIg2.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
    if ((e = mqp::launch_integral2d(d2, dtype, H, W, true, (double*)ctx->IIg2.ptr, isc, s)) != cudaSuccess)
      return cuda_fail(ctx, e, "integral image of img2^2");
    a.IIg2 = (const double*)ctx->IIg2.ptr;
  }
  if (pb.alg == mqp::ALG_ZNCC) {
    ProfileScope ps(ctx, s, 0, 0);
    if ((e = ctx->IIg.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
    if ((e = ctx->II1.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
    if ((e = mqp::launch_integral2d(d2, dtype, H, W, false, (double*)ctx->IIg.ptr, isc, s)) != cudaSuccess)
      return cuda_fail(ctx, e, "integral image of img2");
    if ((e = mqp::launch_integral2d(d1, dtype, H, W, false, (double*)ctx->II1.ptr, isc, s)) != cudaSuccess)
      return cuda_fail(ctx, e, "integral image of img1");
    a.IIg = (const double*)ctx->IIg.ptr;
    a.II1 = (const double*)ctx->II1.ptr;
  }
  a.pred = dpred;
  a.VF = dVF;
  a.SN = dSN;
  a.planes = dplanes;
  a.H = H;
  a.W = W;
  a.IS1 = pb.IS[0];
  a.IS2 = pb.IS[1];
  a.SM1 = pb.SM[0];
  a.SM2 = pb.SM[1];
  a.st1 = pb.st[0];
  a.st2 = pb.st[1];
  a.vf1 = (int)pb.vf[0];
  a.vf2 = (int)pb.vf[1];
  a.ia_begin = ia_begin;
  a.ia_end = ia_end;
  a.threshold = p->threshold;
  a.computeSN = dSN != nullptr;
  std::string err;
  {
    ProfileScope ps(ctx, s, 1, ia_end - ia_begin);
    e = mqp::launch_piv2d(a, pb.alg, s, err);
  }
  if (e != cudaSuccess) return fail(ctx, e == cudaErrorInvalidValue ? MQP_ERR_UNSUPPORTED : MQP_ERR_CUDA, err);
  return MQP_OK;
}

int piv_device_impl(mqp_ctx* ctx, const void* d1, const void* d2, const void* dmask, const void* dmask_skip,
                    int dtype, int ndims, const int64_t dims[3], const mqp_params* p, double* dVF,
                    double* dSN, cudaStream_t s, double* dplanes, int64_t ia_begin, int64_t ia_end) {
  if (dtype != MQP_F32 && dtype != MQP_F64) return fail(ctx, MQP_ERR_INVALID, "dtype must be MQP_F32 or MQP_F64");
  if (!d1 || !d2 || !dVF) return fail(ctx, MQP_ERR_INVALID, "null image or VF pointer");
  const bool masked = dmask != nullptr;
  Problem pb;
  int rc = resolve(ctx, p, ndims, dims, masked, 1, pb);
  if (rc != MQP_OK) return rc;
  if (ndims == 3) return fail(ctx, MQP_ERR_UNSUPPORTED, "3D PIV is not available in this build");
  if (pb.n_ia == 0) return MQP_OK;
  if (ia_end < 0) ia_end = pb.n_ia;
  if (ia_begin < 0 || ia_begin > ia_end || ia_end > pb.n_ia) return fail(ctx, MQP_ERR_INVALID, "IA range outside the vector field");
  if (!p->computeSN) dSN = nullptr;
  // multipass without refinement re-runs the scale-1 geometry with identical
  // results (src/multi_quickPIV.jl:57, Q6): one pass gives the same VF/SN
  return run_pass_2d(ctx, pb, p, d1, d2, dmask, dmask_skip, dtype, dVF, dSN, nullptr, dplanes, ia_begin, ia_end, s);
}

}  // namespace

extern "C" {

int mqp_piv_device(mqp_ctx* ctx, const void* d_img1, const void* d_img2, const void* d_mask,
                   const void* d_mask_skip, int dtype, int ndims, const int64_t dims[3],
                   const mqp_params* p, double* d_VF, double* d_SN, void* stream) {
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : cudaStreamLegacy;
  return piv_device_impl(ctx, d_img1, d_img2, d_mask, d_mask_skip, dtype, ndims, dims, p, d_VF, d_SN, s,
                         nullptr, 0, -1);
}

static int host_roundtrip(mqp_ctx* ctx, const void* img1, const void* img2, const void* mask,
                          const void* mask_skip, int dtype, int ndims, const int64_t dims[3],
                          const mqp_params* p, double* VF, double* SN, int64_t vf_dims_out[3],
                          double* planes, int64_t ia_begin, int64_t ia_end) {
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  if (!img1 || !img2) return fail(ctx, MQP_ERR_INVALID, "null image pointer");
  if (dtype != MQP_F32 && dtype != MQP_F64) return fail(ctx, MQP_ERR_INVALID, "dtype must be MQP_F32 or MQP_F64");
  Problem pb;
  int rc = resolve(ctx, p, ndims, dims, mask != nullptr, 1, pb);
  if (rc != MQP_OK) return rc;
  if (vf_dims_out)
    for (int d = 0; d < 3; ++d) vf_dims_out[d] = pb.vf[d];
  size_t npx = 1;
  for (int d = 0; d < ndims; ++d) npx *= (size_t)dims[d];
  const size_t ib = npx * elem_size(dtype);
  const size_t nvf = (size_t)pb.n_ia;
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  if ((e = ctx->img1.ensure(ib)) != cudaSuccess) return cuda_fail(ctx, e, "image buffer");
  if ((e = ctx->img2.ensure(ib)) != cudaSuccess) return cuda_fail(ctx, e, "image buffer");
  if ((e = cudaMemcpyAsync(ctx->img1.ptr, img1, ib, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy img1");
  if ((e = cudaMemcpyAsync(ctx->img2.ptr, img2, ib, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy img2");
  const void* dmask = nullptr;
  const void* dskip = nullptr;
  if (mask) {
    if ((e = ctx->mask.ensure(ib)) != cudaSuccess) return cuda_fail(ctx, e, "mask buffer");
    if ((e = cudaMemcpyAsync(ctx->mask.ptr, mask, ib, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy mask");
    dmask = ctx->mask.ptr;
  }
  if (mask_skip) {
    if ((e = ctx->mask_skip.ensure(ib)) != cudaSuccess) return cuda_fail(ctx, e, "mask buffer");
    if ((e = cudaMemcpyAsync(ctx->mask_skip.ptr, mask_skip, ib, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy mask");
    dskip = ctx->mask_skip.ptr;
  }
  const size_t vfb = (nvf ? nvf : 1) * ndims * sizeof(double);
  if ((e = ctx->VF.ensure(vfb)) != cudaSuccess) return cuda_fail(ctx, e, "VF buffer");
  if ((e = cudaMemsetAsync(ctx->VF.ptr, 0, vfb, s)) != cudaSuccess) return cuda_fail(ctx, e, "VF memset");
  double* dSN = nullptr;
  if (p->computeSN) {
    if ((e = ctx->SN.ensure((nvf ? nvf : 1) * sizeof(double))) != cudaSuccess) return cuda_fail(ctx, e, "SN buffer");
    if ((e = cudaMemsetAsync(ctx->SN.ptr, 0, (nvf ? nvf : 1) * sizeof(double), s)) != cudaSuccess) return cuda_fail(ctx, e, "SN memset");
    dSN = (double*)ctx->SN.ptr;
  }
  double* dplanes = nullptr;
  size_t planes_bytes = 0;
  if (planes) {
    if (ia_end < 0) ia_end = pb.n_ia;
    size_t per = 1;
    for (int d = 0; d < ndims; ++d) per *= (size_t)(2 * pb.SM[d] + 1);
    planes_bytes = per * (size_t)(ia_end - ia_begin > 0 ? ia_end - ia_begin : 0) * sizeof(double);
    if ((e = ctx->planes.ensure(planes_bytes ? planes_bytes : 8)) != cudaSuccess) return cuda_fail(ctx, e, "planes buffer");
    dplanes = (double*)ctx->planes.ptr;
  }
  rc = piv_device_impl(ctx, ctx->img1.ptr, ctx->img2.ptr, dmask, dskip, dtype, ndims, dims, p,
                       (double*)ctx->VF.ptr, dSN, s, dplanes, planes ? ia_begin : 0, planes ? ia_end : -1);
  if (rc != MQP_OK) {
    cudaStreamSynchronize(s);
    return rc;
  }
  if (nvf && VF && (e = cudaMemcpyAsync(VF, ctx->VF.ptr, nvf * ndims * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy VF");
  if (nvf && SN && dSN && (e = cudaMemcpyAsync(SN, dSN, nvf * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy SN");
  if (planes && planes_bytes && (e = cudaMemcpyAsync(planes, dplanes, planes_bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy planes");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "PIV kernels");
  return MQP_OK;
}

int mqp_piv(mqp_ctx* ctx, const void* img1, const void* img2, const void* mask, const void* mask_skip,
            int dtype, int ndims, const int64_t dims[3], const mqp_params* p, double* VF, double* SN,
            int64_t vf_dims_out[3]) {
  return host_roundtrip(ctx, img1, img2, mask, mask_skip, dtype, ndims, dims, p, VF, SN, vf_dims_out,
                        nullptr, 0, -1);
}

int mqp_profile_enable(mqp_ctx* ctx, int enable) {
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  for (auto& sp : ctx->spans) {
    cudaEventSynchronize(sp.b);
    cudaEventDestroy(sp.a);
    cudaEventDestroy(sp.b);
  }
  ctx->spans.clear();
  ctx->prof = mqp_profile{};
  ctx->profile = enable != 0;
  return MQP_OK;
}

int mqp_profile_read(mqp_ctx* ctx, mqp_profile* out) {
  if (!ctx || !out) return fail(ctx, MQP_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  for (auto& sp : ctx->spans) {
    cudaError_t e = cudaEventSynchronize(sp.b);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "profile event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, sp.a, sp.b);
    if (sp.kind == 0) {
      ctx->prof.launches_integral += 1;
      ctx->prof.ms_integral += ms;
    } else if (sp.kind == 1) {
      ctx->prof.launches_piv += 1;
      ctx->prof.ms_piv += ms;
      ctx->prof.ia_count += sp.ia;
    } else {
      ctx->prof.launches_other += 1;
      ctx->prof.ms_other += ms;
    }
    cudaEventDestroy(sp.a);
    cudaEventDestroy(sp.b);
  }
  ctx->spans.clear();
  *out = ctx->prof;
  return MQP_OK;
}

int mqp_correlation_planes(mqp_ctx* ctx, const void* img1, const void* img2, const void* mask,
                           int dtype, int ndims, const int64_t dims[3], const mqp_params* p,
                           int64_t ia_begin, int64_t ia_end, double* planes) {
  if (!planes) return fail(ctx, MQP_ERR_INVALID, "null planes buffer");
  return host_roundtrip(ctx, img1, img2, mask, nullptr, dtype, ndims, dims, p, nullptr, nullptr, nullptr,
                        planes, ia_begin, ia_end);
}

}  // extern "C"
