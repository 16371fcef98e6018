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
#include "mqp_ctx.h"
#include "mqp_internal.h"

using namespace mqp_host;

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
                    &ctx->VF, &ctx->SN, &ctx->pred, &ctx->planes, &ctx->status, &ctx->iscratch,
                    &ctx->scratch3d, &ctx->passVF[0], &ctx->passVF[1], &ctx->post_in, &ctx->post_mask,
                    &ctx->post_out, &ctx->post_outf, &ctx->post_mask_out, &ctx->post_scratch})
    b->release();
  for (cudaStream_t st : {ctx->in_stream, ctx->out_stream})
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  for (cudaEvent_t ev : ctx->pipe_ev) cudaEventDestroy(ev);
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

namespace mqp_host {

size_t elem_size(int dtype) { return dtype == MQP_F64 ? 8 : 4; }

// The integral images a 2D pass needs (ctx buffers), over image columns
// [x0, x1): the whole image, or one piece of the host-array pipeline.
static int integrals_2d(mqp_ctx* ctx, const Problem& pb, const void* d1, const void* d2, int dtype, cudaStream_t s,
                        int x0, int x1) {
  const int H = (int)pb.dims[0], W = (int)pb.dims[1];
  if (pb.alg != mqp::ALG_NSQECC && pb.alg != mqp::ALG_ZNCC) return MQP_OK;
  const size_t ii_bytes = (size_t)(H + 1) * (size_t)(W + 1) * sizeof(double);
  cudaError_t e;
  // one totals area per integral image: a piece's row offsets read the
  // totals its integral's earlier pieces left
  const size_t tb = mqp::integral2d_scratch_bytes(H, W);
  if ((e = ctx->iscratch.ensure(3 * tb)) != cudaSuccess) return cuda_fail(ctx, e, "integral scratch");
  const bool whole = x0 == 0 && x1 == W;
  auto integral = [&](const void* img, bool sq, double* out, int k) {
    double* isc = (double*)((char*)ctx->iscratch.ptr + k * tb);
    return whole ? mqp::launch_integral2d(img, dtype, H, W, sq, out, isc, s)
                 : mqp::launch_integral2d_cols(img, dtype, H, W, x0, x1, sq, out, isc, s);
  };
  if (!mqp::piv2d_local_sums(pb.IS[0], pb.IS[1], pb.SM[0], pb.SM[1], pb.alg)) {
    ProfileScope ps(ctx, s, 0, 0);
    if ((e = ctx->IIg2.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
    if ((e = integral(d2, true, (double*)ctx->IIg2.ptr, 0)) != cudaSuccess)
      return cuda_fail(ctx, e, "integral image of img2^2");
  }
  if (pb.alg == mqp::ALG_ZNCC) {
    ProfileScope ps(ctx, s, 0, 0);
    if ((e = ctx->IIg.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
    if ((e = ctx->II1.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
    if ((e = integral(d2, false, (double*)ctx->IIg.ptr, 1)) != cudaSuccess)
      return cuda_fail(ctx, e, "integral image of img2");
    if ((e = integral(d1, false, (double*)ctx->II1.ptr, 2)) != cudaSuccess)
      return cuda_fail(ctx, e, "integral image of img1");
  }
  return MQP_OK;
}

// Kernel arguments of a 2D pass over IAs [ia_begin, ia_end) (integral images
// from the ctx buffers).
static mqp::Piv2dArgs args_2d(mqp_ctx* ctx, const Problem& pb, const mqp_params* p, const void* d1, const void* d2,
                              const void* dmask, const void* dskip, int dtype, double* dVF, double* dSN,
                              const int32_t* dpred, double* dplanes, int64_t ia_begin, int64_t ia_end) {
  mqp::Piv2dArgs a;
  memset(&a, 0, sizeof(a));
  a.img1 = d1;
  a.img2 = d2;
  a.mask = dmask;
  a.mask_skip = dskip;
  a.mask_threshold = p->mask_threshold;
  a.dtype = dtype;
  if (pb.alg == mqp::ALG_NSQECC || pb.alg == mqp::ALG_ZNCC) a.IIg2 = (const double*)ctx->IIg2.ptr;
  if (pb.alg == mqp::ALG_ZNCC) {
    a.IIg = (const double*)ctx->IIg.ptr;
    a.II1 = (const double*)ctx->II1.ptr;
  }
  a.pred = dpred;
  a.VF = dVF;
  a.SN = dSN;
  a.planes = dplanes;
  a.H = (int)pb.dims[0];
  a.W = (int)pb.dims[1];
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
  return a;
}

static int launch_2d(mqp_ctx* ctx, const mqp::Piv2dArgs& a, int alg, cudaStream_t s) {
  std::string err;
  cudaError_t e;
  {
    ProfileScope ps(ctx, s, 1, a.ia_end - a.ia_begin);
    e = mqp::launch_piv2d(a, alg, s, err);
  }
  if (e != cudaSuccess) return fail(ctx, e == cudaErrorInvalidValue ? MQP_ERR_UNSUPPORTED : MQP_ERR_CUDA, err);
  return MQP_OK;
}

// Enqueue one pass of the 2D path on device arrays.
int run_pass_2d(mqp_ctx* ctx, const Problem& pb, const mqp_params* p, const void* d1, const void* d2,
                const void* dmask, const void* dskip, int dtype, double* dVF, double* dSN,
                const int32_t* dpred, double* dplanes, int64_t ia_begin, int64_t ia_end, cudaStream_t s) {
  const int H = (int)pb.dims[0], W = (int)pb.dims[1];
  const int SS1 = pb.IS[0] + 2 * pb.SM[0], SS2 = pb.IS[1] + 2 * pb.SM[1];
  const bool huge = mqp::piv2d_fft_len(SS1, SS2) == 0;
  if (huge && !mqp::piv2d_huge_ok(SS1, SS2, pb.IS[0], pb.IS[1], pb.alg))
    return fail(ctx, MQP_ERR_UNSUPPORTED,
                "2D search window (interSize + 2 searchMargin) above 256, or above 128 with an interrogation window "
                "above 128 or a mask, is not supported");
  if (pb.IS[0] > H || pb.IS[1] > W) return MQP_OK;  // empty vector field
  int rc = integrals_2d(ctx, pb, d1, d2, dtype, s, 0, W);
  if (rc != MQP_OK) return rc;
  mqp::Piv2dArgs a = args_2d(ctx, pb, p, d1, d2, dmask, dskip, dtype, dVF, dSN, dpred, dplanes, ia_begin, ia_end);
  if (huge) {
    cudaError_t e = ctx->huge.ensure(mqp::piv2d_huge_scratch_bytes(ctx->device, 2 * pb.SM[0] + 1, 2 * pb.SM[1] + 1));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "scratch of the 2D kernel for search windows above 128");
    a.huge = (float2*)ctx->huge.ptr;
    std::string err;
    {
      ProfileScope ps(ctx, s, 1, ia_end - ia_begin);
      e = mqp::launch_piv2d_huge(a, pb.alg, s, err);
    }
    if (e != cudaSuccess) return fail(ctx, e == cudaErrorInvalidValue ? MQP_ERR_UNSUPPORTED : MQP_ERR_CUDA, err);
    return MQP_OK;
  }
  return launch_2d(ctx, a, pb.alg, s);
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Enqueue one pass of the 3D path on device arrays.
int run_pass_3d(mqp_ctx* ctx, const Problem& pb, const mqp_params* p, const void* d1, const void* d2,
                const void* dmask, const void* dskip, int dtype, double* dVF, double* dSN,
                const int32_t* dpred, double* dplanes, int64_t ia_begin, int64_t ia_end, cudaStream_t s) {
  const int H = (int)pb.dims[0], W = (int)pb.dims[1], D = (int)pb.dims[2];
  const int SS[3] = {pb.IS[0] + 2 * pb.SM[0], pb.IS[1] + 2 * pb.SM[1], pb.IS[2] + 2 * pb.SM[2]};
  if (mqp::piv3d_fft_len(SS) == 0)
    return fail(ctx, MQP_ERR_UNSUPPORTED, "3D search window (interSize + 2 searchMargin) above 64 is not supported yet");
  if (ia_end <= ia_begin) return MQP_OK;
  cudaError_t e;
  mqp::Piv3dArgs a;
  memset(&a, 0, sizeof(a));
  const bool need_g2 = pb.alg == mqp::ALG_NSQECC || pb.alg == mqp::ALG_ZNCC;
  const bool need_g1 = pb.alg == mqp::ALG_ZNCC;
  const size_t ii_bytes = (size_t)(H + 1) * (size_t)(W + 1) * (size_t)(D + 1) * sizeof(double);
  if (need_g2) {
    if ((e = ctx->iscratch.ensure(mqp::integral3d_scratch_bytes(H, W, D))) != cudaSuccess)
      return cuda_fail(ctx, e, "integral scratch");
    double* isc = (double*)ctx->iscratch.ptr;
    ProfileScope ps(ctx, s, 0, 0);
    if ((e = ctx->IIg2.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
    if ((e = mqp::launch_integral3d(d2, dtype, H, W, D, true, (double*)ctx->IIg2.ptr, isc, s)) != cudaSuccess)
      return cuda_fail(ctx, e, "integral volume of img2^2");
    a.IIg2 = (const double*)ctx->IIg2.ptr;
    if (need_g1) {
      if ((e = ctx->IIg.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
      if ((e = ctx->II1.ensure(ii_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "integral buffer");
      if ((e = mqp::launch_integral3d(d2, dtype, H, W, D, false, (double*)ctx->IIg.ptr, isc, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "integral volume of img2");
      if ((e = mqp::launch_integral3d(d1, dtype, H, W, D, false, (double*)ctx->II1.ptr, isc, s)) != cudaSuccess)
        return cuda_fail(ctx, e, "integral volume of img1");
      a.IIg = (const double*)ctx->IIg.ptr;
      a.II1 = (const double*)ctx->II1.ptr;
    }
  }
  const bool direct = mqp::direct3d_ok(pb.IS, pb.SM);  // small windows: spatial correlation, no chunk scratch
  // chunk scratch: Gz | Fz | C | C2 | V | state | K3a parts | K3c parts
  const size_t per_ia = mqp::piv3d_scratch_bytes_per_ia(pb.IS, pb.SM, pb.alg);
  const int64_t n = ia_end - ia_begin;
  int64_t chunk = ctx->chunk3d > 0 ? ctx->chunk3d : (int64_t)(ctx->chunk3d_budget / per_ia);
  if (chunk < 1) chunk = 1;
  if (chunk > 65535) chunk = 65535;
  if (chunk > n) chunk = n;
  for (int d = 0; d < 3; ++d) {
    a.IS[d] = pb.IS[d];
    a.SM[d] = pb.SM[d];
  }
  if (!direct) {
    if ((e = ctx->scratch3d.ensure(mqp::piv3d_scratch_bytes(pb.IS, pb.SM, pb.alg, chunk))) != cudaSuccess)
      return cuda_fail(ctx, e, "3D scratch");
    mqp::piv3d_bind_scratch(a, pb.alg, chunk, (char*)ctx->scratch3d.ptr);
  }
  a.img1 = d1;
  a.img2 = d2;
  a.mask = dmask;
  a.mask_skip = dskip;
  a.dtype = dtype;
  a.pred = dpred;
  a.VF = dVF;
  a.SN = dSN;
  a.planes = dplanes;
  a.planes_begin = ia_begin;
  a.H = H;
  a.W = W;
  a.D = D;
  for (int d = 0; d < 3; ++d) {
    a.IS[d] = pb.IS[d];
    a.SM[d] = pb.SM[d];
    a.st[d] = pb.st[d];
    a.vf[d] = (int)pb.vf[d];
  }
  a.ia_begin = ia_begin;
  a.ia_end = ia_end;
  a.threshold = p->threshold;
  a.mask_threshold = p->mask_threshold;
  std::string err;
  {
    ProfileScope ps(ctx, s, 1, ia_end - ia_begin);
    e = mqp::launch_piv3d(a, pb.alg, chunk, s, err);
  }
  if (e != cudaSuccess) return fail(ctx, e == cudaErrorInvalidValue ? MQP_ERR_UNSUPPORTED : MQP_ERR_CUDA, err);
  return MQP_OK;
}

// Multi-pass refinement (mqp_params.refine): passes at scales 2^(m-1), ..., 1,
// each after the first searching around the whole-pixel predictor taken from
// the previous pass (mqp_multipass.cuh).  SN and the debug planes come from
// the final pass only, as the reference's compute_SN runs at scale 1.
int run_multipass(mqp_ctx* ctx, const mqp_params* p, const void* d1, const void* d2, const void* dmask,
                  const void* dskip, int dtype, int ndims, const int64_t dims[3], double* dVF, double* dSN,
                  cudaStream_t s, double* dplanes, int64_t ia_begin, int64_t ia_end) {
  const bool masked = dmask != nullptr;
  Problem prev;
  const double* prevVF = nullptr;
  cudaError_t e;
  for (int level = p->multipass - 1; level >= 0; --level) {
    if (level > 20) return fail(ctx, MQP_ERR_INVALID, "multipass too large");
    Problem pb;
    int rc = resolve(ctx, p, ndims, dims, masked, 1 << level, pb);
    if (rc != MQP_OK) return rc;
    double* outVF = dVF;
    double* outSN = nullptr;
    if (level == 0) {
      outSN = dSN;
    } else {
      DevBuf& b = ctx->passVF[level & 1];
      if ((e = b.ensure((size_t)(pb.n_ia > 0 ? pb.n_ia : 1) * ndims * sizeof(double))) != cudaSuccess)
        return cuda_fail(ctx, e, "multi-pass vector buffer");
      outVF = (double*)b.ptr;
    }
    const int32_t* dpred = nullptr;
    const bool deform = p->refine == 2 && prevVF && pb.n_ia > 0 && prev.n_ia > 0;
    const void* in1 = d1;
    const void* in2 = d2;
    mqp::DeformArgs da;
    if (deform) {
      // the images resampled around the dense predictor of the previous pass
      // (mqp_deform.cuh); this pass measures the residual
      memset(&da, 0, sizeof(da));
      da.nd = ndims;
      da.dtype = dtype;
      for (int d = 0; d < 3; ++d) da.dims[d] = d < ndims ? dims[d] : 1;
      const size_t img_b = (size_t)(da.dims[0] * da.dims[1] * da.dims[2]) * elem_size(dtype);
      if ((e = ctx->def1.ensure(img_b)) != cudaSuccess || (e = ctx->def2.ensure(img_b)) != cudaSuccess)
        return cuda_fail(ctx, e, "deformed image buffers");
      da.img1 = d1;
      da.img2 = d2;
      da.out1 = ctx->def1.ptr;
      da.out2 = ctx->def2.ptr;
      da.VFc = prevVF;
      for (int d = 0; d < ndims; ++d) {
        da.vf_c[d] = (int)prev.vf[d];
        da.isz_c[d] = prev.IS[d];
        da.st_c[d] = prev.st[d];
        da.vf_f[d] = (int)pb.vf[d];
        da.isz_f[d] = pb.IS[d];
        da.st_f[d] = pb.st[d];
      }
      da.threshold = p->threshold;
      {
        ProfileScope ps(ctx, s, 2, 0);
        if ((e = mqp::launch_deform(da, s)) != cudaSuccess) return cuda_fail(ctx, e, "deform kernel");
      }
      in1 = da.out1;
      in2 = da.out2;
    }
    if (prevVF && pb.n_ia > 0 && !deform && p->refine != 2) {
      if ((e = ctx->pred.ensure((size_t)pb.n_ia * ndims * sizeof(int32_t))) != cudaSuccess)
        return cuda_fail(ctx, e, "predictor buffer");
      mqp::PredArgs pa;
      memset(&pa, 0, sizeof(pa));
      pa.ndims = ndims;
      for (int d = 0; d < ndims; ++d) {
        pa.vf_f[d] = (int)pb.vf[d];
        pa.vf_c[d] = (int)prev.vf[d];
        pa.isz_f[d] = pb.IS[d];
        pa.st_f[d] = pb.st[d];
        pa.isz_c[d] = prev.IS[d];
        pa.st_c[d] = prev.st[d];
      }
      pa.VFc = prevVF;
      pa.pred = (int32_t*)ctx->pred.ptr;
      {
        ProfileScope ps(ctx, s, 2, 0);
        if ((e = mqp::launch_predictor(pa, s)) != cudaSuccess) return cuda_fail(ctx, e, "predictor kernel");
      }
      dpred = pa.pred;
    }
    if (pb.n_ia > 0) {
      const int64_t b0 = level == 0 ? ia_begin : 0, b1 = level == 0 ? ia_end : pb.n_ia;
      double* pl = level == 0 ? dplanes : nullptr;
      rc = ndims == 3 ? run_pass_3d(ctx, pb, p, in1, in2, dmask, dskip, dtype, outVF, outSN, dpred, pl, b0, b1, s)
                      : run_pass_2d(ctx, pb, p, in1, in2, dmask, dskip, dtype, outVF, outSN, dpred, pl, b0, b1, s);
      if (rc != MQP_OK) return rc;
      if (deform) {
        da.VF = outVF;
        ProfileScope ps(ctx, s, 2, 0);
        if ((e = mqp::launch_deform_add(da, s)) != cudaSuccess) return cuda_fail(ctx, e, "deform add kernel");
      }
    }
    prev = pb;
    prevVF = outVF;
  }
  return MQP_OK;
}

int piv_device_impl(mqp_ctx* ctx, const void* d1, const void* d2, const void* dmask, const void* dmask_skip,
                    int dtype, int ndims, const int64_t dims[3], const mqp_params* p, double* dVF,
                    double* dSN, cudaStream_t s, double* dplanes, int64_t ia_begin, int64_t ia_end) {
  NvtxRange nv("mqp_piv_device");
  if (dtype != MQP_F32 && dtype != MQP_F64) return fail(ctx, MQP_ERR_INVALID, "dtype must be MQP_F32 or MQP_F64");
  if (!d1 || !d2) return fail(ctx, MQP_ERR_INVALID, "null image pointer");
  const bool masked = dmask != nullptr;
  Problem pb;
  int rc = resolve(ctx, p, ndims, dims, masked, 1, pb);
  if (rc != MQP_OK) return rc;
  if (pb.n_ia == 0) return MQP_OK;  // empty vector field: nothing to write (an empty VF may have no address)
  if (!dVF) return fail(ctx, MQP_ERR_INVALID, "null VF pointer");
  if (ia_end < 0) ia_end = pb.n_ia;
  if (ia_begin < 0 || ia_begin > ia_end || ia_end > pb.n_ia) return fail(ctx, MQP_ERR_INVALID, "IA range outside the vector field");
  if (!p->computeSN) dSN = nullptr;
  if (p->refine && p->multipass > 1)
    return run_multipass(ctx, p, d1, d2, dmask, dmask_skip, dtype, ndims, dims, dVF, dSN, s, dplanes, ia_begin,
                         ia_end);
  // multipass without refinement re-runs the scale-1 geometry with identical
  // results (src/multi_quickPIV.jl:57, Q6): one pass gives the same VF/SN
  if (ndims == 3)
    return run_pass_3d(ctx, pb, p, d1, d2, dmask, dmask_skip, dtype, dVF, dSN, nullptr, dplanes, ia_begin, ia_end, s);
  return run_pass_2d(ctx, pb, p, d1, d2, dmask, dmask_skip, dtype, dVF, dSN, nullptr, dplanes, ia_begin, ia_end, s);
}

}  // namespace mqp_host

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

// One 2D pass from host arrays, pipelined: the images (and masks) go up in
// pieces of whole columns on a copy-in stream (column-major: a piece is one
// contiguous range, the pieces growing geometrically); the compute stream
// waits for each piece, builds its
// integral columns and runs the IA columns whose windows lie within the
// columns received so far; their vectors go down on a copy-out stream while
// later pieces compute.  Every IA and every integral value is computed as in
// the one-shot path, so the results are identical.
static int host_pipelined_2d(mqp_ctx* ctx, const Problem& pb, const mqp_params* p, const void* img1,
                             const void* img2, const void* mask, const void* mask_skip, int dtype, double* VF,
                             double* SN) {
  const int H = (int)pb.dims[0], W = (int)pb.dims[1];
  const int64_t vf1 = pb.vf[0], vf2 = pb.vf[1];
  const size_t es = elem_size(dtype), colb = (size_t)H * es;
  const int PIPE_PIECES = ctx->host_pieces;
  cudaError_t e;
  if (!ctx->in_stream && (e = cudaStreamCreateWithFlags(&ctx->in_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy stream");
  if (!ctx->out_stream && (e = cudaStreamCreateWithFlags(&ctx->out_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy stream");
  while (ctx->pipe_ev.size() < 2 * PIPE_PIECES + 1) {
    cudaEvent_t ev;
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return cuda_fail(ctx, e, "event");
    ctx->pipe_ev.push_back(ev);
  }
  const size_t ib = colb * (size_t)W;
  for (DevBuf* b : {&ctx->img1, &ctx->img2})
    if ((e = b->ensure(ib)) != cudaSuccess) return cuda_fail(ctx, e, "image buffer");
  if (mask && (e = ctx->mask.ensure(ib)) != cudaSuccess) return cuda_fail(ctx, e, "mask buffer");
  if (mask_skip && (e = ctx->mask_skip.ensure(ib)) != cudaSuccess) return cuda_fail(ctx, e, "mask buffer");
  const size_t nvf = (size_t)pb.n_ia;
  if ((e = ctx->VF.ensure(nvf * 2 * sizeof(double))) != cudaSuccess) return cuda_fail(ctx, e, "VF buffer");
  double* dSN = nullptr;
  if (SN) {
    if ((e = ctx->SN.ensure(nvf * sizeof(double))) != cudaSuccess) return cuda_fail(ctx, e, "SN buffer");
    dSN = (double*)ctx->SN.ptr;
  }
  double* dVF = (double*)ctx->VF.ptr;
  cudaStream_t s = ctx->stream, si = ctx->in_stream, so = ctx->out_stream;
  // the compute stream's earlier work (another call's kernels reading the
  // buffers) precedes this call's copies
  if ((e = cudaEventRecord(ctx->pipe_ev[2 * PIPE_PIECES], s)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(si, ctx->pipe_ev[2 * PIPE_PIECES], 0)) != cudaSuccess)
    return cuda_fail(ctx, e, "pipeline order");
  // IA column v2 reads image columns below need(v2) (IA window, search window
  // data, and the integral columns of its lag windows)
  mqp::Piv2dArgs g0 = args_2d(ctx, pb, p, nullptr, nullptr, nullptr, nullptr, dtype, nullptr, nullptr, nullptr,
                              nullptr, 0, 0);
  auto need = [&](int64_t v2) {
    const mqp::IAGeom g = mqp::ia_geom(g0, 0, (int)v2);
    return std::max(g.ir2 + pb.IS[1], g.g02 + g.hi2);
  };
  int64_t done_cols = 0;  // IA columns launched
  struct Out {
    int k;
    size_t a0, n;  // IAs [a0, a0 + n) finished by piece k
  };
  std::vector<Out> outs;
  int x0 = 0;
  for (int k = 0; k < PIPE_PIECES; ++k) {
    // geometric pieces (each twice the last): a small first piece starts
    // the kernels early, and the later copies hide behind the compute
    const int64_t den = ((int64_t)1 << PIPE_PIECES) - 1, num = ((int64_t)1 << (k + 1)) - 1;
    int x1 = k == PIPE_PIECES - 1 ? W : (int)(((int64_t)W * num / den + 63) / 64 * 64);
    if (x1 > W) x1 = W;
    if (x1 <= x0) continue;
    const size_t off = colb * (size_t)x0, len = colb * (size_t)(x1 - x0);
    const void* src[4] = {img1, img2, mask, mask_skip};
    DevBuf* dst[4] = {&ctx->img1, &ctx->img2, &ctx->mask, &ctx->mask_skip};
    for (int i = 0; i < 4; ++i)
      if (src[i] && (e = cudaMemcpyAsync((char*)dst[i]->ptr + off, (const char*)src[i] + off, len,
                                         cudaMemcpyHostToDevice, si)) != cudaSuccess)
        return cuda_fail(ctx, e, "copy images");
    if ((e = cudaEventRecord(ctx->pipe_ev[k], si)) != cudaSuccess || (e = cudaStreamWaitEvent(s, ctx->pipe_ev[k], 0)) != cudaSuccess)
      return cuda_fail(ctx, e, "pipeline order");
    int rc = integrals_2d(ctx, pb, ctx->img1.ptr, ctx->img2.ptr, dtype, s, x0, x1);
    if (rc != MQP_OK) return rc;
    int64_t c1 = done_cols;
    while (c1 < vf2 && (x1 == W || need(c1) <= x1)) ++c1;
    if (c1 > done_cols) {
      rc = launch_2d(ctx, args_2d(ctx, pb, p, ctx->img1.ptr, ctx->img2.ptr, mask ? ctx->mask.ptr : nullptr,
                                  mask_skip ? ctx->mask_skip.ptr : nullptr, dtype, dVF, dSN, nullptr, nullptr,
                                  vf1 * done_cols, vf1 * c1),
                     pb.alg, s);
      if (rc != MQP_OK) return rc;
      if ((e = cudaEventRecord(ctx->pipe_ev[PIPE_PIECES + k], s)) != cudaSuccess) return cuda_fail(ctx, e, "pipeline order");
      outs.push_back({k, (size_t)(vf1 * done_cols), (size_t)(vf1 * (c1 - done_cols))});
      done_cols = c1;
    }
    x0 = x1;
  }
  // downloads after every upload is enqueued: a copy into pageable memory
  // returns only when done, and would hold back the next piece's upload
  for (const auto& o : outs) {
    if ((e = cudaStreamWaitEvent(so, ctx->pipe_ev[PIPE_PIECES + o.k], 0)) != cudaSuccess)
      return cuda_fail(ctx, e, "pipeline order");
    if (VF && (e = cudaMemcpyAsync(VF + 2 * o.a0, dVF + 2 * o.a0, 2 * o.n * sizeof(double), cudaMemcpyDeviceToHost, so)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy VF");
    if (SN && (e = cudaMemcpyAsync(SN + o.a0, dSN + o.a0, o.n * sizeof(double), cudaMemcpyDeviceToHost, so)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy SN");
  }
  if ((e = cudaStreamSynchronize(so)) != cudaSuccess) return cuda_fail(ctx, e, "PIV kernels");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "PIV kernels");
  return MQP_OK;
}

// The 3D FFTCC pass (no integral volumes) pipelined the same way over z: the
// volumes go up in geometrically growing pieces of whole z-planes (each one
// contiguous range); the IA layers (vector-field z indices) whose windows the
// received planes cover run while later planes copy.
static int host_pipelined_3d(mqp_ctx* ctx, const Problem& pb, const mqp_params* p, const void* img1,
                             const void* img2, int dtype, double* VF, double* SN) {
  const int H = (int)pb.dims[0], W = (int)pb.dims[1], D = (int)pb.dims[2];
  const int64_t layer = pb.vf[0] * pb.vf[1], vf3 = pb.vf[2];
  const size_t planeb = (size_t)H * (size_t)W * elem_size(dtype);
  const int PIECES = ctx->host_pieces;
  cudaError_t e;
  if (!ctx->in_stream && (e = cudaStreamCreateWithFlags(&ctx->in_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy stream");
  if (!ctx->out_stream && (e = cudaStreamCreateWithFlags(&ctx->out_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, e, "copy stream");
  while (ctx->pipe_ev.size() < 2 * (size_t)PIECES + 1) {
    cudaEvent_t ev;
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return cuda_fail(ctx, e, "event");
    ctx->pipe_ev.push_back(ev);
  }
  const size_t ib = planeb * (size_t)D;
  for (DevBuf* b : {&ctx->img1, &ctx->img2})
    if ((e = b->ensure(ib)) != cudaSuccess) return cuda_fail(ctx, e, "image buffer");
  const size_t nvf = (size_t)pb.n_ia;
  if ((e = ctx->VF.ensure(nvf * 3 * sizeof(double))) != cudaSuccess) return cuda_fail(ctx, e, "VF buffer");
  double* dSN = nullptr;
  if (SN) {
    if ((e = ctx->SN.ensure(nvf * sizeof(double))) != cudaSuccess) return cuda_fail(ctx, e, "SN buffer");
    dSN = (double*)ctx->SN.ptr;
  }
  double* dVF = (double*)ctx->VF.ptr;
  cudaStream_t s = ctx->stream, si = ctx->in_stream, so = ctx->out_stream;
  if ((e = cudaEventRecord(ctx->pipe_ev[2 * PIECES], s)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(si, ctx->pipe_ev[2 * PIECES], 0)) != cudaSuccess)
    return cuda_fail(ctx, e, "pipeline order");
  mqp::Piv3dArgs g0;
  memset(&g0, 0, sizeof(g0));
  g0.H = H;
  g0.W = W;
  g0.D = D;
  for (int d = 0; d < 3; ++d) {
    g0.IS[d] = pb.IS[d];
    g0.SM[d] = pb.SM[d];
    g0.st[d] = pb.st[d];
    g0.vf[d] = (int)pb.vf[d];
  }
  auto need = [&](int64_t v3) {  // z-planes below this cover IA layer v3
    const mqp::IAGeom3 g = mqp::ia_geom3(g0, layer * v3);
    return std::max(g.ir[2] + pb.IS[2], g.g0[2] + g.hi[2]);
  };
  struct Out {
    int k;
    size_t a0, n;
  };
  std::vector<Out> outs;
  int64_t done = 0;  // IA layers launched
  int z0 = 0;
  for (int k = 0; k < PIECES; ++k) {
    const int64_t den = ((int64_t)1 << PIECES) - 1, num = ((int64_t)1 << (k + 1)) - 1;
    int z1 = k == PIECES - 1 ? D : (int)((int64_t)D * num / den);
    if (z1 > D) z1 = D;
    if (z1 <= z0) continue;
    const size_t off = planeb * (size_t)z0, len = planeb * (size_t)(z1 - z0);
    if ((e = cudaMemcpyAsync((char*)ctx->img1.ptr + off, (const char*)img1 + off, len, cudaMemcpyHostToDevice, si)) != cudaSuccess ||
        (e = cudaMemcpyAsync((char*)ctx->img2.ptr + off, (const char*)img2 + off, len, cudaMemcpyHostToDevice, si)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy volumes");
    if ((e = cudaEventRecord(ctx->pipe_ev[k], si)) != cudaSuccess || (e = cudaStreamWaitEvent(s, ctx->pipe_ev[k], 0)) != cudaSuccess)
      return cuda_fail(ctx, e, "pipeline order");
    int64_t v1 = done;
    while (v1 < vf3 && (z1 == D || need(v1) <= z1)) ++v1;
    if (v1 > done) {
      const int rc = run_pass_3d(ctx, pb, p, ctx->img1.ptr, ctx->img2.ptr, nullptr, nullptr, dtype, dVF, dSN, nullptr,
                                 nullptr, layer * done, layer * v1, s);
      if (rc != MQP_OK) return rc;
      if ((e = cudaEventRecord(ctx->pipe_ev[PIECES + k], s)) != cudaSuccess) return cuda_fail(ctx, e, "pipeline order");
      outs.push_back({k, (size_t)(layer * done), (size_t)(layer * (v1 - done))});
      done = v1;
    }
    z0 = z1;
  }
  for (const auto& o : outs) {
    if ((e = cudaStreamWaitEvent(so, ctx->pipe_ev[PIECES + o.k], 0)) != cudaSuccess)
      return cuda_fail(ctx, e, "pipeline order");
    if (VF && (e = cudaMemcpyAsync(VF + 3 * o.a0, dVF + 3 * o.a0, 3 * o.n * sizeof(double), cudaMemcpyDeviceToHost, so)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy VF");
    if (SN && (e = cudaMemcpyAsync(SN + o.a0, dSN + o.a0, o.n * sizeof(double), cudaMemcpyDeviceToHost, so)) != cudaSuccess)
      return cuda_fail(ctx, e, "copy SN");
  }
  if ((e = cudaStreamSynchronize(so)) != cudaSuccess) return cuda_fail(ctx, e, "PIV kernels");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "PIV kernels");
  return MQP_OK;
}

static int host_roundtrip(mqp_ctx* ctx, const void* img1, const void* img2, const void* mask,
                          const void* mask_skip, int dtype, int ndims, const int64_t dims[3],
                          const mqp_params* p, double* VF, double* SN, int64_t vf_dims_out[3],
                          double* planes, int64_t ia_begin, int64_t ia_end) {
  NvtxRange nv("mqp_piv");
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
  // one 2D pass into host arrays: pipelined copies (wide images only)
  if (ndims == 2 && !planes && !(p->refine && p->multipass > 1) && pb.n_ia > 0 && pb.dims[1] >= 1024 &&
      ctx->host_pieces > 1 &&
      mqp::piv2d_fft_len(pb.IS[0] + 2 * pb.SM[0], pb.IS[1] + 2 * pb.SM[1]) != 0)
    return host_pipelined_2d(ctx, pb, p, img1, img2, mask, mask_skip, dtype, VF, SN);
  if (ndims == 3 && !planes && !(p->refine && p->multipass > 1) && pb.n_ia > 0 && pb.alg == mqp::ALG_FFTCC &&
      !mask && pb.dims[2] >= 64 && ctx->host_pieces > 1)
    return host_pipelined_3d(ctx, pb, p, img1, img2, dtype, VF, SN);
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

}  // extern "C"

namespace {

// Validates a post-processing request and fills the kernel arguments.
int post_resolve(mqp_ctx* ctx, const mqp_post_params* p, const mqp_field* f, mqp::PostArgs& a) {
  if (!p || !f) return fail(ctx, MQP_ERR_INVALID, "null parameters or field");
  if (f->ndims < 1 || f->ndims > 4) return fail(ctx, MQP_ERR_INVALID, "field ndims must be 1..4");
  if (f->ncomp < 1 || f->ncomp > 4) return fail(ctx, MQP_ERR_INVALID, "field ncomp must be 1..4");
  memset(&a, 0, sizeof(a));
  a.op = p->op;
  a.ncomp = f->ncomp;
  a.nd = f->ndims;
  a.n = 1;
  for (int d = 0; d < 4; ++d) {
    const int64_t n = d < f->ndims ? f->dims[d] : 1;
    if (n < 0 || n > (1 << 30)) return fail(ctx, MQP_ERR_INVALID, "field extents must be in [0, 2^30]");
    a.dims[d] = (int)n;
    a.radius[d] = d < f->ndims ? p->radius[d] : 0;
    if (a.radius[d] < 0) return fail(ctx, MQP_ERR_INVALID, "radius must be >= 0");
    a.n *= n;
  }
  switch (p->op) {
    case MQP_POST_MAGNITUDES:
    case MQP_POST_AVERAGE:
      break;
    case MQP_POST_SIMILARITY_AVG:
      a.p0 = cospi(p->max_angle / 180.0);  // cosd
      a.i0 = p->normalize != 0;
      a.i1 = p->scale_by_similarity != 0;
      a.p1 = p->similarity_exponent;
      break;
    case MQP_POST_COLLECTIVENESS:
      a.p0 = cospi(p->max_angle / 180.0);
      break;
    case MQP_POST_TH_MASK:
      if (f->ncomp != 1) return fail(ctx, MQP_ERR_INVALID, "TH masking takes a scalar map (ncomp = 1)");
      a.p0 = p->threshold;
      a.i0 = p->cmp != 0;
      break;
    case MQP_POST_STD_MASK:
      if (f->ncomp != 1) return fail(ctx, MQP_ERR_INVALID, "STD masking takes a scalar map (ncomp = 1)");
      if (a.n == 1) return fail(ctx, MQP_ERR_INVALID, "STD masking needs at least two values (or none)");
      a.p0 = p->threshold;
      break;
    case MQP_POST_REPLACE:
      if (p->replace < MQP_REPLACE_ZERO || p->replace > MQP_REPLACE_MEAN)
        return fail(ctx, MQP_ERR_INVALID, "replace must be MQP_REPLACE_ZERO, _MEDIAN or _MEAN");
      a.i0 = p->replace;
      break;
    case MQP_POST_LOCAL_MAGNITUDE:
      a.p0 = p->threshold;
      break;
    case MQP_POST_MATLAB_DIVERGENCE:
      if (f->ncomp != f->ndims) return fail(ctx, MQP_ERR_INVALID, "matlab_divergence needs ncomp == ndims");
      break;
    case MQP_POST_DIVERGENCE:
      if (f->ncomp != f->ndims) return fail(ctx, MQP_ERR_INVALID, "divergence needs ncomp == ndims");
      a.i0 = p->normalize != 0;
      a.p1 = p->min_speed;
      a.i1 = p->divide_by;
      a.i2 = p->circle != 0;
      if (a.i1 < MQP_DIVIDE_NONE || a.i1 > MQP_DIVIDE_MAGS) return fail(ctx, MQP_ERR_INVALID, "bad divide_by");
      break;
    default:
      return fail(ctx, MQP_ERR_INVALID, "unknown post-processing op " + std::to_string(p->op));
  }
  return MQP_OK;
}

// which buffers an op reads/writes: in (ncomp-vector or scalar), mask, out
// (Float64, vector or scalar), outf (Float32 scalar), mask_out
struct PostIO {
  bool mask, out_vec, out_scalar, outf, mask_out;
};
PostIO post_io(int op) {
  switch (op) {
    case MQP_POST_MAGNITUDES: return {false, false, true, false, false};
    case MQP_POST_AVERAGE:
    case MQP_POST_SIMILARITY_AVG: return {false, true, false, false, false};
    case MQP_POST_COLLECTIVENESS:
    case MQP_POST_MATLAB_DIVERGENCE: return {false, false, false, true, false};
    case MQP_POST_TH_MASK:
    case MQP_POST_STD_MASK: return {false, false, false, false, true};
    case MQP_POST_REPLACE: return {true, true, false, false, false};
    case MQP_POST_LOCAL_MAGNITUDE: return {false, true, false, false, true};
    case MQP_POST_DIVERGENCE: return {false, false, true, false, false};
    default: return {false, false, false, false, false};
  }
}

int post_run(mqp_ctx* ctx, mqp::PostArgs& a, const double* d_in, const uint8_t* d_mask, double* d_out,
             float* d_outf, uint8_t* d_mask_out, cudaStream_t s) {
  const PostIO io = post_io(a.op);
  if (a.n == 0) return MQP_OK;  // empty field: nothing to compute (its arrays may have no address)
  if (!d_in) return fail(ctx, MQP_ERR_INVALID, "null input field");
  if ((io.mask && !d_mask) || ((io.out_vec || io.out_scalar) && !d_out) || (io.outf && !d_outf) ||
      (io.mask_out && !d_mask_out))
    return fail(ctx, MQP_ERR_INVALID, "a buffer this op needs is null");
  a.VF = d_in;
  a.mask = d_mask;
  a.out = d_out;
  a.outf = d_outf;
  a.mask_out = d_mask_out;
  cudaError_t e;
  if (a.op == MQP_POST_STD_MASK) {
    if ((e = ctx->post_scratch.ensure(mqp::post_scratch_bytes())) != cudaSuccess) return cuda_fail(ctx, e, "scratch");
  }
  ProfileScope ps(ctx, s, 2, 0);
  if ((e = mqp::launch_post(a, (double*)ctx->post_scratch.ptr, s)) != cudaSuccess) return cuda_fail(ctx, e, "post-processing kernel");
  return MQP_OK;
}

}  // namespace

extern "C" {

int mqp_postprocess_device(mqp_ctx* ctx, const mqp_post_params* p, const mqp_field* f, const double* d_in,
                           const uint8_t* d_mask, double* d_out, float* d_outf, uint8_t* d_mask_out, void* stream) {
  NvtxRange nv("mqp_postprocess_device");
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  mqp::PostArgs a;
  int rc = post_resolve(ctx, p, f, a);
  if (rc != MQP_OK) return rc;
  return post_run(ctx, a, d_in, d_mask, d_out, d_outf, d_mask_out, stream ? (cudaStream_t)stream : cudaStreamLegacy);
}

int mqp_postprocess(mqp_ctx* ctx, const mqp_post_params* p, const mqp_field* f, const double* in, const uint8_t* mask,
                    double* out, float* outf, uint8_t* mask_out) {
  NvtxRange nv("mqp_postprocess");
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  mqp::PostArgs a;
  int rc = post_resolve(ctx, p, f, a);
  if (rc != MQP_OK) return rc;
  if (a.n == 0) return MQP_OK;  // empty field
  if (!in) return fail(ctx, MQP_ERR_INVALID, "null input field");
  const PostIO io = post_io(a.op);
  const bool vec_in = !(a.op == MQP_POST_TH_MASK || a.op == MQP_POST_STD_MASK);
  const size_t n = (size_t)a.n, nb = n ? n : 1;
  const size_t in_b = nb * (vec_in ? a.ncomp : 1) * sizeof(double);
  const size_t out_b = nb * (io.out_vec ? a.ncomp : 1) * sizeof(double);
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  if ((e = ctx->post_in.ensure(in_b)) != cudaSuccess) return cuda_fail(ctx, e, "post-processing buffer");
  if ((e = cudaMemcpyAsync(ctx->post_in.ptr, in, in_b, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy in");
  uint8_t* dm = nullptr;
  if (io.mask) {
    if (!mask) return fail(ctx, MQP_ERR_INVALID, "this op needs a mask");
    if ((e = ctx->post_mask.ensure(nb)) != cudaSuccess) return cuda_fail(ctx, e, "post-processing buffer");
    if ((e = cudaMemcpyAsync(ctx->post_mask.ptr, mask, nb, cudaMemcpyHostToDevice, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy mask");
    dm = (uint8_t*)ctx->post_mask.ptr;
  }
  double* dout = nullptr;
  float* doutf = nullptr;
  uint8_t* dmo = nullptr;
  if (io.out_vec || io.out_scalar) {
    if (!out) return fail(ctx, MQP_ERR_INVALID, "this op needs `out`");
    if ((e = ctx->post_out.ensure(out_b)) != cudaSuccess) return cuda_fail(ctx, e, "post-processing buffer");
    dout = (double*)ctx->post_out.ptr;
  }
  if (io.outf) {
    if (!outf) return fail(ctx, MQP_ERR_INVALID, "this op needs `outf`");
    if ((e = ctx->post_outf.ensure(nb * sizeof(float))) != cudaSuccess) return cuda_fail(ctx, e, "post-processing buffer");
    doutf = (float*)ctx->post_outf.ptr;
  }
  if (io.mask_out) {
    if (!mask_out) return fail(ctx, MQP_ERR_INVALID, "this op needs `mask_out`");
    if ((e = ctx->post_mask_out.ensure(nb)) != cudaSuccess) return cuda_fail(ctx, e, "post-processing buffer");
    dmo = (uint8_t*)ctx->post_mask_out.ptr;
  }
  rc = post_run(ctx, a, (const double*)ctx->post_in.ptr, dm, dout, doutf, dmo, s);
  if (rc != MQP_OK) {
    cudaStreamSynchronize(s);
    return rc;
  }
  if (n && dout && (e = cudaMemcpyAsync(out, dout, out_b, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy out");
  if (n && doutf && (e = cudaMemcpyAsync(outf, doutf, n * sizeof(float), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy out");
  if (n && dmo && (e = cudaMemcpyAsync(mask_out, dmo, n, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return cuda_fail(ctx, e, "copy out");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(ctx, e, "post-processing");
  return MQP_OK;
}

int mqp_set_tuning(mqp_ctx* ctx, int key, int64_t value) {
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (value < 0) return fail(ctx, MQP_ERR_INVALID, "tuning values must be >= 0");
  switch (key) {
    case MQP_TUNE_CHUNK3D: ctx->chunk3d = value; return MQP_OK;
    case MQP_TUNE_CHUNK3D_BUDGET: ctx->chunk3d_budget = value > 0 ? (size_t)value : ((size_t)1 << 30); return MQP_OK;
    case MQP_TUNE_HOST_PIECES:
      if (value < 1 || value > 16) return fail(ctx, MQP_ERR_INVALID, "host pieces must be in [1, 16]");
      ctx->host_pieces = (int)value;
      return MQP_OK;
    default: return fail(ctx, MQP_ERR_INVALID, "unknown tuning key " + std::to_string(key));
  }
}

int mqp_correlation_planes(mqp_ctx* ctx, const void* img1, const void* img2, const void* mask,
                           int dtype, int ndims, const int64_t dims[3], const mqp_params* p,
                           int64_t ia_begin, int64_t ia_end, double* planes) {
  if (!planes) return fail(ctx, MQP_ERR_INVALID, "null planes buffer");
  return host_roundtrip(ctx, img1, img2, mask, nullptr, dtype, ndims, dims, p, nullptr, nullptr, nullptr,
                        planes, ia_begin, ia_end);
}

}  // extern "C"
