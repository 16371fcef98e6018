// Private host-side state of the C ABI: the context (mqp_ctx), its grow-only
// device buffers, kernel timing spans and parameter resolution shared by
// the single-pair (mqp_abi.cu) and batched (mqp_batch.cu) entry points.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <string>
#include <vector>

#include "mqp.h"
#include "mqp_internal.h"

namespace mqp_host {

inline thread_local std::string g_create_error;

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

}  // namespace mqp_host

struct mqp_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  std::mutex mu;
  mqp_host::DevBuf img1, img2, mask, mask_skip, II1, IIg, IIg2, VF, SN, pred, planes, status, iscratch, scratch3d;
  mqp_host::DevBuf passVF[2];  // vectors of the coarse passes of a multi-pass refinement
  mqp_host::DevBuf def1, def2;  // deformed images of the deforming refinement
  mqp_host::DevBuf huge;        // scratch slots of the 2D kernel for search windows above 128
  mqp_host::DevBuf post_in, post_mask, post_out, post_outf, post_mask_out, post_scratch;
  mqp_host::DevBuf traj_in, traj_out;  // host-array pseudo-trajectories
  // host-array 2D path: copy-in and copy-out streams, events of its pieces
  cudaStream_t in_stream = nullptr, out_stream = nullptr;
  std::vector<cudaEvent_t> pipe_ev;
  int host_pieces = 3;
  // 3D path: IAs per chunk (0 = sized from chunk3d_budget bytes of scratch)
  int64_t chunk3d = 0;
  size_t chunk3d_budget = (size_t)1 << 30;
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

namespace mqp_host {

// An NVTX range over an entry point's host work (what it enqueues), named
// after the entry point, for Nsight Systems timelines and ncu NVTX filters;
// without a tool attached the push and pop do nothing.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

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

inline int fail(mqp_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  else g_create_error = msg;
  return code;
}

inline int cuda_fail(mqp_ctx* ctx, cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? MQP_ERR_OOM : MQP_ERR_CUDA;
  return fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

// get_vectorfield_size (src/utils/piv_ops.jl:11-14)
inline int64_t vf_len(int64_t size, int IS, int st) {
  const int64_t stop = size - IS + 1;
  return stop < 1 ? 0 : (stop - 1) / st + 1;
}

inline int resolve(mqp_ctx* ctx, const mqp_params* p, int ndims, const int64_t dims[3], bool masked,
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
  if (p->refine < 0 || p->refine > 2) return fail(ctx, MQP_ERR_INVALID, "refine must be 0, 1 or 2");
  if (p->refine == 2 && masked && p->multipass > 1)
    return fail(ctx, MQP_ERR_UNSUPPORTED, "window deformation (refine = 2) does not take masks");
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

// Passes on device arrays (mqp_abi.cu): enqueue one PIV pass of a resolved
// problem on stream s, optionally with a whole-pixel predictor and debug planes.
size_t elem_size(int dtype);
size_t align256(size_t n);
int run_pass_2d(mqp_ctx* ctx, const Problem& pb, const mqp_params* p, const void* d1, const void* d2,
                const void* dmask, const void* dskip, int dtype, double* dVF, double* dSN,
                const int32_t* dpred, double* dplanes, int64_t ia_begin, int64_t ia_end, cudaStream_t s);
int run_pass_3d(mqp_ctx* ctx, const Problem& pb, const mqp_params* p, const void* d1, const void* d2,
                const void* dmask, const void* dskip, int dtype, double* dVF, double* dSN,
                const int32_t* dpred, double* dplanes, int64_t ia_begin, int64_t ia_end, cudaStream_t s);

}  // namespace mqp_host
