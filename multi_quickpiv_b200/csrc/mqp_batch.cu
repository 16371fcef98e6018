// Batched PIV plans (include/mqp.h, mqp_batch_plan_*): many image pairs of
// mixed size, dimensionality, algorithm and pass count computed by a fixed,
// pre-allocated schedule that is captured once into a CUDA graph.
//
// A plan owns all scratch (one arena allocated at creation), so running it
// allocates nothing and synchronises nothing on the host.  The schedule:
//
//   main stream   integral images of the 2D pairs, then per pass round the
//                 multi-pass predictors and ONE persistent launch of the
//                 fused 2D kernel per kernel variant (N, prune, algorithm,
//                 dtype), whose warps take IAs of all pairs of that variant
//                 from a single work queue (large and small pairs balance)
//   3D lanes      up to four side streams; each 3D pair runs all its steps
//                 (integral volumes, predictors, passes) on one lane, with
//                 its own chunk scratch, concurrently with the 2D work and
//                 the other lanes.  Pairs go to lanes longest first by an
//                 estimate of their arithmetic (a coarse pass of a few IAs
//                 cannot fill the GPU alone; lanes let such passes of
//                 different pairs run side by side).
//
// Pass rounds: pair k with L_k passes (refine && multipass > 1, else 1) runs
// its pass at scale 2^(L_k-1-r) in round r, so every pair's coarse pass comes
// first and its predictor is ready before its next round.  Results equal
// mqp_piv_device's for each pair alone.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "mqp.h"
#include "mqp_ctx.h"
#include "mqp_internal.h"

using namespace mqp_host;

struct mqp_plan {
  mqp_ctx* ctx = nullptr;
  int device = 0;
  DevBuf arena;
  // enqueue steps: (main stream, 3D lane streams) -> MQP_OK or an error code
  std::vector<std::function<int(cudaStream_t, const cudaStream_t*)>> ops;
  std::vector<cudaStream_t> lanes;
  std::vector<cudaEvent_t> ev_join;
  // 2D lanes: the kernel variants (groups) of one pass round run side by side
  std::vector<cudaStream_t> lanes2d;
  std::vector<cudaEvent_t> ev_join2d;
  cudaEvent_t ev_fork2d = nullptr;
  cudaStream_t cap = nullptr;
  cudaEvent_t ev_fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t total_ia = 0;
  int64_t launches = 0;
  size_t scratch_bytes = 0;
};

namespace {

// Byte offsets into the arena, resolved to pointers once it is allocated.
struct Arena {
  size_t size = 0;
  size_t take(size_t bytes) {
    const size_t off = size;
    size += align256(bytes ? bytes : 1);
    return off;
  }
};

struct Level {
  Problem pb;
  size_t vf_off = 0;     // this pass's vectors (coarse passes; the final pass writes the caller's VF)
  size_t pred_off = 0;   // this pass's predictor (passes after the first)
  bool has_vf = false, has_pred = false;
};

struct ItemPlan {
  mqp_batch_item it;
  int alg = 0;
  int levels = 1;
  std::vector<Level> lev;   // lev[l] = scale 2^l; the first round runs lev[levels-1]
  size_t ii_off[3] = {0, 0, 0};  // IIg2, IIg, II1
  int n_ii = 0;
  int lane = 0;  // 3D pairs: the side stream all its steps run on
};

constexpr int LANES3D = 4;
constexpr int LANES2D = 4;

// Rough arithmetic of one 3D pass (FLOPs), for balancing pairs over lanes.
double cost3d(const Problem& pb) {
  if (pb.n_ia == 0) return 0.0;
  if (mqp::direct3d_ok(pb.IS, pb.SM)) {
    double nf = 1, np = 1;
    for (int d = 0; d < 3; ++d) {
      nf *= pb.IS[d];
      np *= 2 * pb.SM[d] + 1;
    }
    return 2.0 * nf * np * (double)pb.n_ia;
  }
  const int SS[3] = {pb.IS[0] + 2 * pb.SM[0], pb.IS[1] + 2 * pb.SM[1], pb.IS[2] + 2 * pb.SM[2]};
  const double N = mqp::piv3d_fft_len(SS);
  return 7.5 * N * N * N * std::log2(N * N * N) * (double)pb.n_ia;
}

template <typename T>
T* at(const mqp_plan* p, size_t off) {
  return reinterpret_cast<T*>(static_cast<char*>(p->arena.ptr) + off);
}

int integral_kernels_2d(int W) { return 2 + ((W + 63) / 64 > 1 ? 1 : 0) + ((W + 63) / 64 > 32 ? 1 : 0); }

int64_t chunk_for(const mqp_batch_options& o, size_t per, int64_t n_ia) {
  int64_t chunk = o.chunk3d > 0 ? o.chunk3d
                                : (int64_t)((o.chunk3d_budget > 0 ? (size_t)o.chunk3d_budget : ((size_t)1 << 30)) / per);
  return std::max<int64_t>(1, std::min<int64_t>({chunk, n_ia, 65535}));
}

}  // namespace

extern "C" {

int mqp_batch_plan_create(mqp_ctx* ctx, const mqp_batch_item* items, int32_t n_items, const mqp_batch_options* opt,
                          mqp_plan** out) {
  if (!ctx) return fail(nullptr, MQP_ERR_INVALID, "null context");
  if (!out) return fail(ctx, MQP_ERR_INVALID, "null output pointer");
  *out = nullptr;
  if (n_items < 0 || (n_items > 0 && !items)) return fail(ctx, MQP_ERR_INVALID, "bad item list");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  mqp_batch_options o{};
  o.use_graph = 1;
  o.grab = 2;
  if (opt) o = *opt;
  if (o.grab < 1 || o.grab > 64) return fail(ctx, MQP_ERR_INVALID, "grab must be in [1, 64]");

  Arena ar;
  std::vector<ItemPlan> plan(n_items);
  int rounds = 0;
  size_t isc2d = 0, isc3d = 0, scr3d_per = 0;
  for (int k = 0; k < n_items; ++k) {
    ItemPlan& ip = plan[k];
    ip.it = items[k];
    const mqp_batch_item& it = ip.it;
    const std::string who = "batch item " + std::to_string(k) + ": ";
    if (!it.img1 || !it.img2) return fail(ctx, MQP_ERR_INVALID, who + "null image pointer");
    if (it.dtype != MQP_F32 && it.dtype != MQP_F64) return fail(ctx, MQP_ERR_INVALID, who + "dtype must be MQP_F32 or MQP_F64");
    const bool masked = it.mask != nullptr;
    if (it.params.refine == 2 && it.params.multipass > 1)
      return fail(ctx, MQP_ERR_UNSUPPORTED, who + "batch plans run the whole-pixel refinement (refine = 1), not deformation");
    ip.levels = (it.params.refine && it.params.multipass > 1) ? it.params.multipass : 1;
    if (ip.levels > 16) return fail(ctx, MQP_ERR_INVALID, who + "multipass too large");
    ip.lev.resize(ip.levels);
    for (int l = 0; l < ip.levels; ++l) {
      int rc = resolve(ctx, &it.params, it.ndims, it.dims, masked, 1 << l, ip.lev[l].pb);
      if (rc != MQP_OK) {
        ctx->last_error = who + ctx->last_error;
        return rc;
      }
      const Problem& pb = ip.lev[l].pb;
      if (pb.n_ia == 0) continue;
      if (it.ndims == 2) {
        if (mqp::piv2d_fft_len(pb.IS[0] + 2 * pb.SM[0], pb.IS[1] + 2 * pb.SM[1]) == 0)
          return fail(ctx, MQP_ERR_UNSUPPORTED, who + "2D search window (interSize + 2 searchMargin) too large at pass scale " +
                                                    std::to_string(1 << l));
      } else {
        const int SS[3] = {pb.IS[0] + 2 * pb.SM[0], pb.IS[1] + 2 * pb.SM[1], pb.IS[2] + 2 * pb.SM[2]};
        if (mqp::piv3d_fft_len(SS) == 0)
          return fail(ctx, MQP_ERR_UNSUPPORTED, who + "3D search window (interSize + 2 searchMargin) too large at pass scale " +
                                                    std::to_string(1 << l));
        if (!mqp::direct3d_ok(pb.IS, pb.SM)) {  // the direct kernel needs no chunk scratch
          const size_t per = mqp::piv3d_scratch_bytes_per_ia(pb.IS, pb.SM, pb.alg);
          scr3d_per = std::max(scr3d_per, per * (size_t)chunk_for(o, per, pb.n_ia));
        }
      }
    }
    ip.alg = ip.lev[0].pb.alg;
    rounds = std::max(rounds, ip.levels);
    // integral images once per pair (the images do not change between passes)
    if (ip.alg == mqp::ALG_NSQECC || ip.alg == mqp::ALG_ZNCC) {
      ip.n_ii = ip.alg == mqp::ALG_ZNCC ? 3 : 1;
      size_t b = (size_t)(it.dims[0] + 1) * (size_t)(it.dims[1] + 1) * sizeof(double);
      if (it.ndims == 3) b *= (size_t)(it.dims[2] + 1);
      for (int i = 0; i < ip.n_ii; ++i) ip.ii_off[i] = ar.take(b);
      if (it.ndims == 2) isc2d = std::max(isc2d, mqp::integral2d_scratch_bytes((int)it.dims[0], (int)it.dims[1]));
      else isc3d = std::max(isc3d, mqp::integral3d_scratch_bytes((int)it.dims[0], (int)it.dims[1], (int)it.dims[2]));
    }
    // an empty vector field is never written (an empty VF may have no address)
    if (!it.VF && ip.lev[0].pb.n_ia > 0) return fail(ctx, MQP_ERR_INVALID, who + "null VF pointer");
    for (int l = 0; l < ip.levels; ++l) {
      Level& L = ip.lev[l];
      const size_t n = (size_t)std::max<int64_t>(L.pb.n_ia, 1);
      if (l > 0) {
        L.vf_off = ar.take(n * it.ndims * sizeof(double));
        L.has_vf = true;
      }
      if (l < ip.levels - 1) {
        L.pred_off = ar.take(n * it.ndims * sizeof(int32_t));
        L.has_pred = true;
      }
    }
  }
  // 3D pairs to lanes, longest first onto the least loaded lane
  int n_lanes = 0;
  {
    std::vector<std::pair<double, int>> work;
    for (int k = 0; k < n_items; ++k)
      if (plan[k].it.ndims == 3) {
        double c = 0.0;
        for (const Level& L : plan[k].lev) c += cost3d(L.pb);
        work.push_back({c, k});
      }
    n_lanes = std::min<int>(LANES3D, (int)work.size());
    std::stable_sort(work.begin(), work.end(), [](const std::pair<double, int>& x, const std::pair<double, int>& y) {
      return x.first > y.first;
    });
    std::vector<double> load(n_lanes, 0.0);
    for (const auto& w : work) {
      const int ln = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      plan[w.second].lane = ln;
      load[ln] += w.first;
    }
  }
  // one 2D integral scratch per 2D lane (integral images of different pairs run side by side)
  std::vector<size_t> isc2d_off(LANES2D);
  for (int ln = 0; ln < LANES2D; ++ln) isc2d_off[ln] = isc2d ? ar.take(isc2d) : 0;
  std::vector<size_t> isc3d_off(n_lanes), scr3d_off(n_lanes);
  for (int ln = 0; ln < n_lanes; ++ln) {
    isc3d_off[ln] = ar.take(isc3d);
    scr3d_off[ln] = ar.take(scr3d_per + 8 * 256);
  }

  // 2D groups per round: one work queue per kernel variant
  struct Group {
    int N = 0;
    bool prune = false;
    int alg = 0, dtype = 0;
    bool lw = false;  // window sums on chip (piv2d_local_sums), as the single-pair path
    int wf2 = 0;
    std::vector<int> members;
    size_t items_off = 0, prefix_off = 0, counter_off = 0;
    std::vector<mqp::Piv2dArgs> args;
    std::vector<long long> prefix;
  };
  std::vector<std::vector<Group>> groups(rounds);
  for (int r = 0; r < rounds; ++r) {
    std::map<std::tuple<int, int, int, int, int>, int> idx;
    for (int k = 0; k < n_items; ++k) {
      const ItemPlan& ip = plan[k];
      const int l = ip.levels - 1 - r;
      if (l < 0 || ip.it.ndims != 2) continue;
      const Problem& pb = ip.lev[l].pb;
      if (pb.n_ia == 0) continue;
      // kernel variant: N = 1 marks the direct (spatial) correlation of small windows
      const bool direct = mqp::direct2d_ok(pb.IS[0], pb.IS[1], pb.SM[0], pb.SM[1]);
      const int N = direct ? 1 : mqp::piv2d_fft_len(pb.IS[0] + 2 * pb.SM[0], pb.IS[1] + 2 * pb.SM[1]);
      const bool prune = direct || (pb.IS[0] <= N / 2 && pb.IS[1] <= N / 2);
      const bool lw = !direct && mqp::piv2d_local_sums(pb.IS[0], pb.IS[1], pb.SM[0], pb.SM[1], ip.alg);
      const auto key = std::make_tuple(N, (int)prune, ip.alg, (int)ip.it.dtype, (int)lw);
      auto f = idx.find(key);
      if (f == idx.end()) {
        Group g;
        g.N = N;
        g.prune = prune;
        g.alg = ip.alg;
        g.dtype = ip.it.dtype;
        g.lw = lw;
        idx[key] = (int)groups[r].size();
        groups[r].push_back(g);
        f = idx.find(key);
      }
      Group& g = groups[r][f->second];
      g.members.push_back(k);
      g.wf2 = std::max(g.wf2, direct ? (mqp::piv2d_direct_words(pb.IS[0], pb.IS[1], pb.SM[0], pb.SM[1]) + 1) / 2
                              : lw   ? mqp::piv2d_warp_f2_lw(N, 2 * pb.SM[0] + 1, 2 * pb.SM[1] + 1)
                                     : mqp::piv2d_warp_f2(N, prune, 2 * pb.SM[0] + 1, 2 * pb.SM[1] + 1,
                                                          ip.alg == mqp::ALG_MASK_NSQECC));
    }
    for (Group& g : groups[r]) {
      g.items_off = ar.take(g.members.size() * sizeof(mqp::Piv2dArgs));
      g.prefix_off = ar.take((g.members.size() + 1) * sizeof(long long));
      g.counter_off = ar.take(sizeof(unsigned long long));
    }
  }

  mqp_plan* P = new mqp_plan();
  P->ctx = ctx;
  P->device = ctx->device;
  P->scratch_bytes = ar.size;
  cudaError_t e = P->arena.ensure(ar.size);
  if (e != cudaSuccess) {
    delete P;
    return cuda_fail(ctx, e, "batch plan scratch");
  }
  e = cudaMemset(P->arena.ptr, 0, ar.size);
  P->lanes.assign(n_lanes, nullptr);
  P->ev_join.assign(n_lanes, nullptr);
  for (int ln = 0; ln < n_lanes && e == cudaSuccess; ++ln) {
    e = cudaStreamCreateWithFlags(&P->lanes[ln], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev_join[ln], cudaEventDisableTiming);
  }
  size_t max_groups = 0, n_ii2d = 0;
  for (const auto& gr : groups) max_groups = std::max(max_groups, gr.size());
  for (const ItemPlan& ip : plan) n_ii2d += (ip.n_ii && ip.it.ndims == 2) ? 1 : 0;
  const size_t want2d = std::max(max_groups, n_ii2d);
  const int n_lanes2d = want2d > 1 ? (int)std::min<size_t>(LANES2D, want2d) : 0;
  P->lanes2d.assign(n_lanes2d, nullptr);
  P->ev_join2d.assign(n_lanes2d, nullptr);
  for (int ln = 0; ln < n_lanes2d && e == cudaSuccess; ++ln) {
    e = cudaStreamCreateWithFlags(&P->lanes2d[ln], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev_join2d[ln], cudaEventDisableTiming);
  }
  if (e == cudaSuccess && n_lanes2d) e = cudaEventCreateWithFlags(&P->ev_fork2d, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P->cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    mqp_batch_plan_destroy(P);
    return cuda_fail(ctx, e, "batch plan setup");
  }

  // fill and upload the 2D work lists
  for (int r = 0; r < rounds; ++r)
    for (Group& g : groups[r]) {
      long long total = 0;
      for (int k : g.members) {
        const ItemPlan& ip = plan[k];
        const int l = ip.levels - 1 - r;
        const Level& L = ip.lev[l];
        const Problem& pb = L.pb;
        mqp::Piv2dArgs a;
        memset(&a, 0, sizeof(a));
        a.img1 = ip.it.img1;
        a.img2 = ip.it.img2;
        a.mask = ip.it.mask;
        a.mask_skip = ip.it.mask_skip;
        a.dtype = ip.it.dtype;
        if (ip.n_ii >= 1) a.IIg2 = at<double>(P, ip.ii_off[0]);
        if (ip.n_ii >= 3) {
          a.IIg = at<double>(P, ip.ii_off[1]);
          a.II1 = at<double>(P, ip.ii_off[2]);
        }
        a.pred = L.has_pred ? at<int32_t>(P, L.pred_off) : nullptr;
        a.VF = l == 0 ? ip.it.VF : at<double>(P, L.vf_off);
        a.SN = (l == 0 && ip.it.params.computeSN) ? ip.it.SN : nullptr;
        a.planes = nullptr;
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
        a.ia_begin = 0;
        a.ia_end = pb.n_ia;
        a.threshold = ip.it.params.threshold;
        a.mask_threshold = ip.it.params.mask_threshold;
        a.computeSN = a.SN != nullptr;
        g.args.push_back(a);
        g.prefix.push_back(total);
        total += pb.n_ia;
      }
      g.prefix.push_back(total);
      e = cudaMemcpy(at<char>(P, g.items_off), g.args.data(), g.args.size() * sizeof(mqp::Piv2dArgs), cudaMemcpyHostToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(at<char>(P, g.prefix_off), g.prefix.data(), g.prefix.size() * sizeof(long long), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        mqp_batch_plan_destroy(P);
        return cuda_fail(ctx, e, "batch work lists");
      }
      P->total_ia += total;
    }

  // ---- the schedule ----
  P->ops.push_back([P](cudaStream_t m, const cudaStream_t* lanes) {
    if (P->lanes.empty()) return MQP_OK;
    if (cudaEventRecord(P->ev_fork, m) != cudaSuccess) return fail(P->ctx, MQP_ERR_CUDA, "batch fork");
    for (size_t ln = 0; ln < P->lanes.size(); ++ln)
      if (cudaStreamWaitEvent(lanes[ln], P->ev_fork, 0) != cudaSuccess) return fail(P->ctx, MQP_ERR_CUDA, "batch fork");
    return MQP_OK;
  });
  // 2D integral images: pairs spread over the 2D lanes, joined before round 0
  const int nl2i = n_ii2d > 1 ? (int)P->lanes2d.size() : 0;
  if (nl2i) {
    P->ops.push_back([P, nl2i](cudaStream_t m, const cudaStream_t*) {
      if (cudaEventRecord(P->ev_fork2d, m) != cudaSuccess) return fail(P->ctx, MQP_ERR_CUDA, "batch fork");
      for (int ln = 0; ln < nl2i; ++ln)
        if (cudaStreamWaitEvent(P->lanes2d[ln], P->ev_fork2d, 0) != cudaSuccess)
          return fail(P->ctx, MQP_ERR_CUDA, "batch fork");
      return MQP_OK;
    });
  }
  int ii2d = 0;
  for (int k = 0; k < n_items; ++k) {
    const ItemPlan& ip = plan[k];
    if (!ip.n_ii) continue;
    const bool d3 = ip.it.ndims == 3;
    const int lane2 = (!d3 && nl2i) ? ii2d++ % nl2i : -1;
    const void* i1 = ip.it.img1;
    const void* i2 = ip.it.img2;
    const int dt = ip.it.dtype, n_ii = ip.n_ii;
    const int H = (int)ip.it.dims[0], W = (int)ip.it.dims[1], D = d3 ? (int)ip.it.dims[2] : 1;
    double* ii[3] = {at<double>(P, ip.ii_off[0]), n_ii > 1 ? at<double>(P, ip.ii_off[1]) : nullptr,
                     n_ii > 2 ? at<double>(P, ip.ii_off[2]) : nullptr};
    double* isc = at<double>(P, d3 ? isc3d_off[ip.lane] : isc2d_off[lane2 >= 0 ? lane2 : 0]);
    const int lane = ip.lane;
    P->launches += (int64_t)n_ii * (d3 ? integral_kernels_2d(W) + 1 : integral_kernels_2d(W));
    P->ops.push_back([=](cudaStream_t m, const cudaStream_t* lanes) {
      cudaStream_t st = d3 ? lanes[lane] : (lane2 >= 0 ? P->lanes2d[lane2] : m);
      const void* src[3] = {i2, i2, i1};
      const bool sq[3] = {true, false, false};
      for (int i = 0; i < n_ii; ++i) {
        const cudaError_t e2 = d3 ? mqp::launch_integral3d(src[i], dt, H, W, D, sq[i], ii[i], isc, st)
                                  : mqp::launch_integral2d(src[i], dt, H, W, sq[i], ii[i], isc, st);
        if (e2 != cudaSuccess) return cuda_fail(P->ctx, e2, "batch integral images");
      }
      return MQP_OK;
    });
  }
  if (nl2i) {
    P->ops.push_back([P, nl2i](cudaStream_t m, const cudaStream_t*) {
      for (int ln = 0; ln < nl2i; ++ln)
        if (cudaEventRecord(P->ev_join2d[ln], P->lanes2d[ln]) != cudaSuccess ||
            cudaStreamWaitEvent(m, P->ev_join2d[ln], 0) != cudaSuccess)
          return fail(P->ctx, MQP_ERR_CUDA, "batch join");
      return MQP_OK;
    });
  }
  for (int r = 0; r < rounds; ++r) {
    // predictors of this round (2D on the main stream, 3D on the side stream)
    for (int k = 0; k < n_items; ++k) {
      const ItemPlan& ip = plan[k];
      const int l = ip.levels - 1 - r;
      if (l < 0 || l == ip.levels - 1 || ip.lev[l].pb.n_ia == 0) continue;
      const Level& L = ip.lev[l];
      const Level& C = ip.lev[l + 1];
      mqp::PredArgs pa;
      memset(&pa, 0, sizeof(pa));
      pa.ndims = ip.it.ndims;
      for (int d = 0; d < pa.ndims; ++d) {
        pa.vf_f[d] = (int)L.pb.vf[d];
        pa.vf_c[d] = (int)C.pb.vf[d];
        pa.isz_f[d] = L.pb.IS[d];
        pa.st_f[d] = L.pb.st[d];
        pa.isz_c[d] = C.pb.IS[d];
        pa.st_c[d] = C.pb.st[d];
      }
      pa.VFc = at<double>(P, C.vf_off);
      pa.pred = at<int32_t>(P, L.pred_off);
      const bool d3 = ip.it.ndims == 3;
      const int lane = ip.lane;
      P->launches += 1;
      P->ops.push_back([=](cudaStream_t m, const cudaStream_t* lanes) {
        const cudaError_t e2 = mqp::launch_predictor(pa, d3 ? lanes[lane] : m);
        return e2 == cudaSuccess ? MQP_OK : cuda_fail(P->ctx, e2, "batch predictor");
      });
    }
    // several kernel variants this round: fork them onto the 2D lanes and
    // join them back before the next round's predictors read their vectors
    const int nl2 = groups[r].size() > 1 ? std::min<int>((int)P->lanes2d.size(), (int)groups[r].size()) : 0;
    if (nl2) {
      P->ops.push_back([P, nl2](cudaStream_t m, const cudaStream_t*) {
        if (cudaEventRecord(P->ev_fork2d, m) != cudaSuccess) return fail(P->ctx, MQP_ERR_CUDA, "batch fork");
        for (int ln = 0; ln < nl2; ++ln)
          if (cudaStreamWaitEvent(P->lanes2d[ln], P->ev_fork2d, 0) != cudaSuccess)
            return fail(P->ctx, MQP_ERR_CUDA, "batch fork");
        return MQP_OK;
      });
    }
    int gi = 0;
    for (const Group& g : groups[r]) {
      const int lane2 = nl2 ? gi++ % nl2 : -1;
      mqp::Piv2dBatch b;
      b.items = at<mqp::Piv2dArgs>(P, g.items_off);
      b.prefix = at<long long>(P, g.prefix_off);
      b.n_items = (int)g.members.size();
      b.total = g.prefix.back();
      b.N = g.N;
      b.prune = g.prune;
      b.alg = g.alg;
      b.dtype = g.dtype;
      b.wf2 = g.wf2;
      b.grab = o.grab;
      b.lw = g.lw;
      b.counter = at<unsigned long long>(P, g.counter_off);
      P->launches += 1;
      P->ops.push_back([=](cudaStream_t m, const cudaStream_t*) {
        std::string err;
        const cudaError_t e2 = mqp::launch_piv2d_batch(b, lane2 >= 0 ? P->lanes2d[lane2] : m, err);
        return e2 == cudaSuccess ? MQP_OK : fail(P->ctx, MQP_ERR_CUDA, "batch 2D launch: " + err);
      });
    }
    if (nl2) {
      P->ops.push_back([P, nl2](cudaStream_t m, const cudaStream_t*) {
        for (int ln = 0; ln < nl2; ++ln)
          if (cudaEventRecord(P->ev_join2d[ln], P->lanes2d[ln]) != cudaSuccess ||
              cudaStreamWaitEvent(m, P->ev_join2d[ln], 0) != cudaSuccess)
            return fail(P->ctx, MQP_ERR_CUDA, "batch join");
        return MQP_OK;
      });
    }
    for (int k = 0; k < n_items; ++k) {
      const ItemPlan& ip = plan[k];
      const int l = ip.levels - 1 - r;
      if (l < 0 || ip.it.ndims != 3 || ip.lev[l].pb.n_ia == 0) continue;
      const Level& L = ip.lev[l];
      const Problem& pb = L.pb;
      const size_t per = mqp::piv3d_scratch_bytes_per_ia(pb.IS, pb.SM, pb.alg);
      const int64_t chunk = chunk_for(o, per, pb.n_ia);
      mqp::Piv3dArgs a;
      memset(&a, 0, sizeof(a));
      for (int d = 0; d < 3; ++d) {
        a.IS[d] = pb.IS[d];
        a.SM[d] = pb.SM[d];
      }
      mqp::piv3d_bind_scratch(a, pb.alg, chunk, at<char>(P, scr3d_off[ip.lane]));
      a.img1 = ip.it.img1;
      a.img2 = ip.it.img2;
      a.mask = ip.it.mask;
      a.mask_skip = ip.it.mask_skip;
      a.dtype = ip.it.dtype;
      if (ip.n_ii >= 1) a.IIg2 = at<double>(P, ip.ii_off[0]);
      if (ip.n_ii >= 3) {
        a.IIg = at<double>(P, ip.ii_off[1]);
        a.II1 = at<double>(P, ip.ii_off[2]);
      }
      a.pred = L.has_pred ? at<int32_t>(P, L.pred_off) : nullptr;
      a.VF = l == 0 ? ip.it.VF : at<double>(P, L.vf_off);
      a.SN = (l == 0 && ip.it.params.computeSN) ? ip.it.SN : nullptr;
      a.H = (int)pb.dims[0];
      a.W = (int)pb.dims[1];
      a.D = (int)pb.dims[2];
      for (int d = 0; d < 3; ++d) {
        a.IS[d] = pb.IS[d];
        a.SM[d] = pb.SM[d];
        a.st[d] = pb.st[d];
        a.vf[d] = (int)pb.vf[d];
      }
      a.ia_begin = 0;
      a.ia_end = pb.n_ia;
      a.threshold = ip.it.params.threshold;
      a.mask_threshold = ip.it.params.mask_threshold;
      const int alg = pb.alg;
      const int64_t chunks = (pb.n_ia + chunk - 1) / chunk;
      P->launches += mqp::direct3d_ok(pb.IS, pb.SM) ? 1 : chunks * (alg == mqp::ALG_MASK_NSQECC ? 7 : 5);
      P->total_ia += pb.n_ia;
      const int lane = ip.lane;
      P->ops.push_back([=](cudaStream_t, const cudaStream_t* lanes) {
        std::string err;
        const cudaError_t e2 = mqp::launch_piv3d(a, alg, chunk, lanes[lane], err);
        return e2 == cudaSuccess ? MQP_OK : fail(P->ctx, MQP_ERR_CUDA, "batch 3D launch: " + err);
      });
    }
  }
  P->ops.push_back([P](cudaStream_t m, const cudaStream_t* lanes) {
    for (size_t ln = 0; ln < P->lanes.size(); ++ln)
      if (cudaEventRecord(P->ev_join[ln], lanes[ln]) != cudaSuccess || cudaStreamWaitEvent(m, P->ev_join[ln], 0) != cudaSuccess)
        return fail(P->ctx, MQP_ERR_CUDA, "batch join");
    return MQP_OK;
  });

  if (o.use_graph) {
    e = cudaStreamBeginCapture(P->cap, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? MQP_OK : cuda_fail(ctx, e, "batch graph capture");
    if (rc == MQP_OK)
      for (auto& op : P->ops)
        if ((rc = op(P->cap, P->lanes.data())) != MQP_OK) break;
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(P->cap, &g);
    if (rc == MQP_OK && e2 != cudaSuccess) rc = cuda_fail(ctx, e2, "batch graph capture");
    if (rc == MQP_OK) {
      P->graph = g;
      e = cudaGraphInstantiate(&P->exec, g, 0);
      if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batch graph instantiate");
    } else if (g) {
      cudaGraphDestroy(g);
    }
    if (rc != MQP_OK) {
      cudaGetLastError();
      mqp_batch_plan_destroy(P);
      return rc;
    }
  }
  *out = P;
  return MQP_OK;
}

int mqp_batch_plan_run(mqp_plan* plan, void* stream) {
  NvtxRange nv("mqp_batch_plan_run");
  if (!plan) return fail(nullptr, MQP_ERR_INVALID, "null plan");
  mqp_ctx* ctx = plan->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(plan->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : cudaStreamLegacy;
  if (plan->exec) {
    const cudaError_t e = cudaGraphLaunch(plan->exec, s);
    return e == cudaSuccess ? MQP_OK : cuda_fail(ctx, e, "batch graph launch");
  }
  for (auto& op : plan->ops) {
    const int rc = op(s, plan->lanes.data());
    if (rc != MQP_OK) return rc;
  }
  return MQP_OK;
}

int mqp_batch_plan_info(const mqp_plan* plan, int64_t* total_ia, int64_t* launches, int64_t* scratch_bytes) {
  if (!plan) return fail(nullptr, MQP_ERR_INVALID, "null plan");
  if (total_ia) *total_ia = plan->total_ia;
  if (launches) *launches = plan->launches;
  if (scratch_bytes) *scratch_bytes = (int64_t)plan->scratch_bytes;
  return MQP_OK;
}

int mqp_batch_plan_destroy(mqp_plan* plan) {
  if (!plan) return MQP_OK;
  cudaSetDevice(plan->device);
  for (cudaStream_t ln : plan->lanes)
    if (ln) cudaStreamSynchronize(ln);
  cudaDeviceSynchronize();
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  if (plan->graph) cudaGraphDestroy(plan->graph);
  if (plan->ev_fork) cudaEventDestroy(plan->ev_fork);
  for (cudaEvent_t ev : plan->ev_join)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : plan->ev_join2d)
    if (ev) cudaEventDestroy(ev);
  if (plan->ev_fork2d) cudaEventDestroy(plan->ev_fork2d);
  for (cudaStream_t ln : plan->lanes2d)
    if (ln) {
      cudaStreamSynchronize(ln);
      cudaStreamDestroy(ln);
    }
  for (cudaStream_t ln : plan->lanes)
    if (ln) cudaStreamDestroy(ln);
  if (plan->cap) cudaStreamDestroy(plan->cap);
  plan->arena.release();
  delete plan;
  return MQP_OK;
}

}  // extern "C"
