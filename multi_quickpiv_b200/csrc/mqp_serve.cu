// Serving runtime (include/mqp.h, mqp_server_*): PIV requests of time-lapse
// streams, frame t against frame t+1, admitted continuously as execution
// slots and device memory free up.
//
//   streams   each time-lapse stream (fixed frame size, dtype and PIV
//             parameters) keeps its last frames resident in a ring of three
//             device buffers, with the plain integral image of each frame for
//             ZNCC (it is the next request's integral of img1), so a request
//             uploads only its new frame.
//   slots     `slots` CUDA streams; a request runs entirely on one: upload of
//             its frame from pinned staging, integral images, the PIV kernels
//             (fused 2D or K3a/K3b/K3c), download of VF/SN to pinned memory.
//             Requests on different slots overlap on the device.
//   admission a worker thread admits queued requests (FIFO, skipping requests
//             that must wait for their stream's previous frame) whenever a
//             slot is free and the request's transient device bytes (integral
//             images, 3D chunk scratch, outputs; stream-ordered allocations)
//             fit the free-memory budget.  Frames of one stream are ordered
//             by events: request k waits for request k-1's upload.
//   host side pinned staging and result buffers are allocated when a stream
//             opens (one per slot); submit copies the frame into staging
//             outside the server lock, and a finished request's VF/SN move
//             from pinned memory to host memory the request owns, so requests
//             whose results are collected late hold no pinned memory and the
//             worker never waits on a pinned allocation or a large copy.
//   latency   submit -> result on the host, per request; mqp_server_get_stats
//             reports p50 / p99 of it and of its two parts (queued: submit ->
//             issue; running: issue -> done) and throughput.  With the
//             environment variable MQP_SERVER_TRACE set to a file name, the
//             server writes every finished request's timeline there (CSV) when
//             it is destroyed.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "mqp.h"
#include "mqp_ctx.h"
#include "mqp_internal.h"

using namespace mqp_host;

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

constexpr int RING = 3;

// Pinned host buffers of one size, owned by a stream: staging for its new
// frames, or downloads of its results.  Buffers go back to `free` when the
// request that held them finishes; none is released before the server.
struct HostBufs {
  size_t n = 0;
  std::vector<void*> free, all;
  void* take() {
    if (free.empty()) return nullptr;
    void* p = free.back();
    free.pop_back();
    return p;
  }
  void put(void* p) {
    if (p) free.push_back(p);
  }
  void add(void* p, bool in_use) {
    all.push_back(p);
    if (!in_use) free.push_back(p);
  }
  void release() {
    for (void* p : all) cudaFreeHost(p);
    all.clear();
    free.clear();
  }
};

struct SrvStream {
  int id = 0;
  int ndims = 2;
  int64_t dims[3] = {1, 1, 1};
  int dtype = MQP_F32;
  mqp_params p{};
  Problem pb;
  size_t frame_bytes = 0, ii_bytes = 0;
  void* frames[RING] = {nullptr, nullptr, nullptr};
  double* ii[RING] = {nullptr, nullptr, nullptr};  // plain integral of each frame (ZNCC)
  cudaEvent_t ready[RING] = {nullptr, nullptr, nullptr};
  int64_t submitted = 0;  // frames submitted after the first
  int64_t issued = 0;     // requests issued to a slot
  int64_t done = 0;       // requests completed
  size_t transient = 0;   // device bytes one request allocates while it runs
  HostBufs stage, res;    // pinned frame staging, pinned result downloads
};

struct SrvRequest {
  uint64_t id = 0;
  int stream = 0;
  int64_t k = 0;        // frame index of the new frame (>= 1)
  void* staging = nullptr;  // pinned copy of the new frame
  double* res = nullptr;    // pinned VF then SN, held while the request runs
  std::vector<double> vf, sn;  // results, filled when the request finishes
  size_t vf_n = 0, sn_n = 0;
  double t_submit = 0, t_issue = 0, t_done = 0;
  int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
  int slot = -1;
  std::string err;
};

struct Slot {
  cudaStream_t s = nullptr;
  cudaEvent_t done = nullptr;
  uint64_t req = 0;
  bool busy = false;
};

}  // namespace

struct mqp_server {
  int device = 0;
  mqp_server_options opt{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
  std::map<int, SrvStream> streams;
  int next_stream = 1;
  std::map<uint64_t, SrvRequest> reqs;
  std::deque<uint64_t> queue;
  uint64_t next_req = 1;
  std::vector<Slot> slots;
  size_t budget = 0, in_use = 0;
  std::vector<double> lat, lat_wait, lat_run;  // completed latencies (ms): total, queued, running
  struct TraceRec {
    uint64_t id;
    int stream, slot, state;
    int64_t k;
    double t_submit, t_issue, t_done;
  };
  std::vector<TraceRec> trace;
  std::string trace_path;
  double t_first = 0, t_last = 0;
  int64_t ia_done = 0, completed = 0, failed = 0, admitted_overlap = 0;
  std::string last_error;
};

namespace {

int srv_fail(mqp_server* S, int code, const std::string& m) {
  if (S) S->last_error = m;
  return code;
}

// Transient device bytes of one request of stream st (allocated on the slot's
// stream and freed there when the request finishes).
size_t request_bytes(const SrvStream& st) {
  size_t b = 0;
  const bool norm = st.pb.alg == mqp::ALG_NSQECC || st.pb.alg == mqp::ALG_ZNCC;
  if (norm) {
    b += st.ii_bytes;  // integral of the new frame squared
    b += st.ndims == 2 ? mqp::integral2d_scratch_bytes((int)st.dims[0], (int)st.dims[1])
                       : mqp::integral3d_scratch_bytes((int)st.dims[0], (int)st.dims[1], (int)st.dims[2]);
    if (st.pb.alg == mqp::ALG_ZNCC) b += st.ii_bytes;  // integral of the new frame (kept in the ring)
  }
  b += (size_t)std::max<int64_t>(st.pb.n_ia, 1) * (st.ndims + 1) * sizeof(double);
  if (st.ndims == 3 && !mqp::direct3d_ok(st.pb.IS, st.pb.SM)) {
    const size_t per = mqp::piv3d_scratch_bytes_per_ia(st.pb.IS, st.pb.SM, st.pb.alg);
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(st.pb.n_ia, (int64_t)(st.transient / per)));
    b += per * (size_t)chunk + 8 * 256;
  }
  return b;
}

int64_t chunk3d_of(const SrvStream& st) {
  const size_t per = mqp::piv3d_scratch_bytes_per_ia(st.pb.IS, st.pb.SM, st.pb.alg);
  return std::max<int64_t>(1, std::min<int64_t>({st.pb.n_ia, (int64_t)(st.transient / per), 65535}));
}

// Enqueue request r of stream st on slot stream s.  Returns "" or an error.
std::string issue(mqp_server* S, SrvStream& st, SrvRequest& r, cudaStream_t s) {
  NvtxRange nv("mqp_server_request");
  const int cur = (int)(r.k % RING), prev = (int)((r.k - 1) % RING);
  cudaError_t e;
  auto bad = [](cudaError_t e, const char* what) { return std::string(what) + ": " + cudaGetErrorString(e); };
  if ((e = cudaStreamWaitEvent(s, st.ready[prev], 0)) != cudaSuccess) return bad(e, "frame order");
  if ((e = cudaMemcpyAsync(st.frames[cur], r.staging, st.frame_bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return bad(e, "frame upload");
  const int H = (int)st.dims[0], W = (int)st.dims[1], D = (int)st.dims[2];
  const void* img1 = st.frames[prev];
  const void* img2 = st.frames[cur];
  const bool norm = st.pb.alg == mqp::ALG_NSQECC || st.pb.alg == mqp::ALG_ZNCC;
  double* IIg2 = nullptr;
  double* isc = nullptr;
  std::vector<void*> tmp;
  auto alloc = [&](size_t n) -> void* {
    void* p = nullptr;
    if (cudaMallocAsync(&p, n ? n : 8, s) != cudaSuccess) return nullptr;
    tmp.push_back(p);
    return p;
  };
  std::string err;
  auto integral = [&](const void* img, bool sq, double* out) {
    return st.ndims == 2 ? mqp::launch_integral2d(img, st.dtype, H, W, sq, out, isc, s)
                         : mqp::launch_integral3d(img, st.dtype, H, W, D, sq, out, isc, s);
  };
  if (norm) {
    isc = (double*)alloc(st.ndims == 2 ? mqp::integral2d_scratch_bytes(H, W) : mqp::integral3d_scratch_bytes(H, W, D));
    IIg2 = (double*)alloc(st.ii_bytes);
    if (!isc || !IIg2) err = "transient allocation";
    if (err.empty() && (e = integral(img2, true, IIg2)) != cudaSuccess) err = bad(e, "integral image");
    if (err.empty() && st.pb.alg == mqp::ALG_ZNCC && (e = integral(img2, false, st.ii[cur])) != cudaSuccess)
      err = bad(e, "integral image");
  }
  // frame k (and its plain integral) is now ready for request k+1
  if (err.empty() && (e = cudaEventRecord(st.ready[cur], s)) != cudaSuccess) err = bad(e, "event");
  double* dVF = err.empty() ? (double*)alloc(r.vf_n * sizeof(double)) : nullptr;
  double* dSN = (err.empty() && r.sn_n) ? (double*)alloc(r.sn_n * sizeof(double)) : nullptr;
  if (err.empty() && (!dVF || (r.sn_n && !dSN))) err = "transient allocation";
  if (err.empty() && st.ndims == 2) {
    mqp::Piv2dArgs a;
    memset(&a, 0, sizeof(a));
    a.img1 = img1;
    a.img2 = img2;
    a.dtype = st.dtype;
    a.IIg2 = IIg2;
    if (st.pb.alg == mqp::ALG_ZNCC) {
      a.IIg = st.ii[cur];
      a.II1 = st.ii[prev];
    }
    a.VF = dVF;
    a.SN = dSN;
    a.H = H;
    a.W = W;
    a.IS1 = st.pb.IS[0];
    a.IS2 = st.pb.IS[1];
    a.SM1 = st.pb.SM[0];
    a.SM2 = st.pb.SM[1];
    a.st1 = st.pb.st[0];
    a.st2 = st.pb.st[1];
    a.vf1 = (int)st.pb.vf[0];
    a.vf2 = (int)st.pb.vf[1];
    a.ia_begin = 0;
    a.ia_end = st.pb.n_ia;
    a.threshold = st.p.threshold;
    a.mask_threshold = st.p.mask_threshold;
    a.computeSN = dSN != nullptr;
    if ((e = mqp::launch_piv2d(a, st.pb.alg, s, err)) != cudaSuccess && err.empty()) err = bad(e, "PIV kernel");
  } else if (err.empty()) {
    const int64_t chunk = chunk3d_of(st);
    const size_t per = mqp::piv3d_scratch_bytes_per_ia(st.pb.IS, st.pb.SM, st.pb.alg);
    const bool direct = mqp::direct3d_ok(st.pb.IS, st.pb.SM);  // no chunk scratch
    char* base = direct ? (char*)dVF : (char*)alloc(per * (size_t)chunk + 8 * 256);
    if (!base) {
      err = "transient allocation";
    } else {
      mqp::Piv3dArgs a;
      memset(&a, 0, sizeof(a));
      for (int d = 0; d < 3; ++d) {
        a.IS[d] = st.pb.IS[d];
        a.SM[d] = st.pb.SM[d];
      }
      mqp::piv3d_bind_scratch(a, st.pb.alg, chunk, base);
      a.img1 = img1;
      a.img2 = img2;
      a.dtype = st.dtype;
      a.IIg2 = IIg2;
      if (st.pb.alg == mqp::ALG_ZNCC) {
        a.IIg = st.ii[cur];
        a.II1 = st.ii[prev];
      }
      a.VF = dVF;
      a.SN = dSN;
      a.H = H;
      a.W = W;
      a.D = D;
      for (int d = 0; d < 3; ++d) {
        a.IS[d] = st.pb.IS[d];
        a.SM[d] = st.pb.SM[d];
        a.st[d] = st.pb.st[d];
        a.vf[d] = (int)st.pb.vf[d];
      }
      a.ia_begin = 0;
      a.ia_end = st.pb.n_ia;
      a.threshold = st.p.threshold;
      a.mask_threshold = st.p.mask_threshold;
      if ((e = mqp::launch_piv3d(a, st.pb.alg, chunk, s, err)) != cudaSuccess && err.empty()) err = bad(e, "PIV kernels");
    }
  }
  if (err.empty() &&
      (e = cudaMemcpyAsync(r.res, dVF, r.vf_n * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    err = bad(e, "VF download");
  if (err.empty() && r.sn_n &&
      (e = cudaMemcpyAsync(r.res + r.vf_n, dSN, r.sn_n * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    err = bad(e, "SN download");
  for (void* p : tmp) cudaFreeAsync(p, s);
  return err;
}

void worker_loop(mqp_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  while (!S->stop) {
    bool progress = false;
    // completions
    for (size_t i = 0; i < S->slots.size(); ++i) {
      Slot& sl = S->slots[i];
      if (!sl.busy) continue;
      const cudaError_t q = cudaEventQuery(sl.done);
      if (q == cudaErrorNotReady) continue;
      SrvRequest& r = S->reqs[sl.req];
      SrvStream& st = S->streams[r.stream];
      r.t_done = now_ms();
      if (q != cudaSuccess) {
        r.state = 3;
        r.err = std::string("request: ") + cudaGetErrorString(q);
        ++S->failed;
      } else {
        r.vf.assign(r.res, r.res + r.vf_n);
        if (r.sn_n) r.sn.assign(r.res + r.vf_n, r.res + r.vf_n + r.sn_n);
        r.state = 2;
        S->lat.push_back(r.t_done - r.t_submit);
        S->lat_wait.push_back(r.t_issue - r.t_submit);
        S->lat_run.push_back(r.t_done - r.t_issue);
        S->ia_done += st.pb.n_ia;
        ++S->completed;
        S->t_last = r.t_done;
      }
      st.stage.put(r.staging);
      st.res.put(r.res);
      r.staging = nullptr;
      r.res = nullptr;
      S->in_use -= request_bytes(st);
      if (!S->trace_path.empty()) S->trace.push_back({r.id, r.stream, (int)i, r.state, r.k, r.t_submit, r.t_issue, r.t_done});
      st.done += 1;
      sl.busy = false;
      progress = true;
    }
    // admission: FIFO, requests whose stream is not ready are skipped over
    for (auto it = S->queue.begin(); it != S->queue.end();) {
      int free_slot = -1;
      for (size_t i = 0; i < S->slots.size(); ++i)
        if (!S->slots[i].busy) {
          free_slot = (int)i;
          break;
        }
      if (free_slot < 0) break;
      SrvRequest& r = S->reqs[*it];
      SrvStream& st = S->streams[r.stream];
      const size_t need = request_bytes(st);
      // request k: k-1 issued (its upload precedes ours on the GPU through the
      // stream's events), k-2 finished (its frames leave the ring slot we overwrite)
      const bool ordered = st.issued == r.k - 1 && st.done >= r.k - 2;
      if (!ordered || S->in_use + need > S->budget) {
        ++it;
        continue;
      }
      // the stream's pinned result buffers number the slots and at most
      // slots - 1 requests run now, so one is free (allocated only if
      // open_stream could not make them all)
      r.res = (double*)st.res.take();
      if (!r.res) {
        void* h = nullptr;
        if (cudaMallocHost(&h, st.res.n) != cudaSuccess) {
          ++it;
          continue;
        }
        st.res.add(h, true);
        r.res = (double*)h;
      }
      Slot& sl = S->slots[free_slot];
      int busy = 0;
      for (auto& o : S->slots) busy += o.busy;
      if (busy > 0) ++S->admitted_overlap;
      r.t_issue = now_ms();
      std::string err = issue(S, st, r, sl.s);
      cudaError_t e = cudaEventRecord(sl.done, sl.s);
      if (err.empty() && e != cudaSuccess) err = std::string("event: ") + cudaGetErrorString(e);
      st.issued += 1;
      if (!err.empty()) {
        // the slot stream is still usable: wait for what was enqueued, then fail the request
        cudaStreamSynchronize(sl.s);
        cudaGetLastError();
        r.state = 3;
        r.err = err;
        r.t_done = now_ms();
        ++S->failed;
        st.done += 1;
        st.stage.put(r.staging);
        st.res.put(r.res);
        r.staging = nullptr;
        r.res = nullptr;
      } else {
        r.state = 1;
        r.slot = free_slot;
        sl.busy = true;
        sl.req = r.id;
        S->in_use += need;
      }
      it = S->queue.erase(it);
      progress = true;
    }
    if (progress) S->cv_done.notify_all();
    bool running = false;
    for (auto& sl : S->slots) running = running || sl.busy;
    if (running) S->cv_work.wait_for(lk, std::chrono::microseconds(50));
    else S->cv_work.wait(lk, [S] { return S->stop || !S->queue.empty(); });
  }
}

}  // namespace

extern "C" {

int mqp_server_create(int device, const mqp_server_options* opt, mqp_server** out) {
  if (!out) return MQP_ERR_INVALID;
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return MQP_ERR_CUDA;
  mqp_server* S = new mqp_server();
  S->device = device;
  S->opt.slots = 4;
  S->opt.hbm_reserve_bytes = (int64_t)4 << 30;
  S->opt.chunk3d_budget = (int64_t)512 << 20;
  if (opt) {
    if (opt->slots > 0) S->opt.slots = opt->slots;
    if (opt->hbm_budget_bytes > 0) S->opt.hbm_budget_bytes = opt->hbm_budget_bytes;
    if (opt->hbm_reserve_bytes > 0) S->opt.hbm_reserve_bytes = opt->hbm_reserve_bytes;
    if (opt->chunk3d_budget > 0) S->opt.chunk3d_budget = opt->chunk3d_budget;
  }
  if (S->opt.slots > 64) S->opt.slots = 64;
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  S->budget = S->opt.hbm_budget_bytes > 0 ? (size_t)S->opt.hbm_budget_bytes
                                          : (fr > (size_t)S->opt.hbm_reserve_bytes ? fr - (size_t)S->opt.hbm_reserve_bytes : 0);
  // keep freed transient memory in the device's pool between requests
  // (process-local: the pool of this process's context)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (const char* tp = getenv("MQP_SERVER_TRACE")) S->trace_path = tp;
  S->slots.resize(S->opt.slots);
  for (auto& sl : S->slots) {
    if ((e = cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess) {
      mqp_server_destroy(S);
      return MQP_ERR_CUDA;
    }
  }
  S->worker = std::thread(worker_loop, S);
  *out = S;
  return MQP_OK;
}

const char* mqp_server_last_error(const mqp_server* S) { return S ? S->last_error.c_str() : ""; }

int mqp_server_open_stream(mqp_server* S, const void* first_frame, int dtype, int ndims, const int64_t dims[3],
                           const mqp_params* p, int32_t* stream_id) {
  if (!S || !first_frame || !dims || !p || !stream_id) return srv_fail(S, MQP_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  cudaSetDevice(S->device);
  if (dtype != MQP_F32 && dtype != MQP_F64) return srv_fail(S, MQP_ERR_INVALID, "dtype must be MQP_F32 or MQP_F64");
  if (p->refine && p->multipass > 1) return srv_fail(S, MQP_ERR_UNSUPPORTED, "serving runs single-pass PIV");
  SrvStream st;
  st.id = S->next_stream;
  st.ndims = ndims;
  st.dtype = dtype;
  st.p = *p;
  mqp_ctx tmp;  // resolve() reports into a context
  int rc = resolve(&tmp, p, ndims, dims, false, 1, st.pb);
  if (rc != MQP_OK) return srv_fail(S, rc, tmp.last_error);
  for (int d = 0; d < 3; ++d) st.dims[d] = st.pb.dims[d];
  if (ndims == 2 && mqp::piv2d_fft_len(st.pb.IS[0] + 2 * st.pb.SM[0], st.pb.IS[1] + 2 * st.pb.SM[1]) == 0)
    return srv_fail(S, MQP_ERR_UNSUPPORTED, "2D search window too large");
  if (ndims == 3) {
    const int SS[3] = {st.pb.IS[0] + 2 * st.pb.SM[0], st.pb.IS[1] + 2 * st.pb.SM[1], st.pb.IS[2] + 2 * st.pb.SM[2]};
    if (mqp::piv3d_fft_len(SS) == 0) return srv_fail(S, MQP_ERR_UNSUPPORTED, "3D search window too large");
  }
  size_t npx = 1;
  for (int d = 0; d < ndims; ++d) npx *= (size_t)st.dims[d];
  st.frame_bytes = npx * (dtype == MQP_F64 ? 8 : 4);
  st.ii_bytes = (size_t)(st.dims[0] + 1) * (size_t)(st.dims[1] + 1) * (ndims == 3 ? (size_t)(st.dims[2] + 1) : 1) * sizeof(double);
  st.transient = (size_t)S->opt.chunk3d_budget;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < RING && e == cudaSuccess; ++i) {
    e = cudaMalloc(&st.frames[i], st.frame_bytes);
    if (e == cudaSuccess && st.pb.alg == mqp::ALG_ZNCC) e = cudaMalloc((void**)&st.ii[i], st.ii_bytes);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st.ready[i], cudaEventDisableTiming);
  }
  // frame 0 and its plain integral (ZNCC), synchronously
  if (e == cudaSuccess) e = cudaMemcpy(st.frames[0], first_frame, st.frame_bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && st.pb.alg == mqp::ALG_ZNCC) {
    double* isc = nullptr;
    const size_t ib = ndims == 2 ? mqp::integral2d_scratch_bytes((int)st.dims[0], (int)st.dims[1])
                                 : mqp::integral3d_scratch_bytes((int)st.dims[0], (int)st.dims[1], (int)st.dims[2]);
    e = cudaMalloc((void**)&isc, ib);
    if (e == cudaSuccess)
      e = ndims == 2 ? mqp::launch_integral2d(st.frames[0], dtype, (int)st.dims[0], (int)st.dims[1], false, st.ii[0], isc, 0)
                     : mqp::launch_integral3d(st.frames[0], dtype, (int)st.dims[0], (int)st.dims[1], (int)st.dims[2], false,
                                              st.ii[0], isc, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (isc) cudaFree(isc);
  }
  if (e == cudaSuccess) e = cudaEventRecord(st.ready[0], 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    for (int i = 0; i < RING; ++i) {
      if (st.frames[i]) cudaFree(st.frames[i]);
      if (st.ii[i]) cudaFree(st.ii[i]);
      if (st.ready[i]) cudaEventDestroy(st.ready[i]);
    }
    return srv_fail(S, e == cudaErrorMemoryAllocation ? MQP_ERR_OOM : MQP_ERR_CUDA,
                    std::string("open stream: ") + cudaGetErrorString(e));
  }
  // pinned staging for new frames and result buffers, one per slot (staging
  // bounded to 256 MiB per stream; further frames in flight allocate more)
  st.res.n = (size_t)std::max<int64_t>(st.pb.n_ia, 1) * (st.ndims + (st.p.computeSN ? 1 : 0)) * sizeof(double);
  st.stage.n = st.frame_bytes;
  const size_t n_stage = std::max<size_t>(1, std::min<size_t>(S->slots.size(), ((size_t)256 << 20) / st.frame_bytes));
  for (size_t i = 0; i < S->slots.size() + n_stage; ++i) {
    HostBufs& hb = i < S->slots.size() ? st.res : st.stage;
    void* h = nullptr;
    if (cudaMallocHost(&h, hb.n) != cudaSuccess) break;  // allocated again on demand
    hb.add(h, false);
  }
  // grow the device pool now to hold every slot running a request of this
  // stream: growing it later (two large 3D requests meeting for the first
  // time) would stall the worker inside the allocation for tens of ms
  {
    const size_t need = request_bytes(st);
    std::vector<void*> warm;
    for (size_t i = 0; i < S->slots.size() && S->in_use + (i + 1) * need <= S->budget; ++i) {
      void* d = nullptr;
      if (cudaMallocAsync(&d, need, S->slots[0].s) != cudaSuccess) break;
      warm.push_back(d);
    }
    for (void* d : warm) cudaFreeAsync(d, S->slots[0].s);
    cudaStreamSynchronize(S->slots[0].s);
    cudaGetLastError();
  }
  S->streams[st.id] = st;
  *stream_id = S->next_stream++;
  return MQP_OK;
}

int mqp_server_submit(mqp_server* S, int32_t stream_id, const void* frame, uint64_t* request_id) {
  if (!S || !frame || !request_id) return srv_fail(S, MQP_ERR_INVALID, "null argument");
  SrvRequest r;
  size_t frame_bytes = 0;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto f = S->streams.find(stream_id);
    if (f == S->streams.end()) return srv_fail(S, MQP_ERR_NOT_FOUND, "unknown stream " + std::to_string(stream_id));
    const SrvStream& st = f->second;
    frame_bytes = st.frame_bytes;
    r.vf_n = (size_t)std::max<int64_t>(st.pb.n_ia, 1) * st.ndims;
    r.sn_n = st.p.computeSN ? (size_t)std::max<int64_t>(st.pb.n_ia, 1) : 0;
    r.staging = f->second.stage.take();
  }
  // a pinned allocation (all staging buffers in flight) and the frame copy
  // run without the lock, so the worker keeps admitting and completing
  if (!r.staging) {
    void* h = nullptr;
    if (cudaMallocHost(&h, frame_bytes) != cudaSuccess) return srv_fail(S, MQP_ERR_OOM, "pinned staging");
    r.staging = h;
    std::lock_guard<std::mutex> lk(S->mu);
    auto f = S->streams.find(stream_id);
    if (f == S->streams.end()) {
      cudaFreeHost(h);
      return srv_fail(S, MQP_ERR_NOT_FOUND, "unknown stream " + std::to_string(stream_id));
    }
    f->second.stage.add(h, true);
  }
  memcpy(r.staging, frame, frame_bytes);
  std::lock_guard<std::mutex> lk(S->mu);
  auto f = S->streams.find(stream_id);
  if (f == S->streams.end()) {
    return srv_fail(S, MQP_ERR_NOT_FOUND, "unknown stream " + std::to_string(stream_id));
  }
  SrvStream& st = f->second;
  r.id = S->next_req++;
  r.stream = stream_id;
  r.k = ++st.submitted;
  r.t_submit = now_ms();
  if (S->t_first == 0) S->t_first = r.t_submit;
  const uint64_t id = r.id;
  S->reqs[id] = std::move(r);
  S->queue.push_back(id);
  *request_id = id;
  S->cv_work.notify_one();
  return MQP_OK;
}

int mqp_server_result(mqp_server* S, uint64_t request_id, int32_t wait_ms, double* VF, double* SN,
                      double* latency_ms) {
  if (!S) return MQP_ERR_INVALID;
  std::unique_lock<std::mutex> lk(S->mu);
  auto f = S->reqs.find(request_id);
  if (f == S->reqs.end()) return srv_fail(S, MQP_ERR_NOT_FOUND, "unknown request " + std::to_string(request_id));
  if (f->second.state < 2) {
    if (wait_ms == 0) return MQP_ERR_BUSY;
    const auto pred = [S, request_id] { return S->reqs[request_id].state >= 2; };
    if (wait_ms < 0) S->cv_done.wait(lk, pred);
    else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), pred)) return MQP_ERR_TIMEOUT;
  }
  SrvRequest& r = S->reqs[request_id];
  int rc = MQP_OK;
  if (r.state == 3) {
    rc = srv_fail(S, MQP_ERR_CUDA, r.err);
  } else {
    if (VF) memcpy(VF, r.vf.data(), r.vf_n * sizeof(double));
    if (SN && r.sn_n) memcpy(SN, r.sn.data(), r.sn_n * sizeof(double));
    if (latency_ms) *latency_ms = r.t_done - r.t_submit;
  }
  S->reqs.erase(request_id);
  return rc;
}

int mqp_server_get_stats(mqp_server* S, mqp_server_stats* out) {
  if (!S || !out) return MQP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  memset(out, 0, sizeof(*out));
  auto sorted = [](std::vector<double> v) {
    std::sort(v.begin(), v.end());
    return v;
  };
  const std::vector<double> l = sorted(S->lat), lw = sorted(S->lat_wait), lr = sorted(S->lat_run);
  auto pct_of = [](const std::vector<double>& v, double q) {
    return v.empty() ? 0.0 : v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))];
  };
  auto pct = [&](double q) { return pct_of(l, q); };
  out->wait_p50_ms = pct_of(lw, 0.50);
  out->wait_p99_ms = pct_of(lw, 0.99);
  out->run_p50_ms = pct_of(lr, 0.50);
  out->run_p99_ms = pct_of(lr, 0.99);
  out->completed = S->completed;
  out->failed = S->failed;
  out->queued = (int64_t)S->queue.size();
  int running = 0;
  for (auto& sl : S->slots) running += sl.busy;
  out->running = running;
  out->admitted_while_busy = S->admitted_overlap;
  out->p50_ms = pct(0.50);
  out->p99_ms = pct(0.99);
  out->max_ms = l.empty() ? 0.0 : l.back();
  out->ia_done = S->ia_done;
  const double span = S->t_last - S->t_first;
  out->ia_per_s = span > 0 ? S->ia_done / (span / 1e3) : 0.0;
  out->budget_bytes = (int64_t)S->budget;
  out->in_use_bytes = (int64_t)S->in_use;
  return MQP_OK;
}

int mqp_server_reset_stats(mqp_server* S) {
  if (!S) return MQP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  S->lat.clear();
  S->lat_wait.clear();
  S->lat_run.clear();
  S->trace.clear();
  S->ia_done = 0;
  S->completed = 0;
  S->failed = 0;
  S->admitted_overlap = 0;
  S->t_first = 0;
  S->t_last = 0;
  return MQP_OK;
}

int mqp_server_destroy(mqp_server* S) {
  if (!S) return MQP_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  if (!S->trace_path.empty()) {
    if (FILE* f = fopen(S->trace_path.c_str(), "w")) {
      fprintf(f, "request,stream,frame,slot,state,t_submit_ms,t_issue_ms,t_done_ms\n");
      const double t0 = S->trace.empty() ? 0.0 : S->trace.front().t_submit;
      for (const auto& t : S->trace)
        fprintf(f, "%llu,%d,%lld,%d,%d,%.3f,%.3f,%.3f\n", (unsigned long long)t.id, t.stream, (long long)t.k, t.slot,
                t.state, t.t_submit - t0, t.t_issue - t0, t.t_done - t0);
      fclose(f);
    }
  }
  cudaSetDevice(S->device);
  for (auto& sl : S->slots) {
    if (sl.s) cudaStreamSynchronize(sl.s);
    if (sl.s) cudaStreamDestroy(sl.s);
    if (sl.done) cudaEventDestroy(sl.done);
  }
  for (auto& kv : S->streams) {
    SrvStream& st = kv.second;
    for (int i = 0; i < RING; ++i) {
      if (st.frames[i]) cudaFree(st.frames[i]);
      if (st.ii[i]) cudaFree(st.ii[i]);
      if (st.ready[i]) cudaEventDestroy(st.ready[i]);
    }
    st.stage.release();
    st.res.release();
  }
  delete S;
  return MQP_OK;
}

}  // extern "C"
