// sm_100a kernels of the 2D team variant (mqp_piv2d_team.cuh): one IA per
// team of N threads, TEAMS teams per block, persistent over the IAs of one
// launch or of a batch work queue.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include <string>

#include "mqp_internal.h"
#include "mqp_piv2d_team.cuh"

namespace mqp {

namespace {

// Barrier over the N threads of one team (named barrier 1 + team; one warp
// needs only __syncwarp).
template <int N>
__device__ __forceinline__ void team_sync(int team) {
  if constexpr (N == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(N) : "memory");
  }
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ double wnmax(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = nmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double wmax(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ void wpeak(double& best, int& bidx) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bidx, off);
    peak_merge(best, bidx, ob, oi);
  }
}

// Team scratch (doubles): [0..3] the warps' skip maxima and sums of squares,
// [4..11] the warps' peak and SN partials, [12] sumF2, [13] meanG; the last
// double of the largest workspace is the batch queue head.
constexpr int SCR_SUMF2 = 12, SCR_MEANG = 13;

// The finish of one IA (after phase 3): FP64 similarity plane (into the dead
// G region), first full-overlap peak, SN and the Gaussian fit.  The IA's
// geometry is recomputed here rather than kept live through phases 2 and 3.
template <int N, int ALG, typename Sync>
__device__ __forceinline__ void piv2d_team_finish(const Piv2dArgs& a, long long ia, double* scr, double* plane,
                                                  const float* cc, int tid, Sync sync) {
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const int warp = tid >> 5, lane = tid & 31;
  const int v1 = (int)(ia % a.vf1), v2 = (int)(ia / a.vf1);
  int d1, d2;
  ia_pred(a, v1, v2, d1, d2);
  const IAGeom g = ia_geom(a, v1, v2);
  const long long vfo = (long long)v1 + (long long)a.vf1 * v2;
  IAScalars sc;
  sc.sumF2 = scr[SCR_SUMF2];
  sc.meanG = scr[SCR_MEANG];
  sc.meanF = 0.0;
  LagRanges R;
  R.lo1 = g.tlf1;
  R.hi1 = 2 * a.SM1 - g.brb1;
  R.lo2 = g.tlf2;
  R.hi2 = 2 * a.SM2 - g.brb2;
  R.shi1 = 2 * a.SM1 - 1 - g.brb1;
  R.shi2 = 2 * a.SM2 - 1 - g.brb2;
  PeakAcc acc;
  acc.best = 0.0;
  acc.bidx = -1;
  acc.smax = -INFINITY;
  acc.ssum = 0.0;
  const float sqF = sqrtf((float)sc.sumF2);
  const int nl = P1 * P2;
  double* pdst = a.planes ? a.planes + (ia - a.ia_begin) * (long long)nl : nullptr;
#pragma unroll 1
  for (int l0 = tid; l0 < nl; l0 += 4 * N) {
    // four lags' integral-image lookups in flight together
    double v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int l = l0 + k * N;
      v[k] = 0.0;
      if (l < nl) v[k] = team_similarity<ALG>(a, g, sc, sqF, l % P1, l / P1, (double)cc[l]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int l = l0 + k * N;
      if (l < nl) {
        const int s1 = l % P1, s2 = l / P1;
        plane[s1 * P2 + s2] = v[k];
        acc_take(acc, R, s1, s2, P1, v[k]);
        if (pdst) pdst[l] = v[k];
      }
    }
  }
  double best = acc.best;
  int bidx = acc.bidx;
  wpeak(best, bidx);
  double smax = wnmax(acc.smax), ssum = wsum(acc.ssum);
  if (N > 32) {
    // the warps' partials, merged in warp order: (best, index, SN max, SN sum)
    if (lane == 0) {
      scr[4 + 4 * warp] = best;
      scr[5 + 4 * warp] = (double)bidx;
      scr[6 + 4 * warp] = smax;
      scr[7 + 4 * warp] = ssum;
    }
    sync();
    best = scr[4];
    bidx = (int)scr[5];
    smax = scr[6];
    ssum = scr[7];
    peak_merge(best, bidx, scr[8], (int)scr[9]);
    smax = nmax(smax, scr[10]);
    ssum = ssum + scr[11];
  } else {
    sync();
  }
  if (warp == 0) {
    double r1 = -1.0, r2 = -1.0;  // no peak: 1-based (0, 0), displacement -(SM+1)
    if (bidx >= 0) refine2d_warp(plane, P2, a.SM1, a.SM2, g, bidx % P1, bidx / P1, best, lane, r1, r2);
    if (lane == 0) {
      a.VF[2 * vfo + 0] = r1 - a.SM1 + d1;
      a.VF[2 * vfo + 1] = r2 - a.SM2 + d2;
      if (a.SN) {
        // compute_SN (src/utils/piv_ops.jl:336-367) over [TLF_off, 2SM-1-BRB_off]
        const double len = (double)(R.shi1 - R.lo1 + 1) * (double)(R.shi2 - R.lo2 + 1);
        a.SN[vfo] = smax / ((ssum - smax) / (len - 1.0));
      }
    }
  }
  sync();  // the plane and the scratch are reused by the next IA
}

// The per-IA body for one team (tid = thread within the team).
template <int N, int ALG, typename T>
__device__ __forceinline__ void piv2d_team_ia(const Piv2dArgs& a, long long ia, float2* base, const float2* tw,
                                              int team, int tid) {
  using L = TeamLayout<N>;
  constexpr int M = N / 2;
  constexpr bool ZN = ALG == ALG_ZNCC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  float2* G = base;
  float2* F = base + L::g_f2(P1, P2);
  double* scr = reinterpret_cast<double*>(F + L::f_f2(P1, P2));
  const int warp = tid >> 5, lane = tid & 31;
  auto sync = [team]() { team_sync<N>(team); };

  const IAGeom g = ia_geom(a, (int)(ia % a.vf1), (int)(ia / a.vf1));
  IAScalars sc;
  sc.meanF = 0.0;
  sc.meanG = 0.0;
  if (ZN) {
    // copy_*_minus_mean! (src/utils/zncc_ops.jl:7-25)
    sc.meanF = box_sum(a.II1, a.H, g.ir1, g.ir1 + a.IS1, g.ir2, g.ir2 + a.IS2) / ((double)a.IS1 * a.IS2);
    const double nG = (double)(g.hi1 - g.lo1) * (double)(g.hi2 - g.lo2);
    sc.meanG = box_sum(a.IIg, a.H, g.g01 + g.lo1, g.g01 + g.hi1, g.g02 + g.lo2, g.g02 + g.hi2) / nG;
  }

  // ---- phase 1: F rows (thread pairs, half warp-uniform at N = 64), G rows ----
  double vmax = -INFINITY, sumsq = 0.0;
  {
    team_f_row<N, T, ZN>(a, g, sc.meanF, tid % M, tid / M, F, vmax, sumsq);
  }
  team_g_row<N, T, ZN>(a, g, (float)sc.meanG, tid, G);
  // skip_inter_region (src/utils/piv_ops.jl:134-157) needs the IA maximum
  vmax = wmax(vmax);
  sumsq = wsum(sumsq);
  if (N > 32) {
    if (lane == 0) {
      scr[2 * warp] = vmax;
      scr[2 * warp + 1] = sumsq;
    }
    sync();
    vmax = fmax(scr[0], scr[2]);
    sumsq = scr[1] + scr[3];
  } else {
    sync();
  }
  const bool skip = a.threshold >= 0.0 && vmax < a.threshold;
  if (skip) {
    const long long vfo = ia;  // the IA's linear index is its vector-field offset
    if (tid == 0) {
      a.VF[2 * vfo + 0] = 0.0;
      a.VF[2 * vfo + 1] = 0.0;
      if (a.SN) a.SN[vfo] = 0.0;
    }
    if (a.planes) {
      double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
      for (int i = tid; i < P1 * P2; i += N) dst[i] = 0.0;
    }
    sync();  // the scratch is reused by the next IA
    return;
  }
  // Phases 2 and 3 need every register they can get, so the IA's geometry
  // and scalars are not kept live across them: the scalars wait in the team
  // scratch (no one reads these slots before the barriers of phase 2), and
  // the finish recomputes the geometry from an index the compiler cannot see
  // through.
  if (tid == 0) {
    scr[SCR_SUMF2] = sumsq;
    scr[SCR_MEANG] = sc.meanG;
  }
  asm volatile("" : "+l"(ia));

  // ---- phase 2: spectrum columns, thread pair (u, half) ----
  {
    team_phase2<N>(tid % M, tid / M, G, F, sync);
  }
  sync();

  // ---- phase 3: lag rows (thread pairs), raw correlation to cc (FP32) ----
  float* cc = reinterpret_cast<float*>(F);
  {
    const float scale = (float)cc_scale<N>();
    const bool tail = P1 == M + 1;  // row M alone after one round of pairs
    const int paired = tail ? P1 - 1 : P1;
    const int hh = tid / M, j = tid % M;
    for (int b = 0; b < paired; b += M) {
      const int s1 = b + j;
      if (s1 < paired) team_phase3_row<N>(s1, hh, P1, P2, G, cc, scale);
    }
    if (tail) {
      for (int s2 = tid; s2 < P2; s2 += N) cc[(P1 - 1) + P1 * s2] = team_tail_value<N>(G, tw, s2) * scale;
    }
  }
  sync();

  // ---- finish: similarity plane, peak, SN ----
  piv2d_team_finish<N, ALG>(a, ia, scr, reinterpret_cast<double*>(G), cc, tid, sync);
}

template <int N>
__device__ __forceinline__ void load_twiddles(float2* tw) {
  for (int j = threadIdx.x; j < N; j += blockDim.x) tw[j] = twiddle_rt(j * (TW_N / N));
  __syncthreads();
}

template <int N, int ALG, typename T, int TEAMS, int MINB>
__global__ void __launch_bounds__(TEAMS * N, MINB) piv2d_team_kernel(Piv2dArgs a) {
  extern __shared__ float2 smem[];
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const int team = threadIdx.x / N, tid = threadIdx.x % N;
  float2* tw = smem;
  float2* base = smem + N + (size_t)team * TeamLayout<N>::team_f2(P1, P2);
  load_twiddles<N>(tw);
  const long long nteams = (long long)gridDim.x * TEAMS;
  for (long long ia = a.ia_begin + (long long)blockIdx.x * TEAMS + team; ia < a.ia_end; ia += nteams)
    piv2d_team_ia<N, ALG, T>(a, ia, base, tw, team, tid);
}

// Batched: teams take `grab` consecutive entries of the work queue [0, total)
// at a time (see piv2d_batch_kernel); tf2 = float2 per team, the largest any
// item needs.
template <int N, int ALG, typename T, int TEAMS, int MINB>
__global__ void __launch_bounds__(TEAMS * N, MINB)
    piv2d_team_batch_kernel(const Piv2dArgs* __restrict__ items, const long long* __restrict__ prefix, int n_items,
                            long long total, int tf2, int grab, unsigned long long* counter) {
  extern __shared__ float2 smem[];
  const int team = threadIdx.x / N, tid = threadIdx.x % N;
  float2* tw = smem;
  float2* base = smem + N + (size_t)team * tf2;
  // queue head: the last double of the team's workspace (past every item's
  // own scratch slots)
  unsigned long long* head = reinterpret_cast<unsigned long long*>(base + tf2) - 1;
  load_twiddles<N>(tw);
  for (;;) {
    if (tid == 0) *head = atomicAdd(counter, (unsigned long long)grab);
    team_sync<N>(team);
    const unsigned long long g0 = *head;
    team_sync<N>(team);
    if ((long long)g0 >= total) break;
    for (int t = 0; t < grab; ++t) {
      const long long gi = (long long)g0 + t;
      if (gi >= total) break;
      int lo = 0, hi = n_items - 1;  // last k with prefix[k] <= gi
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= gi) lo = mid;
        else hi = mid - 1;
      }
      const Piv2dArgs& a = items[lo];
      piv2d_team_ia<N, ALG, T>(a, a.ia_begin + (gi - prefix[lo]), base, tw, team, tid);
    }
  }
}

template <int N>
struct TeamCfg;
// length 64: two teams (four warps, ~50 KB) per block, four blocks per SM
// (128 registers); three teams at three blocks (96 registers) spill
template <>
struct TeamCfg<64> {
  static constexpr int TEAMS = 2, MINB = 4;
};
// length 32: eight one-warp teams per block
template <>
struct TeamCfg<32> {
  static constexpr int TEAMS = 8, MINB = 3;
};

template <typename K>
cudaError_t grid_for(K kern, int threads, size_t smem, long long work, long long per_block, long long& blocks,
                     std::string& err) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return e;
  }
  int dev = 0, per_sm = 0;
  cudaGetDevice(&dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess || per_sm < 1) {
    err = "piv2d team kernel does not fit on an SM (shared memory " + std::to_string(smem) + " B)";
    return e != cudaSuccess ? e : cudaErrorInvalidConfiguration;
  }
  blocks = (long long)device_sm_count(dev) * per_sm;
  const long long need = (work + per_block - 1) / per_block;
  if (blocks > need) blocks = need;
  return cudaSuccess;
}

template <int N, int ALG, typename T>
cudaError_t launch_team_t(const Piv2dArgs& a, cudaStream_t s, std::string& err) {
  constexpr int TEAMS = TeamCfg<N>::TEAMS, MINB = TeamCfg<N>::MINB;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const size_t smem = ((size_t)N + (size_t)TEAMS * TeamLayout<N>::team_f2(P1, P2)) * sizeof(float2);
  auto kern = piv2d_team_kernel<N, ALG, T, TEAMS, MINB>;
  long long blocks = 0;
  cudaError_t e = grid_for(kern, TEAMS * N, smem, a.ia_end - a.ia_begin, TEAMS, blocks, err);
  if (e != cudaSuccess || blocks < 1) return e;
  kern<<<(unsigned)blocks, TEAMS * N, smem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("piv2d team launch: ") + cudaGetErrorString(e);
  return e;
}

template <int N, int ALG, typename T>
cudaError_t launch_team_batch_t(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  constexpr int TEAMS = TeamCfg<N>::TEAMS, MINB = TeamCfg<N>::MINB;
  const size_t smem = ((size_t)N + (size_t)TEAMS * b.wf2) * sizeof(float2);
  auto kern = piv2d_team_batch_kernel<N, ALG, T, TEAMS, MINB>;
  long long blocks = 0;
  cudaError_t e = grid_for(kern, TEAMS * N, smem, b.total, TEAMS, blocks, err);
  if (e != cudaSuccess || blocks < 1) return e;
  if ((e = cudaMemsetAsync(b.counter, 0, sizeof(unsigned long long), s)) != cudaSuccess) {
    err = std::string("counter reset: ") + cudaGetErrorString(e);
    return e;
  }
  kern<<<(unsigned)blocks, TEAMS * N, smem, s>>>(b.items, b.prefix, b.n_items, b.total, b.wf2,
                                                 b.grab > 0 ? b.grab : 1, b.counter);
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("piv2d team batch launch: ") + cudaGetErrorString(e);
  return e;
}

template <int N, typename T>
cudaError_t launch_team_alg(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  switch (alg) {
    case ALG_FFTCC: return launch_team_t<N, ALG_FFTCC, T>(a, s, err);
    case ALG_ZNCC: return launch_team_t<N, ALG_ZNCC, T>(a, s, err);
    case ALG_NSQECC: return launch_team_t<N, ALG_NSQECC, T>(a, s, err);
    default: err = "team kernel: unsupported correlation algorithm"; return cudaErrorInvalidValue;
  }
}

template <int N, typename T>
cudaError_t launch_team_batch_alg(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  switch (b.alg) {
    case ALG_FFTCC: return launch_team_batch_t<N, ALG_FFTCC, T>(b, s, err);
    case ALG_ZNCC: return launch_team_batch_t<N, ALG_ZNCC, T>(b, s, err);
    case ALG_NSQECC: return launch_team_batch_t<N, ALG_NSQECC, T>(b, s, err);
    default: err = "team kernel: unsupported correlation algorithm"; return cudaErrorInvalidValue;
  }
}

}  // namespace

bool piv2d_team_ok(int N, bool prune, int alg) {
  // Opt-in (MQP_TUNE_PIV2D_TEAM=1): on the 2048^2 workload the one-warp-per-IA
  // kernel is still faster (2.31 ms against 2.51 ms for two 64-thread teams
  // per block at 128 registers, 2.62 ms for three at 167, 3.58 ms for three
  // at 96 with spills).
  static const bool team = [] {
    const char* v = getenv("MQP_TUNE_PIV2D_TEAM");
    return v && v[0] == '1';
  }();
  return team && (N == 32 || N == 64) && prune && (alg == ALG_FFTCC || alg == ALG_ZNCC || alg == ALG_NSQECC);
}

int piv2d_team_f2(int N, int P1, int P2) {
  return N == 64 ? TeamLayout<64>::team_f2(P1, P2) : TeamLayout<32>::team_f2(P1, P2);
}

cudaError_t launch_piv2d_team(const Piv2dArgs& a, int N, int alg, cudaStream_t s, std::string& err) {
  if (N == 64) return a.dtype == 0 ? launch_team_alg<64, float>(a, alg, s, err) : launch_team_alg<64, double>(a, alg, s, err);
  return a.dtype == 0 ? launch_team_alg<32, float>(a, alg, s, err) : launch_team_alg<32, double>(a, alg, s, err);
}

cudaError_t launch_piv2d_team_batch(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  if (b.N == 64)
    return b.dtype == 0 ? launch_team_batch_alg<64, float>(b, s, err) : launch_team_batch_alg<64, double>(b, s, err);
  return b.dtype == 0 ? launch_team_batch_alg<32, float>(b, s, err) : launch_team_batch_alg<32, double>(b, s, err);
}

}  // namespace mqp
