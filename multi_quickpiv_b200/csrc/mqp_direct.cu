// sm_100a kernels of the direct (spatial) correlation for small windows, 2D
// and 3D (see mqp_direct.cuh): one warp per interrogation area, or for the
// 3D shapes of the register-tiled lag loop one block per interrogation area.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "mqp_direct.cuh"
#include "mqp_internal.h"

namespace mqp {

namespace {

constexpr int DWARPS = 4;

__device__ __forceinline__ double dsum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ double dmax(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double dnmax(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = nmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ void dpeak(double& best, int& bidx) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bidx, off);
    peak_merge(best, bidx, ob, oi);
  }
}

// ---- 2D: one IA per warp -----------------------------------------------------
template <int ALG, typename T>
__device__ __forceinline__ void direct2d_ia(const Piv2dArgs& a, long long ia, float* ws, int lane) {
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const D2Off o = d2_off(a.IS1, a.IS2, a.SM1, a.SM2);
  float* F = ws + o.F;
  float* G = ws + o.G;
  double* plane = reinterpret_cast<double*>(ws + o.plane);
  float* c1 = ws + o.c1;
  const int v1 = (int)(ia % a.vf1), v2 = (int)(ia / a.vf1);
  int d1, d2;
  ia_pred(a, v1, v2, d1, d2);
  const IAGeom g = ia_geom(a, v1, v2);
  IAScalars sc;
  sc.meanF = sc.meanG = sc.sumF2 = 0.0;
  if (ALG == ALG_ZNCC) {
    // copy_*_minus_mean! (src/utils/zncc_ops.jl:7-25)
    sc.meanF = box_sum(a.II1, a.H, g.ir1, g.ir1 + a.IS1, g.ir2, g.ir2 + a.IS2) / ((double)a.IS1 * a.IS2);
    const double nG = (double)(g.hi1 - g.lo1) * (double)(g.hi2 - g.lo2);
    sc.meanG = box_sum(a.IIg, a.H, g.g01 + g.lo1, g.g01 + g.hi1, g.g02 + g.lo2, g.g02 + g.hi2) / nG;
  }
  const long long vfo = (long long)v1 + (long long)a.vf1 * v2;
  constexpr int NPASS = MASKED ? 2 : 1;
  for (int pass = 0; pass < NPASS; ++pass) {
    const int PASS = MASKED ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;
    double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
    direct2d_load<T, ALG>(a, g, sc, PASS, lane, 32, F, G, vmax, mmax, sumsq);
    if (pass == 0) {
      vmax = dmax(vmax);
      mmax = dmax(mmax);
      sc.sumF2 = dsum(sumsq);
      // skip_inter_region (src/utils/piv_ops.jl:134-157): the vector stays zero
      const bool skip = MASKED ? ((a.threshold > 0.0 && vmax < a.threshold) ||
                                  (a.mask_threshold > 0.0 && mmax < a.mask_threshold))
                               : (a.threshold >= 0.0 && vmax < a.threshold);
      if (skip) {
        if (lane == 0) {
          a.VF[2 * vfo] = 0.0;
          a.VF[2 * vfo + 1] = 0.0;
          if (a.SN) a.SN[vfo] = 0.0;
        }
        if (a.planes)
          for (int i = lane; i < P1 * P2; i += 32) a.planes[(ia - a.ia_begin) * (long long)P1 * P2 + i] = 0.0;
        __syncwarp();
        return;
      }
    }
    __syncwarp();
    direct2d_lags(a, lane, 32, F, G, plane);
    __syncwarp();
    if (MASKED && pass == 0) {
      for (int i = lane; i < P1 * P2; i += 32) c1[i] = (float)plane[i];
      __syncwarp();
    }
  }
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
  // similarity of every lag, the lags spread over all lanes (a plane has
  // only 2SM1+1 rows: one row per lane would leave most lanes idle)
  for (int q = lane; q < P1 * P2; q += 32) direct2d_finish_lag<ALG>(a, g, sc, q, P1, P2, plane, c1, R, acc);
  __syncwarp();
  double best = acc.best;
  int bidx = acc.bidx;
  dpeak(best, bidx);
  double sn = 0.0;
  if (a.SN) {
    const double smax = dnmax(acc.smax), ssum = dsum(acc.ssum);
    const double len = (double)(R.shi1 - R.lo1 + 1) * (double)(R.shi2 - R.lo2 + 1);
    sn = smax / ((ssum - smax) / (len - 1.0));
  }
  if (a.planes) {
    double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
    for (int i = lane; i < P1 * P2; i += 32) dst[i] = plane[(i % P1) * P2 + i / P1];
  }
  double r1 = -1.0, r2 = -1.0;
  if (bidx >= 0) refine2d_warp(plane, P2, a.SM1, a.SM2, g, bidx % P1, bidx / P1, best, lane, r1, r2);
  if (lane == 0) {
    a.VF[2 * vfo + 0] = r1 - a.SM1 + d1;
    a.VF[2 * vfo + 1] = r2 - a.SM2 + d2;
    if (a.SN) a.SN[vfo] = sn;
  }
  __syncwarp();
}

template <int ALG, typename T>
// 2D direct kernels: eight blocks (32 warps) per SM for latency hiding (64
// registers; a few bytes of spill for the normalised algorithms)
__global__ void __launch_bounds__(DWARPS * 32, 8) direct2d_kernel(Piv2dArgs a, int words) {
  extern __shared__ float dsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* ws = dsm + (size_t)warp * words;
  const long long nw = (long long)gridDim.x * DWARPS;
  for (long long ia = a.ia_begin + (long long)blockIdx.x * DWARPS + warp; ia < a.ia_end; ia += nw)
    direct2d_ia<ALG, T>(a, ia, ws, lane);
}

template <int ALG, typename T>
__global__ void __launch_bounds__(DWARPS * 32, 8)
    direct2d_batch_kernel(const Piv2dArgs* __restrict__ items, const long long* __restrict__ prefix, int n_items,
                          long long total, int words, int grab, unsigned long long* counter) {
  extern __shared__ float dsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* ws = dsm + (size_t)warp * words;
  for (;;) {
    unsigned long long g0 = 0;
    if (lane == 0) g0 = atomicAdd(counter, (unsigned long long)grab);
    g0 = __shfl_sync(0xffffffffu, g0, 0);
    if ((long long)g0 >= total) break;
    for (int t = 0; t < grab; ++t) {
      const long long gi = (long long)g0 + t;
      if (gi >= total) break;
      int lo = 0, hi = n_items - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= gi) lo = mid;
        else hi = mid - 1;
      }
      const Piv2dArgs& a = items[lo];
      direct2d_ia<ALG, T>(a, a.ia_begin + (gi - prefix[lo]), ws, lane);
    }
  }
}

// ---- 3D: one IA per warp -----------------------------------------------------
template <int ALG, typename T>
__device__ __forceinline__ void direct3d_ia(const Piv3dArgs& a, long long ia, float* ws, int lane) {
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1, P3 = 2 * a.SM[2] + 1;
  const int vol = P1 * P2 * P3;
  const D3Off o = d3_off(a.IS, a.SM);
  float* F = ws + o.F;
  float* G = ws + o.G;
  float* V = ws + o.V;
  float* C1 = ws + o.c1;
  const IAGeom3 g = ia_geom3(a, ia);
  IA3State s;
  ia3_means<ALG>(a, g, s.meanF, s.meanG);
  s.sumF2 = 0.0;
  s.skip = 0;
  constexpr int NPASS = MASKED ? 2 : 1;
  for (int pass = 0; pass < NPASS; ++pass) {
    const int PASS = MASKED ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;
    double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
    direct3d_load<T, ALG>(a, g, s, PASS, lane, 32, F, G, vmax, mmax, sumsq);
    if (pass == 0) {
      vmax = dmax(vmax);
      mmax = dmax(mmax);
      s.sumF2 = dsum(sumsq);
      if (skip_test3(a, ALG, vmax, mmax)) {
        if (lane == 0) {
          for (int d = 0; d < 3; ++d) a.VF[3 * ia + d] = 0.0;
          if (a.SN) a.SN[ia] = 0.0;
        }
        if (a.planes)
          for (int i = lane; i < vol; i += 32) a.planes[(ia - a.planes_begin) * (long long)vol + i] = 0.0;
        __syncwarp();
        return;
      }
    }
    __syncwarp();
    direct3d_lags(a, lane, 32, F, G, V);
    __syncwarp();
    if (MASKED && pass == 0) {
      for (int i = lane; i < vol; i += 32) C1[i] = V[i];
      __syncwarp();
    }
  }
  const LagRanges3 R = lag_ranges3(a, g);
  PeakAcc acc;
  acc.best = 0.0;
  acc.bidx = -1;
  acc.smax = -INFINITY;
  acc.ssum = 0.0;
  for (int q = lane; q < vol; q += 32) {
    const double c = MASKED ? (double)C1[q] : (double)V[q];
    const double c2 = MASKED ? (double)V[q] : 0.0;
    const double v = direct3d_sim<ALG>(a, g, s, q, c, c2);
    V[q] = (float)v;
    if (a.planes) a.planes[(ia - a.planes_begin) * (long long)vol + q] = v;
    acc_take3(acc, R, q % P1, (q / P1) % P2, q / (P1 * P2), q, v);
  }
  __syncwarp();
  double best = acc.best;
  int bidx = acc.bidx;
  dpeak(best, bidx);
  const double smax = dnmax(acc.smax), ssum = dsum(acc.ssum);
  if (lane == 0) direct3d_final(a, g, ia, R, V, best, bidx, smax, ssum);
  __syncwarp();
}

template <int ALG, typename T>
__global__ void __launch_bounds__(DWARPS * 32) direct3d_kernel(Piv3dArgs a, int words) {
  extern __shared__ float dsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* ws = dsm + (size_t)warp * words;
  const long long nw = (long long)gridDim.x * DWARPS;
  for (long long ia = a.ia_begin + (long long)blockIdx.x * DWARPS + warp; ia < a.ia_end; ia += nw)
    direct3d_ia<ALG, T>(a, ia, ws, lane);
}

// ---- 3D, register-tiled lags: one block per IA ------------------------------
constexpr int D3T_MAXT = 256;  // threads of a block (P1 P3 tasks, rounded up to warps)
constexpr int D3T_RED = 4 * (D3T_MAXT / 32) * 2 + D3T_MAXT / 32;  // reduction words

// Block-wide reductions in a fixed warp order (every thread gets the result).
__device__ __forceinline__ void block_max_max_sum(double& a, double& b, double& c, double* red, int tid, int nw) {
  a = dmax(a);
  b = dmax(b);
  c = dsum(c);
  if ((tid & 31) == 0) {
    red[3 * (tid >> 5)] = a;
    red[3 * (tid >> 5) + 1] = b;
    red[3 * (tid >> 5) + 2] = c;
  }
  __syncthreads();
  a = red[0];
  b = red[1];
  c = red[2];
  for (int w = 1; w < nw; ++w) {
    a = fmax(a, red[3 * w]);
    b = fmax(b, red[3 * w + 1]);
    c += red[3 * w + 2];
  }
  __syncthreads();
}

__device__ __forceinline__ void block_peak(PeakAcc& acc, double* red, int* redi, int tid, int nw) {
  dpeak(acc.best, acc.bidx);
  acc.smax = dnmax(acc.smax);
  acc.ssum = dsum(acc.ssum);
  if ((tid & 31) == 0) {
    red[3 * (tid >> 5)] = acc.best;
    red[3 * (tid >> 5) + 1] = acc.smax;
    red[3 * (tid >> 5) + 2] = acc.ssum;
    redi[tid >> 5] = acc.bidx;
  }
  __syncthreads();
  acc.best = red[0];
  acc.smax = red[1];
  acc.ssum = red[2];
  acc.bidx = redi[0];
  for (int w = 1; w < nw; ++w) {
    peak_merge(acc.best, acc.bidx, red[3 * w], redi[w]);
    acc.smax = nmax(acc.smax, red[3 * w + 1]);
    acc.ssum += red[3 * w + 2];
  }
  __syncthreads();
}

template <int ALG, typename T, int IS2, int P2>
__device__ __forceinline__ void direct3d_tiled_ia(const Piv3dArgs& a, long long ia, float* ws, double* red, int* redi,
                                                  int tid, int nt) {
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int nw = nt >> 5;
  const int P1 = 2 * a.SM[0] + 1, P3 = 2 * a.SM[2] + 1;
  const int vol = P1 * P2 * P3;
  const D3Off o = d3_off(a.IS, a.SM);
  float* F = ws + o.F;
  float* G = ws + o.G;
  float* V = ws + o.V;
  float* C1 = ws + o.c1;
  const IAGeom3 g = ia_geom3(a, ia);
  IA3State s;
  ia3_means<ALG>(a, g, s.meanF, s.meanG);
  s.sumF2 = 0.0;
  s.skip = 0;
  constexpr int NPASS = MASKED ? 2 : 1;
  for (int pass = 0; pass < NPASS; ++pass) {
    const int PASS = MASKED ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;
    double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
    direct3d_load<T, ALG>(a, g, s, PASS, tid, nt, F, G, vmax, mmax, sumsq, true);
    if (pass == 0) {
      block_max_max_sum(vmax, mmax, sumsq, red, tid, nw);  // also orders the loads before the lags
      s.sumF2 = sumsq;
      if (skip_test3(a, ALG, vmax, mmax)) {
        if (tid == 0) {
          for (int d = 0; d < 3; ++d) a.VF[3 * ia + d] = 0.0;
          if (a.SN) a.SN[ia] = 0.0;
        }
        if (a.planes)
          for (int i = tid; i < vol; i += nt) a.planes[(ia - a.planes_begin) * (long long)vol + i] = 0.0;
        return;
      }
    } else {
      __syncthreads();
    }
    direct3d_lags_tiled<IS2, P2>(a, tid, nt, F, G, V);
    __syncthreads();
    if (MASKED && pass == 0) {
      for (int i = tid; i < vol; i += nt) C1[i] = V[i];
      __syncthreads();
    }
  }
  const LagRanges3 R = lag_ranges3(a, g);
  PeakAcc acc;
  acc.best = 0.0;
  acc.bidx = -1;
  acc.smax = -INFINITY;
  acc.ssum = 0.0;
  for (int q = tid; q < vol; q += nt) {
    const double c = MASKED ? (double)C1[q] : (double)V[q];
    const double c2 = MASKED ? (double)V[q] : 0.0;
    const double v = direct3d_sim<ALG>(a, g, s, q, c, c2);
    V[q] = (float)v;
    if (a.planes) a.planes[(ia - a.planes_begin) * (long long)vol + q] = v;
    acc_take3(acc, R, q % P1, (q / P1) % P2, q / (P1 * P2), q, v);
  }
  block_peak(acc, red, redi, tid, nw);  // its barriers also publish V
  if (tid < 32) {  // warp 0: the fit's seven logs on seven lanes
    double r[3] = {-1.0, -1.0, -1.0};
    if (acc.bidx >= 0) {
      const int p[3] = {acc.bidx % P1, (acc.bidx / P1) % P2, acc.bidx / (P1 * P2)};
      refine3d_warp(V, P1, P2, a.SM, g, p, acc.best, tid, r);
    }
    if (tid == 0) direct3d_final(a, g, ia, R, V, acc.best, acc.bidx, acc.smax, acc.ssum, r);
  }
  __syncthreads();
}

template <int ALG, typename T, int IS2, int P2>
__global__ void __launch_bounds__(D3T_MAXT) direct3d_tiled_kernel(Piv3dArgs a, int words) {
  extern __shared__ float dsm[];
  double* red = reinterpret_cast<double*>(dsm + words);
  int* redi = reinterpret_cast<int*>(red + 3 * (D3T_MAXT / 32));
  for (long long ia = a.ia_begin + blockIdx.x; ia < a.ia_end; ia += gridDim.x)
    direct3d_tiled_ia<ALG, T, IS2, P2>(a, ia, dsm, red, redi, threadIdx.x, blockDim.x);
}

// grid: resident blocks of `kern` with `smem` bytes, at most enough for n warps' work
cudaError_t grid_for(const void* kern, size_t smem, long long n, long long& blocks, std::string& err) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return e;
  }
  int dev = 0, per_sm = 0;
  cudaGetDevice(&dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, DWARPS * 32, smem);
  if (e != cudaSuccess || per_sm < 1) {
    err = "direct correlation kernel does not fit on an SM (shared memory " + std::to_string(smem) + " B)";
    return e != cudaSuccess ? e : cudaErrorInvalidConfiguration;
  }
  blocks = (long long)device_sm_count(dev) * per_sm;
  const long long need = (n + DWARPS - 1) / DWARPS;
  if (blocks > need) blocks = need;
  return cudaSuccess;
}

template <int ALG, typename T>
cudaError_t d2_launch(const Piv2dArgs* single, const Piv2dBatch* batch, cudaStream_t s, std::string& err) {
  const int words = single ? d2_off(single->IS1, single->IS2, single->SM1, single->SM2).words : 2 * batch->wf2;
  const size_t smem = (size_t)DWARPS * words * sizeof(float);
  const void* kern = single ? (const void*)direct2d_kernel<ALG, T> : (const void*)direct2d_batch_kernel<ALG, T>;
  long long blocks = 0;
  cudaError_t e = grid_for(kern, smem, single ? single->ia_end - single->ia_begin : batch->total, blocks, err);
  if (e != cudaSuccess || blocks < 1) return e;
  if (single) {
    direct2d_kernel<ALG, T><<<(unsigned)blocks, DWARPS * 32, smem, s>>>(*single, words);
  } else {
    if ((e = cudaMemsetAsync(batch->counter, 0, sizeof(unsigned long long), s)) != cudaSuccess) {
      err = std::string("counter reset: ") + cudaGetErrorString(e);
      return e;
    }
    direct2d_batch_kernel<ALG, T><<<(unsigned)blocks, DWARPS * 32, smem, s>>>(
        batch->items, batch->prefix, batch->n_items, batch->total, words, batch->grab > 0 ? batch->grab : 1,
        batch->counter);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("direct 2D launch: ") + cudaGetErrorString(e);
  return e;
}

template <typename T>
cudaError_t d2_alg(int alg, const Piv2dArgs* single, const Piv2dBatch* batch, cudaStream_t s, std::string& err) {
  switch (alg) {
    case ALG_FFTCC: return d2_launch<ALG_FFTCC, T>(single, batch, s, err);
    case ALG_ZNCC: return d2_launch<ALG_ZNCC, T>(single, batch, s, err);
    case ALG_NSQECC: return d2_launch<ALG_NSQECC, T>(single, batch, s, err);
    case ALG_MASK_NSQECC: return d2_launch<ALG_MASK_NSQECC, T>(single, batch, s, err);
    default: err = "unknown correlation algorithm"; return cudaErrorInvalidValue;
  }
}

template <int ALG, typename T, int IS2, int P2>
cudaError_t d3t_launch(const Piv3dArgs& a, cudaStream_t s, std::string& err) {
  const int words = d3_off(a.IS, a.SM).words;
  const size_t smem = (size_t)(words + D3T_RED) * sizeof(float);
  const int tasks = (2 * a.SM[0] + 1) * (2 * a.SM[2] + 1);
  const int nt = std::min(D3T_MAXT, (tasks + 31) / 32 * 32);
  const void* kern = (const void*)direct3d_tiled_kernel<ALG, T, IS2, P2>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, per_sm = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem);
  if (e != cudaSuccess || per_sm < 1) {
    err = "direct 3D kernel does not fit on an SM (shared memory " + std::to_string(smem) + " B)";
    return e != cudaSuccess ? e : cudaErrorInvalidConfiguration;
  }
  const long long n = a.ia_end - a.ia_begin;
  const long long blocks = std::min<long long>((long long)device_sm_count(dev) * per_sm, n);
  direct3d_tiled_kernel<ALG, T, IS2, P2><<<(unsigned)blocks, nt, smem, s>>>(a, words);
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("direct 3D launch: ") + cudaGetErrorString(e);
  return e;
}

template <int ALG, typename T>
cudaError_t d3_launch(const Piv3dArgs& a, cudaStream_t s, std::string& err) {
  const int IS2 = a.IS[1], P2 = 2 * a.SM[1] + 1;
#define MQP_D3_GO(i, p) \
  if (IS2 == i && P2 == p) return d3t_launch<ALG, T, i, p>(a, s, err);
  MQP_D3_TILED_SHAPES(MQP_D3_GO)
#undef MQP_D3_GO
  const int words = d3_off(a.IS, a.SM).words;
  const size_t smem = (size_t)DWARPS * words * sizeof(float);
  long long blocks = 0;
  cudaError_t e = grid_for((const void*)direct3d_kernel<ALG, T>, smem, a.ia_end - a.ia_begin, blocks, err);
  if (e != cudaSuccess || blocks < 1) return e;
  direct3d_kernel<ALG, T><<<(unsigned)blocks, DWARPS * 32, smem, s>>>(a, words);
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("direct 3D launch: ") + cudaGetErrorString(e);
  return e;
}

template <typename T>
cudaError_t d3_alg(int alg, const Piv3dArgs& a, cudaStream_t s, std::string& err) {
  switch (alg) {
    case ALG_FFTCC: return d3_launch<ALG_FFTCC, T>(a, s, err);
    case ALG_ZNCC: return d3_launch<ALG_ZNCC, T>(a, s, err);
    case ALG_NSQECC: return d3_launch<ALG_NSQECC, T>(a, s, err);
    case ALG_MASK_NSQECC: return d3_launch<ALG_MASK_NSQECC, T>(a, s, err);
    default: err = "unknown correlation algorithm"; return cudaErrorInvalidValue;
  }
}

}  // namespace

int piv2d_direct_words(int IS1, int IS2, int SM1, int SM2) { return d2_off(IS1, IS2, SM1, SM2).words; }

cudaError_t launch_piv2d_direct(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  return a.dtype == 0 ? d2_alg<float>(alg, &a, nullptr, s, err) : d2_alg<double>(alg, &a, nullptr, s, err);
}

cudaError_t launch_piv2d_direct_batch(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  if (b.total <= 0 || b.n_items <= 0) return cudaSuccess;
  return b.dtype == 0 ? d2_alg<float>(b.alg, nullptr, &b, s, err) : d2_alg<double>(b.alg, nullptr, &b, s, err);
}

cudaError_t launch_piv3d_direct(const Piv3dArgs& a, int alg, cudaStream_t s, std::string& err) {
  if (a.ia_end <= a.ia_begin) return cudaSuccess;
  return a.dtype == 0 ? d3_alg<float>(alg, a, s, err) : d3_alg<double>(alg, a, s, err);
}

}  // namespace mqp
