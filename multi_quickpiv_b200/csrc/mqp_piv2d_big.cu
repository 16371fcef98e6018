// sm_100a kernels of the 2D path for search windows up to 128 (see
// mqp_piv2d_big.cuh): one block of 128 threads per interrogation area.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>

#include "mqp_internal.h"
#include "mqp_piv2d_big.cuh"

namespace mqp {

namespace {

__device__ __forceinline__ double bwarp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ double bwarp_max(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double bwarp_nmax(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = nmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

// One IA; every thread of the block takes part.  sm: the block's workspace
// (LayBig, sized for this IA's lag plane), red: its last LayBig::RED_F2 slots
// (16 doubles: four per warp for the block reductions).
template <bool FPRUNE, int ALG, typename T>
__device__ __forceinline__ void piv2d_big_ia(const Piv2dArgs& a, long long ia, float2* sm, double* red) {
  using L = LayBig<FPRUNE>;
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  float2* S = sm + L::S_OFF;
  float2* SF = sm + L::F_OFF;
  double* plane = reinterpret_cast<double*>(SF);
  float* c1buf = MASKED ? reinterpret_cast<float*>(SF + L::region2(P1, P2)) : nullptr;
  float2* PK = sm + L::pk_off(P1, P2, MASKED);
  const int v1 = (int)(ia % a.vf1), v2 = (int)(ia / a.vf1);
  int d1, d2;
  ia_pred(a, v1, v2, d1, d2);
  const IAGeom g = ia_geom(a, v1, v2);
  IAScalars sc;
  sc.meanF = 0.0;
  sc.meanG = 0.0;
  sc.sumF2 = 0.0;
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
    big_rows<FPRUNE, T, ALG>(a, g, sc, PASS, t, S, SF, vmax, mmax, sumsq);
    if (pass == 0) {
      vmax = bwarp_max(vmax);
      mmax = bwarp_max(mmax);
      sumsq = bwarp_sum(sumsq);
      if (lane == 0) {
        red[warp] = vmax;
        red[4 + warp] = mmax;
        red[8 + warp] = sumsq;
      }
      __syncthreads();
      vmax = fmax(fmax(red[0], red[1]), fmax(red[2], red[3]));
      mmax = fmax(fmax(red[4], red[5]), fmax(red[6], red[7]));
      sc.sumF2 = ((red[8] + red[9]) + red[10]) + red[11];
      // skip_inter_region (src/utils/piv_ops.jl:134-157): the vector stays zero
      const bool skip = MASKED ? ((a.threshold > 0.0 && vmax < a.threshold) ||
                                  (a.mask_threshold > 0.0 && mmax < a.mask_threshold))
                               : (a.threshold >= 0.0 && vmax < a.threshold);
      if (skip) {
        if (t == 0) {
          a.VF[2 * vfo + 0] = 0.0;
          a.VF[2 * vfo + 1] = 0.0;
          if (a.SN) a.SN[vfo] = 0.0;
        }
        if (a.planes) {
          double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
          for (int i = t; i < P1 * P2; i += BIG_THREADS) dst[i] = 0.0;
        }
        __syncthreads();
        return;
      }
    } else {
      __syncthreads();
    }
    big_columns<FPRUNE>(t, P1, S, SF, PK);
    __syncthreads();
    big_lag_row<FPRUNE>(t, P1, P2, S, plane);
    __syncthreads();
    if (MASKED && pass == 0) {
      // park (F*mask)*G while the second pass reuses the workspace
      for (int i = t; i < P1 * P2; i += BIG_THREADS) c1buf[i] = (float)plane[i];
      __syncthreads();
    }
  }
  // ---- finish: similarity, peak (first_fullovp_peak), SN, Gaussian fit ----
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
  if (t < P1) finish_row<ALG>(a, g, sc, t, P1, P2, plane + (long long)t * P2, R, acc, MASKED ? c1buf + t * P2 : nullptr);
  double best = acc.best;
  int bidx = acc.bidx;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bidx, off);
    peak_merge(best, bidx, ob, oi);
  }
  const double smax = bwarp_nmax(acc.smax);
  const double ssum = bwarp_sum(acc.ssum);
  __syncthreads();  // red[] reuse; the plane is complete
  if (lane == 0) {
    red[warp] = best;
    red[4 + warp] = (double)bidx;
    red[8 + warp] = smax;
    red[12 + warp] = ssum;
  }
  __syncthreads();
  if (a.planes) {
    double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
    for (int i = t; i < P1 * P2; i += BIG_THREADS) dst[i] = plane[(i % P1) * P2 + i / P1];
  }
  if (t == 0) {
    double b = red[0], mx = red[8], sum = red[12];
    int bi = (int)red[4];
    for (int w = 1; w < 4; ++w) {
      peak_merge(b, bi, red[w], (int)red[4 + w]);
      mx = nmax(mx, red[8 + w]);
      sum += red[12 + w];
    }
    double r1, r2;
    if (bi < 0) {
      r1 = -1.0;  // 1-based peak (0, 0): displacement -(SM+1)
      r2 = -1.0;
    } else {
      refine2d(plane, P2, a.SM1, a.SM2, g, bi % P1, bi / P1, b, r1, r2);
    }
    a.VF[2 * vfo + 0] = r1 - a.SM1 + d1;
    a.VF[2 * vfo + 1] = r2 - a.SM2 + d2;
    if (a.SN) {
      // compute_SN (src/utils/piv_ops.jl:336-367) over [TLF_off, 2SM-1-BRB_off]
      const double len = (double)(R.shi1 - R.lo1 + 1) * (double)(R.shi2 - R.lo2 + 1);
      a.SN[vfo] = mx / ((sum - mx) / (len - 1.0));
    }
  }
  __syncthreads();
}

// Persistent over the IAs of one pair; wsz = the block's workspace (float2),
// whose last LayBig::RED_F2 slots are the reduction scratch.
template <bool FPRUNE, int ALG, typename T>
__global__ void __launch_bounds__(BIG_THREADS) piv2d_big_kernel(Piv2dArgs a, int wsz) {
  extern __shared__ float2 smem[];
  double* red = reinterpret_cast<double*>(smem + wsz - LayBig<FPRUNE>::RED_F2);
  for (long long ia = a.ia_begin + blockIdx.x; ia < a.ia_end; ia += gridDim.x) piv2d_big_ia<FPRUNE, ALG, T>(a, ia, smem, red);
}

// Batched: blocks take `grab` IAs at a time from one queue over many pairs
// (prefix[k] = first queue index of pair k).
template <bool FPRUNE, int ALG, typename T>
__global__ void __launch_bounds__(BIG_THREADS)
    piv2d_big_batch_kernel(const Piv2dArgs* __restrict__ items, const long long* __restrict__ prefix, int n_items,
                           long long total, int wsz, int grab, unsigned long long* counter) {
  extern __shared__ float2 smem[];
  double* red = reinterpret_cast<double*>(smem + wsz - LayBig<FPRUNE>::RED_F2);
  __shared__ unsigned long long g0s;
  for (;;) {
    if (threadIdx.x == 0) g0s = atomicAdd(counter, (unsigned long long)grab);
    __syncthreads();
    const long long g0 = (long long)g0s;
    __syncthreads();
    if (g0 >= total) break;
    for (int q = 0; q < grab; ++q) {
      const long long gi = g0 + q;
      if (gi >= total) break;
      int lo = 0, hi = n_items - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= gi) lo = mid;
        else hi = mid - 1;
      }
      const Piv2dArgs& a = items[lo];
      piv2d_big_ia<FPRUNE, ALG, T>(a, a.ia_begin + (gi - prefix[lo]), smem, red);
    }
  }
}

template <bool FPRUNE, int ALG, typename T>
cudaError_t big_launch(const Piv2dArgs* single, const Piv2dBatch* batch, cudaStream_t s, std::string& err) {
  const int wsz = single ? LayBig<FPRUNE>::total_f2(2 * single->SM1 + 1, 2 * single->SM2 + 1, ALG == ALG_MASK_NSQECC)
                         : batch->wf2;
  const size_t smem = (size_t)wsz * sizeof(float2);
  const void* kern = single ? (const void*)piv2d_big_kernel<FPRUNE, ALG, T>
                            : (const void*)piv2d_big_batch_kernel<FPRUNE, ALG, T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return e;
  }
  int dev = 0, per_sm = 0;
  cudaGetDevice(&dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BIG_THREADS, smem);
  if (e != cudaSuccess || per_sm < 1) {
    err = "piv2d (128) kernel does not fit on an SM (shared memory " + std::to_string(smem) + " B)";
    return e != cudaSuccess ? e : cudaErrorInvalidConfiguration;
  }
  long long blocks = (long long)device_sm_count(dev) * per_sm;
  const long long need = single ? single->ia_end - single->ia_begin : batch->total;
  if (blocks > need) blocks = need;
  if (blocks < 1) return cudaSuccess;
  if (single) {
    piv2d_big_kernel<FPRUNE, ALG, T><<<(unsigned)blocks, BIG_THREADS, smem, s>>>(*single, wsz);
  } else {
    if ((e = cudaMemsetAsync(batch->counter, 0, sizeof(unsigned long long), s)) != cudaSuccess) {
      err = std::string("counter reset: ") + cudaGetErrorString(e);
      return e;
    }
    piv2d_big_batch_kernel<FPRUNE, ALG, T><<<(unsigned)blocks, BIG_THREADS, smem, s>>>(
        batch->items, batch->prefix, batch->n_items, batch->total, wsz, batch->grab > 0 ? batch->grab : 1,
        batch->counter);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("piv2d (128) launch: ") + cudaGetErrorString(e);
  return e;
}

template <bool FPRUNE, typename T>
cudaError_t big_alg(int alg, const Piv2dArgs* single, const Piv2dBatch* batch, cudaStream_t s, std::string& err) {
  switch (alg) {
    case ALG_FFTCC: return big_launch<FPRUNE, ALG_FFTCC, T>(single, batch, s, err);
    case ALG_ZNCC: return big_launch<FPRUNE, ALG_ZNCC, T>(single, batch, s, err);
    case ALG_NSQECC: return big_launch<FPRUNE, ALG_NSQECC, T>(single, batch, s, err);
    case ALG_MASK_NSQECC: return big_launch<FPRUNE, ALG_MASK_NSQECC, T>(single, batch, s, err);
    default: err = "unknown correlation algorithm"; return cudaErrorInvalidValue;
  }
}

cudaError_t big_dispatch(bool prune, int dtype, int alg, const Piv2dArgs* single, const Piv2dBatch* batch,
                         cudaStream_t s, std::string& err) {
  if (prune)
    return dtype == 0 ? big_alg<true, float>(alg, single, batch, s, err) : big_alg<true, double>(alg, single, batch, s, err);
  return dtype == 0 ? big_alg<false, float>(alg, single, batch, s, err) : big_alg<false, double>(alg, single, batch, s, err);
}

}  // namespace

int piv2d_big_warp_f2(bool prune, int P1, int P2, bool masked) { return piv2d_big_smem_f2(prune, P1, P2, masked); }

cudaError_t launch_piv2d_big(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  const bool prune = a.IS1 <= MB && a.IS2 <= MB;
  return big_dispatch(prune, a.dtype, alg, &a, nullptr, s, err);
}

cudaError_t launch_piv2d_big_batch(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  if (b.total <= 0 || b.n_items <= 0) return cudaSuccess;
  return big_dispatch(b.prune, b.dtype, b.alg, nullptr, &b, s, err);
}

}  // namespace mqp
