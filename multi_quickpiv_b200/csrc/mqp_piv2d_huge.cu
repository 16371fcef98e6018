// sm_100a kernel of the 2D path for search windows of 129..256
// (mqp_piv2d_huge.cuh): one 256-thread block per IA, persistent over the IAs
// of a launch, each block with its own scratch slot.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>

#include "mqp_internal.h"
#include "mqp_piv2d_huge.cuh"

namespace mqp {

namespace {

__device__ __forceinline__ double hsum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ double hnmax(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = nmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double hmax(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ void hpeak(double& best, int& bidx) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bidx, off);
    peak_merge(best, bidx, ob, oi);
  }
}

constexpr int HW = HUGE_THREADS / 32;  // warps per block

template <int ALG, typename T>
__device__ __forceinline__ void huge_ia(const Piv2dArgs& a, long long ia, float2* slot, float2* sm) {
  constexpr bool ZN = ALG == ALG_ZNCC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const HugeSlot L(P1, P2);
  float2* GS = slot + L.gs;
  float2* FS = slot + L.fs;
  float2* LG = slot + L.lg;
  float* cc = reinterpret_cast<float*>(slot + L.cc);
  double* plane = reinterpret_cast<double*>(slot + L.pl);
  float2* park = sm;
  float2* pack = sm + HugeSmem::PARK;
  const float2* tw = pack + HugeSmem::PACK;
  double* red = reinterpret_cast<double*>(sm + HugeSmem::PARK + HugeSmem::PACK + HugeSmem::TW);

  const int v1 = (int)(ia % a.vf1), v2 = (int)(ia / a.vf1);
  int d1, d2;
  ia_pred(a, v1, v2, d1, d2);
  const IAGeom g = ia_geom(a, v1, v2);
  IAScalars sc;
  sc.meanF = 0.0;
  sc.meanG = 0.0;
  if (ZN) {
    // copy_*_minus_mean! (src/utils/zncc_ops.jl:7-25)
    sc.meanF = box_sum(a.II1, a.H, g.ir1, g.ir1 + a.IS1, g.ir2, g.ir2 + a.IS2) / ((double)a.IS1 * a.IS2);
    const double nG = (double)(g.hi1 - g.lo1) * (double)(g.hi2 - g.lo2);
    sc.meanG = box_sum(a.IIg, a.H, g.g01 + g.lo1, g.g01 + g.hi1, g.g02 + g.lo2, g.g02 + g.hi2) / nG;
  }
  const long long vfo = (long long)v1 + (long long)a.vf1 * v2;

  // ---- A: rows ----
  double vmax = -INFINITY, sumsq = 0.0;
  huge_f_row<T, ZN>(a, g, sc.meanF, t % MH, t / MH, FS, vmax, sumsq);
  huge_g_row<T, ZN>(a, g, (float)sc.meanG, t, GS, reinterpret_cast<float*>(park));
  vmax = hmax(vmax);
  sumsq = hsum(sumsq);
  if (lane == 0) {
    red[2 * warp] = vmax;
    red[2 * warp + 1] = sumsq;
  }
  __syncthreads();
  vmax = red[0];
  sumsq = red[1];
  for (int w = 1; w < HW; ++w) {
    vmax = fmax(vmax, red[2 * w]);
    sumsq = sumsq + red[2 * w + 1];
  }
  sc.sumF2 = sumsq;
  __syncthreads();
  // skip_inter_region (src/utils/piv_ops.jl:134-157)
  if (a.threshold >= 0.0 && vmax < a.threshold) {
    if (t == 0) {
      a.VF[2 * vfo + 0] = 0.0;
      a.VF[2 * vfo + 1] = 0.0;
      if (a.SN) a.SN[vfo] = 0.0;
    }
    if (a.planes) {
      double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
      for (int i = t; i < P1 * P2; i += HUGE_THREADS) dst[i] = 0.0;
    }
    return;
  }

  // ---- B: columns, a thread quad per column (quarter q warp-uniform) ----
  for (int r = 0; r < 2; ++r) {
    float2 f[QH];
    huge_b_part1(r, t, GS, FS, tw, park, pack, f);
    __syncthreads();
    huge_b_part2(r, t, tw, park, pack, f);
    __syncthreads();
    huge_b_part3(r, t, P1, park, LG);
    __syncthreads();
  }

  // ---- C: lag rows, a thread pair per row ----
  {
    const float scale = (float)cc_scale<NH>();
    const int hh = t / MH;
    for (int b = 0; b < P1; b += MH) {
      const int s1 = b + t % MH;
      if (s1 < P1) huge_lag_row(s1, hh, P1, P2, LG, cc, scale);
    }
  }
  __syncthreads();

  // ---- D: similarity plane, peak, SN, Gaussian fit ----
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
  for (int l0 = t; l0 < nl; l0 += 4 * HUGE_THREADS) {
    double v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int l = l0 + k * HUGE_THREADS;
      v[k] = 0.0;
      if (l < nl) v[k] = team_similarity<ALG>(a, g, sc, sqF, l % P1, l / P1, (double)cc[l]);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int l = l0 + k * HUGE_THREADS;
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
  hpeak(best, bidx);
  double smax = hnmax(acc.smax), ssum = hsum(acc.ssum);
  if (lane == 0) {
    red[4 * warp] = best;
    red[4 * warp + 1] = (double)bidx;
    red[4 * warp + 2] = smax;
    red[4 * warp + 3] = ssum;
  }
  __syncthreads();
  if (warp == 0) {
    // the warps' partials in warp order
    best = red[0];
    bidx = (int)red[1];
    smax = red[2];
    ssum = red[3];
    for (int w = 1; w < HW; ++w) {
      peak_merge(best, bidx, red[4 * w], (int)red[4 * w + 1]);
      smax = nmax(smax, red[4 * w + 2]);
      ssum = ssum + red[4 * w + 3];
    }
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
  __syncthreads();  // the reduction slots and the scratch slot are reused by the next IA
}

template <int ALG, typename T>
__global__ void __launch_bounds__(HUGE_THREADS, 1) piv2d_huge_kernel(Piv2dArgs a) {
  extern __shared__ float2 sm[];
  float2* tw = sm + HugeSmem::PARK + HugeSmem::PACK;
  for (int j = threadIdx.x; j < NH; j += blockDim.x) tw[j] = twiddle_rt(j * (TW_N / NH));
  __syncthreads();
  float2* slot = a.huge + (long long)blockIdx.x * HugeSlot(2 * a.SM1 + 1, 2 * a.SM2 + 1).total;
  for (long long ia = a.ia_begin + blockIdx.x; ia < a.ia_end; ia += gridDim.x) huge_ia<ALG, T>(a, ia, slot, sm);
}

template <int ALG, typename T>
cudaError_t launch_huge_t(const Piv2dArgs& a, cudaStream_t s, std::string& err) {
  const size_t smem = (size_t)HugeSmem::TOTAL * sizeof(float2);
  auto kern = piv2d_huge_kernel<ALG, T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return e;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  long long blocks = device_sm_count(dev);
  const long long n = a.ia_end - a.ia_begin;
  if (blocks > n) blocks = n;
  if (blocks < 1) return cudaSuccess;
  kern<<<(unsigned)blocks, HUGE_THREADS, smem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("piv2d huge launch: ") + cudaGetErrorString(e);
  return e;
}

template <typename T>
cudaError_t launch_huge_alg(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  switch (alg) {
    case ALG_FFTCC: return launch_huge_t<ALG_FFTCC, T>(a, s, err);
    case ALG_ZNCC: return launch_huge_t<ALG_ZNCC, T>(a, s, err);
    case ALG_NSQECC: return launch_huge_t<ALG_NSQECC, T>(a, s, err);
    default: err = "search windows above 128 take FFTCC, ZNCC or NSQECC (no masks)"; return cudaErrorInvalidValue;
  }
}

}  // namespace

bool piv2d_huge_ok(int SS1, int SS2, int IS1, int IS2, int alg) {
  const int SS = SS1 > SS2 ? SS1 : SS2;
  return SS > 128 && SS <= NH && IS1 <= MH && IS2 <= MH && (alg == ALG_FFTCC || alg == ALG_ZNCC || alg == ALG_NSQECC);
}

size_t piv2d_huge_scratch_bytes(int device, int P1, int P2) {
  return (size_t)device_sm_count(device) * (size_t)HugeSlot(P1, P2).total * sizeof(float2);
}

cudaError_t launch_piv2d_huge(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  if (!a.huge) {
    err = "search windows above 128 need the per-block scratch (Piv2dArgs::huge)";
    return cudaErrorInvalidValue;
  }
  return a.dtype == 0 ? launch_huge_alg<float>(a, alg, s, err) : launch_huge_alg<double>(a, alg, s, err);
}

}  // namespace mqp
