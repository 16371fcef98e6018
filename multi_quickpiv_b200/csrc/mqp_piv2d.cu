// sm_100a kernels of the 2D path: FP64 integral images and the fused
// per-interrogation-area correlation / peak kernel (see mqp_piv2d.cuh).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>

#include "mqp_internal.h"

namespace mqp {

// ---------------------------------------------------------------------------
// integral images (integralArraySQ!, src/utils/common_ops.jl:142-180, built
// once per image instead of once per search window)
// ---------------------------------------------------------------------------
// pass 1: one warp per image column, prefix sum down the column (dim 1,
// contiguous) with warp scans; writes rows 1..H of out column c+1 and the
// zero first row.
template <typename T, bool SQ>
__global__ void integral_cols_kernel(const T* __restrict__ img, int H, int W, double* __restrict__ out) {
  const int warps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  const long long ld = (long long)H + 1;
  for (int c = blockIdx.x * warps + (threadIdx.x >> 5); c <= W; c += gridDim.x * warps) {
    double* o = out + ld * c;
    if (c == 0) {
      for (int r = lane; r <= H; r += 32) o[r] = 0.0;
      continue;
    }
    const T* col = img + (long long)H * (c - 1);
    if (lane == 0) o[0] = 0.0;
    double carry = 0.0;
    for (int r0 = 0; r0 < H; r0 += 32) {
      const int r = r0 + lane;
      double v = 0.0;
      if (r < H) {
        v = (double)col[r];
        if (SQ) v = v * v;
      }
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += t;
      }
      v += carry;
      if (r < H) o[r + 1] = v;
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

// pass 2: one thread per row of out, running sum across columns (dim 2);
// consecutive threads read consecutive rows, so every step is coalesced.
__global__ void integral_rows_kernel(int H, int W, double* __restrict__ out) {
  const long long ld = (long long)H + 1;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > H) return;
  double acc = 0.0;
  int c = 1;
  for (; c + 8 <= W + 1; c += 8) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = out[r + ld * (c + k)];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      acc += v[k];
      out[r + ld * (c + k)] = acc;
    }
  }
  for (; c <= W; ++c) {
    acc += out[r + ld * c];
    out[r + ld * c] = acc;
  }
}

cudaError_t launch_integral2d(const void* img, int dtype, int H, int W, bool square, double* out,
                              cudaStream_t s) {
  const int threads = 256;
  const int blocks = (W + 1 + 7) / 8 < 4096 ? (W + 1 + 7) / 8 : 4096;
  if (dtype == 0) {
    if (square) integral_cols_kernel<float, true><<<blocks, threads, 0, s>>>((const float*)img, H, W, out);
    else integral_cols_kernel<float, false><<<blocks, threads, 0, s>>>((const float*)img, H, W, out);
  } else {
    if (square) integral_cols_kernel<double, true><<<blocks, threads, 0, s>>>((const double*)img, H, W, out);
    else integral_cols_kernel<double, false><<<blocks, threads, 0, s>>>((const double*)img, H, W, out);
  }
  integral_rows_kernel<<<(H + 1 + 127) / 128, 128, 0, s>>>(H, W, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// warp reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ double warp_nmax(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = nmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ void warp_peak(double& best, int& bidx) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bidx, off);
    peak_merge(best, bidx, ob, oi);
  }
}

// ---------------------------------------------------------------------------
// the fused kernel
// ---------------------------------------------------------------------------
// Persistent: each warp walks IAs ia = first + k * (all warps).  The warp's
// shared-memory workspace holds the spectra rows of G (N/2 x (N+1)) and F
// (N/2 x (NF+1)); after phase 2 the F rows are reused for the FP64 plane.
template <int N, bool FPRUNE, int ALG, typename T, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) piv2d_kernel(Piv2dArgs a) {
  extern __shared__ float2 smem[];
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* GH = smem + (size_t)warp * Lay::warp_f2(P1, P2);
  float2* FH = GH + Lay::F_OFF;
  double* plane = reinterpret_cast<double*>(FH);
  float2* tw = smem + (size_t)WARPS * Lay::warp_f2(P1, P2);  // (cos, sin)(2 pi j / N)
  for (int j = threadIdx.x; j < N; j += blockDim.x) tw[j] = twiddle_cs(j * (TW_N / N));
  __syncthreads();
  const long long nwarps = (long long)gridDim.x * WARPS;
  const double scale = cc_scale<N>();

  for (long long ia = a.ia_begin + (long long)blockIdx.x * WARPS + warp; ia < a.ia_end; ia += nwarps) {
    const int v1 = (int)(ia % a.vf1), v2 = (int)(ia / a.vf1);
    int d1, d2;
    ia_pred(a, v1, v2, d1, d2);
    const IAGeom g = ia_geom(a, v1, v2);
    IAScalars sc;
    sc.meanF = 0.0;
    sc.meanG = 0.0;
    if (ALG == ALG_ZNCC) {
      // copy_*_minus_mean! (src/utils/zncc_ops.jl:7-25): IA mean and the mean
      // of the whole clipped search region
      sc.meanF = box_sum(a.II1, a.H, g.ir1, g.ir1 + a.IS1, g.ir2, g.ir2 + a.IS2) / ((double)a.IS1 * a.IS2);
      const double nG = (double)(g.hi1 - g.lo1) * (double)(g.hi2 - g.lo2);
      sc.meanG = box_sum(a.IIg, a.H, g.g01 + g.lo1, g.g01 + g.hi1, g.g02 + g.lo2, g.g02 + g.hi2) / nG;
    }

    // ---- phase 1: F rows (+ skip test), then G rows; r2c along dim 2 ----
    constexpr int NJF = (Lay::NF + 31) / 32, NJG = N / 32;
    double vmax = -INFINITY, sumsq = 0.0;
#pragma unroll 1
    for (int job = 0; job < NJF; ++job) {
      const int row = lane + 32 * job;
      if (row < Lay::NF) phase1_row<N, FPRUNE, T, ALG == ALG_ZNCC>(a, g, sc, true, row, GH, FH, vmax, sumsq);
    }
    vmax = warp_max(vmax);
    sc.sumF2 = warp_sum(sumsq);
    const long long vfo = (long long)v1 + (long long)a.vf1 * v2;
    if (a.threshold >= 0.0 && vmax < a.threshold) {
      // skip_inter_region (src/utils/piv_ops.jl:140-146): the vector stays zero
      if (lane == 0) {
        a.VF[2 * vfo + 0] = 0.0;
        a.VF[2 * vfo + 1] = 0.0;
        if (a.SN) a.SN[vfo] = 0.0;
      }
      if (a.planes) {
        double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
        for (int i = lane; i < P1 * P2; i += 32) dst[i] = 0.0;
      }
      __syncwarp();
      continue;
    }
#pragma unroll 1
    for (int job = 0; job < NJG; ++job)
      phase1_row<N, FPRUNE, T, ALG == ALG_ZNCC>(a, g, sc, false, lane + 32 * job, GH, FH, vmax, sumsq);
    __syncwarp();

    // ---- phase 2: along dim 1 per spectrum row, product, inverse ----
#pragma unroll 1
    for (int u = lane; u < M; u += 32) phase2_row<N, FPRUNE>(u, P1, GH, FH);
    __syncwarp();

    // ---- phase 3: c2r along dim 2 per lag row, similarity -> plane ----
    // rows [0, lane_rows) one per lane; a short tail of rows (2*SM1+1 just
    // above 32) is computed by the whole warp, lanes over s2.
    const int lane_rows = (P1 - 32 > 0 && P1 - 32 <= 4) ? 32 : P1;
#pragma unroll 1
    for (int s1 = lane; s1 < lane_rows; s1 += 32) {
      float cc[N];
      phase3_row<N, FPRUNE>(s1, GH, cc);
#pragma unroll
      for (int s2 = 0; s2 < N; ++s2)
        if (s2 < P2) plane[s1 + P1 * s2] = (double)cc[s2] * scale;
      similarity_row<ALG>(a, g, sc, s1, P1, P2, plane);
    }
#pragma unroll 1
    for (int s1 = lane_rows; s1 < P1; ++s1)
      for (int s2 = lane; s2 < P2; s2 += 32)
        plane[s1 + P1 * s2] =
            similarity_one<ALG>(a, g, sc, s1, s2, (double)tail_row_value<N, FPRUNE>(GH, tw, s1, s2) * scale);
    __syncwarp();

    // ---- peak (first_fullovp_peak), SN, Gaussian refinement ----
    const int lo1 = g.tlf1, hi1 = 2 * a.SM1 - g.brb1;
    const int lo2 = g.tlf2, hi2 = 2 * a.SM2 - g.brb2;
    double best = 0.0;
    int bidx = -1;
    for (int s1 = lane; s1 < lane_rows && s1 <= hi1; s1 += 32)
      if (s1 >= lo1) peak_scan_row(plane, P1, s1, lo2, hi2, best, bidx);
    for (int s1 = lane_rows > lo1 ? lane_rows : lo1; s1 <= hi1; ++s1)
      for (int s2 = lane; s2 <= hi2; s2 += 32)
        if (s2 >= lo2) peak_take(plane[s1 + P1 * s2], s1 + P1 * s2, best, bidx);
    warp_peak(best, bidx);
    double sn = 0.0;
    if (a.SN) {
      // compute_SN (src/utils/piv_ops.jl:336-367) over [TLF_off, 2SM-1-BRB_off]
      const int shi1 = 2 * a.SM1 - 1 - g.brb1, shi2 = 2 * a.SM2 - 1 - g.brb2;
      double smax = -INFINITY, ssum = 0.0;
      for (int s1 = lane; s1 < lane_rows && s1 <= shi1; s1 += 32) {
        if (s1 < lo1) continue;
        for (int s2 = lo2; s2 <= shi2; ++s2) {
          const double v = plane[s1 + P1 * s2];
          smax = nmax(smax, v);
          ssum += v;
        }
      }
      for (int s1 = lane_rows > lo1 ? lane_rows : lo1; s1 <= shi1; ++s1)
        for (int s2 = lane; s2 <= shi2; s2 += 32) {
          if (s2 < lo2) continue;
          const double v = plane[s1 + P1 * s2];
          smax = nmax(smax, v);
          ssum += v;
        }
      smax = warp_nmax(smax);
      ssum = warp_sum(ssum);
      const double len = (double)(shi1 - lo1 + 1) * (double)(shi2 - lo2 + 1);
      sn = smax / ((ssum - smax) / (len - 1.0));
    }
    if (a.planes) {
      double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
      for (int i = lane; i < P1 * P2; i += 32) dst[i] = plane[i];
    }
    if (lane == 0) {
      double r1, r2;
      if (bidx < 0) {
        r1 = -1.0;  // 1-based peak (0, 0): displacement -(SM+1)
        r2 = -1.0;
      } else {
        refine2d(plane, P1, a.SM1, a.SM2, g, bidx % P1, bidx / P1, best, r1, r2);
      }
      a.VF[2 * vfo + 0] = r1 - a.SM1 + d1;
      a.VF[2 * vfo + 1] = r2 - a.SM2 + d2;
      if (a.SN) a.SN[vfo] = sn;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
int piv2d_fft_len(int SS1, int SS2) {
  const int SS = SS1 > SS2 ? SS1 : SS2;
  if (SS <= 32) return 32;
  if (SS <= 64) return 64;
  return 0;
}

int device_sm_count(int device) {
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  return n;
}

template <int N, bool FPRUNE, int ALG, typename T, int WARPS, int MINB>
static cudaError_t launch_t(const Piv2dArgs& a, cudaStream_t s, std::string& err) {
  using Lay = Layout2d<N, FPRUNE>;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const size_t smem = ((size_t)WARPS * Lay::warp_f2(P1, P2) + N) * sizeof(float2);
  auto kern = piv2d_kernel<N, FPRUNE, ALG, T, WARPS, MINB>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return e;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, smem);
  if (e != cudaSuccess || per_sm < 1) {
    err = "piv2d kernel does not fit on an SM (shared memory " + std::to_string(smem) + " B)";
    return e != cudaSuccess ? e : cudaErrorInvalidConfiguration;
  }
  const long long n_ia = a.ia_end - a.ia_begin;
  long long blocks = (long long)device_sm_count(dev) * per_sm;
  const long long need = (n_ia + WARPS - 1) / WARPS;
  if (blocks > need) blocks = need;
  if (blocks < 1) return cudaSuccess;
  kern<<<(unsigned)blocks, WARPS * 32, smem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("piv2d launch: ") + cudaGetErrorString(e);
  return e;
}

template <int N, bool FPRUNE, typename T, int WARPS, int MINB>
static cudaError_t launch_alg(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  switch (alg) {
    case ALG_FFTCC: return launch_t<N, FPRUNE, ALG_FFTCC, T, WARPS, MINB>(a, s, err);
    case ALG_ZNCC: return launch_t<N, FPRUNE, ALG_ZNCC, T, WARPS, MINB>(a, s, err);
    case ALG_NSQECC: return launch_t<N, FPRUNE, ALG_NSQECC, T, WARPS, MINB>(a, s, err);
    default: err = "unknown correlation algorithm"; return cudaErrorInvalidValue;
  }
}

template <int N, bool FPRUNE, int WARPS, int MINB>
static cudaError_t launch_dt(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  return a.dtype == 0 ? launch_alg<N, FPRUNE, float, WARPS, MINB>(a, alg, s, err)
                      : launch_alg<N, FPRUNE, double, WARPS, MINB>(a, alg, s, err);
}

cudaError_t launch_piv2d(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  const int SS1 = a.IS1 + 2 * a.SM1, SS2 = a.IS2 + 2 * a.SM2;
  const int N = piv2d_fft_len(SS1, SS2);
  const bool prune = (a.IS1 <= N / 2) && (a.IS2 <= N / 2);
  if (N == 64) return prune ? launch_dt<64, true, 4, 2>(a, alg, s, err) : launch_dt<64, false, 4, 2>(a, alg, s, err);
  if (N == 32) return prune ? launch_dt<32, true, 4, 2>(a, alg, s, err) : launch_dt<32, false, 4, 2>(a, alg, s, err);
  err = "search window larger than 64 along some axis is not supported by the 2D kernel";
  return cudaErrorInvalidValue;
}

}  // namespace mqp
