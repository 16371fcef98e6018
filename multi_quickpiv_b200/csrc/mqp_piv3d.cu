// sm_100a kernels of the 3D path (see mqp_piv3d.cuh): K3a (r2c along dim 3),
// K3b (complex 2D correlation per k3 slab), K3c (inverse along k3, similarity,
// peak, Gaussian fit, SN), launched chunk by chunk over the vector field.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>

#include "mqp_internal.h"

namespace mqp {

namespace {

constexpr int K3A_THREADS = 256;

__device__ __forceinline__ double warp_sum3(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ double warp_max3(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}
__device__ __forceinline__ double warp_nmax3(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = nmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  return v;
}

// Blocks (part, IA): each part walks its contiguous share of the IA's lines.
// Pass 0 leaves the part's skip maxima and sumF2 in apart; part 0 records the
// ZNCC means, and k3a_merge_kernel completes the state.
// Two blocks per SM (16 warps): registers capped at 128 (a few bytes of
// spill at length 64) instead of one 147-register block.
template <int N, bool FPRUNE, int ALG, typename T>
__global__ void __launch_bounds__(K3A_THREADS, 2) k3a_kernel(Piv3dArgs a, int pass) {
  constexpr int PARTS = k3a_parts(N);
  const int part = blockIdx.x;
  const long long ci = blockIdx.y;
  const IAGeom3 g = ia_geom3(a, a.ia_begin + ci);
  IA3State s;
  if (pass == 0) {
    ia3_means<ALG>(a, g, s.meanF, s.meanG);
    s.sumF2 = 0.0;
    s.skip = 0;
  } else {
    s = a.state[ci];
  }
  double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
  const int nl = k3a_lines(a, g);
  const int l0 = (int)((long long)nl * part / PARTS), l1 = (int)((long long)nl * (part + 1) / PARTS);
  for (int line = l0 + threadIdx.x; line < l1; line += K3A_THREADS)
    k3a_line<N, FPRUNE, T, ALG>(a, g, s, pass, ci, line, vmax, mmax, sumsq);
  if (pass != 0) return;
  __shared__ double red[3][K3A_THREADS / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  vmax = warp_max3(vmax);
  mmax = warp_max3(mmax);
  sumsq = warp_sum3(sumsq);
  if (lane == 0) {
    red[0][warp] = vmax;
    red[1][warp] = mmax;
    red[2][warp] = sumsq;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < K3A_THREADS / 32; ++w) {
      vmax = fmax(vmax, red[0][w]);
      mmax = fmax(mmax, red[1][w]);
      sumsq += red[2][w];
    }
    a.apart[ci * PARTS + part] = ReducePart3{vmax, mmax, sumsq};
    if (part == 0) a.state[ci] = s;
  }
}

// One thread per IA: its K3a parts in part order -> sumF2 and the skip test.
template <int N, int ALG>
__global__ void k3a_merge_kernel(Piv3dArgs a, long long n) {
  constexpr int PARTS = k3a_parts(N);
  const long long ci = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= n) return;
  const ReducePart3* p = a.apart + ci * PARTS;
  double vmax = p[0].vmax, mmax = p[0].mmax, sumsq = p[0].sumsq;
  for (int k = 1; k < PARTS; ++k) {
    vmax = fmax(vmax, p[k].vmax);
    mmax = fmax(mmax, p[k].mmax);
    sumsq += p[k].sumsq;
  }
  IA3State s = a.state[ci];
  s.sumF2 = sumsq;
  s.skip = skip_test3(a, ALG, vmax, mmax) ? 1 : 0;
  a.state[ci] = s;
}

// One block of 2N threads (a pair per line) per (k3, IA) slab.
template <int N, bool FPRUNE>
__global__ void __launch_bounds__(2 * N) k3b_kernel(Piv3dArgs a, float2* C) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
  extern __shared__ float2 sm[];
  const int k3 = blockIdx.x;
  const long long ci = blockIdx.y;
  if (a.state[ci].skip) return;
  const IAGeom3 g = ia_geom3(a, a.ia_begin + ci);
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1;
  float2* S = sm;
  float2* SF = sm + N * L::SSTR;
  const int t = threadIdx.x % N, h = threadIdx.x / N;
  k3b_rows<N, FPRUNE>(a, g, ci, k3, t, h, S, SF);
  __syncthreads();
  {
    float2 y[M];
    k3b_cols_g<N, FPRUNE>(t, h, S, y);
    __syncthreads();
    k3b_park<N, FPRUNE>(t, h, S, y);
  }
  __syncthreads();
  {
    float2 p[M];
    k3b_cols_f<N, FPRUNE>(t, h, S, SF, p);
    __syncthreads();
    k3b_x1<N, FPRUNE>(t, h, p, S);
  }
  __syncthreads();
  {
    float2 o[M];
    k3b_x2<N, FPRUNE>(t, h, S, o);
    __syncthreads();
    k3b_x3<N, FPRUNE>(t, h, P1, o, S);
  }
  __syncthreads();
  {
    float2 u[M];
    k3b_r2a<N, FPRUNE>(t, h, P1, S, u);
    __syncthreads();
    k3b_r2b<N, FPRUNE>(t, h, P1, u, S);
  }
  __syncthreads();
  k3b_r2c<N, FPRUNE>(ci, k3, t, h, P1, P2, S, C);
}

// Blocks (part, IA): each part walks its contiguous share of the lag pairs;
// the part's peak / SN accumulators go to cpart, and k3c_merge_kernel
// finishes the IA.
template <int N, int ALG>
__global__ void __launch_bounds__(K3C_THREADS) k3c_kernel(Piv3dArgs a) {
  const int part = blockIdx.x, parts = gridDim.x;
  const long long ci = blockIdx.y;
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1, P3 = 2 * a.SM[2] + 1;
  const int q0 = P1 * P2 * part / parts, q1 = P1 * P2 * (part + 1) / parts;
  const IA3State s = a.state[ci];
  if (s.skip) {
    if (a.planes) {
      const long long vol = (long long)P1 * P2 * P3;
      double* dst = a.planes + (a.ia_begin + ci - a.planes_begin) * vol;
      for (int q = q0 + threadIdx.x; q < q1; q += K3C_THREADS)
        for (int s3 = 0; s3 < P3; ++s3) dst[q + (long long)P1 * P2 * s3] = 0.0;
    }
    return;
  }
  const IAGeom3 g = ia_geom3(a, a.ia_begin + ci);
  const LagRanges3 R = lag_ranges3(a, g);
  PeakAcc acc;
  acc.best = 0.0;
  acc.bidx = -1;
  acc.smax = -INFINITY;
  acc.ssum = 0.0;
  for (int q = q0 + threadIdx.x; q < q1; q += K3C_THREADS) k3c_pair<N, ALG>(a, g, s, ci, q, P1, P2, P3, R, acc);
  // block merge: (largest value, lowest column-major index), NaN-propagating max, sum
  __shared__ double rb[K3C_THREADS / 32], rs[K3C_THREADS / 32], rm[K3C_THREADS / 32];
  __shared__ int ri[K3C_THREADS / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double best = acc.best;
  int bidx = acc.bidx;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bidx, off);
    peak_merge(best, bidx, ob, oi);
  }
  const double smax = warp_nmax3(acc.smax);
  const double ssum = warp_sum3(acc.ssum);
  if (lane == 0) {
    rb[warp] = best;
    ri[warp] = bidx;
    rm[warp] = smax;
    rs[warp] = ssum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = rb[0], mx = rm[0], sum = rs[0];
    int bi = ri[0];
    for (int w = 1; w < K3C_THREADS / 32; ++w) {
      peak_merge(b, bi, rb[w], ri[w]);
      mx = nmax(mx, rm[w]);
      sum += rs[w];
    }
    PeakPart3 pp;
    pp.best = b;
    pp.smax = mx;
    pp.ssum = sum;
    pp.bidx = bi;
    pp.pad_ = 0;
    a.cpart[ci * gridDim.x + part] = pp;
  }
}

// One thread per IA: its K3c parts in part order, then the Gaussian fit and
// SN from the similarity volume (k3c_final).
template <int N, int ALG>
__global__ void k3c_merge_kernel(Piv3dArgs a, long long n, int parts) {
  const long long ci = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= n) return;
  if (a.state[ci].skip) {
    k3c_skipped(a, ci);
    return;
  }
  const PeakPart3* p = a.cpart + ci * parts;
  double b = p[0].best, mx = p[0].smax, sum = p[0].ssum;
  int bi = p[0].bidx;
  for (int k = 1; k < parts; ++k) {
    peak_merge(b, bi, p[k].best, p[k].bidx);
    mx = nmax(mx, p[k].smax);
    sum += p[k].ssum;
  }
  const IAGeom3 g = ia_geom3(a, a.ia_begin + ci);
  k3c_final(a, g, ci, lag_ranges3(a, g), b, bi, mx, sum);
}

template <int N, bool FPRUNE, int ALG, typename T>
cudaError_t run_chunks(Piv3dArgs a, long long chunk, cudaStream_t s, std::string& err) {
  using L = Lay3<N, FPRUNE>;
  const size_t smem = (size_t)L::SMEM_F2 * sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(k3b_kernel<N, FPRUNE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return e;
  }
  const long long begin = a.ia_begin, end = a.ia_end;
  constexpr int NPASS = ALG == ALG_MASK_NSQECC ? 2 : 1;
  for (long long c0 = begin; c0 < end; c0 += chunk) {
    const long long n = end - c0 < chunk ? end - c0 : chunk;
    a.ia_begin = c0;
    a.ia_end = c0 + n;
    const unsigned merge_blocks = (unsigned)((n + 127) / 128);
    for (int pass = 0; pass < NPASS; ++pass) {
      k3a_kernel<N, FPRUNE, ALG, T><<<dim3(k3a_parts(N), (unsigned)n), K3A_THREADS, 0, s>>>(a, pass);
      if (pass == 0) k3a_merge_kernel<N, ALG><<<merge_blocks, 128, 0, s>>>(a, n);
      k3b_kernel<N, FPRUNE><<<dim3(L::K3, (unsigned)n), 2 * N, smem, s>>>(a, pass == 0 ? a.C : a.C2);
    }
    const int cparts = k3c_parts(N, (2 * a.SM[0] + 1) * (2 * a.SM[1] + 1));
    k3c_kernel<N, ALG><<<dim3(cparts, (unsigned)n), K3C_THREADS, 0, s>>>(a);
    k3c_merge_kernel<N, ALG><<<merge_blocks, 128, 0, s>>>(a, n, cparts);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
      err = std::string("piv3d launch: ") + cudaGetErrorString(e);
      return e;
    }
  }
  return cudaSuccess;
}

template <int N, bool FPRUNE, typename T>
cudaError_t run_alg(const Piv3dArgs& a, int alg, long long chunk, cudaStream_t s, std::string& err) {
  switch (alg) {
    case ALG_FFTCC: return run_chunks<N, FPRUNE, ALG_FFTCC, T>(a, chunk, s, err);
    case ALG_ZNCC: return run_chunks<N, FPRUNE, ALG_ZNCC, T>(a, chunk, s, err);
    case ALG_NSQECC: return run_chunks<N, FPRUNE, ALG_NSQECC, T>(a, chunk, s, err);
    case ALG_MASK_NSQECC: return run_chunks<N, FPRUNE, ALG_MASK_NSQECC, T>(a, chunk, s, err);
    default: err = "unknown correlation algorithm"; return cudaErrorInvalidValue;
  }
}

template <int N, bool FPRUNE>
cudaError_t run_dt(const Piv3dArgs& a, int alg, long long chunk, cudaStream_t s, std::string& err) {
  return a.dtype == 0 ? run_alg<N, FPRUNE, float>(a, alg, chunk, s, err)
                      : run_alg<N, FPRUNE, double>(a, alg, chunk, s, err);
}

}  // namespace

int piv3d_fft_len(const int SS[3]) {
  int m = SS[0];
  if (SS[1] > m) m = SS[1];
  if (SS[2] > m) m = SS[2];
  if (m <= 32) return 32;
  if (m <= 64) return 64;
  if (m <= 128) return 128;  // only with every interSize <= 64 (launch_piv3d)
  return 0;
}

static bool piv3d_prune(const int IS[3], int N) { return IS[0] <= N / 2 && IS[1] <= N / 2 && IS[2] <= N / 2; }

// Chunk scratch of c IAs: Gz | Fz | C | C2 | V | state | K3a parts | K3c
// parts, each array 256-byte aligned.
namespace {
struct Scr3 {
  size_t b[8];
};
Scr3 scr3(const int IS[3], const int SM[3], int alg, size_t c) {
  Scr3 r{};
  const int SS[3] = {IS[0] + 2 * SM[0], IS[1] + 2 * SM[1], IS[2] + 2 * SM[2]};
  const int N = piv3d_fft_len(SS);
  if (N == 0) return r;
  const size_t K3 = N / 2 + 1;
  const size_t NF = piv3d_prune(IS, N) ? N / 2 : N;
  const size_t P12 = (size_t)(2 * SM[0] + 1) * (2 * SM[1] + 1);
  const size_t P3 = 2 * SM[2] + 1;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  r.b[0] = al(c * K3 * N * N * sizeof(float2));                               // Gz
  r.b[1] = al(c * K3 * NF * NF * sizeof(float2));                             // Fz
  r.b[2] = al(c * K3 * P12 * sizeof(float2));                                 // C
  r.b[3] = alg == ALG_MASK_NSQECC ? r.b[2] : 0;                               // C2
  r.b[4] = al(c * P12 * P3 * sizeof(float));                                  // V
  r.b[5] = al(c * sizeof(IA3State));                                          // state
  r.b[6] = al(c * k3a_parts(N) * sizeof(ReducePart3));                        // K3a parts
  r.b[7] = al(c * (size_t)k3c_parts(N, (int)P12) * sizeof(PeakPart3));        // K3c parts
  return r;
}
}  // namespace

size_t piv3d_scratch_bytes(const int IS[3], const int SM[3], int alg, long long chunk) {
  const Scr3 r = scr3(IS, SM, alg, (size_t)chunk);
  size_t t = 0;
  for (size_t x : r.b) t += x;
  return t;
}

size_t piv3d_scratch_bytes_per_ia(const int IS[3], const int SM[3], int alg) {
  // one IA's share, with the alignment of the eight arrays
  return piv3d_scratch_bytes(IS, SM, alg, 1);
}

void piv3d_bind_scratch(Piv3dArgs& a, int alg, long long chunk, char* base) {
  const Scr3 r = scr3(a.IS, a.SM, alg, (size_t)chunk);
  size_t o = 0;
  a.Gz = (float2*)(base + o);
  o += r.b[0];
  a.Fz = (float2*)(base + o);
  o += r.b[1];
  a.C = (float2*)(base + o);
  o += r.b[2];
  a.C2 = r.b[3] ? (float2*)(base + o) : nullptr;
  o += r.b[3];
  a.V = (float*)(base + o);
  o += r.b[4];
  a.state = (IA3State*)(base + o);
  o += r.b[5];
  a.apart = (ReducePart3*)(base + o);
  o += r.b[6];
  a.cpart = (PeakPart3*)(base + o);
}

cudaError_t launch_piv3d(const Piv3dArgs& a, int alg, long long chunk, cudaStream_t s, std::string& err) {
  const int SS[3] = {a.IS[0] + 2 * a.SM[0], a.IS[1] + 2 * a.SM[1], a.IS[2] + 2 * a.SM[2]};
  const int N = piv3d_fft_len(SS);
  if (!direct3d_ok(a.IS, a.SM) && (chunk < 1 || chunk > 65535)) {
    err = "3D chunk must be in [1, 65535]";
    return cudaErrorInvalidValue;
  }
  if (a.ia_end <= a.ia_begin) return cudaSuccess;
  if (direct3d_ok(a.IS, a.SM)) return launch_piv3d_direct(a, alg, s, err);  // small windows: no chunk scratch
  const bool prune = piv3d_prune(a.IS, N);
  if (N == 64) return prune ? run_dt<64, true>(a, alg, chunk, s, err) : run_dt<64, false>(a, alg, chunk, s, err);
  if (N == 32) return prune ? run_dt<32, true>(a, alg, chunk, s, err) : run_dt<32, false>(a, alg, chunk, s, err);
  // search windows 65..128 (the coarse passes of interSize-64 refinements):
  // the same kernels at length 128, for interrogation windows up to 64
  if (N == 128 && prune) return run_dt<128, true>(a, alg, chunk, s, err);
  err = "3D search window (interSize + 2 searchMargin) above 128, or above 64 with an interSize above 64, is not supported";
  return cudaErrorInvalidValue;
}

}  // namespace mqp
