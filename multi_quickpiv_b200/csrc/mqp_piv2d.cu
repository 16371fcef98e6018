// sm_100a kernels of the 2D path: FP64 integral images and the fused
// per-interrogation-area correlation / peak kernel (see mqp_piv2d.cuh).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include "mqp_internal.h"
#include "mqp_stage.cuh"

namespace mqp {

// ---------------------------------------------------------------------------
// integral images (integralArraySQ!, src/utils/common_ops.jl:142-180, built
// once per image instead of once per search window)
// ---------------------------------------------------------------------------
// pass 1: one warp per image column, prefix sum down the column (dim 1,
// contiguous) with warp scans; writes rows 1..H of out column c+1 and the
// zero first row.
// blockIdx.y selects one of a batch of planes (the z slices of a volume):
// input plane z starts at img + z*in_plane, its output at out + z*out_plane.
// Output columns [cb, ce) of the (W+1)-column integral.
template <typename T, bool SQ>
__global__ void integral_cols_kernel(const T* __restrict__ img, int H, int W, double* __restrict__ out,
                                     long long in_plane, long long out_plane, int cb, int ce) {
  const int warps = blockDim.x >> 5;
  const int lane = threadIdx.x & 31;
  const long long ld = (long long)H + 1;
  img += in_plane * blockIdx.y;
  out += out_plane * blockIdx.y;
  for (int c = cb + blockIdx.x * warps + (threadIdx.x >> 5); c < ce; c += gridDim.x * warps) {
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

// pass 2: running sums across columns (dim 2) in chunks of ICHUNK columns:
// thread (row r, chunk k) scans its chunk in place and records the chunk
// total; consecutive threads take consecutive rows, so every step is a
// coalesced column segment.
constexpr int ICHUNK = 64;

__global__ void integral_rows_chunk_kernel(int H, int W, double* __restrict__ out, double* __restrict__ totals,
                                           long long out_plane, long long tot_plane, int k0) {
  const long long ld = (long long)H + 1;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y + k0;
  if (r > H) return;
  out += out_plane * blockIdx.z;
  totals += tot_plane * blockIdx.z;
  const int c0 = 1 + k * ICHUNK;
  const int c1 = c0 + ICHUNK <= W + 1 ? c0 + ICHUNK : W + 1;
  double acc = 0.0;
  int c = c0;
  for (; c + 8 <= c1; c += 8) {
    double v[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) v[t] = out[r + ld * (c + t)];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      acc += v[t];
      out[r + ld * (c + t)] = acc;
    }
  }
  for (; c < c1; ++c) {
    acc += out[r + ld * c];
    out[r + ld * c] = acc;
  }
  totals[r + ld * k] = acc;
}

// pass 3a: per row, the running sums of the chunk totals,
// offs[k] = ((t_0 + t_1) + ...) + t_{k-1}, for chunks k in [k0, k1), k0 >= 1,
// continuing from offs[k0 - 1] (left by the earlier chunks).  offs lives
// tot_plane / 2 after the totals of its plane.
__global__ void integral_rows_prefix_kernel(int H, double* __restrict__ totals, long long tot_plane, int k0, int k1) {
  const long long ld = (long long)H + 1;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > H) return;
  totals += tot_plane * blockIdx.z;
  double* offs = totals + tot_plane / 2;
  double off = k0 > 1 ? offs[r + ld * (k0 - 1)] : 0.0;
  for (int k = k0; k < k1; ++k) {
    off = (k > 1 ? off : 0.0) + totals[r + ld * (k - 1)];
    offs[r + ld * k] = off;
  }
}

// pass 3b: every chunk k > 0 adds the sum of the totals of chunks 0..k-1
// (chunks k0 + blockIdx.y, k0 >= 1): read from pass 3a's running sums, or
// (few chunks, no pass 3a) summed here in the same order.
__global__ void integral_rows_offset_kernel(int H, int W, double* __restrict__ out,
                                            const double* __restrict__ totals, long long out_plane,
                                            long long tot_plane, int k0, int prefixed) {
  const long long ld = (long long)H + 1;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y + k0;
  if (r > H) return;
  out += out_plane * blockIdx.z;
  totals += tot_plane * blockIdx.z;
  double off = 0.0;
  if (prefixed) {
    off = totals[tot_plane / 2 + r + ld * k];
  } else {
    for (int q = 0; q < k; ++q) off += totals[r + ld * q];
  }
  const int c0 = 1 + k * ICHUNK;
  const int c1 = c0 + ICHUNK <= W + 1 ? c0 + ICHUNK : W + 1;
  for (int c = c0; c < c1; ++c) out[r + ld * c] += off;
}

// pass 4 (volumes): running sums along dim 3, one thread per (row, column)
// walking the planes; consecutive threads take consecutive rows.
__global__ void integral_zscan_kernel(long long plane, int D, double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= plane) return;
  double acc = 0.0;
  for (int z = 1; z <= D; ++z) {
    double* p = out + plane * z + i;
    acc += *p;
    *p = acc;
  }
}

// 2D exclusive-prefix integrals of `planes` consecutive H x W planes of img,
// plane z written to out + z*out_plane: the integral columns that image
// columns [x0, x1) complete (x0 a multiple of 64, x1 one or W), after those
// of image columns < x0.  Piece by piece or at once, every value comes out
// of the same sums in the same order.
static cudaError_t integral_planes(const void* img, int dtype, int H, int W, int planes, bool square, double* out,
                                   long long out_plane, double* scratch, cudaStream_t s, int x0 = 0, int x1 = -1) {
  if (x1 < 0) x1 = W;
  if (x0 % ICHUNK != 0 || x1 <= x0 || x1 > W || (x1 % ICHUNK != 0 && x1 != W)) return cudaErrorInvalidValue;
  const int threads = 256;
  const int cb = x0 == 0 ? 0 : x0 + 1, ce = x1 + 1;  // integral column c sums image columns < c
  const int blocks = (ce - cb + 7) / 8 < 4096 ? (ce - cb + 7) / 8 : 4096;
  const long long in_plane = (long long)H * W;
  const dim3 gc(blocks, planes);
  if (dtype == 0) {
    if (square) integral_cols_kernel<float, true><<<gc, threads, 0, s>>>((const float*)img, H, W, out, in_plane, out_plane, cb, ce);
    else integral_cols_kernel<float, false><<<gc, threads, 0, s>>>((const float*)img, H, W, out, in_plane, out_plane, cb, ce);
  } else {
    if (square) integral_cols_kernel<double, true><<<gc, threads, 0, s>>>((const double*)img, H, W, out, in_plane, out_plane, cb, ce);
    else integral_cols_kernel<double, false><<<gc, threads, 0, s>>>((const double*)img, H, W, out, in_plane, out_plane, cb, ce);
  }
  const int chunks = (W + ICHUNK - 1) / ICHUNK;
  const int k0 = x0 / ICHUNK, k1 = (x1 + ICHUNK - 1) / ICHUNK;  // row chunks of this piece
  // per plane: the chunk totals, then their running sums
  const long long tot_plane = 2LL * (H + 1) * (chunks + 1);
  const dim3 g1((H + 1 + 127) / 128, k1 - k0, planes);
  integral_rows_chunk_kernel<<<g1, 128, 0, s>>>(H, W, out, scratch, out_plane, tot_plane, k0);
  const int ko = k0 > 1 ? k0 : 1;
  if (k1 > ko) {
    // wide images: running sums first (linear work); up to 32 chunks the
    // offsets sum their few totals directly (one launch fewer)
    const int prefixed = chunks > 32;
    if (prefixed) {
      const dim3 gp((H + 1 + 127) / 128, 1, planes);
      integral_rows_prefix_kernel<<<gp, 128, 0, s>>>(H, scratch, tot_plane, ko, k1);
    }
    const dim3 g2((H + 1 + 127) / 128, k1 - ko, planes);
    integral_rows_offset_kernel<<<g2, 128, 0, s>>>(H, W, out, scratch, out_plane, tot_plane, ko, prefixed);
  }
  return cudaGetLastError();
}

cudaError_t launch_integral2d(const void* img, int dtype, int H, int W, bool square, double* out,
                              double* scratch, cudaStream_t s) {
  return integral_planes(img, dtype, H, W, 1, square, out, 0, scratch, s);
}

cudaError_t launch_integral2d_cols(const void* img, int dtype, int H, int W, int x0, int x1, bool square,
                                   double* out, double* scratch, cudaStream_t s) {
  return integral_planes(img, dtype, H, W, 1, square, out, 0, scratch, s, x0, x1);
}

cudaError_t launch_integral3d(const void* img, int dtype, int H, int W, int D, bool square, double* out,
                              double* scratch, cudaStream_t s) {
  const long long plane = (long long)(H + 1) * (W + 1);
  cudaError_t e = cudaMemsetAsync(out, 0, (size_t)plane * sizeof(double), s);
  if (e != cudaSuccess) return e;
  // planes are independent in the 2D passes; the grid's y/z extent bounds a batch
  for (int z0 = 0; z0 < D; z0 += 65535) {
    const int nz = D - z0 < 65535 ? D - z0 : 65535;
    const char* src = (const char*)img + (size_t)z0 * H * W * (dtype == 0 ? 4 : 8);
    e = integral_planes(src, dtype, H, W, nz, square, out + plane * (1 + z0), plane, scratch, s);
    if (e != cudaSuccess) return e;
  }
  integral_zscan_kernel<<<(unsigned)((plane + 255) / 256), 256, 0, s>>>(plane, D, out);
  return cudaGetLastError();
}

size_t integral2d_scratch_bytes(int H, int W) {  // chunk totals and their running sums
  return 2 * (size_t)(H + 1) * (size_t)((W + ICHUNK - 1) / ICHUNK + 1) * sizeof(double);
}

size_t integral3d_scratch_bytes(int H, int W, int D) {
  return integral2d_scratch_bytes(H, W) * (size_t)(D < 65535 ? D : 65535);
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
// One interrogation area, the whole per-IA body of PIV_CPU's loop, for one
// warp.  GH is the warp's shared-memory workspace (Layout2d, sized for this
// IA's lag plane), tw the (cos, sin)(2 pi j / N) table.  LW: ZNCC with an
// N/2 x N/2 interrogation window forms its window sums on chip (lw_rows /
// lw_cols) instead of reading integral images.  STG: this IA's search window
// was staged into GH by the TMA (mqp_stage.cuh) on mbar's phase `phase`, and
// the IA stages window ia_next (>= 0) as soon as its own G spectra are dead.
template <int N, bool FPRUNE, int ALG, typename T, bool LW = false, bool STG = false>
__device__ __forceinline__ void piv2d_ia(const Piv2dArgs& a, long long ia, float2* GH, const float2* tw, int lane,
                                         const CUtensorMap* tmap = nullptr, uint64_t* mbar = nullptr,
                                         unsigned* phase = nullptr, long long ia_next = -1) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  static_assert(!LW || ((ALG == ALG_ZNCC || ALG == ALG_NSQECC) && FPRUNE), "on-chip window sums: ZNCC / NSQECC");
  static_assert(!STG || (!MASKED && sizeof(T) == 4), "staged windows: FP32, unmasked");
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  // the plane follows the largest user of the G region: spectra, the window-sum table, the staged tile
  constexpr int F_OFF = STG ? (LW && Lay::F_OFF_LW > Lay::F_OFF_STG ? Lay::F_OFF_LW : Lay::F_OFF_STG)
                            : (LW ? Lay::F_OFF_LW : Lay::F_OFF);
  float2* FH = GH + F_OFF;
  // the next IA's window into the dead G spectra (every lane calls it)
  auto stage_next = [&]() {
    if (STG && ia_next >= 0 && *phase != STAGE_OFF) {
      stage_fence();
      __syncwarp();
      if (lane == 0) {
        const IAGeom gn = ia_geom(a, (int)(ia_next % a.vf1), (int)(ia_next / a.vf1));
        stage_issue<N>(tmap, reinterpret_cast<float*>(GH), mbar, stage_x0(gn.g01), gn.g02);
      }
    }
  };
  double* lw = LW ? reinterpret_cast<double*>(GH) : nullptr;
  double* plane = reinterpret_cast<double*>(FH);
  float* c1buf = MASKED ? reinterpret_cast<float*>(FH + Lay::region2_f2(P1, P2)) : nullptr;
  const double scale = cc_scale<N>();
  // lag rows [0, lane_rows) go one per lane; a short tail of rows
  // (2*SM1+1 just above 32) is computed by the whole warp, lanes over s2
  const int lane_rows = (P1 - 32 > 0 && P1 - 32 <= 4) ? 32 : P1;
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
  const long long vfo = (long long)v1 + (long long)a.vf1 * v2;
  bool skipped = false;

  // One pass correlates one pair of inputs; masked NSQECC needs two
  // ((F*mask) with G, mask with G^2, mask_nsqecc.jl:151-155).
  constexpr int NPASS = MASKED ? 2 : 1;
#pragma unroll 1
  for (int pass = 0; pass < NPASS; ++pass) {
    const int pmode = MASKED ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;

    // ---- phase 1: F rows and G rows, r2c along dim 2 (one rolled body) ----
    // The loads of the next row are in flight while the current row is
    // transformed.
    constexpr int NJF = (Lay::NF + 31) / 32, NJ = NJF + N / 32;
    double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
    if (STG) {
      // F rows from global memory (row_process reads them itself) while the
      // staged window lands; then every lane reads its G rows from the tile
      // before any lane writes spectra over it
#pragma unroll 1
      for (int job = 0; job < NJF; ++job) {
        const RowJob jf = row_job<N, FPRUNE>(a, g, lane, job);
        float none[N];
#pragma unroll
        for (int x = 0; x < N; ++x) none[x] = 0.f;
        if (jf.row < Lay::NF) row_process<N, FPRUNE, T, ALG == ALG_ZNCC>(a, sc, pmode, jf, none, GH, FH, vmax, mmax, sumsq);
      }
      // a copy that never lands (bounded wait) raises the status flag and
      // turns staging off for this warp: its rows come from global memory
      const bool armed = *phase != STAGE_OFF;
      const bool tiled = __all_sync(0xffffffffu, armed && stage_wait(mbar, *phase));  // one verdict per warp
      if (armed) {
        if (tiled) {
          *phase ^= 1u;
        } else {
          *phase = STAGE_OFF;
          if (a.status && lane == 0) atomicExch(a.status, 1);
        }
      }
      const float* tile = reinterpret_cast<const float*>(GH) + (g.g01 - stage_x0(g.g01));
      float gv[N / 32][N];
      RowJob jg[N / 32];
#pragma unroll
      for (int h = 0; h < N / 32; ++h) {
        jg[h] = row_job<N, FPRUNE>(a, g, lane, NJF + h);
        if (tiled) {
          const float* rowp = tile + jg[h].row;
#pragma unroll
          for (int x = 0; x < N; ++x)
            gv[h][x] = (jg[h].live && x >= jg[h].xlo && x < jg[h].xhi) ? rowp[x * StageTile<N>::ROWS] : 0.f;
        } else {
          row_load<N, T>(a, jg[h], gv[h]);
        }
      }
      __syncwarp();
      // unrolled: a runtime row index would put gv in local memory
#pragma unroll
      for (int h = 0; h < N / 32; ++h)
        row_process<N, FPRUNE, T, ALG == ALG_ZNCC>(a, sc, pmode, jg[h], gv[h], GH, FH, vmax, mmax, sumsq);
    } else {
    float buf[N];
    RowJob jn = row_job<N, FPRUNE>(a, g, lane, 0);
    row_load<N, T>(a, jn, buf);
#pragma unroll 1
    for (int job = 0; job < NJ; ++job) {
      const RowJob jc = jn;
      float cur[N];
#pragma unroll
      for (int x = 0; x < N; ++x) cur[x] = buf[x];
      if (job + 1 < NJ) {
        jn = row_job<N, FPRUNE>(a, g, lane, job + 1);
        row_load<N, T>(a, jn, buf);
      }
      if (!(jc.isF && jc.row >= Lay::NF))
        row_process<N, FPRUNE, T, ALG == ALG_ZNCC>(a, sc, pmode, jc, cur, GH, FH, vmax, mmax, sumsq);
    }
    }
    if (pass == 0) {
      vmax = warp_max(vmax);
      sc.sumF2 = warp_sum(sumsq);
      // skip_inter_region (src/utils/piv_ops.jl:134-157): the vector stays zero
      bool skip;
      if (MASKED) {
        mmax = warp_max(mmax);
        skip = (a.threshold > 0.0 && vmax < a.threshold) || (a.mask_threshold > 0.0 && mmax < a.mask_threshold);
      } else {
        skip = a.threshold >= 0.0 && vmax < a.threshold;
      }
      if (skip) {
        skipped = true;
        break;
      }
    }
    __syncwarp();
#pragma unroll 1
    for (int n = lane; n < M; n += 32) split_G_pair<N, FPRUNE>(GH, tw, n);
    __syncwarp();

    // ---- phases 2 and 3: one rolled loop of stages around one FFT body ----
    // The plane is row-contiguous: element (s1, s2) at s1*P2 + s2.
    {
      constexpr int RU = (M + 31) / 32;  // spectrum rows per lane
      const int NS2 = 6 * RU;            // phase-2 stages
      const int RL = (lane_rows + 31) / 32;
      float2 t[M];  // carried from the F stage (the product) into the I stage
#pragma unroll 1
      for (int job = 0; job < NS2 + RL; ++job) {
        if (job == NS2) __syncwarp();  // all spectra rows finished before phase 3
        bool active;
        int st = 0, h = 0, u = 0, s1 = 0;
        if (job < NS2) {
          const int q = job % 6;
          u = lane + 32 * (job / 6);
          h = q / 3;
          st = q % 3;
          active = u < M;
          if (active) stage_pre<N, FPRUNE>(st, h, GH + u * Lay::GSTR, FH + u * Lay::FSTR, t);
        } else {
          s1 = lane + 32 * (job - NS2);
          active = s1 < lane_rows;
          if (active) c2r_pre<N, FPRUNE>(s1, GH, t);
        }
        if (!active) continue;
        fft_reg<M, false>(t);
        if (job < NS2) {
          stage_post<N, FPRUNE>(st, h, u == 0, P1, GH + u * Lay::GSTR, t);
        } else {
          double* prow = plane + s1 * P2;
#pragma unroll
          for (int n = 0; n < M; ++n) {
            const float2 z = cconj(t[fpos<M>(n)]);
            if (2 * n < P2) prow[2 * n] = (double)z.x * scale;
            if (2 * n + 1 < P2) prow[2 * n + 1] = (double)z.y * scale;
          }
        }
      }
    }
    __syncwarp();
    // raw correlation of the tail lag rows, all lanes over s2
#pragma unroll 1
    for (int s1 = lane_rows; s1 < P1; ++s1)
      for (int s2 = lane; s2 < P2; s2 += 32)
        plane[s1 * P2 + s2] = (double)tail_row_value<N, FPRUNE>(GH, tw, s1, s2) * scale;
    __syncwarp();
    if (!LW) stage_next();  // with LW the table holds the G region until the finish has read it
    if (LW) {
      // the G spectra are dead: their space takes the window-sum table
      lw_rows<N, T, ALG == ALG_ZNCC>(a, g, sc.meanG, lane, P2, lw);
      __syncwarp();
      lw_cols<N>(lane, P1, P2, lw);
      lw_col32<N>(lane, P1, P2, lw);
      __syncwarp();
    }
    if (MASKED && pass == 0) {
      // park (F*mask)*G while the second pass reuses the workspace
      for (int i = lane; i < P1 * P2; i += 32) c1buf[i] = (float)plane[i];
      __syncwarp();
    }
  }
  if (skipped) {
    stage_next();
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
    return;
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
#pragma unroll 1
  for (int s1 = lane; s1 < lane_rows; s1 += 32)
    finish_row<ALG, LW ? N : 0>(a, g, sc, s1, P1, P2, plane + s1 * P2, R, acc, MASKED ? c1buf + s1 * P2 : nullptr,
                                lw);
#pragma unroll 1
  for (int s1 = lane_rows; s1 < P1; ++s1)
    for (int s2 = lane; s2 < P2; s2 += 32) {
      double& e = plane[s1 * P2 + s2];
      e = finish_one<ALG, LW ? N : 0>(a, g, sc, s1, s2, e, MASKED ? (double)c1buf[s1 * P2 + s2] : 0.0, lw);
      acc_take(acc, R, s1, s2, P1, e);
    }
  __syncwarp();
  if (LW) stage_next();
  double best = acc.best;
  int bidx = acc.bidx;
  warp_peak(best, bidx);
  double sn = 0.0;
  if (a.SN) {
    // compute_SN (src/utils/piv_ops.jl:336-367) over [TLF_off, 2SM-1-BRB_off]
    const double smax = warp_nmax(acc.smax);
    const double ssum = warp_sum(acc.ssum);
    const double len = (double)(R.shi1 - R.lo1 + 1) * (double)(R.shi2 - R.lo2 + 1);
    sn = smax / ((ssum - smax) / (len - 1.0));
  }
  if (a.planes) {
    double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
    for (int i = lane; i < P1 * P2; i += 32) dst[i] = plane[(i % P1) * P2 + i / P1];
  }
  double r1 = -1.0, r2 = -1.0;  // no peak: 1-based (0, 0), displacement -(SM+1)
  if (bidx >= 0) refine2d_warp(plane, P2, a.SM1, a.SM2, g, bidx % P1, bidx / P1, best, lane, r1, r2);
  if (lane == 0) {
    a.VF[2 * vfo + 0] = r1 - a.SM1 + d1;
    a.VF[2 * vfo + 1] = r2 - a.SM2 + d2;
    if (a.SN) a.SN[vfo] = sn;
  }
  __syncwarp();
}

// Persistent: each warp walks IAs ia = first + k * (all warps).  The warp's
// shared-memory workspace holds the spectra rows of G (N/2 x (N+1)) and F
// (N/2 x (NF+1)); after phase 2 the F rows are reused for the FP64 plane.
// STG: tmap describes img2 for the staged windows (mqp_stage.cuh); each
// warp stages its first window before the loop and every IA the next one.
template <int N, bool FPRUNE, int ALG, typename T, int WARPS, int MINB, bool LW = false, bool STG = false>
__global__ void __launch_bounds__(WARPS * 32, MINB) piv2d_kernel(Piv2dArgs a, const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) float2 smem[];
  using Lay = Layout2d<N, FPRUNE>;
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wf2 = STG ? Lay::warp_f2_stg(P1, P2) : (LW ? Lay::warp_f2_lw(P1, P2) : Lay::warp_f2(P1, P2, MASKED));
  float2* GH = smem + (size_t)warp * wf2;
  float2* tw = smem + (size_t)WARPS * wf2;  // (cos, sin)(2 pi j / N)
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tw + N) + warp;
  for (int j = threadIdx.x; j < N; j += blockDim.x) tw[j] = twiddle_rt(j * (TW_N / N));
  if (STG && lane == 0) stage_init(mbar);
  __syncthreads();
  const long long nwarps = (long long)gridDim.x * WARPS;
  const long long first = a.ia_begin + (long long)blockIdx.x * WARPS + warp;
  unsigned phase = 0;
  if (STG && first < a.ia_end && lane == 0) {
    const IAGeom g0 = ia_geom(a, (int)(first % a.vf1), (int)(first / a.vf1));
    stage_issue<N>(&tmap, reinterpret_cast<float*>(GH), mbar, stage_x0(g0.g01), g0.g02);
  }
  for (long long ia = first; ia < a.ia_end; ia += nwarps)
    piv2d_ia<N, FPRUNE, ALG, T, LW, STG>(a, ia, GH, tw, lane, &tmap, mbar, &phase,
                                         ia + nwarps < a.ia_end ? ia + nwarps : -1);
}

// Batched: the IAs of many image pairs sharing one kernel variant form one
// work queue [0, total); prefix[k] is the first queue index of item k
// (prefix[n_items] = total).  Warps take `grab` consecutive queue entries at
// a time from `counter` (zeroed before the launch), so large and small pairs
// balance across the SMs.  wf2: float2 per warp, the largest any item needs.
template <int N, bool FPRUNE, int ALG, typename T, int WARPS, int MINB, bool LW = false>
__global__ void __launch_bounds__(WARPS * 32, MINB)
    piv2d_batch_kernel(const Piv2dArgs* __restrict__ items, const long long* __restrict__ prefix, int n_items,
                       long long total, int wf2, int grab, unsigned long long* counter) {
  extern __shared__ float2 smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* GH = smem + (size_t)warp * wf2;
  float2* tw = smem + (size_t)WARPS * wf2;
  for (int j = threadIdx.x; j < N; j += blockDim.x) tw[j] = twiddle_rt(j * (TW_N / N));
  __syncthreads();
  for (;;) {
    unsigned long long g0 = 0;
    if (lane == 0) g0 = atomicAdd(counter, (unsigned long long)grab);
    g0 = __shfl_sync(0xffffffffu, g0, 0);
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
      piv2d_ia<N, FPRUNE, ALG, T, LW>(a, a.ia_begin + (gi - prefix[lo]), GH, tw, lane);
    }
  }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
int piv2d_fft_len(int SS1, int SS2) {
  const int SS = SS1 > SS2 ? SS1 : SS2;
  if (SS <= 32) return 32;
  if (SS <= 64) return 64;
  if (SS <= 128) return 128;  // block kernel, mqp_piv2d_big.cu
  return 0;
}

int device_sm_count(int device) {
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  return n;
}

// Tensor map of an H x W column-major FP32 image for the staged windows of
// FFT length N: dim 0 = rows (contiguous), dim 1 = columns, box (N + 4) x N,
// zero fill outside the image.  False when the image does not qualify (row
// pitch not a multiple of 16 bytes, base not 16-byte aligned) or the driver
// entry point is missing; the caller then launches the unstaged kernel.
static bool stage_tensor_map(CUtensorMap* m, const void* img, long long H, long long W, int N) {
  if (H % 4 != 0 || ((uintptr_t)img & 15) != 0 || H < 1 || W < 1) return false;
  typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  // looked up once (thread-safe static initialisation: serving launches from several threads)
  static const EncodeTiled encode = []() -> EncodeTiled {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return (EncodeTiled)fn;
    return nullptr;
  }();
  if (!encode) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)H, (cuuint64_t)W};
  const cuuint64_t strides[1] = {(cuuint64_t)H * 4};
  const cuuint32_t box[2] = {(cuuint32_t)(N + 4), (cuuint32_t)N};
  const cuuint32_t estr[2] = {1, 1};
  return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(img), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Staged windows are on unless MQP_TUNE_PIV2D_TMA=0 (both kernels give
// identical results; the knob exists for timing comparisons).
static bool stage_enabled() {
  const char* v = getenv("MQP_TUNE_PIV2D_TMA");  // read per launch: a test may switch it between calls
  return !(v && v[0] == '0');
}

template <int N, bool FPRUNE, int ALG, typename T, int WARPS, int MINB, bool LW = false, bool STG = false>
static cudaError_t launch_t(const Piv2dArgs& a, cudaStream_t s, std::string& err, const CUtensorMap* tm = nullptr) {
  using Lay = Layout2d<N, FPRUNE>;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const int wf2 = STG ? Lay::warp_f2_stg(P1, P2) : (LW ? Lay::warp_f2_lw(P1, P2) : Lay::warp_f2(P1, P2, ALG == ALG_MASK_NSQECC));
  const size_t smem = ((size_t)WARPS * wf2 + N + (STG ? WARPS : 0)) * sizeof(float2);
  auto kern = piv2d_kernel<N, FPRUNE, ALG, T, WARPS, MINB, LW, STG>;
  CUtensorMap tmap;
  memset(&tmap, 0, sizeof(tmap));
  if (tm) tmap = *tm;
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
  kern<<<(unsigned)blocks, WARPS * 32, smem, s>>>(a, tmap);
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("piv2d launch: ") + cudaGetErrorString(e);
  return e;
}

// FP32 FFTCC / NSQECC / ZNCC with staged windows when img2 qualifies.
// Measured on B200 (2048^2 vortex, step 8, whole pass, results
// bit-identical): NSQECC interSize 32 2.41 -> 2.22 ms, 24 2.06 -> 1.85, 16
// 0.86 -> 0.82; FFTCC 32 1.42 -> 1.27, 24 1.32 -> 1.18, 16 0.65 -> 0.52;
// ZNCC 24 2.55 -> 2.49 (ZNCC with interSize N/2 goes through launch_lw).
template <int N, bool FPRUNE, int WARPS, int MINB>
static bool launch_stg(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err, cudaError_t& e) {
  if (a.dtype != 0 || !stage_enabled() || (alg != ALG_FFTCC && alg != ALG_NSQECC && alg != ALG_ZNCC)) return false;
  CUtensorMap tm;
  if (!stage_tensor_map(&tm, a.img2, a.H, a.W, N)) return false;
  e = alg == ALG_FFTCC  ? launch_t<N, FPRUNE, ALG_FFTCC, float, WARPS, MINB, false, true>(a, s, err, &tm)
      : alg == ALG_ZNCC ? launch_t<N, FPRUNE, ALG_ZNCC, float, WARPS, MINB, false, true>(a, s, err, &tm)
                        : launch_t<N, FPRUNE, ALG_NSQECC, float, WARPS, MINB, false, true>(a, s, err, &tm);
  return true;
}

template <int N, bool FPRUNE, typename T, int WARPS, int MINB>
static cudaError_t launch_alg(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  switch (alg) {
    case ALG_FFTCC: return launch_t<N, FPRUNE, ALG_FFTCC, T, WARPS, MINB>(a, s, err);
    case ALG_ZNCC: return launch_t<N, FPRUNE, ALG_ZNCC, T, WARPS, MINB>(a, s, err);
    case ALG_NSQECC: return launch_t<N, FPRUNE, ALG_NSQECC, T, WARPS, MINB>(a, s, err);
    // length 64: 29.7 KB per warp, three warps per block keep two blocks per SM
    case ALG_MASK_NSQECC: return launch_t<N, FPRUNE, ALG_MASK_NSQECC, T, N == 32 ? 4 : 3, MINB>(a, s, err);
    default: err = "unknown correlation algorithm"; return cudaErrorInvalidValue;
  }
}

template <int N, bool FPRUNE, int WARPS, int MINB>
static cudaError_t launch_dt(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  return a.dtype == 0 ? launch_alg<N, FPRUNE, float, WARPS, MINB>(a, alg, s, err)
                      : launch_alg<N, FPRUNE, double, WARPS, MINB>(a, alg, s, err);
}

// ZNCC whose interrogation window is half the FFT length in both axes: the
// warp kernel forms the window sums on chip and reads no integral image of
// img2^2 (lw_rows / lw_cols).  Measured on B200 (2048^2 vortex, interSize 32,
// margin 16, step 8, whole pass): ZNCC 2.91 -> 2.77 ms, since it drops eight
// integral-image loads per lag; NSQECC, with four, ran 2.42 -> 2.54 ms (the
// window's second read from L2 costs more than the lookups it replaces), so
// NSQECC keeps the integral image.
bool piv2d_local_sums(int IS1, int IS2, int SM1, int SM2, int alg) {
  if (alg != ALG_ZNCC) return false;
  if (direct2d_ok(IS1, IS2, SM1, SM2)) return false;
  const int N = piv2d_fft_len(IS1 + 2 * SM1, IS2 + 2 * SM2);
  if (N != 32 && N != 64) return false;
  if (piv2d_team_ok(N, true, alg)) return false;
  return IS1 == N / 2 && IS2 == N / 2;
}

template <int N, int MINB>
static cudaError_t launch_lw(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  if (alg != ALG_ZNCC) {
    err = "on-chip window sums are built for ZNCC";
    return cudaErrorInvalidValue;
  }
  // staged windows as well at length 32 (interSize 16: 0.98 -> 0.86 ms per 2048^2 pass); at length 64
  // the tile can only be issued after the finish has read the table, and the pass ran 2.77 -> 3.09 ms
  CUtensorMap tm;
  if (N == 32 && a.dtype == 0 && stage_enabled() && stage_tensor_map(&tm, a.img2, a.H, a.W, N))
    return launch_t<N, true, ALG_ZNCC, float, 4, MINB, true, true>(a, s, err, &tm);
  return a.dtype == 0 ? launch_t<N, true, ALG_ZNCC, float, 4, MINB, true>(a, s, err)
                      : launch_t<N, true, ALG_ZNCC, double, 4, MINB, true>(a, s, err);
}

int piv2d_warp_f2_lw(int N, int P1, int P2) {
  return N == 64 ? Layout2d<64, true>::warp_f2_lw(P1, P2) : Layout2d<32, true>::warp_f2_lw(P1, P2);
}

int piv2d_warp_f2(int N, bool prune, int P1, int P2, bool masked) {
  if (!masked && piv2d_team_ok(N, prune, ALG_NSQECC)) return piv2d_team_f2(N, P1, P2);
  if (N == 128) return piv2d_big_warp_f2(prune, P1, P2, masked);
  if (N == 64) return prune ? Layout2d<64, true>::warp_f2(P1, P2, masked) : Layout2d<64, false>::warp_f2(P1, P2, masked);
  if (N == 32) return prune ? Layout2d<32, true>::warp_f2(P1, P2, masked) : Layout2d<32, false>::warp_f2(P1, P2, masked);
  return 0;
}

template <int N, bool FPRUNE, int ALG, typename T, int WARPS, int MINB, bool LW = false>
static cudaError_t launch_batch_t(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  const size_t smem = ((size_t)WARPS * b.wf2 + N) * sizeof(float2);
  auto kern = piv2d_batch_kernel<N, FPRUNE, ALG, T, WARPS, MINB, LW>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return e;
  }
  int dev = 0, per_sm = 0;
  cudaGetDevice(&dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, smem);
  if (e != cudaSuccess || per_sm < 1) {
    err = "piv2d batch kernel does not fit on an SM (shared memory " + std::to_string(smem) + " B)";
    return e != cudaSuccess ? e : cudaErrorInvalidConfiguration;
  }
  long long blocks = (long long)device_sm_count(dev) * per_sm;
  const long long need = (b.total + WARPS - 1) / WARPS;
  if (blocks > need) blocks = need;
  if (blocks < 1) return cudaSuccess;
  if ((e = cudaMemsetAsync(b.counter, 0, sizeof(unsigned long long), s)) != cudaSuccess) {
    err = std::string("counter reset: ") + cudaGetErrorString(e);
    return e;
  }
  kern<<<(unsigned)blocks, WARPS * 32, smem, s>>>(b.items, b.prefix, b.n_items, b.total, b.wf2,
                                                   b.grab > 0 ? b.grab : 1, b.counter);
  e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("piv2d batch launch: ") + cudaGetErrorString(e);
  return e;
}

template <int N, bool FPRUNE, typename T>
static cudaError_t launch_batch_alg(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  constexpr int MINB = N == 32 ? 3 : 2;  // as launch_piv2d
  switch (b.alg) {
    case ALG_FFTCC: return launch_batch_t<N, FPRUNE, ALG_FFTCC, T, 4, MINB>(b, s, err);
    case ALG_ZNCC: return launch_batch_t<N, FPRUNE, ALG_ZNCC, T, 4, MINB>(b, s, err);
    case ALG_NSQECC: return launch_batch_t<N, FPRUNE, ALG_NSQECC, T, 4, MINB>(b, s, err);
    case ALG_MASK_NSQECC: return launch_batch_t<N, FPRUNE, ALG_MASK_NSQECC, T, N == 32 ? 4 : 3, MINB>(b, s, err);
    default: err = "unknown correlation algorithm"; return cudaErrorInvalidValue;
  }
}

template <int N, int MINB>
static cudaError_t launch_batch_lw(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  if (b.alg != ALG_ZNCC) {
    err = "on-chip window sums are built for ZNCC";
    return cudaErrorInvalidValue;
  }
  return b.dtype == 0 ? launch_batch_t<N, true, ALG_ZNCC, float, 4, MINB, true>(b, s, err)
                      : launch_batch_t<N, true, ALG_ZNCC, double, 4, MINB, true>(b, s, err);
}

template <int N, bool FPRUNE>
static cudaError_t launch_batch_dt(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  return b.dtype == 0 ? launch_batch_alg<N, FPRUNE, float>(b, s, err) : launch_batch_alg<N, FPRUNE, double>(b, s, err);
}

cudaError_t launch_piv2d_batch(const Piv2dBatch& b, cudaStream_t s, std::string& err) {
  if (b.total <= 0 || b.n_items <= 0) return cudaSuccess;
  if (b.N == 128) return launch_piv2d_big_batch(b, s, err);
  if (b.N == 1) return launch_piv2d_direct_batch(b, s, err);
  if (piv2d_team_ok(b.N, b.prune, b.alg)) return launch_piv2d_team_batch(b, s, err);
  if (b.lw) return b.N == 64 ? launch_batch_lw<64, 2>(b, s, err) : launch_batch_lw<32, 3>(b, s, err);
  if (b.N == 64) return b.prune ? launch_batch_dt<64, true>(b, s, err) : launch_batch_dt<64, false>(b, s, err);
  if (b.N == 32) return b.prune ? launch_batch_dt<32, true>(b, s, err) : launch_batch_dt<32, false>(b, s, err);
  err = "search window larger than 64 along some axis is not supported by the 2D kernel";
  return cudaErrorInvalidValue;
}

cudaError_t launch_piv2d(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err) {
  if (direct2d_ok(a.IS1, a.IS2, a.SM1, a.SM2)) return launch_piv2d_direct(a, alg, s, err);
  const int SS1 = a.IS1 + 2 * a.SM1, SS2 = a.IS2 + 2 * a.SM2;
  const int N = piv2d_fft_len(SS1, SS2);
  const bool prune = (a.IS1 <= N / 2) && (a.IS2 <= N / 2);
  if (piv2d_team_ok(N, prune, alg)) return launch_piv2d_team(a, N, alg, s, err);
  if (piv2d_local_sums(a.IS1, a.IS2, a.SM1, a.SM2, alg))
    return N == 64 ? launch_lw<64, 2>(a, alg, s, err) : launch_lw<32, 3>(a, alg, s, err);
  cudaError_t e = cudaSuccess;
  if (N == 64 && (prune ? launch_stg<64, true, 4, 2>(a, alg, s, err, e) : launch_stg<64, false, 4, 2>(a, alg, s, err, e)))
    return e;
  if (N == 32 && (prune ? launch_stg<32, true, 4, 3>(a, alg, s, err, e) : launch_stg<32, false, 4, 3>(a, alg, s, err, e)))
    return e;
  if (N == 64) return prune ? launch_dt<64, true, 4, 2>(a, alg, s, err) : launch_dt<64, false, 4, 2>(a, alg, s, err);
  // length 32 needs fewer registers: three blocks per SM (12 warps) without spill
  if (N == 32) return prune ? launch_dt<32, true, 4, 3>(a, alg, s, err) : launch_dt<32, false, 4, 3>(a, alg, s, err);
  if (N == 128) return launch_piv2d_big(a, alg, s, err);
  err = "search window larger than 128 along some axis is not supported by the 2D kernels";
  return cudaErrorInvalidValue;
}

}  // namespace mqp
