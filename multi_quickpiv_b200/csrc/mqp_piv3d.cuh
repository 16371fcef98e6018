// 3D PIV: the per-IA body of multi_quickPIV's PIV_CPU loop
// (src/multi_quickPIV.jl:63-89) for volumes, as three kernels over a chunk
// of interrogation areas (IAs).  A 64^3 search window's spectrum
// (64 x 64 x 33 complex FP32, 1.08 MB) does not fit on one SM, so the
// transform is split by axis and the pieces meet in an L2/HBM scratch:
//
//   K3a  one thread per window line along dim 3 (z): r2c of the real line
//        (one N/2-point complex FFT), bins k3 = 0..N/2 written to
//        Gz[k3][x2][x1] / Fz[k3][x2][x1].  Threads are consecutive x1, so
//        every image load and every scratch store is one coalesced segment.
//        The block also reduces the skip test's maximum and sumF2.
//   K3b  one block per (IA, k3) slab: the complex 2D correlation of the F
//        slab with the G slab, i.e. rows along dim 2, columns along dim 1,
//        conj(F)*G, inverse along k1 (lags s1 < P1 kept), inverse along k2
//        (lags s2 < P2 kept); every line transform is a register FFT.
//   K3c  one block per IA: the complex-to-real inverse along k3 for every
//        (s1, s2) lag pair (k3 > N/2 follow by Hermitian symmetry), the
//        ZNCC / NSQECC / masked NSQECC normalisation from FP64 integral
//        volumes, the first full-overlap maximum, the 3x3x3 Gaussian fit and
//        the SN ratio.
//
// cc[s] = sum_x F(x) G(x+s) on the lags s in [0, 2SM] exactly as
// _FFTCC! (src/crosscorrelation_algorithms/fftcc.jl:101-126); any cubic FFT
// length N >= IS + 2SM gives the same lags as the reference's
// good_size_real transform.  N is 32 or 64 here.
#pragma once

#include "mqp_piv2d.cuh"

namespace mqp {

// per-IA values K3a hands to K3b / K3c
struct IA3State {
  double sumF2;  // sum of squares of the transformed F (ZNCC: mean removed; masked: sum(maskF^2/wi))
  double meanF;  // ZNCC
  double meanG;  // ZNCC
  int skip;      // skip_inter_region said yes: the vector stays zero
  int pad_;
};

// Per-block partial results: K3a's skip maxima and sumF2 over its share of
// the lines, K3c's peak / SN accumulators over its share of the lag pairs;
// a merge kernel combines an IA's parts in part order.
struct ReducePart3 {
  double vmax, mmax, sumsq;
};
struct PeakPart3 {
  double best, smax, ssum;
  int bidx, pad_;
};

// Blocks per IA of K3a (over its z-lines) and K3c (over its lag pairs): at
// FFT length 128 an IA's lines and lag pairs fill several blocks (the coarse
// passes that use it have few IAs); shorter lengths keep one block per IA.
constexpr int K3C_THREADS = 256;
MQP_HD MQP_FI constexpr int k3a_parts(int N) { return N >= 128 ? 8 : 1; }
MQP_HD MQP_FI int k3c_parts(int N, int P12) { return N >= 128 ? (P12 + K3C_THREADS - 1) / K3C_THREADS : 1; }

struct Piv3dArgs {
  const void* img1;
  const void* img2;
  const void* mask;       // masked NSQECC interrogation-area mask, or null
  const void* mask_skip;  // masked NSQECC skip mask, or null (= mask)
  int dtype;              // 0 = float32 volumes, 1 = float64 volumes
  const double* II1;      // integral volume of img1 (ZNCC), (H+1)(W+1)(D+1)
  const double* IIg;      // integral volume of img2 (ZNCC)
  const double* IIg2;     // integral volume of img2^2 (ZNCC, NSQECC)
  const int32_t* pred;    // whole-voxel predictor (3, vf1, vf2, vf3) or null
  double* VF;             // (3, vf1, vf2, vf3) column-major
  double* SN;             // (vf1, vf2, vf3) or null
  double* planes;         // debug: (P1, P2, P3, n) similarity volumes or null
  long long planes_begin; // IA index of planes[..., 0]
  int H, W, D;            // volume size (dims 1, 2, 3)
  int IS[3], SM[3], st[3], vf[3];
  long long ia_begin, ia_end;  // IAs of this chunk (global linear indices)
  double threshold;       // skip when max(IA) < threshold (threshold >= 0; masked: > 0)
  double mask_threshold;  // masked: skip when max(mask_skip IA) < mask_threshold (> 0)
  // chunk scratch, indexed by ci = ia - ia_begin
  float2* Gz;             // [ci][k3][x2][x1], N x N per slab
  float2* Fz;             // [ci][k3][x2][x1], NF x NF per slab
  float2* C;              // [ci][k3][s2][s1] first (or only) correlation
  float2* C2;             // masked: mask * G^2 correlation
  float* V;               // [ci][s3][s2][s1] similarity volume
  IA3State* state;        // [ci]
  ReducePart3* apart;     // [ci][k3a_parts(N)]
  PeakPart3* cpart;       // [ci][k3c_parts(N, P1 P2)]
};

template <int N, bool FPRUNE>
struct Lay3 {
  static constexpr int M = N / 2;
  static constexpr int K3 = M + 1;                // z bins 0..N/2
  static constexpr int NF = FPRUNE ? N / 2 : N;   // F extent kept along dims 1 and 2
  static constexpr long long GZ = (long long)K3 * N * N;    // float2 per IA
  static constexpr long long FZ = (long long)K3 * NF * NF;  // float2 per IA
  static constexpr int SSTR = N + 1;              // odd strides: conflict-free rows and columns
  static constexpr int FSTR = NF + 1;
  static constexpr int SMEM_F2 = N * SSTR + N * FSTR;  // K3b shared memory per slab
};

// Geometry of one IA in pad coordinates (0-based), per axis d: pad index p
// maps to volume index g0[d] + p and holds data iff lo[d] <= p < hi[d].
struct IAGeom3 {
  int v[3];    // vector-field coordinates
  int d[3];    // clamped whole-voxel predictor
  int ir[3];   // IA origin (0-based volume coordinates)
  int g0[3], lo[3], hi[3];
  int tlf[3], brb[3];  // SR_TLF_off, SR_BRB_off
};

// get_interrogation_coordinates + get_search_coordinates
// (src/utils/piv_ops.jl:38-76) per axis, with linear2cartesian's column-major
// order (src/utils/common_ops.jl:54-67).
MQP_HD MQP_FI IAGeom3 ia_geom3(const Piv3dArgs& a, long long ia) {
  IAGeom3 g;
  const long long plane = (long long)a.vf[0] * a.vf[1];
  g.v[2] = (int)(ia / plane);
  const long long r = ia - (long long)g.v[2] * plane;
  g.v[1] = (int)(r / a.vf[0]);
  g.v[0] = (int)(r - (long long)g.v[1] * a.vf[0]);
  const int size[3] = {a.H, a.W, a.D};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int dd = 0;
    if (a.pred) {
      const int T0 = 1 + g.v[d] * a.st[d];
      dd = clamp_pred(a.pred[3 * ia + d], T0, T0 + a.IS[d] - 1, size[d]);
    }
    g.d[d] = dd;
    axis_geom(g.v[d], a.st[d], a.IS[d], a.SM[d], size[d], dd, g.ir[d], g.g0[d], g.lo[d], g.hi[d], g.tlf[d],
              g.brb[d]);
  }
  return g;
}

// Sum over the volume box [r0, r1) x [c0, c1) x [z0, z1) from an
// exclusive-prefix integral volume of size (H+1) x (W+1) x (D+1).
MQP_HD MQP_FI double box_sum3(const double* II, int H, int W, int r0, int r1, int c0, int c1, int z0, int z1) {
  if (r1 <= r0 || c1 <= c0 || z1 <= z0) return 0.0;
  const long long l1 = (long long)H + 1, l2 = l1 * ((long long)W + 1);
  const double* A = II + l2 * z1;
  const double* B = II + l2 * z0;
  const double top = (A[r1 + l1 * c1] - A[r0 + l1 * c1]) - (A[r1 + l1 * c0] - A[r0 + l1 * c0]);
  const double bot = (B[r1 + l1 * c1] - B[r0 + l1 * c1]) - (B[r1 + l1 * c0] - B[r0 + l1 * c0]);
  return top - bot;
}

// ZNCC means (copy_*_minus_mean!, src/utils/zncc_ops.jl:7-25): of the IA and
// of the whole clipped search region.
template <int ALG>
MQP_HD MQP_FI void ia3_means(const Piv3dArgs& a, const IAGeom3& g, double& meanF, double& meanG) {
  meanF = 0.0;
  meanG = 0.0;
  if (ALG != ALG_ZNCC) return;
  meanF = box_sum3(a.II1, a.H, a.W, g.ir[0], g.ir[0] + a.IS[0], g.ir[1], g.ir[1] + a.IS[1], g.ir[2],
                   g.ir[2] + a.IS[2]) /
          ((double)a.IS[0] * (double)a.IS[1] * (double)a.IS[2]);
  const double nG = (double)(g.hi[0] - g.lo[0]) * (double)(g.hi[1] - g.lo[1]) * (double)(g.hi[2] - g.lo[2]);
  meanG = box_sum3(a.IIg, a.H, a.W, g.g0[0] + g.lo[0], g.g0[0] + g.hi[0], g.g0[1] + g.lo[1], g.g0[1] + g.hi[1],
                   g.g0[2] + g.lo[2], g.g0[2] + g.hi[2]) /
          nG;
}

// ---------------------------------------------------------------------------
// K3a: r2c along dim 3 of one window line
// ---------------------------------------------------------------------------
// z holds the line packed as z[n] = x[2n] + i x[2n+1]; after the N/2-point FFT
// out[k * kstride] receives X2[k] = 2 DFT(x)[k] for k = 0..N/2 (X2[0] and
// X2[N/2] are real).
template <int N, int NZ>
MQP_HD MQP_FI void r2c_line_store(float2 (&z)[N / 2], float2* out, long long kstride) {
  constexpr int M = N / 2;
  fft_reg<M, false, NZ>(z);
  const float2 Z0 = z[fpos<M>(0)];
  out[0] = make_float2(2.f * (Z0.x + Z0.y), 0.f);
  out[M * kstride] = make_float2(2.f * (Z0.x - Z0.y), 0.f);
#pragma unroll
  for (int k = 1; k < M; ++k) {
    const float2 A = z[fpos<M>(k)];
    const float2 B = cconj(z[fpos<M>(M - k)]);
    out[k * kstride] = cadd(cadd(A, B), rotate<N, false>(cmul_mi(csub(A, B)), k));
  }
}

// Lines of one IA: the IS1 x IS2 lines of F first (line = x1 + IS1 x2), then
// the data lines of G (x1 in [lo1, hi1), x2 in [lo2, hi2)).
MQP_HD MQP_FI int k3a_lines(const Piv3dArgs& a, const IAGeom3& g) {
  return a.IS[0] * a.IS[1] + (g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]);
}

// One line of K3a.  F lines: the IA line along z (copy_inter_region!,
// src/utils/piv_ops.jl:99-109), minus the IA mean for ZNCC
// (src/utils/zncc_ops.jl:7-12), times the mask for masked NSQECC
// (copy_inter_masked!, src/utils/masked_nsqecc_ops.jl:19-25) or the mask
// itself for its second correlation; they accumulate the raw maxima of the
// skip tests (src/utils/piv_ops.jl:134-157) and the FP64 sumF2
// (zncc.jl:131-135, nsqecc.jl:349-353; masked sum(maskF^2/wi),
// mask_nsqecc.jl:141-149).  G lines: the search line on its data part
// (copy_search_region!, src/utils/piv_ops.jl:115-127), minus the search
// mean for ZNCC (src/utils/zncc_ops.jl:18-25), squared for the masked second
// correlation (copy_search_squared!, src/utils/masked_nsqecc_ops.jl:35-42).
template <int N, bool FPRUNE, typename T, int ALG>
MQP_HD MQP_FI void k3a_line(const Piv3dArgs& a, const IAGeom3& g, const IA3State& s, int pass, long long ci,
                            int line, double& vmax, double& mmax, double& sumsq) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
  const long long HW = (long long)a.H * a.W;
  const int nFL = a.IS[0] * a.IS[1];
  const int PASS = ALG == ALG_MASK_NSQECC ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;
  float w[N];
  if (line < nFL) {
    const int x1 = line % a.IS[0], x2 = line / a.IS[0];
    const long long base = (long long)(g.ir[0] + x1) + (long long)a.H * ((long long)(g.ir[1] + x2) +
                                                                         (long long)a.W * g.ir[2]);
    const T* p = reinterpret_cast<const T*>(a.img1) + base;
    const T* q = PASS != PASS_PLAIN ? reinterpret_cast<const T*>(a.mask) + base : p;
    const T* qs = PASS == PASS_MASKED ? reinterpret_cast<const T*>(a.mask_skip ? a.mask_skip : a.mask) + base : p;
    constexpr int FLIM = L::NF;  // z extent an IA line can occupy
#pragma unroll
    for (int x = 0; x < N; ++x) {
      w[x] = 0.f;
      if (x < FLIM && x < a.IS[2]) {
        const long long off = HW * x;
        if (PASS == PASS_PLAIN) {
          const T r = ldg_px<T>(p, off);
          vmax = (double)r > vmax ? (double)r : vmax;
          const double val = (double)r - s.meanF;
          sumsq += val * val;
          w[x] = (float)val;
        } else if (PASS == PASS_MASKED) {
          const T r = ldg_px<T>(p, off);
          const T mk = ldg_px<T>(q, off);
          const T ms = ldg_px<T>(qs, off);
          vmax = (double)r > vmax ? (double)r : vmax;
          mmax = (double)ms > mmax ? (double)ms : mmax;
          const double val = (double)r * (double)mk;
          sumsq += val * val / ((double)mk > 0.0 ? (double)mk : 1.0);
          w[x] = (float)val;
        } else {
          w[x] = (float)ldg_px<T>(q, off);
        }
      }
    }
    float2 z[M];
#pragma unroll
    for (int n = 0; n < M; ++n) z[n] = make_float2(w[2 * n], w[2 * n + 1]);
    float2* out = a.Fz + ci * L::FZ + ((long long)x2 * L::NF + x1);
    r2c_line_store<N, FPRUNE ? M / 2 : M>(z, out, (long long)L::NF * L::NF);
    return;
  }
  const int l = line - nFL;
  const int n1 = g.hi[0] - g.lo[0];
  const int x1 = g.lo[0] + l % n1, x2 = g.lo[1] + l / n1;
  const long long base = (long long)(g.g0[0] + x1) + (long long)a.H * ((long long)(g.g0[1] + x2) +
                                                                       (long long)a.W * g.g0[2]);
  const T* p = reinterpret_cast<const T*>(a.img2) + base;
  const float mg = (float)s.meanG;
#pragma unroll
  for (int x = 0; x < N; ++x) {
    w[x] = 0.f;
    if (x >= g.lo[2] && x < g.hi[2]) {
      float v = (float)ldg_px<T>(p, HW * x);
      if (ALG == ALG_ZNCC) v = v - mg;
      if (PASS == PASS_MASK_SQ) v = v * v;
      w[x] = v;
    }
  }
  float2 z[M];
#pragma unroll
  for (int n = 0; n < M; ++n) z[n] = make_float2(w[2 * n], w[2 * n + 1]);
  float2* out = a.Gz + ci * L::GZ + ((long long)x2 * N + x1);
  r2c_line_store<N, M>(z, out, (long long)N * N);
}

MQP_HD MQP_FI bool skip_test3(const Piv3dArgs& a, int alg, double vmax, double mmax) {
  if (alg == ALG_MASK_NSQECC)
    return (a.threshold > 0.0 && vmax < a.threshold) || (a.mask_threshold > 0.0 && mmax < a.mask_threshold);
  return a.threshold >= 0.0 && vmax < a.threshold;
}

// ---------------------------------------------------------------------------
// K3b: the complex 2D correlation of one k3 slab, two threads per line
// ---------------------------------------------------------------------------
// Thread (t, h) of 2N: every N-point line transform is split between a pair.
// Forward (decimation in frequency): X[2m + h] is the M-point FFT (M = N/2)
// of x[n] + x[n+M] (h = 0) or (x[n] - x[n+M]) W_N^n (h = 1).  Inverse
// (decimation in time): z_h = M-point inverse of the bins of parity h, and
// x[n] = z_0[n] + W_N^-n z_1[n], x[n+M] = z_0[n] - W_N^-n z_1[n].  A thread
// holds M values, half the registers of a whole line, so twice the warps fit.
// Phases are separated by block barriers (the kernel, or the host emulation
// running each phase for all threads before the next).

// the half-line input of the forward split from the line's two halves
template <int N>
MQP_HD MQP_FI float2 dif_in(int h, int n, float2 u, float2 v) {
  return h ? rotate<N, false>(csub(u, v), n) : cadd(u, v);
}

// Phase R: thread (t, h) transforms row x1 = t of the G slab and (t < NF) of
// the F slab along dim 2; bins k2 = 2m + h go to S[k2][x1] and SF[k2][x1].
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_rows(const Piv3dArgs& a, const IAGeom3& g, long long ci, int k3, int t, int h, float2* S,
                            float2* SF) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
  const float2 z0 = make_float2(0.f, 0.f);
  if (t >= g.lo[0] && t < g.hi[0]) {
    const float2* src = a.Gz + ci * L::GZ + (long long)k3 * N * N + t;
    float2 y[M];
#pragma unroll
    for (int n = 0; n < M; ++n) {
      const float2 u = (n >= g.lo[1] && n < g.hi[1]) ? src[n * N] : z0;
      const float2 v = (n + M >= g.lo[1] && n + M < g.hi[1]) ? src[(n + M) * N] : z0;
      y[n] = dif_in<N>(h, n, u, v);
    }
    fft_reg<M, false>(y);
#pragma unroll
    for (int m = 0; m < M; ++m) S[(2 * m + h) * L::SSTR + t] = y[fpos<M>(m)];
  } else {
#pragma unroll 4
    for (int m = 0; m < M; ++m) S[(2 * m + h) * L::SSTR + t] = z0;
  }
  if (t < L::NF) {
    if (t < a.IS[0]) {
      const float2* src = a.Fz + ci * L::FZ + (long long)k3 * L::NF * L::NF + t;
      float2 y[M];
#pragma unroll
      for (int n = 0; n < M; ++n) {
        const float2 u = (n < L::NF && n < a.IS[1]) ? src[n * L::NF] : z0;
        const float2 v = (n + M < L::NF && n + M < a.IS[1]) ? src[(n + M) * L::NF] : z0;
        y[n] = dif_in<N>(h, n, u, v);
      }
      fft_reg<M, false>(y);
#pragma unroll
      for (int m = 0; m < M; ++m) SF[(2 * m + h) * L::FSTR + t] = y[fpos<M>(m)];
    } else {
#pragma unroll 4
      for (int m = 0; m < M; ++m) SF[(2 * m + h) * L::FSTR + t] = z0;
    }
  }
}

// Phase C1: thread (t, h) transforms column k2 = t of G along dim 1 (row t
// of S holds x1 = 0..N-1); the bins of parity h are kept in y (fpos slots).
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_cols_g(int t, int h, const float2* S, float2 (&y)[N / 2]) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
  const float2* row = S + t * L::SSTR;
#pragma unroll
  for (int n = 0; n < M; ++n) y[n] = dif_in<N>(h, n, row[n], row[n + M]);
  fft_reg<M, false>(y);
}

// Phase C2 (after a barrier): the G bins parked in their own row of S,
// natural bin order k1, so the F transform has the registers to itself.
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_park(int t, int h, float2* S, const float2 (&y)[N / 2]) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
#pragma unroll
  for (int m = 0; m < M; ++m) S[t * L::SSTR + 2 * m + h] = y[fpos<M>(m)];
}

// Phase C3: column t of F along dim 1, conj(F) G over the bins of parity h,
// and its M-point inverse: z_h (fpos slots) of the lags along dim 1.
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_cols_f(int t, int h, const float2* S, const float2* SF, float2 (&p)[N / 2]) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
  const float2 z0 = make_float2(0.f, 0.f);
  const float2* frow = SF + t * L::FSTR;
  float2 y[M];
#pragma unroll
  for (int n = 0; n < M; ++n) y[n] = dif_in<N>(h, n, n < L::NF ? frow[n] : z0, n + M < L::NF ? frow[n + M] : z0);
  fft_reg<M, false>(y);
  const float2* grow = S + t * L::SSTR;
#pragma unroll
  for (int m = 0; m < M; ++m) p[m] = cmulc(y[fpos<M>(m)], grow[2 * m + h]);
  fft_reg<M, true>(p);
}

// Exchange of a pair's inverse halves through column t of T (T aliases S):
// X1 writes z_0[n] (h = 0) or W_N^-n z_1[n] (h = 1) to row n + hM; X2 (after a
// barrier) reads both and keeps x[n + hM] = z_0[n] +- W_N^-n z_1[n]; X3 (after
// a barrier) stores the lags s1 < P1 to T[s1][t].
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_x1(int t, int h, const float2 (&p)[N / 2], float2* T) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
#pragma unroll
  for (int n = 0; n < M; ++n) {
    const float2 w = p[fpos<M>(n)];
    T[(n + h * M) * L::SSTR + t] = h ? rotate<N, true>(w, n) : w;
  }
}
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_x2(int t, int h, const float2* T, float2 (&o)[N / 2]) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
#pragma unroll
  for (int n = 0; n < M; ++n) {
    const float2 a = T[n * L::SSTR + t], b = T[(n + M) * L::SSTR + t];
    o[n] = h ? csub(a, b) : cadd(a, b);
  }
}
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_x3(int t, int h, int P1, const float2 (&o)[N / 2], float2* T) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
#pragma unroll
  for (int n = 0; n < M; ++n)
    if (n + h * M < P1) T[(n + h * M) * L::SSTR + t] = o[n];
}

// Phase R2a: thread (s1 = t < P1, h) takes the bins k2 of parity h of lag row
// s1 and inverts them (M points); R2b (after a barrier) writes its half to
// the row; R2c (after a barrier) combines the halves into lags s2 = n + hM
// and stores those below P2 to C[ci][k3][s2][s1].
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_r2a(int t, int h, int P1, const float2* T, float2 (&u)[N / 2]) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
  if (t >= P1) return;
#pragma unroll
  for (int m = 0; m < M; ++m) u[m] = T[t * L::SSTR + 2 * m + h];
  fft_reg<M, true>(u);
}
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_r2b(int t, int h, int P1, const float2 (&u)[N / 2], float2* T) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
  if (t >= P1) return;
#pragma unroll
  for (int n = 0; n < M; ++n) {
    const float2 w = u[fpos<M>(n)];
    T[t * L::SSTR + n + h * M] = h ? rotate<N, true>(w, n) : w;
  }
}
template <int N, bool FPRUNE>
MQP_HD MQP_FI void k3b_r2c(long long ci, int k3, int t, int h, int P1, int P2, const float2* T, float2* C) {
  using L = Lay3<N, FPRUNE>;
  constexpr int M = N / 2;
  if (t >= P1) return;
  float2* dst = C + ((ci * L::K3 + k3) * P2) * (long long)P1 + t;
#pragma unroll
  for (int n = 0; n < M; ++n) {
    const int s2 = n + h * M;
    if (s2 < P2) {
      const float2 a = T[t * L::SSTR + n], b = T[t * L::SSTR + n + M];
      dst[(long long)s2 * P1] = h ? csub(a, b) : cadd(a, b);
    }
  }
}

// ---------------------------------------------------------------------------
// K3c: inverse along k3, similarity, peak and SN accumulation
// ---------------------------------------------------------------------------
// cc scale: two r2c (x2 each), two unnormalised 2D inverses over N^2 bins and
// the unnormalised inverse along k3
template <int N>
MQP_HD MQP_FI double cc_scale3() { return 1.0 / (4.0 * (double)N * (double)N * (double)N); }

// Complex-to-real inverse along k3 of one lag pair from bins X[0..N/2]:
// x[n] = sum_{k<N} X[k] e^{+2 pi i k n / N} with X[N-k] = conj X[k].
// t[m] = x[2m] + i x[2m+1] on return (slot fpos(m)).  X[0] and X[N/2] are
// real in exact arithmetic; their rounding-level imaginary parts are dropped.
template <int N>
MQP_HD MQP_FI void c2r_k3(const float2* src, long long kstride, float2 (&t)[N / 2]) {
  constexpr int M = N / 2;
  float2 X[M + 1];
#pragma unroll
  for (int k = 0; k <= M; ++k) X[k] = src[k * kstride];
#pragma unroll
  for (int k = 0; k < M; ++k) {
    float2 E, O;
    if (k == 0) {
      E = make_float2(X[0].x + X[M].x, 0.f);
      O = make_float2(X[0].x - X[M].x, 0.f);
    } else {
      const float2 A = X[k], B = cconj(X[M - k]);
      E = cadd(A, B);
      O = rotate<N, true>(csub(A, B), k);
    }
    t[k] = cadd(E, cmul_pi(O));
  }
  fft_reg<M, true>(t);
}

struct LagRanges3 {
  int lo[3], hi[3], shi[3];
};

MQP_HD MQP_FI LagRanges3 lag_ranges3(const Piv3dArgs& a, const IAGeom3& g) {
  LagRanges3 R;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    R.lo[d] = g.tlf[d];
    R.hi[d] = 2 * a.SM[d] - g.brb[d];
    R.shi[d] = 2 * a.SM[d] - 1 - g.brb[d];
  }
  return R;
}

MQP_HD MQP_FI void acc_take3(PeakAcc& acc, const LagRanges3& R, int s1, int s2, int s3, int idx, double v) {
  if (s1 >= R.lo[0] && s2 >= R.lo[1] && s3 >= R.lo[2]) {
    if (s1 <= R.hi[0] && s2 <= R.hi[1] && s3 <= R.hi[2]) peak_take(v, idx, acc.best, acc.bidx);
    if (s1 <= R.shi[0] && s2 <= R.shi[1] && s3 <= R.shi[2]) {
      acc.smax = nmax(acc.smax, v);
      acc.ssum += v;
    }
  }
}

// One lag pair q = s1 + P1 s2: the P3 lags along dim 3, their similarity
// (similarity_value: fftcc.jl:123, zncc_ops.jl:29-50, nsqecc_ops.jl:1-25,
// masked_nsqecc_ops.jl:123-142) with window sums from the integral volumes,
// written to the similarity volume and taken into the accumulators.
template <int N, int ALG>
MQP_HD MQP_FI void k3c_pair(const Piv3dArgs& a, const IAGeom3& g, const IA3State& s, long long ci, int q, int P1,
                            int P2, int P3, const LagRanges3& R, PeakAcc& acc) {
  constexpr int M = N / 2, K3 = M + 1;
  const int s1 = q % P1, s2 = q / P1;
  const long long cs = (long long)P1 * P2;
  float2 t[M];
  c2r_k3<N>(a.C + ci * K3 * cs + q, cs, t);
  float2 t2[M];
  if constexpr (ALG == ALG_MASK_NSQECC) c2r_k3<N>(a.C2 + ci * K3 * cs + q, cs, t2);
  const double scale = cc_scale3<N>();
  const float sqF = sqrtf((float)s.sumF2);
  int r0 = 0, r1 = 0, c0 = 0, c1 = 0;
  if (ALG == ALG_ZNCC || ALG == ALG_NSQECC) {
    lag_window(s1, a.IS[0], g.g0[0], g.lo[0], g.hi[0], r0, r1);
    lag_window(s2, a.IS[1], g.g0[1], g.lo[1], g.hi[1], c0, c1);
  }
  const long long vol = (long long)P1 * P2 * P3;
  float* vdst = a.V + ci * vol + q;
  double* pdst = a.planes ? a.planes + (a.ia_begin + ci - a.planes_begin) * vol + q : nullptr;
#pragma unroll
  for (int s3 = 0; s3 < N; ++s3) {
    if (s3 < P3) {
      const float2 z = t[fpos<M>(s3 >> 1)];
      const double c = (double)((s3 & 1) ? z.y : z.x) * scale;
      double v;
      if constexpr (ALG == ALG_FFTCC) {
        v = c;
      } else if constexpr (ALG == ALG_MASK_NSQECC) {
        const float2 z2 = t2[fpos<M>(s3 >> 1)];
        const double c2 = (double)((s3 & 1) ? z2.y : z2.x) * scale;
        v = similarity_value<ALG_MASK_NSQECC>(IAScalars{s.sumF2, 0.0, 0.0}, sqF, (double)(float)c, c2, 0.0, 0.0);
      } else {
        int z0, z1;
        lag_window(s3, a.IS[2], g.g0[2], g.lo[2], g.hi[2], z0, z1);
        const double S2 = box_sum3(a.IIg2, a.H, a.W, r0, r1, c0, c1, z0, z1);
        double S1 = 0.0, n = 0.0;
        if (ALG == ALG_ZNCC) {
          S1 = box_sum3(a.IIg, a.H, a.W, r0, r1, c0, c1, z0, z1);
          n = (double)(r1 - r0) * (double)(c1 - c0) * (double)(z1 - z0);
        }
        v = similarity_value<ALG>(IAScalars{s.sumF2, s.meanF, s.meanG}, sqF, c, S2, S1, n);
      }
      vdst[(long long)s3 * P1 * P2] = (float)v;
      if (pdst) pdst[(long long)s3 * P1 * P2] = v;
      acc_take3(acc, R, s1, s2, s3, q + P1 * P2 * s3, v);
    }
  }
}

// gaussian_refinement + gaussian_3D (src/utils/piv_ops.jl:282-291, :321-326)
// around the 0-based peak p of value mx in the similarity volume vol
// (element (s1, s2, s3) at s1 + P1 (s2 + P2 s3)).  The minimum runs over the
// whole 3x3x3 neighbourhood.  r is unchanged when the peak touches the
// search range edge.
MQP_HD MQP_FI bool refine3d_values(const float* vol, int P1, int P2, const int SM[3], const IAGeom3& g,
                                   const int p[3], double mx, double (&v)[7], double& mn) {
  bool inside = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) inside = inside && (p[d] + 1 > 1 + g.tlf[d]) && (p[d] + 1 < 1 + 2 * SM[d] - g.brb[d]);
  if (!inside) return false;
  const long long P12 = (long long)P1 * P2;
  const float* c = vol + p[0] + (long long)P1 * p[1] + P12 * p[2];
  const long long stride[3] = {1, P1, P12};
  mn = (double)c[-1 - P1 - P12];
  for (int k = -1; k <= 1; ++k)
    for (int j = -1; j <= 1; ++j)
      for (int i = -1; i <= 1; ++i) mn = nmin(mn, (double)c[i + P1 * j + P12 * k]);
  v[0] = mx;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    v[1 + 2 * d] = (double)c[-stride[d]];
    v[2 + 2 * d] = (double)c[stride[d]];
  }
  return true;
}

// l[0] = log of the peak term, l[1 + 2d] / l[2 + 2d] of the lower / upper
// neighbour along axis d
MQP_HD MQP_FI void refine3d_from_logs(const int p[3], const double (&l)[7], double r[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double lo = l[1 + 2 * d], hi = l[2 + 2 * d];
    r[d] = p[d] + (lo - hi) / (2.0 * lo - 4.0 * l[0] + 2.0 * hi);
  }
}

MQP_HD MQP_FI void refine3d(const float* vol, int P1, int P2, const int SM[3], const IAGeom3& g, const int p[3],
                            double mx, double r[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) r[d] = p[d];
  double v[7], mn;
  if (!refine3d_values(vol, P1, P2, SM, g, p, mx, v, mn)) return;
  double l[7];
  for (int k = 0; k < 7; ++k) l[k] = log(1.0 + v[k] - mn);
  refine3d_from_logs(p, l, r);
}

#if defined(__CUDACC__)
// refine3d for a whole warp (every lane calls it with the same peak): lanes
// 0-6 take one log each; every lane returns refine3d's position.
__device__ __forceinline__ void refine3d_warp(const float* vol, int P1, int P2, const int SM[3], const IAGeom3& g,
                                              const int p[3], double mx, int lane, double r[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) r[d] = p[d];
  double v[7], mn;
  if (!refine3d_values(vol, P1, P2, SM, g, p, mx, v, mn)) return;
  double x = v[0];
#pragma unroll
  for (int k = 1; k < 7; ++k)
    if (lane == k) x = v[k];
  const double mine = lane < 7 ? log(1.0 + x - mn) : 0.0;
  double l[7];
#pragma unroll
  for (int k = 0; k < 7; ++k) l[k] = __shfl_sync(0xffffffffu, mine, k);
  refine3d_from_logs(p, l, r);
}
#endif

// The vector and SN of one IA from the merged accumulators (thread 0 of K3c).
MQP_HD MQP_FI void k3c_final(const Piv3dArgs& a, const IAGeom3& g, long long ci, const LagRanges3& R, double best,
                             int bidx, double smax, double ssum) {
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1, P3 = 2 * a.SM[2] + 1;
  const long long ia = a.ia_begin + ci;
  double r[3];
  if (bidx < 0) {
    r[0] = r[1] = r[2] = -1.0;  // 1-based peak (0, 0, 0): displacement -(SM+1)
  } else {
    const int p[3] = {bidx % P1, (bidx / P1) % P2, bidx / (P1 * P2)};
    refine3d(a.V + ci * (long long)P1 * P2 * P3, P1, P2, a.SM, g, p, best, r);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) a.VF[3 * ia + d] = r[d] - a.SM[d] + g.d[d];
  if (a.SN) {
    // compute_SN (src/utils/piv_ops.jl:336-367) over [TLF_off, 2SM-1-BRB_off];
    // the reference's 2D-only indexing (:357-360) is extended to the third axis
    const double len = (double)(R.shi[0] - R.lo[0] + 1) * (double)(R.shi[1] - R.lo[1] + 1) *
                       (double)(R.shi[2] - R.lo[2] + 1);
    a.SN[ia] = smax / ((ssum - smax) / (len - 1.0));
  }
}

// skipped IA: zero vector, zero SN, zero debug volume
MQP_HD MQP_FI void k3c_skipped(const Piv3dArgs& a, long long ci) {
  const long long ia = a.ia_begin + ci;
  a.VF[3 * ia + 0] = 0.0;
  a.VF[3 * ia + 1] = 0.0;
  a.VF[3 * ia + 2] = 0.0;
  if (a.SN) a.SN[ia] = 0.0;
}

}  // namespace mqp
