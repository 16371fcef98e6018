// Fused 2D PIV: one warp owns one interrogation area (IA) at a time and runs
// the whole per-IA pipeline of multi_quickPIV's PIV_CPU loop body
// (src/multi_quickPIV.jl:63-89) without leaving the SM:
//
//   phase 1  lane-per-row real FFT along dim 2 (r2c of a length-N real row
//            via one N/2-point complex FFT).  The F and G windows are read
//            straight from the images with the reference's clipping and
//            border offset (src/utils/piv_ops.jl:59-127); lanes are
//            consecutive rows, so every warp load is one coalesced segment
//            of a column.  Spectra rows k2 = 0..N/2-1 go to shared memory
//            (k2 = 0 and k2 = N/2 are both real and share slot 0 as
//            (re, im) = (X[0], X[N/2])).
//   phase 2  lane-per-spectrum-row complex FFT along dim 1 of G, of F (as
//            two half transforms, F being zero past IS1), conj(F)*G, inverse
//            FFT along dim 1; only the 2*SM1+1 fully-overlapping lags stay.
//   phase 3  lane-per-lag-row complex-to-real inverse along dim 2 (one
//            N/2-point complex FFT), giving cc[s1,s2] = sum_x F(x)G(x+s)
//            (src/crosscorrelation_algorithms/fftcc.jl:101-126).
//   then     ZNCC/NSQECC normalisation from FP64 integral images
//            (src/utils/zncc_ops.jl:29-50, src/utils/nsqecc_ops.jl:1-25),
//            full-overlap argmax with column-major first-max semantics
//            (src/utils/common_ops.jl:98-124), 3-point Gaussian fit
//            (src/utils/piv_ops.jl:249-326) and SN (:333-367).
//
// The FFT length only has to cover the search window (N >= IS + 2 SM): the
// lags 0..2SM never wrap, so any N gives the same correlation as the
// reference's good_size_real(IS+2SM) transform up to rounding.  N is a power
// of two here.
#pragma once

#include "mqp_fft.cuh"

#include <stdint.h>

namespace mqp {

enum Alg : int { ALG_FFTCC = 0, ALG_ZNCC = 1, ALG_NSQECC = 2, ALG_MASK_NSQECC = 3 };

struct Piv2dArgs {
  const void* img1;
  const void* img2;
  const void* mask;      // masked NSQECC interrogation-area mask (or null)
  int dtype;             // 0 = float32 images, 1 = float64 images
  const double* II1;     // integral of img1 (ZNCC mean of F), (H+1)x(W+1)
  const double* IIg;     // integral of img2 (ZNCC)
  const double* IIg2;    // integral of img2^2 (ZNCC, NSQECC)
  const int32_t* pred;   // whole-pixel predictor (2, vf1, vf2) or null
  double* VF;            // (2, vf1, vf2) column-major
  double* SN;            // (vf1, vf2) or null
  double* planes;        // debug: (P1, P2, n_ia) similarity planes or null
  int H, W;              // image size (dim 1, dim 2)
  int IS1, IS2, SM1, SM2, st1, st2;
  int vf1, vf2;
  long long ia_begin, ia_end;  // IA linear index range processed by this launch
  double threshold;      // skip when max(IA) < threshold (threshold >= 0)
  int computeSN;
  int* status;           // device error flag (non-zero = failure), or null
};

// Geometry of one IA in pad coordinates (0-based).  Pad index p along an
// axis maps to image index g0 + p and holds data iff lo <= p < hi.
struct IAGeom {
  int ir1, ir2;     // IA origin (0-based image coordinates)
  int g01, g02;     // image coordinate of pad index 0
  int lo1, hi1, lo2, hi2;
  int tlf1, tlf2;   // SR_TLF_off (reference, 1-based semantics)
  int brb1, brb2;   // SR_BRB_off
};

struct IAScalars {
  double sumF2;   // sum of squares of the transformed F (ZNCC: mean removed; masked: sum(maskF^2/wi))
  double meanF;   // ZNCC
  double meanG;   // ZNCC
};

// get_interrogation_coordinates + get_search_coordinates
// (src/utils/piv_ops.jl:38-76) for one axis, 1-based like the reference,
// including the short-by-2 TLF offset of :72.  d = whole-pixel predictor
// (already clamped so the moved IA stays inside the image).
MQP_HD MQP_FI void axis_geom(int v, int st, int IS, int SM, int size, int d,
                             int& ir0, int& g0, int& lo, int& hi, int& tlf, int& brb) {
  const int IR_TLF = 1 + v * st;
  const int IR_BRB = IR_TLF + IS - 1;
  const int vT = IR_TLF + d, vB = IR_BRB + d;
  const int SR_TLF = vT - SM > 1 ? vT - SM : 1;
  const int SR_BRB = vB + SM < size ? vB + SM : size;
  tlf = (SM - 1 - vT) > 0 ? (SM - 1 - vT) : 0;   // |min(0, IR_TLF - (SM - 1))|
  brb = (vB + SM - size) > 0 ? (vB + SM - size) : 0;
  const int len = SR_BRB - SR_TLF + 1;
  lo = tlf;
  hi = tlf + (len > 0 ? len : 0);
  g0 = (SR_TLF - 1) - tlf;
  ir0 = IR_TLF - 1;
}

MQP_HD MQP_FI int clamp_pred(int d, int IR_TLF, int IR_BRB, int size) {
  const int lo = 1 - IR_TLF, hi = size - IR_BRB;
  return d < lo ? lo : (d > hi ? hi : d);
}

MQP_HD MQP_FI IAGeom ia_geom(const Piv2dArgs& a, int v1, int v2) {
  IAGeom g;
  int d1 = 0, d2 = 0;
  if (a.pred) {
    const long long base = 2LL * ((long long)v1 + (long long)a.vf1 * v2);
    const int T1 = 1 + v1 * a.st1, T2 = 1 + v2 * a.st2;
    d1 = clamp_pred(a.pred[base + 0], T1, T1 + a.IS1 - 1, a.H);
    d2 = clamp_pred(a.pred[base + 1], T2, T2 + a.IS2 - 1, a.W);
  }
  axis_geom(v1, a.st1, a.IS1, a.SM1, a.H, d1, g.ir1, g.g01, g.lo1, g.hi1, g.tlf1, g.brb1);
  axis_geom(v2, a.st2, a.IS2, a.SM2, a.W, d2, g.ir2, g.g02, g.lo2, g.hi2, g.tlf2, g.brb2);
  return g;
}

MQP_HD MQP_FI void ia_pred(const Piv2dArgs& a, int v1, int v2, int& d1, int& d2) {
  d1 = d2 = 0;
  if (a.pred) {
    const long long base = 2LL * ((long long)v1 + (long long)a.vf1 * v2);
    const int T1 = 1 + v1 * a.st1, T2 = 1 + v2 * a.st2;
    d1 = clamp_pred(a.pred[base + 0], T1, T1 + a.IS1 - 1, a.H);
    d2 = clamp_pred(a.pred[base + 1], T2, T2 + a.IS2 - 1, a.W);
  }
}

MQP_HD MQP_FI double load_px(const void* img, int dtype, long long idx) {
  return dtype == 0 ? (double)((const float*)img)[idx] : ((const double*)img)[idx];
}

// Sum over the image box [r0, r1) x [c0, c1) from an exclusive-prefix
// integral array II of size (H+1) x (W+1), column-major.
MQP_HD MQP_FI double box_sum(const double* II, int H, int r0, int r1, int c0, int c1) {
  if (r1 <= r0 || c1 <= c0) return 0.0;
  const long long ld = (long long)H + 1;
  return (II[r1 + ld * c1] - II[r0 + ld * c1]) - (II[r1 + ld * c0] - II[r0 + ld * c0]);
}

// Shared-memory layout of one warp's IA workspace, in float2 units.
template <int N, bool FPRUNE>
struct Layout2d {
  static constexpr int M = N / 2;                 // spectrum rows after the r2c along dim 1
  static constexpr int GSTR = N + 1;              // odd row stride: conflict-free rows and columns
  static constexpr int NF = FPRUNE ? N / 2 : N;   // stored F columns
  static constexpr int FSTR = NF + 1;
  static constexpr int G_OFF = 0;
  static constexpr int G_SIZE = M * GSTR;
  static constexpr int F_OFF = G_SIZE;
  static constexpr int F_SIZE = M * FSTR;
  // the FP64 similarity plane (P1 x P2 <= N x N) aliases the F rows after phase 2
  static MQP_HD MQP_FI int region2_f2(int P1, int P2) {
    return F_SIZE > P1 * P2 ? F_SIZE : P1 * P2;   // one double == one float2
  }
  static MQP_HD MQP_FI int warp_f2(int P1, int P2) { return G_SIZE + region2_f2(P1, P2); }
};

// ---------------------------------------------------------------------------
// phase 1: real FFT of one window row along dim 2 -> spectra X2 = 2 * DFT
// ---------------------------------------------------------------------------
// z holds the row packed as z[n] = x[2n] + i x[2n+1]; after the M-point FFT
// the r2c split gives X2[k] = (Z[k] + conj Z[M-k]) - i W^k (Z[k] - conj Z[M-k]).
// out[k * stride] receives X2[k] (k = 1..M-1) and out[0] the packed pair
// (X2[0], X2[M]).
template <int N, int NZ>
MQP_HD MQP_FI void r2c_store(float2 (&z)[N / 2], float2* out, int stride) {
  constexpr int M = N / 2;
  fft_reg<M, false, NZ>(z);
  const float2 Z0 = z[fpos<M>(0)];
  out[0] = make_float2(2.f * (Z0.x + Z0.y), 2.f * (Z0.x - Z0.y));
#pragma unroll
  for (int k = 1; k < M; ++k) {
    const float2 A = z[fpos<M>(k)];
    const float2 B = cconj(z[fpos<M>(M - k)]);
    const float2 e = cadd(A, B);
    const float2 o = cmul_mi(csub(A, B));
    out[k * stride] = cadd(e, rotate<N, false>(o, k));
  }
}

template <typename T>
MQP_HD MQP_FI T ldg_px(const void* img, long long i) {
#if defined(__CUDA_ARCH__)
  return __ldg(reinterpret_cast<const T*>(img) + i);
#else
  return reinterpret_cast<const T*>(img)[i];
#endif
}

MQP_HD MQP_FI void zero_strided(float2* base, int rows, int stride) {
  for (int k = 0; k < rows; ++k) base[k * stride] = make_float2(0.f, 0.f);
}

// One row of phase 1.  Row j of the lane's work: j == 0 is row y = lane of
// the interrogation window F (copy_inter_region!, src/utils/piv_ops.jl:99-109,
// minus its mean for ZNCC, src/utils/zncc_ops.jl:7-12), j >= 1 is row
// p = lane + 32 (j - 1) of the padded search window G: pad (p, x2) <-
// img2(g01+p, g02+x2) on the clipped data region and 0 elsewhere
// (copy_search_region!, src/utils/piv_ops.jl:115-127), minus meanG there for
// ZNCC (src/utils/zncc_ops.jl:18-25).  One rolled body serves both so the
// r2c code exists once.  F rows also accumulate the raw max (skip test,
// src/utils/piv_ops.jl:134-146) and the FP64 sum of squares of the
// transformed values (sumF2, zncc.jl:131-135, nsqecc.jl:349-353).
template <int N, bool FPRUNE, typename T, bool ZNCC>
MQP_HD MQP_FI void phase1_row(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, bool isF, int row,
                              float2* GH, float2* FH, double& vmax, double& sumsq) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2* out = isF ? FH + row : GH + row;
  const int stride = isF ? Lay::FSTR : Lay::GSTR;
  float2 z[M];
  if (isF) {
    if (row >= a.IS1) {
      zero_strided(out, M, stride);
      return;
    }
    const long long base = (long long)(g.ir1 + row) + (long long)a.H * g.ir2;
#pragma unroll
    for (int n = 0; n < M; ++n) {
      float v[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int x2 = 2 * n + h;
        v[h] = 0.f;
        if ((!FPRUNE || x2 < M) && x2 < a.IS2) {
          const double r = (double)ldg_px<T>(a.img1, base + (long long)a.H * x2);
          vmax = r > vmax ? r : vmax;
          const double val = r - sc.meanF;
          sumsq += val * val;
          v[h] = (float)val;
        }
      }
      z[n] = make_float2(v[0], v[1]);
    }
  } else {
    if (row < g.lo1 || row >= g.hi1) {
      zero_strided(out, M, stride);
      return;
    }
    const long long base = (long long)(g.g01 + row) + (long long)a.H * g.g02;
    const float meanG = ZNCC ? (float)sc.meanG : 0.f;
#pragma unroll
    for (int n = 0; n < M; ++n) {
      float v[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int x2 = 2 * n + h;
        v[h] = 0.f;
        if (x2 >= g.lo2 && x2 < g.hi2) {
          const float r = (float)ldg_px<T>(a.img2, base + (long long)a.H * x2);
          v[h] = ZNCC ? r - meanG : r;
        }
      }
      z[n] = make_float2(v[0], v[1]);
    }
  }
  r2c_store<N, M>(z, out, stride);
}

// ---------------------------------------------------------------------------
// phase 2: along dim 1 for one spectrum row u (u = 0 is the packed real pair)
// ---------------------------------------------------------------------------
// F row u as an N/2-point transform of its even (ODD = 0) or odd (ODD = 1)
// output bins: F is zero past NF entries, and for the full width the two
// halves are folded first (the first DIF stage of the N-point transform).
template <int N, bool FPRUNE, int ODD>
MQP_HD MQP_FI void load_F_half(const float2* Frow, float2 (&f)[N / 2]) {
  constexpr int M = N / 2;
#pragma unroll
  for (int n = 0; n < M; ++n) {
    float2 v = Frow[n];
    if (!FPRUNE) {
      const float2 w = Frow[n + M];
      v = ODD ? csub(v, w) : cadd(v, w);
    }
    f[n] = ODD ? rotate<N, false>(v, n) : v;
  }
  fft_reg<M, false>(f);
}

// conj(F)*G over the bins k = 2m + ODD of spectrum row u into p (natural
// order).  Row 0 carries two real rows A + iB (k2 = 0 and k2 = N/2): their
// spectra are A^ = (Z[k] + conj Z[-k]) / 2 and B^ = -i (Z[k] - conj Z[-k]) / 2,
// and the two Hermitian products return together as PA + i PB.
template <int N, int ODD>
MQP_HD MQP_FI void row_product(bool packed, const float2 (&g)[N], const float2 (&f)[N / 2], float2 (&p)[N]) {
  constexpr int M = N / 2;
  if (!packed) {
#pragma unroll
    for (int m = 0; m < M; ++m) p[2 * m + ODD] = cmulc(f[fpos<M>(m)], g[fpos<N>(2 * m + ODD)]);
  } else {
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int k = 2 * m + ODD;
      const int nk = (N - k) & (N - 1);
      if (nk < k) continue;  // written together with its mirror
      const int nm = nk >> 1;  // the mirror bin has the same parity
      const float2 Zk = g[fpos<N>(k)], Zn = cconj(g[fpos<N>(nk)]);
      const float2 Fk = f[fpos<M>(m)], Fn = cconj(f[fpos<M>(nm)]);
      const float2 A = cscale(cadd(Zk, Zn), 0.5f), B = cscale(cmul_mi(csub(Zk, Zn)), 0.5f);
      const float2 Af = cscale(cadd(Fk, Fn), 0.5f), Bf = cscale(cmul_mi(csub(Fk, Fn)), 0.5f);
      const float2 PA = cmulc(Af, A), PB = cmulc(Bf, B);
      p[k] = cadd(PA, cmul_pi(PB));
      if (nk != k) p[nk] = cadd(cconj(PA), cmul_pi(cconj(PB)));
    }
  }
}

template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase2_row(int u, int P1, float2* GH, const float2* FH) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2* Grow = GH + u * Lay::GSTR;
  const float2* Frow = FH + u * Lay::FSTR;
  const bool packed = (u == 0);
  float2 g[N];
#pragma unroll
  for (int n = 0; n < N; ++n) g[n] = Grow[n];
  fft_reg<N, false>(g);
  float2 p[N];
  {
    float2 f[M];
    load_F_half<N, FPRUNE, 0>(Frow, f);
    row_product<N, 0>(packed, g, f, p);
  }
  {
    float2 f[M];
    load_F_half<N, FPRUNE, 1>(Frow, f);
    row_product<N, 1>(packed, g, f, p);
  }
  fft_reg<N, true>(p);
#pragma unroll
  for (int s = 0; s < N; ++s)
    if (s < P1) Grow[s] = p[fpos<N>(s)];
}

// ---------------------------------------------------------------------------
// phase 3: complex-to-real along dim 2 for lag row s1 -> cc[s2], s2 < N
// ---------------------------------------------------------------------------
template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase3_row(int s1, const float2* GH, float (&cc)[N]) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2 X[M];
#pragma unroll
  for (int k = 0; k < M; ++k) X[k] = GH[k * Lay::GSTR + s1];
  const float X0 = X[0].x, XM = X[0].y;  // the packed real bins X[0], X[N/2]
  float2 x[M];
#pragma unroll
  for (int k = 0; k < M; ++k) {
    float2 E, O;
    if (k == 0) {
      E = make_float2(X0 + XM, 0.f);
      O = make_float2(X0 - XM, 0.f);
    } else {
      const float2 A = X[k];
      const float2 B = cconj(X[M - k]);
      E = cadd(A, B);
      O = rotate<N, true>(csub(A, B), k);
    }
    x[k] = cadd(E, cmul_pi(O));
  }
  fft_reg<M, true>(x);
#pragma unroll
  for (int n = 0; n < M; ++n) {
    const float2 v = x[fpos<M>(n)];
    cc[2 * n] = v.x;
    cc[2 * n + 1] = v.y;
  }
}

// Lag row s1 >= 32 (only when 2*SM1+1 > 32) computed by the whole warp: lane
// l evaluates lags s2 = l, l+32, ... of the Hermitian inverse
//   x[s2] = X[0] + (-1)^s2 X[N/2] + 2 sum_{k=1}^{N/2-1} Re(X[k] e^{+2 pi i k s2 / N})
// directly (one row of phase 3 costs a full transform per lane otherwise).
// tw: (cos, sin)(2 pi j / N) for j < N, in shared memory.
template <int N, bool FPRUNE>
MQP_HD MQP_FI float tail_row_value(const float2* GH, const float2* tw, int s1, int s2) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  const float2 X0 = GH[s1];
  float acc = 0.f;
  int t = 0;
#pragma unroll 4
  for (int k = 1; k < M; ++k) {
    t = (t + s2) & (N - 1);
    const float2 X = GH[k * Lay::GSTR + s1];
    const float2 w = tw[t];
    acc += X.x * w.x - X.y * w.y;
  }
  return X0.x + ((s2 & 1) ? -X0.y : X0.y) + 2.f * acc;
}

// cc scale: r2c (x2 per transform, F and G) and the two unnormalised inverses
template <int N>
MQP_HD MQP_FI double cc_scale() { return 1.0 / (4.0 * (double)N * (double)N); }

// ---------------------------------------------------------------------------
// per-IA scalars and the similarity of one lag column
// ---------------------------------------------------------------------------

// Image row (or column) range covered by the interrogation-sized window at
// lag s, clipped to the data of the padded search window.
MQP_HD MQP_FI void lag_window(int s, int IS, int g0, int lo, int hi, int& r0, int& r1) {
  const int a = s > lo ? s : lo;
  const int b = (s + IS) < hi ? (s + IS) : hi;
  r0 = g0 + a;
  r1 = g0 + (b > a ? b : a);
}

// Similarity of lag row s1, in place over plane[s1 + P1*s2] (s2 < P2),
// which holds the raw correlation c = sum_x F(x) G(x+s):
//   FFTCC  c                                           (fftcc.jl:123)
//   ZNCC   c / (sqrt(sum_win G'^2) sqrt(sumF2))        (zncc_ops.jl:29-50)
//   NSQECC den / (den + num), num = sumF2 + sum_win G^2 - 2c,
//          den = sqrt(sum_win G^2) sqrt(sumF2)          (nsqecc_ops.jl:1-25)
// The window sums come from FP64 integral images of img2 / img2^2 (lanes are
// consecutive lag rows, so each lookup is a coalesced column segment) and
// the numerator is formed in FP64 (it cancels near a match); the square
// roots and the final quotient are FP32, whose ~1e-7 relative error is
// below the FP32 correlation's own.
template <int ALG>
MQP_HD MQP_FI void similarity_row(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, int s1, int P1,
                                  int P2, double* plane) {
  if (ALG == ALG_FFTCC) return;
  int r0, r1;
  lag_window(s1, a.IS1, g.g01, g.lo1, g.hi1, r0, r1);
  const float sqF = sqrtf((float)sc.sumF2);
  const long long ld = (long long)a.H + 1;
  const bool rows = r1 > r0;
  for (int s2 = 0; s2 < P2; ++s2) {
    int c0, c1;
    lag_window(s2, a.IS2, g.g02, g.lo2, g.hi2, c0, c1);
    double S2 = 0.0, S1 = 0.0;
    if (rows && c1 > c0) {
      const double* A0 = a.IIg2 + ld * c0;
      const double* A1 = a.IIg2 + ld * c1;
      S2 = (A1[r1] - A1[r0]) - (A0[r1] - A0[r0]);
      if (ALG == ALG_ZNCC) {
        const double* B0 = a.IIg + ld * c0;
        const double* B1 = a.IIg + ld * c1;
        S1 = (B1[r1] - B1[r0]) - (B0[r1] - B0[r0]);
      }
    }
    double& v = plane[s1 + P1 * s2];
    const double c = v;
    if (ALG == ALG_NSQECC) {
      const double num = (sc.sumF2 - 2.0 * c) + S2;
      const float den = sqrtf((float)S2) * sqF;
      v = (double)(den / (float)(num + (double)den));
    } else {
      const double n = (double)(r1 - r0) * (double)(c1 - c0);
      double SG = S2 - 2.0 * sc.meanG * S1 + n * sc.meanG * sc.meanG;
      SG = SG > 0.0 ? SG : 0.0;
      v = (double)((float)c / (sqrtf((float)SG) * sqF));
    }
  }
}

// similarity_row for one element (s1, s2): the tail rows use it with the
// lanes spread over s2.
template <int ALG>
MQP_HD MQP_FI double similarity_one(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, int s1, int s2,
                                    double c) {
  if (ALG == ALG_FFTCC) return c;
  int r0, r1, c0, c1;
  lag_window(s1, a.IS1, g.g01, g.lo1, g.hi1, r0, r1);
  lag_window(s2, a.IS2, g.g02, g.lo2, g.hi2, c0, c1);
  const double S2 = box_sum(a.IIg2, a.H, r0, r1, c0, c1);
  const float sqF = sqrtf((float)sc.sumF2);
  if (ALG == ALG_NSQECC) {
    const double num = (sc.sumF2 - 2.0 * c) + S2;
    const float den = sqrtf((float)S2) * sqF;
    return (double)(den / (float)(num + (double)den));
  }
  const double S1 = box_sum(a.IIg, a.H, r0, r1, c0, c1);
  const double n = (double)(r1 - r0) * (double)(c1 - c0);
  double SG = S2 - 2.0 * sc.meanG * S1 + n * sc.meanG * sc.meanG;
  SG = SG > 0.0 ? SG : 0.0;
  return (double)((float)c / (sqrtf((float)SG) * sqF));
}

// NaN-propagating max / min (Julia's maximum / minimum)
MQP_HD MQP_FI double nmax(double m, double v) { return (v > m || v != v) ? v : m; }
MQP_HD MQP_FI double nmin(double m, double v) { return (v < m || v != v) ? v : m; }

// gaussian_refinement + gaussian_2D (src/utils/piv_ops.jl:282-319) around the
// 0-based peak (p1, p2) of value mx in the P1-row plane; returns the refined
// 0-based position (unchanged when the peak touches the search range edge).
MQP_HD MQP_FI void refine2d(const double* plane, int P1, int SM1, int SM2, const IAGeom& g,
                            int p1, int p2, double mx, double& r1, double& r2) {
  r1 = p1;
  r2 = p2;
  // reference test in 1-based indices: peak > 1 + TLF_off and peak < 1 + 2SM - BRB_off
  const bool inside = (p1 + 1 > 1 + g.tlf1) && (p2 + 1 > 1 + g.tlf2) &&
                      (p1 + 1 < 1 + 2 * SM1 - g.brb1) && (p2 + 1 < 1 + 2 * SM2 - g.brb2);
  if (!inside) return;
  double mn = plane[(p1 - 1) + P1 * (p2 - 1)];
  for (int j = -1; j <= 1; ++j)
    for (int i = -1; i <= 1; ++i) mn = nmin(mn, plane[(p1 + i) + P1 * (p2 + j)]);
  const double lmx = log(1.0 + mx - mn);
  const double up = log(1.0 + plane[(p1 - 1) + P1 * p2] - mn);
  const double down = log(1.0 + plane[(p1 + 1) + P1 * p2] - mn);
  const double left = log(1.0 + plane[p1 + P1 * (p2 - 1)] - mn);
  const double right = log(1.0 + plane[p1 + P1 * (p2 + 1)] - mn);
  r1 = p1 + (up - down) / (2.0 * up - 4.0 * lmx + 2.0 * down);
  r2 = p2 + (left - right) / (2.0 * left - 4.0 * lmx + 2.0 * right);
}

// lane-local part of first_fullovp_peak (src/utils/common_ops.jl:98-124).
// The reference keeps the first maximum > 0 of a column-major scan; every
// lane keeps the (largest value, lowest column-major index) of the elements
// it owns, starting from (0, none), and merging lanes by the same rule gives
// the same element whatever the split.
MQP_HD MQP_FI void peak_take(double v, int idx, double& best, int& bidx) {
  // larger value, or the same value earlier in column-major order
  if (v > best || (v == best && idx < bidx)) {
    best = v;
    bidx = idx;
  }
}

MQP_HD MQP_FI void peak_scan_row(const double* plane, int P1, int s1, int lo2, int hi2, double& best,
                                 int& bidx) {
  for (int s2 = lo2; s2 <= hi2; ++s2) peak_take(plane[s1 + P1 * s2], s1 + P1 * s2, best, bidx);
}

// merge two (value, first index) candidates: larger value, then smaller index
MQP_HD MQP_FI void peak_merge(double& best, int& bidx, double ob, int oi) {
  if (oi < 0) return;
  if (bidx < 0 || ob > best || (ob == best && oi < bidx)) {
    best = ob;
    bidx = oi;
  }
}

}  // namespace mqp
