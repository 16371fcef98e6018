// Fused 2D PIV: one warp owns one interrogation area (IA) at a time and runs
// the whole per-IA pipeline of multi_quickPIV's PIV_CPU loop body
// (src/multi_quickPIV.jl:63-89) without leaving the SM:
//
//   phase 1  lane-per-column real FFT along dim 1 (r2c of a length-N1 real
//            column via one N1/2-point complex FFT), F and G windows loaded
//            straight from the images with the reference's clipping and
//            border offset (src/utils/piv_ops.jl:59-127), written to shared
//            memory as spectra rows k1 = 0..N1/2-1 (rows 0 and N1/2 are both
//            real and share slot 0 as (re, im) = (X[0], X[N1/2])).
//   phase 2  lane-per-row complex FFT along dim 2 of G, of F (as two half
//            transforms, F being zero past IS2), conj(F)*G, inverse FFT
//            along dim 2; only the 2*SM2+1 fully-overlapping lags are kept.
//   phase 3  lane-per-lag-column complex-to-real inverse along dim 1 (one
//            N1/2-point complex FFT), giving cc[s1,s2] = sum_x F(x)G(x+s)
//            (src/crosscorrelation_algorithms/fftcc.jl:101-126).
//   then     ZNCC/NSQECC normalisation from FP64 integral arrays
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
// phase 1: real FFT of one column along dim 1 -> rows of X2 = 2 * DFT
// ---------------------------------------------------------------------------
// z holds the column packed as z[n] = x[2n] + i x[2n+1]; after the M-point
// FFT the r2c split gives X2[k] = (Z[k] + conj Z[M-k]) - i W^k (Z[k] - conj Z[M-k]).
template <int N, int NZ>
MQP_HD MQP_FI void r2c_column_store(float2 (&z)[N / 2], float2* col, int stride) {
  constexpr int M = N / 2;
  fft_reg<M, false, NZ>(z);
  const float2 Z0 = z[fpos<M>(0)];
  // slot 0 packs the two real bins X2[0] = 2(Re+Im) and X2[M] = 2(Re-Im)
  col[0] = make_float2(2.f * (Z0.x + Z0.y), 2.f * (Z0.x - Z0.y));
#pragma unroll
  for (int k = 1; k < M; ++k) {
    const float2 A = z[fpos<M>(k)];
    const float2 B = cconj(z[fpos<M>(M - k)]);
    const float2 e = cadd(A, B);
    const float2 o = cmul_mi(csub(A, B));
    col[k * stride] = cadd(e, rotate<N, false>(o, k));
  }
}

// F column x2 of the IA (x2 < IS2), optionally minus a mean (ZNCC) and times
// a mask (masked NSQECC).  Returns the column's max raw value and
// accumulates sum of squares of the (mean-removed / masked) values.
template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase1_F_column(const Piv2dArgs& a, const IAGeom& g, int x2, double meanF,
                                   bool use_mask, float2* FH, double& vmax, double& sumsq,
                                   double& msum) {
  constexpr int M = N / 2;
  constexpr int NZ = FPRUNE ? M / 2 : M;
  float2 z[M];
  const long long colbase = (long long)(g.ir1) + (long long)a.H * (g.ir2 + x2);
#pragma unroll
  for (int n = 0; n < M; ++n) {
    float v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int y = 2 * n + h;
      v[h] = 0.f;
      if ((!FPRUNE || y < M) && y < a.IS1) {
        const double raw = load_px(a.img1, a.dtype, colbase + y);
        vmax = raw > vmax ? raw : vmax;
        double val = raw - meanF;
        if (use_mask) {
          const double w = load_px(a.mask, a.dtype, colbase + y);
          val = raw * w;
          // sum(maskF^2 / wi), wi = mask if mask > 0 else 1 (mask_nsqecc.jl:145-149)
          sumsq += val * val / (w > 0 ? w : 1.0);
          msum += w;
        } else {
          sumsq += val * val;
        }
        v[h] = (float)val;
      }
    }
    z[n] = make_float2(v[0], v[1]);
  }
  r2c_column_store<N, NZ>(z, FH + x2, Layout2d<N, FPRUNE>::FSTR);
}

// mask column x2 of the IA as its own transform input (masked NSQECC's second
// correlation, mask_nsqecc.jl:155)
template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase1_mask_column(const Piv2dArgs& a, const IAGeom& g, int x2, float2* FH) {
  constexpr int M = N / 2;
  constexpr int NZ = FPRUNE ? M / 2 : M;
  float2 z[M];
  const long long colbase = (long long)(g.ir1) + (long long)a.H * (g.ir2 + x2);
#pragma unroll
  for (int n = 0; n < M; ++n) {
    float v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int y = 2 * n + h;
      v[h] = ((!FPRUNE || y < M) && y < a.IS1) ? (float)load_px(a.mask, a.dtype, colbase + y) : 0.f;
    }
    z[n] = make_float2(v[0], v[1]);
  }
  r2c_column_store<N, NZ>(z, FH + x2, Layout2d<N, FPRUNE>::FSTR);
}

// G column x2 of the padded search window (pad index x2), minus meanG on the
// valid region for ZNCC (zncc_ops.jl:18-25), squared for masked NSQECC's G^2.
template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase1_G_column(const Piv2dArgs& a, const IAGeom& g, int x2, double meanG,
                                   bool square, float2* GH) {
  constexpr int M = N / 2;
  float2 z[M];
  const bool colok = (x2 >= g.lo2) && (x2 < g.hi2);
  const long long colbase = (long long)g.g01 + (long long)a.H * (g.g02 + x2);
#pragma unroll
  for (int n = 0; n < M; ++n) {
    float v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = 2 * n + h;
      v[h] = 0.f;
      if (colok && p >= g.lo1 && p < g.hi1) {
        double raw = load_px(a.img2, a.dtype, colbase + p);
        if (square) raw = raw * raw;
        v[h] = (float)(raw - meanG);
      }
    }
    z[n] = make_float2(v[0], v[1]);
  }
  r2c_column_store<N, M>(z, GH + x2, Layout2d<N, FPRUNE>::GSTR);
}

MQP_HD MQP_FI void zero_column(float2* base, int rows, int stride) {
  for (int k = 0; k < rows; ++k) base[k * stride] = make_float2(0.f, 0.f);
}

// ---------------------------------------------------------------------------
// phase 2: along dim 2 for one spectrum row u (u = 0 is the packed real pair)
// ---------------------------------------------------------------------------
// Loads F row u into fe (even output bins) or fo (odd output bins) as an
// N/2-point transform: F is zero past NF columns, and for the full width the
// two halves are folded first (the first DIF stage of the N-point transform).
template <int N, bool FPRUNE, bool ODD>
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

template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase2_row(int u, int P2, float2* GH, const float2* FH) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2* Grow = GH + u * Lay::GSTR;
  const float2* Frow = FH + u * Lay::FSTR;
  float2 g[N];
#pragma unroll
  for (int n = 0; n < N; ++n) g[n] = Grow[n];
  fft_reg<N, false>(g);
  float2 p[N];
  if (u != 0) {
    float2 f[M];
    load_F_half<N, FPRUNE, false>(Frow, f);
#pragma unroll
    for (int m = 0; m < M; ++m) p[2 * m] = cmulc(f[fpos<M>(m)], g[fpos<N>(2 * m)]);
    load_F_half<N, FPRUNE, true>(Frow, f);
#pragma unroll
    for (int m = 0; m < M; ++m) p[2 * m + 1] = cmulc(f[fpos<M>(m)], g[fpos<N>(2 * m + 1)]);
  } else {
    // rows k1 = 0 (A, real) and k1 = N1/2 (B, real) travel as A + iB:
    // A^ = (Z[k] + conj Z[-k]) / 2, B^ = -i (Z[k] - conj Z[-k]) / 2, and the
    // two products return as one inverse of PA + i PB (PA, PB Hermitian).
    float2 f[M];
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
      if (pass == 0) load_F_half<N, FPRUNE, false>(Frow, f);
      else load_F_half<N, FPRUNE, true>(Frow, f);
#pragma unroll
      for (int k = pass; k < N; k += 2) {
        const int nk = (N - k) & (N - 1);
        if (nk < k) continue;  // handled with its mirror
        const int m = k >> 1, nm = nk >> 1;
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
  fft_reg<N, true>(p);
#pragma unroll
  for (int s = 0; s < N; ++s)
    if (s < P2) Grow[s] = p[fpos<N>(s)];
}

// ---------------------------------------------------------------------------
// phase 3: complex-to-real along dim 1 for lag column s2 -> cc[0..P1) * scale
// ---------------------------------------------------------------------------
template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase3_column(int s2, const float2* GH, float (&cc)[N]) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2 x[M];
  float2 X[M];
#pragma unroll
  for (int k = 0; k < M; ++k) X[k] = GH[k * Lay::GSTR + s2];
  const float X0 = X[0].x, XM = X[0].y;  // the packed real bins X[0], X[N/2]
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

// cc scale: r2c (x2 per transform, F and G) and the two unnormalised inverses
template <int N>
MQP_HD MQP_FI double cc_scale() { return 1.0 / (4.0 * (double)N * (double)N); }

// ---------------------------------------------------------------------------
// per-IA scalars and the similarity of one lag column
// ---------------------------------------------------------------------------
struct IAScalars {
  double sumF2;   // sum of squares of the transformed F (ZNCC: mean removed; masked: sum(maskF^2/wi))
  double meanF;   // ZNCC
  double meanG;   // ZNCC
};

// Image row (or column) range covered by the interrogation-sized window at
// lag s, clipped to the data of the padded search window.
MQP_HD MQP_FI void lag_window(int s, int IS, int g0, int lo, int hi, int& r0, int& r1) {
  const int a = s > lo ? s : lo;
  const int b = (s + IS) < hi ? (s + IS) : hi;
  r0 = g0 + a;
  r1 = g0 + (b > a ? b : a);
}

// Similarity of lag (s1, s2) from the raw correlation c:
//   FFTCC  c                                           (fftcc.jl:123)
//   ZNCC   c / (sqrt(sum_win G'^2) sqrt(sumF2))        (zncc_ops.jl:29-50)
//   NSQECC den / (den + num), num = sumF2 + sum_win G^2 - 2c,
//          den = sqrt(sum_win G^2) sqrt(sumF2)          (nsqecc_ops.jl:1-25)
// The window sums come from FP64 integral images of img2 / img2^2.
template <int ALG>
MQP_HD MQP_FI double similarity(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc,
                                int s1, int s2, double c) {
  if (ALG == ALG_FFTCC) return c;
  int r0, r1, c0, c1;
  lag_window(s1, a.IS1, g.g01, g.lo1, g.hi1, r0, r1);
  lag_window(s2, a.IS2, g.g02, g.lo2, g.hi2, c0, c1);
  const double S2 = box_sum(a.IIg2, a.H, r0, r1, c0, c1);
  if (ALG == ALG_NSQECC) {
    double num = c * -2.0;
    num = num + sc.sumF2;
    num = num + S2;
    const double den = sqrt(S2) * sqrt(sc.sumF2);
    return den / (num + den);
  }
  // ZNCC: sum over the window of (G - meanG)^2 on its data part
  const double S1 = box_sum(a.IIg, a.H, r0, r1, c0, c1);
  const double n = (double)(r1 - r0) * (double)(c1 - c0);
  double SG = S2 - 2.0 * sc.meanG * S1 + n * sc.meanG * sc.meanG;
  SG = SG > 0.0 ? SG : 0.0;
  return c / (sqrt(SG) * sqrt(sc.sumF2));
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

// lane-local part of first_fullovp_peak (src/utils/common_ops.jl:98-124): strict
// '>' from 0 over the lane's lag columns in column-major order.
MQP_HD MQP_FI void peak_scan_column(const double* plane, int P1, int s2, int lo1, int hi1,
                                    double& best, int& bidx) {
  for (int s1 = lo1; s1 <= hi1; ++s1) {
    const double v = plane[s1 + P1 * s2];
    if (v > best) {
      best = v;
      bidx = s1 + P1 * s2;
    }
  }
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
