// Direct (spatial) correlation for small windows, 2D and 3D: one warp per
// interrogation area (IA).  For the small windows of fine multi-pass levels
// (interSize 4-8) the spatial sum cc[s] = sum_x F(x) G(x+s) over the
// fully-overlapping lags s in [0, 2SM] costs fewer operations than any FFT
// the lags need (2D interSize 8, searchMargin 4: 64 x 81 = 5,184 multiply-adds
// against ~15k flops of a 16-point 2D FFT correlation and ~80k of the 32-point
// one the FFT kernels use), so these windows skip the transform.  The values
// are the same correlation the reference's _FFTCC! computes
// (src/crosscorrelation_algorithms/fftcc.jl:101-126), summed in FP32 (each
// lag's sum rounds once per term instead of through an FFT); the
// normalisation, peak, SN and Gaussian fit are the FFT kernels' own
// functions.
//
// Per warp, in shared memory: F (IS1 x IS2 [x IS3]) and the zero-padded
// search window G (SS1 x SS2 [x SS3]) as FP32, with the reference's clipping
// and border offset (Q1), ZNCC mean subtraction, mask products; the lag plane
// (FP64, 2D) or lag volume (FP32, 3D).
#pragma once

#include "mqp_piv2d.cuh"
#include "mqp_piv3d.cuh"

namespace mqp {

// ---- 2D ----------------------------------------------------------------------
constexpr int D2_MAXF = 256;   // IS1 * IS2
constexpr int D2_MAXG = 1056;  // SS1 * (SS2 | 1), SS <= 32
constexpr int D2_MAXP = 289;   // P1 * P2

// Direct correlation is chosen when its multiply-adds per IA are few.
MQP_HD MQP_FI bool direct2d_ok(int IS1, int IS2, int SM1, int SM2) {
  const int SS1 = IS1 + 2 * SM1, SS2 = IS2 + 2 * SM2, P1 = 2 * SM1 + 1, P2 = 2 * SM2 + 1;
  return IS1 * IS2 <= D2_MAXF && SS1 <= 32 && SS2 <= 32 && P1 * P2 <= D2_MAXP &&
         (long long)IS1 * IS2 * P1 * P2 <= 16384;
}

// Per-warp workspace (in 4-byte words): F | G (rows of SS2 | 1) | FP64 plane |
// FP32 parked first correlation (masked NSQECC), sized for the problem.
struct D2Off {
  int F, G, plane, c1, words;
};
MQP_HD MQP_FI D2Off d2_off(int IS1, int IS2, int SM1, int SM2) {
  const int SS1 = IS1 + 2 * SM1, GS = (IS2 + 2 * SM2) | 1, np = (2 * SM1 + 1) * (2 * SM2 + 1);
  D2Off o;
  o.F = 0;
  o.G = IS1 * IS2;
  o.plane = (o.G + SS1 * GS + 1) & ~1;  // 8-byte aligned
  o.c1 = o.plane + 2 * np;
  o.words = (o.c1 + np + 1) & ~1;
  return o;
}

// Lane's share of the F and G loads for one pass (row_process's values: F
// minus the IA mean for ZNCC, F*mask / mask for masked NSQECC; G on its data
// region, minus the search mean for ZNCC, squared for the masked second
// correlation).  Accumulates the skip maxima and sumF2.  G row stride GS.
template <typename T, int ALG>
MQP_HD MQP_FI void direct2d_load(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, int PASS, int lane,
                                 int nl, float* F, float* G, double& vmax, double& mmax, double& sumsq) {
  const int IS1 = a.IS1, IS2 = a.IS2, SS1 = a.IS1 + 2 * a.SM1, SS2 = a.IS2 + 2 * a.SM2, GS = SS2 | 1;
  for (int i = lane; i < IS1 * IS2; i += nl) {
    const int x1 = i % IS1, x2 = i / IS1;
    const long long off = (long long)(g.ir1 + x1) + (long long)a.H * (g.ir2 + x2);
    float w;
    if (PASS == PASS_PLAIN) {
      const T r = ldg_px<T>(a.img1, off);
      vmax = (double)r > vmax ? (double)r : vmax;
      const double val = (double)r - sc.meanF;
      sumsq += val * val;
      w = (float)val;
    } else if (PASS == PASS_MASKED) {
      const T r = ldg_px<T>(a.img1, off);
      const T mk = ldg_px<T>(a.mask, off);
      const T ms = ldg_px<T>(a.mask_skip ? a.mask_skip : a.mask, off);
      vmax = (double)r > vmax ? (double)r : vmax;
      mmax = (double)ms > mmax ? (double)ms : mmax;
      const double val = (double)r * (double)mk;
      sumsq += val * val / ((double)mk > 0.0 ? (double)mk : 1.0);
      w = (float)val;
    } else {
      w = (float)ldg_px<T>(a.mask, off);
    }
    F[x1 * IS2 + x2] = w;
  }
  const float mg = (float)sc.meanG;
  for (int i = lane; i < SS1 * SS2; i += nl) {
    const int p1 = i % SS1, p2 = i / SS1;
    float v = 0.f;
    if (p1 >= g.lo1 && p1 < g.hi1 && p2 >= g.lo2 && p2 < g.hi2) {
      v = (float)ldg_px<T>(a.img2, (long long)(g.g01 + p1) + (long long)a.H * (g.g02 + p2));
      if (ALG == ALG_ZNCC) v = v - mg;
      if (PASS == PASS_MASK_SQ) v = v * v;
    }
    G[p1 * GS + p2] = v;
  }
}

// Similarity of lag q = s1 P2 + s2 from its raw correlation(s), in place in
// the plane, taken into the peak / SN accumulators (finish_one: the same
// values finish_row gives the FFT kernels' rows).
template <int ALG>
MQP_HD MQP_FI void direct2d_finish_lag(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, int q, int P1,
                                       int P2, double* plane, const float* c1, const LagRanges& R, PeakAcc& acc) {
  const int s1 = q / P2, s2 = q - s1 * P2;
  const double v = finish_one<ALG>(a, g, sc, s1, s2, plane[q], ALG == ALG_MASK_NSQECC ? (double)c1[q] : 0.0);
  plane[q] = v;
  acc_take(acc, R, s1, s2, P1, v);
}

// Lane's lags: plane[s1 * P2 + s2] = sum_x F(x) G(x + s).
MQP_HD MQP_FI void direct2d_lags(const Piv2dArgs& a, int lane, int nl, const float* F, const float* G, double* plane) {
  const int IS1 = a.IS1, IS2 = a.IS2, GS = (a.IS2 + 2 * a.SM2) | 1;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  for (int q = lane; q < P1 * P2; q += nl) {
    const int s1 = q % P1, s2 = q / P1;
    float acc = 0.f;
    for (int x1 = 0; x1 < IS1; ++x1) {
      const float* f = F + x1 * IS2;
      const float* gr = G + (x1 + s1) * GS + s2;
      for (int x2 = 0; x2 < IS2; ++x2) acc = fmaf(f[x2], gr[x2], acc);
    }
    plane[s1 * P2 + s2] = (double)acc;
  }
}

// ---- 3D ----------------------------------------------------------------------
constexpr int D3_MAXF = 512;   // IS1 * IS2 * IS3
constexpr int D3_MAXG = 4096;  // SS1 * SS2 * SS3, SS <= 16
constexpr int D3_MAXP = 729;   // P1 * P2 * P3

MQP_HD MQP_FI bool direct3d_ok(const int IS[3], const int SM[3]) {
  long long nf = 1, ng = 1, np = 1;
  for (int d = 0; d < 3; ++d) {
    const int SS = IS[d] + 2 * SM[d];
    if (SS > 16) return false;
    nf *= IS[d];
    ng *= SS;
    np *= 2 * SM[d] + 1;
  }
  return nf <= D3_MAXF && ng <= D3_MAXG && np <= D3_MAXP && nf * np <= (1 << 19);
}

// Workspace of one IA (4-byte words): F | G | similarity volume | parked
// first correlation (masked NSQECC), sized for the problem.  G's planes along
// dim 3 are R2 words apart, R2 = S1 S2 padded to P1 modulo 32: the threads of
// a warp that read G at lags s1 + P1 s3 = 32 consecutive tasks then hit 32
// distinct banks.
struct D3Off {
  int F, G, V, c1, words, R2;
};
MQP_HD MQP_FI D3Off d3_off(const int IS[3], const int SM[3]) {
  int nf = 1, np = 1;
  for (int d = 0; d < 3; ++d) {
    nf *= IS[d];
    np *= 2 * SM[d] + 1;
  }
  const int S0 = IS[0] + 2 * SM[0], S1 = IS[1] + 2 * SM[1], S2 = IS[2] + 2 * SM[2];
  const int P1 = 2 * SM[0] + 1;
  D3Off o;
  o.R2 = S0 * S1 + (((P1 - S0 * S1) % 32) + 32) % 32;
  o.F = 0;
  o.G = (nf + 3) & ~3;
  o.V = o.G + o.R2 * S2;
  o.c1 = o.V + np;
  o.words = (o.c1 + np + 3) & ~3;
  return o;
}

// (interSize, lag count) along dim 2 of the register-tiled lag kernel; other
// shapes take the one-lag-per-lane loop (direct3d_lags).
#define MQP_D3_TILED_SHAPES(X) X(2, 3) X(4, 5) X(6, 7) X(8, 9) X(8, 5) X(4, 9)
MQP_HD MQP_FI bool d3_tiled(int IS2, int P2) {
#define MQP_D3_IS(i, p) if (IS2 == i && P2 == p) return true;
  MQP_D3_TILED_SHAPES(MQP_D3_IS)
#undef MQP_D3_IS
  return false;
}

// F stored x1-fastest (F[x1 + IS1 (x2 + IS2 x3)]) or, for the tiled kernel,
// x2-fastest (F[x2 + IS2 (x1 + IS1 x3)]); G x1-fastest over the pad,
// G[p1 + S1 p2 + R2 p3].
template <typename T, int ALG>
MQP_HD MQP_FI void direct3d_load(const Piv3dArgs& a, const IAGeom3& g, const IA3State& s, int PASS, int lane, int nl,
                                 float* F, float* G, double& vmax, double& mmax, double& sumsq, bool fx2 = false) {
  const long long HW = (long long)a.H * a.W;
  const int I0 = a.IS[0], I1 = a.IS[1], I2 = a.IS[2];
  for (int i = lane; i < I0 * I1 * I2; i += nl) {
    const int x1 = i % I0, x2 = (i / I0) % I1, x3 = i / (I0 * I1);
    const long long off = (long long)(g.ir[0] + x1) + (long long)a.H * (g.ir[1] + x2) + HW * (g.ir[2] + x3);
    float w;
    if (PASS == PASS_PLAIN) {
      const T r = ldg_px<T>(a.img1, off);
      vmax = (double)r > vmax ? (double)r : vmax;
      const double val = (double)r - s.meanF;
      sumsq += val * val;
      w = (float)val;
    } else if (PASS == PASS_MASKED) {
      const T r = ldg_px<T>(a.img1, off);
      const T mk = ldg_px<T>(a.mask, off);
      const T ms = ldg_px<T>(a.mask_skip ? a.mask_skip : a.mask, off);
      vmax = (double)r > vmax ? (double)r : vmax;
      mmax = (double)ms > mmax ? (double)ms : mmax;
      const double val = (double)r * (double)mk;
      sumsq += val * val / ((double)mk > 0.0 ? (double)mk : 1.0);
      w = (float)val;
    } else {
      w = (float)ldg_px<T>(a.mask, off);
    }
    F[fx2 ? x2 + I1 * (x1 + I0 * x3) : i] = w;
  }
  const int S0 = a.IS[0] + 2 * a.SM[0], S1 = a.IS[1] + 2 * a.SM[1], S2 = a.IS[2] + 2 * a.SM[2];
  const int R2 = d3_off(a.IS, a.SM).R2;
  const float mg = (float)s.meanG;
  for (int i = lane; i < S0 * S1 * S2; i += nl) {
    const int p1 = i % S0, p2 = (i / S0) % S1, p3 = i / (S0 * S1);
    float v = 0.f;
    if (p1 >= g.lo[0] && p1 < g.hi[0] && p2 >= g.lo[1] && p2 < g.hi[1] && p3 >= g.lo[2] && p3 < g.hi[2]) {
      v = (float)ldg_px<T>(a.img2, (long long)(g.g0[0] + p1) + (long long)a.H * (g.g0[1] + p2) + HW * (g.g0[2] + p3));
      if (ALG == ALG_ZNCC) v = v - mg;
      if (PASS == PASS_MASK_SQ) v = v * v;
    }
    G[p1 + S0 * p2 + R2 * p3] = v;
  }
}

// raw correlation of lag q (s1 fastest) into V[q]
MQP_HD MQP_FI void direct3d_lags(const Piv3dArgs& a, int lane, int nl, const float* F, const float* G, float* V) {
  const int I0 = a.IS[0], I1 = a.IS[1], I2 = a.IS[2];
  const int S0 = a.IS[0] + 2 * a.SM[0], R2 = d3_off(a.IS, a.SM).R2;
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1, P3 = 2 * a.SM[2] + 1;
  for (int q = lane; q < P1 * P2 * P3; q += nl) {
    const int s1 = q % P1, s2 = (q / P1) % P2, s3 = q / (P1 * P2);
    float acc = 0.f;
    for (int x3 = 0; x3 < I2; ++x3)
      for (int x2 = 0; x2 < I1; ++x2) {
        const float* f = F + I0 * (x2 + I1 * x3);
        const float* gr = G + (s1 + S0 * (x2 + s2) + R2 * (x3 + s3));
        for (int x1 = 0; x1 < I0; ++x1) acc = fmaf(f[x1], gr[x1], acc);
      }
    V[q] = acc;
  }
}

// Register-tiled raw correlation: a task is one (s1, s3) lag pair and owns
// the P2 lags along dim 2 in registers.  Per (x3, x1) it holds F's IS2 values
// along dim 2 (x2-fastest F, one broadcast read per value) and streams the
// SS2 values of its G column, each feeding every lag whose window covers it:
// IS2 P2 fused multiply-adds per IS2 + SS2 shared-memory reads.  Consecutive
// tasks read consecutive banks (R2 = P1 modulo 32).  Sums run over x3, x1,
// then x2 (the one-lag loop sums x3, x2, x1).
template <int IS2, int P2>
MQP_HD MQP_FI void direct3d_lags_tiled(const Piv3dArgs& a, int tid, int nt, const float* F, const float* G, float* V) {
  constexpr int SS2 = IS2 + P2 - 1;
  const int I0 = a.IS[0], I2 = a.IS[2];
  const int S0 = a.IS[0] + 2 * a.SM[0], R2 = d3_off(a.IS, a.SM).R2;
  const int P1 = 2 * a.SM[0] + 1, P3 = 2 * a.SM[2] + 1;
  for (int task = tid; task < P1 * P3; task += nt) {
    const int s1 = task % P1, s3 = task / P1;
    float acc[P2];
#pragma unroll
    for (int j = 0; j < P2; ++j) acc[j] = 0.f;
    for (int x3 = 0; x3 < I2; ++x3) {
      const float* gz = G + s1 + R2 * (x3 + s3);
      const float* fz = F + IS2 * I0 * x3;
      for (int x1 = 0; x1 < I0; ++x1) {
        float f[IS2];
#pragma unroll
        for (int k = 0; k < IS2; ++k) f[k] = fz[IS2 * x1 + k];
        const float* gp = gz + x1;
#pragma unroll
        for (int t = 0; t < SS2; ++t) {
          const float gv = gp[S0 * t];
#pragma unroll
          for (int j = 0; j < P2; ++j)
            if (t - j >= 0 && t - j < IS2) acc[j] = fmaf(f[t - j], gv, acc[j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < P2; ++j) V[s1 + P1 * (j + P2 * s3)] = acc[j];
  }
}

// Similarity of lag q from its raw correlation(s), exactly as k3c_pair forms it.
template <int ALG>
MQP_HD MQP_FI double direct3d_sim(const Piv3dArgs& a, const IAGeom3& g, const IA3State& s, int q, double c,
                                  double c2) {
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1;
  const int s1 = q % P1, s2 = (q / P1) % P2, s3 = q / (P1 * P2);
  const float sqF = sqrtf((float)s.sumF2);
  if (ALG == ALG_FFTCC) return c;
  if (ALG == ALG_MASK_NSQECC)
    return similarity_value<ALG_MASK_NSQECC>(IAScalars{s.sumF2, 0.0, 0.0}, sqF, (double)(float)c, c2, 0.0, 0.0);
  int r0, r1, c0, c1, z0, z1;
  lag_window(s1, a.IS[0], g.g0[0], g.lo[0], g.hi[0], r0, r1);
  lag_window(s2, a.IS[1], g.g0[1], g.lo[1], g.hi[1], c0, c1);
  lag_window(s3, a.IS[2], g.g0[2], g.lo[2], g.hi[2], z0, z1);
  const double S2 = box_sum3(a.IIg2, a.H, a.W, r0, r1, c0, c1, z0, z1);
  double S1 = 0.0, n = 0.0;
  if (ALG == ALG_ZNCC) {
    S1 = box_sum3(a.IIg, a.H, a.W, r0, r1, c0, c1, z0, z1);
    n = (double)(r1 - r0) * (double)(c1 - c0) * (double)(z1 - z0);
  }
  return similarity_value<ALG>(IAScalars{s.sumF2, s.meanF, s.meanG}, sqF, c, S2, S1, n);
}

// Vector and SN of a 3D IA from the merged accumulators and its volume
// (k3c_final's rule; the volume lives in the warp's workspace).  With r
// given (the refined peak, e.g. from refine3d_warp) the fit is not redone.
MQP_HD MQP_FI void direct3d_final(const Piv3dArgs& a, const IAGeom3& g, long long ia, const LagRanges3& R,
                                  const float* V, double best, int bidx, double smax, double ssum,
                                  const double* rgiven = nullptr) {
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1;
  double r[3];
  if (rgiven) {
    for (int d = 0; d < 3; ++d) r[d] = rgiven[d];
  } else if (bidx < 0) {
    r[0] = r[1] = r[2] = -1.0;
  } else {
    const int p[3] = {bidx % P1, (bidx / P1) % P2, bidx / (P1 * P2)};
    refine3d(V, P1, P2, a.SM, g, p, best, r);
  }
  for (int d = 0; d < 3; ++d) a.VF[3 * ia + d] = r[d] - a.SM[d] + g.d[d];
  if (a.SN) {
    const double len = (double)(R.shi[0] - R.lo[0] + 1) * (double)(R.shi[1] - R.lo[1] + 1) *
                       (double)(R.shi[2] - R.lo[2] + 1);
    a.SN[ia] = smax / ((ssum - smax) / (len - 1.0));
  }
}

}  // namespace mqp
