// Host emulation of the direct (spatial) correlation kernels for small
// windows (test infrastructure, not part of the product library): the same
// per-lane functions as direct2d_kernel / direct3d_kernel /
// direct3d_tiled_kernel (mqp_direct.cuh), run as one lane covering every
// element, with sequential reductions.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "mqp_direct.cuh"

using namespace mqp;

template <int ALG, typename T>
static void emu_d2_ia(const Piv2dArgs& a, long long ia, std::vector<float>& ws) {
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const D2Off o = d2_off(a.IS1, a.IS2, a.SM1, a.SM2);
  float* F = ws.data() + o.F;
  float* G = ws.data() + o.G;
  double* plane = reinterpret_cast<double*>(ws.data() + o.plane);
  float* c1 = ws.data() + o.c1;
  const int v1 = (int)(ia % a.vf1), v2 = (int)(ia / a.vf1);
  int d1, d2;
  ia_pred(a, v1, v2, d1, d2);
  const IAGeom g = ia_geom(a, v1, v2);
  IAScalars sc;
  sc.meanF = sc.meanG = sc.sumF2 = 0.0;
  if (ALG == ALG_ZNCC) {
    sc.meanF = box_sum(a.II1, a.H, g.ir1, g.ir1 + a.IS1, g.ir2, g.ir2 + a.IS2) / ((double)a.IS1 * a.IS2);
    const double nG = (double)(g.hi1 - g.lo1) * (double)(g.hi2 - g.lo2);
    sc.meanG = box_sum(a.IIg, a.H, g.g01 + g.lo1, g.g01 + g.hi1, g.g02 + g.lo2, g.g02 + g.hi2) / nG;
  }
  const long long vfo = (long long)v1 + (long long)a.vf1 * v2;
  constexpr int NPASS = MASKED ? 2 : 1;
  for (int pass = 0; pass < NPASS; ++pass) {
    const int PASS = MASKED ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;
    double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
    direct2d_load<T, ALG>(a, g, sc, PASS, 0, 1, F, G, vmax, mmax, sumsq);
    if (pass == 0) {
      sc.sumF2 = sumsq;
      const bool skip = MASKED ? ((a.threshold > 0.0 && vmax < a.threshold) ||
                                  (a.mask_threshold > 0.0 && mmax < a.mask_threshold))
                               : (a.threshold >= 0.0 && vmax < a.threshold);
      if (skip) {
        a.VF[2 * vfo] = a.VF[2 * vfo + 1] = 0.0;
        if (a.SN) a.SN[vfo] = 0.0;
        if (a.planes) memset(a.planes + (ia - a.ia_begin) * (long long)P1 * P2, 0, sizeof(double) * P1 * P2);
        return;
      }
    }
    direct2d_lags(a, 0, 1, F, G, plane);
    if (MASKED && pass == 0)
      for (int i = 0; i < P1 * P2; ++i) c1[i] = (float)plane[i];
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
  for (int q = 0; q < P1 * P2; ++q) direct2d_finish_lag<ALG>(a, g, sc, q, P1, P2, plane, c1, R, acc);
  if (a.planes) {
    double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
    for (int i = 0; i < P1 * P2; ++i) dst[i] = plane[(i % P1) * P2 + i / P1];
  }
  double r1 = -1.0, r2 = -1.0;
  if (acc.bidx >= 0) refine2d(plane, P2, a.SM1, a.SM2, g, acc.bidx % P1, acc.bidx / P1, acc.best, r1, r2);
  a.VF[2 * vfo + 0] = r1 - a.SM1 + d1;
  a.VF[2 * vfo + 1] = r2 - a.SM2 + d2;
  if (a.SN) {
    const double len = (double)(R.shi1 - R.lo1 + 1) * (double)(R.shi2 - R.lo2 + 1);
    a.SN[vfo] = acc.smax / ((acc.ssum - acc.smax) / (len - 1.0));
  }
}

template <int ALG, typename T>
static void emu_d3_ia(const Piv3dArgs& a, long long ia, std::vector<float>& ws) {
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1, P3 = 2 * a.SM[2] + 1, vol = P1 * P2 * P3;
  const D3Off o = d3_off(a.IS, a.SM);
  float* F = ws.data() + o.F;
  float* G = ws.data() + o.G;
  float* V = ws.data() + o.V;
  float* C1 = ws.data() + o.c1;
  const IAGeom3 g = ia_geom3(a, ia);
  IA3State s;
  ia3_means<ALG>(a, g, s.meanF, s.meanG);
  s.sumF2 = 0.0;
  s.skip = 0;
  constexpr int NPASS = MASKED ? 2 : 1;
  for (int pass = 0; pass < NPASS; ++pass) {
    const int PASS = MASKED ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;
    double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
    const bool tiled = d3_tiled(a.IS[1], P2);
    direct3d_load<T, ALG>(a, g, s, PASS, 0, 1, F, G, vmax, mmax, sumsq, tiled);
    if (pass == 0) {
      s.sumF2 = sumsq;
      if (skip_test3(a, ALG, vmax, mmax)) {
        for (int d = 0; d < 3; ++d) a.VF[3 * ia + d] = 0.0;
        if (a.SN) a.SN[ia] = 0.0;
        if (a.planes) memset(a.planes + (ia - a.planes_begin) * (long long)vol, 0, sizeof(double) * vol);
        return;
      }
    }
    if (!tiled) direct3d_lags(a, 0, 1, F, G, V);
#define MQP_D3_EMU(i, p) \
  else if (a.IS[1] == i && P2 == p) direct3d_lags_tiled<i, p>(a, 0, 1, F, G, V);
    MQP_D3_TILED_SHAPES(MQP_D3_EMU)
#undef MQP_D3_EMU
    if (MASKED && pass == 0)
      for (int i = 0; i < vol; ++i) C1[i] = V[i];
  }
  const LagRanges3 R = lag_ranges3(a, g);
  PeakAcc acc;
  acc.best = 0.0;
  acc.bidx = -1;
  acc.smax = -INFINITY;
  acc.ssum = 0.0;
  for (int q = 0; q < vol; ++q) {
    const double c = MASKED ? (double)C1[q] : (double)V[q];
    const double c2 = MASKED ? (double)V[q] : 0.0;
    const double v = direct3d_sim<ALG>(a, g, s, q, c, c2);
    V[q] = (float)v;
    if (a.planes) a.planes[(ia - a.planes_begin) * (long long)vol + q] = v;
    acc_take3(acc, R, q % P1, (q / P1) % P2, q / (P1 * P2), q, v);
  }
  direct3d_final(a, g, ia, R, V, acc.best, acc.bidx, acc.smax, acc.ssum);
}

template <int ALG>
static void emu_d2(const Piv2dArgs& a) {
  std::vector<float> ws((size_t)d2_off(a.IS1, a.IS2, a.SM1, a.SM2).words);
  for (long long ia = a.ia_begin; ia < a.ia_end; ++ia) {
    if (a.dtype == 0) emu_d2_ia<ALG, float>(a, ia, ws);
    else emu_d2_ia<ALG, double>(a, ia, ws);
  }
}

template <int ALG>
static void emu_d3(const Piv3dArgs& a) {
  std::vector<float> ws((size_t)d3_off(a.IS, a.SM).words);
  for (long long ia = a.ia_begin; ia < a.ia_end; ++ia) {
    if (a.dtype == 0) emu_d3_ia<ALG, float>(a, ia, ws);
    else emu_d3_ia<ALG, double>(a, ia, ws);
  }
}

// called by mqp_emu_piv2d / mqp_emu_piv3d for windows direct2d_ok / direct3d_ok accept
int emu_piv2d_direct(const Piv2dArgs& a, int alg) {
  switch (alg) {
    case 0: emu_d2<0>(a); return 0;
    case 1: emu_d2<1>(a); return 0;
    case 2: emu_d2<2>(a); return 0;
    case 3: emu_d2<3>(a); return 0;
    default: return -1;
  }
}

int emu_piv3d_direct(const Piv3dArgs& a, int alg) {
  switch (alg) {
    case 0: emu_d3<0>(a); return 0;
    case 1: emu_d3<1>(a); return 0;
    case 2: emu_d3<2>(a); return 0;
    case 3: emu_d3<3>(a); return 0;
    default: return -1;
  }
}
