// Host emulation of the 2D block kernel for search windows up to 128 (test
// infrastructure, not part of the product library): the same per-thread
// phase functions as piv2d_big_kernel (mqp_piv2d_big.cuh), thread by thread,
// with each barrier replaced by the end of a loop over the block's threads
// and the block reductions by sequential loops.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "mqp_piv2d_big.cuh"

using namespace mqp;

template <bool FPRUNE, int ALG, typename T>
static void emu_big_ia(const Piv2dArgs& a, long long ia, std::vector<float2>& ws) {
  using L = LayBig<FPRUNE>;
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  float2* S = ws.data() + L::S_OFF;
  float2* SF = ws.data() + L::F_OFF;
  double* plane = reinterpret_cast<double*>(SF);
  float* c1buf = MASKED ? reinterpret_cast<float*>(SF + L::region2(P1, P2)) : nullptr;
  float2* PK = ws.data() + L::pk_off(P1, P2, MASKED);
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
  std::vector<float2> reg((size_t)BIG_THREADS * MB);  // one 64-point array per thread across a barrier
  constexpr int NPASS = MASKED ? 2 : 1;
  for (int pass = 0; pass < NPASS; ++pass) {
    const int PASS = MASKED ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;
    double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
    for (int t = 0; t < BIG_THREADS; ++t) big_rows<FPRUNE, T, ALG>(a, g, sc, PASS, t, S, SF, vmax, mmax, sumsq);
    if (pass == 0) {
      sc.sumF2 = sumsq;
      const bool skip = MASKED ? ((a.threshold > 0.0 && vmax < a.threshold) ||
                                  (a.mask_threshold > 0.0 && mmax < a.mask_threshold))
                               : (a.threshold >= 0.0 && vmax < a.threshold);
      if (skip) {
        a.VF[2 * vfo] = 0.0;
        a.VF[2 * vfo + 1] = 0.0;
        if (a.SN) a.SN[vfo] = 0.0;
        if (a.planes) memset(a.planes + (ia - a.ia_begin) * (long long)P1 * P2, 0, sizeof(double) * P1 * P2);
        return;
      }
    }
    auto slot = [&](int t) { return reinterpret_cast<float2(*)[MB]>(&reg[(size_t)t * MB]); };
    for (int t = 0; t < BIG_THREADS; ++t) big_col_g<FPRUNE>(t, S, *slot(t));
    for (int t = 0; t < BIG_THREADS; ++t) big_col_park<FPRUNE>(t, *slot(t), S);
    for (int t = 0; t < BIG_THREADS; ++t) big_col_product<FPRUNE>(t, S, SF, PK, *slot(t));
    for (int t = 0; t < BIG_THREADS; ++t) big_col_park_a<FPRUNE>(t, *slot(t), S);
    for (int t = 0; t < BIG_THREADS; ++t) big_col_combine<FPRUNE>(t, P1, S, *slot(t));
    for (int t = 0; t < BIG_THREADS; ++t) big_col_store<FPRUNE>(t, P1, *slot(t), S);
    for (int t = 0; t < BIG_THREADS; ++t) big_lag_row<FPRUNE>(t, P1, P2, S, plane);
    if (MASKED && pass == 0)
      for (int i = 0; i < P1 * P2; ++i) c1buf[i] = (float)plane[i];
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
  for (int t = 0; t < P1; ++t)
    finish_row<ALG>(a, g, sc, t, P1, P2, plane + (long long)t * P2, R, acc, MASKED ? c1buf + t * P2 : nullptr);
  if (a.planes) {
    double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
    for (int i = 0; i < P1 * P2; ++i) dst[i] = plane[(i % P1) * P2 + i / P1];
  }
  double r1, r2;
  if (acc.bidx < 0) {
    r1 = r2 = -1.0;
  } else {
    refine2d(plane, P2, a.SM1, a.SM2, g, acc.bidx % P1, acc.bidx / P1, acc.best, r1, r2);
  }
  a.VF[2 * vfo + 0] = r1 - a.SM1 + d1;
  a.VF[2 * vfo + 1] = r2 - a.SM2 + d2;
  if (a.SN) {
    const double len = (double)(R.shi1 - R.lo1 + 1) * (double)(R.shi2 - R.lo2 + 1);
    a.SN[vfo] = acc.smax / ((acc.ssum - acc.smax) / (len - 1.0));
  }
}

template <bool FPRUNE, int ALG>
static void emu_big_alg(const Piv2dArgs& a) {
  using L = LayBig<FPRUNE>;
  std::vector<float2> ws((size_t)L::total_f2(2 * a.SM1 + 1, 2 * a.SM2 + 1, ALG == ALG_MASK_NSQECC));
  for (long long ia = a.ia_begin; ia < a.ia_end; ++ia) {
    if (a.dtype == 0) emu_big_ia<FPRUNE, ALG, float>(a, ia, ws);
    else emu_big_ia<FPRUNE, ALG, double>(a, ia, ws);
  }
}

template <bool FPRUNE>
static int emu_big_prune(const Piv2dArgs& a, int alg) {
  switch (alg) {
    case 0: emu_big_alg<FPRUNE, 0>(a); return 0;
    case 1: emu_big_alg<FPRUNE, 1>(a); return 0;
    case 2: emu_big_alg<FPRUNE, 2>(a); return 0;
    case 3: emu_big_alg<FPRUNE, 3>(a); return 0;
    default: return -1;
  }
}

// called by mqp_emu_piv2d (mqp_emu.cu) for search windows 65..128
int emu_piv2d_big(const Piv2dArgs& a, int alg) {
  const bool prune = a.IS1 <= MB && a.IS2 <= MB;
  return prune ? emu_big_prune<true>(a, alg) : emu_big_prune<false>(a, alg);
}
