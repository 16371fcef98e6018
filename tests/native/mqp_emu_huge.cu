// Host emulation of the 2D kernel for search windows of 129..256
// (mqp_piv2d_huge.cuh) for the CPU tests (test infrastructure, not part of
// the product library): every stage runs for all 256 threads of the block,
// thread by thread, between the kernel's block barriers, with the same stage
// functions; the finish reduces sequentially.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "mqp_piv2d_huge.cuh"

using namespace mqp;

template <int ALG, typename T>
static void emu_huge_ia(const Piv2dArgs& a, long long ia, float2* slot, float2* sm) {
  constexpr bool ZN = ALG == ALG_ZNCC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  const HugeSlot L(P1, P2);
  float2* GS = slot + L.gs;
  float2* FS = slot + L.fs;
  float2* LG = slot + L.lg;
  float* cc = reinterpret_cast<float*>(slot + L.cc);
  double* plane = reinterpret_cast<double*>(slot + L.pl);
  float2* park = sm;
  float2* pack = sm + HugeSmem::PARK;
  const float2* tw = pack + HugeSmem::PACK;
  const int v1 = (int)(ia % a.vf1), v2 = (int)(ia / a.vf1);
  int d1, d2;
  ia_pred(a, v1, v2, d1, d2);
  const IAGeom g = ia_geom(a, v1, v2);
  IAScalars sc;
  sc.meanF = sc.meanG = 0.0;
  if (ZN) {
    sc.meanF = box_sum(a.II1, a.H, g.ir1, g.ir1 + a.IS1, g.ir2, g.ir2 + a.IS2) / ((double)a.IS1 * a.IS2);
    const double nG = (double)(g.hi1 - g.lo1) * (double)(g.hi2 - g.lo2);
    sc.meanG = box_sum(a.IIg, a.H, g.g01 + g.lo1, g.g01 + g.hi1, g.g02 + g.lo2, g.g02 + g.hi2) / nG;
  }
  const long long vfo = (long long)v1 + (long long)a.vf1 * v2;
  double vmax = -INFINITY, sumsq = 0.0;
  for (int t = 0; t < HUGE_THREADS; ++t) {
    huge_f_row<T, ZN>(a, g, sc.meanF, t % MH, t / MH, FS, vmax, sumsq);
    huge_g_row<T, ZN>(a, g, (float)sc.meanG, t, GS, reinterpret_cast<float*>(park));
  }
  sc.sumF2 = sumsq;
  if (a.threshold >= 0.0 && vmax < a.threshold) {
    a.VF[2 * vfo] = a.VF[2 * vfo + 1] = 0.0;
    if (a.SN) a.SN[vfo] = 0.0;
    if (a.planes)
      for (int i = 0; i < P1 * P2; ++i) a.planes[(ia - a.ia_begin) * (long long)P1 * P2 + i] = 0.0;
    return;
  }
  std::vector<float2> fs((size_t)HUGE_THREADS * QH);
  for (int r = 0; r < 2; ++r) {
    for (int t = 0; t < HUGE_THREADS; ++t)
      huge_b_part1(r, t, GS, FS, tw, park, pack, *reinterpret_cast<float2(*)[QH]>(&fs[(size_t)t * QH]));
    for (int t = 0; t < HUGE_THREADS; ++t)
      huge_b_part2(r, t, tw, park, pack, *reinterpret_cast<float2(*)[QH]>(&fs[(size_t)t * QH]));
    for (int t = 0; t < HUGE_THREADS; ++t) huge_b_part3(r, t, P1, park, LG);
  }
  const float scale = (float)cc_scale<NH>();
  for (int b = 0; b < P1; b += MH)
    for (int t = 0; t < HUGE_THREADS; ++t) {
      const int s1 = b + t % MH;
      if (s1 < P1) huge_lag_row(s1, t / MH, P1, P2, LG, cc, scale);
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
  const float sqF = sqrtf((float)sc.sumF2);
  for (int l = 0; l < P1 * P2; ++l) {
    const int s1 = l % P1, s2 = l / P1;
    const double v = team_similarity<ALG>(a, g, sc, sqF, s1, s2, (double)cc[l]);
    plane[s1 * P2 + s2] = v;
    acc_take(acc, R, s1, s2, P1, v);
    if (a.planes) a.planes[(ia - a.ia_begin) * (long long)P1 * P2 + l] = v;
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

template <int ALG>
static void emu_huge_run(const Piv2dArgs& a) {
  std::vector<float2> slot((size_t)HugeSlot(2 * a.SM1 + 1, 2 * a.SM2 + 1).total), sm((size_t)HugeSmem::TOTAL);
  float2* tw = sm.data() + HugeSmem::PARK + HugeSmem::PACK;
  for (int j = 0; j < NH; ++j) tw[j] = twiddle_rt(j * (TW_N / NH));
  for (long long ia = a.ia_begin; ia < a.ia_end; ++ia) {
    if (a.dtype == 0) emu_huge_ia<ALG, float>(a, ia, slot.data(), sm.data());
    else emu_huge_ia<ALG, double>(a, ia, slot.data(), sm.data());
  }
}

int emu_piv2d_huge(const Piv2dArgs& a, int alg) {
  if (alg == ALG_FFTCC) emu_huge_run<ALG_FFTCC>(a);
  else if (alg == ALG_ZNCC) emu_huge_run<ALG_ZNCC>(a);
  else if (alg == ALG_NSQECC) emu_huge_run<ALG_NSQECC>(a);
  else return -1;
  return 0;
}
