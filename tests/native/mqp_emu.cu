// Host emulation of the fused 2D kernel for CPU tests (test infrastructure,
// not part of the product library).  It runs the SAME per-lane phase
// functions as piv2d_kernel (mqp_piv2d.cuh), lane by lane, with the warp
// reductions replaced by plain loops, so FFT indexing, scaling, window
// geometry and peak logic can be checked against the oracle without a GPU.
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "mqp_deform.cuh"
#include "mqp_direct.cuh"
#include "mqp_piv2d.cuh"
#include "mqp_piv2d_team.cuh"

using namespace mqp;

static void integral(const void* img, int dtype, int H, int W, bool sq, std::vector<double>& out) {
  const long long ld = H + 1;
  out.assign((size_t)ld * (W + 1), 0.0);
  for (int c = 1; c <= W; ++c) {
    double acc = 0.0;
    for (int r = 1; r <= H; ++r) {
      double v = load_px(img, dtype, (long long)(r - 1) + (long long)H * (c - 1));
      if (sq) v = v * v;
      acc += v;
      out[r + ld * c] = out[r + ld * (c - 1)] + acc;
    }
  }
}

template <int N, bool FPRUNE, int ALG, typename T, bool LW = false>
static void emu_ia(const Piv2dArgs& a, long long ia, std::vector<float2>& ws) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  constexpr bool MASKED = ALG == ALG_MASK_NSQECC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  float2* GH = ws.data();
  float2* FH = GH + (LW ? Lay::F_OFF_LW : Lay::F_OFF);
  double* lw = LW ? reinterpret_cast<double*>(GH) : nullptr;
  double* plane = reinterpret_cast<double*>(FH);
  float* c1buf = MASKED ? reinterpret_cast<float*>(FH + Lay::region2_f2(P1, P2)) : nullptr;
  float2 tw[N];
  for (int j = 0; j < N; ++j) tw[j] = twiddle_rt(j * (TW_N / N));
  const double scale = cc_scale<N>();
  const int lane_rows = (P1 - 32 > 0 && P1 - 32 <= 4) ? 32 : P1;
  const int v1 = (int)(ia % a.vf1), v2 = (int)(ia / a.vf1);
  int d1, d2;
  ia_pred(a, v1, v2, d1, d2);
  const IAGeom g = ia_geom(a, v1, v2);
  IAScalars sc;
  sc.meanF = sc.meanG = 0.0;
  if (ALG == ALG_ZNCC) {
    sc.meanF = box_sum(a.II1, a.H, g.ir1, g.ir1 + a.IS1, g.ir2, g.ir2 + a.IS2) / ((double)a.IS1 * a.IS2);
    const double nG = (double)(g.hi1 - g.lo1) * (double)(g.hi2 - g.lo2);
    sc.meanG = box_sum(a.IIg, a.H, g.g01 + g.lo1, g.g01 + g.hi1, g.g02 + g.lo2, g.g02 + g.hi2) / nG;
  }
  const long long vfo = (long long)v1 + (long long)a.vf1 * v2;
  constexpr int NPASS = MASKED ? 2 : 1;
  for (int pass = 0; pass < NPASS; ++pass) {
    const int pmode = MASKED ? (pass == 0 ? PASS_MASKED : PASS_MASK_SQ) : PASS_PLAIN;
    double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
    constexpr int NJF = (Lay::NF + 31) / 32, NJ = NJF + N / 32;
    for (int lane = 0; lane < 32; ++lane)
      for (int job = 0; job < NJ; ++job) {
        const RowJob j = row_job<N, FPRUNE>(a, g, lane, job);
        if (j.isF && j.row >= Lay::NF) continue;
        float v[N];
        row_load<N, T>(a, j, v);
        row_process<N, FPRUNE, T, ALG == ALG_ZNCC>(a, sc, pmode, j, v, GH, FH, vmax, mmax, sumsq);
      }
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
    for (int n = 0; n < M; ++n) split_G_pair<N, FPRUNE>(GH, tw, n);
    for (int u = 0; u < M; ++u) {
      float2 t[M];
      for (int q = 0; q < 6; ++q) {
        const int h = q / 3, st = q % 3;
        stage_pre<N, FPRUNE>(st, h, GH + u * Lay::GSTR, FH + u * Lay::FSTR, t);
        fft_reg<M, false>(t);
        stage_post<N, FPRUNE>(st, h, u == 0, P1, GH + u * Lay::GSTR, t);
      }
    }
    for (int s1 = 0; s1 < lane_rows; ++s1) {
      float2 t[M];
      c2r_pre<N, FPRUNE>(s1, GH, t);
      fft_reg<M, false>(t);
      double* prow = plane + s1 * P2;
      for (int n = 0; n < M; ++n) {
        const float2 z = cconj(t[fpos<M>(n)]);
        if (2 * n < P2) prow[2 * n] = (double)z.x * scale;
        if (2 * n + 1 < P2) prow[2 * n + 1] = (double)z.y * scale;
      }
    }
    for (int s1 = lane_rows; s1 < P1; ++s1)
      for (int s2 = 0; s2 < P2; ++s2) plane[s1 * P2 + s2] = (double)tail_row_value<N, FPRUNE>(GH, tw, s1, s2) * scale;
    if (LW) {
      // the on-chip window sums: every lane's rows, then every lane's columns
      for (int lane = 0; lane < 32; ++lane) lw_rows<N, T, ALG == ALG_ZNCC>(a, g, sc.meanG, lane, P2, lw);
      for (int lane = 0; lane < 32; ++lane) lw_cols<N>(lane, P1, P2, lw);
      if (N == 64 && P2 > 32) {
        // lw_col32's warp scans, lane by lane
        double* col = lw + 32 * N;
        double suf[32], pre[32], r1[32];
        for (int l = 0; l < 32; ++l) {
          suf[l] = col[l];
          pre[l] = r1[l] = col[l + 32];
        }
        for (int off = 1; off < 32; off <<= 1) {
          double a_[32], b_[32];
          for (int l = 0; l < 32; ++l) {
            a_[l] = l + off < 32 ? suf[l + off] : suf[l];
            b_[l] = l >= off ? pre[l - off] : pre[l];
          }
          for (int l = 0; l < 32; ++l) lw_scan_step(suf[l], pre[l], a_[l], b_[l], l, off);
        }
        for (int l = 0; l < 32 && l < P1; ++l) col[l] = suf[l] + (l ? pre[l - 1] : 0.0);
        if (P1 > 32) col[32] = pre[31];
        (void)r1;
      }
    }
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
  double best = 0.0, smax = -INFINITY, ssum = 0.0;
  int bidx = -1;
  for (int lane = 0; lane < 32; ++lane) {
    PeakAcc acc;
    acc.best = 0.0;
    acc.bidx = -1;
    acc.smax = -INFINITY;
    acc.ssum = 0.0;
    for (int s1 = lane; s1 < lane_rows; s1 += 32)
      finish_row<ALG, LW ? N : 0>(a, g, sc, s1, P1, P2, plane + s1 * P2, R, acc, MASKED ? c1buf + s1 * P2 : nullptr,
                                  lw);
    for (int s1 = lane_rows; s1 < P1; ++s1)
      for (int s2 = lane; s2 < P2; s2 += 32) {
        double& e = plane[s1 * P2 + s2];
        e = finish_one<ALG, LW ? N : 0>(a, g, sc, s1, s2, e, MASKED ? (double)c1buf[s1 * P2 + s2] : 0.0, lw);
        acc_take(acc, R, s1, s2, P1, e);
      }
    peak_merge(best, bidx, acc.best, acc.bidx);
    smax = nmax(smax, acc.smax);
    ssum += acc.ssum;
  }
  double sn = 0.0;
  if (a.SN) {
    const double len = (double)(R.shi1 - R.lo1 + 1) * (double)(R.shi2 - R.lo2 + 1);
    sn = smax / ((ssum - smax) / (len - 1.0));
  }
  if (a.planes) {
    double* dst = a.planes + (ia - a.ia_begin) * (long long)P1 * P2;
    for (int i = 0; i < P1 * P2; ++i) dst[i] = plane[(i % P1) * P2 + i / P1];
  }
  double r1 = -1.0, r2 = -1.0;
  if (bidx >= 0) refine2d(plane, P2, a.SM1, a.SM2, g, bidx % P1, bidx / P1, best, r1, r2);
  a.VF[2 * vfo] = r1 - a.SM1 + d1;
  a.VF[2 * vfo + 1] = r2 - a.SM2 + d2;
  if (a.SN) a.SN[vfo] = sn;
}

template <int N, bool FPRUNE, int ALG, bool LW = false>
static void emu_run(const Piv2dArgs& a) {
  using Lay = Layout2d<N, FPRUNE>;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  std::vector<float2> ws((size_t)(LW ? Lay::warp_f2_lw(P1, P2) : Lay::warp_f2(P1, P2, ALG == ALG_MASK_NSQECC)));
  for (long long ia = a.ia_begin; ia < a.ia_end; ++ia) {
    if (a.dtype == 0) emu_ia<N, FPRUNE, ALG, float, LW>(a, ia, ws);
    else emu_ia<N, FPRUNE, ALG, double, LW>(a, ia, ws);
  }
}

// ZNCC with the on-chip window sums (launch_piv2d's choice for an N/2 x N/2
// interrogation window)
template <int N>
static int emu_lw(const Piv2dArgs& a, int alg) {
  if (alg != 1) return -1;
  emu_run<N, true, 1, true>(a);
  return 0;
}

// The team kernel (mqp_piv2d_team.cuh) thread by thread: each phase runs for
// every thread of the team before the next (the team barriers), phase 2 in
// its two halves around its barrier; the finish uses the same similarity,
// peak and fit functions with sequential reductions.
template <int N, int ALG, typename T>
static void emu_team_ia(const Piv2dArgs& a, long long ia, std::vector<float2>& ws) {
  using L = TeamLayout<N>;
  constexpr int M = N / 2;
  constexpr bool ZN = ALG == ALG_ZNCC;
  const int P1 = 2 * a.SM1 + 1, P2 = 2 * a.SM2 + 1;
  float2* G = ws.data();
  float2* F = G + L::g_f2(P1, P2);
  float2 tw[N];
  for (int j = 0; j < N; ++j) tw[j] = twiddle_rt(j * (TW_N / N));
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
  for (int tid = 0; tid < N; ++tid) {
    team_f_row<N, T, ZN>(a, g, sc.meanF, tid % M, tid / M, F, vmax, sumsq);
  }
  for (int tid = 0; tid < N; ++tid) team_g_row<N, T, ZN>(a, g, (float)sc.meanG, tid, G);
  sc.sumF2 = sumsq;
  if (a.threshold >= 0.0 && vmax < a.threshold) {
    a.VF[2 * vfo] = a.VF[2 * vfo + 1] = 0.0;
    if (a.SN) a.SN[vfo] = 0.0;
    if (a.planes)
      for (int i = 0; i < P1 * P2; ++i) a.planes[(ia - a.ia_begin) * (long long)P1 * P2 + i] = 0.0;
    return;
  }
  std::vector<float2> xs((size_t)N * M);
  for (int st = 0; st < 3; ++st) {
    // every thread's transform of the stage, then every thread's post (the
    // team barrier of stage 0 sits between them)
    for (int tid = 0; tid < N; ++tid) {
      float2(&x)[M] = *reinterpret_cast<float2(*)[M]>(&xs[(size_t)tid * M]);
      team_p2_pre<N>(st, tid % M, tid / M, G, F, x);
      fft_reg<M, false>(x);
    }
    for (int tid = 0; tid < N; ++tid) {
      float2(&x)[M] = *reinterpret_cast<float2(*)[M]>(&xs[(size_t)tid * M]);
      team_p2_post<N>(st, tid % M, tid / M, G, x);
    }
  }
  float* cc = reinterpret_cast<float*>(F);
  const float scale = (float)cc_scale<N>();
  const bool tail = P1 == M + 1;
  const int paired = tail ? P1 - 1 : P1;
  for (int b = 0; b < paired; b += M)
    for (int tid = 0; tid < N; ++tid) {
      const int s1 = b + tid % M;
      if (s1 >= paired) continue;
      team_phase3_row<N>(s1, tid / M, P1, P2, G, cc, scale);
    }
  if (tail)
    for (int s2 = 0; s2 < P2; ++s2) cc[(P1 - 1) + P1 * s2] = team_tail_value<N>(G, tw, s2) * scale;
  double* plane = reinterpret_cast<double*>(G);
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

template <int N, int ALG>
static void emu_team_run(const Piv2dArgs& a) {
  std::vector<float2> ws((size_t)TeamLayout<N>::team_f2(2 * a.SM1 + 1, 2 * a.SM2 + 1));
  for (long long ia = a.ia_begin; ia < a.ia_end; ++ia) {
    if (a.dtype == 0) emu_team_ia<N, ALG, float>(a, ia, ws);
    else emu_team_ia<N, ALG, double>(a, ia, ws);
  }
}

template <int N>
static int emu_team(const Piv2dArgs& a, int alg) {
  if (alg == 0) emu_team_run<N, 0>(a);
  else if (alg == 1) emu_team_run<N, 1>(a);
  else if (alg == 2) emu_team_run<N, 2>(a);
  else return -1;
  return 0;
}

template <int N, bool FPRUNE>
static int emu_alg(const Piv2dArgs& a, int alg) {
  if (alg == 0) emu_run<N, FPRUNE, 0>(a);
  else if (alg == 1) emu_run<N, FPRUNE, 1>(a);
  else if (alg == 2) emu_run<N, FPRUNE, 2>(a);
  else if (alg == 3) emu_run<N, FPRUNE, 3>(a);
  else return -1;
  return 0;
}

int emu_piv2d_big(const Piv2dArgs& a, int alg);     // mqp_emu_big.cu
int emu_piv2d_direct(const Piv2dArgs& a, int alg);  // mqp_emu_direct.cu
int emu_piv2d_huge(const Piv2dArgs& a, int alg);    // mqp_emu_huge.cu

extern "C" __attribute__((visibility("default"))) int mqp_emu_piv2d(
    const void* img1, const void* img2, const void* mask, const void* mask_skip, int dtype, int H, int W,
    int IS1, int IS2, int SM1, int SM2, int st1, int st2, int alg, double threshold, double mask_threshold,
    int computeSN, double* VF, double* SN, double* planes, long long ia_begin, long long ia_end) {
  std::vector<double> II1, IIg, IIg2;
  const int SS = (IS1 + 2 * SM1) > (IS2 + 2 * SM2) ? (IS1 + 2 * SM1) : (IS2 + 2 * SM2);
  const int N = SS <= 32 ? 32 : (SS <= 64 ? 64 : (SS <= 128 ? 128 : (SS <= 256 ? 256 : 0)));
  const bool prune = IS1 <= N / 2 && IS2 <= N / 2;
  // MQP_EMU_PIV2D_TEAM=1 emulates the opt-in team kernel for pruned FFTCC /
  // ZNCC / NSQECC (default: the one-warp-per-IA kernel, as launch_piv2d);
  // MQP_EMU_PIV2D_NO_LW=1 keeps the integral-image window sums where the warp
  // kernel forms them on chip
  const char* team_env = getenv("MQP_EMU_PIV2D_TEAM");
  const char* nolw_env = getenv("MQP_EMU_PIV2D_NO_LW");
  const bool direct = direct2d_ok(IS1, IS2, SM1, SM2);
  const bool team = !direct && prune && alg <= 2 && (N == 32 || N == 64) && team_env && team_env[0] == '1';
  const bool lw = !direct && !team && alg == 1 && (N == 32 || N == 64) && IS1 == N / 2 &&
                  IS2 == N / 2 && !(nolw_env && nolw_env[0] == '1');
  Piv2dArgs a;
  memset(&a, 0, sizeof(a));
  a.img1 = img1;
  a.img2 = img2;
  a.mask = mask;
  a.mask_skip = mask_skip;
  a.mask_threshold = mask_threshold;
  a.dtype = dtype;
  if ((alg == 1 || alg == 2) && !lw) {  // the on-chip sums read no img2^2 integral
    integral(img2, dtype, H, W, true, IIg2);
    a.IIg2 = IIg2.data();
  }
  if (alg == 1) {
    integral(img2, dtype, H, W, false, IIg);
    integral(img1, dtype, H, W, false, II1);
    a.IIg = IIg.data();
    a.II1 = II1.data();
  }
  a.VF = VF;
  a.SN = computeSN ? SN : nullptr;
  a.planes = planes;
  a.H = H; a.W = W; a.IS1 = IS1; a.IS2 = IS2; a.SM1 = SM1; a.SM2 = SM2; a.st1 = st1; a.st2 = st2;
  a.vf1 = (H - IS1) / st1 + 1;
  a.vf2 = (W - IS2) / st2 + 1;
  a.ia_begin = ia_begin;
  a.ia_end = ia_end;
  a.threshold = threshold;
  a.computeSN = computeSN;
  if (direct) return emu_piv2d_direct(a, alg);
  if (N == 128) return emu_piv2d_big(a, alg);
  if (N == 256) return IS1 <= 128 && IS2 <= 128 ? emu_piv2d_huge(a, alg) : -2;
  if (lw) return N == 64 ? emu_lw<64>(a, alg) : emu_lw<32>(a, alg);
  if (N == 64) return team ? emu_team<64>(a, alg) : (prune ? emu_alg<64, true>(a, alg) : emu_alg<64, false>(a, alg));
  if (N == 32) return team ? emu_team<32>(a, alg) : (prune ? emu_alg<32, true>(a, alg) : emu_alg<32, false>(a, alg));
  return -2;
}

// the deforming refinement's resampling (mqp_deform.cuh) over a whole image
extern "C" __attribute__((visibility("default"))) int mqp_emu_deform(
    const void* img1, const void* img2, int dtype, int nd, const long long* dims, const double* VFc,
    const int* vf_c, const int* isz_c, const int* st_c, void* out1, void* out2) {
  DeformArgs a;
  memset(&a, 0, sizeof(a));
  a.nd = nd;
  a.dtype = dtype;
  long long n = 1;
  for (int d = 0; d < 3; ++d) {
    a.dims[d] = d < nd ? dims[d] : 1;
    n *= a.dims[d];
    if (d < nd) {
      a.vf_c[d] = vf_c[d];
      a.isz_c[d] = isz_c[d];
      a.st_c[d] = st_c[d];
    }
  }
  a.img1 = img1;
  a.img2 = img2;
  a.out1 = out1;
  a.out2 = out2;
  a.VFc = VFc;
  for (long long i = 0; i < n; ++i) deform_pixel(a, i);
  return 0;
}

// one register FFT, for direct unit tests of mqp_fft.cuh
extern "C" __attribute__((visibility("default"))) int mqp_emu_fft(int n, int inverse, float* io) {
  auto run = [&](auto tag) {
    constexpr int NN = decltype(tag)::value;
    float2 x[NN];
    for (int i = 0; i < NN; ++i) x[i] = make_float2(io[2 * i], io[2 * i + 1]);
    if (inverse) fft_reg<NN, true>(x);
    else fft_reg<NN, false>(x);
    for (int k = 0; k < NN; ++k) {
      io[2 * k] = x[fpos<NN>(k)].x;
      io[2 * k + 1] = x[fpos<NN>(k)].y;
    }
  };
  switch (n) {
    case 4: run(std::integral_constant<int, 4>()); break;
    case 8: run(std::integral_constant<int, 8>()); break;
    case 16: run(std::integral_constant<int, 16>()); break;
    case 32: run(std::integral_constant<int, 32>()); break;
    case 64: run(std::integral_constant<int, 64>()); break;
    case 128: run(std::integral_constant<int, 128>()); break;
    default: return -1;
  }
  return 0;
}
