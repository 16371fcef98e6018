// Host emulation of the 3D kernels for CPU tests (test infrastructure, not
// part of the product library).  It runs the SAME per-thread phase functions
// as k3a/k3b/k3c (mqp_piv3d.cuh), thread by thread and block by block, with
// the block reductions replaced by plain loops and each __syncthreads by the
// end of a loop over threads.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "mqp_multipass.cuh"
#include "mqp_direct.cuh"
#include "mqp_piv3d.cuh"

using namespace mqp;

int emu_piv3d_direct(const Piv3dArgs& a, int alg);  // mqp_emu_direct.cu

// exclusive-prefix integral volume (H+1) x (W+1) x (D+1)
static void integral3(const void* img, int dtype, int H, int W, int D, bool sq, std::vector<double>& out) {
  const long long l1 = H + 1, l2 = l1 * (W + 1);
  out.assign((size_t)(l2 * (D + 1)), 0.0);
  for (int z = 1; z <= D; ++z)
    for (int c = 1; c <= W; ++c)
      for (int r = 1; r <= H; ++r) {
        double v = load_px(img, dtype, (long long)(r - 1) + (long long)H * ((c - 1) + (long long)W * (z - 1)));
        if (sq) v = v * v;
        auto at = [&](int rr, int cc, int zz) { return out[rr + l1 * cc + l2 * zz]; };
        out[r + l1 * c + l2 * z] = v + at(r - 1, c, z) + at(r, c - 1, z) + at(r, c, z - 1) - at(r - 1, c - 1, z) -
                                   at(r - 1, c, z - 1) - at(r, c - 1, z - 1) + at(r - 1, c - 1, z - 1);
      }
}

template <int N, bool FPRUNE, int ALG, typename T>
static void emu3_run(Piv3dArgs a) {
  using L = Lay3<N, FPRUNE>;
  const long long n = a.ia_end - a.ia_begin;
  const int P1 = 2 * a.SM[0] + 1, P2 = 2 * a.SM[1] + 1, P3 = 2 * a.SM[2] + 1;
  const long long P12 = (long long)P1 * P2;
  std::vector<float2> Gz((size_t)(n * L::GZ)), Fz((size_t)(n * L::FZ));
  std::vector<float2> Cb((size_t)(n * L::K3 * P12)), C2b(ALG == ALG_MASK_NSQECC ? Cb.size() : 0);
  std::vector<float> V((size_t)(n * P12 * P3));
  std::vector<IA3State> st((size_t)n);
  a.Gz = Gz.data();
  a.Fz = Fz.data();
  a.C = Cb.data();
  a.C2 = C2b.empty() ? nullptr : C2b.data();
  a.V = V.data();
  a.state = st.data();
  constexpr int NPASS = ALG == ALG_MASK_NSQECC ? 2 : 1;
  std::vector<float2> sm((size_t)L::SMEM_F2);
  std::vector<float2> pbuf((size_t)N * N);
  for (int pass = 0; pass < NPASS; ++pass) {
    // K3a
    for (long long ci = 0; ci < n; ++ci) {
      const IAGeom3 g = ia_geom3(a, a.ia_begin + ci);
      IA3State s;
      if (pass == 0) {
        ia3_means<ALG>(a, g, s.meanF, s.meanG);
        s.sumF2 = 0.0;
        s.skip = 0;
      } else {
        s = st[ci];
      }
      double vmax = -INFINITY, mmax = -INFINITY, sumsq = 0.0;
      const int nl = k3a_lines(a, g);
      for (int line = 0; line < nl; ++line) k3a_line<N, FPRUNE, T, ALG>(a, g, s, pass, ci, line, vmax, mmax, sumsq);
      if (pass == 0) {
        s.sumF2 = sumsq;
        s.skip = skip_test3(a, ALG, vmax, mmax) ? 1 : 0;
        st[ci] = s;
      }
    }
    // K3b
    float2* Cout = pass == 0 ? a.C : a.C2;
    for (long long ci = 0; ci < n; ++ci) {
      if (st[ci].skip) continue;
      const IAGeom3 g = ia_geom3(a, a.ia_begin + ci);
      // the kernel's phases, each for all 2N threads (t, h) before the next
      // (its block barriers); a thread's M registers live in pbuf between phases
      constexpr int M = N / 2;
      using Reg = float2[M];
      Reg* R = reinterpret_cast<Reg*>(pbuf.data());
      for (int k3 = 0; k3 < L::K3; ++k3) {
        float2* S = sm.data();
        float2* SF = S + N * L::SSTR;
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_rows<N, FPRUNE>(a, g, ci, k3, t, h, S, SF);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_cols_g<N, FPRUNE>(t, h, S, R[h * N + t]);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_park<N, FPRUNE>(t, h, S, R[h * N + t]);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_cols_f<N, FPRUNE>(t, h, S, SF, R[h * N + t]);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_x1<N, FPRUNE>(t, h, R[h * N + t], S);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_x2<N, FPRUNE>(t, h, S, R[h * N + t]);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_x3<N, FPRUNE>(t, h, P1, R[h * N + t], S);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_r2a<N, FPRUNE>(t, h, P1, S, R[h * N + t]);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_r2b<N, FPRUNE>(t, h, P1, R[h * N + t], S);
        for (int h = 0; h < 2; ++h)
          for (int t = 0; t < N; ++t) k3b_r2c<N, FPRUNE>(ci, k3, t, h, P1, P2, S, Cout);
      }
    }
  }
  // K3c
  for (long long ci = 0; ci < n; ++ci) {
    if (st[ci].skip) {
      k3c_skipped(a, ci);
      if (a.planes) {
        const long long vol = P12 * P3;
        memset(a.planes + (a.ia_begin + ci - a.planes_begin) * vol, 0, sizeof(double) * (size_t)vol);
      }
      continue;
    }
    const IAGeom3 g = ia_geom3(a, a.ia_begin + ci);
    const LagRanges3 R = lag_ranges3(a, g);
    PeakAcc acc;
    acc.best = 0.0;
    acc.bidx = -1;
    acc.smax = -INFINITY;
    acc.ssum = 0.0;
    for (int q = 0; q < P1 * P2; ++q) k3c_pair<N, ALG>(a, g, st[ci], ci, q, P1, P2, P3, R, acc);
    k3c_final(a, g, ci, R, acc.best, acc.bidx, acc.smax, acc.ssum);
  }
}

template <int N, bool FPRUNE, int ALG>
static void emu3_dt(const Piv3dArgs& a) {
  if (a.dtype == 0) emu3_run<N, FPRUNE, ALG, float>(a);
  else emu3_run<N, FPRUNE, ALG, double>(a);
}

template <int N, bool FPRUNE>
static int emu3_alg(const Piv3dArgs& a, int alg) {
  switch (alg) {
    case 0: emu3_dt<N, FPRUNE, 0>(a); return 0;
    case 1: emu3_dt<N, FPRUNE, 1>(a); return 0;
    case 2: emu3_dt<N, FPRUNE, 2>(a); return 0;
    case 3: emu3_dt<N, FPRUNE, 3>(a); return 0;
    default: return -1;
  }
}

extern "C" __attribute__((visibility("default"))) int mqp_emu_piv3d(
    const void* img1, const void* img2, const void* mask, const void* mask_skip, int dtype, const int* dims,
    const int* IS, const int* SM, const int* st, int alg, double threshold, double mask_threshold, int computeSN,
    double* VF, double* SN, double* planes, long long ia_begin, long long ia_end) {
  std::vector<double> II1, IIg, IIg2;
  Piv3dArgs a;
  memset(&a, 0, sizeof(a));
  a.img1 = img1;
  a.img2 = img2;
  a.mask = mask;
  a.mask_skip = mask_skip;
  a.dtype = dtype;
  a.H = dims[0];
  a.W = dims[1];
  a.D = dims[2];
  if (alg == 1 || alg == 2) {
    integral3(img2, dtype, a.H, a.W, a.D, true, IIg2);
    a.IIg2 = IIg2.data();
  }
  if (alg == 1) {
    integral3(img2, dtype, a.H, a.W, a.D, false, IIg);
    integral3(img1, dtype, a.H, a.W, a.D, false, II1);
    a.IIg = IIg.data();
    a.II1 = II1.data();
  }
  a.VF = VF;
  a.SN = computeSN ? SN : nullptr;
  a.planes = planes;
  a.planes_begin = ia_begin;
  int SS = 0;
  for (int d = 0; d < 3; ++d) {
    a.IS[d] = IS[d];
    a.SM[d] = SM[d];
    a.st[d] = st[d];
    a.vf[d] = (dims[d] - IS[d]) / st[d] + 1;
    SS = IS[d] + 2 * SM[d] > SS ? IS[d] + 2 * SM[d] : SS;
  }
  a.ia_begin = ia_begin;
  a.ia_end = ia_end;
  a.threshold = threshold;
  a.mask_threshold = mask_threshold;
  if (direct3d_ok(a.IS, a.SM)) return emu_piv3d_direct(a, alg);
  const int N = SS <= 32 ? 32 : (SS <= 64 ? 64 : (SS <= 128 ? 128 : 0));
  const bool prune = IS[0] <= N / 2 && IS[1] <= N / 2 && IS[2] <= N / 2;
  if (N == 128) return prune ? emu3_alg<128, true>(a, alg) : -2;
  if (N == 64) return prune ? emu3_alg<64, true>(a, alg) : emu3_alg<64, false>(a, alg);
  if (N == 32) return prune ? emu3_alg<32, true>(a, alg) : emu3_alg<32, false>(a, alg);
  return -2;
}

// the multi-pass predictor (mqp_multipass.cuh), every fine IA
extern "C" __attribute__((visibility("default"))) int mqp_emu_predictor(
    int ndims, const int* vf_f, const int* vf_c, const int* isz_f, const int* st_f, const int* isz_c,
    const int* st_c, const double* VFc, int32_t* pred) {
  PredArgs a;
  memset(&a, 0, sizeof(a));
  a.ndims = ndims;
  long long n = 1;
  for (int d = 0; d < ndims; ++d) {
    a.vf_f[d] = vf_f[d];
    a.vf_c[d] = vf_c[d];
    a.isz_f[d] = isz_f[d];
    a.st_f[d] = st_f[d];
    a.isz_c[d] = isz_c[d];
    a.st_c[d] = st_c[d];
    n *= vf_f[d];
  }
  a.VFc = VFc;
  a.pred = pred;
  for (long long i = 0; i < n; ++i) predictor_at(a, i);
  return 0;
}
