// Fused 2D PIV, team variant: one interrogation area (IA) per team of N
// threads (N = FFT length = 64: two warps; 32: one warp), several teams per
// block.  It computes the same per-IA body as piv2d_kernel (the loop body of
// PIV_CPU, src/multi_quickPIV.jl:63-89) for search windows up to N with
// interrogation windows up to N/2 (the pruned F), FFTCC / ZNCC / NSQECC:
//
//   phase 1  G rows (thread p = window row p, all N rows): r2c along dim 2
//            (copy_search_region!, src/utils/piv_ops.jl:111-127); F rows
//            (thread pair per row, each half of a decimation-in-frequency
//            split: copy_inter_region!, src/utils/piv_ops.jl:95-109), with
//            the skip maximum and the FP64 sumF2.
//   phase 2  spectrum column u by the thread pair (u, h): half h of the
//            length-N transforms along dim 1 of G and F, conj(F) G, inverse
//            (src/crosscorrelation_algorithms/fftcc.jl:101-126).
//   phase 3  lag row s1 by a thread pair: complex-to-real inverse along
//            dim 2, each thread one half of the split; the raw correlation
//            goes to shared memory as FP32.
//   finish   every team thread over the lags: ZNCC/NSQECC normalisation from
//            the FP64 integral images (src/utils/zncc_ops.jl:29-50,
//            src/utils/nsqecc_ops.jl:1-25), the FP64 similarity plane, the
//            first full-overlap peak (src/utils/common_ops.jl:98-124), SN
//            (src/utils/piv_ops.jl:333-367), Gaussian fit (:249-326).
//
// Each thread of a pair runs half-length register FFTs, so the pair does a
// line's transform with half the registers of one thread doing all of it,
// and twice the warps fit on an SM (a team holds about 25 KB of shared
// memory at N = 64: nine IAs, eighteen warps per SM).  The split half is
// uniform across a warp at N = 64 (warp 0 takes half 0, warp 1 half 1); the
// two halves share every transform body and differ only in the short steps
// around it, so the kernel's code stays small enough for the instruction
// cache (a version with one copy of each phase per half stalled on
// instruction fetch).
#pragma once

#include "mqp_piv2d.cuh"

namespace mqp {

// mqp_no_hoist (mqp_fft.cuh) opens each half-specialised phase function, so
// the compiler keeps the two halves' identical loads inside their branches
// of the warp-uniform dispatch instead of hoisting them (which holds both
// halves' data live and spills).

// Shared-memory layout of one team (float2 units).
//   G region: spectrum columns u = 0..M-1 of the G rows (stride GS = N + 1 over
//             the N window rows); after phase 3 the FP64 similarity plane
//             (P1 x P2, row-contiguous).
//   F region: spectrum columns of the F rows (stride FS = M + 1 over M rows);
//             after phase 2 the FP32 raw correlation (column-major P1 x P2).
//   scratch:  team reductions, the IA's scalars and the batch queue head.
template <int N>
struct TeamLayout {
  static constexpr int M = N / 2;
  static constexpr int GS = N + 1;
  static constexpr int FS = M + 1;
  static constexpr int G_MIN = M * GS;
  static constexpr int F_MIN = M * FS;
  static constexpr int SCR = 16;
  static MQP_HD MQP_FI int g_f2(int P1, int P2) { return G_MIN > P1 * P2 ? G_MIN : P1 * P2; }
  static MQP_HD MQP_FI int f_f2(int P1, int P2) {
    const int c = (P1 * P2 + 1) / 2;
    return F_MIN > c ? F_MIN : c;
  }
  static MQP_HD MQP_FI int team_f2(int P1, int P2) { return g_f2(P1, P2) + f_f2(P1, P2) + SCR; }
};

// ---------------------------------------------------------------------------
// phase 1
// ---------------------------------------------------------------------------
// G row p of the padded search window (data on the clipped region only,
// minus the search-region mean there for ZNCC) -> r2c along dim 2 into
// G[u * GS + p] (slot 0 packs the real bins 0 and N/2).
template <int N, typename T, bool ZNCC>
MQP_HD MQP_FI void team_g_row(const Piv2dArgs& a, const IAGeom& g, float mg, int p, float2* G) {
  constexpr int M = N / 2;
  const bool live = p >= g.lo1 && p < g.hi1;
  if (!live) {
#pragma unroll
    for (int u = 0; u < M; ++u) G[u * TeamLayout<N>::GS + p] = make_float2(0.f, 0.f);
    return;
  }
  const T* src = reinterpret_cast<const T*>(a.img2) + ((long long)(g.g01 + p) + (long long)a.H * g.g02);
  const long long H = a.H;
  float2 z[M];
#pragma unroll
  for (int n = 0; n < M; ++n) {
    const int x0 = 2 * n, x1 = 2 * n + 1;
    float v0 = 0.f, v1 = 0.f;
    if (x0 >= g.lo2 && x0 < g.hi2) v0 = (float)ldg_px<T>(src, H * x0);
    if (x1 >= g.lo2 && x1 < g.hi2) v1 = (float)ldg_px<T>(src, H * x1);
    if (ZNCC) {
      v0 = (x0 >= g.lo2 && x0 < g.hi2) ? v0 - mg : 0.f;
      v1 = (x1 >= g.lo2 && x1 < g.hi2) ? v1 - mg : 0.f;
    }
    z[n] = make_float2(v0, v1);
  }
  r2c_store<N, M>(z, G + p, TeamLayout<N>::GS);
}

// F row q (interrogation window row, zero past IS1; minus the IA mean for
// ZNCC), half hh of its length-M complex FFT.  The row's packed input
// z[n] = x[2n] + i x[2n+1] is zero for n >= M/2 (F is at most M wide), so the
// first decimation-in-frequency stage reduces to Z[2k] = FFT_{M/2}(z)[k] and
// Z[2k+1] = FFT_{M/2}(z W_M^n)[k].  Bin k' of the real transform needs Z[k']
// and Z[M-k'], which share k''s parity, so this thread finishes the bins of
// parity hh and writes them to F[k' * FS + q].  The hh = 0 thread also takes
// the raw maximum (skip test) and the FP64 sum of squares of the values.
// Only the twiddle and the bin finishing depend on hh, so the transform
// body exists once for both halves (instruction-cache footprint).
template <int N, int HH>
MQP_HD MQP_FI void team_f_bins(int q, const float2 (&w)[N / 4], float2* F) {
  constexpr int M = N / 2, Q = M / 2, FS = TeamLayout<N>::FS;
  mqp_no_hoist();
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    const int kp = 2 * k + HH;  // bin of the real transform
    if (kp == 0) {
      const float2 Z0 = w[fpos<Q>(0)];
      F[q] = make_float2(2.f * (Z0.x + Z0.y), 2.f * (Z0.x - Z0.y));
      continue;
    }
    const int kk = (M - kp - HH) / 2;  // M - kp = 2 kk + HH
    const float2 A = w[fpos<Q>(k)];
    const float2 B = cconj(w[fpos<Q>(kk)]);
    const float2 e = cadd(A, B);
    const float2 o = cmul_mi(csub(A, B));
    F[kp * FS + q] = cadd(e, rotate<N, false>(o, kp));
  }
}

template <int N, typename T, bool ZNCC>
MQP_HD MQP_FI void team_f_row(const Piv2dArgs& a, const IAGeom& g, double meanF, int q, int hh, float2* F,
                              double& vmax, double& sumsq) {
  constexpr int M = N / 2, Q = M / 2, FS = TeamLayout<N>::FS;
  if (q >= a.IS1) {
    for (int k = 0; k < Q; ++k) F[(2 * k + hh) * FS + q] = make_float2(0.f, 0.f);
    return;
  }
  const T* src = reinterpret_cast<const T*>(a.img1) + ((long long)(g.ir1 + q) + (long long)a.H * g.ir2);
  const long long H = a.H;
  float2 w[Q];
#pragma unroll
  for (int n = 0; n < Q; ++n) {
    float v[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int x = 2 * n + e;
      v[e] = 0.f;
      if (x < a.IS2) {
        const T r = ldg_px<T>(src, H * x);
        const double val = (double)r - meanF;
        if (hh == 0) {
          vmax = (double)r > vmax ? (double)r : vmax;
          sumsq += val * val;
        }
        v[e] = (float)val;
      }
    }
    w[n] = make_float2(v[0], v[1]);
  }
  if (hh) {
#pragma unroll
    for (int n = 1; n < Q; ++n) w[n] = rotate<M, false>(w[n], n);
  }
  fft_reg<Q, false>(w);  // Z[2k + hh] = w[fpos<Q>(k)]
  if (hh) team_f_bins<N, 1>(q, w, F);
  else team_f_bins<N, 0>(q, w, F);
}

// ---------------------------------------------------------------------------
// phase 2: spectrum column u, half H2 (bins k1 = 2m + H2 along dim 1)
// ---------------------------------------------------------------------------
// The first DIF stage along dim 1 folds the N rows of G into the half
// (g[n] + g[n+M] for H2 = 0, (g[n] - g[n+M]) W_N^n for H2 = 1); F has M rows
// (zero past them), so its half is f[n] or f[n] W_N^n.  The pair meets in
// shared memory twice: every thread of the team has read the G columns before
// any writes its transformed half back (team barrier `sync`), and phase 3
// combines the two halves' inverses A0[s] + W_N^-s A1[s] (s < M) and
// A0[s] - W_N^-s A1[s] (s + M).  On return G[u] holds A0 in slots 0..M-1 and
// W_N^-s A1[s] in slots M..N-1.
// The three transforms of a column half (G forward, F forward, the product's
// inverse through the forward transform of its conjugate) run as stages
// st = 0, 1, 2 of one loop around a single FFT body; team_p2_pre loads the
// stage's input into t, team_p2_post consumes the transform.  Between the
// transform and the post of stage 0 the team synchronises (every column has
// been read before the halves are written back into it).
template <int N, int H2>
MQP_HD MQP_FI void team_p2_fold(const float2* Gc, float2 (&t)[N / 2]) {
  constexpr int M = N / 2;
  mqp_no_hoist();
#pragma unroll
  for (int n = 0; n < M; ++n) {
    const float2 a0 = Gc[n], a1 = Gc[n + M];
    t[n] = H2 ? rotate<N, false>(csub(a0, a1), n) : cadd(a0, a1);
  }
}

template <int N, int H2>
MQP_HD MQP_FI void team_p2_fload(const float2* Fc, float2 (&t)[N / 2]) {
  constexpr int M = N / 2;
  mqp_no_hoist();
#pragma unroll
  for (int n = 0; n < M; ++n) t[n] = H2 ? rotate<N, false>(Fc[n], n) : Fc[n];
}

template <int N>
MQP_HD MQP_FI void team_p2_pre(int st, int u, int h, const float2* G, const float2* F, float2 (&t)[N / 2]) {
  if (st == 0) {
    const float2* Gc = G + u * TeamLayout<N>::GS;
    if (h) team_p2_fold<N, 1>(Gc, t);
    else team_p2_fold<N, 0>(Gc, t);
  } else if (st == 1) {
    const float2* Fc = F + u * TeamLayout<N>::FS;
    if (h) team_p2_fload<N, 1>(Fc, t);
    else team_p2_fload<N, 0>(Fc, t);
  }
}

// t = conj(conj(F^) G^) in natural order from F^ (fpos slots of t) and the
// column's G^ half; column 0 carries the two real rows k2 = 0 and k2 = N/2 as
// A + iB (see half_product)
template <int N, int H2>
MQP_HD MQP_FI void team_p2_product(bool packed, const float2* Gh, float2 (&t)[N / 2]) {
  constexpr int M = N / 2;
  float2 p[M];
  if (!packed) {
    mqp_no_hoist();
#pragma unroll
    for (int m = 0; m < M; ++m) p[m] = cconj(cmulc(t[fpos<M>(m)], Gh[m]));
  } else {
    mqp_no_hoist();
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const int mm = H2 ? M - 1 - m : (M - m) & (M - 1);  // the mirror bin's index in this half
      if (mm < m) continue;
      const float2 Zk = Gh[m], Zn = cconj(Gh[mm]);
      const float2 Fk = t[fpos<M>(m)], Fn = cconj(t[fpos<M>(mm)]);
      const float2 A = cscale(cadd(Zk, Zn), 0.5f), B = cscale(cmul_mi(csub(Zk, Zn)), 0.5f);
      const float2 Af = cscale(cadd(Fk, Fn), 0.5f), Bf = cscale(cmul_mi(csub(Fk, Fn)), 0.5f);
      const float2 PA = cmulc(Af, A), PB = cmulc(Bf, B);
      p[m] = cconj(cadd(PA, cmul_pi(PB)));
      if (mm != m) p[mm] = cconj(cadd(cconj(PA), cmul_pi(cconj(PB))));
    }
  }
#pragma unroll
  for (int m = 0; m < M; ++m) t[m] = p[m];
}

template <int N, int H2>
MQP_HD MQP_FI void team_p2_store_inverse(float2* Gh, const float2 (&t)[N / 2]) {
  constexpr int M = N / 2;
#pragma unroll
  for (int s = 0; s < M; ++s) {
    const float2 A = cconj(t[fpos<M>(s)]);
    Gh[s] = H2 ? rotate<N, true>(A, s) : A;
  }
}

template <int N>
MQP_HD MQP_FI void team_p2_post(int st, int u, int h, float2* G, float2 (&t)[N / 2]) {
  constexpr int M = N / 2;
  float2* Gh = G + u * TeamLayout<N>::GS + h * M;
  if (st == 0) {
#pragma unroll
    for (int m = 0; m < M; ++m) Gh[m] = t[fpos<M>(m)];
  } else if (st == 1) {
    if (h) team_p2_product<N, 1>(u == 0, Gh, t);
    else team_p2_product<N, 0>(u == 0, Gh, t);
  } else {
    if (h) team_p2_store_inverse<N, 1>(Gh, t);
    else team_p2_store_inverse<N, 0>(Gh, t);
  }
}

// On return G[u] holds A0 in slots 0..M-1 and W_N^-s A1[s] in slots M..N-1.
template <int N, typename Sync>
MQP_HD MQP_FI void team_phase2(int u, int h, float2* G, const float2* F, Sync sync) {
  float2 t[N / 2];
#pragma unroll 1
  for (int st = 0; st < 3; ++st) {
    team_p2_pre<N>(st, u, h, G, F, t);
    fft_reg<N / 2, false>(t);
    if (st == 0) sync();
    team_p2_post<N>(st, u, h, G, t);
  }
}

// ---------------------------------------------------------------------------
// phase 3: lag row s1, half HH of the complex-to-real inverse along dim 2
// ---------------------------------------------------------------------------
// Row s1's spectrum X[u] = A0[u][s] + R1[u][s] (s1 = s < M) or A0 - R1
// (s1 = s + M).  The c2r input t[k] (conjugated, see c2r_pre) goes through
// one decimation-in-frequency step: outputs n = 2j + HH come from a length-M/2
// FFT of t[k] + t[k+M/2] (HH = 0) or (t[k] - t[k+M/2]) W_M^k (HH = 1).  Output
// n gives cc[2n] and cc[2n+1]; they go to cc[s1 + P1 * s2] as FP32 (scaled).
template <int N>
MQP_HD MQP_FI void team_phase3_row(int s1, int hh, int P1, int P2, const float2* G, float* cc, float scale) {
  mqp_no_hoist();
  constexpr int M = N / 2, Q = M / 2, GS = TeamLayout<N>::GS;
  const int s = s1 < M ? s1 : s1 - M;
  const float sg = s1 < M ? 1.f : -1.f;
  auto X = [&](int u) {
    const float2 a0 = G[u * GS + s], r1 = G[u * GS + M + s];
    return make_float2(a0.x + sg * r1.x, a0.y + sg * r1.y);
  };
  // c2r input bin k from X[k] and X[M-k] (see c2r_pre)
  auto tk = [](float2 A, float2 Bm, int k) {
    const float2 B = cconj(Bm);
    const float2 E = cadd(A, B);
    const float2 O = rotate<N, true>(csub(A, B), k);
    return cconj(cadd(E, cmul_pi(O)));
  };
  // the DIF fold of the half: lo + hi (hh = 0) or (lo - hi) W_M^k (hh = 1),
  // selected per element so both halves share this code
  const float fs = hh ? -1.f : 1.f;
  auto fold = [&](float2 lo, float2 hi, int k) {
    const float2 d = make_float2(lo.x + fs * hi.x, lo.y + fs * hi.y);
    const float2 r = rotate<M, false>(d, k);
    return hh ? r : d;
  };
  // bins {k, Q-k, Q+k, M-k} close under both pairings (k with M-k for the
  // c2r split, k with k+Q for the DIF fold): four spectrum reads give y[k]
  // and y[Q-k], so only the half-length input stays live
  float2 y[Q];
  {
    const float2 X0 = X(0), XQ = X(Q);
    const float2 t0 = cconj(cadd(make_float2(X0.x + X0.y, 0.f), cmul_pi(make_float2(X0.x - X0.y, 0.f))));
    const float2 tq = tk(XQ, XQ, Q);
    y[0] = fold(t0, tq, 0);
  }
#pragma unroll
  for (int k = 1; k <= Q / 2; ++k) {
    const int k2 = Q - k, k3 = Q + k, k4 = M - k;
    const float2 a = X(k), b = X(k2), c = X(k3), d = X(k4);
    const float2 ta = tk(a, d, k), td = tk(d, a, k4);
    const float2 tb = tk(b, c, k2), tc = tk(c, b, k3);
    y[k] = fold(ta, tc, k);
    if (k2 != k) y[k2] = fold(tb, td, k2);
  }
  fft_reg<Q, false>(y);
#pragma unroll
  for (int j = 0; j < Q; ++j) {
    const int n = 2 * j + hh;
    const float2 T = y[fpos<Q>(j)];
    if (2 * n < P2) cc[s1 + P1 * (2 * n)] = T.x * scale;
    if (2 * n + 1 < P2) cc[s1 + P1 * (2 * n + 1)] = -T.y * scale;
  }
}

// Lag row s1 = M (when 2*SM1+1 = M+1) at lag s2, computed directly:
// x[s2] = X[0] + (-1)^s2 X[N/2] + 2 sum_{k=1}^{M-1} Re(X[k] e^{+2 pi i k s2 / N})
// with X[u] = A0[u][0] - R1[u][0]; tw = (cos, sin)(2 pi j / N).
template <int N>
MQP_HD MQP_FI float team_tail_value(const float2* G, const float2* tw, int s2) {
  constexpr int M = N / 2, GS = TeamLayout<N>::GS;
  const float2 X0 = csub(G[0], G[M]);
  float acc = 0.f;
  int t = 0;
#pragma unroll 4
  for (int k = 1; k < M; ++k) {
    t = (t + s2) & (N - 1);
    const float2 X = csub(G[k * GS], G[k * GS + M]);
    const float2 w = tw[t];
    acc += X.x * w.x - X.y * w.y;
  }
  return X0.x + ((s2 & 1) ? -X0.y : X0.y) + 2.f * acc;
}

// Similarity at lag (s1, s2) from the raw correlation c (finish_row's sums).
template <int ALG>
MQP_HD MQP_FI double team_similarity(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, float sqF, int s1,
                                     int s2, double c) {
  if (ALG == ALG_FFTCC) return c;
  int r0, r1, c0, c1;
  lag_window(s1, a.IS1, g.g01, g.lo1, g.hi1, r0, r1);
  lag_window(s2, a.IS2, g.g02, g.lo2, g.hi2, c0, c1);
  double S2 = 0.0, S1 = 0.0, n = 0.0;
  if (r1 > r0 && c1 > c0) {
    const long long ld = (long long)a.H + 1;
    const double* A0 = a.IIg2 + ld * c0;
    const double* A1 = a.IIg2 + ld * c1;
    S2 = (A1[r1] - A1[r0]) - (A0[r1] - A0[r0]);
    if (ALG == ALG_ZNCC) {
      const double* B0 = a.IIg + ld * c0;
      const double* B1 = a.IIg + ld * c1;
      S1 = (B1[r1] - B1[r0]) - (B0[r1] - B0[r0]);
      n = (double)(r1 - r0) * (double)(c1 - c0);
    }
  }
  return similarity_value<ALG>(sc, sqF, c, S2, S1, n);
}

}  // namespace mqp
