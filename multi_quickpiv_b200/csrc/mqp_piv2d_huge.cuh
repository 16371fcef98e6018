// 2D PIV for search windows of 129..256 per axis (FFT length 256), the
// coarse passes of interSize-128 refinements or large margins: one block of
// 256 threads per interrogation area (IA), the per-IA body of PIV_CPU's loop
// (src/multi_quickPIV.jl:63-89).  A 256 x 256 spectrum does not fit in shared
// memory, so the stages meet in a per-block scratch slot in global memory
// (L2-resident: one slot per resident block):
//
//   A  rows: G row t (256 rows) by a thread pair per round, the 128-point
//      packed complex transform split by one decimation-in-frequency step
//      (each thread a 64-point register FFT) and finished into bins of its
//      parity (the r2c split pairs k with 128-k, same parity); F rows
//      (interrogation window up to 128) likewise, one round.  Spectra to
//      GS[k2][x1] and FS[k2][x1] (copy_*_region!, src/utils/piv_ops.jl:95-127).
//   B  columns: column k2 by a thread quad, the 256-point transform split by
//      one radix-4 decimation-in-frequency step (bins 4m + q to thread q);
//      conj(F) G; the inverses recombined across the quad through shared
//      memory; lags s1 < P1 to LG[k2][s1].
//      (src/crosscorrelation_algorithms/fftcc.jl:101-126)
//   C  lag rows: the complex-to-real inverse along k2 split over a thread
//      pair, raw correlation (FP32) to CC[s1 + P1 s2].
//   D  finish: ZNCC / NSQECC similarity from the FP64 integral images into the
//      FP64 plane PL, first full-overlap peak, SN, Gaussian fit
//      (src/utils/zncc_ops.jl:29-50, nsqecc_ops.jl:1-25,
//      src/utils/common_ops.jl:98-124, src/utils/piv_ops.jl:249-367).
#pragma once

#include "mqp_piv2d_team.cuh"

namespace mqp {

constexpr int NH = 256;          // FFT length
constexpr int MH = NH / 2;       // packed spectrum columns, complex row length
constexpr int QH = 64;           // register FFT length of every split transform
constexpr int HUGE_THREADS = 256;

// Per-block scratch slot (float2 units), sized for the pass's lags so that
// all resident blocks' slots stay in L2:
//   stages A-B  LG [k2][s1] (128 x P1) | GS [k2][x1] (128 x 256) | FS [k2][x1] (128 x 128)
//   stages C-D  LG | CC (P1 P2 floats, over the dead GS) | PL (P1 P2 doubles, after CC)
struct HugeSlot {
  long long lg, gs, fs, cc, pl, total;
  MQP_HD HugeSlot(int P1, int P2) {
    lg = 0;
    gs = (long long)MH * P1;
    fs = gs + (long long)MH * NH;
    cc = gs;
    pl = cc + ((long long)P1 * P2 + 1) / 2;
    const long long ab = fs + (long long)MH * MH, cd = pl + (long long)P1 * P2;
    total = ((ab > cd ? ab : cd) + 15) / 16 * 16;  // slots on 128-byte boundaries
  }
};

// Shared memory (float2 units): the park/exchange area of stage B (64
// columns x 4 quarters x 64 values, element (col, q, m) at m * 256 + q * 64 +
// col so that a warp's 32 columns fall in distinct banks), the packed column's staging (2 x 256),
// the twiddle table (256) and reduction slots.
struct HugeSmem {
  static constexpr int PARK = 64 * 4 * QH;
  static constexpr int PACK = 2 * NH;
  static constexpr int TW = NH;
  static constexpr int RED = 32;
  static constexpr int TOTAL = PARK + PACK + TW + RED;
};

// ---------------------------------------------------------------------------
// stage A: rows
// ---------------------------------------------------------------------------
// The 64-point halves of the packed 128-point row transform finished into
// the real transform's bins of parity HH (r2c split, as team_f_bins).
template <int HH>
MQP_HD MQP_FI void huge_row_bins(const float2 (&w)[QH], float2* out, long long kstride) {
  mqp_no_hoist();
#pragma unroll
  for (int k = 0; k < QH; ++k) {
    const int kp = 2 * k + HH;
    if (kp == 0) {
      const float2 Z0 = w[fpos<QH>(0)];
      out[0] = make_float2(2.f * (Z0.x + Z0.y), 2.f * (Z0.x - Z0.y));
      continue;
    }
    const int kk = (MH - kp - HH) / 2;  // MH - kp = 2 kk + HH
    const float2 A = w[fpos<QH>(k)];
    const float2 B = cconj(w[fpos<QH>(kk)]);
    out[kp * kstride] = cadd(cadd(A, B), rotate<NH, false>(cmul_mi(csub(A, B)), kp));
  }
}

// G row t: data on the clipped search region (minus the search mean for
// ZNCC), packed z[n] = x[2n] + i x[2n+1], folded z[n] + z[n+64] (half 0) and
// (z[n] - z[n+64]) W_128^n (half 1), each transformed and finished into the
// bins of its parity at GS[k2 * 256 + t].  Every pixel is loaded once: the
// first 128 pass through the thread's column of `stage` (stage[x * 256 + t],
// 128 KB of shared memory), the second 128 meet them there, half 0's fold
// stays in registers and half 1's difference goes back to the stage.
template <typename T, bool ZNCC>
MQP_HD MQP_FI void huge_g_row(const Piv2dArgs& a, const IAGeom& g, float mg, int t, float2* GS, float* stage) {
  const bool live = t >= g.lo1 && t < g.hi1;
  const T* src = reinterpret_cast<const T*>(a.img2) + ((long long)(g.g01 + t) + (long long)a.H * g.g02);
  const long long H = a.H;
  float* col = stage + t;
  auto px = [&](int xx) {
    float v = 0.f;
    if (live && xx >= g.lo2 && xx < g.hi2) {
      v = (float)ldg_px<T>(src, H * xx);
      if (ZNCC) v -= mg;
    }
    return v;
  };
#pragma unroll 16
  for (int x = 0; x < MH; ++x) col[x * NH] = px(x);
  float2 w[QH];
#pragma unroll
  for (int n = 0; n < QH; ++n) {
    if (n % 8 == 0) mqp_no_hoist();
    const float h0 = px(MH + 2 * n), h1 = px(MH + 2 * n + 1);
    const float l0 = col[(2 * n) * NH], l1 = col[(2 * n + 1) * NH];
    w[n] = make_float2(l0 + h0, l1 + h1);
    col[(2 * n) * NH] = l0 - h0;
    col[(2 * n + 1) * NH] = l1 - h1;
  }
  fft_reg<QH, false>(w);
  huge_row_bins<0>(w, GS + t, NH);
  mqp_no_hoist();
#pragma unroll
  for (int n = 0; n < QH; ++n) {
    const float2 d = make_float2(col[(2 * n) * NH], col[(2 * n + 1) * NH]);
    w[n] = n ? rotate<MH, false>(d, n) : d;
  }
  fft_reg<QH, false>(w);
  huge_row_bins<1>(w, GS + t, NH);
}

// F row q (< 128), half hh: the IA row (minus the IA mean for ZNCC), at most
// 128 wide, so z[n] = 0 for n >= 64 and the fold is z[n] (times W_128^n for
// hh = 1); bins of parity hh to FS[k2 * 128 + q].  The hh = 0 thread takes the
// raw maximum and the FP64 sum of squares.
template <typename T, bool ZNCC>
MQP_HD MQP_FI void huge_f_row(const Piv2dArgs& a, const IAGeom& g, double meanF, int q, int hh, float2* FS,
                              double& vmax, double& sumsq) {
  float2 w[QH];
  if (q < a.IS1) {
    const T* src = reinterpret_cast<const T*>(a.img1) + ((long long)(g.ir1 + q) + (long long)a.H * g.ir2);
    const long long H = a.H;
#pragma unroll
    for (int n = 0; n < QH; ++n) {
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
      for (int n = 1; n < QH; ++n) w[n] = rotate<MH, false>(w[n], n);
    }
  } else {
#pragma unroll
    for (int n = 0; n < QH; ++n) w[n] = make_float2(0.f, 0.f);
  }
  fft_reg<QH, false>(w);
  float2* out = FS + q;
  if (hh) huge_row_bins<1>(w, out, MH);
  else huge_row_bins<0>(w, out, MH);
}

// ---------------------------------------------------------------------------
// stage B: columns (thread quad per column, quarter q warp-uniform)
// ---------------------------------------------------------------------------
// Radix-4 fold of a 256-point column into quarter q:
//   y[n] = W_256^{nq} sum_j x[n + 64 j] W_4^{jq}   (n < 64)
// whose 64-point transform gives the bins 4m + q.  src(j, n) = x[n + 64 j].
template <typename Src>
MQP_HD MQP_FI void huge_fold4(int q, Src src, const float2* tw, float2 (&y)[QH]) {
#pragma unroll
  for (int n = 0; n < QH; ++n) {
    const float2 x0 = src(0, n), x1 = src(1, n), x2 = src(2, n), x3 = src(3, n);
    float2 s;
    // W_4^{jq} = (-i)^{jq}
    if (q == 0) s = cadd(cadd(x0, x1), cadd(x2, x3));
    else if (q == 1) s = cadd(csub(x0, x2), cmul_mi(csub(x1, x3)));
    else if (q == 2) s = csub(cadd(x0, x2), cadd(x1, x3));
    else s = cadd(csub(x0, x2), cmul_pi(csub(x1, x3)));
    const float2 w = tw[(n * q) & (NH - 1)];  // (cos, sin)(2 pi n q / 256): W_256^{nq} = cos - i sin
    y[n] = make_float2(s.x * w.x + s.y * w.y, s.y * w.x - s.x * w.y);
  }
}

// Element stride of one thread's park slots (see HugeSmem).
constexpr int HPS = 4 * 64;

// Part 1 of a column: G's quarter transformed and parked in shared memory
// (park[m * HPS] = G^[4m + q], natural m) and F's quarter transformed into f.
MQP_HD MQP_FI void huge_col_forward(int k2, int q, const float2* GS, const float2* FS, const float2* tw,
                                    float2* park, float2 (&f)[QH]) {
  mqp_no_hoist();
  {
    float2 y[QH];
    const float2* gc = GS + (long long)k2 * NH;
    huge_fold4(q, [&](int j, int n) { return gc[n + QH * j]; }, tw, y);
    fft_reg<QH, false>(y);
#pragma unroll
    for (int m = 0; m < QH; ++m) park[m * HPS] = y[fpos<QH>(m)];
  }
  mqp_no_hoist();
  const float2* fc = FS + (long long)k2 * MH;
  const float2 z0 = make_float2(0.f, 0.f);
  huge_fold4(q, [&](int j, int n) { return j < 2 ? fc[n + QH * j] : z0; }, tw, f);
  fft_reg<QH, false>(f);  // F^[4m + q] at f[fpos(m)]
}

// Part 2: t = conj(conj(F^) G^) for the quarter's bins, written over the
// park (park[m * HPS] for bin 4m + q) so that f dies before the inverse loads it.
// The packed column k2 = 0 carries the real rows k2 = 0 and 128 as A + iB;
// its product pairs bin k with -k, whose quarter is (-q) mod 4, so the quad
// stages both spectra in `pack` (G^ then F^, natural bin order) first.
MQP_HD MQP_FI void huge_col_product(int k2, int q, float2* park, const float2* pack, const float2 (&f)[QH]) {
  if (k2 != 0) {
#pragma unroll
    for (int m = 0; m < QH; ++m) park[m * HPS] = cconj(cmulc(f[fpos<QH>(m)], park[m * HPS]));
    return;
  }
  const float2* Gp = pack;
  const float2* Fp = pack + NH;
  for (int m = 0; m < QH; ++m) {
    const int k = 4 * m + q, kn = (NH - k) & (NH - 1);
    const float2 Zk = Gp[k], Zn = cconj(Gp[kn]);
    const float2 Fk = Fp[k], Fn = cconj(Fp[kn]);
    const float2 A = cscale(cadd(Zk, Zn), 0.5f), B = cscale(cmul_mi(csub(Zk, Zn)), 0.5f);
    const float2 Af = cscale(cadd(Fk, Fn), 0.5f), Bf = cscale(cmul_mi(csub(Fk, Fn)), 0.5f);
    const float2 PA = cmulc(Af, A), PB = cmulc(Bf, B);
    park[m * HPS] = cconj(cadd(PA, cmul_pi(PB)));
  }
}

// Part 3: the quarter's 64-point inverse (through the forward transform of
// the conjugate products parked at park[m * HPS]), twiddled W_256^{-s q}
// z_q[s], written back over the park: park[s * HPS] = xch[q][s].
MQP_HD MQP_FI void huge_col_inverse(int q, float2* park, const float2* tw) {
  mqp_no_hoist();
  float2 t[QH];
#pragma unroll
  for (int m = 0; m < QH; ++m) t[m] = park[m * HPS];
  fft_reg<QH, false>(t);
#pragma unroll
  for (int s = 0; s < QH; ++s) {
    const float2 z = cconj(t[fpos<QH>(s)]);
    const float2 w = tw[(s * q) & (NH - 1)];  // W_256^{-sq} = cos + i sin
    park[s * HPS] = make_float2(z.x * w.x - z.y * w.y, z.x * w.y + z.y * w.x);
  }
}

// Part 4 (after the quad's exchange): lags s1 = s + 64 p of the column,
//   x[s + 64p] = sum_q W_4^{-pq} xch[q][s],   xch[q][s] = xch[s * HPS + q * 64],
// those below P1 to LG[k2 * P1 + s1].
MQP_HD MQP_FI void huge_col_combine(int k2, int p, int P1, const float2* xch, float2* LG) {
#pragma unroll 4
  for (int s = 0; s < QH; ++s) {
    const int s1 = s + QH * p;
    if (s1 >= P1) break;
    const float2* e = xch + s * HPS;
    const float2 a0 = e[0], a1 = e[QH], a2 = e[2 * QH], a3 = e[3 * QH];
    float2 v;
    // W_4^{-pq} = (+i)^{pq}
    if (p == 0) v = cadd(cadd(a0, a1), cadd(a2, a3));
    else if (p == 1) v = cadd(csub(a0, a2), cmul_pi(csub(a1, a3)));
    else if (p == 2) v = csub(cadd(a0, a2), cadd(a1, a3));
    else v = cadd(csub(a0, a2), cmul_mi(csub(a1, a3)));
    LG[(long long)k2 * P1 + s1] = v;
  }
}

// Stage B for thread t in round r (columns k2 = 64 r + t % 64, quarter
// q = t / 64): part 1, then (block barrier) part 2, then (block barrier)
// part 3, then a block barrier before the next round reuses the park.
// park: 64 columns x 4 quarters x 64 values (HugeSmem); the quad of column c
// exchanges through its own slots, based at park[c].
MQP_HD MQP_FI void huge_b_part1(int r, int t, const float2* GS, const float2* FS, const float2* tw, float2* park,
                                float2* pack, float2 (&f)[QH]) {
  const int col = t % 64, q = t / 64, k2 = r * 64 + col;
  float2* mine = park + q * 64 + col;
  huge_col_forward(k2, q, GS, FS, tw, mine, f);
  if (k2 == 0) {
    // the packed column's spectra in natural bin order for its mirror pairs
#pragma unroll
    for (int m = 0; m < QH; ++m) {
      pack[4 * m + q] = mine[m * HPS];
      pack[NH + 4 * m + q] = f[fpos<QH>(m)];
    }
  }
}
MQP_HD MQP_FI void huge_b_part2(int r, int t, const float2* tw, float2* park, const float2* pack,
                                const float2 (&f)[QH]) {
  const int col = t % 64, q = t / 64, k2 = r * 64 + col;
  float2* mine = park + q * 64 + col;
  huge_col_product(k2, q, mine, pack, f);
  huge_col_inverse(q, mine, tw);
}
MQP_HD MQP_FI void huge_b_part3(int r, int t, int P1, const float2* park, float2* LG) {
  const int col = t % 64, q = t / 64, k2 = r * 64 + col;
  huge_col_combine(k2, q, P1, park + col, LG);
}

// ---------------------------------------------------------------------------
// stage C: lag row s1, half hh of the complex-to-real inverse along k2
// ---------------------------------------------------------------------------
// As team_phase3_row with the row's spectrum X[u] = LG[u * P1 + s1].
MQP_HD MQP_FI void huge_lag_row(int s1, int hh, int P1, int P2, const float2* LG, float* cc, float scale) {
  mqp_no_hoist();
  constexpr int M = MH, Q = QH;
  auto X = [&](int u) { return LG[(long long)u * P1 + s1]; };
  auto tk = [](float2 A, float2 Bm, int k) {
    const float2 B = cconj(Bm);
    const float2 E = cadd(A, B);
    const float2 O = rotate<NH, true>(csub(A, B), k);
    return cconj(cadd(E, cmul_pi(O)));
  };
  const float fs = hh ? -1.f : 1.f;
  auto fold = [&](float2 lo, float2 hi, int k) {
    const float2 d = make_float2(lo.x + fs * hi.x, lo.y + fs * hi.y);
    const float2 r = rotate<M, false>(d, k);
    return hh ? r : d;
  };
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

}  // namespace mqp
