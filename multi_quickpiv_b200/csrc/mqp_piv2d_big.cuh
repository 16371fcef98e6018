// 2D PIV for search windows up to 128 (FFT length NB = 128): one block of
// 128 threads per interrogation area (IA), the per-IA body of PIV_CPU's loop
// (src/multi_quickPIV.jl:63-89) for the large windows of coarse multi-pass
// levels (interSize 64, searchMargin 32).  Same mathematics as the warp
// kernel (mqp_piv2d.cuh), laid out for a 128-point transform that does not
// fit one thread:
//
//   rows     thread t = window row: r2c of the real 128-point row along dim 2
//            through one 64-point complex FFT (r2c_store); spectra rows
//            k2 = 0..63 go to shared memory, k2 = 0 and k2 = 64 (both real)
//            packed as one complex row.
//   columns  lanes (2c, 2c+1) own spectrum column c: a first radix-2 DIF
//            stage splits each 128-point column transform into its even and
//            odd bins, one 64-point FFT per lane, for G and F; conj(F) G; the
//            64-point inverses are recombined as
//              x[s] = A0[s] + W^-s A1[s],  x[s+64] = A0[s] - W^-s A1[s]
//            with the partner's half read through the pair's own row of
//            shared memory.  Lags s1 < P1 stay.
//   lags     thread t = lag row s1: complex-to-real inverse along k2.
//   finish   ZNCC / NSQECC / masked normalisation from the FP64 integral
//            images, first full-overlap maximum, SN and the Gaussian fit,
//            shared with the warp kernel (finish_row, refine2d).
#pragma once

#include "mqp_piv2d.cuh"

namespace mqp {

// The phases are separate (not inlined) functions on the device so that each
// 64-point transform gets the whole register file; their arrays never cross a
// phase boundary.
#if defined(__CUDACC__)
#define MQP_PHASE __host__ __device__ __noinline__
#else
#define MQP_PHASE inline
#endif

constexpr int NB = 128;      // FFT length
constexpr int MB = NB / 2;   // spectrum rows / complex half length
constexpr int BIG_THREADS = 128;

template <bool FPRUNE>
struct LayBig {
  static constexpr int NF = FPRUNE ? MB : NB;  // F columns (dim 1 extent) kept
  static constexpr int SSTR = NB + 1;          // G spectra rows: k2 x x1
  static constexpr int FSTR = NF + 1;          // F spectra rows
  static constexpr int TSTR = MB + 1;          // lag rows after the columns: s1 x k2
  static constexpr int S_OFF = 0;
  static constexpr int S_SIZE = MB * SSTR;
  static constexpr int F_OFF = S_SIZE;
  static constexpr int F_SIZE = MB * FSTR;
  // the FP64 plane (P1 x P2 doubles) reuses the F rows after the columns
  static MQP_HD MQP_FI int region2(int P1, int P2) { return F_SIZE > P1 * P2 ? F_SIZE : P1 * P2; }
  static MQP_HD MQP_FI int extra(bool masked, int P1, int P2) { return masked ? (P1 * P2 + 1) / 2 : 0; }
  // after the plane (and the parked masked correlation): the packed column's
  // F bins (2 x 64) and RED_F2 slots (16 doubles) of block reduction
  static constexpr int RED_F2 = 16;
  static MQP_HD MQP_FI int pk_off(int P1, int P2, bool masked) { return S_SIZE + region2(P1, P2) + extra(masked, P1, P2); }
  static MQP_HD MQP_FI int total_f2(int P1, int P2, bool masked) { return pk_off(P1, P2, masked) + 2 * MB + RED_F2; }
};

// ---- rows -------------------------------------------------------------------
// Row t of G (the padded search window, data on the clipped region only;
// minus the search mean for ZNCC; squared for the masked second
// correlation) and, for t < NF, row t of F (the IA row; minus the IA mean
// for ZNCC; times the mask, or the mask, for masked NSQECC).  Accumulates
// the F row's skip maxima and sumF2 like row_process.
template <bool FPRUNE, typename T, int ALG>
MQP_PHASE void big_rows(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, int PASS, int t, float2* S,
                        float2* SF, double& vmax, double& mmax, double& sumsq) {
  using L = LayBig<FPRUNE>;
  {  // G row t
    float2 z[MB];
    const bool live = t >= g.lo1 && t < g.hi1;
    if (live) {
      const T* p = reinterpret_cast<const T*>(a.img2) + ((long long)(g.g01 + t) + (long long)a.H * g.g02);
      const float mg = (float)sc.meanG;
      float w[NB];
#pragma unroll
      for (int x = 0; x < NB; ++x) {
        w[x] = 0.f;
        if (x >= g.lo2 && x < g.hi2) {
          float v = (float)ldg_px<T>(p, (long long)a.H * x);
          if (ALG == ALG_ZNCC) v = v - mg;
          if (PASS == PASS_MASK_SQ) v = v * v;
          w[x] = v;
        }
      }
#pragma unroll
      for (int n = 0; n < MB; ++n) z[n] = make_float2(w[2 * n], w[2 * n + 1]);
      r2c_store<NB, MB>(z, S + t, L::SSTR);
    } else {
      zero_strided(S + t, MB, L::SSTR);
    }
  }
  if (t < L::NF) {  // F row t
    float2* out = SF + t;
    if (t >= a.IS1) {
      zero_strided(out, MB, L::FSTR);
      return;
    }
    const long long base = (long long)(g.ir1 + t) + (long long)a.H * g.ir2;
    const T* p = reinterpret_cast<const T*>(a.img1) + base;
    const T* q = PASS != PASS_PLAIN ? reinterpret_cast<const T*>(a.mask) + base : p;
    const T* qs = PASS == PASS_MASKED ? reinterpret_cast<const T*>(a.mask_skip ? a.mask_skip : a.mask) + base : p;
    float w[NB];
#pragma unroll
    for (int x = 0; x < NB; ++x) {
      w[x] = 0.f;
      if (x < L::NF && x < a.IS2) {
        const long long off = (long long)a.H * x;
        if (PASS == PASS_PLAIN) {
          const T r = ldg_px<T>(p, off);
          vmax = (double)r > vmax ? (double)r : vmax;
          const double val = (double)r - sc.meanF;
          sumsq += val * val;
          w[x] = (float)val;
        } else if (PASS == PASS_MASKED) {
          const T r = ldg_px<T>(p, off);
          const T mk = ldg_px<T>(q, off);
          const T ms = ldg_px<T>(qs, off);
          vmax = (double)r > vmax ? (double)r : vmax;
          mmax = (double)ms > mmax ? (double)ms : mmax;
          const double val = (double)r * (double)mk;
          sumsq += val * val / ((double)mk > 0.0 ? (double)mk : 1.0);
          w[x] = (float)val;
        } else {
          w[x] = (float)ldg_px<T>(q, off);
        }
      }
    }
    float2 z[MB];
#pragma unroll
    for (int n = 0; n < MB; ++n) z[n] = make_float2(w[2 * n], w[2 * n + 1]);
    r2c_store<NB, FPRUNE ? MB / 2 : MB>(z, out, L::FSTR);
  }
}

// ---- columns ----------------------------------------------------------------
// Step 1 (lane t: column c = t/2, half h = t%2): the DIF split and 64-point
// FFT of G column c; y[fpos(m)] = bin 2m+h.
template <bool FPRUNE>
MQP_HD MQP_FI void big_col_g(int t, const float2* S, float2 (&y)[MB]) {
  using L = LayBig<FPRUNE>;
  const int c = t >> 1, h = t & 1;
  const float2* row = S + c * L::SSTR;
  if (h) {
#pragma unroll
    for (int n = 0; n < MB; ++n) y[n] = rotate<NB, false>(csub(row[n], row[n + MB]), n);
  } else {
#pragma unroll
    for (int n = 0; n < MB; ++n) y[n] = cadd(row[n], row[n + MB]);
  }
  fft_reg<MB, false>(y);
}

// Step 2 (after the pair finished reading the column): park the bins of this
// half in natural order in the pair's row, slots 64h + m.
template <bool FPRUNE>
MQP_HD MQP_FI void big_col_park(int t, const float2 (&y)[MB], float2* S) {
  using L = LayBig<FPRUNE>;
  const int c = t >> 1, h = t & 1;
  float2* row = S + c * L::SSTR + MB * h;
#pragma unroll
  for (int m = 0; m < MB; ++m) row[m] = y[fpos<MB>(m)];
}

// Step 3: F column c (F is zero past NF along dim 1), the product conj(F) G
// for this half's bins and the 64-point inverse; p[fpos(s)] = A_h[s].
// Column 0 carries the packed real pair k2 = 0 / 64: both products return
// together as PA + i PB, built from each bin and its mirror -k (which lies in
// the same half); its F bins go through PK (2 x 64 slots) so the mirror
// lookup needs no second register copy.
template <bool FPRUNE>
MQP_HD MQP_FI void big_col_product(int t, const float2* S, const float2* SF, float2* PK, float2 (&p)[MB]) {
  using L = LayBig<FPRUNE>;
  const int c = t >> 1, h = t & 1;
  const float2* frow = SF + c * L::FSTR;
  const float2* G = S + c * L::SSTR + MB * h;
  float2 f[MB];
  if (h) {
#pragma unroll
    for (int n = 0; n < MB; ++n)
      f[n] = rotate<NB, false>((L::NF > MB) ? csub(frow[n], frow[n + MB]) : frow[n], n);
  } else {
#pragma unroll
    for (int n = 0; n < MB; ++n) f[n] = (L::NF > MB) ? cadd(frow[n], frow[n + MB]) : frow[n];
  }
  fft_reg<MB, false>(f);
  if (c != 0) {
#pragma unroll
    for (int m = 0; m < MB; ++m) p[m] = cmulc(f[fpos<MB>(m)], G[m]);
  } else {
    float2* F = PK + MB * h;
#pragma unroll
    for (int m = 0; m < MB; ++m) F[m] = f[fpos<MB>(m)];
#pragma unroll 4
    for (int m = 0; m < MB; ++m) {
      const int mm = h ? MB - 1 - m : (MB - m) & (MB - 1);
      const float2 Zk = G[m], Zn = cconj(G[mm]);
      const float2 Fk = F[m], Fn = cconj(F[mm]);
      const float2 A = cscale(cadd(Zk, Zn), 0.5f), B = cscale(cmul_mi(csub(Zk, Zn)), 0.5f);
      const float2 Af = cscale(cadd(Fk, Fn), 0.5f), Bf = cscale(cmul_mi(csub(Fk, Fn)), 0.5f);
      p[m] = cadd(cmulc(Af, A), cmul_pi(cmulc(Bf, B)));
    }
  }
  fft_reg<MB, true>(p);
}

// Step 4 (after the product): park A_h[s] in natural order in the pair's
// row, slots 64h + s (this half's G bins, already consumed).
template <bool FPRUNE>
MQP_HD MQP_FI void big_col_park_a(int t, const float2 (&p)[MB], float2* S) {
  big_col_park<FPRUNE>(t, p, S);
}

// Step 5 (after the pair parked both halves): recombine.  Lane h keeps the
// lags 64h + s < P1 in out[s]: x[s] = A0[s] + W^-s A1[s] (h = 0) and
// x[s + 64] = A0[s] - W^-s A1[s] (h = 1).
template <bool FPRUNE>
MQP_HD MQP_FI void big_col_combine(int t, int P1, const float2* S, float2 (&out)[MB]) {
  using L = LayBig<FPRUNE>;
  const int c = t >> 1, h = t & 1;
  const float2* row = S + c * L::SSTR;
  const int n = P1 - MB * h;  // lags this lane keeps
#pragma unroll
  for (int s = 0; s < MB; ++s) {
    if (s < n) {
      const float2 w = rotate<NB, true>(row[MB + s], s);
      out[s] = h ? csub(row[s], w) : cadd(row[s], w);
    }
  }
}

// Step 6 (after every lane finished with S): lag rows s1 < P1 of column c into
// T[s1][c] (T aliases S; P1 <= 127 rows of TSTR fit in the G spectra area).
template <bool FPRUNE>
MQP_HD MQP_FI void big_col_store(int t, int P1, const float2 (&out)[MB], float2* T) {
  using L = LayBig<FPRUNE>;
  const int c = t >> 1, h = t & 1;
  const int n = P1 - MB * h;
#pragma unroll
  for (int s = 0; s < MB; ++s)
    if (s < n) T[(MB * h + s) * L::TSTR + c] = out[s];
}

#if defined(__CUDACC__)
// The column phase of one block on the device: steps 1-6 with the pair and
// block barriers between them, split so that at most one 64-point array is
// live in each function.
template <bool FPRUNE>
__device__ __noinline__ void big_columns_g(int t, float2* S) {
  float2 y[MB];
  big_col_g<FPRUNE>(t, S, y);
  __syncwarp();
  big_col_park<FPRUNE>(t, y, S);
}
template <bool FPRUNE>
__device__ __noinline__ void big_columns_product(int t, float2* S, const float2* SF, float2* PK) {
  float2 p[MB];
  big_col_product<FPRUNE>(t, S, SF, PK, p);
  big_col_park_a<FPRUNE>(t, p, S);
}
template <bool FPRUNE>
__device__ __noinline__ void big_columns_combine(int t, int P1, float2* S) {
  float2 out[MB];
  big_col_combine<FPRUNE>(t, P1, S, out);
  __syncthreads();
  big_col_store<FPRUNE>(t, P1, out, S);
}
template <bool FPRUNE>
__device__ __forceinline__ void big_columns(int t, int P1, float2* S, const float2* SF, float2* PK) {
  big_columns_g<FPRUNE>(t, S);
  big_columns_product<FPRUNE>(t, S, SF, PK);
  __syncwarp();
  big_columns_combine<FPRUNE>(t, P1, S);
}
#endif

// ---- lag rows -----------------------------------------------------------------
// Lag row s1 = t < P1: complex-to-real inverse along k2 from the 65 bins
// (k2 = 0 and 64 packed in slot 0), lags s2 < P2 into the FP64 plane row.
template <bool FPRUNE>
MQP_PHASE void big_lag_row(int t, int P1, int P2, const float2* T, double* plane) {
  using L = LayBig<FPRUNE>;
  if (t >= P1) return;
  const float2* row = T + t * L::TSTR;
  float2 X[MB];
#pragma unroll
  for (int k = 0; k < MB; ++k) X[k] = row[k];
  float2 z[MB];
#pragma unroll
  for (int k = 0; k < MB; ++k) {
    float2 E, O;
    if (k == 0) {
      E = make_float2(X[0].x + X[0].y, 0.f);
      O = make_float2(X[0].x - X[0].y, 0.f);
    } else {
      const float2 A = X[k], B = cconj(X[MB - k]);
      E = cadd(A, B);
      O = rotate<NB, true>(csub(A, B), k);
    }
    z[k] = cadd(E, cmul_pi(O));
  }
  fft_reg<MB, true>(z);
  const double scale = cc_scale<NB>();
  double* prow = plane + (long long)t * P2;
#pragma unroll
  for (int n = 0; n < MB; ++n) {
    const float2 v = z[fpos<MB>(n)];
    if (2 * n < P2) prow[2 * n] = (double)v.x * scale;
    if (2 * n + 1 < P2) prow[2 * n + 1] = (double)v.y * scale;
  }
}

MQP_HD MQP_FI int piv2d_big_smem_f2(bool prune, int P1, int P2, bool masked) {
  return prune ? LayBig<true>::total_f2(P1, P2, masked) : LayBig<false>::total_f2(P1, P2, masked);
}

}  // namespace mqp
