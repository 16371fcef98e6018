// Fused 2D PIV: one warp owns one interrogation area (IA) at a time and runs
// the whole per-IA pipeline of multi_quickPIV's PIV_CPU loop body
// (src/multi_quickPIV.jl:63-89) without leaving the SM:
//
//   phase 1  lane-per-row real FFT along dim 2 (r2c of a length-N real row
//            via one N/2-point complex FFT).  The F and G windows are read
//            straight from the images with the reference's clipping and
//            border offset (src/utils/piv_ops.jl:59-127); lanes are
//            consecutive rows, so every warp load is one coalesced segment
//            of a column.  Spectra rows k2 = 0..N/2-1 go to shared memory
//            (k2 = 0 and k2 = N/2 are both real and share slot 0 as
//            (re, im) = (X[0], X[N/2])).
//   phase 2  lane-per-spectrum-row complex FFT along dim 1 of G, of F (as
//            two half transforms, F being zero past IS1), conj(F)*G, inverse
//            FFT along dim 1; only the 2*SM1+1 fully-overlapping lags stay.
//   phase 3  lane-per-lag-row complex-to-real inverse along dim 2 (one
//            N/2-point complex FFT), giving cc[s1,s2] = sum_x F(x)G(x+s)
//            (src/crosscorrelation_algorithms/fftcc.jl:101-126).
//   then     ZNCC/NSQECC normalisation from FP64 integral images
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
  const void* mask_skip; // masked NSQECC skip mask (the double-masked method), or null = mask
  int dtype;             // 0 = float32 images, 1 = float64 images (masks share it)
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
  double threshold;      // skip when max(IA) < threshold (threshold >= 0; masked: > 0)
  double mask_threshold; // masked: skip when max(mask_skip IA) < mask_threshold (> 0)
  int computeSN;
  int* status;           // device error flag (non-zero = failure), or null
  float2* huge;          // FFT length 256 (mqp_piv2d_huge.cuh): one scratch slot per resident block
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

struct IAScalars {
  double sumF2;   // sum of squares of the transformed F (ZNCC: mean removed; masked: sum(maskF^2/wi))
  double meanF;   // ZNCC
  double meanG;   // ZNCC
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
  // masked NSQECC parks its first correlation (FP32, P1 x P2) after the plane
  static MQP_HD MQP_FI int extra_f2(bool masked, int P1, int P2) { return masked ? (P1 * P2 + 1) / 2 : 0; }
  static MQP_HD MQP_FI int warp_f2(int P1, int P2, bool masked = false) {
    return G_SIZE + region2_f2(P1, P2) + extra_f2(masked, P1, P2);
  }
  // kernels that form the window sums on chip (lw_rows / lw_cols): the
  // (N/2 + 1) x N FP64 table overlays the dead G spectra and may run past
  // them, so their plane starts after the larger of the two
  static constexpr int TBL = (N / 2 + 1) * N;
  static constexpr int F_OFF_LW = G_SIZE > TBL ? G_SIZE : TBL;
  static MQP_HD MQP_FI int warp_f2_lw(int P1, int P2) { return F_OFF_LW + region2_f2(P1, P2); }
  // kernels that stage the next search window with the TMA (mqp_stage.cuh):
  // the (N + 4) x N FP32 tile lands over the dead G spectra and may run past
  // them; each warp's region starts on a 128-byte boundary
  static constexpr int TILE_F2 = ((N + 4) * N + 1) / 2;
  static constexpr int F_OFF_STG = G_SIZE > TILE_F2 ? G_SIZE : TILE_F2;
  static MQP_HD MQP_FI int warp_f2_stg(int P1, int P2) { return (F_OFF_STG + region2_f2(P1, P2) + 15) / 16 * 16; }
  static_assert(F_OFF_STG >= F_OFF_LW, "the staged layout also holds the window-sum table");
};

// ---------------------------------------------------------------------------
// phase 1: real FFT of one window row along dim 2 -> spectra X2 = 2 * DFT
// ---------------------------------------------------------------------------
// z holds the row packed as z[n] = x[2n] + i x[2n+1]; after the M-point FFT
// the r2c split gives X2[k] = (Z[k] + conj Z[M-k]) - i W^k (Z[k] - conj Z[M-k]).
// out[k * stride] receives X2[k] (k = 1..M-1) and out[0] the packed pair
// (X2[0], X2[M]).
template <int N, int NZ>
MQP_HD MQP_FI void r2c_store(float2 (&z)[N / 2], float2* out, int stride) {
  constexpr int M = N / 2;
  fft_reg<M, false, NZ>(z);
  const float2 Z0 = z[fpos<M>(0)];
  out[0] = make_float2(2.f * (Z0.x + Z0.y), 2.f * (Z0.x - Z0.y));
#pragma unroll
  for (int k = 1; k < M; ++k) {
    const float2 A = z[fpos<M>(k)];
    const float2 B = cconj(z[fpos<M>(M - k)]);
    const float2 e = cadd(A, B);
    const float2 o = cmul_mi(csub(A, B));
    out[k * stride] = cadd(e, rotate<N, false>(o, k));
  }
}

template <typename T>
MQP_HD MQP_FI T ldg_px(const void* img, long long i) {
#if defined(__CUDA_ARCH__)
  return __ldg(reinterpret_cast<const T*>(img) + i);
#else
  return reinterpret_cast<const T*>(img)[i];
#endif
}

MQP_HD MQP_FI void zero_strided(float2* base, int rows, int stride) {
  for (int k = 0; k < rows; ++k) base[k * stride] = make_float2(0.f, 0.f);
}

// One row of phase 1.  Row j of the lane's work: j == 0 is row y = lane of
// the interrogation window F (copy_inter_region!, src/utils/piv_ops.jl:99-109,
// minus its mean for ZNCC, src/utils/zncc_ops.jl:7-12), j >= 1 is row
// p = lane + 32 (j - 1) of the padded search window G: pad (p, x2) <-
// img2(g01+p, g02+x2) on the clipped data region and 0 elsewhere
// (copy_search_region!, src/utils/piv_ops.jl:115-127), minus meanG there for
// ZNCC (src/utils/zncc_ops.jl:18-25).  One rolled body serves both so the
// r2c code exists once.  F rows also accumulate the raw max (skip test,
// src/utils/piv_ops.jl:134-146) and the FP64 sum of squares of the
// transformed values (sumF2, zncc.jl:131-135, nsqecc.jl:349-353).
// Phase 1 works through the lane's rows ("jobs": NJF rows of F, then the
// N/32 rows of G) with the raw loads of the next job in flight while the
// current one is transformed.  A job's loads read one row of the window
// along dim 2; lanes are consecutive rows, so each warp load is one
// coalesced column segment.
struct RowJob {
  bool isF;
  bool live;      // the row holds data (else it is all zero)
  int row;        // window row (dim 1)
  int xlo, xhi;   // data columns [xlo, xhi) along dim 2
  long long base; // image index of (row, column 0)
};

template <int N, bool FPRUNE>
MQP_HD MQP_FI RowJob row_job(const Piv2dArgs& a, const IAGeom& g, int lane, int job) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int NJF = (Lay::NF + 31) / 32;
  RowJob j;
  j.isF = job < NJF;
  j.row = lane + 32 * (j.isF ? job : job - NJF);
  if (j.isF) {
    // row y of the interrogation window (copy_inter_region!, src/utils/piv_ops.jl:99-109)
    j.live = j.row < a.IS1;
    j.xlo = 0;
    j.xhi = a.IS2 < (FPRUNE ? N / 2 : N) ? a.IS2 : (FPRUNE ? N / 2 : N);
    j.base = (long long)(g.ir1 + j.row) + (long long)a.H * g.ir2;
  } else {
    // row p of the padded search window: data on the clipped region only
    // (copy_search_region!, src/utils/piv_ops.jl:115-127)
    j.live = j.row >= g.lo1 && j.row < g.hi1;
    j.xlo = g.lo2;
    j.xhi = g.hi2;
    j.base = (long long)(g.g01 + j.row) + (long long)a.H * g.g02;
  }
  return j;
}

// raw values of a G job's row (0 outside the data columns).  F rows are read
// by row_process itself, in the images' own precision.
template <int N, typename T>
MQP_HD MQP_FI void row_load(const Piv2dArgs& a, const RowJob& j, float (&v)[N]) {
  const T* p = reinterpret_cast<const T*>(a.img2) + j.base;
  const bool live = j.live && !j.isF;
#pragma unroll
  for (int x = 0; x < N; ++x)
    v[x] = (live && x >= j.xlo && x < j.xhi) ? (float)ldg_px<T>(p, (long long)a.H * x) : 0.f;
}

// Which inputs a phase-1 pass correlates.
enum Pass1 : int {
  PASS_PLAIN = 0,   // F (minus mean for ZNCC) with G (minus mean for ZNCC)
  PASS_MASKED = 1,  // masked NSQECC, first correlation: F*mask with G
  PASS_MASK_SQ = 2  // masked NSQECC, second correlation: mask with G^2
};

// Transform one row of phase 1 into its spectra (r2c along dim 2).
// F rows: the IA row (copy_inter_region!, src/utils/piv_ops.jl:99-109), minus
// the IA mean for ZNCC (src/utils/zncc_ops.jl:7-12), times the mask for
// masked NSQECC (copy_inter_masked!, src/utils/masked_nsqecc_ops.jl:19-25) or
// the mask itself for its second correlation; they accumulate the raw
// maxima of the skip tests (src/utils/piv_ops.jl:134-157) in the images'
// precision and the FP64 sum of squares of the transformed values (sumF2:
// zncc.jl:131-135, nsqecc.jl:349-353; masked sum(maskF^2/wi),
// mask_nsqecc.jl:141-149).  G rows come loaded in v and subtract the
// search-region mean on their data part for ZNCC (src/utils/zncc_ops.jl:18-25),
// or are squared for the masked second correlation (copy_search_squared!,
// src/utils/masked_nsqecc_ops.jl:35-42).
template <int N, bool FPRUNE, typename T, bool ZNCC>
MQP_HD MQP_FI void row_process(const Piv2dArgs& a, const IAScalars& sc, int PASS, const RowJob& j,
                               const float (&v)[N], float2* GH, float2* FH, double& vmax, double& mmax,
                               double& sumsq) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2* out = j.isF ? FH + j.row : GH + j.row;
  const int stride = j.isF ? Lay::FSTR : Lay::GSTR;
  if (!j.live) {
    zero_strided(out, M, stride);
    return;
  }
  float2 z[M];
  if (j.isF) {
    constexpr int FLIM = FPRUNE ? N / 2 : N;  // columns an IA row can occupy
    const T* p = reinterpret_cast<const T*>(a.img1) + j.base;
    const T* q = PASS != PASS_PLAIN ? reinterpret_cast<const T*>(a.mask) + j.base : p;
    const T* qs = PASS == PASS_MASKED ? reinterpret_cast<const T*>(a.mask_skip ? a.mask_skip : a.mask) + j.base : p;
    float w[N];
#pragma unroll
    for (int x = 0; x < N; ++x) {
      w[x] = 0.f;
      if (x < FLIM && x < j.xhi) {
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
#pragma unroll
    for (int n = 0; n < M; ++n) z[n] = make_float2(w[2 * n], w[2 * n + 1]);
  } else if (ZNCC) {
    const float mg = (float)sc.meanG;
#pragma unroll
    for (int n = 0; n < M; ++n) {
      const int x0 = 2 * n, x1 = 2 * n + 1;
      z[n] = make_float2((x0 >= j.xlo && x0 < j.xhi) ? v[x0] - mg : 0.f,
                         (x1 >= j.xlo && x1 < j.xhi) ? v[x1] - mg : 0.f);
    }
  } else if (PASS == PASS_MASK_SQ) {
#pragma unroll
    for (int n = 0; n < M; ++n) z[n] = make_float2(v[2 * n] * v[2 * n], v[2 * n + 1] * v[2 * n + 1]);
  } else {
#pragma unroll
    for (int n = 0; n < M; ++n) z[n] = make_float2(v[2 * n], v[2 * n + 1]);
  }
  r2c_store<N, M>(z, out, stride);
}

// ---------------------------------------------------------------------------
// after phase 1: first DIF stage along dim 1 for the G spectra
// ---------------------------------------------------------------------------
// Splits every G spectrum row u (length N along dim 1) into its even-bin
// half Ge[n] = g[n] + g[n+N/2] (slots 0..N/2) and odd-bin half
// Go[n] = (g[n] - g[n+N/2]) W_N^n (slots N/2..N), in place, so phase 2
// works on half-length transforms.  Lane handles window rows n = lane + 32j.
// tw: (cos, sin)(2 pi j / N).
template <int N, bool FPRUNE>
MQP_HD MQP_FI void split_G_pair(float2* GH, const float2* tw, int n) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  const float2 w = tw[n];
  for (int u = 0; u < M; ++u) {
    float2* r = GH + u * Lay::GSTR;
    const float2 a = r[n], b = r[n + M];
    const float2 d = csub(a, b);
    r[n] = cadd(a, b);
    r[n + M] = make_float2(d.x * w.x + d.y * w.y, d.y * w.x - d.x * w.y);  // d * conj(w)
  }
}

// ---------------------------------------------------------------------------
// phase 2: along dim 1 for one spectrum row u (u = 0 is the packed real pair)
// ---------------------------------------------------------------------------
// conj(F)*G over the N/2 bins k = 2m + h of one half (natural order m).  Row 0
// carries two real rows A + iB (k2 = 0 and k2 = N/2): their spectra are
// A^ = (Z[k] + conj Z[-k]) / 2 and B^ = -i (Z[k] - conj Z[-k]) / 2, and the two
// Hermitian products return together as PA + i PB; the mirror -k of a bin
// lies in the same half (m' = -m mod N/2 for even bins, N/2-1-m for odd).
template <int M>
MQP_HD MQP_FI void half_product(bool packed, int h, const float2 (&x)[M], const float2 (&f)[M], float2 (&p)[M]) {
  if (!packed) {
#pragma unroll
    for (int m = 0; m < M; ++m) p[m] = cmulc(f[fpos<M>(m)], x[fpos<M>(m)]);
    return;
  }
#pragma unroll
  for (int m = 0; m < M; ++m) {
    // the mirror of bin 2m+h is 2m'+h with m' = (h ? M-1-m : (M-m) % M)
    const int me = (M - m) & (M - 1), mo = M - 1 - m;
    const int mm = h ? mo : me;
    if (mm < m) continue;  // written together with its mirror
    const float2 Zk = x[fpos<M>(m)], Zn = cconj(h ? x[fpos<M>(mo)] : x[fpos<M>(me)]);
    const float2 Fk = f[fpos<M>(m)], Fn = cconj(h ? f[fpos<M>(mo)] : f[fpos<M>(me)]);
    const float2 A = cscale(cadd(Zk, Zn), 0.5f), B = cscale(cmul_mi(csub(Zk, Zn)), 0.5f);
    const float2 Af = cscale(cadd(Fk, Fn), 0.5f), Bf = cscale(cmul_mi(csub(Fk, Fn)), 0.5f);
    const float2 PA = cmulc(Af, A), PB = cmulc(Bf, B);
    const float2 q = cadd(PA, cmul_pi(PB));
    const float2 qm = cadd(cconj(PA), cmul_pi(cconj(PB)));
    if (h) {
      p[m] = q;
      if (mo != m) p[mo] = qm;
    } else {
      p[m] = q;
      if (me != m) p[me] = qm;
    }
  }
}

// One spectrum row: two half passes (even bins, then odd bins) of forward
// N/2-point transforms of G (already split by split_G_pair) and F, the
// product, and an N/2-point inverse; the halves recombine as
//   R[s] = A0[s] + W_N^-s A1[s],  R[s + N/2] = A0[s] - W_N^-s A1[s].
// The even pass parks A0 in the consumed Ge slots.  Lags s < P1 stay in
// slots 0..P1 of the row.
template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase2_row(int u, int P1, float2* GH, const float2* FH, const float2* tw) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2* Grow = GH + u * Lay::GSTR;
  const float2* Frow = FH + u * Lay::FSTR;
  const bool packed = (u == 0);
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {
    float2 x[M];
#pragma unroll
    for (int n = 0; n < M; ++n) x[n] = Grow[h * M + n];
    fft_reg<M, false>(x);
    float2 f[M];
#pragma unroll
    for (int n = 0; n < M; ++n) {
      float2 v = Frow[n];
      if (!FPRUNE) {
        const float2 w = Frow[n + M];
        v = h ? csub(v, w) : cadd(v, w);
      }
      f[n] = v;
    }
    if (h) {
#pragma unroll
      for (int n = 1; n < M; ++n) f[n] = rotate<N, false>(f[n], n);
    }
    fft_reg<M, false>(f);
    float2 p[M];
    half_product<M>(packed, h, x, f, p);
    fft_reg<M, true>(p);
    if (h == 0) {
#pragma unroll
      for (int n = 0; n < M; ++n) Grow[n] = p[fpos<M>(n)];
    } else {
#pragma unroll
      for (int n = 0; n < M; ++n) {
        const float2 a0 = Grow[n];
        const float2 t = rotate<N, true>(p[fpos<M>(n)], n);
        if (n < P1) Grow[n] = cadd(a0, t);
        if (n + M < P1) Grow[n + M] = csub(a0, t);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// phase 3: complex-to-real along dim 2 for lag row s1 -> cc[s2], s2 < N
// ---------------------------------------------------------------------------
template <int N, bool FPRUNE>
MQP_HD MQP_FI void phase3_row(int s1, const float2* GH, float (&cc)[N]) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2 X[M];
#pragma unroll
  for (int k = 0; k < M; ++k) X[k] = GH[k * Lay::GSTR + s1];
  const float X0 = X[0].x, XM = X[0].y;  // the packed real bins X[0], X[N/2]
  float2 x[M];
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

// ---------------------------------------------------------------------------
// phases 2 and 3 through one forward FFT body
// ---------------------------------------------------------------------------
// Every transform of phases 2 and 3 is an N/2-point complex FFT; running them
// as the stages of one rolled loop around a single fft_reg call keeps one
// copy of the transform code in the kernel (the fully unrolled transforms are
// most of the instruction footprint).  Inverses use
// IFFT(x) = conj(FFT(conj(x))), the conjugations folded into the
// neighbouring arithmetic.
//
// Stages of one spectrum row (phase 2), h = 0 (even bins) then h = 1:
//   G : t <- Ge/Go half of the row            -> FFT -> row half <- G^_h
//   F : t <- F row (folded / twiddled for h)  -> FFT -> t <- conj(conj(F^_h) G^_h)
//   I : (t holds the conjugated product)      -> FFT -> A_h = conj(t): park (h=0)
//                                                     or recombine (h=1)
// and of one lag row (phase 3):
//   C : t <- conj(E + iO) of the c2r split    -> FFT -> cc = conj(t)
enum Stage2 : int { ST_G = 0, ST_F = 1, ST_I = 2 };

template <int N, bool FPRUNE>
MQP_HD MQP_FI void stage_pre(int st, int h, const float2* Grow, const float2* Frow, float2 (&t)[N / 2]) {
  constexpr int M = N / 2;
  if (st == ST_G) {
#pragma unroll
    for (int n = 0; n < M; ++n) t[n] = Grow[h * M + n];
  } else if (st == ST_F) {
#pragma unroll
    for (int n = 0; n < M; ++n) {
      float2 v = Frow[n];
      if (!FPRUNE) {
        const float2 w = Frow[n + M];
        v = h ? csub(v, w) : cadd(v, w);
      }
      t[n] = v;
    }
    if (h) {
#pragma unroll
      for (int n = 1; n < M; ++n) t[n] = rotate<N, false>(t[n], n);
    }
  }
}

// conj of the product conj(F^)G^ over one half (natural order m), from the
// transformed F half in t (fpos slots) and the transformed G half in x
// (natural order), computed in place in x and then moved to t (keeping two
// half spectra live, not three); see half_product for the packed row 0.
template <int M>
MQP_HD MQP_FI void stage_product(bool packed, int h, float2 (&x)[M], float2 (&t)[M]) {
  if (!packed) {
#pragma unroll
    for (int m = 0; m < M; ++m) x[m] = cconj(cmulc(t[fpos<M>(m)], x[m]));
  } else {
#pragma unroll
    for (int m = 0; m < M; ++m) {
      // the mirror of bin 2m+h is 2m'+h with m' = (M-m) % M (h = 0) or M-1-m
      // (h = 1); h is a runtime value, so both candidates stay compile-time
      // register indices and a select picks one
      const int me = (M - m) & (M - 1), mo = M - 1 - m;
      if (me < m && mo < m) continue;
      const bool lead = h ? (mo >= m) : (me >= m);  // this m writes the pair
      const float2 Zk = x[m], Fk = t[fpos<M>(m)];
      const float2 Zn = cconj(h ? x[mo] : x[me]);
      const float2 Fn = cconj(h ? t[fpos<M>(mo)] : t[fpos<M>(me)]);
      const float2 A = cscale(cadd(Zk, Zn), 0.5f), B = cscale(cmul_mi(csub(Zk, Zn)), 0.5f);
      const float2 Af = cscale(cadd(Fk, Fn), 0.5f), Bf = cscale(cmul_mi(csub(Fk, Fn)), 0.5f);
      const float2 PA = cmulc(Af, A), PB = cmulc(Bf, B);
      const float2 qk = cconj(cadd(PA, cmul_pi(PB)));
      const float2 qn = cconj(cadd(cconj(PA), cmul_pi(cconj(PB))));
      if (lead) {
        x[m] = qk;
        if (h) {
          if (mo != m) x[mo] = qn;
        } else {
          if (me != m) x[me] = qn;
        }
      }
    }
  }
#pragma unroll
  for (int m = 0; m < M; ++m) t[m] = x[m];
}

template <int N, bool FPRUNE>
MQP_HD MQP_FI void stage_post(int st, int h, bool packed, int P1, float2* Grow, float2 (&t)[N / 2]) {
  constexpr int M = N / 2;
  if (st == ST_G) {
#pragma unroll
    for (int n = 0; n < M; ++n) Grow[h * M + n] = t[fpos<M>(n)];
  } else if (st == ST_F) {
    float2 x[M];
#pragma unroll
    for (int n = 0; n < M; ++n) x[n] = Grow[h * M + n];
    stage_product<M>(packed, h, x, t);
  } else {
    if (h == 0) {
#pragma unroll
      for (int n = 0; n < M; ++n) Grow[n] = cconj(t[fpos<M>(n)]);
    } else {
#pragma unroll
      for (int n = 0; n < M; ++n) {
        const float2 a0 = Grow[n];
        const float2 r = rotate<N, true>(cconj(t[fpos<M>(n)]), n);
        if (n < P1) Grow[n] = cadd(a0, r);
        if (n + M < P1) Grow[n + M] = csub(a0, r);
      }
    }
  }
}

// phase 3 input: the c2r split of lag column s1 of the spectra rows,
// conjugated for the inverse through the forward transform
template <int N, bool FPRUNE>
MQP_HD MQP_FI void c2r_pre(int s1, const float2* GH, float2 (&t)[N / 2]) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  float2 X[M];
#pragma unroll
  for (int k = 0; k < M; ++k) X[k] = GH[k * Lay::GSTR + s1];
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
    t[k] = cconj(cadd(E, cmul_pi(O)));
  }
}

// Lag row s1 >= 32 (only when 2*SM1+1 > 32) computed by the whole warp: lane
// l evaluates lags s2 = l, l+32, ... of the Hermitian inverse
//   x[s2] = X[0] + (-1)^s2 X[N/2] + 2 sum_{k=1}^{N/2-1} Re(X[k] e^{+2 pi i k s2 / N})
// directly (one row of phase 3 costs a full transform per lane otherwise).
// tw: (cos, sin)(2 pi j / N) for j < N, in shared memory.
template <int N, bool FPRUNE>
MQP_HD MQP_FI float tail_row_value(const float2* GH, const float2* tw, int s1, int s2) {
  using Lay = Layout2d<N, FPRUNE>;
  constexpr int M = N / 2;
  const float2 X0 = GH[s1];
  float acc = 0.f;
  int t = 0;
#pragma unroll 4
  for (int k = 1; k < M; ++k) {
    t = (t + s2) & (N - 1);
    const float2 X = GH[k * Lay::GSTR + s1];
    const float2 w = tw[t];
    acc += X.x * w.x - X.y * w.y;
  }
  return X0.x + ((s2 & 1) ? -X0.y : X0.y) + 2.f * acc;
}

// cc scale: r2c (x2 per transform, F and G) and the two unnormalised inverses
template <int N>
MQP_HD MQP_FI double cc_scale() { return 1.0 / (4.0 * (double)N * (double)N); }

// ---------------------------------------------------------------------------
// per-IA scalars and the similarity of one lag column
// ---------------------------------------------------------------------------

// Image row (or column) range covered by the interrogation-sized window at
// lag s, clipped to the data of the padded search window.
MQP_HD MQP_FI void lag_window(int s, int IS, int g0, int lo, int hi, int& r0, int& r1) {
  const int a = s > lo ? s : lo;
  const int b = (s + IS) < hi ? (s + IS) : hi;
  r0 = g0 + a;
  r1 = g0 + (b > a ? b : a);
}

// NaN-propagating max / min (Julia's maximum / minimum)
MQP_HD MQP_FI double nmax(double m, double v) { return (v > m || v != v) ? v : m; }
MQP_HD MQP_FI double nmin(double m, double v) { return (v < m || v != v) ? v : m; }

// lane-local part of first_fullovp_peak (src/utils/common_ops.jl:98-124).
// The reference keeps the first maximum > 0 of a column-major scan; every
// lane keeps the (largest value, lowest column-major index) of the elements
// it owns, starting from (0, none), and merging lanes by the same rule gives
// the same element whatever the split.
MQP_HD MQP_FI void peak_take(double v, int idx, double& best, int& bidx) {
  if (v > best || (v == best && idx < bidx)) {
    best = v;
    bidx = idx;
  }
}

// Per-lane accumulators of the peak search and of compute_SN
// (src/utils/piv_ops.jl:336-367), and the 0-based inclusive lag ranges:
// peak [lo, hi] = [TLF_off, 2SM - BRB_off], SN rows/cols up to 2SM-1-BRB_off.
struct PeakAcc {
  double best;
  int bidx;
  double smax, ssum;
};
struct LagRanges {
  int lo1, hi1, lo2, hi2, shi1, shi2;
};

MQP_HD MQP_FI void acc_take(PeakAcc& acc, const LagRanges& R, int s1, int s2, int P1, double v) {
  if (s1 >= R.lo1 && s2 >= R.lo2) {
    if (s1 <= R.hi1 && s2 <= R.hi2) peak_take(v, s1 + P1 * s2, acc.best, acc.bidx);
    if (s1 <= R.shi1 && s2 <= R.shi2) {
      acc.smax = nmax(acc.smax, v);
      acc.ssum += v;
    }
  }
}

// Similarity from the raw correlation c and the window sums:
//   FFTCC  c                                           (fftcc.jl:123)
//   ZNCC   c / (sqrt(sum_win G'^2) sqrt(sumF2))        (zncc_ops.jl:29-50)
//   NSQECC den / (den + num), num = sumF2 + sum_win G^2 - 2c,
//          den = sqrt(sum_win G^2) sqrt(sumF2)          (nsqecc_ops.jl:1-25)
// The numerator is formed in FP64 (it cancels near a match); the square
// roots and the final quotient are FP32, whose ~1e-7 relative error is below
// the FP32 correlation's own.
template <int ALG>
MQP_HD MQP_FI double similarity_value(const IAScalars& sc, float sqF, double c, double S2, double S1, double n) {
  if (ALG == ALG_FFTCC) return c;
  if (ALG == ALG_MASK_NSQECC) {
    // fftcc2masknsqecc! (src/utils/masked_nsqecc_ops.jl:123-142): c = (F*mask)*G,
    // S2 = mask*G^2, both correlations
    const double num = (sc.sumF2 - 2.0 * c) + S2;
    const float den = sqrtf(fabsf((float)S2)) * sqF;
    return (double)(den / (float)(num + (double)den));
  }
  if (ALG == ALG_NSQECC) {
    const double num = (sc.sumF2 - 2.0 * c) + S2;
    const float den = sqrtf((float)S2) * sqF;
    return (double)(den / (float)(num + (double)den));
  }
  double SG = S2 - 2.0 * sc.meanG * S1 + n * sc.meanG * sc.meanG;
  SG = SG > 0.0 ? SG : 0.0;
  return (double)((float)c / (sqrtf((float)SG) * sqF));
}

// ---------------------------------------------------------------------------
// window sums on chip (interrogation window = half the FFT length)
// ---------------------------------------------------------------------------
// The reference forms sum_win(pad_G^2) for every fully-overlapping lag from
// an integral array of the IA's squared padded search window
// (integralArraySQ! and add_numerator_nsqecc, src/utils/common_ops.jl:142-245;
// pad_G minus the search-region mean for ZNCC, src/utils/zncc_ops.jl:18-25).
// When the lag window (the interrogation window) is H x H with H = N/2, the
// warp kernel forms the same sums in FP64 from the window's pixels, in two
// passes over a table in its own shared memory (the G spectra are dead by
// then), instead of four lookups per lag in whole-image integral images.  A
// window [s, s + H) of a length-N line splits at H into the suffix
// [s, H) of the first half and the prefix [H, H + s) of the second, so each
// pass is two independent running sums of non-negative terms (no
// cancellation, half the dependency chain of one sliding sum):
//   lw_rows  lane = pad row p1 (p1 = lane + 32 h): R[p1][s2] over columns;
//   lw_cols  lane = lag column s2: S[s1][s2] over rows of R, written over R;
//            a 33rd column (P2 = H + 1 = 33) by warp scans, lanes over rows.
// Element (p1, s2) sits at s2 * N + (p1 ^ (s2 & 31)): lanes over p1, over s2
// and over s1 (the finish) all hit distinct bank pairs.
MQP_HD MQP_FI int lw_at(int N, int p1, int s2) { return s2 * N + (p1 ^ (s2 & 31)); }

template <int N, typename T, bool ZNCC>
MQP_HD MQP_FI void lw_rows(const Piv2dArgs& a, const IAGeom& g, double meanG, int lane, int P2, double* lw) {
  constexpr int H = N / 2;
  // one row per batch of loads (two rows of 64 live values spill)
  constexpr int RB = 1;
#pragma unroll 1
  for (int h0 = 0; h0 < N / 32; h0 += RB) {
    T v[RB][N];
    bool live[RB];
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      const int p1 = lane + 32 * (h0 + b);
      live[b] = p1 >= g.lo1 && p1 < g.hi1;
      const T* src = reinterpret_cast<const T*>(a.img2) + ((long long)(g.g01 + p1) + (long long)a.H * g.g02);
#pragma unroll
      for (int x = 0; x < N; ++x)
        v[b][x] = (live[b] && x >= g.lo2 && x < g.hi2) ? ldg_px<T>(src, (long long)a.H * x) : T(0);
    }
    mqp_no_hoist();  // every load of the batch is issued before the first use
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      const int p1 = lane + 32 * (h0 + b);
      // pad_G^2 (0 outside the clipped search region)
      auto q = [&](int x) {
        const double d = ZNCC ? (double)v[b][x] - meanG : (double)v[b][x];
        return (live[b] && x >= g.lo2 && x < g.hi2) ? d * d : 0.0;
      };
      double A[H + 1];  // A[s] = sum of q over [s, H)
      A[H] = 0.0;
#pragma unroll
      for (int x = H - 1; x >= 0; --x) A[x] = A[x + 1] + q(x);
      double B = 0.0;  // sum of q over [H, H + s2)
#pragma unroll
      for (int s2 = 0; s2 <= H; ++s2) {
        if (s2 < P2) lw[lw_at(N, p1, s2)] = A[s2] + B;
        if (s2 < H) B = B + q(H + s2);
      }
    }
  }
}

template <int N>
MQP_HD MQP_FI void lw_cols(int lane, int P1, int P2, double* lw) {
  constexpr int H = N / 2;
  const int s2 = lane;
  if (s2 < P2) {
    const int sw = s2 & 31;
    double* col = lw + s2 * N;
    double r[N];
#pragma unroll
    for (int p = 0; p < N; ++p) r[p] = col[p ^ sw];
    double A[H + 1];  // A[s1] = sum of r over [s1, H)
    A[H] = 0.0;
#pragma unroll
    for (int p = H - 1; p >= 0; --p) A[p] = A[p + 1] + r[p];
    double B = 0.0;
#pragma unroll
    for (int s1 = 0; s1 <= H; ++s1) {
      if (s1 < P1) col[s1 ^ sw] = A[s1] + B;
      if (s1 < H) B = B + r[H + s1];
    }
  }
}

// Column 32 of lw_cols (N = 64, P2 = 33): lanes over rows, r0 = R[lane],
// r1 = R[32 + lane]; S[s1] = (rows [s1, 32)) + (rows [32, 32 + s1)) by two
// log-step scans.  The scan steps, shared with the host emulation:
MQP_HD MQP_FI void lw_scan_step(double& suf, double& pre, double suf_from_above, double pre_from_below, int lane,
                                int off) {
  if (lane + off < 32) suf += suf_from_above;
  if (lane >= off) pre += pre_from_below;
}
template <int N>
MQP_HD MQP_FI void lw_col32(int lane, int P1, int P2, double* lw) {
#if defined(__CUDA_ARCH__)
  if (N != 64 || P2 <= 32) return;
  double* col = lw + 32 * N;  // (p1 ^ (32 & 31)) = p1: no swizzle in this column
  const double r0 = col[lane], r1 = col[lane + 32];
  __syncwarp();
  double suf = r0, pre = r1;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double a = __shfl_down_sync(0xffffffffu, suf, off);
    const double b = __shfl_up_sync(0xffffffffu, pre, off);
    lw_scan_step(suf, pre, a, b, lane, off);
  }
  double ex = __shfl_up_sync(0xffffffffu, pre, 1);  // rows [32, 32 + lane)
  if (lane == 0) ex = 0.0;
  if (lane < P1) col[lane] = suf + ex;
  if (lane == 31 && P1 > 32) col[32] = pre;  // S[32]: rows [32, 64)
#else
  (void)lane, (void)P1, (void)P2, (void)lw;  // the host emulation runs the scan lane by lane
#endif
}

// Finishes lag row s1: prow[s2] (s2 < P2) holds the raw correlation on entry
// and the similarity on exit; the row's elements enter the peak / SN
// accumulators.  Window sums come from the FP64 integral images of img2 and
// img2^2; lanes are consecutive lag rows, so each lookup is a coalesced
// column segment, and four lags' lookups are issued before any is used.
// LWN = N: the window sums come from the on-chip table lw (lw_rows /
// lw_cols; for ZNCC already about the search mean), not from the images.
template <int ALG, int LWN = 0>
MQP_HD MQP_FI void finish_row(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, int s1, int P1,
                              int P2, double* prow, const LagRanges& R, PeakAcc& acc, const float* c1row = nullptr,
                              const double* lw = nullptr) {
  const float sqF = sqrtf((float)sc.sumF2);
  if (ALG == ALG_MASK_NSQECC) {
    // prow holds mask*G^2, c1row the parked (F*mask)*G
    for (int s2 = 0; s2 < P2; ++s2) {
      const double v = similarity_value<ALG>(sc, sqF, (double)c1row[s2], prow[s2], 0.0, 0.0);
      prow[s2] = v;
      acc_take(acc, R, s1, s2, P1, v);
    }
    return;
  }
  int r0 = 0, r1 = 0;
  if (ALG != ALG_FFTCC) lag_window(s1, a.IS1, g.g01, g.lo1, g.hi1, r0, r1);
  const long long ld = (long long)a.H + 1;
  for (int b = 0; b < P2; b += 4) {
    double S2v[4], S1v[4], nv[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      S2v[t] = 0.0;
      S1v[t] = 0.0;
      nv[t] = 0.0;
      const int s2 = b + t;
      if (LWN && s2 < P2) {
        S2v[t] = lw[lw_at(LWN, s1, s2)];
      } else if (ALG != ALG_FFTCC && s2 < P2) {
        int c0, c1;
        lag_window(s2, a.IS2, g.g02, g.lo2, g.hi2, c0, c1);
        if (r1 > r0 && c1 > c0) {
          const double* A0 = a.IIg2 + ld * c0;
          const double* A1 = a.IIg2 + ld * c1;
          S2v[t] = (A1[r1] - A1[r0]) - (A0[r1] - A0[r0]);
          if (ALG == ALG_ZNCC) {
            const double* B0 = a.IIg + ld * c0;
            const double* B1 = a.IIg + ld * c1;
            S1v[t] = (B1[r1] - B1[r0]) - (B0[r1] - B0[r0]);
            nv[t] = (double)(r1 - r0) * (double)(c1 - c0);
          }
        }
      }
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int s2 = b + t;
      if (s2 < P2) {
        const double v = similarity_value<ALG>(sc, sqF, prow[s2], S2v[t], S1v[t], nv[t]);
        prow[s2] = v;
        acc_take(acc, R, s1, s2, P1, v);
      }
    }
  }
}

// One element (s1, s2) of a tail lag row (the whole warp shares such rows,
// lanes over s2); c is the raw correlation.
template <int ALG, int LWN = 0>
MQP_HD MQP_FI double finish_one(const Piv2dArgs& a, const IAGeom& g, const IAScalars& sc, int s1, int s2,
                                double c, double cmask = 0.0, const double* lw = nullptr) {
  if (ALG == ALG_FFTCC) return c;
  if (LWN) return similarity_value<ALG>(sc, sqrtf((float)sc.sumF2), c, lw[lw_at(LWN, s1, s2)], 0.0, 0.0);
  // masked: c = mask*G^2, cmask = (F*mask)*G
  if (ALG == ALG_MASK_NSQECC) return similarity_value<ALG>(sc, sqrtf((float)sc.sumF2), cmask, c, 0.0, 0.0);
  int r0, r1, c0, c1;
  lag_window(s1, a.IS1, g.g01, g.lo1, g.hi1, r0, r1);
  lag_window(s2, a.IS2, g.g02, g.lo2, g.hi2, c0, c1);
  const double S2 = box_sum(a.IIg2, a.H, r0, r1, c0, c1);
  const double S1 = ALG == ALG_ZNCC ? box_sum(a.IIg, a.H, r0, r1, c0, c1) : 0.0;
  const double n = (double)(r1 - r0) * (double)(c1 - c0);
  return similarity_value<ALG>(sc, sqrtf((float)sc.sumF2), c, S2, S1, n);
}

// gaussian_refinement + gaussian_2D (src/utils/piv_ops.jl:282-319) around the
// 0-based peak (p1, p2) of value mx; the plane is row-contiguous (element
// (s1, s2) at s1*P2 + s2).  refine2d_values gives the five values whose logs
// the fit takes (peak, up, down, left, right) and the 3x3 minimum, or false
// when the peak touches the search range edge (position unchanged);
// refine2d_from_logs the refined 0-based position from their logs.
MQP_HD MQP_FI bool refine2d_values(const double* plane, int P2, int SM1, int SM2, const IAGeom& g, int p1, int p2,
                                   double mx, double (&v)[5], double& mn) {
  // reference test in 1-based indices: peak > 1 + TLF_off and peak < 1 + 2SM - BRB_off
  const bool inside = (p1 + 1 > 1 + g.tlf1) && (p2 + 1 > 1 + g.tlf2) &&
                      (p1 + 1 < 1 + 2 * SM1 - g.brb1) && (p2 + 1 < 1 + 2 * SM2 - g.brb2);
  if (!inside) return false;
  auto at = [&](int i, int j) { return plane[i * P2 + j]; };
  mn = at(p1 - 1, p2 - 1);
  for (int j = -1; j <= 1; ++j)
    for (int i = -1; i <= 1; ++i) mn = nmin(mn, at(p1 + i, p2 + j));
  v[0] = mx;
  v[1] = at(p1 - 1, p2);
  v[2] = at(p1 + 1, p2);
  v[3] = at(p1, p2 - 1);
  v[4] = at(p1, p2 + 1);
  return true;
}

MQP_HD MQP_FI void refine2d_from_logs(int p1, int p2, const double (&l)[5], double& r1, double& r2) {
  r1 = p1 + (l[1] - l[2]) / (2.0 * l[1] - 4.0 * l[0] + 2.0 * l[2]);
  r2 = p2 + (l[3] - l[4]) / (2.0 * l[3] - 4.0 * l[0] + 2.0 * l[4]);
}

MQP_HD MQP_FI void refine2d(const double* plane, int P2, int SM1, int SM2, const IAGeom& g, int p1, int p2,
                            double mx, double& r1, double& r2) {
  r1 = p1;
  r2 = p2;
  double v[5], mn;
  if (!refine2d_values(plane, P2, SM1, SM2, g, p1, p2, mx, v, mn)) return;
  double l[5];
  for (int k = 0; k < 5; ++k) l[k] = log(1.0 + v[k] - mn);
  refine2d_from_logs(p1, p2, l, r1, r2);
}

#if defined(__CUDACC__)
// refine2d for a whole warp (every lane calls it with the same peak): lanes
// 0-4 take one log each instead of lane 0 taking all five in a row; every
// lane returns the same position, equal to refine2d's.
__device__ __forceinline__ void refine2d_warp(const double* plane, int P2, int SM1, int SM2, const IAGeom& g, int p1,
                                              int p2, double mx, int lane, double& r1, double& r2) {
  r1 = p1;
  r2 = p2;
  double v[5], mn;
  if (!refine2d_values(plane, P2, SM1, SM2, g, p1, p2, mx, v, mn)) return;
  double x = v[0];
#pragma unroll
  for (int k = 1; k < 5; ++k)
    if (lane == k) x = v[k];
  const double mine = lane < 5 ? log(1.0 + x - mn) : 0.0;
  double l[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) l[k] = __shfl_sync(0xffffffffu, mine, k);
  refine2d_from_logs(p1, p2, l, r1, r2);
}
#endif

// merge two (value, first index) candidates: larger value, then smaller index
MQP_HD MQP_FI void peak_merge(double& best, int& bidx, double ob, int oi) {
  if (oi < 0) return;
  if (bidx < 0 || ob > best || (ob == best && oi < bidx)) {
    best = ob;
    bidx = oi;
  }
}

}  // namespace mqp
