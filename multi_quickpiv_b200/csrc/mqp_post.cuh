// Vector-field post-processing on the device: the local-window operations of
// multi_quickPIV's src/postprocessing/postprocessing.jl, one thread per
// vector.  A vector field is Float64 (ncomp, d1, ..., dnd) column-major,
// exactly the VF array PIV returns (component fastest); windows are clamped
// at the field border (localOp, postprocessing.jl:62-72: the window shrinks).
//
// Every per-vector function here is __host__ __device__ so the CPU tests run
// the same code through a host loop.
#pragma once

#include "mqp_fft.cuh"

#include <math.h>
#include <stdint.h>

namespace mqp {

enum PostOp : int {
  POST_MAGNITUDES = 0,
  POST_AVERAGE = 1,
  POST_SIMILARITY_AVERAGING = 2,
  POST_COLLECTIVENESS = 3,
  POST_TH_MASK = 4,
  POST_STD_MASK = 5,
  POST_REPLACE = 6,
  POST_LOCAL_MAGNITUDE = 7,
  POST_MATLAB_DIVERGENCE = 8,
  POST_DIVERGENCE = 9
};

enum ReplaceKind : int { REPLACE_ZERO = 0, REPLACE_MEDIAN = 1, REPLACE_MEAN = 2 };
enum DivideBy : int { DIVIDE_NONE = 0, DIVIDE_N = 1, DIVIDE_MAGS = 2 };

constexpr int POST_MAXD = 4;

struct PostArgs {
  int op;
  int ncomp;               // vector components (1 for a scalar map)
  int nd;                  // field dimensions, 1..4
  int dims[POST_MAXD];     // field size (unused dims 1)
  int radius[POST_MAXD];   // window radius per dim (unused dims 0)
  long long n;             // prod(dims)
  const double* VF;        // (ncomp, dims...) or the scalar map (dims...)
  const uint8_t* mask;     // POST_REPLACE: vectors to replace
  double* out;             // Float64 output (ncomp, dims...) or (dims...)
  float* outf;             // Float32 output (dims...)
  uint8_t* mask_out;       // mask output (dims...)
  double p0, p1, p2;       // op parameters (see each op)
  int i0, i1, i2;          // op flags (see each op)
};

MQP_HD MQP_FI void post_coords(const PostArgs& a, long long i, int (&c)[POST_MAXD]) {
#pragma unroll
  for (int d = 0; d < POST_MAXD; ++d) {
    c[d] = (int)(i % a.dims[d]);
    i /= a.dims[d];
  }
}

// clamped window [lo, hi] (inclusive) around c, as localOp's
// max(1, c - r) : min(size, c + r)
MQP_HD MQP_FI void post_window(const PostArgs& a, const int (&c)[POST_MAXD], int (&lo)[POST_MAXD],
                               int (&hi)[POST_MAXD]) {
#pragma unroll
  for (int d = 0; d < POST_MAXD; ++d) {
    lo[d] = c[d] - a.radius[d] > 0 ? c[d] - a.radius[d] : 0;
    hi[d] = c[d] + a.radius[d] < a.dims[d] - 1 ? c[d] + a.radius[d] : a.dims[d] - 1;
  }
}

MQP_HD MQP_FI long long post_lin(const PostArgs& a, int i0, int i1, int i2, int i3) {
  return (long long)i0 + (long long)a.dims[0] * ((long long)i1 + (long long)a.dims[1] * ((long long)i2 +
                                                                                       (long long)a.dims[2] * i3));
}

// Products and sums rounded separately, as Julia's broadcast-then-sum
// (`sum(x .^ 2)`, `sum(a .* b)`) rounds them: no fused multiply-add.
MQP_HD MQP_FI double pmul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
MQP_HD MQP_FI double padd(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}

// magnitudes (postprocessing.jl:184-192): sqrt(sum(VF[:, i].^2))
MQP_HD MQP_FI double post_mag(const double* VF, int ncomp, long long i) {
  double s = 0.0;
  for (int c = 0; c < ncomp; ++c) {
    const double v = VF[(long long)ncomp * i + c];
    s = padd(s, pmul(v, v));
  }
  return sqrt(s);
}

MQP_HD MQP_FI long long post_count(const int (&lo)[POST_MAXD], const int (&hi)[POST_MAXD]) {
  long long n = 1;
#pragma unroll
  for (int d = 0; d < POST_MAXD; ++d) n *= (long long)(hi[d] - lo[d] + 1);
  return n;
}

// Statistics.median of component comp over the window: the middle element,
// or the mean of the two middle elements for an even count; NaN if any value
// is NaN.  Selection by counting (no storage): value x is the k-th smallest
// iff #{< x} <= k < #{<= x}.
MQP_HD MQP_FI double post_median(const PostArgs& a, const int (&lo)[POST_MAXD], const int (&hi)[POST_MAXD],
                                 int comp) {
  const long long n = post_count(lo, hi);
  const long long k1 = (n - 1) / 2, k2 = n / 2;
  double v1 = 0.0, v2 = 0.0;
  bool f1 = false, f2 = false;
  for (int w3 = lo[3]; w3 <= hi[3]; ++w3)
    for (int w2 = lo[2]; w2 <= hi[2]; ++w2)
      for (int w1 = lo[1]; w1 <= hi[1]; ++w1)
        for (int w0 = lo[0]; w0 <= hi[0]; ++w0) {
          const double x = a.VF[(long long)a.ncomp * post_lin(a, w0, w1, w2, w3) + comp];
          if (x != x) return x;
          if (f1 && f2) continue;
          long long lt = 0, le = 0;
          for (int u3 = lo[3]; u3 <= hi[3]; ++u3)
            for (int u2 = lo[2]; u2 <= hi[2]; ++u2)
              for (int u1 = lo[1]; u1 <= hi[1]; ++u1)
                for (int u0 = lo[0]; u0 <= hi[0]; ++u0) {
                  const double y = a.VF[(long long)a.ncomp * post_lin(a, u0, u1, u2, u3) + comp];
                  lt += y < x;
                  le += y <= x;
                }
          if (!f1 && lt <= k1 && k1 < le) {
            v1 = x;
            f1 = true;
          }
          if (!f2 && lt <= k2 && k2 < le) {
            v2 = x;
            f2 = true;
          }
        }
  return k1 == k2 ? v1 : (v1 + v2) / 2.0;
}

// Statistics.mean of component comp over the window (sequential sum in
// column-major order, then / count)
MQP_HD MQP_FI double post_mean(const PostArgs& a, const int (&lo)[POST_MAXD], const int (&hi)[POST_MAXD], int comp) {
  double s = 0.0;
  for (int w3 = lo[3]; w3 <= hi[3]; ++w3)
    for (int w2 = lo[2]; w2 <= hi[2]; ++w2)
      for (int w1 = lo[1]; w1 <= hi[1]; ++w1)
        for (int w0 = lo[0]; w0 <= hi[0]; ++w0) s += a.VF[(long long)a.ncomp * post_lin(a, w0, w1, w2, w3) + comp];
  return s / (double)post_count(lo, hi);
}

// average(radius, VF) (postprocessing.jl:364-381): the window mean of each component
MQP_HD MQP_FI void post_average_at(const PostArgs& a, long long i) {
  int c[POST_MAXD], lo[POST_MAXD], hi[POST_MAXD];
  post_coords(a, i, c);
  post_window(a, c, lo, hi);
  for (int k = 0; k < a.ncomp; ++k) a.out[(long long)a.ncomp * i + k] = post_mean(a, lo, hi, k);
}

// collectiveness(radius, VF; max_angle) (postprocessing.jl:291-331): the
// fraction of window vectors whose normalised dot product with the centre's
// exceeds cosd(max_angle) (p0 = cosd(max_angle)); Float32 output.  A zero
// vector normalises to NaN and is similar to nothing.
MQP_HD MQP_FI void post_collectiveness_at(const PostArgs& a, long long i) {
  int c[POST_MAXD], lo[POST_MAXD], hi[POST_MAXD];
  post_coords(a, i, c);
  post_window(a, c, lo, hi);
  const double mag = post_mag(a.VF, a.ncomp, i);
  long long similar = 0;
  for (int w3 = lo[3]; w3 <= hi[3]; ++w3)
    for (int w2 = lo[2]; w2 <= hi[2]; ++w2)
      for (int w1 = lo[1]; w1 <= hi[1]; ++w1)
        for (int w0 = lo[0]; w0 <= hi[0]; ++w0) {
          const long long l = post_lin(a, w0, w1, w2, w3);
          const double mag_ = post_mag(a.VF, a.ncomp, l);
          double dot = 0.0;
          for (int k = 0; k < a.ncomp; ++k)
            dot = padd(dot, pmul(a.VF[(long long)a.ncomp * i + k] / mag, a.VF[(long long)a.ncomp * l + k] / mag_));
          similar += dot > a.p0;
        }
  a.outf[i] = (float)((double)similar / (double)post_count(lo, hi));
}

// similarityAveraging(radius, VF; max_angle, normalize, scale_by_similarity,
// similarity_exponent) (postprocessing.jl:475-523), the VF method: the sum of
// the window vectors similar to the centre (dot of the normalised vectors >
// cosd(max_angle) = p0), divided by its norm if normalize (i0), times
// (similar / count)^similarity_exponent (p1) if scale_by_similarity (i1).
// Zero vectors are left as they are; a zero neighbour adds nothing (Julia's
// `false * NaN == 0`).
MQP_HD MQP_FI void post_similarity_averaging_at(const PostArgs& a, long long i) {
  const int nc = a.ncomp;
  const double mag = post_mag(a.VF, nc, i);
  if (mag == 0.0) {
    for (int k = 0; k < nc; ++k) a.out[(long long)nc * i + k] = a.VF[(long long)nc * i + k];
    return;
  }
  int c[POST_MAXD], lo[POST_MAXD], hi[POST_MAXD];
  post_coords(a, i, c);
  post_window(a, c, lo, hi);
  double avg[4] = {0.0, 0.0, 0.0, 0.0};
  long long similar = 0;
  for (int w3 = lo[3]; w3 <= hi[3]; ++w3)
    for (int w2 = lo[2]; w2 <= hi[2]; ++w2)
      for (int w1 = lo[1]; w1 <= hi[1]; ++w1)
        for (int w0 = lo[0]; w0 <= hi[0]; ++w0) {
          const long long l = post_lin(a, w0, w1, w2, w3);
          const double mag_ = post_mag(a.VF, nc, l);
          double dot = 0.0;
          for (int k = 0; k < nc; ++k)
            dot = padd(dot, pmul(a.VF[(long long)nc * i + k] / mag, a.VF[(long long)nc * l + k] / mag_));
          if (dot > a.p0) {
            for (int k = 0; k < nc && k < 4; ++k) avg[k] = padd(avg[k], pmul(a.VF[(long long)nc * l + k] / mag_, mag_));
            ++similar;
          }
        }
  double fac = 1.0;
  if (a.i0) {
    double s = 0.0;
    for (int k = 0; k < nc && k < 4; ++k) s = padd(s, pmul(avg[k], avg[k]));
    fac /= sqrt(s);
  }
  if (a.i1) fac *= pow((double)similar / (double)post_count(lo, hi), a.p1);
  for (int k = 0; k < nc && k < 4; ++k) a.out[(long long)nc * i + k] = avg[k] * fac;
}

// TH_masking (postprocessing.jl:660-670): cmp(map, th), i0 = 0 for x > th
// (the default cmp) and 1 for x < th (remove_low_SN's), p0 = th
MQP_HD MQP_FI void post_th_mask_at(const PostArgs& a, long long i) {
  const double x = a.VF[i];
  a.mask_out[i] = (uint8_t)(a.i0 == 0 ? (x > a.p0) : (x < a.p0));
}

// STD_masking (postprocessing.jl:598-609): |map - mean| > n * std with
// p0 = n, p1 = mean, p2 = std (n-1 normalised) of the whole map
MQP_HD MQP_FI void post_std_mask_at(const PostArgs& a, long long i) {
  a.mask_out[i] = (uint8_t)(fabs(a.VF[i] - a.p1) > a.p0 * a.p2);
}

// The replacement step of STD_filtering / TH_filtering / remove_low_SN
// (postprocessing.jl:630-643, :692-706, :723-732): masked vectors take the
// zero vector (zeroReplace), the window median (medianReplace) or the window
// mean (meanReplace) of the ORIGINAL field, per component (i0 = kind);
// others are copied.
MQP_HD MQP_FI void post_replace_at(const PostArgs& a, long long i) {
  const int nc = a.ncomp;
  if (!a.mask[i]) {
    for (int k = 0; k < nc; ++k) a.out[(long long)nc * i + k] = a.VF[(long long)nc * i + k];
    return;
  }
  int c[POST_MAXD], lo[POST_MAXD], hi[POST_MAXD];
  post_coords(a, i, c);
  post_window(a, c, lo, hi);
  for (int k = 0; k < nc; ++k) {
    double v = 0.0;
    if (a.i0 == REPLACE_MEDIAN) v = post_median(a, lo, hi, k);
    else if (a.i0 == REPLACE_MEAN) v = post_mean(a, lo, hi, k);
    a.out[(long long)nc * i + k] = v;
  }
}

// local_magnitude_mask(ratio, VF; radius) (postprocessing.jl:202-218): keep
// a vector when |v| / mean(|w| over the window without v) < ratio (p0);
// out = VF times the keep mask, mask_out = 1 where removed
MQP_HD MQP_FI void post_local_magnitude_at(const PostArgs& a, long long i) {
  int c[POST_MAXD], lo[POST_MAXD], hi[POST_MAXD];
  post_coords(a, i, c);
  post_window(a, c, lo, hi);
  const int nc = a.ncomp;
  double s = 0.0;
  for (int w3 = lo[3]; w3 <= hi[3]; ++w3)
    for (int w2 = lo[2]; w2 <= hi[2]; ++w2)
      for (int w1 = lo[1]; w1 <= hi[1]; ++w1)
        for (int w0 = lo[0]; w0 <= hi[0]; ++w0) s += post_mag(a.VF, nc, post_lin(a, w0, w1, w2, w3));
  const double m = post_mag(a.VF, nc, i);
  const double mean = (s - m) / (double)(post_count(lo, hi) - 1);
  const bool keep = m / mean < a.p0;
  // VF .* mask with a Bool mask: Julia's false is a strong zero (signed zero, also for NaN)
  for (int k = 0; k < nc; ++k) {
    const double v = a.VF[(long long)nc * i + k];
    a.out[(long long)nc * i + k] = keep ? v : copysign(0.0, v);
  }
  a.mask_out[i] = (uint8_t)!keep;
}

// matlab_divergence(VF) (postprocessing.jl:918-941): sum over components of
// the central difference along that component's axis, one-sided at the
// border (clamped neighbours, divided by their distance); Float32 output
MQP_HD MQP_FI void post_matlab_divergence_at(const PostArgs& a, long long i) {
  int c[POST_MAXD];
  post_coords(a, i, c);
  float acc = 0.f;
  for (int k = 0; k < a.ncomp && k < a.nd; ++k) {
    int cm[POST_MAXD], cp[POST_MAXD];
    for (int d = 0; d < POST_MAXD; ++d) {
      cm[d] = c[d];
      cp[d] = c[d];
    }
    cm[k] = c[k] - 1 < 0 ? 0 : (c[k] - 1 > a.dims[k] - 1 ? a.dims[k] - 1 : c[k] - 1);
    cp[k] = c[k] + 1 > a.dims[k] - 1 ? a.dims[k] - 1 : c[k] + 1;
    const double vp = a.VF[(long long)a.ncomp * post_lin(a, cp[0], cp[1], cp[2], cp[3]) + k];
    const double vm = a.VF[(long long)a.ncomp * post_lin(a, cm[0], cm[1], cm[2], cm[3]) + k];
    acc += (float)((vp - vm) / (double)abs(cm[k] - cp[k]));
  }
  a.outf[i] = acc;
}

// ---- divergence by correlation with a sink pattern -------------------------
// normalize_sink (postprocessing.jl:757-773) at sink offset k (0-based, size
// 2r+1 per axis, centre r): |centre - k|, zero outside max(r) when circle,
// 1 at the centre
MQP_HD MQP_FI double sink_magnitude(const PostArgs& a, const int (&k)[POST_MAXD], bool circle) {
  double s = 0.0;
  int rmax = 0;
  bool centre = true;
  for (int d = 0; d < a.nd; ++d) {
    const double t = (double)(a.radius[d] - k[d]);
    s = padd(s, pmul(t, t));
    rmax = a.radius[d] > rmax ? a.radius[d] : rmax;
    centre = centre && k[d] == a.radius[d];
  }
  if (centre) return 1.0;
  double m = sqrt(s);
  if (circle && !(m <= (double)rmax)) m = 0.0;
  return m;
}

// normalize_vectorfield (postprocessing.jl:826-845) for one vector: zeroed
// below min_speed (p1 > 0), divided by its magnitude (zero magnitude -> 1)
// when normalize (i0); component comp
MQP_HD MQP_FI double post_vfnorm(const PostArgs& a, long long l, int comp) {
  const double M = post_mag(a.VF, a.ncomp, l);
  double v = a.VF[(long long)a.ncomp * l + comp];
  if (a.p1 > 0.0) v *= (double)(M > a.p1);
  if (a.i0) v /= (M == 0.0 ? 1.0 : M);
  return v;
}

// divergence(radii, VF; normalize, min_speed, divide_by, circle): the
// reference (postprocessing.jl:853-903) cannot run (it passes keywords to the
// positional allocate_tmp_data, :872, and FFTCC_crop does the same); its
// intent, computed here directly: for every vector i,
//   sum_c sum_k sink_c(k) * VFn_c(i + k - r)       (zero outside the field)
// which is FFTCC_crop's centred zero-padded correlation, with
// sink_c(k) = (r_c - k_c) / |centre - k| (sink!, :783-798, NaN -> 0), then
// divided by the number of non-zero sink magnitudes (divide_by "N", i1 = 1)
// or by the window sum of the normalised field's magnitudes ("mags", i1 = 2).
// i2 = circle.
MQP_HD MQP_FI void post_divergence_at(const PostArgs& a, long long i) {
  int c[POST_MAXD];
  post_coords(a, i, c);
  const bool circle = a.i2 != 0;
  double acc = 0.0, nsink = 0.0, smags = 0.0;
  int k[POST_MAXD] = {0, 0, 0, 0};
  int ext[POST_MAXD];
  for (int d = 0; d < POST_MAXD; ++d) ext[d] = d < a.nd ? 2 * a.radius[d] + 1 : 1;
  for (k[3] = 0; k[3] < ext[3]; ++k[3])
    for (k[2] = 0; k[2] < ext[2]; ++k[2])
      for (k[1] = 0; k[1] < ext[1]; ++k[1])
        for (k[0] = 0; k[0] < ext[0]; ++k[0]) {
          const double sm = sink_magnitude(a, k, circle);
          nsink += sm > 0.0;
          int p[POST_MAXD];
          bool in = true;
          for (int d = 0; d < POST_MAXD; ++d) {
            p[d] = d < a.nd ? c[d] + k[d] - a.radius[d] : 0;
            in = in && p[d] >= 0 && p[d] < a.dims[d];
          }
          if (!in) continue;
          const long long l = post_lin(a, p[0], p[1], p[2], p[3]);
          if (a.i1 == DIVIDE_MAGS) {
            double s = 0.0;
            for (int q = 0; q < a.ncomp; ++q) {
              const double v = post_vfnorm(a, l, q);
              s = padd(s, pmul(v, v));
            }
            smags += sqrt(s);
          }
          if (sm == 0.0) continue;
          for (int q = 0; q < a.ncomp && q < a.nd; ++q) {
            double sv = (double)(a.radius[q] - k[q]) / sm;
            if (sv != sv) sv = 0.0;
            acc = padd(acc, pmul(sv, post_vfnorm(a, l, q)));
          }
        }
  if (a.i1 == DIVIDE_N) acc /= nsink;
  else if (a.i1 == DIVIDE_MAGS) acc /= smags;
  a.out[i] = acc;
}

MQP_HD MQP_FI void post_at(const PostArgs& a, long long i) {
  switch (a.op) {
    case POST_MAGNITUDES: a.out[i] = post_mag(a.VF, a.ncomp, i); break;
    case POST_AVERAGE: post_average_at(a, i); break;
    case POST_SIMILARITY_AVERAGING: post_similarity_averaging_at(a, i); break;
    case POST_COLLECTIVENESS: post_collectiveness_at(a, i); break;
    case POST_TH_MASK: post_th_mask_at(a, i); break;
    case POST_STD_MASK: post_std_mask_at(a, i); break;
    case POST_REPLACE: post_replace_at(a, i); break;
    case POST_LOCAL_MAGNITUDE: post_local_magnitude_at(a, i); break;
    case POST_MATLAB_DIVERGENCE: post_matlab_divergence_at(a, i); break;
    case POST_DIVERGENCE: post_divergence_at(a, i); break;
    default: break;
  }
}

}  // namespace mqp
