// Multi-pass refinement with window deformation (mqp_params.refine = 2).
//
// The reference's pass loop leaves the multi-pass step as a TODO
// (src/multi_quickPIV.jl:55 "replace by the new multi-pass code", with the
// displacement hook of get_search_coordinates unused, src/utils/piv_ops.jl:64,
// and interpolate_vectorfield! commented out, :92).  This build's deforming
// pass, after the coarsest one:
//
//   1. The previous (coarser) pass's vectors, which sit at its IA centres
//      c_j = j * step_c + (interSize_c - 1) / 2 (0-based pixels), are
//      interpolated multilinearly to a dense predictor D(p) (clamped to the
//      outermost centres; non-finite vectors count as 0).
//   2. Both images are resampled symmetrically around it, multilinear and
//      clamped at the image border: img1'(p) = img1(p - D(p)/2),
//      img2'(p) = img2(p + D(p)/2), computed in FP64 and stored in the
//      images' precision.  If img2(y) = img1(y - u), the deformed pair is
//      shifted by the residual u - D.
//   3. The ordinary pass runs on the deformed pair (no whole-pixel shift)
//      and each vector becomes D(c) + residual, D taken at the fine IA's
//      centre c; IAs the threshold skips (tested on img1') stay 0.
#pragma once

#include "mqp_fft.cuh"

#include <math.h>
#include <stdint.h>

namespace mqp {

// FP64 products and sums rounded one at a time (no fused multiply-add), so
// the deformed images equal a plain FP64 restatement's bit for bit
MQP_HD MQP_FI double dmul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
MQP_HD MQP_FI double dadd(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}

struct DeformArgs {
  int nd;
  long long dims[3];       // image extents (dims[2] = 1 for 2D)
  int dtype;               // 0 float32, 1 float64
  const void* img1;
  const void* img2;
  void* out1;              // deformed images, same layout and precision
  void* out2;
  // the coarse vector field
  const double* VFc;       // (nd, vf_c...) column-major
  int vf_c[3];
  int isz_c[3], st_c[3];
  // the fine pass (add step)
  double* VF;              // (nd, vf_f...) column-major: residuals in, vectors out
  int vf_f[3];
  int isz_f[3], st_f[3];
  double threshold;        // skip test of the fine pass (threshold >= 0)
};

// The dense predictor at 0-based position pos (one value per component).
MQP_HD MQP_FI void deform_predictor(const DeformArgs& a, const double (&pos)[3], double (&D)[3]) {
  int j0[3] = {0, 0, 0}, j1[3] = {0, 0, 0};
  double t[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < a.nd; ++d) {
    double f = (pos[d] - 0.5 * (a.isz_c[d] - 1)) / a.st_c[d];
    const double hi = (double)(a.vf_c[d] - 1);
    f = f < 0.0 ? 0.0 : (f > hi ? hi : f);
    int j = (int)floor(f);
    if (j > a.vf_c[d] - 1) j = a.vf_c[d] - 1;
    j0[d] = j;
    j1[d] = j + 1 < a.vf_c[d] ? j + 1 : j;
    t[d] = f - (double)j;
  }
  for (int c = 0; c < a.nd; ++c) D[c] = 0.0;
  const int corners = 1 << a.nd;
  for (int k = 0; k < corners; ++k) {
    double w = 1.0;
    long long idx = 0, mul = 1;
    for (int d = 0; d < a.nd; ++d) {
      const bool up = (k >> d) & 1;
      w = dmul(w, up ? t[d] : 1.0 - t[d]);
      idx += (long long)(up ? j1[d] : j0[d]) * mul;
      mul *= a.vf_c[d];
    }
    for (int c = 0; c < a.nd; ++c) {
      const double v = a.VFc[(long long)a.nd * idx + c];
      D[c] = dadd(D[c], dmul(w, (v == v && v < 1e300 && v > -1e300) ? v : 0.0));
    }
  }
}

MQP_HD MQP_FI double deform_load(const void* img, int dtype, long long i) {
  return dtype == 0 ? (double)((const float*)img)[i] : ((const double*)img)[i];
}

// Multilinear sample of an image at 0-based position pos, clamped to the
// image (the border values extend outwards).
MQP_HD MQP_FI double deform_sample(const DeformArgs& a, const void* img, const double (&pos)[3]) {
  long long i0[3] = {0, 0, 0}, i1[3] = {0, 0, 0};
  double t[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < a.nd; ++d) {
    const double hi = (double)(a.dims[d] - 1);
    double f = pos[d] < 0.0 ? 0.0 : (pos[d] > hi ? hi : pos[d]);
    if (!(f == f)) f = 0.0;
    long long j = (long long)floor(f);
    if (j > a.dims[d] - 1) j = a.dims[d] - 1;
    i0[d] = j;
    i1[d] = j + 1 < a.dims[d] ? j + 1 : j;
    t[d] = f - (double)j;
  }
  double s = 0.0;
  const int corners = 1 << a.nd;
  for (int k = 0; k < corners; ++k) {
    double w = 1.0;
    long long idx = 0, mul = 1;
    for (int d = 0; d < a.nd; ++d) {
      const bool up = (k >> d) & 1;
      w = dmul(w, up ? t[d] : 1.0 - t[d]);
      idx += (up ? i1[d] : i0[d]) * mul;
      mul *= a.dims[d];
    }
    s = dadd(s, dmul(w, deform_load(img, a.dtype, idx)));
  }
  return s;
}

// Pixel i (column-major linear index): the two deformed images there.
MQP_HD MQP_FI void deform_pixel(const DeformArgs& a, long long i) {
  double p[3] = {0.0, 0.0, 0.0};
  long long r = i;
  for (int d = 0; d < a.nd; ++d) {
    p[d] = (double)(r % a.dims[d]);
    r /= a.dims[d];
  }
  double D[3];
  deform_predictor(a, p, D);
  double q1[3] = {0.0, 0.0, 0.0}, q2[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < a.nd; ++d) {
    q1[d] = dadd(p[d], -0.5 * D[d]);  // 0.5 D is exact
    q2[d] = dadd(p[d], 0.5 * D[d]);
  }
  const double v1 = deform_sample(a, a.img1, q1), v2 = deform_sample(a, a.img2, q2);
  if (a.dtype == 0) {
    ((float*)a.out1)[i] = (float)v1;
    ((float*)a.out2)[i] = (float)v2;
  } else {
    ((double*)a.out1)[i] = v1;
    ((double*)a.out2)[i] = v2;
  }
}

// Fine IA i: VF += D(centre) unless the threshold skip test (on the
// deformed img1) left it at zero.
MQP_HD MQP_FI void deform_add(const DeformArgs& a, long long i) {
  int jf[3] = {0, 0, 0};
  long long r = i;
  for (int d = 0; d < a.nd; ++d) {
    jf[d] = (int)(r % a.vf_f[d]);
    r /= a.vf_f[d];
  }
  if (a.threshold >= 0.0) {
    // skip_inter_region (src/utils/piv_ops.jl:134-146) on the deformed img1
    double m = -INFINITY;
    const int n2 = a.nd == 3 ? a.isz_f[2] : 1;
    for (int z = 0; z < n2; ++z)
      for (int x = 0; x < a.isz_f[1]; ++x)
        for (int y = 0; y < a.isz_f[0]; ++y) {
          const long long yy = (long long)jf[0] * a.st_f[0] + y, xx = (long long)jf[1] * a.st_f[1] + x;
          const long long zz = a.nd == 3 ? (long long)jf[2] * a.st_f[2] + z : 0;
          const double v = deform_load(a.out1, a.dtype, yy + a.dims[0] * (xx + a.dims[1] * zz));
          m = v > m ? v : m;
        }
    if (m < a.threshold) return;
  }
  double c[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < a.nd; ++d) c[d] = (double)jf[d] * a.st_f[d] + 0.5 * (a.isz_f[d] - 1);
  double D[3];
  deform_predictor(a, c, D);
  for (int d = 0; d < a.nd; ++d) a.VF[(long long)a.nd * i + d] = dadd(a.VF[(long long)a.nd * i + d], D[d]);
}

}  // namespace mqp
