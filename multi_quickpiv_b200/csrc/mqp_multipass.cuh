// Multi-pass refinement: the whole-pixel predictor a finer pass takes from
// the previous (coarser) pass.
//
// The reference's pass loop (src/multi_quickPIV.jl:55-93) re-runs the
// scale-1 geometry on every pass and never hands a displacement to
// get_search_coordinates (src/utils/piv_ops.jl:64, :84), so its multipass is
// a stub.  With mqp_params.refine set, passes run at scales 2^(m-1), ..., 2,
// 1 (interSize, searchMargin and step times the scale, the reference's own
// _isize/_smarg/_step accessors, src/piv_parameters.jl:83-87), and every
// fine IA's search window moves by the rounded displacement of the coarse IA
// whose centre is nearest to its own, per axis (ties to the higher index).
#pragma once

#include "mqp_fft.cuh"

#include <math.h>
#include <stdint.h>

namespace mqp {

struct PredArgs {
  int ndims;
  int vf_f[3];                 // fine vector field
  int vf_c[3];                 // coarse vector field
  int isz_f[3], st_f[3];       // fine interSize, step
  int isz_c[3], st_c[3];       // coarse interSize, step
  const double* VFc;           // (ndims, vf_c...) column-major
  int32_t* pred;               // (ndims, vf_f...) column-major
};

MQP_HD MQP_FI long long floor_div(long long a, long long b) {  // b > 0
  const long long q = a / b;
  return (a % b != 0 && a < 0) ? q - 1 : q;
}

// Nearest coarse index along one axis for fine index jf.  Centres are taken in
// doubled coordinates, 2 (TLF - 1) + isize - 1, to stay in integers; the
// nearest coarse centre minimises |2 jc st_c + isz_c - 1 - cf|.
MQP_HD MQP_FI int nearest_coarse(int jf, int isz_f, int st_f, int isz_c, int st_c, int vf_c) {
  const long long cf = 2LL * jf * st_f + isz_f - 1;
  long long jc = floor_div(cf - (isz_c - 1) + st_c, 2LL * st_c);
  if (jc < 0) jc = 0;
  if (jc > vf_c - 1) jc = vf_c - 1;
  return (int)jc;
}

// round half away from zero; non-finite (NaN from a degenerate coarse
// window) gives no shift
MQP_HD MQP_FI int32_t round_pred(double v) {
  if (!(v == v) || v > 1e9 || v < -1e9) return 0;
  const double r = floor(fabs(v) + 0.5);
  return (int32_t)(v < 0 ? -r : r);
}

// predictor of fine IA i (column-major linear index over vf_f)
MQP_HD MQP_FI void predictor_at(const PredArgs& a, long long i) {
  int jf[3] = {0, 0, 0};
  long long r = i;
  for (int d = 0; d < a.ndims; ++d) {
    jf[d] = (int)(r % a.vf_f[d]);
    r /= a.vf_f[d];
  }
  long long lc = 0, mul = 1;
  bool empty = false;
  for (int d = 0; d < a.ndims; ++d) {
    if (a.vf_c[d] < 1) empty = true;
    const int jc = empty ? 0 : nearest_coarse(jf[d], a.isz_f[d], a.st_f[d], a.isz_c[d], a.st_c[d], a.vf_c[d]);
    lc += jc * mul;
    mul *= a.vf_c[d] > 0 ? a.vf_c[d] : 1;
  }
  for (int d = 0; d < a.ndims; ++d)
    a.pred[(long long)a.ndims * i + d] = empty ? 0 : round_pred(a.VFc[(long long)a.ndims * lc + d]);
}

}  // namespace mqp
