// Host emulation of the post-processing kernels for CPU tests (test
// infrastructure, not part of the product library): the same per-vector
// functions as post_kernel (mqp_post.cuh), run over every vector in a host
// loop; the STD mean / deviation reductions are plain sequential sums.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "mqp_post.cuh"

using namespace mqp;

extern "C" __attribute__((visibility("default"))) int mqp_emu_post(
    int op, int ncomp, int nd, const int* dims, const int* radius, const double* in, const uint8_t* mask,
    double* out, float* outf, uint8_t* mask_out, double p0, double p1, double p2, int i0, int i1, int i2) {
  PostArgs a;
  memset(&a, 0, sizeof(a));
  a.op = op;
  a.ncomp = ncomp;
  a.nd = nd;
  a.n = 1;
  for (int d = 0; d < POST_MAXD; ++d) {
    a.dims[d] = d < nd ? dims[d] : 1;
    a.radius[d] = d < nd ? radius[d] : 0;
    a.n *= a.dims[d];
  }
  a.VF = in;
  a.mask = mask;
  a.out = out;
  a.outf = outf;
  a.mask_out = mask_out;
  a.p0 = p0;
  a.p1 = p1;
  a.p2 = p2;
  a.i0 = i0;
  a.i1 = i1;
  a.i2 = i2;
  if (op == POST_STD_MASK) {
    double s = 0.0;
    for (long long i = 0; i < a.n; ++i) s += in[i];
    const double mean = s / (double)a.n;
    double v = 0.0;
    for (long long i = 0; i < a.n; ++i) v += (in[i] - mean) * (in[i] - mean);
    a.p1 = mean;
    a.p2 = sqrt(v / (double)(a.n - 1));
  }
  for (long long i = 0; i < a.n; ++i) post_at(a, i);
  return 0;
}
