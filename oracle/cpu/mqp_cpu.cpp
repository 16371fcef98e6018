// C++17/OpenMP Float64 restatement of multi_quickPIV's per-IA PIV loop
// (TEST ORACLE + CPU BASELINE; never part of the CUDA product).
//
// It follows the same reference lines as oracle/piv_oracle.py
// (src/multi_quickPIV.jl:40-96, src/utils/piv_ops.jl:6-127,134-157,249-367,
// src/utils/fft_ops.jl:95-105,145-198, src/utils/common_ops.jl:98-124,142-245,
// the four src/crosscorrelation_algorithms files and their *_ops.jl helpers),
// with two differences in HOW, not WHAT:
//  - FFTW (not vendored, FFTW_jll 3.3.10) is replaced by a self-written
//    mixed-radix (2,3,4,5) complex FFT in double; the two real transforms of
//    F and G ride in one complex transform (z = F + iG), so each IA costs two
//    complex N-D transforms of the reference's good_size_real size.
//  - the interrogation areas are spread over OpenMP threads (the reference's
//    loop is serial; FFTW threads inside each tiny transform).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <complex>
#include <vector>

#include "mqp.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cd = std::complex<double>;

// ---- FFT -------------------------------------------------------------------
struct Plan1D {
  int n = 0;
  std::vector<int> radices;
  std::vector<cd> tw;  // exp(-2 pi i k / n)
  void init(int n_) {
    n = n_;
    radices.clear();
    int m = n;
    while (m % 4 == 0) { radices.push_back(4); m /= 4; }
    while (m % 2 == 0) { radices.push_back(2); m /= 2; }
    while (m % 3 == 0) { radices.push_back(3); m /= 3; }
    while (m % 5 == 0) { radices.push_back(5); m /= 5; }
    if (m > 1) radices.push_back(m);  // generic DFT radix
    tw.resize(n);
    for (int k = 0; k < n; ++k) tw[k] = std::polar(1.0, -2.0 * M_PI * k / n);
  }
};

// Self-sorting (Stockham) decimation-in-frequency FFT, out-of-place
// ping-pong; sign = -1 forward, +1 inverse (unnormalised).  Stage with
// current length L, stride s, radix r (m = L/r):
//   y[q + s(r p + u)] = W_L^(p u) * sum_j x[q + s(p + m j)] W_r^(j u)
void fft1d(const Plan1D& pl, cd* x, cd* work, int sign) {
  const int n = pl.n;
  if (n == 1) return;
  cd* src = x;
  cd* dst = work;
  int L = n, s = 1;
  for (int r : pl.radices) {
    const int m = L / r;
    const int step = n / L;  // W_L^k == W_n^(k*step)
    for (int p = 0; p < m; ++p) {
      for (int q = 0; q < s; ++q) {
        cd a[64], b[64];
        for (int j = 0; j < r; ++j) a[j] = src[q + s * (p + m * j)];
        if (r == 2) {
          b[0] = a[0] + a[1];
          b[1] = a[0] - a[1];
        } else if (r == 4) {
          const cd s02 = a[0] + a[2], d02 = a[0] - a[2], s13 = a[1] + a[3], d13 = a[1] - a[3];
          // forward: W_4 = -i
          const cd jd = sign < 0 ? cd(d13.imag(), -d13.real()) : cd(-d13.imag(), d13.real());
          b[0] = s02 + s13;
          b[2] = s02 - s13;
          b[1] = d02 + jd;
          b[3] = d02 - jd;
        } else {
          for (int u = 0; u < r; ++u) {
            cd acc = 0.0;
            for (int j = 0; j < r; ++j) {
              cd w = pl.tw[(size_t)((j * u) % r) * (n / r)];
              if (sign > 0) w = std::conj(w);
              acc += a[j] * w;
            }
            b[u] = acc;
          }
        }
        for (int u = 0; u < r; ++u) {
          cd w = pl.tw[(size_t)((long long)p * u * step % n)];
          if (sign > 0) w = std::conj(w);
          dst[q + s * (r * p + u)] = b[u] * w;
        }
      }
    }
    L = m;
    s *= r;
    std::swap(src, dst);
  }
  if (src != x) memcpy(x, src, sizeof(cd) * n);
}

struct PlanND {
  int nd = 2;
  int cs[3] = {1, 1, 1};
  Plan1D p[3];
  void init(int nd_, const int* c) {
    nd = nd_;
    for (int d = 0; d < 3; ++d) cs[d] = d < nd ? c[d] : 1;
    for (int d = 0; d < nd; ++d) p[d].init(cs[d]);
  }
  size_t size() const { return (size_t)cs[0] * cs[1] * cs[2]; }
  // column-major, axis 0 fastest
  void run(cd* a, int sign, std::vector<cd>& line, std::vector<cd>& work) const {
    const int n0 = cs[0], n1 = cs[1], n2 = cs[2];
    int mx = n0 > n1 ? n0 : n1;
    mx = mx > n2 ? mx : n2;
    line.resize(mx);
    work.resize(mx);
    for (int z = 0; z < n2; ++z)
      for (int y = 0; y < n1; ++y) fft1d(p[0], a + (size_t)n0 * (y + (size_t)n1 * z), work.data(), sign);
    for (int z = 0; z < n2; ++z)
      for (int x = 0; x < n0; ++x) {
        for (int y = 0; y < n1; ++y) line[y] = a[x + (size_t)n0 * (y + (size_t)n1 * z)];
        fft1d(p[1], line.data(), work.data(), sign);
        for (int y = 0; y < n1; ++y) a[x + (size_t)n0 * (y + (size_t)n1 * z)] = line[y];
      }
    if (nd == 3)
      for (int y = 0; y < n1; ++y)
        for (int x = 0; x < n0; ++x) {
          for (int z = 0; z < n2; ++z) line[z] = a[x + (size_t)n0 * (y + (size_t)n1 * z)];
          fft1d(p[2], line.data(), work.data(), sign);
          for (int z = 0; z < n2; ++z) a[x + (size_t)n0 * (y + (size_t)n1 * z)] = line[z];
        }
  }
};

// ---- reference helpers -------------------------------------------------------
int root_(int base, int goal, int mul) {  // root (src/utils/fft_ops.jl:165-171)
  int n = 0;
  long long v = (long long)mul * base;
  while (v < goal) {
    ++n;
    v *= base;
  }
  return n;
}

int good_size_real(int n) {  // src/utils/fft_ops.jl:175-198
  if (n <= 6) return n;
  int bestfac = 2 * n;
  for (int n5 = 0; n5 <= root_(11, bestfac, 5); ++n5) {
    long long x = 1;
    for (int i = 0; i < n5; ++i) x *= 5;
    while (x < n) x *= 2;
    while (true) {
      if (x < n) x *= 3;
      else if (x > n) {
        if (x < bestfac) bestfac = (int)x;
        if (x & 1) break;
        x >>= 1;
      } else return n;
    }
  }
  return bestfac;
}

double px(const void* img, int dtype, long long i) {
  return dtype == MQP_F64 ? ((const double*)img)[i] : (double)((const float*)img)[i];
}

struct Geo {
  int IR_TLF[3], IR_BRB[3], SR_TLF[3], SR_BRB[3], toff[3], boff[3];
};

struct Ctx {
  int nd;
  int64_t dims[3];
  int IS[3], SM[3], st[3], cs[3], P[3], SS[3];
  int64_t vf[3];
  int alg;
  double thr, mthr;
  int sn;
};

// get_interrogation_coordinates / get_search_coordinates (src/utils/piv_ops.jl:38-76)
Geo geo(const Ctx& c, int64_t ia) {
  Geo g;
  int64_t rem = ia;
  for (int d = 0; d < 3; ++d) {
    int64_t v = 0;
    if (d < c.nd) {
      v = rem % c.vf[d];
      rem /= c.vf[d];
    }
    const int T = 1 + (int)v * c.st[d];
    const int B = T + c.IS[d] - 1;
    const int S = c.SM[d];
    g.IR_TLF[d] = T;
    g.IR_BRB[d] = B;
    g.SR_TLF[d] = T - S > 1 ? T - S : 1;
    g.SR_BRB[d] = (B + S) < (int)c.dims[d] ? (B + S) : (int)c.dims[d];
    const int t = T - (S - 1);
    g.toff[d] = t < 0 ? -t : 0;
    const int b = (int)c.dims[d] - (B + S);
    g.boff[d] = b < 0 ? -b : 0;
  }
  return g;
}

inline size_t cidx(const int* n, int a, int b, int z) { return (size_t)a + (size_t)n[0] * (b + (size_t)n[1] * z); }

struct Work {
  std::vector<cd> z1, z2, line, wk;
  std::vector<double> padF, padG, pad3, pad4, integ, cc, cc2;
};

// window sums over pad_G[1:SS] squared (integralArraySQ! + add_numerator_nsqecc)
void window_sums(const Ctx& c, const std::vector<double>& padG, std::vector<double>& integ, std::vector<double>& out) {
  const int h = c.SS[0], w = c.SS[1], dd = c.nd == 3 ? c.SS[2] : 1;
  const int ih = h + 1, iw = w + 1, idd = dd + 1;
  integ.assign((size_t)ih * iw * (c.nd == 3 ? idd : 1), 0.0);
  auto I = [&](int r, int q, int z) -> double& { return integ[(size_t)r + (size_t)ih * (q + (size_t)iw * z)]; };
  auto G = [&](int r, int q, int z) { return padG[cidx(c.cs, r, q, z)]; };
  if (c.nd == 2) {
    for (int q = 1; q <= w; ++q)
      for (int r = 1; r <= h; ++r) {
        const double v = G(r - 1, q - 1, 0);
        I(r, q, 0) = v * v + I(r - 1, q, 0) + I(r, q - 1, 0) - I(r - 1, q - 1, 0);
      }
  } else {
    for (int z = 1; z <= dd; ++z)
      for (int q = 1; q <= w; ++q) {
        double tmp = 0.0;
        for (int r = 1; r <= h; ++r) {
          const double v = G(r - 1, q - 1, z - 1);
          const double v2 = v * v;
          I(r, q, z) = v2 + I(r, q - 1, z) + I(r, q, z - 1) - I(r, q - 1, z - 1) + tmp;
          tmp += v2;
        }
      }
  }
  const int P0 = c.P[0], P1 = c.P[1], P2 = c.nd == 3 ? c.P[2] : 1;
  out.assign((size_t)P0 * P1 * P2, 0.0);
  for (int z = 0; z < P2; ++z)
    for (int q = 0; q < P1; ++q)
      for (int r = 0; r < P0; ++r) {
        double s;
        if (c.nd == 2) {
          const int Tr = r, L = q, D = r + c.IS[0], R = q + c.IS[1];
          s = 0.0;
          s += I(D, R, 0);
          s += I(Tr, L, 0);
          s -= I(Tr, R, 0);
          s -= I(D, L, 0);
        } else {
          const int Tr = r, L = q, F = z, D = r + c.IS[0], R = q + c.IS[1], B = z + c.IS[2];
          s = 0.0;
          s += I(D, R, B);
          s -= I(Tr, L, F);
          s -= I(Tr, R, B);
          s -= I(D, L, B);
          s -= I(D, R, F);
          s += I(D, L, F);
          s += I(Tr, R, F);
          s += I(Tr, L, B);
        }
        out[(size_t)r + (size_t)P0 * (q + (size_t)P1 * z)] = s;
      }
}

// pad arrays: column-major of size cs
void fill_pads(const Ctx& c, const Geo& g, const void* img1, const void* img2, const void* mask, int dtype,
               Work& w, double& sumF2) {
  const size_t n = (size_t)c.cs[0] * c.cs[1] * c.cs[2];
  w.padF.assign(n, 0.0);
  w.padG.assign(n, 0.0);
  const int64_t H = c.dims[0], W = c.dims[1];
  const int D3 = c.nd == 3 ? c.IS[2] : 1;
  double mF = 0.0, mG = 0.0;
  auto img_idx = [&](int r, int q, int z) { return (long long)r + H * ((long long)q + W * z); };
  if (c.alg == MQP_ZNCC) {  // copy_*_minus_mean! (src/utils/zncc_ops.jl:7-25)
    double s = 0.0;
    for (int z = 0; z < D3; ++z)
      for (int q = 0; q < c.IS[1]; ++q)
        for (int r = 0; r < c.IS[0]; ++r)
          s += px(img1, dtype, img_idx(g.IR_TLF[0] - 1 + r, g.IR_TLF[1] - 1 + q, (c.nd == 3 ? g.IR_TLF[2] - 1 : 0) + z));
    mF = s / ((double)c.IS[0] * c.IS[1] * D3);
    s = 0.0;
    long long cnt = 0;
    const int z0 = c.nd == 3 ? g.SR_TLF[2] : 1, z1 = c.nd == 3 ? g.SR_BRB[2] : 1;
    for (int z = z0; z <= z1; ++z)
      for (int q = g.SR_TLF[1]; q <= g.SR_BRB[1]; ++q)
        for (int r = g.SR_TLF[0]; r <= g.SR_BRB[0]; ++r, ++cnt) s += px(img2, dtype, img_idx(r - 1, q - 1, z - 1));
    mG = s / (double)cnt;
  }
  sumF2 = 0.0;
  for (int z = 0; z < D3; ++z)
    for (int q = 0; q < c.IS[1]; ++q)
      for (int r = 0; r < c.IS[0]; ++r) {
        const long long ii = img_idx(g.IR_TLF[0] - 1 + r, g.IR_TLF[1] - 1 + q, (c.nd == 3 ? g.IR_TLF[2] - 1 : 0) + z);
        double v = px(img1, dtype, ii) - mF;
        if (mask) {
          const double m = px(mask, dtype, ii);
          v = px(img1, dtype, ii) * m;
          sumF2 += v * v / (m > 0 ? m : 1.0);
        } else {
          sumF2 += v * v;
        }
        w.padF[cidx(c.cs, r, q, z)] = v;
      }
  if (mask) {
    w.pad3.assign(n, 0.0);
    for (int z = 0; z < D3; ++z)
      for (int q = 0; q < c.IS[1]; ++q)
        for (int r = 0; r < c.IS[0]; ++r)
          w.pad3[cidx(c.cs, r, q, z)] = px(mask, dtype, img_idx(g.IR_TLF[0] - 1 + r, g.IR_TLF[1] - 1 + q, (c.nd == 3 ? g.IR_TLF[2] - 1 : 0) + z));
  }
  const int z0 = c.nd == 3 ? g.SR_TLF[2] : 1, z1 = c.nd == 3 ? g.SR_BRB[2] : 1;
  for (int z = z0; z <= z1; ++z)
    for (int q = g.SR_TLF[1]; q <= g.SR_BRB[1]; ++q)
      for (int r = g.SR_TLF[0]; r <= g.SR_BRB[0]; ++r) {
        const int pr = r - g.SR_TLF[0] + g.toff[0];
        const int pq = q - g.SR_TLF[1] + g.toff[1];
        const int pz = c.nd == 3 ? z - g.SR_TLF[2] + g.toff[2] : 0;
        w.padG[cidx(c.cs, pr, pq, pz)] = px(img2, dtype, img_idx(r - 1, q - 1, z - 1)) - mG;
      }
}

// cc = IFFT(conj(FFT(a)) FFT(b)) / prod(cs) for two real pads via z = a + i b
void corr2(const PlanND& pl, const std::vector<double>& a, const std::vector<double>& b, Work& w,
           std::vector<double>& out) {
  const size_t n = pl.size();
  w.z1.resize(n);
  for (size_t i = 0; i < n; ++i) w.z1[i] = cd(a[i], b[i]);
  pl.run(w.z1.data(), -1, w.line, w.wk);
  w.z2.resize(n);
  const int n0 = pl.cs[0], n1 = pl.cs[1], n2 = pl.cs[2];
  for (int z = 0; z < n2; ++z)
    for (int y = 0; y < n1; ++y)
      for (int x = 0; x < n0; ++x) {
        const size_t k = (size_t)x + (size_t)n0 * (y + (size_t)n1 * z);
        const size_t mk = (size_t)((n0 - x) % n0) + (size_t)n0 * (((n1 - y) % n1) + (size_t)n1 * ((n2 - z) % n2));
        const cd Z = w.z1[k], Zm = std::conj(w.z1[mk]);
        const cd A = 0.5 * (Z + Zm);
        const cd B = cd(0, -0.5) * (Z - Zm);
        w.z2[k] = std::conj(A) * B;
      }
  pl.run(w.z2.data(), +1, w.line, w.wk);
  out.resize(n);
  const double inv = 1.0 / (double)n;
  for (size_t i = 0; i < n; ++i) out[i] = w.z2[i].real() * inv;
}

// diag (nullable): per IA, MQP_CPU_DIAG doubles describing the similarity block on the lags
// first_fullovp_peak searches: [0] largest value, [1] second largest (-inf if none), [2] largest
// magnitude, [3] compute_SN's denominator (mean of the SN region without its maximum), [4] 1 when
// the IA was skipped.  Test infrastructure: near-tie and SN-conditioning counts.
constexpr int MQP_CPU_DIAG = 5;

void ia_piv(const Ctx& c, const PlanND& pl, int64_t ia, const void* img1, const void* img2, const void* mask,
            const void* mskip, int dtype, double* VF, double* SN, Work& w, double* diag = nullptr) {
  if (diag) {
    double* d = diag + MQP_CPU_DIAG * ia;
    d[0] = d[1] = -INFINITY;
    d[2] = 0.0;
    d[3] = NAN;
    d[4] = 0.0;
  }
  const Geo g = geo(c, ia);
  const int nd = c.nd;
  const int64_t H = c.dims[0], Wd = c.dims[1];
  // skip_inter_region (src/utils/piv_ops.jl:134-157)
  auto ia_max = [&](const void* im) {
    double m = -INFINITY;
    const int D3 = nd == 3 ? c.IS[2] : 1;
    for (int z = 0; z < D3; ++z)
      for (int q = 0; q < c.IS[1]; ++q)
        for (int r = 0; r < c.IS[0]; ++r) {
          const double v = px(im, dtype, (long long)(g.IR_TLF[0] - 1 + r) +
                                             H * ((long long)(g.IR_TLF[1] - 1 + q) + Wd * ((nd == 3 ? g.IR_TLF[2] - 1 : 0) + z)));
          m = v > m ? v : m;
        }
    return m;
  };
  bool skip = false;
  if (mask) {
    if (c.thr > 0) skip = ia_max(img1) < c.thr;
    if (c.mthr > 0) skip = skip || ia_max(mskip ? mskip : mask) < c.mthr;
  } else if (c.thr >= 0) {
    skip = ia_max(img1) < c.thr;
  }
  if (skip) {
    for (int d = 0; d < nd; ++d) VF[nd * ia + d] = 0.0;
    if (SN) SN[ia] = 0.0;
    if (diag) diag[MQP_CPU_DIAG * ia + 4] = 1.0;
    return;
  }
  double sumF2 = 0.0;
  fill_pads(c, g, img1, img2, mask, dtype, w, sumF2);
  const int P0 = c.P[0], P1 = c.P[1], P2 = nd == 3 ? c.P[2] : 1;
  std::vector<double>& cc = w.cc;
  if (mask) {
    // masked NSQECC (src/crosscorrelation_algorithms/mask_nsqecc.jl:126-160)
    w.pad4.resize(w.padG.size());
    for (size_t i = 0; i < w.padG.size(); ++i) w.pad4[i] = w.padG[i] * w.padG[i];
    corr2(pl, w.padF, w.padG, w, w.cc);
    corr2(pl, w.pad3, w.pad4, w, w.cc2);
  } else {
    if (c.alg != MQP_FFTCC) window_sums(c, w.padG, w.integ, w.cc2);
    corr2(pl, w.padF, w.padG, w, w.cc);
  }
  // fully-overlapping similarity block
  std::vector<double> sim((size_t)P0 * P1 * P2);
  for (int z = 0; z < P2; ++z)
    for (int q = 0; q < P1; ++q)
      for (int r = 0; r < P0; ++r) {
        const size_t k = (size_t)r + (size_t)P0 * (q + (size_t)P1 * z);
        const double v = cc[cidx(c.cs, r, q, z)];
        double s;
        if (mask) {
          const double c2 = w.cc2[cidx(c.cs, r, q, z)];
          double num = v * -2.0;
          num += sumF2;
          num += c2;
          const double den = sqrt(fabs(c2)) * sqrt(sumF2);
          s = den / (num + den);
        } else if (c.alg == MQP_FFTCC) {
          s = v;
        } else if (c.alg == MQP_NSQECC) {
          double num = v * -2.0;
          num += sumF2;
          num += w.cc2[k];
          const double den = sqrt(w.cc2[k]) * sqrt(sumF2);
          s = den / (num + den);
        } else {
          s = v / (sqrt(w.cc2[k]) * sqrt(sumF2));
        }
        sim[k] = s;
      }
  // first_fullovp_peak (src/utils/common_ops.jl:98-124)
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = d < nd ? g.toff[d] : 0;
    hi[d] = d < nd ? 2 * c.SM[d] - g.boff[d] : 0;
  }
  double best = 0.0;
  int pk[3] = {-1, -1, -1};
  for (int z = lo[2]; z <= hi[2]; ++z)
    for (int q = lo[1]; q <= hi[1]; ++q)
      for (int r = lo[0]; r <= hi[0]; ++r) {
        const double v = sim[(size_t)r + (size_t)P0 * (q + (size_t)P1 * z)];
        if (v > best) {
          best = v;
          pk[0] = r;
          pk[1] = q;
          pk[2] = z;
        }
      }
  auto S = [&](int r, int q, int z) { return sim[(size_t)r + (size_t)P0 * (q + (size_t)P1 * z)]; };
  if (diag) {
    double t1 = -INFINITY, t2 = -INFINITY, sc = 0.0;
    for (int z = lo[2]; z <= hi[2]; ++z)
      for (int q = lo[1]; q <= hi[1]; ++q)
        for (int r = lo[0]; r <= hi[0]; ++r) {
          const double v = S(r, q, z);
          if (!std::isfinite(v)) continue;
          sc = fabs(v) > sc ? fabs(v) : sc;
          if (v > t1) {
            t2 = t1;
            t1 = v;
          } else if (v > t2) {
            t2 = v;
          }
        }
    double* d = diag + MQP_CPU_DIAG * ia;
    d[0] = t1;
    d[1] = t2;
    d[2] = sc;
  }
  double disp[3] = {0, 0, 0};
  if (pk[0] < 0) {
    for (int d = 0; d < nd; ++d) disp[d] = -(double)(c.SM[d] + 1);
  } else {
    bool inside = true;
    for (int d = 0; d < nd; ++d)
      inside = inside && (pk[d] + 1 > 1 + g.toff[d]) && (pk[d] + 1 < 1 + 2 * c.SM[d] - g.boff[d]);
    double ref[3] = {(double)pk[0], (double)pk[1], (double)pk[2]};
    if (inside) {
      double mn = INFINITY;
      const int zlo = nd == 3 ? pk[2] - 1 : 0, zhi = nd == 3 ? pk[2] + 1 : 0;
      for (int z = zlo; z <= zhi; ++z)
        for (int q = pk[1] - 1; q <= pk[1] + 1; ++q)
          for (int r = pk[0] - 1; r <= pk[0] + 1; ++r) {
            const double v = S(r, q, z);
            mn = (v < mn || v != v) ? v : mn;
          }
      const double lmx = log(1 + best - mn);
      for (int d = 0; d < nd; ++d) {
        int a[3] = {pk[0], pk[1], pk[2]}, b[3] = {pk[0], pk[1], pk[2]};
        a[d] -= 1;
        b[d] += 1;
        const double la = log(1 + S(a[0], a[1], a[2]) - mn);
        const double lb = log(1 + S(b[0], b[1], b[2]) - mn);
        ref[d] += (la - lb) / (2 * la - 4 * lmx + 2 * lb);
      }
    }
    for (int d = 0; d < nd; ++d) disp[d] = ref[d] - c.SM[d];
  }
  for (int d = 0; d < nd; ++d) VF[nd * ia + d] = disp[d];
  if (SN) {  // compute_SN (src/utils/piv_ops.jl:336-367), 3D extended
    int shi[3];
    for (int d = 0; d < 3; ++d) shi[d] = d < nd ? 2 * c.SM[d] - 1 - g.boff[d] : 0;
    double mx = -INFINITY, sum = 0.0;
    double len = 1.0;
    for (int d = 0; d < nd; ++d) len *= (double)(shi[d] - lo[d] + 1);
    for (int z = lo[2]; z <= shi[2]; ++z)
      for (int q = lo[1]; q <= shi[1]; ++q)
        for (int r = lo[0]; r <= shi[0]; ++r) {
          const double v = S(r, q, z);
          mx = (v > mx || v != v) ? v : mx;
          sum += v;
        }
    SN[ia] = mx / ((sum - mx) / (len - 1.0));
    if (diag) diag[MQP_CPU_DIAG * ia + 3] = (sum - mx) / (len - 1.0);
  }
}

}  // namespace

static int cpu_piv(const void* img1, const void* img2, const void* mask, const void* mask_skip, int dtype,
                   int ndims, const int64_t dims[3], const mqp_params* p, double* VF, double* SN, int nthreads,
                   int64_t ia_begin, int64_t ia_end, double* diag) {
  if (ndims != 2 && ndims != 3) return MQP_ERR_INVALID;
  if (!p->unpadded) return MQP_ERR_UNSUPPORTED;
  Ctx c;
  c.nd = ndims;
  c.alg = mask ? MQP_MASK_NSQECC : p->corr_alg;
  c.thr = p->threshold;
  c.mthr = p->mask_threshold;
  c.sn = p->computeSN;
  int64_t n_ia = 1;
  for (int d = 0; d < 3; ++d) {
    c.dims[d] = d < ndims ? dims[d] : 1;
    c.IS[d] = d < ndims ? p->interSize[d] : 1;
    c.SM[d] = d < ndims ? p->searchMargin[d] : 0;
    c.st[d] = d < ndims ? (p->has_step ? p->step[d] : p->interSize[d] - p->overlap[d]) : 1;
    c.SS[d] = c.IS[d] + 2 * c.SM[d];
    // compute_csize_and_paddings with the stored flags (src/utils/fft_ops.jl:145-158)
    c.cs[d] = d < ndims ? (p->good_pad ? good_size_real(c.SS[d]) : c.SS[d] + ((c.SS[d] & 1) && p->odd_pad)) : 1;
    c.P[d] = 2 * c.SM[d] + 1;
    if (d < ndims) {
      const int64_t stop = c.dims[d] - c.IS[d] + 1;
      c.vf[d] = stop < 1 ? 0 : (stop - 1) / c.st[d] + 1;
      n_ia *= c.vf[d];
    } else {
      c.vf[d] = 1;
    }
  }
  if (ia_end < 0 || ia_end > n_ia) ia_end = n_ia;
  PlanND pl;
  pl.init(ndims, c.cs);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    Work w;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int64_t ia = ia_begin; ia < ia_end; ++ia)
      ia_piv(c, pl, ia, img1, img2, mask, mask_skip, dtype, VF, p->computeSN ? SN : nullptr, w, diag);
  }
  return MQP_OK;
}

extern "C" __attribute__((visibility("default"))) int mqp_cpu_piv(
    const void* img1, const void* img2, const void* mask, const void* mask_skip, int dtype, int ndims,
    const int64_t dims[3], const mqp_params* p, double* VF, double* SN, int nthreads, int64_t ia_begin,
    int64_t ia_end) {
  return cpu_piv(img1, img2, mask, mask_skip, dtype, ndims, dims, p, VF, SN, nthreads, ia_begin, ia_end, nullptr);
}

// mqp_cpu_piv plus MQP_CPU_DIAG doubles per IA into diag (indexed by the IA's linear index)
extern "C" __attribute__((visibility("default"))) int mqp_cpu_piv_diag(
    const void* img1, const void* img2, const void* mask, const void* mask_skip, int dtype, int ndims,
    const int64_t dims[3], const mqp_params* p, double* VF, double* SN, int nthreads, int64_t ia_begin,
    int64_t ia_end, double* diag) {
  return cpu_piv(img1, img2, mask, mask_skip, dtype, ndims, dims, p, VF, SN, nthreads, ia_begin, ia_end, diag);
}

extern "C" __attribute__((visibility("default"))) int mqp_cpu_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// test hook: one 1-D transform of length n (interleaved re/im doubles)
extern "C" __attribute__((visibility("default"))) int mqp_cpu_fft(int n, int sign, double* io) {
  Plan1D pl;
  pl.init(n);
  std::vector<cd> x(n), w(n);
  for (int i = 0; i < n; ++i) x[i] = cd(io[2 * i], io[2 * i + 1]);
  fft1d(pl, x.data(), w.data(), sign);
  for (int i = 0; i < n; ++i) {
    io[2 * i] = x[i].real();
    io[2 * i + 1] = x[i].imag();
  }
  return 0;
}
