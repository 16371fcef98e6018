// Register-resident complex FFTs for one thread (sm_100a device code, also
// compiled for the host so the same code can be exercised without a GPU).
//
// A length-N transform lives in a thread's registers as float2 x[N]; every
// loop is fully unrolled, so all indices, twiddles and zero-skips are
// compile-time constants and x never touches local memory.  The algorithm
// is in-place decimation-in-frequency with radix-4 butterflies (plus one
// radix-2 stage when log2 N is odd).  Input is in natural order; frequency k
// ends up in slot fpos<N>(k) (a digit reversal), which callers resolve at
// compile time instead of permuting.
//
// Transforms are unnormalised: forward uses exp(-2*pi*i*nk/N), inverse
// exp(+2*pi*i*nk/N).
#pragma once

#include <cuda_runtime.h>

#if defined(__CUDACC__)
#define MQP_HD __host__ __device__
#define MQP_FI __forceinline__
#else
#define MQP_HD
#define MQP_FI inline
#endif

namespace mqp {

// An empty asm statement with a memory clobber: memory operations cannot
// move across it (loads before it are issued before it, loads after it stay
// after it).
MQP_HD MQP_FI void mqp_no_hoist() {
#if defined(__CUDA_ARCH__)
  asm volatile("" ::: "memory");
#endif
}

constexpr int TW_N = 256;  // twiddle table resolution: exp(2*pi*i*m/256)

// {cos, sin}(2*pi*m/256).  Each translation unit gets its own 2 KB copy
// (device variables cannot be shared across units without relocatable
// device code).
#if defined(__CUDACC__)
static __constant__ float2 c_twiddle[TW_N] = {
#include "mqp_twiddles.inc"
};
#endif
static const float2 h_twiddle[TW_N] = {
#include "mqp_twiddles.inc"
};

// (cos, sin)(2*pi*m/256) for an index that is a compile-time constant once
// the caller is inlined and unrolled (every twiddle of the register FFTs):
// the table is a constant expression, so each use folds to immediate
// operands.  Read from the __constant__ table instead, the twiddles of an
// unrolled transform were hoisted into registers ahead of use and spilled.
// A runtime index would build the table per thread: use twiddle_rt.
MQP_HD MQP_FI float2 twiddle_cs(int m) {
  constexpr float2 t[TW_N] = {
#include "mqp_twiddles.inc"
  };
  return t[m & (TW_N - 1)];
}

// (cos, sin)(2*pi*m/256) for a runtime index (table set-up loops)
MQP_HD MQP_FI float2 twiddle_rt(int m) {
#if defined(__CUDA_ARCH__)
  return c_twiddle[m & (TW_N - 1)];
#else
  return h_twiddle[m & (TW_N - 1)];
#endif
}

MQP_HD MQP_FI float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
MQP_HD MQP_FI float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
MQP_HD MQP_FI float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// a * (-i)
MQP_HD MQP_FI float2 cmul_mi(float2 a) { return make_float2(a.y, -a.x); }
// a * (+i)
MQP_HD MQP_FI float2 cmul_pi(float2 a) { return make_float2(-a.y, a.x); }
MQP_HD MQP_FI float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
MQP_HD MQP_FI float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
MQP_HD MQP_FI float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// a * exp(sign * 2*pi*i * m / L), sign = -1 forward, +1 inverse.  Multiples
// of a quarter or an eighth turn take their exact short forms.
template <int L, bool INV>
MQP_HD MQP_FI float2 rotate(float2 a, int m) {
  static_assert(TW_N % L == 0, "twiddle table too coarse");
  const int t = (m * (TW_N / L)) & (TW_N - 1);  // in 1/256 turns
  if (t == 0) return a;
  if (t == TW_N / 2) return make_float2(-a.x, -a.y);
  if (t == TW_N / 4) return INV ? cmul_pi(a) : cmul_mi(a);
  if (t == 3 * TW_N / 4) return INV ? cmul_mi(a) : cmul_pi(a);
  const float2 cs = twiddle_cs(t);
  // forward: (c - i s); inverse: (c + i s)
  const float s = INV ? cs.y : -cs.y;
  if (t == TW_N / 8 || t == 3 * TW_N / 8 || t == 5 * TW_N / 8 || t == 7 * TW_N / 8) {
    // |c| == |s| == sqrt(1/2): (a.x c - a.y s, a.x s + a.y c) with one multiply each
    const float h = cs.x;  // +-sqrt(1/2)
    const float sg = (s * h > 0.f) ? 1.f : -1.f;  // s == sg * h
    return make_float2((a.x - sg * a.y) * h, (sg * a.x + a.y) * h);
  }
  return make_float2(a.x * cs.x - a.y * s, a.x * s + a.y * cs.x);
}

// ---- digit-reversed output positions --------------------------------------
MQP_HD constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

// Slot of frequency k after the DIF transform of length N (radix-4 stages
// while the remaining span is >= 4, then one radix-2 stage if log2 N is
// odd): the base-4 digits of k reversed, i.e. the closed form of
//   pos_L(k) = (k % 4) * (L / 4) + pos_{L/4}(k / 4),  pos_2(k) = k, pos_1 = 0.
// Kept loop-based (not recursive) so it folds to a constant when k is one.
template <int N>
MQP_HD MQP_FI constexpr int fpos(int k) {
  constexpr int LG = ilog2c(N);
  constexpr int R = LG / 2;
  int p = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) p += ((k >> (2 * i)) & 3) * (N >> (2 * i + 2));
  if (LG & 1) p += (k >> (2 * R));
  return p;
}

// ---- one DIF stage ---------------------------------------------------------
// x: register array of the whole transform; blocks of span L, each split in 4
// quarters of Q = L/4.  NZ = number of leading input elements that may be
// non-zero in the FIRST stage (the rest are known zeros and are skipped).
template <int N, bool INV, int L, int NZ>
MQP_HD MQP_FI void dif_stage4(float2 (&x)[N]) {
  constexpr int Q = L / 4;
#pragma unroll
  for (int b = 0; b < N / L; ++b) {
#pragma unroll
    for (int j = 0; j < Q; ++j) {
      const int i0 = b * L + j, i1 = i0 + Q, i2 = i0 + 2 * Q, i3 = i0 + 3 * Q;
      const bool z1 = (L == N) && (j + Q >= NZ);
      const bool z2 = (L == N) && (j + 2 * Q >= NZ);
      const bool z3 = (L == N) && (j + 3 * Q >= NZ);
      const float2 a0 = x[i0];
      float2 y0, y1, y2, y3;
      if (z1) {  // only a0 non-zero
        y0 = a0; y1 = a0; y2 = a0; y3 = a0;
      } else if (z2) {  // a0, a1
        const float2 a1 = x[i1];
        y0 = cadd(a0, a1);
        y2 = csub(a0, a1);
        y1 = INV ? cadd(a0, cmul_pi(a1)) : cadd(a0, cmul_mi(a1));
        y3 = INV ? cadd(a0, cmul_mi(a1)) : cadd(a0, cmul_pi(a1));
      } else {
        const float2 a1 = x[i1], a2 = x[i2];
        const float2 a3 = z3 ? make_float2(0.f, 0.f) : x[i3];
        const float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
        const float2 s13 = z3 ? a1 : cadd(a1, a3);
        const float2 d13 = z3 ? a1 : csub(a1, a3);
        y0 = cadd(s02, s13);
        y2 = csub(s02, s13);
        // forward: y1 = d02 - i d13, y3 = d02 + i d13 ; inverse swaps the signs
        y1 = INV ? cadd(d02, cmul_pi(d13)) : cadd(d02, cmul_mi(d13));
        y3 = INV ? cadd(d02, cmul_mi(d13)) : cadd(d02, cmul_pi(d13));
      }
      x[i0] = y0;
      x[i1] = rotate<L, INV>(y1, j);
      x[i2] = rotate<L, INV>(y2, 2 * j);
      x[i3] = rotate<L, INV>(y3, 3 * j);
    }
  }
}

template <int N, int L, int NZ>
MQP_HD MQP_FI void dif_stage2(float2 (&x)[N]) {
  static_assert(L == 2, "radix-2 stage is only used last");
#pragma unroll
  for (int b = 0; b < N / 2; ++b) {
    const float2 a0 = x[2 * b], a1 = x[2 * b + 1];
    if ((L == N) && NZ <= 1) {
      x[2 * b + 1] = a0;
    } else {
      x[2 * b] = cadd(a0, a1);
      x[2 * b + 1] = csub(a0, a1);
    }
  }
}

template <int N, bool INV, int L, int NZ>
struct DifRec {
  MQP_HD MQP_FI static void run(float2 (&x)[N]) {
    if constexpr (L >= 4) {
      dif_stage4<N, INV, L, NZ>(x);
      DifRec<N, INV, L / 4, NZ>::run(x);
    } else if constexpr (L == 2) {
      dif_stage2<N, 2, NZ>(x);
    }
  }
};

// In-place FFT of length N (power of two, 2..256) held in registers.
// NZ: the inputs x[NZ..N) are known to be zero (NZ in {N, N/2, N/4}).
template <int N, bool INV, int NZ = N>
MQP_HD MQP_FI void fft_reg(float2 (&x)[N]) {
  static_assert((N & (N - 1)) == 0 && N >= 2 && N <= TW_N, "N must be a power of two <= 256");
  static_assert(NZ == N || NZ == N / 2 || NZ == N / 4, "NZ must be N, N/2 or N/4");
  DifRec<N, INV, N, NZ>::run(x);
}

}  // namespace mqp
