// Internal interface between the C ABI (mqp_abi.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "mqp_piv2d.cuh"

namespace mqp {

// FP64 exclusive-prefix integral image of img (or img^2) for a column-major
// H x W image: out is (H+1) x (W+1), first row/column zero.  scratch holds
// integral2d_scratch_bytes(H, W) bytes of per-chunk totals.
cudaError_t launch_integral2d(const void* img, int dtype, int H, int W, bool square,
                              double* out, double* scratch, cudaStream_t s);
size_t integral2d_scratch_bytes(int H, int W);

// Smallest supported power-of-two FFT length covering the search window,
// or 0 when the window is too large for the fused 2D kernel.
int piv2d_fft_len(int SS1, int SS2);

// Launch the fused 2D kernel over [a.ia_begin, a.ia_end).  `alg` picks the
// similarity; returns cudaSuccess or the launch error (err filled).
cudaError_t launch_piv2d(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err);

int device_sm_count(int device);

}  // namespace mqp
