// Internal interface between the C ABI (mqp_abi.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "mqp_piv2d.cuh"
#include "mqp_piv3d.cuh"
#include "mqp_multipass.cuh"
#include "mqp_deform.cuh"
#include "mqp_post.cuh"
#include "mqp_direct.cuh"

namespace mqp {

// FP64 exclusive-prefix integral image of img (or img^2) for a column-major
// H x W image: out is (H+1) x (W+1), first row/column zero.  scratch holds
// integral2d_scratch_bytes(H, W) bytes of per-chunk totals.
cudaError_t launch_integral2d(const void* img, int dtype, int H, int W, bool square,
                              double* out, double* scratch, cudaStream_t s);
// the integral columns of image columns [x0, x1) (x0 a multiple of 64, x1 one
// or W) after those of columns < x0: a piece of launch_integral2d's result
cudaError_t launch_integral2d_cols(const void* img, int dtype, int H, int W, int x0, int x1, bool square,
                                   double* out, double* scratch, cudaStream_t s);
size_t integral2d_scratch_bytes(int H, int W);

// The same for a column-major H x W x D volume: out is (H+1) x (W+1) x (D+1),
// first plane zero; scratch holds integral3d_scratch_bytes(H, W, D) bytes.
cudaError_t launch_integral3d(const void* img, int dtype, int H, int W, int D, bool square,
                              double* out, double* scratch, cudaStream_t s);
size_t integral3d_scratch_bytes(int H, int W, int D);

// Smallest supported power-of-two FFT length covering the search window
// (32, 64: the warp kernel; 128: the block kernel), or 0 when too large.
int piv2d_fft_len(int SS1, int SS2);

// Launch the fused 2D kernel over [a.ia_begin, a.ia_end).  `alg` picks the
// similarity; returns cudaSuccess or the launch error (err filled).
cudaError_t launch_piv2d(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err);

int device_sm_count(int device);

// One persistent launch of the fused 2D kernel over the IAs of many image
// pairs that share a kernel variant (N, prune, alg, dtype): items[k] (device
// array) is pair k's arguments, prefix[k] the first work-queue index of its
// IAs (n_items + 1 entries, prefix[n_items] = total).  wf2 is the per-warp
// workspace (piv2d_warp_f2) of the largest lag plane among the items;
// counter is one device word the launch resets and uses as the queue head;
// grab is the queue entries a warp takes at once.
struct Piv2dBatch {
  const Piv2dArgs* items;
  const long long* prefix;
  int n_items;
  long long total;
  int N;
  bool prune;
  int alg;
  int dtype;
  int wf2;
  int grab;
  unsigned long long* counter;
  bool lw;  // every item forms its window sums on chip (piv2d_local_sums)
};
int piv2d_warp_f2(int N, bool prune, int P1, int P2, bool masked);
int piv2d_warp_f2_lw(int N, int P1, int P2);
cudaError_t launch_piv2d_batch(const Piv2dBatch& b, cudaStream_t s, std::string& err);

// Search windows of 129..256 (FFT length 256, interrogation windows up to
// 128, FFTCC / ZNCC / NSQECC): one 256-thread block per IA over a scratch
// slot per resident block (mqp_piv2d_huge.cu); a.huge must point at
// piv2d_huge_scratch_bytes(device, P1, P2) bytes.
bool piv2d_huge_ok(int SS1, int SS2, int IS1, int IS2, int alg);
// ZNCC passes whose kernel forms the window sums on chip: they need no
// integral image of img2^2 (mqp_piv2d.cu).
bool piv2d_local_sums(int IS1, int IS2, int SM1, int SM2, int alg);
size_t piv2d_huge_scratch_bytes(int device, int P1, int P2);
cudaError_t launch_piv2d_huge(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err);

// Team variant of the fused 2D kernel (mqp_piv2d_team.cu): one IA per team
// of N threads for FFT lengths 32 and 64 with pruned F (interrogation window
// up to N/2) and FFTCC / ZNCC / NSQECC.  piv2d_team_ok says whether a variant
// runs on it (launch_piv2d and launch_piv2d_batch then route there);
// piv2d_team_f2 is a team's workspace (float2 units), which piv2d_warp_f2
// returns for those variants.
bool piv2d_team_ok(int N, bool prune, int alg);
int piv2d_team_f2(int N, int P1, int P2);
cudaError_t launch_piv2d_team(const Piv2dArgs& a, int N, int alg, cudaStream_t s, std::string& err);
cudaError_t launch_piv2d_team_batch(const Piv2dBatch& b, cudaStream_t s, std::string& err);

// Small windows (direct2d_ok / direct3d_ok): spatial correlation, one warp
// per IA (mqp_direct.cu).  Batch plans mark these groups with N = 1; their
// Piv2dBatch::wf2 is half the per-warp word count (piv2d_direct_words).
int piv2d_direct_words(int IS1, int IS2, int SM1, int SM2);
cudaError_t launch_piv2d_direct(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err);
cudaError_t launch_piv2d_direct_batch(const Piv2dBatch& b, cudaStream_t s, std::string& err);
cudaError_t launch_piv3d_direct(const Piv3dArgs& a, int alg, cudaStream_t s, std::string& err);

// Search windows 65..128 (FFT length 128): one 128-thread block per IA
// (mqp_piv2d_big.cu); for these, Piv2dBatch::wf2 is the block's whole
// workspace (piv2d_warp_f2 with N = 128).
int piv2d_big_warp_f2(bool prune, int P1, int P2, bool masked);
cudaError_t launch_piv2d_big(const Piv2dArgs& a, int alg, cudaStream_t s, std::string& err);
cudaError_t launch_piv2d_big_batch(const Piv2dBatch& b, cudaStream_t s, std::string& err);

// 3D path: cubic FFT length for the search window (0 = unsupported), chunk
// scratch bytes per IA, and the three-kernel launch over [a.ia_begin,
// a.ia_end) in chunks of `chunk` IAs (the scratch pointers of `a` must hold
// chunk IAs).
int piv3d_fft_len(const int SS[3]);
size_t piv3d_scratch_bytes_per_ia(const int IS[3], const int SM[3], int alg);
// chunk scratch of the 3D kernels for `chunk` IAs, and Piv3dArgs' scratch
// pointers bound into it (a.IS / a.SM set)
size_t piv3d_scratch_bytes(const int IS[3], const int SM[3], int alg, long long chunk);
void piv3d_bind_scratch(Piv3dArgs& a, int alg, long long chunk, char* base);
cudaError_t launch_piv3d(const Piv3dArgs& a, int alg, long long chunk, cudaStream_t s, std::string& err);

// Multi-pass refinement: the fine pass's predictor from the coarse vectors.
cudaError_t launch_predictor(const PredArgs& a, cudaStream_t s);
// Deforming refinement: both images resampled around the dense predictor
// (a.out1/out2), and the predictor added back to the fine pass's vectors.
cudaError_t launch_deform(const DeformArgs& a, cudaStream_t s);
cudaError_t launch_deform_add(const DeformArgs& a, cudaStream_t s);

// Vector-field post-processing (one op); scratch holds post_scratch_bytes().
cudaError_t launch_post(const PostArgs& a, double* scratch, cudaStream_t s);
size_t post_scratch_bytes();

}  // namespace mqp
