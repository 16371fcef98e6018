// Window staging with the tensor memory accelerator (TMA) for the 2D warp
// kernel: one elected lane copies the next IA's N x N search window of img2
// (the window copy_search_region! takes, src/utils/piv_ops.jl:115-127) into
// the warp's shared memory with cp.async.bulk.tensor, completing on a
// per-warp mbarrier, while the warp still finishes the current IA.  Phase 1
// then reads the rows from shared memory instead of global memory.
//
// The tile is the window's N columns (dim 2) by N + 4 rows (dim 1, the
// contiguous axis): a tiled copy must start the innermost coordinate on a
// 16-byte boundary, so the first row is rounded down to a multiple of four
// FP32 pixels and the row offset (0..3) is applied when reading.  Rows and
// columns outside the image read as zero (the copy's out-of-bounds fill);
// the clipped search region's own bounds are applied on read.  Each copy
// lands in the issuing CTA's own shared memory only, and its tensor map
// covers only this GPU's img2.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace mqp {

// Tile extents of a staged window for FFT length N (FP32 pixels).
template <int N>
struct StageTile {
  static constexpr int ROWS = N + 4;             // dim 1, contiguous in the image
  static constexpr int COLS = N;                 // dim 2
  static constexpr int FLOATS = ROWS * COLS;
  static constexpr unsigned BYTES = FLOATS * 4;  // 17,408 at N = 64
};

// Bounded waits: a copy that has not landed after this many polls raises the
// status flag and the warp reads its windows from global memory from then
// on, instead of hanging.
constexpr int STAGE_WAIT_POLLS = 1 << 22;
// phase value of a warp whose staging is off (after a wait ran out)
constexpr unsigned STAGE_OFF = 0xffffffffu;

// (The bodies are device code only; the host pass sees empty functions.)
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
#if defined(__CUDA_ARCH__)
  return (uint32_t)__cvta_generic_to_shared(p);
#else
  (void)p;
  return 0;
#endif
}

// Called by one lane per warp, then a block barrier before first use.
__device__ __forceinline__ void stage_init(uint64_t* mbar) {
#if defined(__CUDA_ARCH__)
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
#else
  (void)mbar;
#endif
}

// Every lane: its earlier generic accesses to the destination are ordered
// before the copy's asynchronous writes.  Then __syncwarp and stage_issue
// from one lane.
__device__ __forceinline__ void stage_fence() {
#if defined(__CUDA_ARCH__)
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#endif
}

// One lane: arm the mbarrier with the tile's bytes and start the copy of
// the tile whose first element is image (x0, y0) = (row, column), x0 a
// multiple of 4.
template <int N>
__device__ __forceinline__ void stage_issue(const CUtensorMap* tmap, float* dst, uint64_t* mbar, int x0, int y0) {
#if defined(__CUDA_ARCH__)
  const uint32_t b = smem_u32(mbar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(StageTile<N>::BYTES)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"((uint64_t)tmap), "r"(x0), "r"(y0), "r"(b)
      : "memory");
#else
  (void)tmap, (void)dst, (void)mbar, (void)x0, (void)y0;
#endif
}

// Every lane: wait for the phase with the given parity to complete.
__device__ __forceinline__ bool stage_wait(uint64_t* mbar, unsigned parity) {
#if defined(__CUDA_ARCH__)
  const uint32_t b = smem_u32(mbar);
  for (int i = 0; i < STAGE_WAIT_POLLS; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
#else
  (void)mbar, (void)parity;
  return true;
#endif
}

// The tile's first row for a window whose pad row 0 is image row g01.
__host__ __device__ __forceinline__ int stage_x0(int g01) { return g01 & ~3; }

}  // namespace mqp
