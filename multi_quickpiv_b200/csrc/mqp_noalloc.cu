// Allocation-free 2D PIV on device-resident arrays (mqp_piv2d_noalloc).
//
// Some callers cannot allocate GPU memory at the moment they want a vector
// field: code running inside a framework that owns all device memory through
// its own pool (and forbids side allocations), real-time loops that must not
// hit cudaMalloc's implicit synchronisation or its failure modes mid-run, and
// hosts that pre-plan every byte of a device budget up front.  For them this
// entry point does the same 2D work as mqp_piv_device without creating a
// context and without allocating: the only memory beyond the caller's inputs
// and outputs is the file-scope scratch array below, whose size is fixed when
// the library is built.
//
// What the scratch holds: the FP64 integral images the ZNCC and NSQECC
// normalisations need ((H+1) x (W+1) doubles: one for NSQECC, three for ZNCC,
// none for FFTCC) and the per-chunk totals of their row scan.  The scan
// kernels write every element they later read, so nothing needs clearing
// between calls.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <string>

#include "mqp.h"
#include "mqp_internal.h"

namespace {

// The scratch array.  Every GPU that loads this library's module holds it
// (MQP_NOALLOC_SCRATCH_BYTES bytes) until the process exits.  In host code its
// name is only a host-side stand-in for the device symbol: the device address
// must come from cudaGetSymbolAddress with the device current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MQP_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

int report(char* err, int errlen, int code, const std::string& msg) {
  if (err && errlen > 0) {
    snprintf(err, (size_t)errlen, "%s", msg.c_str());
  }
  return code;
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

extern "C" int mqp_piv2d_noalloc(const void* d_img1, const void* d_img2, int dtype, const int64_t dims[2],
                                 const mqp_params* p, double* d_VF, double* d_SN, void* stream, char* err,
                                 int errlen) {
  if (err && errlen > 0) err[0] = '\0';
  if (!p || !dims || !d_img1 || !d_img2) return report(err, errlen, MQP_ERR_INVALID, "null argument");
  if (dtype != MQP_F32 && dtype != MQP_F64) return report(err, errlen, MQP_ERR_INVALID, "dtype must be MQP_F32 or MQP_F64");
  if (!p->unpadded)
    return report(err, errlen, MQP_ERR_UNSUPPORTED,
                  "ERROR: all gaussian_displacement should be unpadded (stored unpadded must be true)");
  if (p->multipass < 1) return report(err, errlen, MQP_ERR_INVALID, "multipass must be >= 1");
  // the refinement passes keep predictor and coarse vector fields between
  // passes, which this entry point has no memory for
  if (p->refine && p->multipass > 1)
    return report(err, errlen, MQP_ERR_UNSUPPORTED,
                  "multi-pass refinement (refine with multipass > 1) needs per-pass buffers; use mqp_piv_device");
  if (p->corr_alg < MQP_FFTCC || p->corr_alg > MQP_NSQECC)
    return report(err, errlen, MQP_ERR_INVALID, "corr_alg must be MQP_FFTCC, MQP_ZNCC or MQP_NSQECC");
  if (dims[0] < 1 || dims[1] < 1 || dims[0] > (1 << 30) || dims[1] > (1 << 30))
    return report(err, errlen, MQP_ERR_INVALID, "image extents must be in [1, 2^30]");
  const int H = (int)dims[0], W = (int)dims[1];
  int IS[2], SM[2], st[2];
  long long vf[2];
  for (int d = 0; d < 2; ++d) {
    IS[d] = p->interSize[d];
    SM[d] = p->searchMargin[d];
    st[d] = p->has_step ? p->step[d] : p->interSize[d] - p->overlap[d];
    if (IS[d] < 1 || SM[d] < 0 || st[d] < 1)
      return report(err, errlen, MQP_ERR_INVALID, "interSize >= 1, searchMargin >= 0 and step >= 1 are required");
    const long long stop = (long long)dims[d] - IS[d] + 1;
    vf[d] = stop < 1 ? 0 : (stop - 1) / st[d] + 1;
  }
  if (mqp::piv2d_fft_len(IS[0] + 2 * SM[0], IS[1] + 2 * SM[1]) == 0)
    return report(err, errlen, MQP_ERR_UNSUPPORTED, "2D search window (interSize + 2 searchMargin) above 128");
  if (vf[0] * vf[1] == 0) return MQP_OK;  // empty vector field: nothing to write (VF may have no address)
  if (!d_VF) return report(err, errlen, MQP_ERR_INVALID, "null VF pointer");

  // scratch plan: [II of img2^2 | II of img2 | II of img1 | scan totals]
  const int n_ii = p->corr_alg == MQP_NSQECC ? 1 : (p->corr_alg == MQP_ZNCC ? 3 : 0);
  const size_t ii_bytes = align256((size_t)(H + 1) * (size_t)(W + 1) * sizeof(double));
  const size_t tot_bytes = n_ii ? align256(mqp::integral2d_scratch_bytes(H, W)) : 0;
  const size_t need = (size_t)n_ii * ii_bytes + tot_bytes;
  if (need > (size_t)MQP_NOALLOC_SCRATCH_BYTES)
    return report(err, errlen, MQP_ERR_INVALID,
                  "image needs " + std::to_string(need) + " bytes of scratch, above the " +
                      std::to_string((size_t)MQP_NOALLOC_SCRATCH_BYTES) +
                      " bytes built into mqp_piv2d_noalloc (MQP_NOALLOC_SCRATCH_BYTES); use mqp_piv_device");

  // The device address of the scratch array, with the device current.  The
  // first call on a device looks it up; later calls look it up again unless
  // their stream is capturing (a module reloaded after cudaDeviceReset can
  // place the array elsewhere), and a capturing call uses the address cached
  // by an earlier call on the device, so make one call before any capture.
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return report(err, errlen, MQP_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  cudaStream_t s = stream ? (cudaStream_t)stream : cudaStreamLegacy;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();  // clear the query's error; treat the stream as capturing
    cap = cudaStreamCaptureStatusActive;
  }
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (cap == cudaStreamCaptureStatusNone || !g_scratch_addr[dev]) {
      if (cap != cudaStreamCaptureStatusNone)
        return report(err, errlen, MQP_ERR_INVALID,
                      "the first call on a device must come before any stream capture (it looks up the scratch "
                      "array's address)");
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr)
        return report(err, errlen, MQP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch_addr[dev] = ptr;
    }
    base = static_cast<unsigned char*>(g_scratch_addr[dev]);
  }

  double* IIg2 = n_ii >= 1 ? reinterpret_cast<double*>(base) : nullptr;
  double* IIg = n_ii >= 3 ? reinterpret_cast<double*>(base + ii_bytes) : nullptr;
  double* II1 = n_ii >= 3 ? reinterpret_cast<double*>(base + 2 * ii_bytes) : nullptr;
  double* totals = n_ii ? reinterpret_cast<double*>(base + (size_t)n_ii * ii_bytes) : nullptr;
  if (IIg2 && (e = mqp::launch_integral2d(d_img2, dtype, H, W, true, IIg2, totals, s)) != cudaSuccess)
    return report(err, errlen, MQP_ERR_CUDA, std::string("integral image: ") + cudaGetErrorString(e));
  if (IIg && (e = mqp::launch_integral2d(d_img2, dtype, H, W, false, IIg, totals, s)) != cudaSuccess)
    return report(err, errlen, MQP_ERR_CUDA, std::string("integral image: ") + cudaGetErrorString(e));
  if (II1 && (e = mqp::launch_integral2d(d_img1, dtype, H, W, false, II1, totals, s)) != cudaSuccess)
    return report(err, errlen, MQP_ERR_CUDA, std::string("integral image: ") + cudaGetErrorString(e));

  mqp::Piv2dArgs a;
  memset(&a, 0, sizeof(a));
  a.img1 = d_img1;
  a.img2 = d_img2;
  a.dtype = dtype;
  a.II1 = II1;
  a.IIg = IIg;
  a.IIg2 = IIg2;
  a.VF = d_VF;
  a.SN = p->computeSN ? d_SN : nullptr;
  a.H = H;
  a.W = W;
  a.IS1 = IS[0];
  a.IS2 = IS[1];
  a.SM1 = SM[0];
  a.SM2 = SM[1];
  a.st1 = st[0];
  a.st2 = st[1];
  a.vf1 = (int)vf[0];
  a.vf2 = (int)vf[1];
  a.ia_begin = 0;
  a.ia_end = vf[0] * vf[1];
  a.threshold = p->threshold;
  a.mask_threshold = p->mask_threshold;
  a.computeSN = a.SN != nullptr;
  std::string msg;
  e = mqp::launch_piv2d(a, p->corr_alg, s, msg);
  if (e != cudaSuccess) return report(err, errlen, MQP_ERR_CUDA, msg);
  return MQP_OK;
}
