// Allocation-free entry point: the fused filter-bank convolution on the
// tensor cores (split BF16), with its scratch memory in a fixed device array.
//
// Who needs this.  A plan (cct_conv_plan_create) allocates its workspace with
// cudaMalloc.  Some callers cannot do that at the moment they want to
// convolve:
//  - hosts that reserve all device memory up front in their own arena (the
//    reference runtime pre-plans every field buffer; a serving process that
//    admits work by free HBM must not see hidden allocations);
//  - latency-sensitive callers: cudaMalloc and cudaFree may synchronise the
//    device and stall every stream, not just the caller's.
// Those callers pass device pointers for the image, filter and output; the
// only scratch, the packed bf16 hi/lo filter operand, lives in the
// file-scope array below.
//
// Failure reporting: the kernel's bounded waits record a timeout in the
// library's device error word, which is itself a statically allocated device
// word (nothing allocates it), the same word every plan's kernels use.  It
// is not cleared per call: a timeout stays recorded until cct_device_status()
// reads and clears it.
//
// Limits and sharing:
//  - the packed filter operand must fit in kNoAllocScratchBytes (4 MiB);
//    larger filter banks are rejected with CCT_EINVAL and a message;
//  - every GPU that loads this library holds the array until the process
//    exits;
//  - all calls on a device share the array and it keeps the last call's
//    contents: each call rewrites the whole packed operand it uses, so
//    nothing stale is read, but calls that overlap on the GPU (different
//    streams, no ordering between them) race on it;
//  - the array's device address (and the error word's) is looked up on the
//    first call on each device and cached for the life of the CUDA context:
//    make that first call before any stream capture, and not across a
//    cudaDeviceReset.
#include <mutex>

#include "bank_tc.h"
#include "cct_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;  // packed filter operand limit

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
uint8_t *g_noalloc_addr[64];  // device address of g_noalloc_scratch, per device

// Set-up, once per device, with that device current: the array's name is a
// host-side stand-in, so its device address must be looked up.
int scratch_address(int dev, uint8_t **out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return cct::set_error(CCT_ECUDA, "cudaGetSymbolAddress(no-alloc scratch): %s",
                            cudaGetErrorString(e));
    g_noalloc_addr[dev] = static_cast<uint8_t *>(p);
  }
  *out = g_noalloc_addr[dev];
  return CCT_OK;
}

}  // namespace

extern "C" int cct_conv_run_noalloc(const cct_conv_desc *desc, const float *image,
                                    const float *filter, float *out, void *stream) {
  using namespace cct;
  ConvGeom g;
  int rc = resolve_geom(desc, &g);
  if (rc) return rc;
  if (!image || !filter || !out) return set_error(CCT_EINVAL, "null image, filter or output pointer");
  if (desc->precision != CCT_PREC_BF16X3 ||
      (g.mode != CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM && g.mode != CCT_BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM))
    return set_error(CCT_ENOTSUP,
                     "the allocation-free entry point runs the BF16X3 BlockReduceSum frame kernel only");

  int dev = 0, major = 0, sms = 0;
  rc = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= 64) return set_error(CCT_ENODEV, "device index %d out of range", dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) return set_error(CCT_ENODEV, "device %d is not sm_100 (major %d)", dev, major);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

  FrameTcChoice tc;  // the same kernel and tile plan a plan for this descriptor runs
  if (!frame_tc_choose(g, CCT_PREC_BF16X3, sms, &tc))
    return set_error(CCT_ENOTSUP, "shape outside the tensor-core frame kernels (sampling or tile size)");
  if (tc.pack_bytes > kNoAllocScratchBytes)
    return set_error(CCT_EINVAL,
                     "packed filter operand needs %zu bytes; the allocation-free entry point holds "
                     "at most %zu",
                     tc.pack_bytes, kNoAllocScratchBytes);

  uint8_t *scratch = nullptr;
  rc = scratch_address(dev, &scratch);
  if (rc) return rc;
  unsigned *status = device_error_word();
  if (!status) return set_error(CCT_ECUDA, "device error word: symbol address lookup failed");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  rc = frame_tc_pack(tc, filter, scratch, st);
  if (rc) return rc;
  return frame_tc_run(tc, image, out, scratch, status, st, true);
}
