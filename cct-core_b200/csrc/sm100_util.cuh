// sm_100a device utilities: mbarriers with bounded waits, TMA tile loads,
// a device-side error word, and the host-side tensor-map encoder.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cct {

// Device error word (one per device, allocated by the library and passed to
// kernels): bit 0 = a bounded wait gave up.  Read and cleared by
// cct_device_status().
constexpr unsigned kErrWaitTimeout = 1u;

// Upper bound on mbarrier polls before a wait gives up.  Each try_wait
// suspends for up to the hardware's time limit, so this is seconds of
// waiting -- only reachable if a copy never lands.
constexpr uint32_t kMaxWaitPolls = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

// Returns true when the phase with the given parity has completed; false if
// the poll budget ran out (the error word is set).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned *err) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t i = 0; i < kMaxWaitPolls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  atomicOr(err, kErrWaitTimeout);
  return false;
}

// 3-D tiled TMA load (x innermost) into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// Host: encode a 3-D fp32 tensor map (cols, rows, planes) with the given box;
// out-of-bounds elements read as zero.  Returns CCT_OK or an error status.
int encode_tensor_map_3d(CUtensorMap *map, const float *base, uint64_t cols, uint64_t rows,
                         uint64_t planes, uint32_t box_c, uint32_t box_r);

}  // namespace cct
