// Failure-detection self-test: a kernel whose mbarrier wait can never
// complete (nothing arrives), so the product's bounded wait runs out, records
// kErrWaitTimeout in the device error word and returns.  The host then reads
// CCT_ETIMEOUT from cct_device_status() and the context stays usable.  This
// is the device half of the reference's failure surfacing, where a kernel
// error becomes a CLEvent status and a RuntimeException
// (src/main/scala/cogx/platform/opencl/OpenCLDeviceKernel.scala:106-147).
#include <chrono>

#include "cct_internal.h"
#include "sm100_util.cuh"

namespace cct {
namespace {

__global__ void wait_never_arrives(unsigned *err, unsigned *waited) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival expected; none is ever made
    fence_barrier_init();
  }
  __syncthreads();
  const bool ok = mbar_wait(&bar, 0, err);
  if (threadIdx.x == 0) *waited = ok ? 0u : 1u;
}

}  // namespace
}  // namespace cct

using namespace cct;

extern "C" int cct_selftest_wait_timeout(double *elapsed_ms) {
  unsigned *err = device_error_word();
  if (!err) return set_error(CCT_ENODEV, "no device error word");
  unsigned *waited = nullptr;
  int rc = check_cuda(cudaMalloc(&waited, sizeof(unsigned)), "cudaMalloc(selftest)");
  if (rc) return rc;
  const auto t0 = std::chrono::steady_clock::now();
  wait_never_arrives<<<1, 32>>>(err, waited);
  count_launches(1);
  rc = check_cuda(cudaGetLastError(), "selftest launch");
  if (!rc) rc = check_cuda(cudaDeviceSynchronize(), "selftest synchronise");
  const auto t1 = std::chrono::steady_clock::now();
  unsigned w = 0;
  if (!rc) rc = check_cuda(cudaMemcpy(&w, waited, sizeof(w), cudaMemcpyDeviceToHost), "selftest result");
  cudaFree(waited);
  if (elapsed_ms) *elapsed_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  if (!rc && w != 1) rc = set_error(CCT_ECUDA, "selftest wait completed without an arrival");
  return rc;
}
