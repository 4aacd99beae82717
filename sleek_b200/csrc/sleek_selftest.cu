// sleek_selftest.cu -- exercises the codec kernels' bounded waits on the device
// without faulting or hanging it: one CTA waits on an mbarrier that nothing
// arrives on, and one warp looks back over a predecessor flag that nothing
// publishes, each with a caller-given limit, using the same wait helpers as the
// encode and decode kernels (sleek_device.cuh).  Both must give up, report it,
// and return; the context stays usable.
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/sleek_capi.h"
#include "sleek_device.cuh"

namespace sleek {
namespace {

// result[0]: 1 if the mbarrier wait gave up; result[1]: the look-back's return
// value (-1 when it gave up); result[2]: nanoseconds the two waits took
__global__ void __launch_bounds__(32) k_selftest_waits(unsigned long long limit_ns, uint64_t* flags, long long* result)
{
  __shared__ __align__(8) uint64_t bar;
  const int lane = threadIdx.x;
  if (lane == 0) {
    mbar_init(&bar, 1);  // expects one arrival, which never comes
    mbar_fence_init();
  }
  __syncwarp();
  const unsigned long long t0 = globaltimer_ns();
  const bool got = mbar_wait_bounded(&bar, 0, limit_ns);
  // flags[0] is the unpublished predecessor of item 1; flags[2..] hold the
  // workspace header the look-back reads for errors (status word 0: none)
  const long long lb = lookback(flags + 2 + WS_HDR_WORDS, 1, 0, flags + 2, limit_ns);
  const unsigned long long t1 = globaltimer_ns();
  if (lane == 0) {
    result[0] = got ? 0 : 1;
    result[1] = lb;
    result[2] = static_cast<long long>(t1 - t0);
  }
}

}  // namespace
}  // namespace sleek

extern "C" int sleek_selftest_bounded_waits(long long limit_ns, long long* h_result)
{
  if (!h_result || limit_ns <= 0 || limit_ns > 10000000000ll) return SLEEK_ERR_INVALID_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  // [0..1] spare, [2..33] a zeroed workspace header, [34] the flag nobody sets
  const size_t words = 2 + sleek::WS_HDR_WORDS + 1;
  uint64_t* d = nullptr;
  long long* d_res = nullptr;
  int rc = SLEEK_OK;
  if (cudaMalloc(&d, words * sizeof(uint64_t)) != cudaSuccess ||
      cudaMalloc(&d_res, 3 * sizeof(long long)) != cudaSuccess ||
      cudaMemset(d, 0, words * sizeof(uint64_t)) != cudaSuccess) {
    rc = SLEEK_ERR_CUDA;
  } else {
    sleek::k_selftest_waits<<<1, 32>>>(static_cast<unsigned long long>(limit_ns), d, d_res);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(h_result, d_res, 3 * sizeof(long long), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = SLEEK_ERR_CUDA;
  }
  cudaFree(d);
  cudaFree(d_res);
  if (rc) cudaGetLastError();
  return rc;
}
