// sleek_selftest.cu -- device self-tests of the codec's building blocks.
//
// Bounded waits: without faulting or hanging the device, one CTA waits on an
// mbarrier that nothing arrives on, and one warp looks back over a predecessor
// flag that nothing publishes, each with a caller-given limit, using the same
// wait helpers as the encode and decode kernels (sleek_device.cuh).  Both must
// give up, report it, and return; the context stays usable.
//
// Value maps: the transforms, quantizers and dequantizers the kernels compute
// (sleek_device.cuh, rewritten forms) against a literal restatement of the
// reference's integer steps, over every 32-bit word and over every 64-bit
// sign/exponent field with seeded mantissas; mismatches are counted, never
// trapped.
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

// ----------------------------------------------------------------------------
// Value maps against the reference's integer formulation.  The codec kernels
// compute the forward transform's exponent step as one conditional add, the
// 64-bit maps on 32-bit halves, and quantize / dequantize with the rounding
// division in floating point (sleek_device.cuh).  These are the reference's own
// steps, restated literally in 32- and 64-bit integer arithmetic
// (include/sleek_common_gpu.h: forward :356-374, inverse :614-632, quantize
// :776-802, dequantize :1077-1108), to compare against on the device.
// ----------------------------------------------------------------------------
template <typename U>
__device__ __forceinline__ U lit_fwd(U v)
{
  constexpr int TB = 8 * sizeof(U);
  constexpr U top = sizeof(U) == 4 ? static_cast<U>(0xff000000u) : static_cast<U>(0xffe0000000000000ull);
  constexpr U unit = sizeof(U) == 4 ? static_cast<U>(0x01000000u) : static_cast<U>(0x0020000000000000ull);
  constexpr U sgn = static_cast<U>(1) << (TB - 1);
  v = (v << 1) | (v >> (TB - 1));  // sign to the lowest bit
  if (v & top) {
    v -= sgn;
    if ((v & top) == 0 || v >= sgn) v -= unit;
  }
  return (v << 1) ^ ((v & sgn) ? ~static_cast<U>(0) : static_cast<U>(0));
}

template <typename U>
__device__ __forceinline__ U lit_quant(U val, int eb_e, int thr_e, U offs)
{
  constexpr int TB = 8 * sizeof(U);
  constexpr int M = sizeof(U) == 4 ? 23 : 52;  // mantissa bits
  const U a = val & ~(static_cast<U>(1) << (TB - 1));
  const int e = static_cast<int>(a >> M);
  U enc = 0;
  if (e >= thr_e) {
    enc = a - offs;
  } else if (e >= eb_e) {
    const int sh = thr_e - e;
    U mant = (val & ((static_cast<U>(1) << M) - 1)) | (static_cast<U>(1) << M);
    mant += static_cast<U>(1) << (sh - 1);
    enc = mant >> sh;
  }
  enc = (enc << 1) | ((~val) >> (TB - 1));
  return enc ? enc - 1 : 0;
}

template <typename U>
__device__ __forceinline__ U lit_dequant(U enc, int thr_e, U offs)
{
  constexpr int TB = 8 * sizeof(U);
  constexpr int M = sizeof(U) == 4 ? 23 : 52;
  if (enc == 0) return 0;
  const U a = (enc + 1) >> 1;
  U dec = 0;
  if (a >= (static_cast<U>(1) << M)) {
    dec = a + offs;
  } else if (a > 0) {
    const int lz = sizeof(U) == 4 ? __clz(static_cast<uint32_t>(a)) : __clzll(static_cast<unsigned long long>(a));
    const int sh = lz - (TB - 1 - M);
    dec = (a << sh) & ((static_cast<U>(1) << M) - 1);
    dec |= static_cast<U>(thr_e - sh) << M;
  }
  return dec | (enc << (TB - 1));
}

__device__ __forceinline__ uint64_t mix64(uint64_t x)  // splitmix64 finaliser
{
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// error-bound exponents checked: the smallest, small, mid, large and the largest legal
__constant__ int c_eb32[8] = {0, 1, 2, 24, 100, 127, 200, 230};
__constant__ int c_eb64[9] = {0, 1, 2, 53, 500, 1000, 1023, 1500, 1993};

__device__ __forceinline__ QParams q32(int k)
{
  QParams q;
  q.eb_e = c_eb32[k];
  q.thr_e = q.eb_e + 24;
  q.offs = (static_cast<uint64_t>(q.thr_e) << 23) - (1u << 23);
  return q;
}

__device__ __forceinline__ QParams q64(int k)
{
  QParams q;
  q.eb_e = c_eb64[k];
  q.thr_e = q.eb_e + 53;
  q.offs = (static_cast<uint64_t>(q.thr_e) << 52) - (1ull << 52);
  return q;
}

// a 64-bit word with sign and exponent field `top` (12 bits) and a seeded
// mantissa; the first samples of each field are the mantissa's edge values
__device__ __forceinline__ uint64_t word64(uint64_t top, uint64_t j)
{
  constexpr uint64_t MM = (1ull << 52) - 1;
  uint64_t m;
  switch (j) {
    case 0: m = 0; break;
    case 1: m = 1; break;
    case 2: m = MM; break;
    case 3: m = 1ull << 51; break;
    case 4: m = (1ull << 51) - 1; break;
    default: m = mix64(top * 0x100000000ull + j) & MM;
  }
  return (top << 52) | m;
}

// One check over index space [0, n): counts[check] += mismatches, first[check]
// = the smallest failing index.
template <int CHECK>
__global__ void __launch_bounds__(256) k_selftest_maps(unsigned long long n, unsigned long long* counts,
                                                       unsigned long long* first)
{
  unsigned long long bad = 0, fi = ~0ull;
  const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
  for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < n;
       i += stride) {
    bool ok = true;
    if constexpr (CHECK == 0) {  // f32 forward transform and its inverse, every word
      const uint32_t v = static_cast<uint32_t>(i);
      const uint32_t t = fwd(v);
      ok = t == lit_fwd<uint32_t>(v) && inv(t) == v;
    } else if constexpr (CHECK == 1) {  // f32 quantize, every word x 8 bounds
      const uint32_t v = static_cast<uint32_t>(i);
      const QParams q = q32(static_cast<int>(i >> 32));
      ok = quant_fp(v, q) == lit_quant<uint32_t>(v, q.eb_e, q.thr_e, static_cast<uint32_t>(q.offs));
    } else if constexpr (CHECK == 2) {  // f32 dequantize, every code x 8 bounds
      const uint32_t e = static_cast<uint32_t>(i);
      const QParams q = q32(static_cast<int>(i >> 32));
      ok = dequant_fp(e, q) == lit_dequant<uint32_t>(e, q.thr_e, static_cast<uint32_t>(q.offs));
    } else if constexpr (CHECK == 3) {  // f64 forward transform and inverse, every sign/exponent x 2^20
      const uint64_t v = word64(i >> 20, i & 0xfffff);
      const uint64_t t = fwd(v);
      ok = t == lit_fwd<uint64_t>(v) && inv(t) == v;
    } else if constexpr (CHECK == 4) {  // f64 quantize, every sign/exponent x 2^20, x 9 bounds
      const uint64_t v = word64((i >> 20) & 0xfff, i & 0xfffff);
      const QParams q = q64(static_cast<int>(i >> 32));
      const uint64_t want = lit_quant<uint64_t>(v, q.eb_e, q.thr_e, q.offs);
      ok = quant_fp(v, q) == want && quant(v, q) == want;
    } else {  // f64 dequantize x 9 bounds: every code below 2^32 (also the narrow
              // form), then codes of every bit length
      const QParams q = q64(static_cast<int>((i >> 32) % 9));
      if ((i >> 32) < 9) {
        const uint32_t e = static_cast<uint32_t>(i);
        const uint64_t want = lit_dequant<uint64_t>(e, q.thr_e, q.offs);
        ok = dequant_fp(static_cast<uint64_t>(e), q) == want && dequant_fp_narrow(e, q) == want &&
             dequant(static_cast<uint64_t>(e), q) == want;
      } else {
        const int len = static_cast<int>((i >> 26) & 63) + 1;
        const uint64_t e = (mix64(i) & (len == 64 ? ~0ull : ((1ull << len) - 1))) | (1ull << (len - 1));
        const uint64_t want = lit_dequant<uint64_t>(e, q.thr_e, q.offs);
        ok = dequant_fp(e, q) == want && dequant(e, q) == want;
      }
    }
    if (!ok) {
      ++bad;
      if (i < fi) fi = i;
    }
  }
  if (bad) {
    atomicAdd(&counts[CHECK], bad);
    atomicMin(&first[CHECK], fi);
  }
}

}  // namespace
}  // namespace sleek

extern "C" int sleek_selftest_value_maps(long long* h_counts, long long* h_first)
{
  if (!h_counts) return SLEEK_ERR_INVALID_ARG;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  constexpr int K = SLEEK_SELFTEST_VALUE_CHECKS;
  unsigned long long* d = nullptr;
  int rc = SLEEK_OK;
  if (cudaMalloc(&d, 2 * K * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemset(d, 0, K * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMemset(d + K, 0xff, K * sizeof(unsigned long long)) != cudaSuccess) {
    rc = SLEEK_ERR_CUDA;
  } else {
    const unsigned grid = static_cast<unsigned>((sms > 0 ? sms : 148) * 8);
    const unsigned long long w32 = 1ull << 32;
    sleek::k_selftest_maps<0><<<grid, 256>>>(w32, d, d + K);
    sleek::k_selftest_maps<1><<<grid, 256>>>(8 * w32, d, d + K);
    sleek::k_selftest_maps<2><<<grid, 256>>>(8 * w32, d, d + K);
    sleek::k_selftest_maps<3><<<grid, 256>>>(w32, d, d + K);
    sleek::k_selftest_maps<4><<<grid, 256>>>(9 * w32, d, d + K);
    sleek::k_selftest_maps<5><<<grid, 256>>>(18 * w32, d, d + K);
    unsigned long long h[2 * K];
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) {
      rc = SLEEK_ERR_CUDA;
    } else {
      for (int k = 0; k < K; ++k) {
        h_counts[k] = static_cast<long long>(h[k]);
        if (h_first) h_first[k] = static_cast<long long>(h[K + k]);
      }
    }
  }
  cudaFree(d);
  if (rc) cudaGetLastError();
  return rc;
}

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
