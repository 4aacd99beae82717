// sleek_reduce.cu -- value range of a device array (min and max, NaN ignored).
//
// The reference's range-relative ("ARTIFACT") drivers derive the absolute error
// bound as (max - min) * parameter with an OpenMP loop on the host copy of the
// input (computeNOAeb, lossy_compressors_gpu/sleek_single_compressor_lossy.cu:59-75).
// Here the range comes from the device copy in one HBM-bound pass: every value is
// mapped to an order-preserving unsigned key (negative values bit-inverted,
// non-negative ones with the sign bit set), NaNs are skipped, and each CTA folds
// its keys into two 64-bit maxima in the workspace -- keys[0] the maximum of the
// inverted keys (the minimum), keys[1] the maximum key -- so the workspace only
// needs zeroing first.
#include <cstdint>

#include <cuda_runtime.h>

#include "sleek_launch.h"

namespace sleek {

namespace {

constexpr int MM_NT = 256;
constexpr int MM_UNROLL = 4;  // 16-byte loads in flight per thread

template <typename U>
struct KeyOf;

template <>
struct KeyOf<uint32_t> {
  // 0 never occurs as a key or an inverted key of a non-NaN value (it would be
  // the key of 0xffffffff or the inverted key of 0x7fffffff, both NaNs), so 0
  // means "no value"
  __device__ static void fold(uint32_t u, uint32_t& kmax, uint32_t& kinv)
  {
    if ((u & 0x7fffffffu) > 0x7f800000u) return;  // NaN
    const uint32_t k = u ^ (static_cast<uint32_t>(static_cast<int32_t>(u) >> 31) | 0x80000000u);
    kmax = max(kmax, k);
    kinv = max(kinv, ~k);
  }
};

template <>
struct KeyOf<uint64_t> {
  __device__ static void fold(uint64_t u, uint64_t& kmax, uint64_t& kinv)
  {
    if ((u & 0x7fffffffffffffffull) > 0x7ff0000000000000ull) return;  // NaN
    const uint64_t k = u ^ (static_cast<uint64_t>(static_cast<int64_t>(u) >> 63) | 0x8000000000000000ull);
    kmax = max(kmax, k);
    kinv = max(kinv, ~k);
  }
};

template <typename U>
__device__ __forceinline__ void fold_vec(const uint4 w, U& kmax, U& kinv)
{
  if constexpr (sizeof(U) == 4) {
    KeyOf<U>::fold(w.x, kmax, kinv);
    KeyOf<U>::fold(w.y, kmax, kinv);
    KeyOf<U>::fold(w.z, kmax, kinv);
    KeyOf<U>::fold(w.w, kmax, kinv);
  } else {
    KeyOf<U>::fold((static_cast<uint64_t>(w.y) << 32) | w.x, kmax, kinv);
    KeyOf<U>::fold((static_cast<uint64_t>(w.w) << 32) | w.z, kmax, kinv);
  }
}

template <typename U>
__global__ void __launch_bounds__(MM_NT) k_minmax(const U* __restrict__ in, long long n, unsigned long long* keys)
{
  constexpr int E = 16 / sizeof(U);  // values per 16-byte load
  U kmax = 0, kinv = 0;
  // element-aligned inputs: a head of up to E - 1 values before the first 16-byte boundary
  const uintptr_t p = reinterpret_cast<uintptr_t>(in);
  long long head = static_cast<long long>(((16u - (p & 15u)) & 15u) / sizeof(U));
  if (head > n) head = n;
  const long long nv = (n - head) / E;
  const uint4* const v = reinterpret_cast<const uint4*>(in + head);
  const long long gt = static_cast<long long>(blockIdx.x) * MM_NT + threadIdx.x;
  const long long gs = static_cast<long long>(gridDim.x) * MM_NT;
  long long i = gt;
  for (; i + (MM_UNROLL - 1) * gs < nv; i += MM_UNROLL * gs) {
    uint4 w[MM_UNROLL];
#pragma unroll
    for (int u = 0; u < MM_UNROLL; ++u) w[u] = __ldcs(v + i + u * gs);
#pragma unroll
    for (int u = 0; u < MM_UNROLL; ++u) fold_vec<U>(w[u], kmax, kinv);
  }
  for (; i < nv; i += gs) fold_vec<U>(__ldcs(v + i), kmax, kinv);
  if (gt < head) KeyOf<U>::fold(in[gt], kmax, kinv);
  const long long tail = head + nv * E + gt;
  if (gt < E && tail < n) KeyOf<U>::fold(in[tail], kmax, kinv);

  // CTA reduction, then one atomic per maximum
  unsigned long long mx = kmax, mi = kinv;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mi = max(mi, __shfl_xor_sync(0xffffffffu, mi, o));
  }
  __shared__ unsigned long long s_mx[MM_NT / 32], s_mi[MM_NT / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    s_mx[warp] = mx;
    s_mi[warp] = mi;
  }
  __syncthreads();
  if (warp == 0) {
    mx = lane < MM_NT / 32 ? s_mx[lane] : 0ull;
    mi = lane < MM_NT / 32 ? s_mi[lane] : 0ull;
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      mi = max(mi, __shfl_xor_sync(0xffffffffu, mi, o));
    }
    if (lane == 0) {
      if (mi) atomicMax(&keys[0], mi);  // inverted key of the minimum
      if (mx) atomicMax(&keys[1], mx);  // key of the maximum
    }
  }
}

}  // namespace

cudaError_t launch_minmax(int width, const void* in, long long n, unsigned long long* keys, int sms, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  const long long per_cta = static_cast<long long>(MM_NT) * MM_UNROLL * 16 / width;  // values per CTA sweep
  long long grid = static_cast<long long>(sms) * 8;
  const long long need = (n + per_cta - 1) / per_cta;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  if (width == 8) {
    k_minmax<uint64_t><<<static_cast<unsigned>(grid), MM_NT, 0, st>>>(static_cast<const uint64_t*>(in), n, keys);
  } else {
    k_minmax<uint32_t><<<static_cast<unsigned>(grid), MM_NT, 0, st>>>(static_cast<const uint32_t*>(in), n, keys);
  }
  return cudaGetLastError();
}

}  // namespace sleek
