// sleek_lossy_gpu.h -- drop-in replacement for SLEEK's include/sleek_lossy_gpu.h.
// Same types and overloads (:47-127).  sleek_error_bound reports a too-large bound
// and returns parameters that every call rejects with SLEEK_ERR_ERROR_BOUND,
// where the reference exits (:68).
#pragma once

#include <type_traits>

#include "sleek_common_gpu.h"

template <typename T>
struct sleek_error_bound_info
{
  const int eb_e;
  const int thr_e;
  const T offs_e;
};

template <typename F>
static inline sleek_error_bound_info<typename std::conditional<sizeof(F) == 4, unsigned int, unsigned long long>::type> sleek_error_bound(const F eb)
{
  static_assert(sizeof(F) == 4 || sizeof(F) == 8, "float or double");
  if constexpr (sizeof(F) == 4) {
    sleek_eb_info_f32 i;
    if (sleek_report(sleek_error_bound_f32((float)eb, &i), "sleek_error_bound") != SLEEK_OK) return {-1, -1, 0u};
    return {i.eb_e, i.thr_e, i.offs_e};
  } else {
    sleek_eb_info_f64 i;
    if (sleek_report(sleek_error_bound_f64((double)eb, &i), "sleek_error_bound") != SLEEK_OK) return {-1, -1, 0ull};
    return {i.eb_e, i.thr_e, i.offs_e};
  }
}

static inline int sleek_compress_gpu(const int blocks, const sleek_error_bound_info<unsigned int> eb_info, const float* const __restrict__ d_input,
                                     const long long num_elements, byte* const __restrict__ d_encoded, long long* const __restrict__ d_encsize)
{
  (void)blocks;
  const sleek_eb_info_f32 e = {eb_info.eb_e, eb_info.thr_e, eb_info.offs_e};
  const int rc = sleek_compress_lossy_f32(e, d_input, num_elements, d_encoded, d_encsize, nullptr, 0, nullptr);
  return rc ? sleek_report(rc, "sleek_compress_gpu") : sleek_finish(d_encsize, "sleek_compress_gpu");
}

static inline int sleek_decompress_gpu(const int blocks, const sleek_error_bound_info<unsigned int> eb_info, const byte* const __restrict__ d_encoded,
                                       float* const __restrict__ d_decoded, long long* const __restrict__ d_decsize)
{
  (void)blocks;
  const sleek_eb_info_f32 e = {eb_info.eb_e, eb_info.thr_e, eb_info.offs_e};
  const int rc = sleek_decompress_lossy_f32(e, d_encoded, -1, d_decoded, -1, d_decsize, nullptr, 0, nullptr);
  return rc ? sleek_report(rc, "sleek_decompress_gpu") : sleek_finish(d_decsize, "sleek_decompress_gpu");
}

static inline int sleek_compress_gpu(const int blocks, const sleek_error_bound_info<unsigned long long> eb_info, const double* const __restrict__ d_input,
                                     const long long num_elements, byte* const __restrict__ d_encoded, long long* const __restrict__ d_encsize)
{
  (void)blocks;
  const sleek_eb_info_f64 e = {eb_info.eb_e, eb_info.thr_e, eb_info.offs_e};
  const int rc = sleek_compress_lossy_f64(e, d_input, num_elements, d_encoded, d_encsize, nullptr, 0, nullptr);
  return rc ? sleek_report(rc, "sleek_compress_gpu") : sleek_finish(d_encsize, "sleek_compress_gpu");
}

static inline int sleek_decompress_gpu(const int blocks, const sleek_error_bound_info<unsigned long long> eb_info, const byte* const __restrict__ d_encoded,
                                       double* const __restrict__ d_decoded, long long* const __restrict__ d_decsize)
{
  (void)blocks;
  const sleek_eb_info_f64 e = {eb_info.eb_e, eb_info.thr_e, eb_info.offs_e};
  const int rc = sleek_decompress_lossy_f64(e, d_encoded, -1, d_decoded, -1, d_decsize, nullptr, 0, nullptr);
  return rc ? sleek_report(rc, "sleek_decompress_gpu") : sleek_finish(d_decsize, "sleek_decompress_gpu");
}
