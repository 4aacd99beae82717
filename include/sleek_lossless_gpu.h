// sleek_lossless_gpu.h -- drop-in replacement for SLEEK's include/sleek_lossless_gpu.h.
// Same overloads (:47-100); each forwards to the C ABI on the legacy default stream
// and waits for it, as the reference's cudaFree did.  They return a status
// (SLEEK_OK = 0) instead of void; callers that ignore it compile unchanged.  The
// blocks argument is accepted and ignored.
#pragma once

#include "sleek_common_gpu.h"

static inline int sleek_compress_gpu(const int blocks, const float* const __restrict__ d_input, const long long num_elements,
                                     byte* const __restrict__ d_encoded, long long* const __restrict__ d_encsize)
{
  (void)blocks;
  const int rc = sleek_compress_f32(d_input, num_elements, d_encoded, d_encsize, nullptr, 0, nullptr);
  return rc ? sleek_report(rc, "sleek_compress_gpu") : sleek_finish(d_encsize, "sleek_compress_gpu");
}

static inline int sleek_decompress_gpu(const int blocks, const byte* const __restrict__ d_encoded, float* const __restrict__ d_decoded,
                                       long long* const __restrict__ d_decsize)
{
  (void)blocks;
  const int rc = sleek_decompress_f32(d_encoded, -1, d_decoded, -1, d_decsize, nullptr, 0, nullptr);
  return rc ? sleek_report(rc, "sleek_decompress_gpu") : sleek_finish(d_decsize, "sleek_decompress_gpu");
}

static inline int sleek_compress_gpu(const int blocks, const double* const __restrict__ d_input, const long long num_elements,
                                     byte* const __restrict__ d_encoded, long long* const __restrict__ d_encsize)
{
  (void)blocks;
  const int rc = sleek_compress_f64(d_input, num_elements, d_encoded, d_encsize, nullptr, 0, nullptr);
  return rc ? sleek_report(rc, "sleek_compress_gpu") : sleek_finish(d_encsize, "sleek_compress_gpu");
}

static inline int sleek_decompress_gpu(const int blocks, const byte* const __restrict__ d_encoded, double* const __restrict__ d_decoded,
                                       long long* const __restrict__ d_decsize)
{
  (void)blocks;
  const int rc = sleek_decompress_f64(d_encoded, -1, d_decoded, -1, d_decsize, nullptr, 0, nullptr);
  return rc ? sleek_report(rc, "sleek_decompress_gpu") : sleek_finish(d_decsize, "sleek_decompress_gpu");
}
