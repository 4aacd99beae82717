// ref_gpu_shim.cu -- C entry points around the reference's own GPU codec.
//
// Test infrastructure only: the second parity oracle and the kernels to beat.
// oracle/Makefile compiles this file for sm_100a against the UNMODIFIED
// reference headers where they lie (include/sleek_lossless_gpu.h,
// include/sleek_lossy_gpu.h of the SLEEK sources, passed in with -I), producing
// oracle/_ref/libsleek_ref_gpu.so.  Each function forwards to the reference's
// overloads (include/sleek_lossless_gpu.h:47-100, include/sleek_lossy_gpu.h:74-127),
// which allocate and free their own scratch on the legacy default stream.
#include <cstdio>
#include "sleek_lossless_gpu.h"
#include "sleek_lossy_gpu.h"

extern "C" {

int ref_gpu_blocks(void) { return sleek_thread_blocks(); }

void ref_gpu_compress_f32(int blocks, const float* d_in, long long n, unsigned char* d_out, long long* d_size)
{ sleek_compress_gpu(blocks, d_in, n, d_out, d_size); }

void ref_gpu_compress_f64(int blocks, const double* d_in, long long n, unsigned char* d_out, long long* d_size)
{ sleek_compress_gpu(blocks, d_in, n, d_out, d_size); }

void ref_gpu_decompress_f32(int blocks, const unsigned char* d_in, float* d_out, long long* d_size)
{ sleek_decompress_gpu(blocks, d_in, d_out, d_size); }

void ref_gpu_decompress_f64(int blocks, const unsigned char* d_in, double* d_out, long long* d_size)
{ sleek_decompress_gpu(blocks, d_in, d_out, d_size); }

void ref_gpu_compress_lossy_f32(int blocks, float eb, const float* d_in, long long n, unsigned char* d_out, long long* d_size)
{ sleek_compress_gpu(blocks, sleek_error_bound(eb), d_in, n, d_out, d_size); }

void ref_gpu_compress_lossy_f64(int blocks, double eb, const double* d_in, long long n, unsigned char* d_out, long long* d_size)
{ sleek_compress_gpu(blocks, sleek_error_bound(eb), d_in, n, d_out, d_size); }

void ref_gpu_decompress_lossy_f32(int blocks, float eb, const unsigned char* d_in, float* d_out, long long* d_size)
{ sleek_decompress_gpu(blocks, sleek_error_bound(eb), d_in, d_out, d_size); }

void ref_gpu_decompress_lossy_f64(int blocks, double eb, const unsigned char* d_in, double* d_out, long long* d_size)
{ sleek_decompress_gpu(blocks, sleek_error_bound(eb), d_in, d_out, d_size); }

}

// The same kernels launched directly with caller-allocated scratch (the chunk
// carries + ticket counter for encode, the ticket counter for decode), i.e. the
// reference's API bodies (include/sleek_lossless_gpu.h:47-60, 63-72; lossy
// :74-87, 90-99) without their per-call cudaMalloc / cudaFree.
template <typename T, typename F>
static void enc_prealloc(int blocks, const F* d_in, long long n, unsigned char* d_out, long long* d_size,
                         long long* d_carry, int lossy, double eb)
{
  const long long insize = n * (long long)sizeof(F);
  const long long chunks = (insize + SLEEK_CS - 1) / SLEEK_CS + 1;
  cudaMemsetAsync(d_carry, 0, chunks * sizeof(long long));
  unsigned long long* const counter = (unsigned long long*)&d_carry[chunks - 1];
  if (lossy) {
    const auto e = sleek_error_bound((F)eb);
    d_encode<T><<<blocks, SLEEK_TPB>>>((byte*)d_in, insize, d_out, d_size, d_carry, counter, e.eb_e, e.thr_e, e.offs_e);
  } else {
    d_encode<T><<<blocks, SLEEK_TPB>>>((byte*)d_in, insize, d_out, d_size, d_carry, counter);
  }
}

template <typename T, typename F>
static void dec_prealloc(int blocks, const unsigned char* d_in, F* d_out, long long* d_size,
                         unsigned long long* d_counter, int lossy, double eb)
{
  cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long));
  if (lossy) {
    const auto e = sleek_error_bound((F)eb);
    d_decode<T><<<blocks, SLEEK_TPB>>>(d_in, (byte*)d_out, d_size, d_counter, e.thr_e, e.offs_e);
  } else {
    d_decode<T><<<blocks, SLEEK_TPB>>>(d_in, (byte*)d_out, d_size, d_counter);
  }
}

extern "C" {

void ref_gpu_encode_prealloc_f64(int blocks, const double* d_in, long long n, unsigned char* d_out, long long* d_size,
                                 long long* d_carry, int lossy, double eb)
{ enc_prealloc<unsigned long long, double>(blocks, d_in, n, d_out, d_size, d_carry, lossy, eb); }

void ref_gpu_decode_prealloc_f64(int blocks, const unsigned char* d_in, double* d_out, long long* d_size,
                                 unsigned long long* d_counter, int lossy, double eb)
{ dec_prealloc<unsigned long long, double>(blocks, d_in, d_out, d_size, d_counter, lossy, eb); }

void ref_gpu_encode_prealloc_f32(int blocks, const float* d_in, long long n, unsigned char* d_out, long long* d_size,
                                 long long* d_carry, int lossy, double eb)
{ enc_prealloc<unsigned int, float>(blocks, d_in, n, d_out, d_size, d_carry, lossy, eb); }

void ref_gpu_decode_prealloc_f32(int blocks, const unsigned char* d_in, float* d_out, long long* d_size,
                                 unsigned long long* d_counter, int lossy, double eb)
{ dec_prealloc<unsigned int, float>(blocks, d_in, d_out, d_size, d_counter, lossy, eb); }

}
