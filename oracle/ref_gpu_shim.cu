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
