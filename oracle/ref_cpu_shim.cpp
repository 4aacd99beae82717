// ref_cpu_shim.cpp -- C entry points around the reference's own CPU codec.
//
// Test infrastructure only.  oracle/Makefile compiles this file against the
// UNMODIFIED reference headers where they lie (include/sleek_lossless_cpu.h,
// include/sleek_lossy_cpu.h of the SLEEK sources, passed in with -I), producing
// oracle/_ref/libsleek_ref_cpu.so.  Nothing from the reference is copied here:
// this file only forwards plain pointers to the reference's overloads
// (include/sleek_lossless_cpu.h:46-73, include/sleek_lossy_cpu.h:56-101).
#include "sleek_lossless_cpu.h"
#include "sleek_lossy_cpu.h"

extern "C" {

long long ref_cpu_compress_f32(const float* in, long long n, unsigned char* out)
{ long long sz = 0; sleek_compress_cpu(in, n, out, sz); return sz; }

long long ref_cpu_compress_f64(const double* in, long long n, unsigned char* out)
{ long long sz = 0; sleek_compress_cpu(in, n, out, sz); return sz; }

long long ref_cpu_decompress_f32(const unsigned char* in, float* out)
{ long long sz = 0; sleek_decompress_cpu(in, out, sz); return sz; }

long long ref_cpu_decompress_f64(const unsigned char* in, double* out)
{ long long sz = 0; sleek_decompress_cpu(in, out, sz); return sz; }

long long ref_cpu_compress_lossy_f32(float eb, const float* in, long long n, unsigned char* out)
{ long long sz = 0; sleek_compress_cpu(sleek_error_bound(eb), in, n, out, sz); return sz; }

long long ref_cpu_compress_lossy_f64(double eb, const double* in, long long n, unsigned char* out)
{ long long sz = 0; sleek_compress_cpu(sleek_error_bound(eb), in, n, out, sz); return sz; }

long long ref_cpu_decompress_lossy_f32(float eb, const unsigned char* in, float* out)
{ long long sz = 0; sleek_decompress_cpu(sleek_error_bound(eb), in, out, sz); return sz; }

long long ref_cpu_decompress_lossy_f64(double eb, const unsigned char* in, double* out)
{ long long sz = 0; sleek_decompress_cpu(sleek_error_bound(eb), in, out, sz); return sz; }

void ref_cpu_error_bound_f32(float eb, int* eb_e, int* thr_e, unsigned int* offs)
{ const auto i = sleek_error_bound(eb); *eb_e = i.eb_e; *thr_e = i.thr_e; *offs = i.offs_e; }

void ref_cpu_error_bound_f64(double eb, int* eb_e, int* thr_e, unsigned long long* offs)
{ const auto i = sleek_error_bound(eb); *eb_e = i.eb_e; *thr_e = i.thr_e; *offs = i.offs_e; }

}
