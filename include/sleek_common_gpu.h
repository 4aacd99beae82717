// sleek_common_gpu.h -- drop-in replacement for SLEEK's include/sleek_common_gpu.h
// (constants and helpers, :53-119).  The codec itself lives in the sm_100a
// library (libsleek_b200.so); this header only forwards to its C ABI
// (sleek_capi.h).  Link with -lsleek_b200.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#include "sleek_capi.h"

using byte = unsigned char;
static const int SLEEK_CS = 1024 * 16;  // chunk size in bytes (part of the stream format)
static const int SLEEK_TPB = 512;       // kept for source compatibility; the library sizes its own CTAs
#ifndef SLEEK_WS
#define SLEEK_WS 32
#endif

// CheckCuda of the reference (include/sleek_common_gpu.h:68-76), which its command-line
// drivers call after each phase: waits for the device and exits with the same
// message when a CUDA error is pending.
static inline void CheckCuda(const int line)
{
  cudaDeviceSynchronize();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "CUDA error %d on line %d: %s\n\n", e, line, cudaGetErrorString(e));
    exit(-1);
  }
}

// Reports a host- or device-side status the way the reference reports CUDA errors
// (to stderr), but returns it instead of exiting.
static inline int sleek_report(const int status, const char* where)
{
  if (status != SLEEK_OK) fprintf(stderr, "SLEEK ERROR in %s: %s (status %d)\n", where, sleek_status_string(status), status);
  return status;
}

// Waits for the default stream and turns a negative size written by the device
// (-status) into that status.  The reference's calls end in cudaFree, which
// synchronises, so results were visible on return; the forwarders keep that.
static inline int sleek_finish(const long long* d_size, const char* where)
{
  long long v = 0;
  if (cudaMemcpy(&v, d_size, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return sleek_report(SLEEK_ERR_CUDA, where);
  }
  return v < 0 ? sleek_report((int)-v, where) : SLEEK_OK;
}
