// sleek_noalloc.cu -- lossless float32 compress that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs where the device memory is
// owned by someone else (a framework or pool allocator that forbids allocations
// behind its back, a fixed memory budget in a long-running service), and code that
// must not risk the implicit device synchronisation an allocation can cause.  For
// them this entry point compresses with a scratch area that is part of the library
// image itself: a file-scope __device__ array, allocated once per device when the
// library's device code is loaded on that device (with lazy module loading, the
// CUDA default, that happens at the first call's address lookup below, which is
// why the first call belongs at initialisation time) and held until the process
// exits.  The caller still passes the input, the output stream buffer and the size
// output.
//
// The scratch holds the same things the regular entry point's workspace holds (a
// header of 32 words and one look-back flag per 16 KB chunk), so its fixed size
// bounds the input: at most SLEEK_STATIC_MAX_INPUT_BYTES (1 GiB) per call.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/sleek_capi.h"

namespace {

constexpr long long kChunk = 16384;
constexpr long long kMaxChunks = SLEEK_STATIC_MAX_INPUT_BYTES / kChunk;
constexpr size_t kScratchWords = 32 + static_cast<size_t>(kMaxChunks);  // header + one flag per chunk
constexpr size_t kScratchBytes = 8 * kScratchWords;                     // 512 KiB + 256 B

// The scratch itself.  In host code this name is only a handle for the CUDA
// runtime: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned long long g_static_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch on the current device; looked up once per
// device, with that device current, on the first call made on it.
int scratch_address(void** out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) return SLEEK_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return SLEEK_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return SLEEK_OK;
}

}  // namespace

extern "C" int sleek_compress_f32_static(const float* d_input, long long num_elements, unsigned char* d_encoded,
                                         long long* d_encsize, void* stream)
{
  if (num_elements < 0 || (!d_input && num_elements > 0) || !d_encoded || !d_encsize) return SLEEK_ERR_INVALID_ARG;
  if (num_elements > SLEEK_STATIC_MAX_INPUT_BYTES / static_cast<long long>(sizeof(float))) return SLEEK_ERR_TOO_LARGE;
  void* scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc != SLEEK_OK) return rc;
  // The regular entry point with a caller workspace allocates nothing: it clears the
  // part of the scratch this call uses (cudaMemsetAsync on `stream`) and launches.
  return sleek_compress_f32(d_input, num_elements, d_encoded, d_encsize, scratch, kScratchBytes, stream);
}
