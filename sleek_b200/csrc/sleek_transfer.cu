// sleek_transfer.cu -- compressing device-to-host and decompressing host-to-device
// copies: the "compressed memcpy" use of SLEEK (its README's first line), where
// only the stream's S bytes cross PCIe instead of the array's N bytes.
//
// The buffer is cut into chunk-aligned segments, and each segment is encoded on
// its own by the single-buffer encoder.  A chunk's payload and csize do not depend
// on where the chunk sits, so a segment's stream is a slice of the whole stream:
// its size table is a slice of the whole size table and its payloads are a
// contiguous run of the whole payload area.  The host therefore receives exactly
// the stream a one-shot compress writes, assembled in place:
//
//   compress_to_host:  encode(k) on `stream` | D2H of segment k-1's table slice
//                      and payload run on a copy stream, straight to their final
//                      offsets in the host buffer (two device staging slots)
//   decompress_from_host: H2D of segment k (a fresh 8-byte header, the table
//                      slice, the payload run) on the copy stream | decode(k-1)
//                      on `stream` into its place in the output
//
// so the PCIe transfer of one segment overlaps the codec work of the next.  The
// host checks a received stream's header, size table and payload bounds before
// the first copy; the device decoder checks every chunk.  Resources (copy
// stream, events, staging, pinned size slots) are kept per (device, caller
// stream); calls on one stream are serialised by a mutex, calls on different
// streams run concurrently, so uploads and downloads can share the PCIe link
// in both directions.
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/sleek_capi.h"
#include "sleek_launch.h"

namespace {

constexpr long long CS = 16384;
constexpr long long DEFAULT_SEGMENT = 32ll << 20;

long long upper_bound(long long insize)
{
  const long long chunks = (insize + CS - 1) / CS;
  return 12 + 2 * chunks + chunks * CS;
}

struct Slots {
  std::mutex mu;
  bool ready = false;
  cudaStream_t copy = nullptr;
  cudaEvent_t done_codec[2] = {nullptr, nullptr};  // segment's encode / decode finished
  cudaEvent_t done_copy[2] = {nullptr, nullptr};   // segment's copies finished
  unsigned char* staging[2] = {nullptr, nullptr};
  size_t staging_bytes = 0;
  long long* d_sizes = nullptr;  // one device size per segment
  size_t d_sizes_n = 0;
  long long* h_sizes = nullptr;  // pinned mirror of d_sizes
  long long* h_headers = nullptr;  // pinned segment headers (decompress)
  size_t h_n = 0;
};

std::mutex g_map_mu;
std::map<std::pair<int, void*>, Slots*> g_slots;

// resources of one (device, caller stream): calls on different streams of a
// device run concurrently (each with its own copy stream and staging)
Slots* slots_for(int dev, void* stream)
{
  std::lock_guard<std::mutex> lk(g_map_mu);
  Slots*& s = g_slots[{dev, stream}];
  if (!s) s = new Slots();  // kept until exit, like the library's workspaces
  return s;
}

int cuda_fail()
{
  cudaGetLastError();
  return SLEEK_ERR_CUDA;
}

// makes room for segments of `seg_bytes` and `nseg` size slots (s->mu held)
int prepare(Slots* s, long long seg_bytes, long long nseg)
{
  if (!s->ready) {
    if (cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking) != cudaSuccess) return cuda_fail();
    for (int i = 0; i < 2; ++i)
      if (cudaEventCreateWithFlags(&s->done_codec[i], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&s->done_copy[i], cudaEventDisableTiming) != cudaSuccess)
        return cuda_fail();
    s->ready = true;
  }
  const size_t need = static_cast<size_t>(upper_bound(seg_bytes));
  if (s->staging_bytes < need) {
    cudaStreamSynchronize(s->copy);
    for (int i = 0; i < 2; ++i) {
      if (s->staging[i]) cudaFree(s->staging[i]);
      s->staging[i] = nullptr;
    }
    s->staging_bytes = 0;
    for (int i = 0; i < 2; ++i)
      if (cudaMalloc(&s->staging[i], need) != cudaSuccess) return cuda_fail();
    s->staging_bytes = need;
  }
  if (s->d_sizes_n < static_cast<size_t>(nseg)) {
    if (s->d_sizes) cudaFree(s->d_sizes);
    s->d_sizes = nullptr;
    s->d_sizes_n = 0;
    if (cudaMalloc(&s->d_sizes, sizeof(long long) * nseg) != cudaSuccess) return cuda_fail();
    s->d_sizes_n = static_cast<size_t>(nseg);
  }
  if (s->h_n < static_cast<size_t>(nseg)) {
    if (s->h_sizes) cudaFreeHost(s->h_sizes);
    if (s->h_headers) cudaFreeHost(s->h_headers);
    s->h_sizes = s->h_headers = nullptr;
    s->h_n = 0;
    if (cudaMallocHost(&s->h_sizes, sizeof(long long) * nseg) != cudaSuccess ||
        cudaMallocHost(&s->h_headers, sizeof(long long) * nseg) != cudaSuccess)
      return cuda_fail();
    s->h_n = static_cast<size_t>(nseg);
  }
  return SLEEK_OK;
}

long long segment_bytes_of(long long requested)
{
  long long b = requested > 0 ? requested : DEFAULT_SEGMENT;
  b = (b + CS - 1) / CS * CS;
  return b;
}

int check_codec(int elem_bytes, int lossy, double eb, sleek::QParams* q)
{
  if (elem_bytes != 4 && elem_bytes != 8) return SLEEK_ERR_INVALID_ARG;
  return sleek::host_qparams(elem_bytes, lossy != 0, eb, q);
}

}  // namespace

extern "C" {

int sleek_compress_to_host(const void* d_input, long long num_elements, int elem_bytes, int lossy, double error_bound,
                           unsigned char* h_encoded, long long h_capacity, long long* encoded_bytes,
                           long long segment_bytes, void* stream)
{
  sleek::QParams q;
  int rc = check_codec(elem_bytes, lossy, error_bound, &q);
  if (rc) return rc;
  if (!h_encoded || !encoded_bytes || num_elements < 0 || (num_elements > 0 && !d_input)) return SLEEK_ERR_INVALID_ARG;
  if (reinterpret_cast<uintptr_t>(d_input) % elem_bytes) return SLEEK_ERR_ALIGNMENT;
  if (num_elements > (1ll << 52) / elem_bytes) return SLEEK_ERR_INVALID_ARG;
  const long long insize = num_elements * elem_bytes;
  const long long chunks = (insize + CS - 1) / CS;
  const long long table_end = 8 + 2 * chunks;
  if (h_capacity < table_end) return SLEEK_ERR_CAPACITY;
  std::memcpy(h_encoded, &insize, 8);
  *encoded_bytes = 8;
  if (chunks == 0) return SLEEK_OK;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  const long long seg = segment_bytes_of(segment_bytes);
  const long long seg_chunks = seg / CS;
  const long long nseg = (chunks + seg_chunks - 1) / seg_chunks;
  Slots* s = slots_for(dev, stream);
  std::lock_guard<std::mutex> lk(s->mu);
  rc = prepare(s, seg, 2);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned char* in = static_cast<const unsigned char*>(d_input);
  long long run = table_end;  // host offset of the next payload run
  int status = SLEEK_OK;

  // copies segment j (encoded, its size arriving in h_sizes[j & 1]) to its place
  auto flush = [&](long long j) {
    const int slot = static_cast<int>(j & 1);
    if (cudaEventSynchronize(s->done_codec[slot]) != cudaSuccess) {
      status = cuda_fail();
      return;
    }
    const long long size = s->h_sizes[slot];
    if (size < 0) {
      status = static_cast<int>(-size);
      return;
    }
    const long long c0 = j * seg_chunks;
    const long long nch = chunks - c0 < seg_chunks ? chunks - c0 : seg_chunks;
    const long long payload = size - 8 - 2 * nch;
    if (run + payload > h_capacity) {
      status = SLEEK_ERR_CAPACITY;
      return;
    }
    if (cudaMemcpyAsync(h_encoded + 8 + 2 * c0, s->staging[slot] + 8, static_cast<size_t>(2 * nch),
                        cudaMemcpyDeviceToHost, s->copy) != cudaSuccess ||
        cudaMemcpyAsync(h_encoded + run, s->staging[slot] + 8 + 2 * nch, static_cast<size_t>(payload),
                        cudaMemcpyDeviceToHost, s->copy) != cudaSuccess ||
        cudaEventRecord(s->done_copy[slot], s->copy) != cudaSuccess) {
      status = cuda_fail();
      return;
    }
    run += payload;
  };

  for (long long k = 0; k < nseg && status == SLEEK_OK; ++k) {
    const int slot = static_cast<int>(k & 1);
    const long long c0 = k * seg_chunks;
    const long long bytes = insize - c0 * CS < seg ? insize - c0 * CS : seg;
    // the staging slot is free once segment k - 2 has been copied out of it
    if (k >= 2 && cudaStreamWaitEvent(st, s->done_copy[slot], 0) != cudaSuccess) {
      status = cuda_fail();
      break;
    }
    rc = sleek::host_compress(elem_bytes, lossy != 0, q, in + c0 * CS, bytes / elem_bytes, s->staging[slot],
                              s->d_sizes + slot, stream);
    if (rc) {
      status = rc;
      break;
    }
    if (cudaMemcpyAsync(s->h_sizes + slot, s->d_sizes + slot, sizeof(long long), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaEventRecord(s->done_codec[slot], st) != cudaSuccess) {
      status = cuda_fail();
      break;
    }
    if (k >= 1) flush(k - 1);
  }
  if (status == SLEEK_OK) flush(nseg - 1);
  // nothing of this call stays in flight, whatever happened
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaStreamSynchronize(s->copy) != cudaSuccess) {
    if (status == SLEEK_OK) status = cuda_fail();
  }
  if (status == SLEEK_OK) *encoded_bytes = run;
  return status;
}

int sleek_decompress_from_host(const unsigned char* h_encoded, long long encoded_bytes, int elem_bytes, int lossy,
                               double error_bound, void* d_decoded, long long capacity_bytes, long long* decoded_bytes,
                               long long segment_bytes, void* stream)
{
  sleek::QParams q;
  int rc = check_codec(elem_bytes, lossy, error_bound, &q);
  if (rc) return rc;
  if (!h_encoded || !decoded_bytes || encoded_bytes < 0) return SLEEK_ERR_INVALID_ARG;
  if (reinterpret_cast<uintptr_t>(d_decoded) % elem_bytes) return SLEEK_ERR_ALIGNMENT;
  // pre-flight on the host: header, size table and payload bounds, which every
  // copy below relies on; each chunk's widths, size and trailer are checked by
  // the device decoder (reading every chunk's header here would cost as much as
  // a lossy stream's whole transfer)
  sleek_stream_info info;
  rc = sleek::validate_stream(h_encoded, encoded_bytes, elem_bytes, &info, false);
  if (rc) return rc;
  const long long insize = info.insize;
  if (insize > capacity_bytes) return SLEEK_ERR_CAPACITY;
  *decoded_bytes = 0;
  const long long chunks = info.chunks;
  if (chunks == 0) return SLEEK_OK;
  if (!d_decoded) return SLEEK_ERR_INVALID_ARG;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  const long long seg = segment_bytes_of(segment_bytes);
  const long long seg_chunks = seg / CS;
  const long long nseg = (chunks + seg_chunks - 1) / seg_chunks;
  Slots* s = slots_for(dev, stream);
  std::lock_guard<std::mutex> lk(s->mu);
  rc = prepare(s, seg, nseg);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* out = static_cast<unsigned char*>(d_decoded);
  const unsigned char* table = h_encoded + 8;
  long long off = 8 + 2 * chunks;  // host offset of segment k's payload run
  int status = SLEEK_OK;

  for (long long k = 0; k < nseg; ++k) {
    const int slot = static_cast<int>(k & 1);
    const long long c0 = k * seg_chunks;
    const long long nch = chunks - c0 < seg_chunks ? chunks - c0 : seg_chunks;
    const long long bytes = insize - c0 * CS < seg ? insize - c0 * CS : seg;
    long long payload = 0;
    for (long long c = c0; c < c0 + nch; ++c) {
      uint16_t cs;
      std::memcpy(&cs, table + 2 * c, 2);
      payload += cs;
    }
    s->h_headers[k] = bytes;
    unsigned char* const stg = s->staging[slot];
    // the staging slot is free once segment k - 2 has been decoded out of it
    if ((k >= 2 && cudaStreamWaitEvent(s->copy, s->done_codec[slot], 0) != cudaSuccess) ||
        cudaMemcpyAsync(stg, s->h_headers + k, 8, cudaMemcpyHostToDevice, s->copy) != cudaSuccess ||
        cudaMemcpyAsync(stg + 8, table + 2 * c0, static_cast<size_t>(2 * nch), cudaMemcpyHostToDevice, s->copy) !=
            cudaSuccess ||
        cudaMemcpyAsync(stg + 8 + 2 * nch, h_encoded + off, static_cast<size_t>(payload), cudaMemcpyHostToDevice,
                        s->copy) != cudaSuccess ||
        cudaEventRecord(s->done_copy[slot], s->copy) != cudaSuccess || cudaStreamWaitEvent(st, s->done_copy[slot], 0) != cudaSuccess) {
      status = cuda_fail();
      break;
    }
    rc = sleek::host_decompress(elem_bytes, lossy != 0, q, stg, 8 + 2 * nch + payload, out + c0 * CS, bytes,
                                s->d_sizes + k, stream);
    if (rc) {
      status = rc;
      break;
    }
    if (cudaEventRecord(s->done_codec[slot], st) != cudaSuccess) {
      status = cuda_fail();
      break;
    }
    off += payload;
  }
  if (status == SLEEK_OK &&
      cudaMemcpyAsync(s->h_sizes, s->d_sizes, sizeof(long long) * nseg, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    status = cuda_fail();
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaStreamSynchronize(s->copy) != cudaSuccess) {
    if (status == SLEEK_OK) status = cuda_fail();
  }
  if (status != SLEEK_OK) return status;
  long long total = 0;
  for (long long k = 0; k < nseg; ++k) {
    if (s->h_sizes[k] < 0) return static_cast<int>(-s->h_sizes[k]);
    total += s->h_sizes[k];
  }
  if (total != insize) return SLEEK_ERR_CORRUPT_STREAM;
  *decoded_bytes = total;
  return SLEEK_OK;
}

}  // extern "C"
