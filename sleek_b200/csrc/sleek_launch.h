// sleek_launch.h -- host-side launch interface between the C ABI (sleek_capi.cu)
// and the kernels (sleek_kernels.cu).  Internal to the library.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

struct sleek_stream_info;

namespace sleek {

constexpr int NT_MAX_WARPS = 32;

// lossy quantizer parameters, as sleek_error_bound derives them
// (include/sleek_lossy_gpu.h:47-71 of the reference)
struct QParams {
  int eb_e;
  int thr_e;
  uint64_t offs;
};

struct EncArgs {
  const uint8_t* in;     // device input values (element aligned)
  long long insize;      // input bytes
  uint8_t* out;          // device stream, >= upper bound size, 8-byte aligned
  long long* outsize;    // device: stream bytes, or -status on a device-detected error
  uint64_t* ws;          // workspace: header words + flag regions (self-resetting, see WsPhase)
  long long flag_cap;    // flags per region (at least one per chunk)
  QParams q;
};

struct DecArgs {
  const uint8_t* in;     // device stream, 8-byte aligned
  long long in_len;      // stream bytes, or -1 when unknown (no payload bound check)
  uint8_t* out;          // device output values (element aligned)
  long long out_cap;     // output capacity in bytes, or -1 when unknown
  long long* outsize;    // device: decoded bytes, or -status
  uint64_t* ws;          // workspace: header words + flag regions (self-resetting, see WsPhase)
  long long flag_cap;    // flags per region (at least one per CTA)
  QParams q;
};

// One buffer of a batched launch (device table entry).
struct BatchJob {
  const uint8_t* in;     // compress: values; decompress: stream
  uint8_t* out;          // compress: stream; decompress: values
  long long* outsize;    // device: bytes written, or -status
  long long insize;      // compress: input bytes; decompress: stream bytes (-1 = unknown)
  long long cap;         // decompress: output capacity in bytes
  long long chunks;      // compress: chunks; decompress: chunks the capacity allows
  QParams q;
  int kind;              // bit 0: 64-bit values, bit 1: lossy
  int pad_;
};

constexpr int BATCH_MAX_JOBS = 1024;  // buffers per launch (the chunk table lives in shared memory)

struct BatchEncArgs {
  const BatchJob* jobs;         // device table
  const long long* chunk_base;  // device: first chunk id of each job, then the total (njobs + 1)
  int njobs;
  uint64_t* ws;                 // zeroed workspace: header words + one flag per chunk
};

struct BatchDecArgs {
  const BatchJob* jobs;         // device table (in: stream, insize: stream bytes or -1, cap: output bytes)
  const long long* chunk_base;  // device: first chunk id of each job by capacity, then the total
  int njobs;
  uint64_t* ws;                 // zeroed workspace header words
  long long* offsets;           // workspace: payload offset of every chunk id
  long long* actual;            // workspace: chunks in each stream (from its header)
  long long* actual_insize;     // workspace: bytes each stream decodes to
};

// Launch shapes of the single-buffer kernels (sleek_kernels.cu: EncShape*,
// DecShape*); shape 0 is the default.  Every shape produces the same bytes.
struct ShapeInfo {
  int threads;        // per CTA
  int warps;          // compute warps (encode) / warps (decode)
  int stages;         // shared-memory chunk stages
  int ctas_per_sm;    // CTAs per SM the registers are budgeted for
};
int shape_count(bool enc);
ShapeInfo shape_info(bool enc, int shape);
cudaError_t launch_encode(int width, bool lossy, int shape, const EncArgs& a, int grid, cudaStream_t st);
cudaError_t launch_decode(int width, bool lossy, int shape, const DecArgs& a, int grid, cudaStream_t st);
int blocks_per_sm(int width, bool lossy, bool enc, int shape);
cudaError_t launch_decode_batch(const BatchDecArgs& a, int grid, cudaStream_t st);
int decode_batch_blocks_per_sm();
cudaError_t launch_encode_batch(const BatchEncArgs& a, int grid, cudaStream_t st);
int encode_batch_blocks_per_sm();
// the single-buffer entry points for other host sources of the library (they use
// the library-owned workspace of `stream`); host_qparams derives the quantizer
// parameters of an error bound (SLEEK_ERR_ERROR_BOUND when it is too large)
int host_compress(int width, bool lossy, QParams q, const void* in, long long n, unsigned char* out,
                  long long* outsize, void* stream);
int host_decompress(int width, bool lossy, QParams q, const unsigned char* in, long long in_len, void* out,
                    long long cap, long long* outsize, void* stream);
int host_qparams(int width, bool lossy, double eb, QParams* q);
// stream checks of sleek_validate_stream; with payloads = false only the header,
// the size table and the payload bounds (what every copy of the stream depends
// on), without reading the payloads themselves
int validate_stream(const unsigned char* s, long long len, int elem_bytes, sleek_stream_info* info, bool payloads);
// min / max keys of a device array into keys[0] (inverted minimum) and keys[1]
// (maximum); keys must be zero before the launch
cudaError_t launch_minmax(int width, const void* in, long long n, unsigned long long* keys, int sms, cudaStream_t st);

}  // namespace sleek
