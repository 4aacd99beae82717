/*
 * sleek_capi.h -- C ABI of the B200 (sm_100a) SLEEK compress / decompress path.
 *
 * Drop-in boundary for the reference's GPU API (include/sleek_lossless_gpu.h and
 * include/sleek_lossy_gpu.h of SLEEK).  Plain pointers and sizes only; every entry
 * point is asynchronous on the given CUDA stream (NULL = legacy default stream) and
 * returns a status code for everything it can check on the host.  Errors found on
 * the device (malformed stream, a look-back wait that exceeded its time limit)
 * never trap: the kernel writes -status into the size output (*d_encsize or
 * *d_decsize), and the status is also readable with sleek_workspace_status().
 *
 * The compressed byte stream is SLEEK's own (8-byte insize, uint16 size per 16 KB
 * chunk, byte-packed chunk payloads) and is bit-identical to the reference's CPU
 * and GPU output for the same input and error bound.
 *
 * Pointers: device inputs/outputs must be aligned to their element size (4 for
 * float, 8 for double); the stream buffer must be 8-byte aligned.  16-byte
 * aligned inputs take the TMA path; others are loaded with ordinary loads.
 *
 * Workspace: pass NULL to use a workspace the library owns (one per device and
 * stream, grown on demand -- growth calls cudaMalloc, so size it up front with a
 * first call outside stream capture), or pass a device buffer of at least
 * sleek_*_workspace_size() bytes.  A caller's workspace is cleared with
 * cudaMemsetAsync on the same stream before each launch.  The library's own
 * workspace is cleared once, when it is allocated, and then kept ready by the
 * kernels themselves (each launch leaves the half it did not use clean for the
 * next), so calls with NULL issue no clearing work.  Calls that share one
 * workspace must be ordered on one stream; a CUDA graph that holds calls with the
 * library-owned workspace of a stream must run in that stream's order.  A
 * library-owned workspace is replaced (after a synchronisation of its stream)
 * when a call needs more than it holds, so host threads that issue calls on the
 * same stream must not overlap their calls; threads on different streams need no
 * coordination.
 */
#ifndef SLEEK_CAPI_H
#define SLEEK_CAPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SLEEK_OK                 0
#define SLEEK_ERR_INVALID_ARG    1  /* null pointer, negative size, size not a multiple of the element */
#define SLEEK_ERR_ALIGNMENT      2  /* pointer not aligned as documented above */
#define SLEEK_ERR_CUDA           3  /* a CUDA runtime call failed (launch, memset, allocation) */
#define SLEEK_ERR_ERROR_BOUND    4  /* error bound too large (the reference exits, sleek_lossy_gpu.h:68) */
#define SLEEK_ERR_CORRUPT_STREAM 5  /* malformed stream (the reference traps, sleek_common_gpu.h:753,1264) */
#define SLEEK_ERR_TIMEOUT        6  /* a device-side wait exceeded its time limit */
#define SLEEK_ERR_WORKSPACE      7  /* caller workspace smaller than required */
#define SLEEK_ERR_NO_DEVICE      8  /* no CUDA device */
#define SLEEK_ERR_CAPACITY       9  /* output buffer smaller than required */
#define SLEEK_ERR_TOO_LARGE     10  /* input larger than SLEEK_STATIC_MAX_INPUT_BYTES (static-scratch entry point) */

/* Human-readable name of a status code. */
const char* sleek_status_string(int status);

/* Replaces sleek_upper_bound_size (include/sleek_common_gpu.h:79-83): bytes to
 * allocate for a stream of an insize-byte input: 12 + 2*chunks + 16384*chunks. */
long long sleek_upper_bound_size(long long insize);

/* Replaces sleek_system_checks (include/sleek_common_gpu.h:86-105): 0 when the
 * host is little-endian with the expected integer sizes, -1 otherwise. */
int sleek_system_checks(void);

/* Replaces sleek_thread_blocks (include/sleek_common_gpu.h:108-119): the
 * persistent grid size this library uses on the current device (the reference
 * value is accepted and ignored by the compress / decompress calls). */
int sleek_thread_blocks(void);

/* Workspace bytes for one compress of insize bytes / one decompress. */
size_t sleek_compress_workspace_size(long long insize);
size_t sleek_decompress_workspace_size(void);

/* Error-bound parameters; replace sleek_error_bound_info<T> and
 * sleek_error_bound<F> (include/sleek_lossy_gpu.h:47-71).  The sign of eb is
 * ignored, as in the reference.  Returns SLEEK_ERR_ERROR_BOUND where the
 * reference would exit(-1). */
typedef struct { int eb_e; int thr_e; unsigned int offs_e; } sleek_eb_info_f32;
typedef struct { int eb_e; int thr_e; unsigned long long offs_e; } sleek_eb_info_f64;
int sleek_error_bound_f32(float eb, sleek_eb_info_f32* info);
int sleek_error_bound_f64(double eb, sleek_eb_info_f64* info);

/* Lossless compress; replaces sleek_compress_gpu(blocks, const float* or const double*, ...)
 * (include/sleek_lossless_gpu.h:47-60, 75-88).  d_encoded must hold
 * sleek_upper_bound_size(num_elements * elemsize) bytes; *d_encsize (device)
 * receives the stream size in bytes. */
int sleek_compress_f32(const float* d_input, long long num_elements, unsigned char* d_encoded,
                       long long* d_encsize, void* d_workspace, size_t workspace_bytes, void* stream);
int sleek_compress_f64(const double* d_input, long long num_elements, unsigned char* d_encoded,
                       long long* d_encsize, void* d_workspace, size_t workspace_bytes, void* stream);

/* Lossless decompress; replaces sleek_decompress_gpu(blocks, const byte*, float* or double*, ...)
 * (include/sleek_lossless_gpu.h:63-72, 91-100).  encoded_bytes bounds every read
 * of the stream and decoded_capacity bounds the output (pass -1 for either to
 * trust the stream, as the reference does); *d_decsize (device) receives the
 * decoded size in bytes. */
int sleek_decompress_f32(const unsigned char* d_encoded, long long encoded_bytes, float* d_decoded,
                         long long decoded_capacity, long long* d_decsize, void* d_workspace,
                         size_t workspace_bytes, void* stream);
int sleek_decompress_f64(const unsigned char* d_encoded, long long encoded_bytes, double* d_decoded,
                         long long decoded_capacity, long long* d_decsize, void* d_workspace,
                         size_t workspace_bytes, void* stream);

/* Absolute-error-bounded lossy compress / decompress; replace the
 * sleek_error_bound_info overloads (include/sleek_lossy_gpu.h:74-99, 102-127).
 * Decompress needs the same eb parameters that compress used (the stream does
 * not record them). */
int sleek_compress_lossy_f32(sleek_eb_info_f32 eb, const float* d_input, long long num_elements,
                             unsigned char* d_encoded, long long* d_encsize, void* d_workspace,
                             size_t workspace_bytes, void* stream);
int sleek_compress_lossy_f64(sleek_eb_info_f64 eb, const double* d_input, long long num_elements,
                             unsigned char* d_encoded, long long* d_encsize, void* d_workspace,
                             size_t workspace_bytes, void* stream);
int sleek_decompress_lossy_f32(sleek_eb_info_f32 eb, const unsigned char* d_encoded, long long encoded_bytes,
                               float* d_decoded, long long decoded_capacity, long long* d_decsize,
                               void* d_workspace, size_t workspace_bytes, void* stream);
int sleek_decompress_lossy_f64(sleek_eb_info_f64 eb, const unsigned char* d_encoded, long long encoded_bytes,
                               double* d_decoded, long long decoded_capacity, long long* d_decsize,
                               void* d_workspace, size_t workspace_bytes, void* stream);

/* Lossless float32 compress that allocates no device memory, for callers that cannot
 * call cudaMalloc (device memory owned by a framework or pool allocator, a fixed memory
 * budget, or a path that must not risk the device synchronisation an allocation can
 * cause).  This entry point has no counterpart in the reference.  Its scratch is a
 * file-scope device array inside the library (512 KiB per device, held until the process
 * exits), so inputs are limited to SLEEK_STATIC_MAX_INPUT_BYTES (1 GiB); larger ones are
 * rejected with SLEEK_ERR_TOO_LARGE.  The first call on a device looks up the scratch's
 * device address (cudaGetSymbolAddress, with that device current); with lazy module
 * loading that lookup may load the library's device code, a one-time device allocation
 * and possibly a synchronisation, so make that first call at initialisation time, before
 * any stream capture.  The address is cached per device: calls must not span a
 * cudaDeviceReset of that device.  All calls share the one scratch and it keeps the last
 * call's contents (each call clears what it needs on `stream`), so calls whose executions
 * overlap on the GPU (different streams, no ordering between them) race: order them on
 * one stream.  Output, stream format and host-detected errors are those of
 * sleek_compress_f32; a device-detected error shows only as -status in *d_encsize
 * (sleek_workspace_status does not read the static scratch). */
#define SLEEK_STATIC_MAX_INPUT_BYTES (1ll << 30)
int sleek_compress_f32_static(const float* d_input, long long num_elements, unsigned char* d_encoded,
                              long long* d_encsize, void* stream);

/* Tuning: CTAs per SM used by the single-buffer entry points of one kind on the current
 * device, for every input size (0 = as many as fit, the default).  Set by
 * sleek_b200.autotune; no counterpart in the reference, whose grid size comes from
 * sleek_thread_blocks and whose block size is the constant SLEEK_TPB
 * (include/sleek_common_gpu.h:54-56, 108-119). */
int sleek_set_ctas_per_sm(int decompress, int elem_bytes, int lossy, int ctas_per_sm);

/* Tuning: launch shapes.  The single-buffer kernels are built in a few shapes (threads per
 * CTA, compute warps, shared-memory chunk stages, and the CTAs per SM their registers are
 * budgeted for); shape 0 is the default, and every shape writes the same bytes.
 * sleek_launch_shape_info describes shape `shape` of the compress (decompress = 0) or
 * decompress kernels (any output pointer may be NULL) and returns SLEEK_ERR_INVALID_ARG
 * past the last one.  sleek_set_launch_shape selects the shape and the CTAs per SM (0 = as
 * many as fit) of the single-buffer calls of one kind on the current device for inputs of
 * [2^size_log2, 2^(size_log2 + 1)) bytes -- decompress: the decoded size, taken from
 * decoded_capacity, else encoded_bytes -- or for every size with size_log2 = -1.  Set by
 * sleek_b200.autotune from timings on the caller's data. */
int sleek_launch_shape_info(int decompress, int shape, int* threads, int* warps, int* stages, int* ctas_per_sm);
int sleek_set_launch_shape(int decompress, int elem_bytes, int lossy, int size_log2, int shape, int ctas_per_sm);

/* ---- batched compress / decompress ---------------------------------------------
 * Many buffers of uneven sizes with mixed float32 / float64 and mixed error bounds in
 * one persistent launch (per group of up to 1024 buffers).  The batched form has no
 * single counterpart in the reference, whose API takes one buffer per call
 * (include/sleek_lossless_gpu.h:47-100, include/sleek_lossy_gpu.h:74-127); every buffer's
 * stream is bit-identical to what the single-buffer call produces for it. */
typedef struct {
  const void* input;        /* compress: device values; decompress: device stream (8-byte aligned) */
  void* output;             /* compress: device stream, >= sleek_upper_bound_size bytes; decompress: device values */
  long long* size_out;      /* device: bytes written (stream or decoded), or -status */
  long long num_elements;   /* compress: input elements; decompress: output capacity in elements */
  long long stream_bytes;   /* decompress: stream length, -1 = trust the stream; ignored by compress */
  int elem_bytes;           /* 4 = float, 8 = double */
  int lossy;                /* 0 = lossless, 1 = absolute error bound */
  double error_bound;       /* lossy only; same rules as sleek_error_bound_f32/_f64 */
} sleek_batch_item;

typedef struct sleek_batch_plan sleek_batch_plan;

/* Validates the items, derives the quantizer parameters and uploads the job tables
 * (allocates device memory and synchronises: call it outside stream capture). */
int sleek_batch_plan_create(const sleek_batch_item* items, int n, int decompress, sleek_batch_plan** plan);
/* A reusable plan with room for `capacity` items (at most 1024): device tables and a
 * pinned staging area are allocated once, then sleek_batch_plan_set_items replaces the
 * item list with an asynchronous upload on `stream` (no allocation, no host wait), so a
 * serving loop can launch batch after batch.  Call set_items again only after the
 * previous run of the same plan has completed (the staging area is reused). */
int sleek_batch_plan_create_reusable(int capacity, int decompress, sleek_batch_plan** plan);
int sleek_batch_plan_set_items(sleek_batch_plan* plan, const sleek_batch_item* items, int n, void* stream);
/* Workspace bytes a run of the plan needs. */
size_t sleek_batch_plan_workspace_size(const sleek_batch_plan* plan);
/* Tuning: CTAs per SM of the plan's launches (0 = as many as fit). */
int sleek_batch_plan_set_grid(sleek_batch_plan* plan, int ctas_per_sm);
/* Clears the workspace and launches on `stream`: no host work and no allocation, so a
 * run can be captured in a CUDA graph.  Runs sharing a workspace must be stream-ordered. */
int sleek_batch_plan_run(sleek_batch_plan* plan, void* d_workspace, size_t workspace_bytes, void* stream);
int sleek_batch_plan_destroy(sleek_batch_plan* plan);
/* One-shot forms: create a plan, run it, wait for `stream`, destroy it (d_workspace
 * may be NULL: then a temporary one is allocated). */
int sleek_compress_batch(const sleek_batch_item* items, int n, void* d_workspace, size_t workspace_bytes, void* stream);
int sleek_decompress_batch(const sleek_batch_item* items, int n, void* d_workspace, size_t workspace_bytes, void* stream);

/* Synchronises `stream` and reads the device status of the last call that used
 * d_workspace (NULL = the library-owned workspace of the current device and
 * `stream`).  *status receives SLEEK_OK or the first device-side error. */
int sleek_workspace_status(const void* d_workspace, void* stream, int* status);

/* ---- compressed transfers between device and host --------------------------
 * The "compressing memory copy" use of the codec (the reference's README:1,4;
 * its copy baseline is memcpy.cu:111-139): only the stream crosses PCIe.
 *
 * sleek_compress_to_host compresses a device array (elem_bytes 4 or 8, lossy 0/1,
 * error_bound used when lossy) and leaves the complete stream -- byte for byte
 * what sleek_compress_* writes -- in HOST memory h_encoded (h_capacity bytes;
 * sleek_upper_bound_size always suffices), its length in *encoded_bytes.
 * sleek_decompress_from_host checks the header, size table and payload bounds
 * of a stream held in host memory (the device decoder checks every chunk),
 * then decompresses it into device memory d_decoded (capacity_bytes), the byte
 * count in *decoded_bytes; a malformed stream is SLEEK_ERR_CORRUPT_STREAM either way.
 *
 * Both cut the array into segments of segment_bytes (0 = 32 MiB, rounded up to
 * whole 16 KB chunks) so that the copy of one segment, on a library-owned copy
 * stream, overlaps the codec work of the next on `stream` (NULL = legacy default
 * stream).  Host buffers should be pinned (cudaMallocHost / cudaHostRegister) for
 * the copies to overlap.  Both return when the result is complete; calls on one
 * (device, stream) are serialised, calls on different streams run concurrently
 * (e.g. a download thread and an upload thread keep both PCIe directions busy).
 * Device staging: two segments' worth, kept per (device, stream). */
int sleek_compress_to_host(const void* d_input, long long num_elements, int elem_bytes, int lossy, double error_bound,
                           unsigned char* h_encoded, long long h_capacity, long long* encoded_bytes,
                           long long segment_bytes, void* stream);
int sleek_decompress_from_host(const unsigned char* h_encoded, long long encoded_bytes, int elem_bytes, int lossy,
                               double error_bound, void* d_decoded, long long capacity_bytes, long long* decoded_bytes,
                               long long segment_bytes, void* stream);

/* ---- stream validation (host) ----------------------------------------------
 * Parses a stream in HOST memory (no device call) and checks every rule the
 * device decoders enforce: the 8-byte header (original size non-negative and a
 * multiple of elem_bytes), the size table and every payload inside stream_len,
 * each csize in [1, chunk bytes] and at least 34 for a compressed chunk, every
 * subchunk bit width <= 8 * elem_bytes, the widths adding up to the csize, and
 * the trailer equal to the chunk's byte count.  A stream passes exactly when
 * the device decoders, given the same stream_len, accept it.  Returns SLEEK_OK
 * or SLEEK_ERR_CORRUPT_STREAM (info says where and why), SLEEK_ERR_INVALID_ARG
 * for a null pointer or an element size other than 4 or 8.  The reference has
 * no such tool; its decoders trap on a malformed chunk (sleek_common_gpu.h:753,1264)
 * and read out of bounds on a malformed table. */
#define SLEEK_STREAM_OK             0
#define SLEEK_STREAM_SHORT_HEADER   1  /* fewer than 8 bytes */
#define SLEEK_STREAM_BAD_SIZE       2  /* original size negative or not a multiple of elem_bytes */
#define SLEEK_STREAM_SHORT_TABLE    3  /* the size table runs past stream_len */
#define SLEEK_STREAM_BAD_CHUNK_SIZE 4  /* csize 0, above the chunk's bytes, or below 34 while compressed */
#define SLEEK_STREAM_SHORT_PAYLOAD  5  /* a payload runs past stream_len */
#define SLEEK_STREAM_BAD_WIDTH      6  /* a subchunk bit width above the element width */
#define SLEEK_STREAM_SIZE_MISMATCH  7  /* the bit widths do not add up to the csize */
#define SLEEK_STREAM_BAD_TRAILER    8  /* the trailer differs from the chunk's byte count */

/* ---- Serving loop (continuous batching in a thread of the library) ---------------
 * No counterpart in the reference, whose calls take one buffer each.  Requests are
 * admitted once their arrival time (on the server's clock, sleek_server_now) has come
 * and their output fits in the server's device arena (next-fit, coalescing), and run
 * with the batched kernels on `slots` streams: an idle stream takes every admitted
 * request waiting at that moment (at most max_batch, at most max_batch_chunks 16 KB
 * chunks).  A request that can never run (output larger than the arena, more chunks
 * than a launch holds) completes at once with -SLEEK_ERR_CAPACITY, and so do waiting
 * requests when nothing on the GPU can free memory.  Results equal the single-buffer
 * entry points' for the same request alone. */
typedef struct sleek_server_s* sleek_server;

typedef struct {
  const void* input;        /* device: values (compress) or stream (decompress) */
  long long num_elements;   /* compress: input elements; decompress: elements it decodes to */
  long long stream_bytes;   /* decompress: stream length (>= 8); ignored by compress */
  double arrival_s;         /* admitted from this time on the server's clock (<= now: at once) */
  double error_bound;       /* lossy only */
  long long tag;            /* the caller's id, returned with the completion */
  int op;                   /* 0 = compress, 1 = decompress */
  int elem_bytes;           /* 4 = float, 8 = double */
  int lossy;                /* 0 = lossless, 1 = absolute error bound */
  int keep;                 /* 1: the output stays in the arena until sleek_server_release */
} sleek_server_request;

typedef struct {
  long long tag;
  long long result_bytes;   /* bytes written (stream or values), or -status */
  void* output;             /* kept outputs: device address in the arena; otherwise NULL */
  double arrival_s;         /* the request's arrival time */
  double done_s;            /* when the server saw its launch complete (server clock) */
} sleek_server_completion;

/* d_arena: device memory for the outputs (256-byte aligned; NULL = the server allocates
 * arena_bytes itself).  Starts the server's thread and its clock. */
int sleek_server_create(void* d_arena, long long arena_bytes, int slots, int max_batch, long long max_batch_chunks,
                        sleek_server* server);
int sleek_server_now(sleek_server server, double* seconds);
/* Thread-safe; the requests' inputs must stay valid until they complete. */
int sleek_server_submit(sleek_server server, const sleek_server_request* requests, long long n);
/* Moves up to `capacity` completions into `out` (*n of them), waiting up to wait_ms
 * for the first one; returns a CUDA failure of the server's own loop, if any. */
int sleek_server_poll(sleek_server server, sleek_server_completion* out, long long capacity, long long* n,
                      int wait_ms);
/* Requests submitted and not yet delivered as completions (queued or in `poll`'s list). */
int sleek_server_outstanding(sleek_server server, long long* n);
/* The arena's free bytes as the server's loop last left them, and its size. */
int sleek_server_arena_info(sleek_server server, long long* free_bytes, long long* size_bytes);
/* Returns a kept output's memory to the arena. */
int sleek_server_release(sleek_server server, void* output);
/* Finishes every admitted request, then stops the thread and frees the server's
 * resources (requests whose arrival time has not come are dropped). */
int sleek_server_destroy(sleek_server server);
/* Host-only check of the arena's policy: ops[i] > 0 allocates ops[i] bytes (offsets[i]
 * = its offset, -1 if nothing fits); ops[i] <= 0 releases the allocation made by the
 * (-ops[i])-th allocating op (offsets[i] = free bytes afterwards). */
int sleek_server_arena_replay(long long arena_bytes, const long long* ops, long long n, long long* offsets);

typedef struct sleek_stream_info {
  long long insize;        /* original bytes (header), -1 if unreadable */
  long long chunks;        /* chunks the header implies */
  long long stream_bytes;  /* 8 + 2 * chunks + sum of the csizes seen (the whole stream when valid) */
  long long raw_chunks;    /* chunks stored verbatim */
  long long bad_chunk;     /* first malformed chunk, -1 for header / table problems or none */
  int reason;              /* SLEEK_STREAM_* */
  int pad_;
} sleek_stream_info;

int sleek_validate_stream(const unsigned char* h_stream, long long stream_len, int elem_bytes, sleek_stream_info* info);
const char* sleek_stream_reason_string(int reason);

/* Self-test of the device-side time limits (no counterpart in the reference, whose
 * waits are unbounded): a one-warp kernel waits on an mbarrier that nothing arrives
 * on and looks back over a predecessor flag that nothing publishes, each limited to
 * limit_ns (0 < limit_ns <= 10 s), with the same wait helpers as the codec kernels.
 * h_result[0] = 1 if the barrier wait gave up, h_result[1] = the look-back's result
 * (-1 when it gave up), h_result[2] = nanoseconds both waits took.  Synchronous on
 * the legacy default stream; the device stays usable. */
int sleek_selftest_bounded_waits(long long limit_ns, long long* h_result);

/* Self-test of the device value maps (no counterpart in the reference): on the current
 * device, compares what the codec kernels compute -- the lossless transform and its
 * inverse, quantize and dequantize (whose rounding division runs in floating point) --
 * with a literal restatement of the reference's integer steps (include/sleek_common_gpu.h:
 * forward :356-374, inverse :614-632, quantize :776-802, dequantize :1077-1108).
 * Checks, in h_counts[0..SLEEK_SELFTEST_VALUE_CHECKS-1]:
 *   0  float32 transform and inverse, every 32-bit word
 *   1  float32 quantize, every word, error-bound exponents 0 1 2 24 100 127 200 230
 *   2  float32 dequantize, every code, the same exponents
 *   3  float64 transform and inverse, every sign/exponent field x 2^20 seeded mantissas
 *   4  float64 quantize, the same words, error-bound exponents 0 1 2 53 500 1000 1023 1500 1993
 *   5  float64 dequantize, every code below 2^32 (also the narrow form) and 2^32 codes
 *      spread over every bit length, the same exponents
 * Each entry receives the number of mismatching inputs (0 when the maps agree), and
 * h_first (optional) the first failing index of each check (-1 if none).  Synchronous
 * on the legacy default stream, well under a second on a B200. */
#define SLEEK_SELFTEST_VALUE_CHECKS 6
int sleek_selftest_value_maps(long long* h_counts, long long* h_first);

/* Value range of a device array, NaNs ignored: *h_min and *h_max (host memory)
 * receive its smallest and largest value (NaN when the array has no non-NaN
 * value or is empty).  One HBM-bound pass on `stream` (NULL = legacy default
 * stream), then a wait for it; uses the library-owned workspace of `stream`.
 * Replaces the host loop of the range-relative error bound in the reference's
 * ARTIFACT drivers (computeNOAeb, lossy_compressors_gpu/sleek_single_compressor_lossy.cu:59-75,
 * sleek_double_compressor_lossy.cu:59-75), whose eb is (max - min) * parameter.
 * Where the input holds NaNs the reference's result depends on its OpenMP
 * schedule; this one ignores them. */
int sleek_minmax_f32(const float* d_input, long long num_elements, float* h_min, float* h_max, void* stream);
int sleek_minmax_f64(const double* d_input, long long num_elements, double* h_min, double* h_max, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SLEEK_CAPI_H */
