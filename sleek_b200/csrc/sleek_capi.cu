// sleek_capi.cu -- the C ABI declared in include/sleek_capi.h.
//
// Host-side argument checks, grid sizing from the occupancy of the kernels on
// the current device, workspace handling and error-bound derivation.  All
// compute happens in sleek_kernels.cu; there is no CPU fallback.
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include <cuda_runtime.h>

#include "../../include/sleek_capi.h"
#include "sleek_launch.h"

namespace {

constexpr long long CS = 16384;
// workspace header layout, as in sleek_device.cuh (WsWord)
constexpr int HDR_WORDS = 32;
constexpr int WS_STATUS = 2;
constexpr int WS_BLOCK = 8;
constexpr int WS_EPOCH = 16;
constexpr int WS_MINMAX = 24;

constexpr int SHAPES_MAX = 8;
constexpr int BUCKETS = 64;  // input sizes by their base-2 logarithm

// what the single-buffer calls of one kind launch for one size bucket
struct Choice {
  int shape = 0;  // launch shape (sleek_kernels.cu: EncShape*, DecShape*)
  int ctas = 0;   // CTAs per SM, 0 = as many as fit
};

struct DeviceInfo {
  int sms = 0;
  int bps[2][2][2][SHAPES_MAX] = {};  // [width==8][lossy][enc][shape]: CTAs per SM that fit
  Choice choice[2][2][2][BUCKETS];    // [width==8][lossy][enc][size bucket]
};

int size_bucket(long long bytes)
{
  if (bytes <= 0) return 0;
  int b = 0;
  while (b < BUCKETS - 1 && (bytes >> (b + 1)) != 0) ++b;
  return b;
}

// A library-owned workspace: zeroed once when allocated, then kept clean by the
// kernels themselves (two counter blocks and two flag regions used by alternate
// launches, see WsPhase in sleek_device.cuh), so calls need no clearing pass.
struct OwnedWs {
  void* ptr = nullptr;
  long long flag_cap = 0;  // flags per region
};

std::mutex g_mu;
std::map<int, DeviceInfo> g_dev;
std::map<std::pair<int, cudaStream_t>, OwnedWs> g_ws;

int current_device(int* dev)
{
  if (cudaGetDevice(dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  return SLEEK_OK;
}

// Persistent grid and launch shape of a single-buffer call of `bytes` bytes
// (bytes < 0: unknown, the default shape).
int persistent_grid(int dev, int width, bool lossy, bool enc, long long bytes, int* shape)
{
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceInfo& d = g_dev[dev];
  if (d.sms == 0) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    d.sms = sms > 0 ? sms : 1;
  }
  const Choice c = bytes < 0 ? Choice{} : d.choice[width == 8][lossy][enc][size_bucket(bytes)];
  int& b = d.bps[width == 8][lossy][enc][c.shape];
  if (b == 0) {
    const int n = sleek::blocks_per_sm(width, lossy, enc, c.shape);
    b = n > 0 ? n : 1;
  }
  *shape = c.shape;
  return d.sms * ((c.ctas > 0 && c.ctas < b) ? c.ctas : b);
}

// library-owned workspace for (device, stream) with room for `need_flags` flags per
// region; grows, never shrinks.  A new one is zeroed on `st` (the only clearing it
// ever needs).
int owned_workspace(int dev, cudaStream_t st, long long need_flags, OwnedWs* out)
{
  std::lock_guard<std::mutex> lk(g_mu);
  OwnedWs& e = g_ws[{dev, st}];
  if (e.ptr == nullptr || e.flag_cap < need_flags) {
    if (e.ptr) {
      cudaStreamSynchronize(st);
      cudaFree(e.ptr);
      e.ptr = nullptr;
      e.flag_cap = 0;
    }
    long long cap = 1 << 10;  // flags per region: 16 MB of input, doubling as needed
    while (cap < need_flags) cap <<= 1;
    const size_t bytes = static_cast<size_t>(8 * (HDR_WORDS + 2 * cap));
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return SLEEK_ERR_CUDA;
    }
    if (cudaMemsetAsync(p, 0, bytes, st) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(p);
      return SLEEK_ERR_CUDA;
    }
    e.ptr = p;
    e.flag_cap = cap;
  }
  *out = e;
  return SLEEK_OK;
}

// The workspace of one single-buffer launch that uses `need_flags` look-back flags:
// the library-owned one of (device, stream) when user_ws is NULL (no clearing: it
// resets itself), else the caller's, checked and cleared on `st` (epoch 0, so only
// the first flag region is used).
int prepare_workspace(cudaStream_t st, void* user_ws, size_t user_bytes, long long need_flags, uint64_t** ws,
                      long long* flag_cap)
{
  int dev = 0;
  int rc = current_device(&dev);
  if (rc) return rc;
  if (user_ws == nullptr) {
    OwnedWs o;
    rc = owned_workspace(dev, st, need_flags, &o);
    if (rc) return rc;
    *ws = static_cast<uint64_t*>(o.ptr);
    *flag_cap = o.flag_cap;
    return SLEEK_OK;
  }
  const size_t need = static_cast<size_t>(8 * (HDR_WORDS + need_flags));
  if (user_bytes < need) return SLEEK_ERR_WORKSPACE;
  if (reinterpret_cast<uintptr_t>(user_ws) & 7u) return SLEEK_ERR_ALIGNMENT;
  if (cudaMemsetAsync(user_ws, 0, need, st) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  *ws = static_cast<uint64_t*>(user_ws);
  *flag_cap = need_flags;
  return SLEEK_OK;
}

long long enc_flags(long long insize) { return (insize + CS - 1) / CS; }

size_t enc_ws_bytes(long long insize) { return static_cast<size_t>(8 * (HDR_WORDS + enc_flags(insize))); }

size_t dec_ws_bytes(int grid) { return static_cast<size_t>(8 * (HDR_WORDS + grid)); }

int do_compress(int width, bool lossy, sleek::QParams q, const void* in, long long n, unsigned char* out,
                long long* outsize, void* ws, size_t wsb, void* stream)
{
  if (!in && n > 0) return SLEEK_ERR_INVALID_ARG;
  if (!out || !outsize || n < 0) return SLEEK_ERR_INVALID_ARG;
  if (reinterpret_cast<uintptr_t>(in) % width) return SLEEK_ERR_ALIGNMENT;
  if (reinterpret_cast<uintptr_t>(out) & 7u) return SLEEK_ERR_ALIGNMENT;
  if (n > (1ll << 52) / width) return SLEEK_ERR_INVALID_ARG;
  int dev = 0;
  int rc = current_device(&dev);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long insize = n * width;
  const long long chunks = (insize + CS - 1) / CS;
  uint64_t* w = nullptr;
  long long cap = 0;
  rc = prepare_workspace(st, ws, wsb, enc_flags(insize), &w, &cap);
  if (rc) return rc;
  sleek::EncArgs a;
  a.in = static_cast<const uint8_t*>(in);
  a.insize = insize;
  a.out = out;
  a.outsize = outsize;
  a.ws = w;
  a.flag_cap = cap;
  a.q = q;
  int shape = 0;
  long long grid = persistent_grid(dev, width, lossy, true, insize, &shape);
  if (grid > chunks) grid = chunks > 0 ? chunks : 1;
  if (sleek::launch_encode(width, lossy, shape, a, static_cast<int>(grid), st) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  return SLEEK_OK;
}

int do_decompress(int width, bool lossy, sleek::QParams q, const unsigned char* in, long long in_len, void* out,
                  long long out_cap, long long* outsize, void* ws, size_t wsb, void* stream)
{
  if (!in || !outsize) return SLEEK_ERR_INVALID_ARG;
  if (!out && out_cap != 0) return SLEEK_ERR_INVALID_ARG;
  if (reinterpret_cast<uintptr_t>(in) & 7u) return SLEEK_ERR_ALIGNMENT;
  if (reinterpret_cast<uintptr_t>(out) % width) return SLEEK_ERR_ALIGNMENT;
  if (in_len >= 0 && in_len < 8) return SLEEK_ERR_CORRUPT_STREAM;
  int dev = 0;
  int rc = current_device(&dev);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int shape = 0;
  const int grid = persistent_grid(dev, width, lossy, false, out_cap >= 0 ? out_cap : in_len, &shape);
  uint64_t* w = nullptr;
  long long cap = 0;
  rc = prepare_workspace(st, ws, wsb, grid, &w, &cap);
  if (rc) return rc;
  sleek::DecArgs a;
  a.in = in;
  a.in_len = in_len < 0 ? -1 : in_len;
  a.out = static_cast<uint8_t*>(out);
  a.out_cap = out_cap < 0 ? -1 : out_cap;
  a.outsize = outsize;
  a.ws = w;
  a.flag_cap = cap;
  a.q = q;
  if (sleek::launch_decode(width, lossy, shape, a, grid, st) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  return SLEEK_OK;
}

sleek::QParams qp(int eb_e, int thr_e, unsigned long long offs)
{
  sleek::QParams q;
  q.eb_e = eb_e;
  q.thr_e = thr_e;
  q.offs = offs;
  return q;
}

}  // namespace

namespace sleek {

// entry points for other host sources of the library (library-owned workspace of `stream`)
int host_compress(int width, bool lossy, QParams q, const void* in, long long n, unsigned char* out,
                  long long* outsize, void* stream)
{
  return do_compress(width, lossy, q, in, n, out, outsize, nullptr, 0, stream);
}

int host_decompress(int width, bool lossy, QParams q, const unsigned char* in, long long in_len, void* out,
                    long long cap, long long* outsize, void* stream)
{
  return do_decompress(width, lossy, q, in, in_len, out, cap, outsize, nullptr, 0, stream);
}

int host_qparams(int width, bool lossy, double eb, QParams* q)
{
  q->eb_e = 0;
  q->thr_e = 0;
  q->offs = 0;
  if (!lossy) return SLEEK_OK;
  if (width == 4) {
    sleek_eb_info_f32 e;
    const int rc = sleek_error_bound_f32(static_cast<float>(eb), &e);
    if (rc) return rc;
    *q = qp(e.eb_e, e.thr_e, e.offs_e);
  } else {
    sleek_eb_info_f64 e;
    const int rc = sleek_error_bound_f64(eb, &e);
    if (rc) return rc;
    *q = qp(e.eb_e, e.thr_e, e.offs_e);
  }
  return SLEEK_OK;
}

}  // namespace sleek

namespace {

template <typename F, typename U>
int minmax(const F* in, long long n, F* h_min, F* h_max, void* stream)
{
  if (!h_min || !h_max || n < 0 || (n > 0 && !in)) return SLEEK_ERR_INVALID_ARG;
  if (reinterpret_cast<uintptr_t>(in) % sizeof(F)) return SLEEK_ERR_ALIGNMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0;
  int rc = current_device(&dev);
  if (rc) return rc;
  // the two keys live in the range-reduction words of the library-owned workspace
  OwnedWs o;
  rc = owned_workspace(dev, st, 0, &o);
  if (rc) return rc;
  uint64_t* const w = static_cast<uint64_t*>(o.ptr) + WS_MINMAX;
  if (cudaMemsetAsync(w, 0, 16, st) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  unsigned long long keys[2] = {0ull, 0ull};
  if (sleek::launch_minmax(static_cast<int>(sizeof(F)), in, n, reinterpret_cast<unsigned long long*>(w),
                           sms > 0 ? sms : 1, st) != cudaSuccess ||
      cudaMemcpyAsync(keys, w, sizeof(keys), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  constexpr U top = static_cast<U>(1) << (8 * sizeof(U) - 1);
  // a key with the top bit set came from a non-negative value, otherwise from a negative one
  auto value = [&](U k) {
    const U bits = (k & top) ? static_cast<U>(k ^ top) : static_cast<U>(~k);
    F f;
    std::memcpy(&f, &bits, sizeof(F));
    return f;
  };
  if (keys[1] == 0ull) {  // no value that is not NaN
    const U nan = sizeof(U) == 4 ? static_cast<U>(0x7fc00000u) : static_cast<U>(0x7ff8000000000000ull);
    std::memcpy(h_min, &nan, sizeof(F));
    std::memcpy(h_max, &nan, sizeof(F));
    return SLEEK_OK;
  }
  *h_min = value(static_cast<U>(~static_cast<U>(keys[0])));  // keys[0]: inverted key of the minimum
  *h_max = value(static_cast<U>(keys[1]));                   // keys[1]: key of the maximum
  return SLEEK_OK;
}

}  // namespace

extern "C" {

const char* sleek_status_string(int s)
{
  switch (s) {
    case SLEEK_OK: return "ok";
    case SLEEK_ERR_INVALID_ARG: return "invalid argument";
    case SLEEK_ERR_ALIGNMENT: return "misaligned pointer";
    case SLEEK_ERR_CUDA: return "CUDA runtime error";
    case SLEEK_ERR_ERROR_BOUND: return "error bound too large";
    case SLEEK_ERR_CORRUPT_STREAM: return "corrupt compressed stream";
    case SLEEK_ERR_TIMEOUT: return "device wait timed out";
    case SLEEK_ERR_WORKSPACE: return "workspace too small";
    case SLEEK_ERR_NO_DEVICE: return "no CUDA device";
    case SLEEK_ERR_CAPACITY: return "output capacity exceeded";
    case SLEEK_ERR_TOO_LARGE: return "input larger than the static scratch allows";
    default: return "unknown status";
  }
}

long long sleek_upper_bound_size(long long insize)
{
  const long long chunks = (insize + CS - 1) / CS;
  return 3 * 4 + chunks * 2 + chunks * CS;
}

int sleek_system_checks(void)
{
  const int one = 1;
  unsigned char c;
  std::memcpy(&c, &one, 1);
  if (c != 1) return -1;
  if (sizeof(long long) != 8 || sizeof(int) != 4 || sizeof(short) != 2 || sizeof(char) != 1) return -1;
  return 0;
}

int sleek_thread_blocks(void)
{
  int dev = 0;
  if (current_device(&dev)) return 0;
  int shape = 0;
  return persistent_grid(dev, 4, false, true, -1, &shape);
}

size_t sleek_compress_workspace_size(long long insize) { return insize < 0 ? 0 : enc_ws_bytes(insize); }

size_t sleek_decompress_workspace_size(void)
{
  int dev = 0;
  if (current_device(&dev)) return dec_ws_bytes(148 * 32);
  // the largest persistent grid of any decode kind and shape
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int g = 0;
  for (int w = 4; w <= 8; w += 4)
    for (int l = 0; l < 2; l++)
      for (int sh = 0; sh < sleek::shape_count(false); ++sh) {
        const int x = (sms > 0 ? sms : 1) * sleek::blocks_per_sm(w, l != 0, false, sh);
        g = x > g ? x : g;
      }
  return dec_ws_bytes(g);
}

int sleek_error_bound_f32(float eb, sleek_eb_info_f32* info)
{
  if (!info) return SLEEK_ERR_INVALID_ARG;
  uint32_t bits;
  std::memcpy(&bits, &eb, 4);
  const int e = static_cast<int>((bits >> 23) & 0xffu);
  const int t = e + 24;
  if (t >= 255) return SLEEK_ERR_ERROR_BOUND;
  info->eb_e = e;
  info->thr_e = t;
  info->offs_e = (static_cast<uint32_t>(t) << 23) - (1u << 23);
  return SLEEK_OK;
}

int sleek_error_bound_f64(double eb, sleek_eb_info_f64* info)
{
  if (!info) return SLEEK_ERR_INVALID_ARG;
  uint64_t bits;
  std::memcpy(&bits, &eb, 8);
  const int e = static_cast<int>((bits >> 52) & 0x7ffu);
  const int t = e + 53;
  if (t >= 2047) return SLEEK_ERR_ERROR_BOUND;
  info->eb_e = e;
  info->thr_e = t;
  info->offs_e = (static_cast<uint64_t>(t) << 52) - (1ull << 52);
  return SLEEK_OK;
}

int sleek_compress_f32(const float* in, long long n, unsigned char* out, long long* outsize, void* ws, size_t wsb,
                       void* stream)
{
  return do_compress(4, false, qp(0, 0, 0), in, n, out, outsize, ws, wsb, stream);
}

int sleek_compress_f64(const double* in, long long n, unsigned char* out, long long* outsize, void* ws, size_t wsb,
                       void* stream)
{
  return do_compress(8, false, qp(0, 0, 0), in, n, out, outsize, ws, wsb, stream);
}

int sleek_decompress_f32(const unsigned char* in, long long in_len, float* out, long long cap, long long* outsize,
                         void* ws, size_t wsb, void* stream)
{
  return do_decompress(4, false, qp(0, 0, 0), in, in_len, out, cap, outsize, ws, wsb, stream);
}

int sleek_decompress_f64(const unsigned char* in, long long in_len, double* out, long long cap, long long* outsize,
                         void* ws, size_t wsb, void* stream)
{
  return do_decompress(8, false, qp(0, 0, 0), in, in_len, out, cap, outsize, ws, wsb, stream);
}

int sleek_compress_lossy_f32(sleek_eb_info_f32 eb, const float* in, long long n, unsigned char* out,
                             long long* outsize, void* ws, size_t wsb, void* stream)
{
  if (eb.thr_e != eb.eb_e + 24 || eb.thr_e >= 255 || eb.eb_e < 0) return SLEEK_ERR_ERROR_BOUND;
  return do_compress(4, true, qp(eb.eb_e, eb.thr_e, eb.offs_e), in, n, out, outsize, ws, wsb, stream);
}

int sleek_compress_lossy_f64(sleek_eb_info_f64 eb, const double* in, long long n, unsigned char* out,
                             long long* outsize, void* ws, size_t wsb, void* stream)
{
  if (eb.thr_e != eb.eb_e + 53 || eb.thr_e >= 2047 || eb.eb_e < 0) return SLEEK_ERR_ERROR_BOUND;
  return do_compress(8, true, qp(eb.eb_e, eb.thr_e, eb.offs_e), in, n, out, outsize, ws, wsb, stream);
}

int sleek_decompress_lossy_f32(sleek_eb_info_f32 eb, const unsigned char* in, long long in_len, float* out,
                               long long cap, long long* outsize, void* ws, size_t wsb, void* stream)
{
  if (eb.thr_e != eb.eb_e + 24 || eb.thr_e >= 255 || eb.eb_e < 0) return SLEEK_ERR_ERROR_BOUND;
  return do_decompress(4, true, qp(eb.eb_e, eb.thr_e, eb.offs_e), in, in_len, out, cap, outsize, ws, wsb, stream);
}

int sleek_decompress_lossy_f64(sleek_eb_info_f64 eb, const unsigned char* in, long long in_len, double* out,
                               long long cap, long long* outsize, void* ws, size_t wsb, void* stream)
{
  if (eb.thr_e != eb.eb_e + 53 || eb.thr_e >= 2047 || eb.eb_e < 0) return SLEEK_ERR_ERROR_BOUND;
  return do_decompress(8, true, qp(eb.eb_e, eb.thr_e, eb.offs_e), in, in_len, out, cap, outsize, ws, wsb, stream);
}

int sleek_set_ctas_per_sm(int decompress, int elem_bytes, int lossy, int ctas_per_sm)
{
  if ((elem_bytes != 4 && elem_bytes != 8) || ctas_per_sm < 0) return SLEEK_ERR_INVALID_ARG;
  int dev = 0;
  const int rc = current_device(&dev);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_mu);
  for (Choice& c : g_dev[dev].choice[elem_bytes == 8][lossy != 0][decompress == 0]) c.ctas = ctas_per_sm;
  return SLEEK_OK;
}

int sleek_launch_shape_info(int decompress, int shape, int* threads, int* warps, int* stages, int* ctas_per_sm)
{
  if (shape < 0 || shape >= sleek::shape_count(decompress == 0)) return SLEEK_ERR_INVALID_ARG;
  const sleek::ShapeInfo i = sleek::shape_info(decompress == 0, shape);
  if (threads) *threads = i.threads;
  if (warps) *warps = i.warps;
  if (stages) *stages = i.stages;
  if (ctas_per_sm) *ctas_per_sm = i.ctas_per_sm;
  return SLEEK_OK;
}

int sleek_set_launch_shape(int decompress, int elem_bytes, int lossy, int size_log2, int shape, int ctas_per_sm)
{
  if ((elem_bytes != 4 && elem_bytes != 8) || ctas_per_sm < 0 || size_log2 < -1 || size_log2 >= BUCKETS ||
      shape < 0 || shape >= sleek::shape_count(decompress == 0))
    return SLEEK_ERR_INVALID_ARG;
  int dev = 0;
  const int rc = current_device(&dev);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_mu);
  Choice* row = g_dev[dev].choice[elem_bytes == 8][lossy != 0][decompress == 0];
  for (int b = 0; b < BUCKETS; ++b)
    if (size_log2 < 0 || b == size_log2) row[b] = Choice{shape, ctas_per_sm};
  return SLEEK_OK;
}

int sleek_minmax_f32(const float* in, long long n, float* h_min, float* h_max, void* stream)
{
  return minmax<float, uint32_t>(in, n, h_min, h_max, stream);
}

int sleek_minmax_f64(const double* in, long long n, double* h_min, double* h_max, void* stream)
{
  return minmax<double, uint64_t>(in, n, h_min, h_max, stream);
}

int sleek_workspace_status(const void* ws, void* stream, int* status)
{
  if (!status) return SLEEK_ERR_INVALID_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const void* p = ws;
  if (!p) {
    int dev = 0;
    int rc = current_device(&dev);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_ws.find({dev, st});
    if (it == g_ws.end()) {
      *status = SLEEK_OK;
      return SLEEK_OK;
    }
    p = it->second.ptr;
  }
  unsigned long long h[HDR_WORDS];
  if (cudaStreamSynchronize(st) != cudaSuccess ||
      cudaMemcpy(h, p, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  // the last single-buffer launch worked in the counter block of parity epoch - 1;
  // batched runs (epoch 0) in block 0
  const unsigned long long e = h[WS_EPOCH];
  *status = static_cast<int>(h[(e ? ((e - 1) & 1) : 0) * WS_BLOCK + WS_STATUS]);
  return SLEEK_OK;
}

}  // extern "C"
