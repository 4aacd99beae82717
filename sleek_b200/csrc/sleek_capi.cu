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
constexpr int HDR_WORDS = 32;  // workspace header words, as in sleek_device.cuh

struct DeviceInfo {
  int sms = 0;
  int bps[2][2][2] = {};       // [width==8][lossy][enc]: CTAs per SM that fit
  int override_[2][2][2] = {};  // tuned CTAs per SM (0 = as many as fit)
};

std::mutex g_mu;
std::map<int, DeviceInfo> g_dev;
std::map<std::pair<int, cudaStream_t>, std::pair<void*, size_t>> g_ws;

int current_device(int* dev)
{
  if (cudaGetDevice(dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  return SLEEK_OK;
}

int persistent_grid(int dev, int width, bool lossy, bool enc)
{
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceInfo& d = g_dev[dev];
  if (d.sms == 0) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    d.sms = sms > 0 ? sms : 1;
  }
  int& b = d.bps[width == 8][lossy][enc];
  if (b == 0) {
    const int n = sleek::blocks_per_sm(width, lossy, enc);
    b = n > 0 ? n : 1;
  }
  const int o = d.override_[width == 8][lossy][enc];
  return d.sms * ((o > 0 && o < b) ? o : b);
}

// library-owned workspace for (device, stream); grows, never shrinks
int owned_workspace(int dev, cudaStream_t st, size_t need, void** ptr)
{
  std::lock_guard<std::mutex> lk(g_mu);
  auto& e = g_ws[{dev, st}];
  if (e.second < need) {
    if (e.first) {
      cudaStreamSynchronize(st);
      cudaFree(e.first);
      e.first = nullptr;
      e.second = 0;
    }
    size_t sz = 1 << 20;
    while (sz < need) sz <<= 1;
    void* p = nullptr;
    if (cudaMalloc(&p, sz) != cudaSuccess) {
      cudaGetLastError();
      return SLEEK_ERR_CUDA;
    }
    e.first = p;
    e.second = sz;
  }
  *ptr = e.first;
  return SLEEK_OK;
}

int prepare_workspace(cudaStream_t st, void* user_ws, size_t user_bytes, size_t need, uint64_t** ws)
{
  int dev = 0;
  int rc = current_device(&dev);
  if (rc) return rc;
  void* p = user_ws;
  if (p == nullptr) {
    rc = owned_workspace(dev, st, need, &p);
    if (rc) return rc;
  } else {
    if (user_bytes < need) return SLEEK_ERR_WORKSPACE;
    if (reinterpret_cast<uintptr_t>(p) & 7u) return SLEEK_ERR_ALIGNMENT;
  }
  if (cudaMemsetAsync(p, 0, need, st) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  *ws = static_cast<uint64_t*>(p);
  return SLEEK_OK;
}

size_t enc_ws_bytes(long long insize)
{
  const long long chunks = (insize + CS - 1) / CS;
  return static_cast<size_t>(8 * (HDR_WORDS + chunks));
}

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
  rc = prepare_workspace(st, ws, wsb, enc_ws_bytes(insize), &w);
  if (rc) return rc;
  sleek::EncArgs a;
  a.in = static_cast<const uint8_t*>(in);
  a.insize = insize;
  a.out = out;
  a.outsize = outsize;
  a.ws = w;
  a.q = q;
  long long grid = persistent_grid(dev, width, lossy, true);
  if (grid > chunks) grid = chunks > 0 ? chunks : 1;
  if (sleek::launch_encode(width, lossy, a, static_cast<int>(grid), st) != cudaSuccess) {
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
  const int grid = persistent_grid(dev, width, lossy, false);
  uint64_t* w = nullptr;
  rc = prepare_workspace(st, ws, wsb, dec_ws_bytes(grid), &w);
  if (rc) return rc;
  sleek::DecArgs a;
  a.in = in;
  a.in_len = in_len < 0 ? -1 : in_len;
  a.out = static_cast<uint8_t*>(out);
  a.out_cap = out_cap < 0 ? -1 : out_cap;
  a.outsize = outsize;
  a.ws = w;
  a.q = q;
  if (sleek::launch_decode(width, lossy, a, grid, st) != cudaSuccess) {
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
  uint64_t* w = nullptr;
  rc = prepare_workspace(st, nullptr, 0, 8 * 3, &w);  // the two keys and a clear status word
  if (rc) return rc;
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
  return persistent_grid(dev, 4, false, true);
}

size_t sleek_compress_workspace_size(long long insize) { return insize < 0 ? 0 : enc_ws_bytes(insize); }

size_t sleek_decompress_workspace_size(void)
{
  int dev = 0;
  if (current_device(&dev)) return dec_ws_bytes(148 * 8);
  int g = 0;
  for (int w = 4; w <= 8; w += 4)
    for (int l = 0; l < 2; l++) {
      const int x = persistent_grid(dev, w, l != 0, false);
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
  g_dev[dev].override_[elem_bytes == 8][lossy != 0][decompress == 0] = ctas_per_sm;
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
    p = it->second.first;
  }
  unsigned long long v = 0;
  if (cudaStreamSynchronize(st) != cudaSuccess ||
      cudaMemcpy(&v, static_cast<const unsigned long long*>(p) + 2, 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  *status = static_cast<int>(v);
  return SLEEK_OK;
}

}  // extern "C"
