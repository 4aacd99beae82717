// sleek_driver.cpp -- command-line compressor / decompressor over the sm_100a
// library, with the argv and stdout of the reference's GPU drivers
// (lossless_compressors_gpu/sleek_{single,double}_{compressor,decompressor}.cu,
// lossy_compressors_gpu/sleek_{single,double}_{compressor,decompressor}_lossy.cu),
// so that scripts which run those programs and parse their output
// (compress_decompress_inputs_*.py, verify_cpu_gpu_*.py) run unchanged.
//
// One source, built sixteen ways:
//   SLEEK_DOUBLE      0: float data, 1: double data
//   SLEEK_LOSSY       0: lossless,   1: absolute-error-bounded lossy
//   SLEEK_DECOMPRESS  0: compressor, 1: decompressor
//   ARTIFACT          defined: warm-up + timed call, time and throughput lines, and
//                     a range-relative error bound, (max - min) * parameter, with
//                     max and min taken on the device (sleek_minmax_*); the lossy
//                     decompressor also takes the original file and checks the
//                     point-wise bound (the reference's MAXABS report)
//
// Every line the reference prints is printed with the same format, in the same
// order, except the two banner lines, which name this implementation.  Errors
// that the reference leaves to an assert, a trap or a crash (unreadable files,
// malformed streams) are reported on stderr with exit status 255.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "sleek_capi.h"

#ifndef SLEEK_DOUBLE
#define SLEEK_DOUBLE 0
#endif
#ifndef SLEEK_LOSSY
#define SLEEK_LOSSY 0
#endif
#ifndef SLEEK_DECOMPRESS
#define SLEEK_DECOMPRESS 0
#endif

#if SLEEK_DOUBLE
using F = double;
static const char* const PREC = "double";
[[maybe_unused]] static const char* const CHECK_NAME = "MAXABS_d64";
[[maybe_unused]] static F parse_value(const char* s) { return std::stod(s); }
#else
using F = float;
static const char* const PREC = "single";
[[maybe_unused]] static const char* const CHECK_NAME = "MAXABS_f32";
[[maybe_unused]] static F parse_value(const char* s) { return std::stof(s); }
#endif

using byte = unsigned char;

namespace {

struct Timer {
  cudaEvent_t beg, end;
  Timer()
  {
    cudaEventCreate(&beg);
    cudaEventCreate(&end);
  }
  ~Timer()
  {
    cudaEventDestroy(beg);
    cudaEventDestroy(end);
  }
  void start() { cudaEventRecord(beg, 0); }
  double stop()
  {
    cudaEventRecord(end, 0);
    cudaEventSynchronize(end);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, beg, end);
    return 0.001 * ms;
  }
};

void check_cuda(const int line)
{
  cudaDeviceSynchronize();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "CUDA error %d on line %d: %s\n\n", e, line, cudaGetErrorString(e));
    exit(-1);
  }
}

int fail(const char* what, const int status)
{
  fprintf(stderr, "ERROR: %s: %s\n\n", what, sleek_status_string(status));
  return -1;
}

// whole file into pinned host memory; -1 if unreadable
long long read_file(const char* name, byte** buf)
{
  FILE* const f = fopen(name, "rb");
  if (!f) return -1;
  fseek(f, 0, SEEK_END);
  const long long size = ftell(f);
  fseek(f, 0, SEEK_SET);
  *buf = nullptr;
  if (size > 0) {
    if (cudaMallocHost(reinterpret_cast<void**>(buf), static_cast<size_t>(size)) != cudaSuccess) {
      fclose(f);
      return -1;
    }
    const long long got = static_cast<long long>(fread(*buf, 1, static_cast<size_t>(size), f));
    if (got != size) {
      fclose(f);
      return -1;
    }
  }
  fclose(f);
  return size;
}

// allocation or copy that must succeed; otherwise report and exit with 255
void must(const cudaError_t e, const char* what)
{
  if (e != cudaSuccess) {
    fprintf(stderr, "ERROR: %s failed: %s\n\n", what, cudaGetErrorString(e));
    exit(-1);
  }
}

bool write_file(const char* name, const byte* buf, long long size)
{
  FILE* const f = fopen(name, "wb");
  if (!f) return false;
  const bool ok = static_cast<long long>(fwrite(buf, 1, static_cast<size_t>(size), f)) == size;
  return fclose(f) == 0 && ok;
}

#if SLEEK_LOSSY
int error_bound_info(const F eb, sleek_eb_info_f32* i32, sleek_eb_info_f64* i64)
{
#if SLEEK_DOUBLE
  (void)i32;
  const int rc = sleek_error_bound_f64(eb, i64);
#else
  (void)i64;
  const int rc = sleek_error_bound_f32(eb, i32);
#endif
  if (rc == SLEEK_ERR_ERROR_BOUND) {
    fprintf(stderr, "ERROR: error_bound is too large\n");
    exit(-1);
  }
  return rc;
}
#endif

#if defined(ARTIFACT) && SLEEK_LOSSY
// (max - min) * parameter of the values in device memory, with the range lines
F range_relative_bound(const F* d_values, long long n, const F parameter)
{
  F lo = 0, hi = 0;
#if SLEEK_DOUBLE
  const int rc = sleek_minmax_f64(d_values, n, &lo, &hi, nullptr);
#else
  const int rc = sleek_minmax_f32(d_values, n, &lo, &hi, nullptr);
#endif
  if (rc != SLEEK_OK) exit(fail("sleek_minmax", rc));
  printf("min_val: %.10f\n", lo);
  printf("max_val: %.10f\n", hi);
  printf("diff between max and min values: %.10f\n", (hi - lo));
  return (hi - lo) * parameter;
}
#endif

#if defined(ARTIFACT) && SLEEK_LOSSY && SLEEK_DECOMPRESS
// Point-wise check of a reconstruction against the original, reported in the
// reference's MAXABS format (lossy_compressors_gpu/MAXABS_f32.h:40-95): values
// where either side is infinite or NaN must be equal (two NaNs count as equal);
// every other value must lie within [orig - eb, orig + eb] and |orig - recon| <= eb
// in the data's own precision.
void check_bound(const long long size, const F* recon, const F* orig, const F eb)
{
  if (size % static_cast<long long>(sizeof(F)) != 0) {
    fprintf(stderr, "ERROR: %s requires data to be a multiple of %ld bytes long\n", CHECK_NAME, sizeof(F));
    exit(-1);
  }
  if (eb <= 0) {
    fprintf(stderr, "ERROR: %s requires the maximum allowed absolute error to be greater than zero\n", CHECK_NAME);
    exit(-1);
  }
  const long long len = size / static_cast<long long>(sizeof(F));
  F max_diff = 0;
  long long over = 0, nonfinite = 0;
  F lo = orig[0], hi = orig[0];  // NaN in the first place stays: every comparison with it is false
  for (long long i = 0; i < len; i++) {
    const F o = orig[i], r = recon[i];
    if (o < lo) lo = o;
    else if (o > hi) hi = o;
    if (!std::isfinite(o) || !std::isfinite(r)) {
      if (r != o && !(std::isnan(o) && std::isnan(r))) {
        if (nonfinite == 0)
          fprintf(stderr,
                  "%s ERROR: absolute error bound exceeded due to NaN or INF at position %lld: reconstructed value is "
                  "'%.10f' vs original value: '%.10f'\n\n",
                  CHECK_NAME, i, r, o);
        nonfinite++;
      }
    } else {
      const F d = std::abs(o - r);
      max_diff = std::max(max_diff, d);
      const F lower = o - eb, upper = o + eb;
      if (r < lower || r > upper || d > eb) over++;
    }
  }
  if (over == 0 && nonfinite == 0) printf("%s verification passed\n", CHECK_NAME);
  printf("min_val: %.10f\n", lo);
  printf("max_val: %.10f\n", hi);
  printf("diff between max and min values in original input: %.10f\n", (hi - lo));
  printf("num_eb_violations: %lld (%.2f%%) \n", over, 100.0 * (static_cast<float>(over) / len));
  printf("max_diff between original and reconstructed values: %.10f\n", max_diff);
  printf("inf_nan_violations: %lld (%.2f%%) \n", nonfinite, 100.0 * static_cast<float>(nonfinite) / len);
  printf("Number of values in original file: %lld\n", len);
}
#endif

// one library call on the legacy default stream (no wait)
#if !SLEEK_DECOMPRESS
int run(const F* d_in, long long n, byte* d_out, long long* d_size, const sleek_eb_info_f32& e32,
        const sleek_eb_info_f64& e64)
{
  (void)e32;
  (void)e64;
#if SLEEK_LOSSY && SLEEK_DOUBLE
  return sleek_compress_lossy_f64(e64, d_in, n, d_out, d_size, nullptr, 0, nullptr);
#elif SLEEK_LOSSY
  return sleek_compress_lossy_f32(e32, d_in, n, d_out, d_size, nullptr, 0, nullptr);
#elif SLEEK_DOUBLE
  return sleek_compress_f64(d_in, n, d_out, d_size, nullptr, 0, nullptr);
#else
  return sleek_compress_f32(d_in, n, d_out, d_size, nullptr, 0, nullptr);
#endif
}
#else
int run(const byte* d_in, long long in_len, F* d_out, long long cap, long long* d_size, const sleek_eb_info_f32& e32,
        const sleek_eb_info_f64& e64)
{
  (void)e32;
  (void)e64;
#if SLEEK_LOSSY && SLEEK_DOUBLE
  return sleek_decompress_lossy_f64(e64, d_in, in_len, d_out, cap, d_size, nullptr, 0, nullptr);
#elif SLEEK_LOSSY
  return sleek_decompress_lossy_f32(e32, d_in, in_len, d_out, cap, d_size, nullptr, 0, nullptr);
#elif SLEEK_DOUBLE
  return sleek_decompress_f64(d_in, in_len, d_out, cap, d_size, nullptr, 0, nullptr);
#else
  return sleek_decompress_f32(d_in, in_len, d_out, cap, d_size, nullptr, 0, nullptr);
#endif
}
#endif

// the size a call wrote, or exit with the status it reported
long long result_size(const long long* d_size, const char* what)
{
  long long v = 0;
  if (cudaMemcpy(&v, d_size, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) exit(fail(what, SLEEK_ERR_CUDA));
  if (v < 0) exit(fail(what, static_cast<int>(-v)));
  return v;
}

}  // namespace

int main(int argc, char* argv[])
{
  printf("SLEEK-B200 GPU codec: %s-precision %s %s\n", PREC, SLEEK_LOSSY ? "lossy" : "lossless",
         SLEEK_DECOMPRESS ? "decompressor" : "compressor");
  printf("sm_100a build of the SLEEK stream format\n\n");

  const char* const in_name = SLEEK_DECOMPRESS ? "compressed_file_name" : "input_file_name";
  const char* const out_name = SLEEK_DECOMPRESS ? "decompressed_file_name" : "compressed_file_name";
#if SLEEK_LOSSY && SLEEK_DECOMPRESS && defined(ARTIFACT)
  if (argc != 5) {
    printf("USAGE: %s %s %s error_bound original_file_name\n\n", argv[0], in_name, out_name);
    return -1;
  }
#elif SLEEK_LOSSY
  if (argc != 4) {
    printf("USAGE: %s %s %s error_bound\n\n", argv[0], in_name, out_name);
    return -1;
  }
#else
  if (argc != 3) {
    printf("USAGE: %s %s %s\n\n", argv[0], in_name, out_name);
    return -1;
  }
#endif

  if (sleek_system_checks() != 0) return -1;

  sleek_eb_info_f32 e32{};
  sleek_eb_info_f64 e64{};

#if !SLEEK_DECOMPRESS
  // ---------------------------------- compressor ----------------------------------
  byte* input = nullptr;
  const long long insize = read_file(argv[1], &input);
  if (insize == -1) {
    fprintf(stderr, "ERROR: cannot read %s\n\n", argv[1]);
    return -1;
  }
  if (insize <= 0) {
    fprintf(stderr, "ERROR: input file too small\n\n");
    return -1;
  }
  const long long num_elements = insize / static_cast<long long>(sizeof(F));
  printf("original size: %lld bytes\n", insize);
  if (insize % static_cast<long long>(sizeof(F)) != 0) {
    fprintf(stderr, "ERROR: size of input must be a multiple of %ld bytes\n", sizeof(F));
    return -1;
  }

  const long long maxsize = sleek_upper_bound_size(insize);
  byte* encoded = nullptr;
  F* d_input = nullptr;
  byte* d_encoded = nullptr;
  long long* d_encsize = nullptr;
  must(cudaMallocHost(reinterpret_cast<void**>(&encoded), static_cast<size_t>(maxsize)), "host allocation");
  must(cudaMalloc(reinterpret_cast<void**>(&d_input), static_cast<size_t>(insize)), "device allocation");
  must(cudaMemcpy(d_input, input, static_cast<size_t>(insize), cudaMemcpyHostToDevice), "copy to the device");
  must(cudaMalloc(reinterpret_cast<void**>(&d_encoded), static_cast<size_t>(maxsize)), "device allocation");
  must(cudaMalloc(reinterpret_cast<void**>(&d_encsize), sizeof(long long)), "device allocation");
  check_cuda(__LINE__);

#if defined(ARTIFACT)
#if SLEEK_LOSSY
  const F parameter = parse_value(argv[3]);
  const F eb = range_relative_bound(d_input, num_elements, parameter);
  if (int rc = error_bound_info(eb, &e32, &e64)) return fail("sleek_error_bound", rc);
#endif
  int rc = run(d_input, num_elements, d_encoded, d_encsize, e32, e64);  // warm up
  if (rc) return fail("compress", rc);
  check_cuda(__LINE__);
  Timer timer;
  timer.start();
  rc = run(d_input, num_elements, d_encoded, d_encsize, e32, e64);
  const double runtime = timer.stop();
  if (rc) return fail("compress", rc);
  const long long encsize = result_size(d_encsize, "compress");
  must(cudaMemcpy(encoded, d_encoded, static_cast<size_t>(encsize), cudaMemcpyDeviceToHost), "copy to the host");
  printf("encoded size: %lld bytes\n", encsize);
  check_cuda(__LINE__);
  const float CR = (100.0 * encsize) / insize;
  printf("ratio: %6.2f%% %7.3fx\n", CR, 100.0 / CR);
  printf("encoding time: %.6f s\n", runtime);
  const double throughput = insize * 0.000000001 / runtime;
  printf("encoding throughput: %8.3f Gbytes/s\n", throughput);
  check_cuda(__LINE__);
#else
#if SLEEK_LOSSY
  const F eb = parse_value(argv[3]);
  if (int rc = error_bound_info(eb, &e32, &e64)) return fail("sleek_error_bound", rc);
#endif
  if (int rc = run(d_input, num_elements, d_encoded, d_encsize, e32, e64)) return fail("compress", rc);
  const long long encsize = result_size(d_encsize, "compress");
  must(cudaMemcpy(encoded, d_encoded, static_cast<size_t>(encsize), cudaMemcpyDeviceToHost), "copy to the host");
  printf("encoded size: %lld bytes\n", encsize);
  check_cuda(__LINE__);
  const float CR = (100.0 * encsize) / insize;
  printf("ratio: %6.2f%% %7.3fx\n", CR, 100.0 / CR);
#endif

  if (!write_file(argv[2], encoded, encsize)) {
    fprintf(stderr, "ERROR: cannot write %s\n\n", argv[2]);
    return -1;
  }
  cudaFree(d_input);
  cudaFree(d_encoded);
  cudaFree(d_encsize);
  check_cuda(__LINE__);
  cudaFreeHost(input);
  cudaFreeHost(encoded);
  return 0;

#else
  // --------------------------------- decompressor ---------------------------------
  byte* encoded = nullptr;
  const long long insize = read_file(argv[1], &encoded);
  if (insize < 8) {
    fprintf(stderr, "ERROR: cannot read a stream header from %s\n\n", argv[1]);
    return -1;
  }
  // pre-flight: the whole stream is checked on the host before any device work
  sleek_stream_info info;
  if (sleek_validate_stream(encoded, insize, static_cast<int>(sizeof(F)), &info) != SLEEK_OK) {
    fprintf(stderr, "ERROR: %s: %s (chunk %lld)\n\n", sleek_status_string(SLEEK_ERR_CORRUPT_STREAM),
            sleek_stream_reason_string(info.reason), info.bad_chunk);
    return -1;
  }
  const long long pre_size = info.insize;
  printf("encoded size: %lld bytes\n", insize);

  byte* decoded = nullptr;
  byte* d_encoded = nullptr;
  F* d_decoded = nullptr;
  long long* d_decsize = nullptr;
  must(cudaMallocHost(reinterpret_cast<void**>(&decoded), static_cast<size_t>(std::max(pre_size, 1ll))),
       "host allocation");
  must(cudaMalloc(reinterpret_cast<void**>(&d_encoded), static_cast<size_t>(insize)), "device allocation");
  must(cudaMemcpy(d_encoded, encoded, static_cast<size_t>(insize), cudaMemcpyHostToDevice), "copy to the device");
  must(cudaMalloc(reinterpret_cast<void**>(&d_decoded), static_cast<size_t>(std::max(pre_size, 1ll))),
       "device allocation");
  must(cudaMalloc(reinterpret_cast<void**>(&d_decsize), sizeof(long long)), "device allocation");

#if defined(ARTIFACT)
#if SLEEK_LOSSY
  byte* orig = nullptr;
  const long long insize_orig = read_file(argv[4], &orig);
  if (insize_orig == -1) {
    fprintf(stderr, "ERROR: cannot read %s\n\n", argv[4]);
    return -1;
  }
  if (insize_orig <= 0) {
    fprintf(stderr, "ERROR: original input file too small\n\n");
    return -1;
  }
  const F parameter = parse_value(argv[3]);
  F* d_orig = nullptr;
  must(cudaMalloc(reinterpret_cast<void**>(&d_orig), static_cast<size_t>(insize_orig)), "device allocation");
  must(cudaMemcpy(d_orig, orig, static_cast<size_t>(insize_orig), cudaMemcpyHostToDevice), "copy to the device");
  const F eb = range_relative_bound(d_orig, insize_orig / static_cast<long long>(sizeof(F)), parameter);
  cudaFree(d_orig);
  if (int rc = error_bound_info(eb, &e32, &e64)) return fail("sleek_error_bound", rc);
#endif
  int rc = run(d_encoded, insize, d_decoded, pre_size, d_decsize, e32, e64);  // warm up
  if (rc) return fail("decompress", rc);
  (void)result_size(d_decsize, "decompress");
  Timer timer;
  timer.start();
  rc = run(d_encoded, insize, d_decoded, pre_size, d_decsize, e32, e64);
  const double runtime = timer.stop();
  if (rc) return fail("decompress", rc);
  const long long decsize = result_size(d_decsize, "decompress");
  must(cudaMemcpy(decoded, d_decoded, static_cast<size_t>(decsize), cudaMemcpyDeviceToHost), "copy to the host");
  printf("decoded size: %lld bytes\n", decsize);
  check_cuda(__LINE__);
#if SLEEK_LOSSY
  check_bound(insize_orig, reinterpret_cast<const F*>(decoded), reinterpret_cast<const F*>(orig), eb);
#endif
  const float CR = (100.0 * insize) / decsize;
  printf("ratio: %6.2f%% %7.3fx\n", CR, 100.0 / CR);
  printf("decoding time: %.6f s\n", runtime);
  const double throughput = decsize * 0.000000001 / runtime;
  printf("decoding throughput: %8.3f Gbytes/s\n", throughput);
  check_cuda(__LINE__);
#else
#if SLEEK_LOSSY
  const F eb = parse_value(argv[3]);
  if (int rc = error_bound_info(eb, &e32, &e64)) return fail("sleek_error_bound", rc);
#endif
  if (int rc = run(d_encoded, insize, d_decoded, pre_size, d_decsize, e32, e64)) return fail("decompress", rc);
  const long long decsize = result_size(d_decsize, "decompress");
  must(cudaMemcpy(decoded, d_decoded, static_cast<size_t>(decsize), cudaMemcpyDeviceToHost), "copy to the host");
  printf("decoded size: %lld bytes\n", decsize);
  check_cuda(__LINE__);
  const float CR = (100.0 * insize) / decsize;
  printf("ratio: %6.2f%% %7.3fx\n", CR, 100.0 / CR);
#endif

  if (!write_file(argv[2], decoded, decsize)) {
    fprintf(stderr, "ERROR: cannot write %s\n\n", argv[2]);
    return -1;
  }
  cudaFree(d_encoded);
  cudaFree(d_decoded);
  cudaFree(d_decsize);
  check_cuda(__LINE__);
  cudaFreeHost(encoded);
  cudaFreeHost(decoded);
  return 0;
#endif
}
