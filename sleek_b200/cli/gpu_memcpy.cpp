// gpu_memcpy.cpp -- the copy baseline of the reference's measurement scripts
// (memcpy.cu): host-to-device, device-to-device and device-to-host cudaMemcpy of
// one file's bytes, each timed once with CUDA events on the legacy default stream.
// Same argv and the same stdout lines after the banner, so that
// compress_decompress_inputs_*.py can read the DtD throughput from line 8.
#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

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

void report(const char* what, const double seconds, const long long bytes)
{
  printf("%s time: %.6f s\n", what, seconds);
  printf("%s throughput: %8.3f Gbytes/s\n", what, bytes * 0.000000001 / seconds);
}

}  // namespace

int main(int argc, char* argv[])
{
  printf("SLEEK-B200 GPU_memcpy\n");
  printf("copy baseline for the SLEEK codec measurements\n\n");
  if (argc < 2) {
    printf("USAGE: %s file_name\n\n", argv[0]);
    return -1;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    fprintf(stderr, "ERROR: no CUDA capable device detected\n\n");
    exit(-1);
  }
  cudaSetDevice(0);

  FILE* const fin = fopen(argv[1], "rb");
  if (!fin) {
    fprintf(stderr, "ERROR: cannot read %s\n\n", argv[1]);
    return -1;
  }
  fseek(fin, 0, SEEK_END);
  const long long size = ftell(fin);
  if (size <= 0) {
    fprintf(stderr, "ERROR: input file too small\n\n");
    fclose(fin);
    return -1;
  }
  // pageable host memory, as in the reference, so HtD / DtH measure the same path
  unsigned char* const host = new unsigned char[size];
  fseek(fin, 0, SEEK_SET);
  const long long got = static_cast<long long>(fread(host, 1, static_cast<size_t>(size), fin));
  fclose(fin);
  if (got != size) {
    fprintf(stderr, "ERROR: cannot read %s\n\n", argv[1]);
    return -1;
  }
  printf("original size: %lld bytes\n", size);

  unsigned char *d_a = nullptr, *d_b = nullptr;
  cudaMalloc(reinterpret_cast<void**>(&d_a), static_cast<size_t>(size));
  cudaMalloc(reinterpret_cast<void**>(&d_b), static_cast<size_t>(size));
  check_cuda(__LINE__);

  Timer t;
  t.start();
  cudaMemcpy(d_a, host, static_cast<size_t>(size), cudaMemcpyHostToDevice);
  cudaDeviceSynchronize();
  report("HtD", t.stop(), size);

  t.start();
  cudaMemcpy(d_b, d_a, static_cast<size_t>(size), cudaMemcpyDeviceToDevice);
  cudaDeviceSynchronize();
  report("DtD", t.stop(), size);

  t.start();
  cudaMemcpy(host, d_a, static_cast<size_t>(size), cudaMemcpyDeviceToHost);
  cudaDeviceSynchronize();
  report("DtH", t.stop(), size);

  cudaFree(d_a);
  cudaFree(d_b);
  check_cuda(__LINE__);
  delete[] host;
  return 0;
}
