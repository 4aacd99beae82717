// sleek_batch.cu -- batched compress / decompress: many buffers of uneven sizes,
// mixed float32 / float64 and mixed error bounds in one persistent launch per
// group of up to BATCH_MAX_JOBS buffers.
//
// A plan validates the buffers, derives each buffer's quantizer parameters and
// chunk ids, and uploads the job tables once; running it only clears the
// workspace and launches (no host work, no allocation), so a run can be captured
// in a CUDA graph and replayed.  Streams are bit-identical to the single-buffer
// entry points (the batched look-back is segmented per buffer).
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/sleek_capi.h"
#include "sleek_launch.h"

namespace {

constexpr long long CS = 16384;
constexpr int HDR_WORDS = 32;

struct Group {
  sleek::BatchJob* d_jobs = nullptr;
  long long* d_cb = nullptr;
  int njobs = 0;
  long long chunks = 0;  // compress: chunks; decompress: chunks the capacities allow
  size_t ws_bytes = 0;
};

}  // namespace

struct sleek_batch_plan {
  int decompress = 0;
  int device = 0;
  int grid_scale = 0;  // CTAs per SM; 0 = as many as fit
  std::vector<Group> groups;
  size_t ws_bytes = 0;
  // reusable plans: one group whose tables are refilled from pinned staging
  int capacity = 0;
  sleek::BatchJob* h_jobs = nullptr;
  long long* h_cb = nullptr;
};

namespace {

int fill_job(const sleek_batch_item& it, int decompress, sleek::BatchJob& j)
{
  if (it.elem_bytes != 4 && it.elem_bytes != 8) return SLEEK_ERR_INVALID_ARG;
  if (!it.size_out || it.num_elements < 0) return SLEEK_ERR_INVALID_ARG;
  if (it.num_elements > 0 && (!it.input || !it.output)) return SLEEK_ERR_INVALID_ARG;
  if (!it.output || (decompress && !it.input)) return SLEEK_ERR_INVALID_ARG;
  const int w = it.elem_bytes;
  // the largest input the single-buffer entry points accept (2^52 bytes): larger
  // counts would overflow the byte and chunk arithmetic below
  if (it.num_elements > (1ll << 52) / w) return SLEEK_ERR_INVALID_ARG;
  const uintptr_t in = reinterpret_cast<uintptr_t>(it.input);
  const uintptr_t out = reinterpret_cast<uintptr_t>(it.output);
  if (decompress ? ((in & 7u) || (out % w)) : ((in % w) || (out & 7u))) return SLEEK_ERR_ALIGNMENT;
  j.in = static_cast<const uint8_t*>(it.input);
  j.out = static_cast<uint8_t*>(it.output);
  j.outsize = it.size_out;
  j.kind = (w == 8 ? 1 : 0) | (it.lossy ? 2 : 0);
  j.q.eb_e = 0;
  j.q.thr_e = 0;
  j.q.offs = 0;
  if (it.lossy) {
    if (w == 4) {
      sleek_eb_info_f32 e;
      const int rc = sleek_error_bound_f32(static_cast<float>(it.error_bound), &e);
      if (rc) return rc;
      j.q.eb_e = e.eb_e;
      j.q.thr_e = e.thr_e;
      j.q.offs = e.offs_e;
    } else {
      sleek_eb_info_f64 e;
      const int rc = sleek_error_bound_f64(it.error_bound, &e);
      if (rc) return rc;
      j.q.eb_e = e.eb_e;
      j.q.thr_e = e.thr_e;
      j.q.offs = e.offs_e;
    }
  }
  const long long bytes = it.num_elements * w;
  j.chunks = (bytes + CS - 1) / CS;
  if (decompress) {
    j.insize = it.stream_bytes < 0 ? -1 : it.stream_bytes;
    j.cap = bytes;
    if (j.insize >= 0 && j.insize < 8) return SLEEK_ERR_CORRUPT_STREAM;
  } else {
    j.insize = bytes;
    j.cap = 0;
  }
  return SLEEK_OK;
}

void free_plan(sleek_batch_plan* p)
{
  for (auto& g : p->groups) {
    if (g.d_jobs) cudaFree(g.d_jobs);
    if (g.d_cb) cudaFree(g.d_cb);
  }
  if (p->h_jobs) cudaFreeHost(p->h_jobs);
  if (p->h_cb) cudaFreeHost(p->h_cb);
  delete p;
}

int grid_for(const sleek_batch_plan* p, long long chunks)
{
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
  int bps = p->decompress ? sleek::decode_batch_blocks_per_sm() : sleek::encode_batch_blocks_per_sm();
  if (bps < 1) bps = 1;
  if (p->grid_scale > 0 && p->grid_scale < bps) bps = p->grid_scale;
  long long g = static_cast<long long>(sms > 0 ? sms : 1) * bps;
  if (!p->decompress && g > chunks) g = chunks > 0 ? chunks : 1;
  return static_cast<int>(g);
}

}  // namespace

extern "C" {

int sleek_batch_plan_create(const sleek_batch_item* items, int n, int decompress, sleek_batch_plan** plan)
{
  if (!plan || n < 0 || (n > 0 && !items)) return SLEEK_ERR_INVALID_ARG;
  *plan = nullptr;
  // every item is checked before anything touches the device
  for (int i = 0; i < n; ++i) {
    sleek::BatchJob scratch;
    const int rc = fill_job(items[i], decompress ? 1 : 0, scratch);
    if (rc) return rc;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  sleek_batch_plan* p = new (std::nothrow) sleek_batch_plan();
  if (!p) return SLEEK_ERR_INVALID_ARG;
  p->decompress = decompress ? 1 : 0;
  p->device = dev;
  for (int b = 0; b < n; b += sleek::BATCH_MAX_JOBS) {
    const int m = (n - b) < sleek::BATCH_MAX_JOBS ? (n - b) : sleek::BATCH_MAX_JOBS;
    std::vector<sleek::BatchJob> jobs(m);
    std::vector<long long> cb(m + 1);
    long long total = 0;
    for (int i = 0; i < m; ++i) {
      const int rc = fill_job(items[b + i], p->decompress, jobs[i]);
      if (rc) {
        free_plan(p);
        return rc;
      }
      cb[i] = total;
      total += jobs[i].chunks;
    }
    cb[m] = total;
    Group g;
    g.njobs = m;
    g.chunks = total;
    g.ws_bytes = p->decompress ? static_cast<size_t>(8 * (HDR_WORDS + total + 2 * m))
                               : static_cast<size_t>(8 * (HDR_WORDS + total));
    if (cudaMalloc(&g.d_jobs, sizeof(sleek::BatchJob) * m) != cudaSuccess ||
        cudaMalloc(&g.d_cb, sizeof(long long) * (m + 1)) != cudaSuccess ||
        cudaMemcpy(g.d_jobs, jobs.data(), sizeof(sleek::BatchJob) * m, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g.d_cb, cb.data(), sizeof(long long) * (m + 1), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      p->groups.push_back(g);
      free_plan(p);
      return SLEEK_ERR_CUDA;
    }
    p->groups.push_back(g);
    if (g.ws_bytes > p->ws_bytes) p->ws_bytes = g.ws_bytes;
  }
  *plan = p;
  return SLEEK_OK;
}

int sleek_batch_plan_create_reusable(int capacity, int decompress, sleek_batch_plan** plan)
{
  if (!plan || capacity < 1 || capacity > sleek::BATCH_MAX_JOBS) return SLEEK_ERR_INVALID_ARG;
  *plan = nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_NO_DEVICE;
  }
  sleek_batch_plan* p = new (std::nothrow) sleek_batch_plan();
  if (!p) return SLEEK_ERR_INVALID_ARG;
  p->decompress = decompress ? 1 : 0;
  p->device = dev;
  p->capacity = capacity;
  Group g;
  if (cudaMalloc(&g.d_jobs, sizeof(sleek::BatchJob) * capacity) != cudaSuccess ||
      cudaMalloc(&g.d_cb, sizeof(long long) * (capacity + 1)) != cudaSuccess ||
      cudaMallocHost(&p->h_jobs, sizeof(sleek::BatchJob) * capacity) != cudaSuccess ||
      cudaMallocHost(&p->h_cb, sizeof(long long) * (capacity + 1)) != cudaSuccess) {
    cudaGetLastError();
    p->groups.push_back(g);
    free_plan(p);
    return SLEEK_ERR_CUDA;
  }
  p->groups.push_back(g);
  *plan = p;
  return SLEEK_OK;
}

int sleek_batch_plan_set_items(sleek_batch_plan* plan, const sleek_batch_item* items, int n, void* stream)
{
  if (!plan || plan->capacity == 0 || n < 0 || n > plan->capacity || (n > 0 && !items)) return SLEEK_ERR_INVALID_ARG;
  Group& g = plan->groups[0];
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    const int rc = fill_job(items[i], plan->decompress, plan->h_jobs[i]);
    if (rc) return rc;
    plan->h_cb[i] = total;
    total += plan->h_jobs[i].chunks;
  }
  plan->h_cb[n] = total;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((n > 0 && cudaMemcpyAsync(g.d_jobs, plan->h_jobs, sizeof(sleek::BatchJob) * n, cudaMemcpyHostToDevice, st) !=
                    cudaSuccess) ||
      cudaMemcpyAsync(g.d_cb, plan->h_cb, sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, st) != cudaSuccess) {
    cudaGetLastError();
    return SLEEK_ERR_CUDA;
  }
  g.njobs = n;
  g.chunks = total;
  g.ws_bytes = plan->decompress ? static_cast<size_t>(8 * (HDR_WORDS + total + 2 * n))
                                : static_cast<size_t>(8 * (HDR_WORDS + total));
  plan->ws_bytes = g.ws_bytes;
  return SLEEK_OK;
}

size_t sleek_batch_plan_workspace_size(const sleek_batch_plan* plan) { return plan ? plan->ws_bytes : 0; }

int sleek_batch_plan_set_grid(sleek_batch_plan* plan, int ctas_per_sm)
{
  if (!plan || ctas_per_sm < 0) return SLEEK_ERR_INVALID_ARG;
  plan->grid_scale = ctas_per_sm;
  return SLEEK_OK;
}

int sleek_batch_plan_run(sleek_batch_plan* plan, void* d_workspace, size_t workspace_bytes, void* stream)
{
  if (!plan || !d_workspace) return SLEEK_ERR_INVALID_ARG;
  if (workspace_bytes < plan->ws_bytes) return SLEEK_ERR_WORKSPACE;
  if (reinterpret_cast<uintptr_t>(d_workspace) & 7u) return SLEEK_ERR_ALIGNMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint64_t* const ws = static_cast<uint64_t*>(d_workspace);
  for (const Group& g : plan->groups) {
    if (g.njobs == 0) continue;
    if (cudaMemsetAsync(ws, 0, g.ws_bytes, st) != cudaSuccess) {
      cudaGetLastError();
      return SLEEK_ERR_CUDA;
    }
    cudaError_t e;
    if (plan->decompress) {
      sleek::BatchDecArgs a;
      a.jobs = g.d_jobs;
      a.chunk_base = g.d_cb;
      a.njobs = g.njobs;
      a.ws = ws;
      a.offsets = reinterpret_cast<long long*>(ws + HDR_WORDS);
      a.actual = a.offsets + g.chunks;
      a.actual_insize = a.actual + g.njobs;
      e = sleek::launch_decode_batch(a, grid_for(plan, g.chunks), st);
    } else {
      sleek::BatchEncArgs a;
      a.jobs = g.d_jobs;
      a.chunk_base = g.d_cb;
      a.njobs = g.njobs;
      a.ws = ws;
      e = sleek::launch_encode_batch(a, grid_for(plan, g.chunks), st);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      return SLEEK_ERR_CUDA;
    }
  }
  return SLEEK_OK;
}

int sleek_batch_plan_destroy(sleek_batch_plan* plan)
{
  if (plan) free_plan(plan);
  return SLEEK_OK;
}

static int one_shot(const sleek_batch_item* items, int n, int decompress, void* ws, size_t wsb, void* stream)
{
  sleek_batch_plan* p = nullptr;
  int rc = sleek_batch_plan_create(items, n, decompress, &p);
  if (rc) return rc;
  void* w = ws;
  bool own = false;
  if (!w) {
    if (cudaMalloc(&w, p->ws_bytes > 0 ? p->ws_bytes : 8) != cudaSuccess) {
      cudaGetLastError();
      free_plan(p);
      return SLEEK_ERR_CUDA;
    }
    wsb = p->ws_bytes;
    own = true;
  }
  rc = sleek_batch_plan_run(p, w, wsb, stream);
  if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess && rc == SLEEK_OK) {
    cudaGetLastError();
    rc = SLEEK_ERR_CUDA;
  }
  if (own) cudaFree(w);
  free_plan(p);
  return rc;
}

int sleek_compress_batch(const sleek_batch_item* items, int n, void* d_workspace, size_t workspace_bytes, void* stream)
{
  return one_shot(items, n, 0, d_workspace, workspace_bytes, stream);
}

int sleek_decompress_batch(const sleek_batch_item* items, int n, void* d_workspace, size_t workspace_bytes,
                           void* stream)
{
  return one_shot(items, n, 1, d_workspace, workspace_bytes, stream);
}

}  // extern "C"
