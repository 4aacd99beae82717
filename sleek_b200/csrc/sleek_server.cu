// sleek_server.cu -- the serving loop in native code: compress / decompress
// requests of any size, admitted as they arrive and run with continuous batching
// by one thread of the library, so that no interpreter sits between a request's
// arrival, its launch and its completion.
//
// - Outputs live in one device arena (the caller's memory or the server's own),
//   allocated next-fit with coalescing: a request is admitted only when its
//   output fits, and its memory returns to the arena when it completes (or when
//   the caller releases an output it asked to keep).  A request that can never
//   run (output larger than the arena, more chunks than a launch holds) fails at
//   once with SLEEK_ERR_CAPACITY, and so do the waiting requests when nothing on
//   the GPU can free memory: the loop never stalls.
// - `slots` CUDA streams each own a reusable compress plan and a reusable
//   decompress plan (the batched kernels, no allocation per launch); any idle
//   slot takes every admitted request waiting at that moment, up to the plan's
//   capacity and its chunk budget, so requests that arrive while others run join
//   the next launch and launches on different slots overlap on the device.  A
//   launch's sizes come back by an asynchronous copy; the loop completes a slot
//   when its event has passed.
// - Requests carry an arrival time on the server's clock; the loop admits each
//   one once that time has come (a trace can be submitted ahead and replayed),
//   and records when it saw the request's launch complete.
//
// Every result is the stream (or the values) the single-buffer entry points
// produce for the same request alone.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/sleek_capi.h"

namespace {

constexpr long long CS = 16384;
constexpr long long GRANULE = 256;

long long upper_bound(long long insize)
{
  const long long chunks = (insize + CS - 1) / CS;
  return 12 + 2 * chunks + chunks * CS;
}

// Next-fit allocator over [0, size) with coalescing free ranges.  The search
// starts at the free range holding the end of the last allocation and wraps
// around: with outputs freed roughly in arrival order it finds a fit at once
// instead of walking the small holes near the arena's start.
class Arena {
 public:
  explicit Arena(long long size) : size_(size / GRANULE * GRANULE), free_bytes_(size_)
  {
    if (size_ > 0) free_[0] = size_;
  }
  static long long rounded(long long n) { return std::max(GRANULE, (n + GRANULE - 1) / GRANULE * GRANULE); }
  long long size() const { return size_; }
  long long free_bytes() const { return free_bytes_; }

  long long alloc(long long n)
  {
    n = rounded(n);
    if (free_.empty()) return -1;
    auto it = free_.upper_bound(rover_);
    if (it != free_.begin()) --it;
    for (size_t k = 0; k < free_.size(); ++k) {
      const long long s = it->first, e = it->second;
      if (e - s >= n) {
        free_.erase(it);
        if (e - s > n) free_[s + n] = e;
        free_bytes_ -= n;
        rover_ = s + n;
        return s;
      }
      if (++it == free_.end()) it = free_.begin();
    }
    return -1;
  }

  void release(long long off, long long n)
  {
    n = rounded(n);
    long long s = off, e = off + n;
    auto nx = free_.find(e);
    if (nx != free_.end()) {  // merge with the next range
      e = nx->second;
      free_.erase(nx);
    }
    auto it = free_.lower_bound(s);
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->second == s) {  // merge with the previous range
        pv->second = e;
        free_bytes_ += n;
        return;
      }
    }
    free_[s] = e;
    free_bytes_ += n;
  }

 private:
  long long size_;
  long long free_bytes_;
  long long rover_ = 0;
  std::map<long long, long long> free_;  // start -> end
};

using Clock = std::chrono::steady_clock;

struct Req {
  sleek_server_request r;
  long long seq = 0;  // submission order (ties in arrival)
  long long chunks = 0;
  long long out_bytes = 0;
  long long off = -1;
  int index = 0;  // position in its launch's size array
};

struct Earlier {  // arrival, then submission order
  bool operator()(const Req& a, const Req& b) const
  {
    if (a.r.arrival_s != b.r.arrival_s) return a.r.arrival_s < b.r.arrival_s;
    return a.seq < b.seq;
  }
};

struct Slot {
  cudaStream_t st = nullptr;
  sleek_batch_plan* plan[2] = {nullptr, nullptr};  // compress, decompress
  void* ws[2] = {nullptr, nullptr};
  size_t ws_bytes = 0;
  long long* d_sizes = nullptr;
  long long* h_sizes = nullptr;  // pinned
  cudaEvent_t ev = nullptr;
  bool busy = false;
  std::vector<Req> reqs;
};

}  // namespace

struct sleek_server_s {
  int dev = 0;
  unsigned char* base = nullptr;
  bool own_arena = false;
  Arena arena{0};
  int max_batch = 0;
  long long max_chunks = 0;
  std::vector<Slot> slots;
  Clock::time_point t0;

  std::mutex mu;  // guards the members below it
  std::condition_variable cv_in, cv_out;
  std::vector<Req> incoming;
  std::vector<void*> releases;
  std::deque<sleek_server_completion> done;
  long long submitted = 0, finished = 0;
  long long seq = 0;
  bool stop = false;
  int error = SLEEK_OK;  // a CUDA failure of the loop itself
  std::atomic<long long> free_bytes{0};  // the arena's free bytes, as the loop last left them

  // the loop thread's own state
  // requests not yet arrived, in arrival order (a trace submitted in order is
  // appended in constant time per request)
  std::deque<Req> pending;
  std::deque<Req> queue;
  std::unordered_map<const void*, long long> kept;  // kept output -> its bytes
  std::thread th;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

sleek_server_completion completion_of(const Req& q, long long result, void* out, double t)
{
  sleek_server_completion c{};
  c.tag = q.r.tag;
  c.result_bytes = result;
  c.output = out;
  c.arrival_s = q.r.arrival_s;
  c.done_s = t;
  return c;
}

void finish(sleek_server_s* s, std::vector<sleek_server_completion>& out)
{
  if (out.empty()) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto& c : out) s->done.push_back(c);
    s->finished += static_cast<long long>(out.size());
  }
  s->cv_out.notify_all();
  out.clear();
}

// launches one slot's requests: one plan run per direction, then the sizes
int launch(sleek_server_s* s, Slot& sl, std::vector<Req>& reqs, std::vector<sleek_server_completion>& failed)
{
  std::vector<sleek_batch_item> items;
  items.reserve(reqs.size());
  int k = 0;
  std::vector<Req> ok;
  for (int op = 0; op < 2; ++op) {
    items.clear();
    std::vector<size_t> which;
    for (size_t i = 0; i < reqs.size(); ++i) {
      const sleek_server_request& r = reqs[i].r;
      if (r.op != op) continue;
      sleek_batch_item it{};
      it.input = r.input;
      it.output = s->base + reqs[i].off;
      it.size_out = sl.d_sizes + k + static_cast<int>(items.size());
      it.num_elements = r.num_elements;
      it.stream_bytes = op == 0 ? -1 : r.stream_bytes;
      it.elem_bytes = r.elem_bytes;
      it.lossy = r.lossy;
      it.error_bound = r.error_bound;
      items.push_back(it);
      which.push_back(i);
    }
    if (items.empty()) continue;
    int rc = sleek_batch_plan_set_items(sl.plan[op], items.data(), static_cast<int>(items.size()), sl.st);
    if (rc == SLEEK_OK) rc = sleek_batch_plan_run(sl.plan[op], sl.ws[op], sl.ws_bytes, sl.st);
    if (rc != SLEEK_OK) {
      // the whole launch of this direction fails with the plan's status
      const double t = s->now();
      for (size_t i : which) {
        s->arena.release(reqs[i].off, reqs[i].out_bytes);
        failed.push_back(completion_of(reqs[i], -rc, nullptr, t));
      }
      continue;
    }
    for (size_t j = 0; j < which.size(); ++j) {
      Req q = reqs[which[j]];
      q.index = k + static_cast<int>(j);
      ok.push_back(q);
    }
    k += static_cast<int>(items.size());
  }
  if (ok.empty()) return SLEEK_OK;
  if (cudaMemcpyAsync(sl.h_sizes, sl.d_sizes, sizeof(long long) * k, cudaMemcpyDeviceToHost, sl.st) != cudaSuccess ||
      cudaEventRecord(sl.ev, sl.st) != cudaSuccess) {
    cudaGetLastError();
    // the launch cannot be completed by its event: its requests fail now (their
    // memory is returned once the stream has finished with it)
    cudaStreamSynchronize(sl.st);
    cudaGetLastError();
    const double t = s->now();
    for (const Req& q : ok) {
      s->arena.release(q.off, q.out_bytes);
      failed.push_back(completion_of(q, -SLEEK_ERR_CUDA, nullptr, t));
    }
    return SLEEK_ERR_CUDA;
  }
  sl.reqs = std::move(ok);
  sl.busy = true;
  return SLEEK_OK;
}

// admitted requests for one launch, in arrival order: those whose output fits
// now, up to the plan's capacity and chunk budget; the rest keep their places
std::vector<Req> take(sleek_server_s* s)
{
  std::vector<Req> got;
  long long chunks = 0;
  std::deque<Req> keep;
  while (!s->queue.empty()) {
    if (static_cast<int>(got.size()) == s->max_batch) break;
    Req q = std::move(s->queue.front());
    s->queue.pop_front();
    if (chunks + q.chunks <= s->max_chunks) {
      const long long off = s->arena.alloc(q.out_bytes);
      if (off >= 0) {
        q.off = off;
        chunks += q.chunks;
        got.push_back(std::move(q));
        continue;
      }
    }
    keep.push_back(std::move(q));
  }
  while (!keep.empty()) {
    s->queue.push_front(std::move(keep.back()));
    keep.pop_back();
  }
  return got;
}

void loop(sleek_server_s* s)
{
  cudaSetDevice(s->dev);
  std::vector<sleek_server_completion> out;
  std::vector<Req> in;
  std::vector<void*> rel;
  while (true) {
    bool stopping;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      in.swap(s->incoming);
      rel.swap(s->releases);
      stopping = s->stop;
    }
    for (Req& q : in) {
      if (s->pending.empty() || !Earlier()(q, s->pending.back()))
        s->pending.push_back(std::move(q));
      else
        s->pending.insert(std::upper_bound(s->pending.begin(), s->pending.end(), q, Earlier()), std::move(q));
    }
    in.clear();
    for (void* p : rel) {
      auto it = s->kept.find(p);
      if (it != s->kept.end()) {
        s->arena.release(static_cast<unsigned char*>(p) - s->base, it->second);
        s->kept.erase(it);
      }
    }
    rel.clear();

    // completions
    for (Slot& sl : s->slots) {
      if (!sl.busy) continue;
      const cudaError_t e = cudaEventQuery(sl.ev);
      if (e == cudaErrorNotReady) continue;
      const double t = s->now();
      for (const Req& q : sl.reqs) {
        const long long res = e == cudaSuccess ? sl.h_sizes[q.index] : -SLEEK_ERR_CUDA;
        void* p = nullptr;
        if (q.r.keep && res >= 0) {
          p = s->base + q.off;
          s->kept[p] = q.out_bytes;
        } else {
          s->arena.release(q.off, q.out_bytes);
        }
        out.push_back(completion_of(q, res, p, t));
      }
      if (e != cudaSuccess) cudaGetLastError();
      sl.reqs.clear();
      sl.busy = false;
    }

    // arrivals: requests whose time has come join the admission queue
    const double t = s->now();
    while (!s->pending.empty() && s->pending.front().r.arrival_s <= t) {
      Req q = std::move(s->pending.front());
      s->pending.pop_front();
      if (Arena::rounded(q.out_bytes) > s->arena.size() || q.chunks > s->max_chunks)
        out.push_back(completion_of(q, -SLEEK_ERR_CAPACITY, nullptr, t));
      else
        s->queue.push_back(std::move(q));
    }

    // dispatch to idle slots (again after a launch that failed: it returned its
    // requests' memory, which may admit others)
    bool busy = false;
    for (bool retry = true; retry;) {
      retry = false;
      for (Slot& sl : s->slots) {
        if (s->queue.empty()) break;
        if (sl.busy) continue;
        std::vector<Req> reqs = take(s);
        if (reqs.empty()) break;
        if (launch(s, sl, reqs, out) != SLEEK_OK) {
          std::lock_guard<std::mutex> lk(s->mu);
          s->error = SLEEK_ERR_CUDA;
        }
        if (!sl.busy) retry = true;
      }
      busy = false;
      for (const Slot& sl : s->slots) busy = busy || sl.busy;
      retry = retry && !busy && !s->queue.empty();
    }
    if (!s->queue.empty() && !busy) {
      // nothing on the GPU can free memory: what waits cannot be admitted
      const double tf = s->now();
      for (const Req& q : s->queue) out.push_back(completion_of(q, -SLEEK_ERR_CAPACITY, nullptr, tf));
      s->queue.clear();
    }
    s->free_bytes.store(s->arena.free_bytes(), std::memory_order_relaxed);
    finish(s, out);

    if (stopping && !busy && s->queue.empty()) break;
    // idle policy: while launches are in flight, poll them back to back (a timed
    // sleep rounds up to tens of microseconds, which would land in every
    // request's latency); otherwise sleep until the next arrival or a submission
    if (busy) {
      std::this_thread::yield();
    } else {
      std::unique_lock<std::mutex> lk(s->mu);
      if (!s->incoming.empty() || !s->releases.empty() || s->stop) continue;
      double wait = 1e-3;
      if (!s->pending.empty()) wait = std::min(wait, std::max(0.0, s->pending.front().r.arrival_s - s->now()));
      // a timed wait overshoots by tens of microseconds: arrivals that close are
      // waited for by yielding
      if (wait < 200e-6) {
        lk.unlock();
        std::this_thread::yield();
        continue;
      }
      s->cv_in.wait_for(lk, std::chrono::duration<double>(wait - 100e-6));
    }
  }
}

void destroy_resources(sleek_server_s* s)
{
  for (Slot& sl : s->slots) {
    if (sl.st) cudaStreamSynchronize(sl.st);
    for (int op = 0; op < 2; ++op) {
      if (sl.plan[op]) sleek_batch_plan_destroy(sl.plan[op]);
      if (sl.ws[op]) cudaFree(sl.ws[op]);
    }
    if (sl.d_sizes) cudaFree(sl.d_sizes);
    if (sl.h_sizes) cudaFreeHost(sl.h_sizes);
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.st) cudaStreamDestroy(sl.st);
  }
  s->slots.clear();
  if (s->own_arena && s->base) cudaFree(s->base);
  s->base = nullptr;
}

}  // namespace

extern "C" {

int sleek_server_create(void* d_arena, long long arena_bytes, int slots, int max_batch, long long max_batch_chunks,
                        sleek_server* out)
{
  if (!out || arena_bytes < GRANULE || slots < 1 || slots > 64 || max_batch < 1 || max_batch > 1024 ||
      max_batch_chunks < 1)
    return SLEEK_ERR_INVALID_ARG;
  if (d_arena && reinterpret_cast<uintptr_t>(d_arena) % GRANULE) return SLEEK_ERR_ALIGNMENT;
  *out = nullptr;
  auto* s = new sleek_server_s();
  if (cudaGetDevice(&s->dev) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return SLEEK_ERR_NO_DEVICE;
  }
  s->max_batch = max_batch;
  s->max_chunks = max_batch_chunks;
  int rc = SLEEK_OK;
  if (d_arena) {
    s->base = static_cast<unsigned char*>(d_arena);
  } else if (cudaMalloc(&s->base, static_cast<size_t>(arena_bytes)) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return SLEEK_ERR_CUDA;
  } else {
    s->own_arena = true;
  }
  s->arena = Arena(arena_bytes);
  s->free_bytes.store(s->arena.free_bytes());
  // the batched workspace: 32 header words, a flag per chunk, two words per job
  const size_t ws_bytes = 8 * static_cast<size_t>(32 + max_batch_chunks + 2 * max_batch);
  s->slots.resize(static_cast<size_t>(slots));
  for (Slot& sl : s->slots) {
    sl.ws_bytes = ws_bytes;
    if (cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&sl.d_sizes, sizeof(long long) * 2 * max_batch) != cudaSuccess ||
        cudaMallocHost(&sl.h_sizes, sizeof(long long) * 2 * max_batch) != cudaSuccess ||
        cudaMalloc(&sl.ws[0], ws_bytes) != cudaSuccess || cudaMalloc(&sl.ws[1], ws_bytes) != cudaSuccess) {
      cudaGetLastError();
      rc = SLEEK_ERR_CUDA;
      break;
    }
    for (int op = 0; op < 2 && rc == SLEEK_OK; ++op)
      rc = sleek_batch_plan_create_reusable(max_batch, op, &sl.plan[op]);
    if (rc != SLEEK_OK) break;
  }
  if (rc != SLEEK_OK) {
    destroy_resources(s);
    delete s;
    return rc;
  }
  s->t0 = Clock::now();
  s->th = std::thread(loop, s);
  *out = s;
  return SLEEK_OK;
}

int sleek_server_now(sleek_server s, double* seconds)
{
  if (!s || !seconds) return SLEEK_ERR_INVALID_ARG;
  *seconds = s->now();
  return SLEEK_OK;
}

int sleek_server_submit(sleek_server s, const sleek_server_request* reqs, long long n)
{
  if (!s || n < 0 || (n > 0 && !reqs)) return SLEEK_ERR_INVALID_ARG;
  std::vector<Req> add;
  add.reserve(static_cast<size_t>(n));
  for (long long i = 0; i < n; ++i) {
    const sleek_server_request& r = reqs[i];
    if ((r.op != 0 && r.op != 1) || (r.elem_bytes != 4 && r.elem_bytes != 8) || r.num_elements < 0 ||
        (r.num_elements > 0 && !r.input) || (r.op == 1 && r.stream_bytes < 8))
      return SLEEK_ERR_INVALID_ARG;
    Req q;
    q.r = r;
    const long long raw = r.num_elements * r.elem_bytes;
    q.chunks = (raw + CS - 1) / CS;
    q.out_bytes = r.op == 0 ? upper_bound(raw) : raw;
    add.push_back(q);
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return SLEEK_ERR_INVALID_ARG;
    for (Req& q : add) {
      q.seq = s->seq++;
      s->incoming.push_back(q);
    }
    s->submitted += n;
  }
  s->cv_in.notify_one();
  return SLEEK_OK;
}

int sleek_server_poll(sleek_server s, sleek_server_completion* out, long long capacity, long long* n, int wait_ms)
{
  if (!s || !n || capacity < 0 || (capacity > 0 && !out)) return SLEEK_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->done.empty() && wait_ms > 0)
    s->cv_out.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
  long long k = 0;
  while (k < capacity && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.pop_front();
  }
  *n = k;
  return s->error;
}

int sleek_server_outstanding(sleek_server s, long long* n)
{
  if (!s || !n) return SLEEK_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *n = s->submitted - s->finished;
  return SLEEK_OK;
}

int sleek_server_arena_info(sleek_server s, long long* free_bytes, long long* size_bytes)
{
  if (!s || !free_bytes || !size_bytes) return SLEEK_ERR_INVALID_ARG;
  *free_bytes = s->free_bytes.load(std::memory_order_relaxed);
  *size_bytes = s->arena.size();
  return SLEEK_OK;
}

int sleek_server_release(sleek_server s, void* output)
{
  if (!s || !output) return SLEEK_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->releases.push_back(output);
  }
  s->cv_in.notify_one();
  return SLEEK_OK;
}

int sleek_server_destroy(sleek_server s)
{
  if (!s) return SLEEK_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_in.notify_one();
  if (s->th.joinable()) s->th.join();
  destroy_resources(s);
  delete s;
  return SLEEK_OK;
}

int sleek_server_arena_replay(long long arena_bytes, const long long* ops, long long n, long long* offsets)
{
  if (arena_bytes < 0 || n < 0 || (n > 0 && (!ops || !offsets))) return SLEEK_ERR_INVALID_ARG;
  Arena a(arena_bytes);
  std::vector<std::pair<long long, long long>> live;  // per allocation op: offset, bytes
  live.reserve(static_cast<size_t>(n));
  for (long long i = 0; i < n; ++i) {
    const long long v = ops[i];
    if (v > 0) {
      const long long off = a.alloc(v);
      offsets[i] = off;
      live.emplace_back(off, v);
    } else {
      const long long j = -v;  // release of the j-th allocation op (0-based, in order)
      if (j >= static_cast<long long>(live.size()) || live[j].first < 0) return SLEEK_ERR_INVALID_ARG;
      a.release(live[j].first, live[j].second);
      live[j].first = -1;
      offsets[i] = a.free_bytes();
    }
  }
  return SLEEK_OK;
}

}  // extern "C"
