// staging.cu — host <-> device copies of the host-buffer entry points (see
// runtime.cuh: h2d_copy / d2h_copy).
//
// The reference's callers hand over pageable memory (Rust Vec<Fr>).  A copy
// from or to pageable memory cannot be DMA'd directly; the driver stages it
// through its own bounce buffer with one host thread, which ran at about a
// third of the pinned rate on B200 hosts.  Here pageable buffers go through
// a per-thread ring of pinned chunks instead: the host side of each chunk is
// a memcpy split over a small pool of helper threads, and chunk i's DMA
// overlaps chunk i+1's memcpy.  Pinned (page-locked or registered) buffers
// are copied directly.
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "runtime.cuh"

namespace zk {
namespace {

constexpr size_t kChunk = 16u << 20;  // bytes per pinned chunk
constexpr int kSlots = 4;             // chunks in flight per thread

// Fork-join pool for the host memcpys: run(f, parts) calls f(i) for
// i < parts on the helper threads and the caller, and returns when all ran.
class CopyPool {
 public:
  CopyPool() {
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    const unsigned helpers = std::min(7u, hw / 2);
    for (unsigned i = 0; i < helpers; i++) workers_.emplace_back([this] { loop(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  int width() const { return (int)workers_.size() + 1; }
  void run(const std::function<void(int)>& f, int parts) {
    std::unique_lock<std::mutex> serial(run_mu_);  // one parallel copy at a time
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &f;
      parts_ = parts;
      next_ = 0;
      done_ = 0;
      gen_++;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return done_ == parts_; });
    job_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      int i;
      const std::function<void(int)>* f;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (!job_ || next_ >= parts_) return;
        i = next_++;
        f = job_;
      }
      (*f)(i);
      std::lock_guard<std::mutex> lk(mu_);
      if (++done_ == parts_) done_cv_.notify_all();
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || (gen_ != seen && job_ && next_ < parts_); });
        if (stop_) return;
        seen = gen_;
      }
      work();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_, run_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int parts_ = 0, next_ = 0, done_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

CopyPool& pool() {
  static CopyPool* p = new CopyPool();  // lives until exit; its threads are never joined at teardown
  return *p;
}

void par_memcpy(void* dst, const void* src, size_t n) {
  CopyPool& cp = pool();
  const int parts = (int)std::min<size_t>((size_t)cp.width(), std::max<size_t>(1, n >> 20));
  if (parts <= 1) {
    std::memcpy(dst, src, n);
    return;
  }
  const size_t per = (n + parts - 1) / parts;
  cp.run([&](int i) {
    const size_t o = per * i;
    if (o < n) std::memcpy((char*)dst + o, (const char*)src + o, std::min(per, n - o));
  }, parts);
}

struct Ring {
  char* buf[kSlots] = {nullptr};
  cudaEvent_t ev[kSlots] = {nullptr};
  int dev = -1;
  bool ok = false;
};
thread_local Ring t_ring;

cudaError_t ring_get(Ring** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  Ring& r = t_ring;
  if (!r.ok || r.dev != dev) {
    // pinned host memory is usable from every device; events belong to one
    for (int i = 0; i < kSlots; i++) {
      if (!r.buf[i]) {
        e = cudaMallocHost((void**)&r.buf[i], kChunk);
        if (e != cudaSuccess) return e;
      }
      if (r.ev[i]) cudaEventDestroy(r.ev[i]);
      e = cudaEventCreateWithFlags(&r.ev[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    r.dev = dev;
    r.ok = true;
  }
  *out = &r;
  return cudaSuccess;
}

}  // namespace

bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

cudaError_t h2d_copy(void* dst, const void* src, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (host_pinned(src) || n < kChunk / 4) return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s);
  Ring* r;
  cudaError_t e = ring_get(&r);
  if (e != cudaSuccess) return e;
  int k = 0;
  for (size_t off = 0; off < n; off += kChunk, k = (k + 1) % kSlots) {
    const size_t len = std::min(kChunk, n - off);
    e = cudaEventSynchronize(r->ev[k]);  // the slot's previous DMA has finished
    if (e != cudaSuccess) return e;
    par_memcpy(r->buf[k], (const char*)src + off, len);
    e = cudaMemcpyAsync((char*)dst + off, r->buf[k], len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(r->ev[k], s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;  // the source is fully staged: the caller may reuse it
}

cudaError_t d2h_copy(void* dst, const void* src, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (host_pinned(dst) || n < kChunk / 4) return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s);
  Ring* r;
  cudaError_t e = ring_get(&r);
  if (e != cudaSuccess) return e;
  const size_t chunks = (n + kChunk - 1) / kChunk;
  auto issue = [&](size_t c) {
    const size_t off = c * kChunk, len = std::min(kChunk, n - off);
    const int k = (int)(c % kSlots);
    cudaError_t x = cudaMemcpyAsync(r->buf[k], (const char*)src + off, len, cudaMemcpyDeviceToHost, s);
    if (x == cudaSuccess) x = cudaEventRecord(r->ev[k], s);
    return x;
  };
  for (size_t c = 0; c < chunks && c < (size_t)kSlots; c++)
    if ((e = issue(c)) != cudaSuccess) return e;
  for (size_t c = 0; c < chunks; c++) {
    const int k = (int)(c % kSlots);
    const size_t off = c * kChunk, len = std::min(kChunk, n - off);
    e = cudaEventSynchronize(r->ev[k]);
    if (e != cudaSuccess) return e;
    par_memcpy((char*)dst + off, r->buf[k], len);
    if (c + kSlots < chunks && (e = issue(c + kSlots)) != cudaSuccess) return e;
  }
  return cudaSuccess;  // dst holds the data
}

}  // namespace zk
