// Copies between large host buffers and the device for the host-buffer entry points
// (fx_run_host, fx_walk_host, fx_fetch_u, fx_batch_walk_host).
//
// The drop-in contract hands over numpy arrays: the input is whatever the caller has (usually
// pageable memory) and `run` returns a new array (MatrixExpCalculator<T>::run,
// src/main.cu:17-19), which numpy allocates without touching its pages.  A plain cudaMemcpy
// from or to such memory goes through the driver's own small bounce buffer on one thread and,
// for a fresh output array, takes every first-touch page fault on that thread: at N = 10000
// (800 MB each way for complex64) that is about ten times slower than the link.
//
// Here a buffer that the CUDA driver already knows as page-locked is copied directly by DMA.
// Anything else goes through two page-locked chunk buffers owned by the handle: the host
// side of chunk c (a copy split over several threads, which also spreads the page faults)
// overlaps the DMA of chunk c - 1.
#include <sched.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "fx_kernels.cuh"

namespace fx {

namespace {

constexpr size_t kStageChunk = (size_t)32 << 20;   // bytes per page-locked chunk buffer
constexpr size_t kParallelMin = (size_t)1 << 20;   // below this a host copy stays on one thread

int host_threads() {
  cpu_set_t set;
  CPU_ZERO(&set);
  int n = 0;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) n = CPU_COUNT(&set);
  if (n <= 0) n = (int)std::thread::hardware_concurrency();
  return std::max(1, std::min(n, 16));
}

// Process-wide workers for the host side of the chunked copies: started once, so that a
// copy of N = 10000 (25 chunks of 32 MiB) does not start and join hundreds of threads.
// run(n, f) calls f(0) .. f(n - 1), piece 0 on the caller's thread and the others on the
// workers, and returns when all are done; one run at a time.
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool pool(host_threads() - 1);
    return pool;
  }
  int size() const { return (int)workers_.size() + 1; }
  void run(int n, const std::function<void(int)>& f) {
    std::lock_guard<std::mutex> one(run_mu_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &f;
      pieces_ = n;
      next_ = 1;
      left_ = n - 1;
      ++gen_;
    }
    cv_.notify_all();
    if (n > 0) f(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return left_ <= 0; });
    job_ = nullptr;
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }

 private:
  explicit CopyPool(int nworkers) {
    for (int i = 0; i < nworkers; ++i) workers_.emplace_back([this] { loop(); });
  }
  void loop() {
    unsigned long seen = 0;
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return stop_ || (gen_ != seen && next_ < pieces_); });
      if (stop_) return;
      seen = gen_;
      while (job_ && next_ < pieces_) {
        const int i = next_++;
        const std::function<void(int)>* f = job_;
        lk.unlock();
        (*f)(i);
        lk.lock();
        if (--left_ <= 0) done_cv_.notify_all();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::mutex run_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int pieces_ = 0, next_ = 0, left_ = 0;
  unsigned long gen_ = 0;
  bool stop_ = false;
};

// memcpy split over up to host_threads() threads (page-aligned pieces).
void parallel_memcpy(void* dst, const void* src, size_t bytes) {
  CopyPool& pool = CopyPool::get();
  const int nt = bytes < kParallelMin ? 1 : pool.size();
  if (nt == 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t per = ((bytes + nt - 1) / nt + 4095) & ~(size_t)4095;
  const int pieces = (int)((bytes + per - 1) / per);
  pool.run(pieces, [&](int i) {
    const size_t o = (size_t)i * per;
    std::memcpy((char*)dst + o, (const char*)src + o, std::min(per, bytes - o));
  });
}

}  // namespace

bool host_is_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Touches every page of a host buffer (one write per 4 KiB, split over the copy workers), so
// that a fresh allocation takes its first-touch page faults at this point -- while the device
// computes, when called from a thread of its own -- instead of inside the copy that fills it.
// Page-locked and small buffers are left alone.  The bytes written are overwritten by that copy.
void prefault_host(void* p, size_t bytes) {
  if (bytes < kParallelMin || host_is_pinned(p)) return;
  CopyPool& pool = CopyPool::get();
  const int nt = pool.size();
  const size_t per = ((bytes + nt - 1) / nt + 4095) & ~(size_t)4095;
  const int pieces = (int)((bytes + per - 1) / per);
  pool.run(pieces, [&](int i) {
    volatile char* b = (volatile char*)p + (size_t)i * per;
    const size_t len = std::min(per, bytes - (size_t)i * per);
    for (size_t o = 0; o < len; o += 4096) b[o] = 0;
    b[len - 1] = 0;
  });
}

HostStage::~HostStage() { release(); }

void HostStage::release() {
  for (int i = 0; i < 2; ++i) {
    if (ev[i]) {
      cudaEventSynchronize(ev[i]);
      cudaEventDestroy(ev[i]);
    }
    if (buf[i]) cudaFreeHost(buf[i]);
    ev[i] = nullptr;
    buf[i] = nullptr;
  }
}

void HostStage::ensure() {
  for (int i = 0; i < 2; ++i) {
    if (!buf[i] && cudaHostAlloc(&buf[i], kStageChunk, cudaHostAllocDefault) != cudaSuccess) {
      buf[i] = nullptr;
      cudaGetLastError();
      throw Error{FX_ERR_NOMEM, "page-locked staging allocation failed"};
    }
    if (!ev[i]) FX_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
  }
}

void HostStage::h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (bytes < kParallelMin || host_is_pinned(src)) {
    FX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return;
  }
  ensure();
  for (size_t o = 0, c = 0; o < bytes; o += kStageChunk, ++c) {
    const int b = (int)(c & 1);
    const size_t len = std::min(kStageChunk, bytes - o);
    FX_CUDA(cudaEventSynchronize(ev[b]));   // the DMA that last read this buffer is done
    parallel_memcpy(buf[b], (const char*)src + o, len);
    FX_CUDA(cudaMemcpyAsync((char*)dst + o, buf[b], len, cudaMemcpyHostToDevice, s));
    FX_CUDA(cudaEventRecord(ev[b], s));
  }
}

void HostStage::d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (bytes < kParallelMin || host_is_pinned(dst)) {
    FX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaStreamSynchronize(s));
    return;
  }
  ensure();
  const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
  auto piece = [&](size_t c) { return std::min(kStageChunk, bytes - c * kStageChunk); };
  for (size_t c = 0; c <= nch; ++c) {
    if (c < nch) {   // DMA of chunk c into buffer c % 2 (its previous chunk was copied out below)
      const int b = (int)(c & 1);
      FX_CUDA(cudaMemcpyAsync(buf[b], (const char*)src + c * kStageChunk, piece(c), cudaMemcpyDeviceToHost, s));
      FX_CUDA(cudaEventRecord(ev[b], s));
    }
    if (c >= 1) {    // meanwhile the host copies chunk c - 1 out of the other buffer
      const int b = (int)((c - 1) & 1);
      FX_CUDA(cudaEventSynchronize(ev[b]));
      parallel_memcpy((char*)dst + (c - 1) * kStageChunk, buf[b], piece(c - 1));
    }
  }
}

}  // namespace fx
