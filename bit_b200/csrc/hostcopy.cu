// Host <-> device copies of caller arrays.
//
// A pageable cudaMemcpy goes through the driver's own staging at ~20 GB/s on the B200
// hosts, against ~53 GB/s for DMA from pinned memory.  Large copies of pageable arrays
// therefore go through two pinned chunks per context: the host-side copy of chunk k+1 into
// one chunk (split over a few worker threads) overlaps the DMA of chunk k from the other.
// Arrays the caller has page-locked (cudaHostAlloc, cudaHostRegister, a pinned tensor) are
// copied by DMA directly, with no staging.  Small copies stay plain cudaMemcpyAsync.
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"

namespace bit {
namespace {

constexpr size_t kStageChunk = 8u << 20;   // bytes per pinned chunk
constexpr size_t kDirectBelow = 4u << 20;  // plain copies below this size

// A few threads that copy slices of one buffer in parallel (process-wide).
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool p;
    return p;
  }
  // dst[0, n) = src[0, n), split over the workers and the calling thread.
  void copy(void* dst, const void* src, size_t n) {
    const int parts = (int)workers_.size() + 1;
    if (n < (1u << 20) || parts == 1) {
      std::memcpy(dst, src, n);
      return;
    }
    std::unique_lock<std::mutex> call(call_mu_);  // one parallel copy at a time
    const size_t per = (n / parts + 4095) / 4096 * 4096;
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_dst_ = static_cast<char*>(dst);
      job_src_ = static_cast<const char*>(src);
      job_n_ = n;
      job_per_ = per;
      pending_ = parts - 1;
      gen_++;
    }
    cv_.notify_all();
    copy_part(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return pending_ == 0; });
  }

 private:
  CopyPool() {
    unsigned hw = std::thread::hardware_concurrency();
    const int nw = hw >= 8 ? 3 : (hw >= 4 ? 1 : 0);
    for (int i = 0; i < nw; i++) workers_.emplace_back([this, i] { run(i + 1); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      gen_++;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  void copy_part(int k) {
    const size_t b = std::min(job_n_, job_per_ * k), e = std::min(job_n_, b + job_per_);
    if (e > b) std::memcpy(job_dst_ + b, job_src_ + b, e - b);
  }
  void run(int k) {
    long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
      }
      copy_part(k);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) done_cv_.notify_all();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_, call_mu_;
  std::condition_variable cv_, done_cv_;
  char* job_dst_ = nullptr;
  const char* job_src_ = nullptr;
  size_t job_n_ = 0, job_per_ = 0;
  int pending_ = 0;
  long long gen_ = 0;
  bool stop_ = false;
};

void ensure_stage(Ctx* c) {
  if (c->stage[0]) return;
  for (int i = 0; i < 2; i++) {
    BIT_CUDA(cudaMallocHost(&c->stage[i], kStageChunk));
    BIT_CUDA(cudaEventCreateWithFlags(&c->stage_ev[i], cudaEventDisableTiming));
  }
}

// The host array is page-locked memory the device can DMA from or to.
bool host_pinned(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

}  // namespace

void copy_h2d(Ctx* c, void* dst, const void* src, size_t bytes) {
  cudaStream_t s = c->stream;
  if (bytes < kDirectBelow) {
    BIT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return;
  }
  if (host_pinned(src)) {
    // DMA straight from the caller's array; it may be reused once the copy is done
    BIT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    return;
  }
  ensure_stage(c);
  const char* p = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
  int k = 0;
  for (size_t off = 0; off < bytes; off += kStageChunk, k++) {
    const size_t n = std::min(kStageChunk, bytes - off);
    const int b = k & 1;
    BIT_CUDA(cudaEventSynchronize(c->stage_ev[b]));  // the chunk's last DMA is done
    CopyPool::get().copy(c->stage[b], p + off, n);
    BIT_CUDA(cudaMemcpyAsync(d + off, c->stage[b], n, cudaMemcpyHostToDevice, s));
    BIT_CUDA(cudaEventRecord(c->stage_ev[b], s));
  }
}

void copy_d2h(Ctx* c, void* dst, const void* src, size_t bytes) {
  cudaStream_t s = c->stream;
  if (bytes < kDirectBelow || host_pinned(dst)) {
    BIT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaStreamSynchronize(s));
    return;
  }
  ensure_stage(c);
  const char* p = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
  const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
  auto issue = [&](size_t k) {
    const size_t off = k * kStageChunk, n = std::min(kStageChunk, bytes - off);
    BIT_CUDA(cudaMemcpyAsync(c->stage[k & 1], p + off, n, cudaMemcpyDeviceToHost, s));
    BIT_CUDA(cudaEventRecord(c->stage_ev[k & 1], s));
  };
  // a staging chunk may still feed an earlier host-to-device copy: wait for it first
  for (int b = 0; b < 2; b++) BIT_CUDA(cudaEventSynchronize(c->stage_ev[b]));
  issue(0);
  for (size_t k = 0; k < nch; k++) {
    BIT_CUDA(cudaEventSynchronize(c->stage_ev[k & 1]));
    if (k + 1 < nch) issue(k + 1);  // the other chunk was copied out last round
    const size_t off = k * kStageChunk, n = std::min(kStageChunk, bytes - off);
    CopyPool::get().copy(d + off, c->stage[k & 1], n);
  }
}

}  // namespace bit
