// Host <-> device copies of the host-array entry points.
//
// A caller array in page-locked (pinned) memory is moved by one cudaMemcpyAsync.  A pageable
// array -- a .NET array fixed for P/Invoke is pageable memory -- would otherwise be staged by
// the CUDA driver through its own small pinned buffers, copied on the calling thread alone, and
// its transfer then runs well below the host link's bandwidth.  Instead it is cut into chunks:
// a few host worker threads copy each chunk into a slot of a pinned ring that the context owns,
// and one cudaMemcpyAsync per chunk moves it, so the host copies of later chunks overlap the
// DMA of earlier ones.  Device-to-host runs the same ring backwards.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>
#if defined(__x86_64__)
#include <emmintrin.h>
#endif

#include "sort_host.cuh"

namespace hpcs {

// memcpy with streaming (non-temporal) stores on x86-64: the destination's cache lines are
// written without being read first, so a copy moves two bytes of host memory traffic per byte
// instead of three, and it does not evict the caches.  The stores are fenced before return
// (the DMA engine reads the destination after the copying thread signals completion).
inline void stream_copy(void* dst_v, const void* src_v, size_t bytes) {
#if defined(__x86_64__)
  auto* dst = static_cast<unsigned char*>(dst_v);
  const auto* src = static_cast<const unsigned char*>(src_v);
  size_t head = (16u - (reinterpret_cast<uintptr_t>(dst) & 15u)) & 15u;
  if (head > bytes) head = bytes;
  std::memcpy(dst, src, head);
  dst += head;
  src += head;
  bytes -= head;
  const size_t blocks = bytes / 64;
  for (size_t i = 0; i < blocks; i++, dst += 64, src += 64) {
    const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src));
    const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + 16));
    const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + 32));
    const __m128i d = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + 48));
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst), a);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + 16), b);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + 32), c);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + 48), d);
  }
  std::memcpy(dst, src, bytes - blocks * 64);
  _mm_sfence();
#else
  std::memcpy(dst_v, src_v, bytes);
#endif
}

// A fixed set of worker threads that run one memcpy split into equal pieces; the calling thread
// copies the first piece itself and returns when every piece is done.
class CopyPool {
 public:
  explicit CopyPool(int workers) {
    for (int i = 0; i < workers; i++) threads_.emplace_back([this, i] { loop(i + 1); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  int parts() const { return int(threads_.size()) + 1; }
  void copy(void* dst, const void* src, size_t bytes) {
    if (bytes < (size_t(1) << 20) || threads_.empty()) {
      std::memcpy(dst, src, bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      dst_ = static_cast<unsigned char*>(dst);
      src_ = static_cast<const unsigned char*>(src);
      bytes_ = bytes;
      pending_ = int(threads_.size());
      gen_++;
    }
    cv_.notify_all();
    piece(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return pending_ == 0; });
  }

 private:
  void piece(int idx) {
    const size_t per = ((bytes_ + size_t(parts()) - 1) / size_t(parts()) + 63) & ~size_t(63);  // covers bytes_
    const size_t lo = std::min(bytes_, per * size_t(idx));
    const size_t hi = std::min(bytes_, lo + per);
    if (hi > lo) stream_copy(dst_ + lo, src_ + lo, hi - lo);
  }
  void loop(int idx) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      piece(idx);
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (--pending_ == 0) done_cv_.notify_one();
      }
    }
  }
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  bool stop_ = false;
  uint64_t gen_ = 0;
  int pending_ = 0;
  unsigned char* dst_ = nullptr;
  const unsigned char* src_ = nullptr;
  size_t bytes_ = 0;
};

struct HostStager {
  static constexpr int SLOTS = 4;
  static constexpr size_t CHUNK = size_t(16) << 20;
  unsigned char* ring = nullptr;  // SLOTS x CHUNK bytes of pinned host memory
  cudaEvent_t slot_done[SLOTS] = {};
  CopyPool* pool = nullptr;
  ~HostStager() {
    delete pool;
    for (auto& e : slot_done)
      if (e) cudaEventDestroy(e);
    if (ring) cudaFreeHost(ring);
  }
};

// Copy threads: the host's hardware threads, at most 8.  Measured on a 16-core host of a B200
// node (1 GiB through 16 MiB chunks): pageable -> pinned 10 GB/s on one thread, 46-48 GB/s on
// 8, 44-45 GB/s on 16; pinned -> pageable with streaming stores 61 GB/s on 8 and 51 GB/s on
// 16.  The DMA engine moves about 56 GB/s each way over the host link.
inline int stager_threads() {
  const unsigned hw = std::thread::hardware_concurrency();
  return int(std::max(1u, std::min(8u, hw ? hw : 1u)));
}

inline int get_stager(hpcs_ctx* ctx, HostStager** out) {
  if (!ctx->stager) {
    auto* st = new HostStager();
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&st->ring), HostStager::SLOTS * HostStager::CHUNK,
                                  cudaHostAllocDefault);
    for (int i = 0; e == cudaSuccess && i < HostStager::SLOTS; i++)
      e = cudaEventCreateWithFlags(&st->slot_done[i], cudaEventDisableTiming);
    if (e != cudaSuccess) {
      delete st;
      return cuda_fail(e, "pinned staging ring");
    }
    st->pool = new CopyPool(stager_threads() - 1);
    ctx->stager = st;
  }
  *out = ctx->stager;
  return HPCS_OK;
}

// True when the copy should be staged: a pageable host range of at least a few chunks, and the
// context allows staging.
inline bool stage_copy(hpcs_ctx* ctx, const void* host, size_t bytes) {
  if (!ctx->cfg.staged_host_copies || bytes < 2 * HostStager::CHUNK) return false;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, host) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return attr.type == cudaMemoryTypeUnregistered;
}

// Host -> device on stream s.  Returns when the last chunk is enqueued (the host array may be
// reused once the stream has passed that point: the caller synchronises before returning).
inline int copy_to_device(hpcs_ctx* ctx, void* dev, const void* host, size_t bytes, cudaStream_t s) {
  if (!stage_copy(ctx, host, bytes)) {
    HPCS_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s));
    return HPCS_OK;
  }
  HostStager* st = nullptr;
  int rc = get_stager(ctx, &st);
  if (rc != HPCS_OK) return rc;
  const auto* src = static_cast<const unsigned char*>(host);
  auto* dst = static_cast<unsigned char*>(dev);
  size_t off = 0;
  for (int c = 0; off < bytes; c++) {
    const int slot = c % HostStager::SLOTS;
    const size_t sz = std::min(HostStager::CHUNK, bytes - off);
    unsigned char* buf = st->ring + size_t(slot) * HostStager::CHUNK;
    HPCS_CUDA(cudaEventSynchronize(st->slot_done[slot]));  // the slot's previous DMA is done
    st->pool->copy(buf, src + off, sz);
    HPCS_CUDA(cudaMemcpyAsync(dst + off, buf, sz, cudaMemcpyHostToDevice, s));
    HPCS_CUDA(cudaEventRecord(st->slot_done[slot], s));
    off += sz;
  }
  return HPCS_OK;
}

// Device -> host after the work already on stream s; returns with the data in the host array.
inline int copy_to_host(hpcs_ctx* ctx, void* host, const void* dev, size_t bytes, cudaStream_t s) {
  if (!stage_copy(ctx, host, bytes)) {
    HPCS_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
    HPCS_CUDA(cudaStreamSynchronize(s));
    return HPCS_OK;
  }
  HostStager* st = nullptr;
  int rc = get_stager(ctx, &st);
  if (rc != HPCS_OK) return rc;
  auto* dst = static_cast<unsigned char*>(host);
  const auto* src = static_cast<const unsigned char*>(dev);
  const int64_t chunks = int64_t((bytes + HostStager::CHUNK - 1) / HostStager::CHUNK);
  auto chunk_size = [&](int64_t c) { return std::min(HostStager::CHUNK, bytes - size_t(c) * HostStager::CHUNK); };
  // keep SLOTS chunks in flight: issue chunk c, then drain chunk c - SLOTS + 1 ... in order
  int64_t drained = 0;
  for (int64_t c = 0; c < chunks; c++) {
    const int slot = int(c % HostStager::SLOTS);
    if (c >= HostStager::SLOTS) {  // the slot's previous chunk must be copied out first
      const int64_t d = c - HostStager::SLOTS;
      HPCS_CUDA(cudaEventSynchronize(st->slot_done[slot]));
      st->pool->copy(dst + size_t(d) * HostStager::CHUNK, st->ring + size_t(slot) * HostStager::CHUNK, chunk_size(d));
      drained = d + 1;
    }
    HPCS_CUDA(cudaMemcpyAsync(st->ring + size_t(slot) * HostStager::CHUNK, src + size_t(c) * HostStager::CHUNK,
                              chunk_size(c), cudaMemcpyDeviceToHost, s));
    HPCS_CUDA(cudaEventRecord(st->slot_done[slot], s));
  }
  for (int64_t d = drained; d < chunks; d++) {
    const int slot = int(d % HostStager::SLOTS);
    HPCS_CUDA(cudaEventSynchronize(st->slot_done[slot]));
    st->pool->copy(dst + size_t(d) * HostStager::CHUNK, st->ring + size_t(slot) * HostStager::CHUNK, chunk_size(d));
  }
  return HPCS_OK;
}

}  // namespace hpcs
