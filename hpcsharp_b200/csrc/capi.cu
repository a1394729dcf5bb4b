// C ABI of libhpcs_gpu.so (declared in include/hpcs_gpu.h): contexts, argument checks that
// mirror the reference's exceptions, host-array and device-pointer entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/hpcs_gpu.h"
#include "sort_host.cuh"
#include "counting.cuh"
#include "segmented_host.cuh"
#include "topk_host.cuh"
#include "shard.cuh"
#include "host_copy.cuh"

namespace hpcs {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int status, const std::string& msg) {
  set_error(msg);
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return fail(HPCS_ERR_OOM, m);
  return fail(HPCS_ERR_CUDA, m);
}

int ensure(hpcs_ctx* ctx, DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return HPCS_OK;
  if (b.borrowed) return fail(HPCS_ERR_OOM, "borrowed scratch is smaller than the request needs");
  size_t want = bytes < 256 ? 256 : bytes;
  if (ctx->cfg.pool_bytes > 0 && ctx->held_bytes - b.bytes + want > size_t(ctx->cfg.pool_bytes))
    return fail(HPCS_ERR_OOM, "request exceeds the context's pool_bytes budget");
  if (b.ptr) {
    // earlier work on the context's streams may still read the old buffer
    cudaError_t e = cudaStreamSynchronize(ctx->last_stream ? ctx->last_stream : ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    cudaFree(b.ptr);
    ctx->held_bytes -= b.bytes;
    b.ptr = nullptr;
    b.bytes = 0;
  }
  cudaError_t e = cudaMalloc(&b.ptr, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.ptr = nullptr;
    return cuda_fail(e, "cudaMalloc");
  }
  b.bytes = want;
  ctx->held_bytes += want;
  return HPCS_OK;
}

int enter_stream(hpcs_ctx* ctx, cudaStream_t s) {
  if (ctx->last_stream != nullptr && ctx->last_stream != s) {
    HPCS_CUDA(cudaEventRecord(ctx->order_event, ctx->last_stream));
    HPCS_CUDA(cudaStreamWaitEvent(s, ctx->order_event, 0));
  }
  ctx->last_stream = s;
  return HPCS_OK;
}

static cudaEvent_t take_event(hpcs_ctx* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

KernelTimer::KernelTimer(hpcs_ctx* c, cudaStream_t st, int k) : ctx(c), s(st), cls(k) {
  if (!ctx->profile) return;
  a = take_event(ctx);
  b = take_event(ctx);
  if (a) cudaEventRecord(a, s);
}

KernelTimer::~KernelTimer() {
  if (!ctx->profile || !a || !b) return;
  cudaEventRecord(b, s);
  ctx->timed.push_back({cls, a, b});
}

uint32_t* device_error_word(hpcs_ctx* ctx) { return static_cast<uint32_t*>(ctx->err_accum.ptr); }

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

cudaStream_t pick_stream(hpcs_ctx* ctx, void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
}

// Runs the lane-order probe once per device (result cached per device).
int probe_rank_order(hpcs_ctx* ctx, int* ordered) {
  static std::mutex mu;
  static int cache[64];  // 0 unknown, 1 ordered, 2 not ordered
  std::lock_guard<std::mutex> lock(mu);
  int& c = cache[ctx->device & 63];
  if (c == 0) {
    uint32_t* bad = nullptr;
    HPCS_CUDA(cudaMalloc(&bad, 4));
    cudaError_t e = cudaMemset(bad, 0, 4);
    if (e == cudaSuccess) {
      rank_probe_kernel<512, 16><<<ctx->sms * 2, 512>>>(bad, 0x2545F491u);
      e = cudaGetLastError();
    }
    uint32_t h = 1;
    if (e == cudaSuccess) e = cudaMemcpy(&h, bad, 4, cudaMemcpyDeviceToHost);
    cudaFree(bad);
    if (e != cudaSuccess) return cuda_fail(e, "rank order probe");
    c = h == 0 ? 1 : 2;
  }
  *ordered = c == 1;
  return HPCS_OK;
}

int check_device_errors(hpcs_ctx* ctx);

// ---- probe of the shipping pass kernels ---------------------------------------------------
// Keys whose digits take few values, so many lanes of a warp instruction share a counter: with
// `values` = 20 every byte digit has at most 20 values, with 3 at most 3; items are the input
// positions.
__global__ void probe_fill_kernel(uint32_t* keys, uint32_t* items, int64_t n, uint32_t values) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t x = uint32_t(i) * 0x9E3779B1u ^ 0x85EBCA6Bu;
    x ^= x >> 15;
    x *= 0x2C1B3C6Du;
    x ^= x >> 12;
    const uint32_t y = x * 0x27D4EB2Fu;
    keys[i] = ((x & 0xFFFFu) % values) | (((x >> 16) % values) << 8) | (((y >> 8) % values) << 16) |
              (((y >> 20) % values) << 24);
    if (items) items[i] = uint32_t(i);
  }
}

// Counts positions where the keys descend or, with items, equal keys' items do not ascend.
__global__ void probe_check_kernel(const uint32_t* keys, const uint32_t* items, int64_t n, uint32_t* bad) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  uint32_t v = 0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x + 1; i < n; i += stride) {
    if (keys[i] < keys[i - 1]) v++;
    else if (items && keys[i] == keys[i - 1] && items[i] <= items[i - 1]) v++;
  }
  if (v) atomicAdd(bad, v);
}

// Runs the shipping ordered-atomic pass kernels -- the chunked passes and the look-back passes,
// keys only and with items -- on inputs with many equal digits per warp instruction and checks
// the results for order and stability.  Any violation sends the context to the peer-mask
// ranking, which is defined by PTX.  The same code generation and occupancy as a real sort: the
// probe calls the sort's own enqueue functions.
int probe_shipping_kernels(hpcs_ctx* ctx, int* ok) {
  constexpr int64_t n = (int64_t(1) << 20) + 12345;
  uint32_t *keys = nullptr, *items = nullptr, *bad = nullptr;
  cudaError_t e = cudaMalloc(&keys, size_t(n) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&items, size_t(n) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&bad, 4);
  if (e == cudaSuccess) e = cudaMemset(bad, 0, 4);
  int rc = e == cudaSuccess ? HPCS_OK : cuda_fail(e, "probe buffers");
  const int saved_mode = ctx->rank_mode;
  const int saved_scheme = ctx->cfg.pass_scheme;
  ctx->rank_mode = RANK_ORDERED_ATOMIC;
  cudaStream_t s = ctx->stream;
  for (int scheme : {int(HPCS_PASSES_CHUNKED), int(HPCS_PASSES_LOOKBACK)}) {
    ctx->cfg.pass_scheme = scheme;
    for (uint32_t values : {20u, 3u}) {
      for (int with_items = 0; with_items < 2 && rc == HPCS_OK; with_items++) {
        uint32_t* it = with_items ? items : nullptr;
        probe_fill_kernel<<<ctx->sms * 4, 256, 0, s>>>(keys, it, n, values);
        if ((e = cudaGetLastError()) != cudaSuccess) rc = cuda_fail(e, "probe fill");
        if (rc == HPCS_OK)
          rc = with_items ? enqueue_sort<uint32_t, KIND_UNSIGNED, uint32_t>(ctx, keys, items, n, s)
                          : enqueue_sort<uint32_t, KIND_UNSIGNED, NoValue>(ctx, keys, nullptr, n, s);
        if (rc == HPCS_OK) {
          probe_check_kernel<<<ctx->sms * 4, 256, 0, s>>>(keys, it, n, bad);
          if ((e = cudaGetLastError()) != cudaSuccess) rc = cuda_fail(e, "probe check");
        }
      }
    }
  }
  // the one-launch sort of small arrays (small_sort.cuh), taken by the default scheme
  ctx->cfg.pass_scheme = HPCS_PASSES_AUTO;
  constexpr int64_t n_small = 100003;
  for (uint32_t values : {20u, 3u}) {
    for (int with_items = 0; with_items < 2 && rc == HPCS_OK; with_items++) {
      uint32_t* it = with_items ? items : nullptr;
      probe_fill_kernel<<<ctx->sms * 4, 256, 0, s>>>(keys, it, n_small, values);
      if ((e = cudaGetLastError()) != cudaSuccess) rc = cuda_fail(e, "probe fill");
      if (rc == HPCS_OK)
        rc = with_items ? enqueue_sort<uint32_t, KIND_UNSIGNED, uint32_t>(ctx, keys, items, n_small, s)
                        : enqueue_sort<uint32_t, KIND_UNSIGNED, NoValue>(ctx, keys, nullptr, n_small, s);
      if (rc == HPCS_OK) {
        probe_check_kernel<<<ctx->sms * 4, 256, 0, s>>>(keys, it, n_small, bad);
        if ((e = cudaGetLastError()) != cudaSuccess) rc = cuda_fail(e, "probe check");
      }
    }
  }
  ctx->rank_mode = saved_mode;
  ctx->cfg.pass_scheme = saved_scheme;
  uint32_t h = 1;
  if (rc == HPCS_OK && (e = cudaStreamSynchronize(s)) != cudaSuccess) rc = cuda_fail(e, "probe");
  if (rc == HPCS_OK && (e = cudaMemcpy(&h, bad, 4, cudaMemcpyDeviceToHost)) != cudaSuccess) rc = cuda_fail(e, "probe");
  if (rc == HPCS_OK) rc = check_device_errors(ctx);
  cudaFree(keys);
  cudaFree(items);
  cudaFree(bad);
  *ok = rc == HPCS_OK && h == 0;
  return rc;
}

// Reads and clears the accumulated device error bits (synchronous).
int check_device_errors(hpcs_ctx* ctx) {
  uint32_t bits = 0;
  HPCS_CUDA(cudaMemcpy(&bits, ctx->err_accum.ptr, 4, cudaMemcpyDeviceToHost));
  if (bits) {
    HPCS_CUDA(cudaMemset(ctx->err_accum.ptr, 0, 4));
    char buf[160];
    std::snprintf(buf, sizeof buf,
                  "device-side wait ran out (error bits 0x%x: 1=look-back, 2=bulk copy, 4=bounds, 8=queue)",
                  bits);
    return fail(HPCS_ERR_DEVICE_TIMEOUT, buf);
  }
  return HPCS_OK;
}

int check_common(hpcs_ctx* ctx, const void* p, int64_t n) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  if (!p) return fail(HPCS_ERR_NULL, "array is NULL");
  if (n < 0) return fail(HPCS_ERR_RANGE, "length is negative");
  if (n > HPCS_MAX_KEYS) return fail(HPCS_ERR_RANGE, "length exceeds HPCS_MAX_KEYS");
  return HPCS_OK;
}

template <class T, class U, int KIND>
int sort_host(hpcs_ctx* ctx, T* keys, int64_t n) {
  int rc = check_common(ctx, keys, n);
  if (rc != HPCS_OK || n == 0) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t s = ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_a, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  U* d = static_cast<U*>(ctx->keys_a.ptr);
  if ((rc = copy_to_device(ctx, d, keys, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  if ((rc = enqueue_sort<U, KIND, NoValue>(ctx, d, nullptr, n, s)) != HPCS_OK) return rc;
  if ((rc = copy_to_host(ctx, keys, d, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  return check_device_errors(ctx);
}

template <class T, class U, int KIND>
int sort_dev(hpcs_ctx* ctx, T* keys, int64_t n, void* stream) {
  int rc = check_common(ctx, keys, n);
  if (rc != HPCS_OK || n == 0) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  return enqueue_sort<U, KIND, NoValue>(ctx, reinterpret_cast<U*>(keys), nullptr, n, s);
}

// Counting sort of 8/16-bit keys in device memory (histogram, scan, fill), in place.
template <class U>
int enqueue_count_sort(hpcs_ctx* ctx, U* d, int64_t n, uint32_t flip, cudaStream_t s) {
  constexpr int BINS = CountTraits<U>::BINS;
  int rc;
  if ((rc = ensure(ctx, ctx->counts, size_t(BINS) * 4)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->aux2, size_t(BINS + 1) * 8)) != HPCS_OK) return rc;
  uint32_t* counts = static_cast<uint32_t*>(ctx->counts.ptr);
  int64_t* starts = static_cast<int64_t*>(ctx->aux2.ptr);
  const size_t smem = BINS == 256 ? size_t(256) * 32 * 4 : size_t(BINS / 2) * 4;
  auto kh = count_hist_kernel<U>;
  static int attr_set[64] = {0};
  if (!attr_set[ctx->device & 63]) {
    HPCS_CUDA(cudaFuncSetAttribute(kh, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    attr_set[ctx->device & 63] = 1;
  }
  HPCS_CUDA(cudaMemsetAsync(counts, 0, size_t(BINS) * 4, s));
  const int64_t want = (n + int64_t(COUNT_NT) * 16 - 1) / (int64_t(COUNT_NT) * 16);
  const int64_t hcap = int64_t(ctx->sms) * (BINS == 256 ? 2 : 1);  // CTAs per SM that fit the counters
  const int hgrid = int(want < 1 ? 1 : (want > hcap ? hcap : want));
  {
    KernelTimer kt(ctx, s, HPCS_K_HISTOGRAM);
    kh<<<hgrid, COUNT_NT, smem, s>>>(d, n, flip, counts);
    HPCS_CUDA(cudaGetLastError());
  }
  const int64_t range = count_fill_range<U>();
  const int64_t ranges = (n + range - 1) / range;
  if ((rc = ensure(ctx, ctx->aux1, size_t(ranges) * 2 * 4)) != HPCS_OK) return rc;
  int32_t* range_lo = static_cast<int32_t*>(ctx->aux1.ptr);
  int32_t* range_hi = range_lo + ranges;
  count_scan_kernel<BINS><<<BINS / count_scan_nt<BINS>(), count_scan_nt<BINS>(), 0, s>>>(counts, n, range, starts,
                                                                                          range_lo, range_hi);
  HPCS_CUDA(cudaGetLastError());
  const int fgrid = int(ranges > int64_t(ctx->sms) * 8 ? int64_t(ctx->sms) * 8 : ranges);
  {
    KernelTimer kt(ctx, s, HPCS_K_FINALIZE);
    count_fill_kernel<U><<<fgrid, COUNT_FILL_NT, 0, s>>>(d, n, starts, range_lo, range_hi, flip);
    HPCS_CUDA(cudaGetLastError());
  }
  return HPCS_OK;
}

template <class T, class U>
int count_sort_host(hpcs_ctx* ctx, T* keys, int64_t n, uint32_t flip) {
  int rc = check_common(ctx, keys, n);
  if (rc != HPCS_OK || n == 0) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t s = ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_a, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  U* d = static_cast<U*>(ctx->keys_a.ptr);
  if ((rc = copy_to_device(ctx, d, keys, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  if ((rc = enqueue_count_sort<U>(ctx, d, n, flip, s)) != HPCS_OK) return rc;
  if ((rc = copy_to_host(ctx, keys, d, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  return check_device_errors(ctx);
}

template <class T, class U>
int count_sort_dev(hpcs_ctx* ctx, T* keys, int64_t n, uint32_t flip, void* stream) {
  int rc = check_common(ctx, keys, n);
  if (rc != HPCS_OK || n == 0) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  return enqueue_count_sort<U>(ctx, reinterpret_cast<U*>(keys), n, flip, s);
}

template <class T, class U, int KIND>
int pairs_host(hpcs_ctx* ctx, T* keys, uint32_t* items, int64_t n) {
  int rc = check_common(ctx, keys, n);
  if (rc != HPCS_OK) return rc;
  if (!items) return fail(HPCS_ERR_NULL, "items is NULL");
  if (n == 0) return HPCS_OK;
  DeviceGuard g(ctx->device);
  cudaStream_t s = ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_a, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->vals_a, size_t(n) * 4)) != HPCS_OK) return rc;
  U* dk = static_cast<U*>(ctx->keys_a.ptr);
  uint32_t* dv = static_cast<uint32_t*>(ctx->vals_a.ptr);
  if ((rc = copy_to_device(ctx, dk, keys, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  if ((rc = copy_to_device(ctx, dv, items, size_t(n) * 4, s)) != HPCS_OK) return rc;
  if ((rc = enqueue_sort<U, KIND, uint32_t>(ctx, dk, dv, n, s)) != HPCS_OK) return rc;
  if ((rc = copy_to_host(ctx, keys, dk, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  if ((rc = copy_to_host(ctx, items, dv, size_t(n) * 4, s)) != HPCS_OK) return rc;
  return check_device_errors(ctx);
}

template <class T, class U, int KIND>
int pairs_dev(hpcs_ctx* ctx, T* keys, uint32_t* items, int64_t n, void* stream) {
  int rc = check_common(ctx, keys, n);
  if (rc != HPCS_OK) return rc;
  if (!items) return fail(HPCS_ERR_NULL, "items is NULL");
  if (n == 0) return HPCS_OK;
  DeviceGuard g(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  return enqueue_sort<U, KIND, uint32_t>(ctx, reinterpret_cast<U*>(keys), items, n, s);
}

// Histogram of n keys at device pointer d into device counts[P][256] (zeroed here).
template <class U, int KIND>
int enqueue_histogram(hpcs_ctx* ctx, const U* d, int64_t n, uint32_t* counts, cudaStream_t s) {
  constexpr int P = int(sizeof(U));
  HPCS_CUDA(cudaMemsetAsync(counts, 0, size_t(P) * RADIX * 4, s));
  if (n <= 0) return HPCS_OK;
  const U* src = d;
  int rc;
  if ((reinterpret_cast<uintptr_t>(d) & 15) != 0) {  // the vector loads need 16-byte alignment
    if ((rc = ensure(ctx, ctx->keys_b, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
    HPCS_CUDA(cudaMemcpyAsync(ctx->keys_b.ptr, d, size_t(n) * sizeof(U), cudaMemcpyDeviceToDevice, s));
    src = static_cast<const U*>(ctx->keys_b.ptr);
  }
  SortArgs none{};
  KernelTimer kt(ctx, s, HPCS_K_HISTOGRAM);
  return launch_histogram<U, KIND>(ctx, src, n, counts, none, 0, s);
}

template <class T, class U, int KIND>
int histogram_host(hpcs_ctx* ctx, const T* a, int64_t l, int64_t r, uint32_t* counts) {
  constexpr int P = int(sizeof(U));
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  if (!a) return fail(HPCS_ERR_NULL, "array is NULL");
  if (!counts) return fail(HPCS_ERR_NULL, "counts is NULL");
  if (l < 0) return fail(HPCS_ERR_RANGE, "l is negative");
  const int64_t n = r - l + 1;
  if (n > HPCS_MAX_KEYS) return fail(HPCS_ERR_RANGE, "range exceeds HPCS_MAX_KEYS");
  if (n <= 0) {
    std::memset(counts, 0, size_t(P) * RADIX * 4);
    return HPCS_OK;
  }
  DeviceGuard g(ctx->device);
  cudaStream_t s = ctx->stream;
  int rc;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_a, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->counts, size_t(MAX_PASSES) * RADIX * 4)) != HPCS_OK) return rc;
  U* d = static_cast<U*>(ctx->keys_a.ptr);
  uint32_t* dc = static_cast<uint32_t*>(ctx->counts.ptr);
  if ((rc = copy_to_device(ctx, d, a + l, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  if ((rc = enqueue_histogram<U, KIND>(ctx, d, n, dc, s)) != HPCS_OK) return rc;
  HPCS_CUDA(cudaMemcpyAsync(counts, dc, size_t(P) * RADIX * 4, cudaMemcpyDeviceToHost, s));
  HPCS_CUDA(cudaStreamSynchronize(s));
  return HPCS_OK;
}

int check_select_args(hpcs_ctx* ctx, const void* a, int64_t n, int64_t k) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  if (!a) return fail(HPCS_ERR_NULL, "array is NULL");
  // SelectTopK(a, k): length must be positive and k a valid index (SelectionTopKRadix.cs:164-167;
  // k == Length passes the reference's check but then indexes past its bins).
  if (n <= 0) return fail(HPCS_ERR_RANGE, "array length is invalid");
  if (n > HPCS_MAX_SEGMENT_KEYS) return fail(HPCS_ERR_RANGE, "length exceeds HPCS_MAX_SEGMENT_KEYS");
  if (k < 0 || k >= n) return fail(HPCS_ERR_RANGE, "k must be in [0, length)");
  return HPCS_OK;
}

template <class T, class U, int KIND>
int select_topk_host(hpcs_ctx* ctx, T* a, int64_t n, int64_t k) {
  int rc = check_select_args(ctx, a, n, k);
  if (rc != HPCS_OK) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t s = ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_a, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_b, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  U* d = static_cast<U*>(ctx->keys_a.ptr);
  U* o = static_cast<U*>(ctx->keys_b.ptr);
  if ((rc = copy_to_device(ctx, d, a, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  SelectState* st = nullptr;
  if ((rc = enqueue_select<U, KIND>(ctx, d, n, k, s, &st)) != HPCS_OK) return rc;
  if ((rc = enqueue_partition<U, KIND>(ctx, d, n, st, o, s)) != HPCS_OK) return rc;
  if ((rc = copy_to_host(ctx, a, o, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  return check_device_errors(ctx);
}

template <class T, class U, int KIND>
int select_topk_dev(hpcs_ctx* ctx, T* a, int64_t n, int64_t k, void* stream) {
  int rc = check_select_args(ctx, a, n, k);
  if (rc != HPCS_OK) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_b, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  U* d = reinterpret_cast<U*>(a);
  U* o = static_cast<U*>(ctx->keys_b.ptr);
  SelectState* st = nullptr;
  if ((rc = enqueue_select<U, KIND>(ctx, d, n, k, s, &st)) != HPCS_OK) return rc;
  if ((rc = enqueue_partition<U, KIND>(ctx, d, n, st, o, s)) != HPCS_OK) return rc;
  HPCS_CUDA(cudaMemcpyAsync(d, o, size_t(n) * sizeof(U), cudaMemcpyDeviceToDevice, s));
  return HPCS_OK;
}

// ---- PartitionRadix / SelectRadix(Par) ---------------------------------------------------
// Up to this many distinct k indices are placed by successive radix selects and three-way
// partitions of the part above the previous one; more indices sort the subarray, which places
// every index at once (a sorted array is a valid partition for any k).
constexpr int64_t PARTITION_MAX_SELECTS = 4;
static_assert(offsetof(SelectState, eq) == offsetof(SelectState, less) + sizeof(int64_t), "less, eq adjacent");

int check_partition_args(hpcs_ctx* ctx, const void* a, int64_t start, int64_t length, const int64_t* ks,
                         int64_t nk) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  if (!a) return fail(HPCS_ERR_NULL, "array is NULL");
  if (nk > 0 && !ks) return fail(HPCS_ERR_NULL, "k is NULL");
  // PartitionRadix.cs:139-140, :173-174; SelectionRadixParallel.cs:258-261
  if (start < 0 || length <= 0) return fail(HPCS_ERR_RANGE, "array length or length is invalid");
  if (length > HPCS_MAX_SEGMENT_KEYS) return fail(HPCS_ERR_RANGE, "length exceeds HPCS_MAX_SEGMENT_KEYS");
  if (nk < 0) return fail(HPCS_ERR_RANGE, "the number of k indices is negative");
  for (int64_t i = 0; i < nk; i++)
    if (ks[i] < start || ks[i] >= start + length)
      return fail(HPCS_ERR_RANGE, "k must be between start and (start + length)");
  return HPCS_OK;
}

// Places the (ascending, distinct) relative ranks r[] in d[0..n) on the device: afterwards d[r_i]
// is the key the sorted range has at r_i, and the keys between two consecutive r's lie between
// their values.  o is scratch of n keys.  Successive selects and three-way partitions of the part
// above the previous rank's run of equal keys, or one sort when there are many ranks.
template <class U, int KIND>
int enqueue_partition_ranks(hpcs_ctx* ctx, U* d, U* o, int64_t n, const std::vector<int64_t>& r, cudaStream_t s) {
  int rc;
  if (int64_t(r.size()) > PARTITION_MAX_SELECTS) return enqueue_sort<U, KIND, NoValue>(ctx, d, nullptr, n, s);
  int64_t lo = 0;  // keys below lo are placed: every later rank lies at or above it
  for (int64_t rank : r) {
    if (rank < lo) continue;  // inside the previous rank's run of keys equal to its key
    SelectState* st = nullptr;
    if ((rc = enqueue_select<U, KIND>(ctx, d + lo, n - lo, rank - lo, s, &st)) != HPCS_OK) return rc;
    if ((rc = enqueue_partition<U, KIND>(ctx, d + lo, n - lo, st, o + lo, s)) != HPCS_OK) return rc;
    HPCS_CUDA(cudaMemcpyAsync(d + lo, o + lo, size_t(n - lo) * sizeof(U), cudaMemcpyDeviceToDevice, s));
    int64_t less_eq[2] = {0, 0};  // SelectState::less and ::eq are adjacent
    HPCS_CUDA(cudaMemcpyAsync(less_eq, &st->less, sizeof(less_eq), cudaMemcpyDeviceToHost, s));
    HPCS_CUDA(cudaStreamSynchronize(s));
    lo += less_eq[0] + less_eq[1];
  }
  return HPCS_OK;
}

// PartitionRadix(this T[] a, int start, int length, int k / int[] k): host array, in place.
template <class T, class U, int KIND>
int partition_radix_host(hpcs_ctx* ctx, T* a, int64_t start, int64_t length, const int64_t* ks, int64_t nk) {
  int rc = check_partition_args(ctx, a, start, length, ks, nk);
  if (rc != HPCS_OK || nk == 0) return rc;
  std::vector<int64_t> r(ks, ks + nk);
  for (auto& x : r) x -= start;
  std::sort(r.begin(), r.end());
  r.erase(std::unique(r.begin(), r.end()), r.end());
  DeviceGuard g(ctx->device);
  cudaStream_t s = ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_a, size_t(length) * sizeof(U))) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->vals_a, size_t(length) * sizeof(U))) != HPCS_OK) return rc;
  U* d = static_cast<U*>(ctx->keys_a.ptr);
  U* o = static_cast<U*>(ctx->vals_a.ptr);
  if ((rc = copy_to_device(ctx, d, a + start, size_t(length) * sizeof(U), s)) != HPCS_OK) return rc;
  if ((rc = enqueue_partition_ranks<U, KIND>(ctx, d, o, length, r, s)) != HPCS_OK) return rc;
  if ((rc = copy_to_host(ctx, a + start, d, size_t(length) * sizeof(U), s)) != HPCS_OK) return rc;
  return check_device_errors(ctx);
}

// SelectRadix / SelectRadixPar(this T[] a, int start, int length, int k): the k-th smallest key of
// a[start, start + length) (k absolute) into *out, left at a[k]; a is partitioned around it.
template <class T, class U, int KIND>
int select_radix_host(hpcs_ctx* ctx, T* a, int64_t start, int64_t length, int64_t k, T* out) {
  if (!out) return fail(HPCS_ERR_NULL, "out is NULL");
  int rc = partition_radix_host<T, U, KIND>(ctx, a, start, length, &k, 1);
  if (rc != HPCS_OK) return rc;
  *out = a[k];
  return HPCS_OK;
}

int check_topk_args(hpcs_ctx* ctx, const void* in, const void* out, int64_t n, int64_t k) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  if (!in || !out) return fail(HPCS_ERR_NULL, "array is NULL");
  if (n < 0 || n > HPCS_MAX_SEGMENT_KEYS) return fail(HPCS_ERR_RANGE, "length out of range");
  if (k < 0 || k > n) return fail(HPCS_ERR_RANGE, "k must be in [0, length]");
  return HPCS_OK;
}

template <class T, class U, int KIND>
int topk_largest_dev(hpcs_ctx* ctx, const T* in, int64_t n, int64_t k, T* out, void* stream) {
  int rc = check_topk_args(ctx, in, out, n, k);
  if (rc != HPCS_OK || k == 0) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  return topk_largest_enqueue<T, U, KIND>(ctx, reinterpret_cast<const U*>(in), n, k, reinterpret_cast<U*>(out), s);
}

template <class T, class U, int KIND>
int topk_largest_host(hpcs_ctx* ctx, const T* in, int64_t n, int64_t k, T* out) {
  int rc = check_topk_args(ctx, in, out, n, k);
  if (rc != HPCS_OK || k == 0) return rc;
  DeviceGuard g(ctx->device);
  cudaStream_t s = ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->keys_a, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->vals_a, size_t(k) * sizeof(U))) != HPCS_OK) return rc;
  U* d = static_cast<U*>(ctx->keys_a.ptr);
  U* o = static_cast<U*>(ctx->vals_a.ptr);
  if ((rc = copy_to_device(ctx, d, in, size_t(n) * sizeof(U), s)) != HPCS_OK) return rc;
  if ((rc = topk_largest_enqueue<T, U, KIND>(ctx, d, n, k, o, s)) != HPCS_OK) return rc;
  HPCS_CUDA(cudaMemcpyAsync(out, o, size_t(k) * sizeof(U), cudaMemcpyDeviceToHost, s));
  HPCS_CUDA(cudaStreamSynchronize(s));
  return check_device_errors(ctx);
}

// Count, scan and scatter of one shard into `parts` parts (shard.cuh), the kernels built
// for LOG = ceil(log2(parts)).  shard_ctas_per_sm CTAs per SM (the scatter kernel's register
// budget), each a contiguous range of whole tiles; both passes use the same ranges.
template <class U, int KIND, int LOG>
int launch_shard_partition(hpcs_ctx* ctx, const U* keys, const uint32_t* items, int64_t n, int64_t gpos0,
                           const U* split_keys, const int64_t* split_gpos, int parts, U* keys_out,
                           uint32_t* items_out, int64_t* counts_out, cudaStream_t s) {
  const int64_t tiles = (n + SHARD_TILE - 1) / SHARD_TILE;
  const int64_t cap = int64_t(ctx->sms) * (items ? shard_ctas_per_sm<U, true>() : shard_ctas_per_sm<U, false>());
  const int grid = int(tiles < cap ? tiles : cap);
  const int64_t per_cta = (tiles + grid - 1) / grid * SHARD_TILE;
  int rc;
  if ((rc = ensure(ctx, ctx->aux0, size_t(grid) * parts * 4)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->aux1, size_t(grid) * parts * 8)) != HPCS_OK) return rc;
  uint32_t* cta_counts = static_cast<uint32_t*>(ctx->aux0.ptr);
  int64_t* cta_offsets = static_cast<int64_t*>(ctx->aux1.ptr);
  static int attr_set[64] = {0};  // per instance: the scatter kernels' shared memory limit
  if (!attr_set[ctx->device & 63]) {
    HPCS_CUDA(cudaFuncSetAttribute(shard_scatter_kernel<U, KIND, true, LOG>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(shard_scatter_smem<U, true>(SHARD_MAX_PARTS))));
    HPCS_CUDA(cudaFuncSetAttribute(shard_scatter_kernel<U, KIND, false, LOG>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(shard_scatter_smem<U, false>(SHARD_MAX_PARTS))));
    attr_set[ctx->device & 63] = 1;
  }
  KernelTimer kt(ctx, s, HPCS_K_SHARD);
  shard_count_kernel<U, KIND, LOG><<<grid, SHARD_COUNT_NT, 0, s>>>(keys, n, per_cta, gpos0, split_keys, split_gpos,
                                                                   parts, cta_counts);
  HPCS_CUDA(cudaGetLastError());
  shard_scan_kernel<<<1, 1024, 0, s>>>(cta_counts, grid, parts, cta_offsets, counts_out);
  HPCS_CUDA(cudaGetLastError());
  if (items)
    shard_scatter_kernel<U, KIND, true, LOG><<<grid, SHARD_NT, shard_scatter_smem<U, true>(parts), s>>>(
        keys, items, n, per_cta, gpos0, split_keys, split_gpos, parts, cta_offsets, keys_out, items_out);
  else
    shard_scatter_kernel<U, KIND, false, LOG><<<grid, SHARD_NT, shard_scatter_smem<U, false>(parts), s>>>(
        keys, nullptr, n, per_cta, gpos0, split_keys, split_gpos, parts, cta_offsets, keys_out, nullptr);
  HPCS_CUDA(cudaGetLastError());
  return HPCS_OK;
}

template <class U, int KIND>
int enqueue_shard_partition(hpcs_ctx* ctx, const U* keys, const uint32_t* items, int64_t n, int64_t gpos0,
                            const U* split_keys, const int64_t* split_gpos, int parts, U* keys_out,
                            uint32_t* items_out, int64_t* counts_out, cudaStream_t s) {
  if (n == 0) {
    HPCS_CUDA(cudaMemsetAsync(counts_out, 0, size_t(parts) * 8, s));
    return HPCS_OK;
  }
  int log = 0;
  while ((1 << log) < parts) log++;
#define HPCS_SHARD_LOG(L)                                                                                      \
  case L:                                                                                                      \
    return launch_shard_partition<U, KIND, L>(ctx, keys, items, n, gpos0, split_keys, split_gpos, parts, keys_out, \
                                              items_out, counts_out, s);
  switch (log) {
    HPCS_SHARD_LOG(0)
    HPCS_SHARD_LOG(1)
    HPCS_SHARD_LOG(2)
    HPCS_SHARD_LOG(3)
    HPCS_SHARD_LOG(4)
    HPCS_SHARD_LOG(5)
    HPCS_SHARD_LOG(6)
    default: return fail(HPCS_ERR_RANGE, "parts must be in [1, HPCS_MAX_PARTS]");
  }
#undef HPCS_SHARD_LOG
}

template <class U, int KIND>
int shard_partition_typed(hpcs_ctx* ctx, const void* keys, const uint32_t* items, int64_t n, int64_t gpos0,
                          const void* split_keys, const int64_t* split_gpos, int parts, void* keys_out,
                          uint32_t* items_out, int64_t* counts_out, cudaStream_t s) {
  return enqueue_shard_partition<U, KIND>(ctx, static_cast<const U*>(keys), items, n, gpos0,
                                          static_cast<const U*>(split_keys), split_gpos, parts,
                                          static_cast<U*>(keys_out), items_out, counts_out, s);
}

}  // namespace
}  // namespace hpcs

using namespace hpcs;

extern "C" {

void hpcs_config_default(hpcs_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->pool_bytes = 0;
  cfg->skip_trivial_passes = 1;
  cfg->spin_limit_ns = 2000000000LL;
  cfg->poison_tile = -1;
  cfg->rank_mode = 0;
  cfg->staged_host_copies = 1;
}

int hpcs_abi_version(void) { return HPCS_ABI_VERSION; }

const char* hpcs_last_error_message(void) { return g_last_error.c_str(); }

const char* hpcs_status_string(int status) {
  switch (status) {
    case HPCS_OK: return "HPCS_OK";
    case HPCS_ERR_NULL: return "HPCS_ERR_NULL";
    case HPCS_ERR_RANGE: return "HPCS_ERR_RANGE";
    case HPCS_ERR_OOM: return "HPCS_ERR_OOM";
    case HPCS_ERR_CUDA: return "HPCS_ERR_CUDA";
    case HPCS_ERR_DEVICE_TIMEOUT: return "HPCS_ERR_DEVICE_TIMEOUT";
    case HPCS_ERR_UNSUPPORTED: return "HPCS_ERR_UNSUPPORTED";
    case HPCS_ERR_NO_DEVICE: return "HPCS_ERR_NO_DEVICE";
    case HPCS_ERR_BUSY: return "HPCS_ERR_BUSY";
    default: return "HPCS_ERR_UNKNOWN";
  }
}

int hpcs_ctx_create(int device, const hpcs_config* cfg, hpcs_ctx** out) {
  if (!out) return fail(HPCS_ERR_NULL, "out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(HPCS_ERR_NO_DEVICE, "no CUDA device is available");
  }
  if (device < 0 || device >= count) return fail(HPCS_ERR_RANGE, "device index out of range");
  DeviceGuard g(device);
  auto* ctx = new hpcs_ctx();
  ctx->device = device;
  if (cfg) ctx->cfg = *cfg;
  else hpcs_config_default(&ctx->cfg);
  if (ctx->cfg.spin_limit_ns <= 0) ctx->cfg.spin_limit_ns = 2000000000LL;
  cudaDeviceProp prop{};
  if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) {
    delete ctx;
    return cuda_fail(e, "cudaGetDeviceProperties");
  }
  if (prop.major < 10) {
    delete ctx;
    return fail(HPCS_ERR_UNSUPPORTED, "libhpcs_gpu is built for sm_100a (B200)");
  }
  ctx->sms = prop.multiProcessorCount;
  ctx->seg_tuning = seg_default_tuning();
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&ctx->order_event, cudaEventDisableTiming)) != cudaSuccess) {
    delete ctx;
    return cuda_fail(e, "stream/event create");
  }
  int rc = ensure(ctx, ctx->err_accum, 256);
  if (rc != HPCS_OK || cudaMemset(ctx->err_accum.ptr, 0, 256) != cudaSuccess) {
    hpcs_ctx_destroy(ctx);
    return rc != HPCS_OK ? rc : fail(HPCS_ERR_CUDA, "cudaMemset");
  }
  ctx->rank_mode = RANK_PEER_MASK;
  if (ctx->cfg.rank_mode == 0) {
    int ordered = 0;
    if ((rc = probe_rank_order(ctx, &ordered)) != HPCS_OK) {
      hpcs_ctx_destroy(ctx);
      return rc;
    }
    if (ordered) {
      // once per device and process, with the first context: the shipping kernels themselves
      static std::mutex probe_mu;
      static int shipping[64];  // 0 unknown, 1 passed, 2 failed
      std::lock_guard<std::mutex> lock(probe_mu);
      int& sp = shipping[device & 63];
      if (sp == 0) {
        int ok = 0;
        if ((rc = probe_shipping_kernels(ctx, &ok)) != HPCS_OK) {
          hpcs_ctx_destroy(ctx);
          return rc;
        }
        sp = ok ? 1 : 2;
      }
      if (sp == 1) ctx->rank_mode = RANK_ORDERED_ATOMIC;
    }
  }
  *out = ctx;
  return HPCS_OK;
}

int hpcs_ctx_destroy(hpcs_ctx* ctx) {
  if (!ctx) return HPCS_OK;
  DeviceGuard g(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->last_stream && ctx->last_stream != ctx->stream) cudaStreamSynchronize(ctx->last_stream);
  DevBuf* bufs[] = {&ctx->keys_a, &ctx->keys_b,  &ctx->vals_a,    &ctx->vals_b, &ctx->status0,
                    &ctx->status1, &ctx->status2, &ctx->plan, &ctx->counts, &ctx->err_accum,
                    &ctx->aux0,   &ctx->aux1,    &ctx->aux2};
  for (DevBuf* b : bufs)
    if (b->ptr && !b->borrowed) cudaFree(b->ptr);
  for (auto& t : ctx->timed) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
  if (ctx->order_event) cudaEventDestroy(ctx->order_event);
  for (int b = 0; b < hpcs_ctx::SEG_BRANCHES; b++) {
    if (ctx->seg_streams[b]) cudaStreamSynchronize(ctx->seg_streams[b]);
    if (ctx->seg_streams[b]) cudaStreamDestroy(ctx->seg_streams[b]);
    if (ctx->seg_join[b]) cudaEventDestroy(ctx->seg_join[b]);
  }
  if (ctx->seg_fork) cudaEventDestroy(ctx->seg_fork);
  if (ctx->seg_grid_stream) {
    cudaStreamSynchronize(ctx->seg_grid_stream);
    cudaStreamDestroy(ctx->seg_grid_stream);
  }
  if (ctx->seg_grid_fork) cudaEventDestroy(ctx->seg_grid_fork);
  if (ctx->seg_grid_join) cudaEventDestroy(ctx->seg_grid_join);
  delete ctx->stager;
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return HPCS_OK;
}

int hpcs_ctx_synchronize(hpcs_ctx* ctx) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  DeviceGuard g(ctx->device);
  HPCS_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ctx->last_stream && ctx->last_stream != ctx->stream) HPCS_CUDA(cudaStreamSynchronize(ctx->last_stream));
  return check_device_errors(ctx);
}

int hpcs_ctx_profile_enable(hpcs_ctx* ctx, int enable) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  ctx->profile = enable != 0;
  return HPCS_OK;
}

int hpcs_ctx_profile_read(hpcs_ctx* ctx, hpcs_profile* out) {
  if (!ctx || !out) return fail(HPCS_ERR_NULL, "ctx or out is NULL");
  DeviceGuard g(ctx->device);
  std::memset(out, 0, sizeof(*out));
  for (auto& t : ctx->timed) {
    HPCS_CUDA(cudaEventSynchronize(t.b));
    float ms = 0.f;
    HPCS_CUDA(cudaEventElapsedTime(&ms, t.a, t.b));
    if (t.cls >= 0 && t.cls < HPCS_K_CLASSES) {
      out->launches[t.cls] += 1;
      out->total_ms[t.cls] += ms;
    }
    ctx->event_pool.push_back(t.a);
    ctx->event_pool.push_back(t.b);
  }
  ctx->timed.clear();
  return HPCS_OK;
}

void* hpcs_ctx_stream(hpcs_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int hpcs_ctx_trace_tiles(hpcs_ctx* ctx, uint64_t* trace, int capacity_tiles, int pass) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  if (trace && capacity_tiles <= 0) return fail(HPCS_ERR_RANGE, "capacity must be positive");
  ctx->trace = trace;
  ctx->trace_capacity = trace ? capacity_tiles : 0;
  ctx->trace_pass = pass;
  return HPCS_OK;
}

int hpcs_ctx_rank_mode(hpcs_ctx* ctx) { return ctx ? ctx->rank_mode : -HPCS_ERR_NULL; }

// ---- plain sorts ----
int hpcs_sort_u32(hpcs_ctx* c, uint32_t* k, int64_t n) { return sort_host<uint32_t, uint32_t, KIND_UNSIGNED>(c, k, n); }
int hpcs_sort_i32(hpcs_ctx* c, int32_t* k, int64_t n) { return sort_host<int32_t, uint32_t, KIND_SIGNED>(c, k, n); }
int hpcs_sort_f32(hpcs_ctx* c, float* k, int64_t n) { return sort_host<float, uint32_t, KIND_FLOAT>(c, k, n); }
int hpcs_sort_u64(hpcs_ctx* c, uint64_t* k, int64_t n) { return sort_host<uint64_t, uint64_t, KIND_UNSIGNED>(c, k, n); }
int hpcs_sort_i64(hpcs_ctx* c, int64_t* k, int64_t n) { return sort_host<int64_t, uint64_t, KIND_SIGNED>(c, k, n); }
int hpcs_sort_f64(hpcs_ctx* c, double* k, int64_t n) { return sort_host<double, uint64_t, KIND_FLOAT>(c, k, n); }

int hpcs_sort_u32_dev(hpcs_ctx* c, uint32_t* k, int64_t n, void* s) {
  return sort_dev<uint32_t, uint32_t, KIND_UNSIGNED>(c, k, n, s);
}
int hpcs_sort_i32_dev(hpcs_ctx* c, int32_t* k, int64_t n, void* s) {
  return sort_dev<int32_t, uint32_t, KIND_SIGNED>(c, k, n, s);
}
int hpcs_sort_f32_dev(hpcs_ctx* c, float* k, int64_t n, void* s) { return sort_dev<float, uint32_t, KIND_FLOAT>(c, k, n, s); }
int hpcs_sort_u64_dev(hpcs_ctx* c, uint64_t* k, int64_t n, void* s) {
  return sort_dev<uint64_t, uint64_t, KIND_UNSIGNED>(c, k, n, s);
}
int hpcs_sort_i64_dev(hpcs_ctx* c, int64_t* k, int64_t n, void* s) {
  return sort_dev<int64_t, uint64_t, KIND_SIGNED>(c, k, n, s);
}
int hpcs_sort_f64_dev(hpcs_ctx* c, double* k, int64_t n, void* s) {
  return sort_dev<double, uint64_t, KIND_FLOAT>(c, k, n, s);
}

// ---- pairs ----
int hpcs_sort_pairs_u32(hpcs_ctx* c, uint32_t* k, uint32_t* v, int64_t n) {
  return pairs_host<uint32_t, uint32_t, KIND_UNSIGNED>(c, k, v, n);
}
int hpcs_sort_pairs_i32(hpcs_ctx* c, int32_t* k, uint32_t* v, int64_t n) {
  return pairs_host<int32_t, uint32_t, KIND_SIGNED>(c, k, v, n);
}
int hpcs_sort_pairs_f32(hpcs_ctx* c, float* k, uint32_t* v, int64_t n) {
  return pairs_host<float, uint32_t, KIND_FLOAT>(c, k, v, n);
}
int hpcs_sort_pairs_u64(hpcs_ctx* c, uint64_t* k, uint32_t* v, int64_t n) {
  return pairs_host<uint64_t, uint64_t, KIND_UNSIGNED>(c, k, v, n);
}
int hpcs_sort_pairs_i64(hpcs_ctx* c, int64_t* k, uint32_t* v, int64_t n) {
  return pairs_host<int64_t, uint64_t, KIND_SIGNED>(c, k, v, n);
}
int hpcs_sort_pairs_f64(hpcs_ctx* c, double* k, uint32_t* v, int64_t n) {
  return pairs_host<double, uint64_t, KIND_FLOAT>(c, k, v, n);
}
int hpcs_sort_pairs_u32_dev(hpcs_ctx* c, uint32_t* k, uint32_t* v, int64_t n, void* s) {
  return pairs_dev<uint32_t, uint32_t, KIND_UNSIGNED>(c, k, v, n, s);
}
int hpcs_sort_pairs_i32_dev(hpcs_ctx* c, int32_t* k, uint32_t* v, int64_t n, void* s) {
  return pairs_dev<int32_t, uint32_t, KIND_SIGNED>(c, k, v, n, s);
}
int hpcs_sort_pairs_f32_dev(hpcs_ctx* c, float* k, uint32_t* v, int64_t n, void* s) {
  return pairs_dev<float, uint32_t, KIND_FLOAT>(c, k, v, n, s);
}
int hpcs_sort_pairs_u64_dev(hpcs_ctx* c, uint64_t* k, uint32_t* v, int64_t n, void* s) {
  return pairs_dev<uint64_t, uint64_t, KIND_UNSIGNED>(c, k, v, n, s);
}
int hpcs_sort_pairs_i64_dev(hpcs_ctx* c, int64_t* k, uint32_t* v, int64_t n, void* s) {
  return pairs_dev<int64_t, uint64_t, KIND_SIGNED>(c, k, v, n, s);
}
int hpcs_sort_pairs_f64_dev(hpcs_ctx* c, double* k, uint32_t* v, int64_t n, void* s) {
  return pairs_dev<double, uint64_t, KIND_FLOAT>(c, k, v, n, s);
}

// ---- histograms ----
int hpcs_histogram_byte_components_u32(hpcs_ctx* c, const uint32_t* a, int64_t l, int64_t r, uint32_t* o) {
  return histogram_host<uint32_t, uint32_t, KIND_UNSIGNED>(c, a, l, r, o);
}
int hpcs_histogram_byte_components_i32(hpcs_ctx* c, const int32_t* a, int64_t l, int64_t r, uint32_t* o) {
  return histogram_host<int32_t, uint32_t, KIND_SIGNED>(c, a, l, r, o);
}
int hpcs_histogram_byte_components_f32(hpcs_ctx* c, const float* a, int64_t l, int64_t r, uint32_t* o) {
  return histogram_host<float, uint32_t, KIND_FLOAT>(c, a, l, r, o);
}
int hpcs_histogram_byte_components_u64(hpcs_ctx* c, const uint64_t* a, int64_t l, int64_t r, uint32_t* o) {
  return histogram_host<uint64_t, uint64_t, KIND_UNSIGNED>(c, a, l, r, o);
}
int hpcs_histogram_byte_components_i64(hpcs_ctx* c, const int64_t* a, int64_t l, int64_t r, uint32_t* o) {
  return histogram_host<int64_t, uint64_t, KIND_SIGNED>(c, a, l, r, o);
}
int hpcs_histogram_byte_components_f64(hpcs_ctx* c, const double* a, int64_t l, int64_t r, uint32_t* o) {
  return histogram_host<double, uint64_t, KIND_FLOAT>(c, a, l, r, o);
}

int hpcs_sort_u8(hpcs_ctx* c, uint8_t* k, int64_t n) { return count_sort_host<uint8_t, uint8_t>(c, k, n, 0u); }
int hpcs_sort_i8(hpcs_ctx* c, int8_t* k, int64_t n) { return count_sort_host<int8_t, uint8_t>(c, k, n, 0x80u); }
int hpcs_sort_u16(hpcs_ctx* c, uint16_t* k, int64_t n) { return count_sort_host<uint16_t, uint16_t>(c, k, n, 0u); }
int hpcs_sort_i16(hpcs_ctx* c, int16_t* k, int64_t n) { return count_sort_host<int16_t, uint16_t>(c, k, n, 0x8000u); }
int hpcs_sort_u8_dev(hpcs_ctx* c, uint8_t* k, int64_t n, void* s) { return count_sort_dev<uint8_t, uint8_t>(c, k, n, 0u, s); }
int hpcs_sort_i8_dev(hpcs_ctx* c, int8_t* k, int64_t n, void* s) { return count_sort_dev<int8_t, uint8_t>(c, k, n, 0x80u, s); }
int hpcs_sort_u16_dev(hpcs_ctx* c, uint16_t* k, int64_t n, void* s) {
  return count_sort_dev<uint16_t, uint16_t>(c, k, n, 0u, s);
}
int hpcs_sort_i16_dev(hpcs_ctx* c, int16_t* k, int64_t n, void* s) {
  return count_sort_dev<int16_t, uint16_t>(c, k, n, 0x8000u, s);
}

#define HPCS_TOPK_EXPORTS(NAME, T, U, KIND)                                                          \
  int hpcs_select_topk_##NAME(hpcs_ctx* c, T* a, int64_t n, int64_t k) {                            \
    return select_topk_host<T, U, KIND>(c, a, n, k);                                                 \
  }                                                                                                  \
  int hpcs_select_topk_##NAME##_dev(hpcs_ctx* c, T* a, int64_t n, int64_t k, void* s) {             \
    return select_topk_dev<T, U, KIND>(c, a, n, k, s);                                               \
  }                                                                                                  \
  int hpcs_topk_largest_##NAME(hpcs_ctx* c, const T* in, int64_t n, int64_t k, T* out) {            \
    return topk_largest_host<T, U, KIND>(c, in, n, k, out);                                          \
  }                                                                                                  \
  int hpcs_topk_largest_##NAME##_dev(hpcs_ctx* c, const T* in, int64_t n, int64_t k, T* out, void* s) { \
    return topk_largest_dev<T, U, KIND>(c, in, n, k, out, s);                                        \
  }
HPCS_TOPK_EXPORTS(u32, uint32_t, uint32_t, KIND_UNSIGNED)
HPCS_TOPK_EXPORTS(i32, int32_t, uint32_t, KIND_SIGNED)
HPCS_TOPK_EXPORTS(f32, float, uint32_t, KIND_FLOAT)
HPCS_TOPK_EXPORTS(u64, uint64_t, uint64_t, KIND_UNSIGNED)
HPCS_TOPK_EXPORTS(i64, int64_t, uint64_t, KIND_SIGNED)
HPCS_TOPK_EXPORTS(f64, double, uint64_t, KIND_FLOAT)

#define HPCS_PARTITION_EXPORTS(NAME, T, U, KIND)                                                      \
  int hpcs_partition_radix_##NAME(hpcs_ctx* c, T* a, int64_t start, int64_t length, const int64_t* k,     \
                                  int64_t nk) {                                                            \
    return partition_radix_host<T, U, KIND>(c, a, start, length, k, nk);                                   \
  }                                                                                                        \
  int hpcs_select_radix_##NAME(hpcs_ctx* c, T* a, int64_t start, int64_t length, int64_t k, T* out) {     \
    return select_radix_host<T, U, KIND>(c, a, start, length, k, out);                                     \
  }
HPCS_PARTITION_EXPORTS(u32, uint32_t, uint32_t, KIND_UNSIGNED)
HPCS_PARTITION_EXPORTS(i32, int32_t, uint32_t, KIND_SIGNED)
HPCS_PARTITION_EXPORTS(f32, float, uint32_t, KIND_FLOAT)
HPCS_PARTITION_EXPORTS(u64, uint64_t, uint64_t, KIND_UNSIGNED)
HPCS_PARTITION_EXPORTS(i64, int64_t, uint64_t, KIND_SIGNED)
HPCS_PARTITION_EXPORTS(f64, double, uint64_t, KIND_FLOAT)

int hpcs_histogram_byte_components_dev(hpcs_ctx* ctx, int dtype, const void* a, int64_t n, uint32_t* counts,
                                       void* stream) {
  int rc = check_common(ctx, a, n);
  if (rc != HPCS_OK) return rc;
  if (!counts) return fail(HPCS_ERR_NULL, "counts is NULL");
  DeviceGuard g(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  switch (dtype) {
    case HPCS_U32: return enqueue_histogram<uint32_t, KIND_UNSIGNED>(ctx, static_cast<const uint32_t*>(a), n, counts, s);
    case HPCS_I32: return enqueue_histogram<uint32_t, KIND_SIGNED>(ctx, static_cast<const uint32_t*>(a), n, counts, s);
    case HPCS_F32: return enqueue_histogram<uint32_t, KIND_FLOAT>(ctx, static_cast<const uint32_t*>(a), n, counts, s);
    case HPCS_U64: return enqueue_histogram<uint64_t, KIND_UNSIGNED>(ctx, static_cast<const uint64_t*>(a), n, counts, s);
    case HPCS_I64: return enqueue_histogram<uint64_t, KIND_SIGNED>(ctx, static_cast<const uint64_t*>(a), n, counts, s);
    case HPCS_F64: return enqueue_histogram<uint64_t, KIND_FLOAT>(ctx, static_cast<const uint64_t*>(a), n, counts, s);
    default: return fail(HPCS_ERR_UNSUPPORTED, "unknown dtype");
  }
}

int hpcs_shard_partition_dev(hpcs_ctx* ctx, int dtype, const void* keys, const uint32_t* items, int64_t n,
                             int64_t gpos0, const void* split_keys, const int64_t* split_gpos, int parts,
                             void* keys_out, uint32_t* items_out, int64_t* counts_out, void* stream) {
  int rc = check_common(ctx, keys, n);
  if (rc != HPCS_OK) return rc;
  if (!keys_out || !counts_out) return fail(HPCS_ERR_NULL, "keys_out or counts_out is NULL");
  if ((items == nullptr) != (items_out == nullptr)) return fail(HPCS_ERR_NULL, "items and items_out must both be set");
  if (parts < 1 || parts > HPCS_MAX_PARTS) return fail(HPCS_ERR_RANGE, "parts must be in [1, HPCS_MAX_PARTS]");
  if (parts > 1 && (!split_keys || !split_gpos)) return fail(HPCS_ERR_NULL, "splitters are NULL");
  if (gpos0 < 0) return fail(HPCS_ERR_RANGE, "gpos0 is negative");
  if (keys_out == keys) return fail(HPCS_ERR_RANGE, "keys_out must not overlap keys");
  DeviceGuard g(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
#define HPCS_SHARD_CASE(DT, U, KIND) \
  case DT:                          \
    return shard_partition_typed<U, KIND>(ctx, keys, items, n, gpos0, split_keys, split_gpos, parts, keys_out, \
                                          items_out, counts_out, s);
  switch (dtype) {
    HPCS_SHARD_CASE(HPCS_U32, uint32_t, KIND_UNSIGNED)
    HPCS_SHARD_CASE(HPCS_I32, uint32_t, KIND_SIGNED)
    HPCS_SHARD_CASE(HPCS_F32, uint32_t, KIND_FLOAT)
    HPCS_SHARD_CASE(HPCS_U64, uint64_t, KIND_UNSIGNED)
    HPCS_SHARD_CASE(HPCS_I64, uint64_t, KIND_SIGNED)
    HPCS_SHARD_CASE(HPCS_F64, uint64_t, KIND_FLOAT)
    default: return fail(HPCS_ERR_UNSUPPORTED, "unknown dtype");
  }
#undef HPCS_SHARD_CASE
}

}  // extern "C"
