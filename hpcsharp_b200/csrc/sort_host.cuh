// Host-side launch logic for the LSD sort kernels: context state, scratch buffers,
// per-dtype kernel configuration and the enqueue sequence K1 -> K3 x P -> finalize.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hpcs_gpu.h"
#include "radix_kernels.cuh"

namespace hpcs {

// ---- thread-local error text ---------------------------------------------------------
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define HPCS_CUDA(call)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return ::hpcs::cuda_fail(e_, #call); \
  } while (0)

// Grow-only device buffer owned by a context.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace hpcs

struct hpcs_ctx {
  int device = 0;
  int sms = 0;
  hpcs_config cfg{};
  cudaStream_t stream = nullptr;
  cudaStream_t last_stream = nullptr;
  cudaEvent_t order_event = nullptr;
  size_t held_bytes = 0;
  // per-kernel timing
  bool profile = false;
  struct Timed {
    int cls;
    cudaEvent_t a, b;
  };
  std::vector<Timed> timed;
  std::vector<cudaEvent_t> event_pool;
  // scratch
  hpcs::DevBuf keys_a, keys_b, vals_a, vals_b, status0, status1, plan, counts, err_accum;
  hpcs::DevBuf aux0, aux1, aux2;
};

namespace hpcs {

int ensure(hpcs_ctx* ctx, DevBuf& b, size_t bytes);

// Brackets one kernel launch with an event pair when the context profiles.
struct KernelTimer {
  hpcs_ctx* ctx;
  cudaStream_t s;
  int cls;
  cudaEvent_t a = nullptr, b = nullptr;
  KernelTimer(hpcs_ctx* c, cudaStream_t st, int k);
  ~KernelTimer();
};
// Orders work on `s` after all earlier work of the context (scratch is shared).
int enter_stream(hpcs_ctx* ctx, cudaStream_t s);
uint32_t* device_error_word(hpcs_ctx* ctx);

template <class U, class V>
struct SortConfig;
// 32-bit keys: 512 threads x 16 keys = 8192-key tiles, 2 stages, 2 CTAs/SM.
template <>
struct SortConfig<uint32_t, NoValue> {
  static constexpr int NT = 512, KPT = 16, STAGES = 2, MINB = 2;
};
template <>
struct SortConfig<uint64_t, NoValue> {
  static constexpr int NT = 512, KPT = 8, STAGES = 2, MINB = 2;
};
template <>
struct SortConfig<uint32_t, uint32_t> {
  static constexpr int NT = 512, KPT = 8, STAGES = 2, MINB = 2;
};
template <>
struct SortConfig<uint64_t, uint32_t> {
  static constexpr int NT = 512, KPT = 6, STAGES = 2, MINB = 2;
};

constexpr int HIST_NT = 512;

template <class Kernel>
int occupancy_blocks(Kernel k, int nt, size_t smem) {
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, nt, smem) != cudaSuccess) return 1;
  return blocks > 0 ? blocks : 1;
}

// Enqueue a full LSD sort of n keys (and optional 4-byte items) in device memory.
// keys/vals are sorted in place (with scratch B owned by the context).
template <class U, int KIND, class V>
int enqueue_sort(hpcs_ctx* ctx, U* keys, uint32_t* vals, int64_t n, cudaStream_t s) {
  using C = SortConfig<U, V>;
  using L = OnesweepSmem<U, V, C::NT, C::KPT, C::STAGES>;
  constexpr bool PAIRS = !std::is_same<V, NoValue>::value;
  constexpr int P = int(sizeof(U));
  if (n <= 1) return HPCS_OK;
  if (n > MAX_KEYS_PER_SORT) return fail(HPCS_ERR_RANGE, "n exceeds HPCS_MAX_KEYS");
  const int64_t num_tiles = (n + L::TILE - 1) / L::TILE;

  // 16-byte alignment is required by the bulk copies; unaligned callers go through A'.
  U* a = keys;
  uint32_t* va = vals;
  const bool keys_unaligned = (reinterpret_cast<uintptr_t>(keys) & 15) != 0;
  const bool vals_unaligned = PAIRS && (reinterpret_cast<uintptr_t>(vals) & 15) != 0;
  int rc;
  if ((rc = ensure(ctx, ctx->keys_b, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  if (PAIRS && (rc = ensure(ctx, ctx->vals_b, size_t(n) * 4)) != HPCS_OK) return rc;
  if (keys_unaligned) {
    if ((rc = ensure(ctx, ctx->keys_a, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
    a = static_cast<U*>(ctx->keys_a.ptr);
    HPCS_CUDA(cudaMemcpyAsync(a, keys, size_t(n) * sizeof(U), cudaMemcpyDeviceToDevice, s));
  }
  if (vals_unaligned) {
    if ((rc = ensure(ctx, ctx->vals_a, size_t(n) * 4)) != HPCS_OK) return rc;
    va = static_cast<uint32_t*>(ctx->vals_a.ptr);
    HPCS_CUDA(cudaMemcpyAsync(va, vals, size_t(n) * 4, cudaMemcpyDeviceToDevice, s));
  }
  const size_t status_bytes = size_t(num_tiles) * RADIX * 4;
  if ((rc = ensure(ctx, ctx->status0, status_bytes)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->status1, status_bytes)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->plan, sizeof(SortPlan))) != HPCS_OK) return rc;

  SortArgs args{};
  args.keys_a = a;
  args.keys_b = ctx->keys_b.ptr;
  args.vals_a = va;
  args.vals_b = PAIRS ? ctx->vals_b.ptr : nullptr;
  args.n = n;
  args.plan = static_cast<SortPlan*>(ctx->plan.ptr);
  args.status[0] = static_cast<uint32_t*>(ctx->status0.ptr);
  args.status[1] = static_cast<uint32_t*>(ctx->status1.ptr);
  args.num_tiles = int(num_tiles);
  args.skip_trivial = ctx->cfg.skip_trivial_passes;
  args.poison_tile = ctx->cfg.poison_tile;
  args.spin_limit_ns = uint64_t(ctx->cfg.spin_limit_ns);

  HPCS_CUDA(cudaMemsetAsync(args.plan, 0, sizeof(SortPlan), s));

  // K1: fused histogram + plan
  {
    auto k = hist_all_digits_kernel<U, KIND, HIST_NT>;
    static int hist_blocks = 0;
    if (!hist_blocks) hist_blocks = occupancy_blocks(k, HIST_NT, 0);
    const int64_t vec = n * int64_t(sizeof(U)) / 16;
    int64_t want = (vec + HIST_NT * 4 - 1) / (HIST_NT * 4);
    int64_t cap = int64_t(ctx->sms) * hist_blocks;
    int grid = int(want < 1 ? 1 : (want > cap ? cap : want));
    KernelTimer kt(ctx, s, HPCS_K_HISTOGRAM);
    k<<<grid, HIST_NT, 0, s>>>(a, n, &args.plan->hist[0][0], args, 1);
    HPCS_CUDA(cudaGetLastError());
  }
  // K3: one onesweep launch per digit
  {
    auto k = onesweep_pass_kernel<U, KIND, V, C::NT, C::KPT, C::STAGES, C::MINB>;
    static int os_blocks = 0;
    if (!os_blocks) {
      HPCS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::BYTES)));
      os_blocks = occupancy_blocks(k, C::NT, L::BYTES);
    }
    int64_t cap = int64_t(ctx->sms) * os_blocks;
    int grid = int(num_tiles < cap ? num_tiles : cap);
    for (int p = 0; p < P; p++) {
      args.pass = p;
      KernelTimer kt(ctx, s, HPCS_K_ONESWEEP);
      k<<<grid, C::NT, L::BYTES, s>>>(args);
      HPCS_CUDA(cudaGetLastError());
    }
  }
  // finalize: result back into the caller's buffer if it ended in B; collect errors
  {
    int64_t want = (n + 255) / 256;
    int grid = int(want > int64_t(ctx->sms) * 8 ? int64_t(ctx->sms) * 8 : want);
    KernelTimer kt(ctx, s, HPCS_K_FINALIZE);
    finalize_kernel<U><<<grid, 256, 0, s>>>(args, PAIRS ? 1 : 0, device_error_word(ctx));
    HPCS_CUDA(cudaGetLastError());
  }
  if (keys_unaligned)
    HPCS_CUDA(cudaMemcpyAsync(keys, a, size_t(n) * sizeof(U), cudaMemcpyDeviceToDevice, s));
  if (vals_unaligned) HPCS_CUDA(cudaMemcpyAsync(vals, va, size_t(n) * 4, cudaMemcpyDeviceToDevice, s));
  return HPCS_OK;
}

}  // namespace hpcs
