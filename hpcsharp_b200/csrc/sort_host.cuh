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
#include "chunk_pass.cuh"
#include "radix_kernels.cuh"
#include "small_sort.cuh"

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

// Grow-only device buffer owned by a context.  A borrowed buffer is a slice of memory that
// someone else owns (the serving arena): it is never grown or freed by the context.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  bool borrowed = false;
};

}  // namespace hpcs

namespace hpcs {
struct HostStager;
}

struct hpcs_ctx {
  int device = 0;
  int sms = 0;
  int rank_mode = 1;  // hpcs::RankMode actually used
  hpcs_config cfg{};
  cudaStream_t stream = nullptr;
  cudaStream_t last_stream = nullptr;
  cudaEvent_t order_event = nullptr;
  size_t held_bytes = 0;
  // tile trace (debug)
  uint64_t* trace = nullptr;
  int trace_pass = -1;
  int trace_capacity = 0;
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
  hpcs::DevBuf status2;  // second look-back buffer when the device chooses the scheme
  hpcs::DevBuf aux0, aux1, aux2;
  // pinned ring and copy threads for host arrays in pageable memory (host_copy.cuh)
  hpcs::HostStager* stager = nullptr;
  // batched segmented sort: variant per (key width, length class), and the helper streams
  // and events that run the launches of different variants concurrently
  hpcs_seg_tuning seg_tuning{};
  static constexpr int SEG_BRANCHES = 3;
  cudaStream_t seg_streams[SEG_BRANCHES] = {};
  cudaEvent_t seg_fork = nullptr;
  cudaEvent_t seg_join[SEG_BRANCHES] = {};
  // the grid-level path of the batched sort runs on its own branch
  cudaStream_t seg_grid_stream = nullptr;
  cudaEvent_t seg_grid_fork = nullptr, seg_grid_join = nullptr;
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

template <class U, class V, int MODE>
struct SortConfig;
// Tile shapes (threads x keys per thread), prefetch stages, CTAs per SM and CTAs per
// look-back unit (cluster size), per key/payload type and ranking mode.  The 32-bit
// keys-only shape of the ordered-atomic ranking can be overridden at build time for
// tuning sweeps.
#ifndef HPCS_K32_NT
#define HPCS_K32_NT 1024
#endif
#ifndef HPCS_K32_KPT
#define HPCS_K32_KPT 16
#endif
#ifndef HPCS_K32_MINB
#define HPCS_K32_MINB 1
#endif
#ifndef HPCS_CL
#define HPCS_CL 1
#endif
template <>
struct SortConfig<uint32_t, NoValue, RANK_ORDERED_ATOMIC> {
  static constexpr int NT = HPCS_K32_NT, KPT = HPCS_K32_KPT, STAGES = 2, MINB = HPCS_K32_MINB, CL = HPCS_CL;
};
template <>
struct SortConfig<uint32_t, NoValue, RANK_PEER_MASK> {  // + 32 KiB of lane masks
  static constexpr int NT = 512, KPT = 16, STAGES = 2, MINB = 1, CL = 1;
};
template <int MODE>
struct SortConfig<uint64_t, NoValue, MODE> {
  static constexpr int NT = 512, KPT = 8, STAGES = 2, MINB = 2, CL = HPCS_CL;
};
template <int MODE>
struct SortConfig<uint32_t, uint32_t, MODE> {
  static constexpr int NT = 512, KPT = 8, STAGES = 2, MINB = 2, CL = HPCS_CL;
};
template <int MODE>
struct SortConfig<uint64_t, uint32_t, MODE> {
  static constexpr int NT = 512, KPT = 6, STAGES = 2, MINB = 2, CL = HPCS_CL;
};

// Chunked-pass tile shapes (threads x keys per thread).  Every shape keeps its two stage
// buffers within 128 KiB, which leaves room for 148 ranges x 512 bytes of next-digit
// counters within the 227 KiB of shared memory a CTA may use.
#ifndef HPCS_C32_NT
#define HPCS_C32_NT 512
#endif
#ifndef HPCS_C32_KPT
#define HPCS_C32_KPT 32
#endif
#ifndef HPCS_C64_KPT
#define HPCS_C64_KPT 16
#endif
#ifndef HPCS_CP32_KPT
#define HPCS_CP32_KPT 16
#endif
#ifndef HPCS_CP64_KPT
#define HPCS_CP64_KPT 10
#endif
template <class U, class V, int MODE>
struct ChunkConfig;
template <>
struct ChunkConfig<uint32_t, NoValue, RANK_ORDERED_ATOMIC> {
  static constexpr int NT = HPCS_C32_NT, KPT = HPCS_C32_KPT;
};
template <>
struct ChunkConfig<uint32_t, NoValue, RANK_PEER_MASK> {  // + lane masks: fewer warps
  static constexpr int NT = 512, KPT = 20;
};
template <>
struct ChunkConfig<uint64_t, NoValue, RANK_ORDERED_ATOMIC> {
  static constexpr int NT = 512, KPT = HPCS_C64_KPT;
};
template <>
struct ChunkConfig<uint32_t, uint32_t, RANK_ORDERED_ATOMIC> {
  static constexpr int NT = 512, KPT = HPCS_CP32_KPT;
};
template <>
struct ChunkConfig<uint64_t, uint32_t, RANK_ORDERED_ATOMIC> {
  static constexpr int NT = 512, KPT = HPCS_CP64_KPT;
};
// peer-mask ranking: 32 KiB of lane masks on top, 48 KiB stages
template <>
struct ChunkConfig<uint64_t, NoValue, RANK_PEER_MASK> {
  static constexpr int NT = 512, KPT = 12;
};
template <>
struct ChunkConfig<uint32_t, uint32_t, RANK_PEER_MASK> {
  static constexpr int NT = 512, KPT = 12;
};
template <>
struct ChunkConfig<uint64_t, uint32_t, RANK_PEER_MASK> {
  static constexpr int NT = 512, KPT = 8;
};
constexpr size_t MAX_DYN_SMEM = 232448;  // 227 KiB per CTA on sm_100

// Automatic scheme: below these sizes the look-back passes were measured faster on B200 (the
// chunked passes' per-range count tables cost about J^2 x 256 global adds per pass, which
// small sorts do not amortise).  u32 keys: equal at 32 Mi, chunked 2% ahead at 64 Mi;
// u64 keys and u32 pairs: chunked ahead from 8 Mi; u64 + u32 pairs: from 4 Mi.
template <class U, class V>
struct ChunkMinKeys;
template <>
struct ChunkMinKeys<uint32_t, NoValue> {
  static constexpr int64_t value = int64_t(48) << 20;
};
template <>
struct ChunkMinKeys<uint64_t, NoValue> {
  static constexpr int64_t value = int64_t(6) << 20;
};
template <>
struct ChunkMinKeys<uint32_t, uint32_t> {
  static constexpr int64_t value = int64_t(6) << 20;
};
template <>
struct ChunkMinKeys<uint64_t, uint32_t> {
  static constexpr int64_t value = int64_t(3) << 20;
};

template <class U, class V, int MODE>
struct ChunkShape {
  using C = ChunkConfig<U, V, MODE>;
  using L = ChunkSmem<U, V, C::NT, C::KPT, MODE>;
  static constexpr int TILE = L::TILE;
  static constexpr int MAX_RANGES = 2 * int((MAX_DYN_SMEM - L::BASE_BYTES) / (RADIX * 4));
};

constexpr int HIST_NT = 1024;

// Launches K1 (one CTA per SM, 128 KiB of lane-private counters).
template <class U, int KIND>
int launch_histogram(hpcs_ctx* ctx, const U* keys, int64_t n, uint32_t* hist_out, const SortArgs& args,
                     int make_plan, cudaStream_t s);

template <class Kernel>
int occupancy_blocks(Kernel k, int nt, size_t smem) {
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, nt, smem) != cudaSuccess) return 1;
  return blocks > 0 ? blocks : 1;
}

template <class U, int KIND>
int launch_histogram(hpcs_ctx* ctx, const U* keys, int64_t n, uint32_t* hist_out, const SortArgs& args,
                     int make_plan, cudaStream_t s) {
  auto k = hist_all_digits_kernel<U, KIND, HIST_NT>;
  static int attr_set[64] = {0};
  if (!attr_set[ctx->device & 63]) {
    HPCS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(HistSmem<U>::BYTES)));
    attr_set[ctx->device & 63] = 1;
  }
  const int64_t vec = n * int64_t(sizeof(U)) / 16;
  const int64_t want = (vec + HIST_NT * 4 - 1) / (HIST_NT * 4);
  int grid = int(want < 1 ? 1 : (want > ctx->sms ? ctx->sms : want));
  if (args.chunk_hist) grid = args.chunks;  // CTA j counts key range j
  k<<<grid, HIST_NT, HistSmem<U>::BYTES, s>>>(keys, n, hist_out, args, make_plan);
  HPCS_CUDA(cudaGetLastError());
  return HPCS_OK;
}

// Onesweep launches for every digit pass, with the context's ranking mode.  Persistent
// grid of as many CL-CTA clusters as fit on the GPU at once.
template <class U, int KIND, class V, int MODE>
int launch_onesweep_passes(hpcs_ctx* ctx, SortArgs args, cudaStream_t s) {
  using C = SortConfig<U, V, MODE>;
  using L = OnesweepSmem<U, V, C::NT, C::KPT, C::STAGES, MODE>;
  constexpr int P = int(sizeof(U));
  auto k = onesweep_pass_kernel<U, KIND, V, C::NT, C::KPT, C::STAGES, C::MINB, MODE, C::CL>;
  static int clusters_by_dev[64] = {0};
  int& clusters = clusters_by_dev[ctx->device & 63];
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C::CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(C::NT, 1, 1);
  cfg.dynamicSmemBytes = L::BYTES;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (!clusters) {
    HPCS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::BYTES)));
    if (C::CL > 1) HPCS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 0));
    cfg.gridDim = dim3(C::CL * ctx->sms, 1, 1);
    int mc = 0;
    HPCS_CUDA(cudaOccupancyMaxActiveClusters(&mc, k, &cfg));
    clusters = mc > 0 ? mc : 1;
  }
  const int64_t units = args.num_tiles;
  const int grid_clusters = int(units < clusters ? units : clusters);
  cfg.gridDim = dim3(grid_clusters * C::CL, 1, 1);
  for (int p = 0; p < P; p++) {
    args.pass = p;
    KernelTimer kt(ctx, s, HPCS_K_LOOKBACK);
    HPCS_CUDA(cudaLaunchKernelEx(&cfg, k, args));
  }
  return HPCS_OK;
}

// Chunked digit passes: one CTA per key range, one launch per digit.
template <class U, int KIND, class V, int MODE>
int launch_chunk_passes(hpcs_ctx* ctx, SortArgs args, cudaStream_t s) {
  using C = ChunkConfig<U, V, MODE>;
  using L = ChunkSmem<U, V, C::NT, C::KPT, MODE>;
  constexpr int P = int(sizeof(U));
  auto k = chunk_pass_kernel<U, KIND, V, C::NT, C::KPT, MODE>;
  static int attr_set[64] = {0};
  if (!attr_set[ctx->device & 63]) {
    HPCS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(MAX_DYN_SMEM)));
    attr_set[ctx->device & 63] = 1;
  }
  const size_t bytes = L::bytes(args.chunks);
  for (int p = 0; p < P; p++) {
    args.pass = p;
    KernelTimer kt(ctx, s, HPCS_K_ONESWEEP);
    k<<<args.chunks, C::NT, bytes, s>>>(args);
    HPCS_CUDA(cudaGetLastError());
  }
  return HPCS_OK;
}

// Key ranges of the chunked passes: as many as there are SMs (capped by the counters'
// shared memory), each a whole number of tiles.
struct ChunkGeometry {
  int chunks;
  uint32_t chunk_keys;
  uint32_t magic;
};
inline ChunkGeometry chunk_geometry(int64_t n, int tile, int max_ranges) {
  const int64_t tiles = (n + tile - 1) / tile;
  const int64_t per = (tiles + max_ranges - 1) / max_ranges;  // tiles per range
  ChunkGeometry g;
  g.chunks = int((tiles + per - 1) / per);
  g.chunk_keys = uint32_t(per * tile);
  g.magic = uint32_t(((uint64_t(1) << 32) + g.chunk_keys - 1) / g.chunk_keys);
  return g;
}

// Enqueue a full LSD sort of n keys (and optional 4-byte items) in device memory.
// A sort of at most SMALL_MAX_KEYS keys (and items) in one cooperative launch (small_sort.cuh),
// with the context's ranking mode; scratch: B, the per-CTA digit totals and the barrier words.
template <class U, int KIND, class V>
int enqueue_small_sort(hpcs_ctx* ctx, U* keys, uint32_t* vals, int64_t n, cudaStream_t s) {
  constexpr bool PAIRS = !std::is_same<V, NoValue>::value;
  const int G = int((n + SMALL_TILE - 1) / SMALL_TILE);
  int rc;
  if ((rc = ensure(ctx, ctx->keys_b, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  if (PAIRS && (rc = ensure(ctx, ctx->vals_b, size_t(n) * 4)) != HPCS_OK) return rc;
  uint32_t* vb = PAIRS ? static_cast<uint32_t*>(ctx->vals_b.ptr) : nullptr;
  if ((rc = ensure(ctx, ctx->status0, (size_t(G) * RADIX + 2) * 4)) != HPCS_OK) return rc;
  U* b = static_cast<U*>(ctx->keys_b.ptr);
  uint32_t* counts = static_cast<uint32_t*>(ctx->status0.ptr);
  uint32_t* bar = counts + size_t(G) * RADIX;
  uint32_t* err = device_error_word(ctx);
  int n32 = int(n);
  uint64_t spin = uint64_t(ctx->cfg.spin_limit_ns);
  HPCS_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(uint32_t), s));
  void* args[] = {&keys, &b, &vals, &vb, &n32, &counts, &bar, &err, &spin};
  const void* k = ctx->rank_mode == RANK_ORDERED_ATOMIC
                      ? reinterpret_cast<const void*>(small_sort_kernel<U, KIND, V, RANK_ORDERED_ATOMIC>)
                      : reinterpret_cast<const void*>(small_sort_kernel<U, KIND, V, RANK_PEER_MASK>);
  KernelTimer kt(ctx, s, HPCS_K_LOOKBACK);
  HPCS_CUDA(cudaLaunchCooperativeKernel(k, dim3(G), dim3(SMALL_NT), args, 0, s));
  return HPCS_OK;
}

// keys/vals are sorted in place (with scratch B owned by the context).
template <class U, int KIND, class V>
int enqueue_sort(hpcs_ctx* ctx, U* keys, uint32_t* vals, int64_t n, cudaStream_t s) {
  using CA = SortConfig<U, V, RANK_ORDERED_ATOMIC>;
  using CP = SortConfig<U, V, RANK_PEER_MASK>;
  constexpr bool PAIRS = !std::is_same<V, NoValue>::value;
  if (n <= 1) return HPCS_OK;
  if (n > MAX_KEYS_PER_SORT) return fail(HPCS_ERR_RANGE, "n exceeds HPCS_MAX_KEYS");
  // small sorts: one cooperative launch (not inside a stream capture, and not when a pass
  // scheme is forced)
  if (n <= SMALL_MAX_KEYS && ctx->cfg.pass_scheme == HPCS_PASSES_AUTO) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    HPCS_CUDA(cudaStreamIsCapturing(s, &cap));
    if (cap == cudaStreamCaptureStatusNone) return enqueue_small_sort<U, KIND, V>(ctx, keys, vals, n, s);
  }
  if (ctx->cfg.pass_scheme == HPCS_PASSES_LOOKBACK && n > MAX_KEYS_LOOKBACK)
    return fail(HPCS_ERR_RANGE, "look-back passes take at most 2^30 - 1 keys (30-bit prefixes)");
  const bool lookback = ctx->cfg.pass_scheme == HPCS_PASSES_LOOKBACK ||
                        (ctx->cfg.pass_scheme != HPCS_PASSES_CHUNKED && n < ChunkMinKeys<U, V>::value);
  // 4-byte float keys without items, AUTO scheme, large sorts: K1 picks the scheme from the
  // digit counts (normally distributed floats sort faster with the look-back passes, floats
  // with a dominant exponent with the chunked ones).  Not on borrowed (serving) scratch.
  const bool choose = !lookback && ctx->cfg.pass_scheme == HPCS_PASSES_AUTO && KIND == KIND_FLOAT &&
                      sizeof(U) == 4 && !PAIRS && n <= MAX_KEYS_LOOKBACK && !ctx->status1.borrowed;
  const bool ordered = ctx->rank_mode == RANK_ORDERED_ATOMIC;
  const int64_t unit = ordered ? int64_t(CA::NT) * CA::KPT * CA::CL : int64_t(CP::NT) * CP::KPT * CP::CL;
  const int64_t num_tiles = lookback || choose ? (n + unit - 1) / unit : 0;  // look-back units
  ChunkGeometry geo{0, 0, 0};
  if (!lookback) {
    using SA = ChunkShape<U, V, RANK_ORDERED_ATOMIC>;
    using SP = ChunkShape<U, V, RANK_PEER_MASK>;
    const int cap = ordered ? SA::MAX_RANGES : SP::MAX_RANGES;
    geo = chunk_geometry(n, ordered ? SA::TILE : SP::TILE, ctx->sms < cap ? ctx->sms : cap);
  }

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
  constexpr int P = int(sizeof(U));
  const size_t status_bytes = lookback ? size_t(num_tiles) * RADIX * 4 : size_t(geo.chunks) * (P + 3) * RADIX * 4;
  if ((rc = ensure(ctx, ctx->status0, status_bytes)) != HPCS_OK) return rc;
  if (lookback && (rc = ensure(ctx, ctx->status1, status_bytes)) != HPCS_OK) return rc;
  const size_t lb_bytes = size_t(num_tiles) * RADIX * 4;  // one look-back buffer (choose)
  if (choose && (rc = ensure(ctx, ctx->status1, lb_bytes)) != HPCS_OK) return rc;
  if (choose && (rc = ensure(ctx, ctx->status2, lb_bytes)) != HPCS_OK) return rc;
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
  args.trace = ctx->trace;
  args.trace_pass = ctx->trace_pass;
  args.trace_capacity = ctx->trace_capacity;
  if (!lookback) {
    // status0 holds [chunks][P][256] per-range input counts, then [3][chunks][256] tables
    args.chunk_hist = static_cast<uint32_t*>(ctx->status0.ptr);
    args.ctab = args.chunk_hist + size_t(geo.chunks) * P * RADIX;
    args.chunks = geo.chunks;
    args.chunk_keys = geo.chunk_keys;
    args.chunk_magic = geo.magic;
  }
  if (choose) {
    // the look-back passes' buffers are status1 and status2; K1 (chunked mode) does not
    // zero the first one, so it is cleared here
    args.choose_lookback = 1;
    args.status[0] = static_cast<uint32_t*>(ctx->status1.ptr);
    args.status[1] = static_cast<uint32_t*>(ctx->status2.ptr);
    HPCS_CUDA(cudaMemsetAsync(args.status[0], 0, lb_bytes, s));
  }

  HPCS_CUDA(cudaMemsetAsync(args.plan, 0, sizeof(SortPlan), s));

  // K1: fused histogram + plan
  {
    KernelTimer kt(ctx, s, HPCS_K_HISTOGRAM);
    if ((rc = launch_histogram<U, KIND>(ctx, a, n, &args.plan->hist[0][0], args, 1, s)) != HPCS_OK) return rc;
  }
  // K3: one launch per digit (with `choose`, both kinds; the ones K1 did not choose return)
  if (!lookback)
    rc = ordered ? launch_chunk_passes<U, KIND, V, RANK_ORDERED_ATOMIC>(ctx, args, s)
                 : launch_chunk_passes<U, KIND, V, RANK_PEER_MASK>(ctx, args, s);
  if (rc == HPCS_OK && (lookback || choose))
    rc = ordered ? launch_onesweep_passes<U, KIND, V, RANK_ORDERED_ATOMIC>(ctx, args, s)
                 : launch_onesweep_passes<U, KIND, V, RANK_PEER_MASK>(ctx, args, s);
  if (rc != HPCS_OK) return rc;
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
