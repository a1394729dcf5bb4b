// Host side of the batched segmented sort (C ABI in include/hpcs_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/hpcs_gpu.h"
#include "seg_grid.cuh"
#include "segmented_host.cuh"

struct hpcs_segplan {
  hpcs_ctx* ctx = nullptr;
  int64_t nsegs = 0;
  hpcs::SegDesc* d_desc = nullptr;
  uint32_t* d_queue = nullptr;
  void* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  void* d_grid = nullptr;  // grid-level path: per-array sort arguments and the CTA map
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t capture_stream = nullptr;
};

namespace hpcs {
namespace {


int key_bytes(int dtype) { return dtype >= HPCS_U64 ? 8 : 4; }

int validate(const hpcs_segment* segs, int64_t nsegs) {
  if (!segs && nsegs > 0) return fail(HPCS_ERR_NULL, "segments is NULL");
  if (nsegs < 0 || nsegs > (int64_t(1) << 31) - 1) return fail(HPCS_ERR_RANGE, "segment count out of range");
  for (int64_t i = 0; i < nsegs; i++) {
    if (segs[i].n < 0 || segs[i].n > HPCS_MAX_SEGMENT_KEYS) return fail(HPCS_ERR_RANGE, "segment length out of range");
    if (segs[i].n > 0 && !segs[i].keys) return fail(HPCS_ERR_NULL, "segment keys is NULL");
    if (segs[i].dtype < HPCS_U32 || segs[i].dtype > HPCS_F64) return fail(HPCS_ERR_UNSUPPORTED, "unknown dtype");
  }
  return HPCS_OK;
}

struct DeviceGuard2 {
  int prev = -1;
  explicit DeviceGuard2(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard2() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

int ensure_seg_streams(hpcs_ctx* ctx) {
  if (ctx->seg_fork) return HPCS_OK;
  HPCS_CUDA(cudaStreamCreateWithFlags(&ctx->seg_grid_stream, cudaStreamNonBlocking));
  HPCS_CUDA(cudaEventCreateWithFlags(&ctx->seg_grid_fork, cudaEventDisableTiming));
  HPCS_CUDA(cudaEventCreateWithFlags(&ctx->seg_grid_join, cudaEventDisableTiming));
  for (int b = 0; b < hpcs_ctx::SEG_BRANCHES; b++) {
    HPCS_CUDA(cudaStreamCreateWithFlags(&ctx->seg_streams[b], cudaStreamNonBlocking));
    HPCS_CUDA(cudaEventCreateWithFlags(&ctx->seg_join[b], cudaEventDisableTiming));
  }
  HPCS_CUDA(cudaEventCreateWithFlags(&ctx->seg_fork, cudaEventDisableTiming));
  return HPCS_OK;
}

}  // namespace

int seg_build_groups(const hpcs_seg_tuning& tuning, const hpcs_segment* segs, int64_t nsegs,
                     std::vector<SegDesc>& table, std::vector<SegGroup>& groups, size_t& scratch) {
  int rc = validate(segs, nsegs);
  if (rc != HPCS_OK) return rc;
  // group id = 2 x variant + (tiled path)
  constexpr int NG = 2 * SEG_NVARIANTS;
  std::vector<int> var(static_cast<size_t>(nsegs));
  std::vector<double> group_bytes(NG, 0.0);
  for (int64_t i = 0; i < nsegs; i++) {
    const int w = key_bytes(segs[i].dtype);
    const int v = tuning.variant[w == 8 ? 1 : 0][seg_class_of(segs[i].n)];
    var[i] = 2 * v + (seg_variant_large(v, segs[i].n, w) ? 1 : 0);
    group_bytes[var[i]] += double(segs[i].n) * w;
  }
  // groups in decreasing total bytes (the heaviest is launched first, on the caller's
  // stream), arrays within a group largest first
  std::vector<int> vorder(NG);
  std::iota(vorder.begin(), vorder.end(), 0);
  std::stable_sort(vorder.begin(), vorder.end(), [&](int a, int b) { return group_bytes[a] > group_bytes[b]; });
  std::vector<int> vrank(NG);
  for (int r = 0; r < NG; r++) vrank[vorder[r]] = r;
  std::vector<int64_t> order(static_cast<size_t>(nsegs));
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    if (vrank[var[a]] != vrank[var[b]]) return vrank[var[a]] < vrank[var[b]];
    return segs[a].n * key_bytes(segs[a].dtype) > segs[b].n * key_bytes(segs[b].dtype);
  });
  table.resize(size_t(nsegs));
  groups.clear();
  scratch = 0;
  for (int64_t j = 0; j < nsegs; j++) {
    const hpcs_segment& sg = segs[order[j]];
    const int gid = var[order[j]];
    const int v = gid / 2;
    const bool large = (gid & 1) != 0;
    if (groups.empty() || 2 * groups.back().variant + (groups.back().large ? 1 : 0) != gid)
      groups.push_back({v, large, int(j), 0});
    groups.back().count++;
    SegDesc& d = table[j];
    d.keys = sg.keys;
    d.n = sg.n;
    d.dtype = sg.dtype;
    d.pad = 0;
    d.scratch = nullptr;
    const int w = key_bytes(sg.dtype);
    if (large) {
      d.scratch = reinterpret_cast<void*>(scratch + 1);  // offset + 1 for now (0 = none)
      scratch += (size_t(sg.n) * w + 255) / 256 * 256;
    }
  }
  return HPCS_OK;
}

void seg_relocate(std::vector<SegDesc>& table, const std::vector<SegGroup>&, void* base) {
  for (auto& d : table)
    if (d.scratch) d.scratch = static_cast<unsigned char*>(base) + (reinterpret_cast<size_t>(d.scratch) - 1);
}

namespace {
template <int MODE>
int launch_groups_mode(hpcs_ctx* ctx, const SegDesc* d_desc, const std::vector<SegGroup>& groups,
                       uint32_t* d_queues, cudaStream_t s) {
  int rc;
  const int ng = int(groups.size());
  if (ng > 1) {
    if ((rc = ensure_seg_streams(ctx)) != HPCS_OK) return rc;
    HPCS_CUDA(cudaEventRecord(ctx->seg_fork, s));
    for (int b = 0; b < hpcs_ctx::SEG_BRANCHES && b < ng - 1; b++)
      HPCS_CUDA(cudaStreamWaitEvent(ctx->seg_streams[b], ctx->seg_fork, 0));
  }
  for (int g = 0; g < ng; g++) {
    cudaStream_t st = g == 0 ? s : ctx->seg_streams[(g - 1) % hpcs_ctx::SEG_BRANCHES];
    if ((rc = launch_seg_variant<MODE>(ctx, groups[g].variant, groups[g].large, d_desc + groups[g].first,
                                       groups[g].count, d_queues + g, st)) != HPCS_OK)
      return rc;
  }
  for (int b = 0; b < hpcs_ctx::SEG_BRANCHES && b < ng - 1; b++) {
    HPCS_CUDA(cudaEventRecord(ctx->seg_join[b], ctx->seg_streams[b]));
    HPCS_CUDA(cudaStreamWaitEvent(s, ctx->seg_join[b], 0));
  }
  return HPCS_OK;
}
}  // namespace

int seg_launch_groups(hpcs_ctx* ctx, const SegDesc* d_desc, const std::vector<SegGroup>& groups,
                      uint32_t* d_queues, cudaStream_t s) {
  if (groups.empty()) return HPCS_OK;
  HPCS_CUDA(cudaMemsetAsync(d_queues, 0, groups.size() * 4, s));
  return ctx->rank_mode == RANK_ORDERED_ATOMIC ? launch_groups_mode<RANK_ORDERED_ATOMIC>(ctx, d_desc, groups, d_queues, s)
                                               : launch_groups_mode<RANK_PEER_MASK>(ctx, d_desc, groups, d_queues, s);
}

// ---- grid-level path (seg_grid.cuh) -------------------------------------------------------
namespace {
int dtype_bytes(int dtype) { return dtype >= HPCS_U64 ? 8 : 4; }

template <class U, int MODE>
void grid_geometry(int64_t n, int tiles_per_range, ChunkGeometry& g) {
  using S = ChunkShape<U, NoValue, MODE>;
  const int64_t tiles = (n + S::TILE - 1) / S::TILE;
  int64_t want = (tiles + tiles_per_range - 1) / tiles_per_range;
  if (want > S::MAX_RANGES) want = S::MAX_RANGES;
  if (want < 1) want = 1;
  g = chunk_geometry(n, S::TILE, int(want));
}

template <class U, int KIND, int MODE>
int grid_launch_set(hpcs_ctx* ctx, const SegGridSet& set, const SortArgs* d_args, const int2* d_map,
                    cudaStream_t s) {
  using C = ChunkConfig<U, NoValue, MODE>;
  using L = ChunkSmem<U, NoValue, C::NT, C::KPT, MODE>;
  constexpr int P = int(sizeof(U));
  const SortArgs* a = d_args + set.first;
  const int2* m = d_map + set.map_first;
  seg_hist_all_digits_kernel<U, KIND, HIST_NT><<<set.ctas, HIST_NT, HistSmem<U>::BYTES, s>>>(a, m);
  HPCS_CUDA(cudaGetLastError());
  for (int p = 0; p < P; p++) {
    seg_chunk_pass_kernel<U, KIND, NoValue, C::NT, C::KPT, MODE><<<set.ctas, C::NT, L::bytes(set.max_ranges), s>>>(a, m, p);
    HPCS_CUDA(cudaGetLastError());
  }
  seg_finalize_kernel<U><<<set.ctas, 256, 0, s>>>(a, m, device_error_word(ctx));
  HPCS_CUDA(cudaGetLastError());
  return HPCS_OK;
}

template <class U, int KIND, int MODE>
int grid_setup_type(hpcs_ctx* ctx) {
  using C = ChunkConfig<U, NoValue, MODE>;
  static int done[64] = {0};
  if (done[ctx->device & 63]) return HPCS_OK;
  HPCS_CUDA(cudaFuncSetAttribute(seg_hist_all_digits_kernel<U, KIND, HIST_NT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(HistSmem<U>::BYTES)));
  HPCS_CUDA(cudaFuncSetAttribute(seg_chunk_pass_kernel<U, KIND, NoValue, C::NT, C::KPT, MODE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(MAX_DYN_SMEM)));
  done[ctx->device & 63] = 1;
  return HPCS_OK;
}

template <int MODE>
int grid_dispatch(hpcs_ctx* ctx, const SegGridSet* set, const SortArgs* d_args, const int2* d_map, cudaStream_t s) {
  const bool setup = set == nullptr;
  for (int dt = HPCS_U32; dt <= HPCS_F64; dt++) {
    if (!setup && set->dtype != dt) continue;
    int rc = HPCS_OK;
    switch (dt) {
      case HPCS_U32: rc = setup ? grid_setup_type<uint32_t, KIND_UNSIGNED, MODE>(ctx) : grid_launch_set<uint32_t, KIND_UNSIGNED, MODE>(ctx, *set, d_args, d_map, s); break;
      case HPCS_I32: rc = setup ? grid_setup_type<uint32_t, KIND_SIGNED, MODE>(ctx) : grid_launch_set<uint32_t, KIND_SIGNED, MODE>(ctx, *set, d_args, d_map, s); break;
      case HPCS_F32: rc = setup ? grid_setup_type<uint32_t, KIND_FLOAT, MODE>(ctx) : grid_launch_set<uint32_t, KIND_FLOAT, MODE>(ctx, *set, d_args, d_map, s); break;
      case HPCS_U64: rc = setup ? grid_setup_type<uint64_t, KIND_UNSIGNED, MODE>(ctx) : grid_launch_set<uint64_t, KIND_UNSIGNED, MODE>(ctx, *set, d_args, d_map, s); break;
      case HPCS_I64: rc = setup ? grid_setup_type<uint64_t, KIND_SIGNED, MODE>(ctx) : grid_launch_set<uint64_t, KIND_SIGNED, MODE>(ctx, *set, d_args, d_map, s); break;
      default: rc = setup ? grid_setup_type<uint64_t, KIND_FLOAT, MODE>(ctx) : grid_launch_set<uint64_t, KIND_FLOAT, MODE>(ctx, *set, d_args, d_map, s); break;
    }
    if (rc != HPCS_OK) return rc;
  }
  return HPCS_OK;
}
}  // namespace

int seg_grid_build(const hpcs_segment* segs, const std::vector<int64_t>& idx, int mode, int skip_trivial,
                   uint64_t spin_limit_ns, int tiles_per_range, SegGrid& grid) {
  grid = SegGrid();
  grid.mode = mode;
  auto align = [](size_t x) { return (x + 255) / 256 * 256; };
  for (int dt = HPCS_U32; dt <= HPCS_F64; dt++) {
    std::vector<int64_t> mine;
    for (int64_t i : idx)
      if (segs[i].dtype == dt) mine.push_back(i);
    if (mine.empty()) continue;
    SegGridSet set;
    set.dtype = dt;
    set.first = int(grid.args.size());
    set.count = int(mine.size());
    set.map_first = int(grid.map.size());
    set.plan_off = grid.scratch;
    set.plan_bytes = align(mine.size() * sizeof(SortPlan));
    grid.scratch += set.plan_bytes;
    const int w = dtype_bytes(dt);
    const int P = w;
    for (size_t q = 0; q < mine.size(); q++) {
      const hpcs_segment& sg = segs[mine[q]];
      ChunkGeometry g;
      if (w == 4) {
        if (mode == RANK_ORDERED_ATOMIC) grid_geometry<uint32_t, RANK_ORDERED_ATOMIC>(sg.n, tiles_per_range, g);
        else grid_geometry<uint32_t, RANK_PEER_MASK>(sg.n, tiles_per_range, g);
      } else {
        if (mode == RANK_ORDERED_ATOMIC) grid_geometry<uint64_t, RANK_ORDERED_ATOMIC>(sg.n, tiles_per_range, g);
        else grid_geometry<uint64_t, RANK_PEER_MASK>(sg.n, tiles_per_range, g);
      }
      SortArgs a{};
      a.keys_a = sg.keys;
      a.n = sg.n;
      // scratch offsets (+1, so 0 stays "none") until relocation
      a.keys_b = reinterpret_cast<void*>(grid.scratch + 1);
      grid.scratch += align(size_t(sg.n) * w);
      a.chunk_hist = reinterpret_cast<uint32_t*>(grid.scratch + 1);
      grid.scratch += align(size_t(g.chunks) * (P + 3) * RADIX * 4);
      a.plan = reinterpret_cast<SortPlan*>(set.plan_off + q * sizeof(SortPlan) + 1);
      a.chunks = g.chunks;
      a.chunk_keys = g.chunk_keys;
      a.chunk_magic = g.magic;
      a.skip_trivial = skip_trivial;
      a.poison_tile = -1;
      a.spin_limit_ns = spin_limit_ns;
      a.trace_pass = -1;
      grid.args.push_back(a);
      for (int r = 0; r < g.chunks; r++) grid.map.push_back(make_int2(int(q), r));
      if (g.chunks > set.max_ranges) set.max_ranges = g.chunks;
    }
    set.ctas = int(grid.map.size()) - set.map_first;
    grid.sets.push_back(set);
  }
  return HPCS_OK;
}

void seg_grid_relocate(SegGrid& grid, void* base) {
  unsigned char* b = static_cast<unsigned char*>(base);
  auto fix = [&](auto* p) { return reinterpret_cast<decltype(p)>(b + (reinterpret_cast<size_t>(p) - 1)); };
  for (auto& a : grid.args) {
    a.keys_b = fix(static_cast<unsigned char*>(a.keys_b));
    a.chunk_hist = fix(a.chunk_hist);
    a.plan = fix(a.plan);
  }
  // the next-digit tables follow each array's per-range counts
  for (const auto& set : grid.sets) {
    const int P = dtype_bytes(set.dtype);
    for (int q = 0; q < set.count; q++) {
      SortArgs& a = grid.args[size_t(set.first + q)];
      a.ctab = a.chunk_hist + size_t(a.chunks) * P * RADIX;
    }
  }
}

int seg_grid_setup(hpcs_ctx* ctx, const SegGrid& grid) {
  if (grid.sets.empty()) return HPCS_OK;
  return grid.mode == RANK_ORDERED_ATOMIC ? grid_dispatch<RANK_ORDERED_ATOMIC>(ctx, nullptr, nullptr, nullptr, nullptr)
                                          : grid_dispatch<RANK_PEER_MASK>(ctx, nullptr, nullptr, nullptr, nullptr);
}

int seg_grid_launch(hpcs_ctx* ctx, const SegGrid& grid, const SortArgs* d_args, const int2* d_map, cudaStream_t s) {
  for (const auto& set : grid.sets) {
    const SortPlan* plan0 = grid.args[size_t(set.first)].plan;
    HPCS_CUDA(cudaMemsetAsync(const_cast<SortPlan*>(plan0), 0, set.plan_bytes, s));
    const int rc = grid.mode == RANK_ORDERED_ATOMIC ? grid_dispatch<RANK_ORDERED_ATOMIC>(ctx, &set, d_args, d_map, s)
                                                    : grid_dispatch<RANK_PEER_MASK>(ctx, &set, d_args, d_map, s);
    if (rc != HPCS_OK) return rc;
  }
  return HPCS_OK;
}

namespace {
// Splits a batch into the grid-level arrays (their indices) and the others (copied out).
void seg_split(const hpcs_segment* segs, int64_t nsegs, int64_t min_keys, std::vector<hpcs_segment>& rest,
               std::vector<int64_t>& grid_idx) {
  rest.clear();
  grid_idx.clear();
  for (int64_t i = 0; i < nsegs; i++) {
    if (seg_grid_eligible(segs[i], min_keys)) grid_idx.push_back(i);
    else rest.push_back(segs[i]);
  }
}

// The whole batch on stream s: the grid-level sets on their own branch, the other arrays' groups
// as before (the heaviest on s, the others on the helper streams).
int seg_launch_all(hpcs_ctx* ctx, const SegDesc* d_desc, const std::vector<SegGroup>& groups, uint32_t* d_queues,
                   const SegGrid& grid, const SortArgs* d_args, const int2* d_map, cudaStream_t s) {
  int rc;
  const bool branch = !grid.sets.empty();
  if (branch) {
    if ((rc = ensure_seg_streams(ctx)) != HPCS_OK) return rc;
    HPCS_CUDA(cudaEventRecord(ctx->seg_grid_fork, s));
    HPCS_CUDA(cudaStreamWaitEvent(ctx->seg_grid_stream, ctx->seg_grid_fork, 0));
    if ((rc = seg_grid_launch(ctx, grid, d_args, d_map, ctx->seg_grid_stream)) != HPCS_OK) return rc;
  }
  if ((rc = seg_launch_groups(ctx, d_desc, groups, d_queues, s)) != HPCS_OK) return rc;
  if (branch) {
    HPCS_CUDA(cudaEventRecord(ctx->seg_grid_join, ctx->seg_grid_stream));
    HPCS_CUDA(cudaStreamWaitEvent(s, ctx->seg_grid_join, 0));
  }
  return HPCS_OK;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }
}  // namespace

}  // namespace hpcs

using namespace hpcs;

extern "C" {

int hpcs_sort_segmented_dev(hpcs_ctx* ctx, const hpcs_segment* segs, int64_t nsegs, void* stream) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  int rc = validate(segs, nsegs);
  if (rc != HPCS_OK || nsegs == 0) return rc;
  std::vector<hpcs_segment> rest;
  std::vector<int64_t> grid_idx;
  seg_split(segs, nsegs, seg_grid_min_keys(ctx->cfg), rest, grid_idx);
  std::vector<SegDesc> table;
  std::vector<SegGroup> groups;
  size_t scratch = 0;
  if ((rc = seg_build_groups(ctx->seg_tuning, rest.data(), int64_t(rest.size()), table, groups, scratch)) != HPCS_OK)
    return rc;
  SegGrid grid;
  if ((rc = seg_grid_build(segs, grid_idx, ctx->rank_mode, ctx->cfg.skip_trivial_passes,
                           uint64_t(ctx->cfg.spin_limit_ns), seg_grid_tiles(ctx->cfg), grid)) != HPCS_OK)
    return rc;
  DeviceGuard2 g(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  if ((rc = seg_grid_setup(ctx, grid)) != HPCS_OK) return rc;
  const size_t block_scratch = align256(scratch);
  const size_t desc_bytes = table.size() * sizeof(SegDesc);
  const size_t args_bytes = align256(grid.args.size() * sizeof(SortArgs));
  const size_t map_bytes = grid.map.size() * sizeof(int2);
  if ((rc = ensure(ctx, ctx->aux0, block_scratch + grid.scratch + 256)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->aux1, desc_bytes + 256 + groups.size() * 4)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->aux2, args_bytes + map_bytes + 256)) != HPCS_OK) return rc;
  seg_relocate(table, groups, ctx->aux0.ptr);
  seg_grid_relocate(grid, static_cast<unsigned char*>(ctx->aux0.ptr) + block_scratch);
  SegDesc* d_desc = static_cast<SegDesc*>(ctx->aux1.ptr);
  uint32_t* d_queues = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(ctx->aux1.ptr) + (desc_bytes + 255) / 256 * 256);
  SortArgs* d_args = static_cast<SortArgs*>(ctx->aux2.ptr);
  int2* d_map = reinterpret_cast<int2*>(static_cast<unsigned char*>(ctx->aux2.ptr) + args_bytes);
  // the host tables must outlive the copies: copy synchronously with respect to this stream
  if (desc_bytes) HPCS_CUDA(cudaMemcpyAsync(d_desc, table.data(), desc_bytes, cudaMemcpyHostToDevice, s));
  if (!grid.args.empty()) {
    HPCS_CUDA(cudaMemcpyAsync(d_args, grid.args.data(), grid.args.size() * sizeof(SortArgs), cudaMemcpyHostToDevice, s));
    HPCS_CUDA(cudaMemcpyAsync(d_map, grid.map.data(), map_bytes, cudaMemcpyHostToDevice, s));
  }
  HPCS_CUDA(cudaStreamSynchronize(s));
  KernelTimer kt(ctx, s, HPCS_K_SEGMENTED);
  return seg_launch_all(ctx, d_desc, groups, d_queues, grid, d_args, d_map, s);
}

int hpcs_segplan_create(hpcs_ctx* ctx, const hpcs_segment* segs, int64_t nsegs, hpcs_segplan** out) {
  if (!ctx || !out) return fail(HPCS_ERR_NULL, "ctx or out is NULL");
  *out = nullptr;
  int rc = validate(segs, nsegs);
  if (rc != HPCS_OK) return rc;
  std::vector<hpcs_segment> rest;
  std::vector<int64_t> grid_idx;
  seg_split(segs, nsegs, seg_grid_min_keys(ctx->cfg), rest, grid_idx);
  std::vector<SegDesc> table;
  std::vector<SegGroup> groups;
  size_t scratch = 0;
  if ((rc = seg_build_groups(ctx->seg_tuning, rest.data(), int64_t(rest.size()), table, groups, scratch)) != HPCS_OK)
    return rc;
  SegGrid grid;
  if ((rc = seg_grid_build(segs, grid_idx, ctx->rank_mode, ctx->cfg.skip_trivial_passes,
                           uint64_t(ctx->cfg.spin_limit_ns), seg_grid_tiles(ctx->cfg), grid)) != HPCS_OK)
    return rc;
  DeviceGuard2 g(ctx->device);
  auto* p = new hpcs_segplan();
  p->ctx = ctx;
  p->nsegs = nsegs;
  auto cleanup = [&](int code) {
    hpcs_segplan_destroy(p);
    return code;
  };
  const size_t desc_bytes = table.size() * sizeof(SegDesc);
  const size_t queue_off = (desc_bytes + 255) / 256 * 256;
  const size_t block_scratch = align256(scratch);
  const size_t args_bytes = align256(grid.args.size() * sizeof(SortArgs));
  const size_t map_bytes = grid.map.size() * sizeof(int2);
  cudaError_t e;
  if ((e = cudaMalloc(&p->d_desc, queue_off + 256 + groups.size() * 4)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaMalloc"));
  p->d_queue = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(p->d_desc) + queue_off);
  const size_t all_scratch = block_scratch + grid.scratch;
  if (all_scratch && (e = cudaMalloc(&p->d_scratch, all_scratch)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaMalloc"));
  p->scratch_bytes = all_scratch;
  seg_relocate(table, groups, p->d_scratch);
  SortArgs* d_args = nullptr;
  int2* d_map = nullptr;
  if (!grid.sets.empty()) {
    seg_grid_relocate(grid, static_cast<unsigned char*>(p->d_scratch) + block_scratch);
    if ((e = cudaMalloc(&p->d_grid, args_bytes + map_bytes)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc"));
    d_args = static_cast<SortArgs*>(p->d_grid);
    d_map = reinterpret_cast<int2*>(static_cast<unsigned char*>(p->d_grid) + args_bytes);
    if ((e = cudaMemcpy(d_args, grid.args.data(), grid.args.size() * sizeof(SortArgs), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(d_map, grid.map.data(), map_bytes, cudaMemcpyHostToDevice)) != cudaSuccess)
      return cleanup(cuda_fail(e, "cudaMemcpy"));
  }
  if (desc_bytes && (e = cudaMemcpy(p->d_desc, table.data(), desc_bytes, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaMemcpy"));
  if ((e = cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaStreamCreate"));
  // set the kernels' attributes and the helper streams up outside capture: launch every
  // group over zero arrays once
  {
    std::vector<SegGroup> warm = groups;
    for (auto& wg : warm) wg.count = 0;
    if ((rc = seg_launch_groups(ctx, p->d_desc, warm, p->d_queue, p->capture_stream)) != HPCS_OK) return cleanup(rc);
    if ((rc = seg_grid_setup(ctx, grid)) != HPCS_OK) return cleanup(rc);
    if (!grid.sets.empty() && (rc = ensure_seg_streams(ctx)) != HPCS_OK) return cleanup(rc);
    if ((e = cudaStreamSynchronize(p->capture_stream)) != cudaSuccess) return cleanup(cuda_fail(e, "sync"));
  }
  const bool was_profiling = ctx->profile;
  ctx->profile = false;  // no event records inside the graph
  if ((e = cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
    ctx->profile = was_profiling;
    return cleanup(cuda_fail(e, "cudaStreamBeginCapture"));
  }
  rc = seg_launch_all(ctx, p->d_desc, groups, p->d_queue, grid, d_args, d_map, p->capture_stream);
  e = cudaStreamEndCapture(p->capture_stream, &p->graph);
  ctx->profile = was_profiling;
  if (rc != HPCS_OK) return cleanup(rc);
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaStreamEndCapture"));
  if ((e = cudaGraphInstantiate(&p->exec, p->graph, 0)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaGraphInstantiate"));
  *out = p;
  return HPCS_OK;
}

int hpcs_segplan_execute(hpcs_segplan* p, void* stream) {
  if (!p) return fail(HPCS_ERR_NULL, "plan is NULL");
  DeviceGuard2 g(p->ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->ctx->stream;
  int rc = enter_stream(p->ctx, s);
  if (rc != HPCS_OK) return rc;
  KernelTimer kt(p->ctx, s, HPCS_K_SEGMENTED);
  HPCS_CUDA(cudaGraphLaunch(p->exec, s));
  return HPCS_OK;
}

int hpcs_segplan_destroy(hpcs_segplan* p) {
  if (!p) return HPCS_OK;
  DeviceGuard2 g(p->ctx->device);
  if (p->ctx->stream) cudaStreamSynchronize(p->ctx->stream);
  if (p->ctx->last_stream) cudaStreamSynchronize(p->ctx->last_stream);
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->capture_stream) cudaStreamDestroy(p->capture_stream);
  if (p->d_scratch) cudaFree(p->d_scratch);
  if (p->d_grid) cudaFree(p->d_grid);
  if (p->d_desc) cudaFree(p->d_desc);
  delete p;
  return HPCS_OK;
}

}  // extern "C"

extern "C" {

int hpcs_seg_variants(hpcs_seg_variant_info* out, int capacity) {
  for (int v = 0; v < SEG_NVARIANTS && out && v < capacity; v++) {
    out[v].kind = SEG_VARIANTS[v].kind;
    out[v].threads = SEG_VARIANTS[v].nt;
    out[v].keys_per_thread = SEG_VARIANTS[v].kpt;
    out[v].digit_bits = SEG_VARIANTS[v].rbits;
    out[v].max_keys[0] = seg_variant_max_keys(v, 4);
    out[v].max_keys[1] = seg_variant_max_keys(v, 8);
  }
  return SEG_NVARIANTS;
}

int64_t hpcs_seg_class_limit(int c) {
  if (c < 0 || c >= HPCS_SEG_CLASSES) return -2;
  return SEG_CLASS_LIMIT[c];
}

int hpcs_ctx_get_seg_tuning(hpcs_ctx* ctx, hpcs_seg_tuning* out) {
  if (!ctx || !out) return fail(HPCS_ERR_NULL, "ctx or out is NULL");
  *out = ctx->seg_tuning;
  return HPCS_OK;
}

int hpcs_ctx_set_seg_tuning(hpcs_ctx* ctx, const hpcs_seg_tuning* t) {
  if (!ctx || !t) return fail(HPCS_ERR_NULL, "ctx or tuning is NULL");
  for (int w = 0; w < 2; w++)
    for (int c = 0; c < HPCS_SEG_CLASSES; c++)
      if (!seg_variant_fits(t->variant[w][c], w, c))
        return fail(HPCS_ERR_RANGE, "segmented-sort variant unknown or too small for its length class");
  ctx->seg_tuning = *t;
  return HPCS_OK;
}

}  // extern "C"
