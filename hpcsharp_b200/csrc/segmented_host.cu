// Host side of the batched segmented sort (C ABI in include/hpcs_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/hpcs_gpu.h"
#include "segmented_host.cuh"

struct hpcs_segplan {
  hpcs_ctx* ctx = nullptr;
  int64_t nsegs = 0;
  hpcs::SegDesc* d_desc = nullptr;
  uint32_t* d_queue = nullptr;
  void* d_scratch = nullptr;
  size_t scratch_bytes = 0;
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

}  // namespace hpcs

using namespace hpcs;

extern "C" {

int hpcs_sort_segmented_dev(hpcs_ctx* ctx, const hpcs_segment* segs, int64_t nsegs, void* stream) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  std::vector<SegDesc> table;
  std::vector<SegGroup> groups;
  size_t scratch = 0;
  int rc = seg_build_groups(ctx->seg_tuning, segs, nsegs, table, groups, scratch);
  if (rc != HPCS_OK || nsegs == 0) return rc;
  DeviceGuard2 g(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  const size_t desc_bytes = table.size() * sizeof(SegDesc);
  if ((rc = ensure(ctx, ctx->aux0, scratch ? scratch : 256)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->aux1, desc_bytes + 256 + groups.size() * 4)) != HPCS_OK) return rc;
  seg_relocate(table, groups, ctx->aux0.ptr);
  SegDesc* d_desc = static_cast<SegDesc*>(ctx->aux1.ptr);
  uint32_t* d_queues = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(ctx->aux1.ptr) + (desc_bytes + 255) / 256 * 256);
  // the host table must outlive the copy: copy synchronously with respect to this stream
  HPCS_CUDA(cudaMemcpyAsync(d_desc, table.data(), desc_bytes, cudaMemcpyHostToDevice, s));
  HPCS_CUDA(cudaStreamSynchronize(s));
  KernelTimer kt(ctx, s, HPCS_K_SEGMENTED);
  return seg_launch_groups(ctx, d_desc, groups, d_queues, s);
}

int hpcs_segplan_create(hpcs_ctx* ctx, const hpcs_segment* segs, int64_t nsegs, hpcs_segplan** out) {
  if (!ctx || !out) return fail(HPCS_ERR_NULL, "ctx or out is NULL");
  *out = nullptr;
  std::vector<SegDesc> table;
  std::vector<SegGroup> groups;
  size_t scratch = 0;
  int rc = seg_build_groups(ctx->seg_tuning, segs, nsegs, table, groups, scratch);
  if (rc != HPCS_OK) return rc;
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
  cudaError_t e;
  if ((e = cudaMalloc(&p->d_desc, queue_off + 256 + groups.size() * 4)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaMalloc"));
  p->d_queue = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(p->d_desc) + queue_off);
  if (scratch && (e = cudaMalloc(&p->d_scratch, scratch)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc"));
  p->scratch_bytes = scratch;
  seg_relocate(table, groups, p->d_scratch);
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
    if ((e = cudaStreamSynchronize(p->capture_stream)) != cudaSuccess) return cleanup(cuda_fail(e, "sync"));
  }
  const bool was_profiling = ctx->profile;
  ctx->profile = false;  // no event records inside the graph
  if ((e = cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
    ctx->profile = was_profiling;
    return cleanup(cuda_fail(e, "cudaStreamBeginCapture"));
  }
  rc = seg_launch_groups(ctx, p->d_desc, groups, p->d_queue, p->capture_stream);
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
