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

// Validates the descriptors and builds the device table in launch order (largest first);
// returns the scratch bytes needed for arrays larger than one tile.
int build_table(const hpcs_segment* segs, int64_t nsegs, std::vector<SegDesc>& table, size_t& scratch) {
  if (!segs && nsegs > 0) return fail(HPCS_ERR_NULL, "segments is NULL");
  if (nsegs < 0 || nsegs > (int64_t(1) << 31) - 1) return fail(HPCS_ERR_RANGE, "segment count out of range");
  std::vector<int64_t> order(static_cast<size_t>(nsegs));
  std::iota(order.begin(), order.end(), 0);
  for (int64_t i = 0; i < nsegs; i++) {
    if (segs[i].n < 0 || segs[i].n > HPCS_MAX_KEYS) return fail(HPCS_ERR_RANGE, "segment length out of range");
    if (segs[i].n > 0 && !segs[i].keys) return fail(HPCS_ERR_NULL, "segment keys is NULL");
    if (segs[i].dtype < HPCS_U32 || segs[i].dtype > HPCS_F64) return fail(HPCS_ERR_UNSUPPORTED, "unknown dtype");
  }
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    return segs[a].n * key_bytes(segs[a].dtype) > segs[b].n * key_bytes(segs[b].dtype);
  });
  table.resize(size_t(nsegs));
  scratch = 0;
  for (int64_t j = 0; j < nsegs; j++) {
    const hpcs_segment& sg = segs[order[j]];
    SegDesc& d = table[j];
    d.keys = sg.keys;
    d.n = sg.n;
    d.dtype = sg.dtype;
    d.pad = 0;
    d.scratch = nullptr;
    const int64_t tile_keys = int64_t(SEG_NT) * SEG_KPT * 4 / key_bytes(sg.dtype);
    if (sg.n > tile_keys) {
      d.scratch = reinterpret_cast<void*>(scratch);  // offset for now
      scratch += (size_t(sg.n) * key_bytes(sg.dtype) + 255) / 256 * 256;
    }
  }
  return HPCS_OK;
}

// Turns the scratch offsets of build_table into device pointers inside `base`.
void relocate(std::vector<SegDesc>& table, void* base) {
  for (auto& d : table) {
    const int64_t tile_keys = int64_t(SEG_NT) * SEG_KPT * 4 / key_bytes(d.dtype);
    if (d.n > tile_keys) d.scratch = static_cast<unsigned char*>(base) + reinterpret_cast<size_t>(d.scratch);
  }
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

}  // namespace
}  // namespace hpcs

using namespace hpcs;

extern "C" {

int hpcs_sort_segmented_dev(hpcs_ctx* ctx, const hpcs_segment* segs, int64_t nsegs, void* stream) {
  if (!ctx) return fail(HPCS_ERR_NULL, "ctx is NULL");
  std::vector<SegDesc> table;
  size_t scratch = 0;
  int rc = build_table(segs, nsegs, table, scratch);
  if (rc != HPCS_OK || nsegs == 0) return rc;
  DeviceGuard2 g(ctx->device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  if ((rc = enter_stream(ctx, s)) != HPCS_OK) return rc;
  const size_t desc_bytes = table.size() * sizeof(SegDesc);
  if ((rc = ensure(ctx, ctx->aux0, scratch ? scratch : 256)) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->aux1, desc_bytes + 256)) != HPCS_OK) return rc;
  relocate(table, ctx->aux0.ptr);
  SegDesc* d_desc = static_cast<SegDesc*>(ctx->aux1.ptr);
  uint32_t* d_queue = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(ctx->aux1.ptr) + desc_bytes);
  // the host table must outlive the copy: copy synchronously with respect to this stream
  HPCS_CUDA(cudaMemcpyAsync(d_desc, table.data(), desc_bytes, cudaMemcpyHostToDevice, s));
  HPCS_CUDA(cudaStreamSynchronize(s));
  return enqueue_segmented(ctx, d_desc, int(nsegs), d_queue, s);
}

int hpcs_segplan_create(hpcs_ctx* ctx, const hpcs_segment* segs, int64_t nsegs, hpcs_segplan** out) {
  if (!ctx || !out) return fail(HPCS_ERR_NULL, "ctx or out is NULL");
  *out = nullptr;
  std::vector<SegDesc> table;
  size_t scratch = 0;
  int rc = build_table(segs, nsegs, table, scratch);
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
  cudaError_t e;
  if ((e = cudaMalloc(&p->d_desc, desc_bytes + 256)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc"));
  p->d_queue = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(p->d_desc) + desc_bytes);
  if (scratch && (e = cudaMalloc(&p->d_scratch, scratch)) != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc"));
  p->scratch_bytes = scratch;
  relocate(table, p->d_scratch);
  if (desc_bytes && (e = cudaMemcpy(p->d_desc, table.data(), desc_bytes, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaMemcpy"));
  if ((e = cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaStreamCreate"));
  // warm the kernel attributes outside capture, then capture the launch
  if ((rc = enqueue_segmented(ctx, p->d_desc, 0, p->d_queue, p->capture_stream)) != HPCS_OK) return cleanup(rc);
  if ((e = cudaStreamSynchronize(p->capture_stream)) != cudaSuccess) return cleanup(cuda_fail(e, "sync"));
  const bool was_profiling = ctx->profile;
  ctx->profile = false;  // no event records inside the graph
  if ((e = cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
    ctx->profile = was_profiling;
    return cleanup(cuda_fail(e, "cudaStreamBeginCapture"));
  }
  rc = enqueue_segmented(ctx, p->d_desc, int(nsegs), p->d_queue, p->capture_stream);
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
