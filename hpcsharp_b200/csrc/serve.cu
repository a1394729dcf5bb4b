// Serving runtime: sort and top-k requests of mixed size and dtype arrive at any time; a
// scheduler thread admits them as device memory and execution slots free up and runs them
// concurrently on the GPU (continuous batching).
//
// No reference counterpart (HPCsharp is a synchronous library); every result equals the plain
// entry point's result for the same input (sort: hpcs_sort_<t>; top-k: hpcs_topk_largest_<t>).
//
//   memory     one device arena of hbm_budget_bytes, reserved at creation; each admitted
//              request takes its keys and scratch from it (first-fit, 256-byte aligned) and
//              gives them back when it completes.  A request waits while it does not fit.
//   slots      `slots` CUDA streams, each with its own context; a large request runs alone on
//              a slot: H2D copy, sort (or select + gather + sort of the k largest), D2H copy.
//   coalescing requests of at most coalesce_max_keys keys are gathered into one batched
//              segmented-sort launch on a separate stream (a top-k request returns the tail of
//              its sorted array, which is exactly its k largest in ascending order).
//   completion per-slot / per-batch CUDA events, polled by the scheduler, which also reads the
//              device error word copied back with each request.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/hpcs_gpu.h"
#include "segmented_host.cuh"
#include "sort_host.cuh"
#include "topk_host.cuh"

namespace hpcs {
namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }
int dtype_bytes(int dt) { return dt >= HPCS_U64 ? 8 : 4; }

// First-fit allocator over [0, size) with coalescing of freed neighbours.
class Arena {
 public:
  void init(size_t size) {
    free_.clear();
    free_[0] = size;
    size_ = size;
    used_ = 0;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = up256(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes;
        const size_t start = it->first + bytes;
        free_.erase(it);
        if (rest) free_[start] = rest;
        used_ += bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = up256(bytes);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t size() const { return size_; }
  size_t used() const { return used_; }

 private:
  std::map<size_t, size_t> free_;
  size_t size_ = 0, used_ = 0;
};

struct Req {
  uint64_t id = 0;
  hpcs_request r{};
  int64_t t_submit = 0, t_admit = 0, t_done = 0;
  int status = HPCS_OK;
  bool done = false;
  bool coalesced = false;
  size_t off = 0, bytes = 0;
};

// Scratch layout of a request that runs on a slot (offsets from its arena slice).
struct SlotLayout {
  size_t a = 0, b = 0, st0 = 0, st1 = 0, plan = 0, cand = 0, state = 0, out = 0, total = 0;
  size_t keys_bytes = 0, status_bytes = 0;
};

SlotLayout slot_layout(const hpcs_request& r) {
  SlotLayout l;
  const size_t w = size_t(dtype_bytes(r.dtype));
  const int64_t units = (r.n + 4095) / 4096;  // the smallest tile of any config
  l.keys_bytes = up256(size_t(r.n) * w);
  // look-back status words, or the chunked passes' per-range count tables (at most one
  // range per tile and per SM)
  const size_t lookback = size_t(units) * 256 * 4;
  const size_t ranges = size_t(units < 256 ? units : 256);
  const size_t chunked = ranges * (w + 3) * 256 * 4;
  l.status_bytes = up256(lookback > chunked ? lookback : chunked);
  size_t o = 0;
  l.a = o;
  o += l.keys_bytes;
  l.b = o;
  o += l.keys_bytes;
  l.st0 = o;
  o += l.status_bytes;
  l.st1 = o;
  o += l.status_bytes;
  l.plan = o;
  o += up256(sizeof(SortPlan));
  if (r.op == HPCS_OP_TOPK) {
    l.cand = o;
    o += l.keys_bytes;
    l.state = o;
    o += up256(sizeof(SelectState));
    l.out = o;
    o += up256(size_t(r.k) * w);
  }
  l.total = o;
  return l;
}

// The segmented-sort variant a coalesced request runs with, and whether it needs scratch
// (a block-level variant whose tile is shorter than the array).
int coalesced_variant(const hpcs_seg_tuning& t, const hpcs_request& r) {
  return t.variant[dtype_bytes(r.dtype) == 8 ? 1 : 0][seg_class_of(r.n)];
}
bool coalesced_needs_scratch(const hpcs_seg_tuning& t, const hpcs_request& r) {
  return seg_variant_large(coalesced_variant(t, r), r.n, dtype_bytes(r.dtype));
}

// Bytes of a coalesced request: its keys, plus segment scratch if its variant needs it.
size_t coalesced_bytes(const hpcs_seg_tuning& t, const hpcs_request& r) {
  const int w = dtype_bytes(r.dtype);
  size_t b = up256(size_t(r.n) * w);
  if (coalesced_needs_scratch(t, r)) b *= 2;
  return b;
}

template <class U, int KIND>
int run_on_slot(hpcs_ctx* c, const hpcs_request& r, unsigned char* base, const SlotLayout& l, cudaStream_t s) {
  const size_t w = sizeof(U);
  U* a = reinterpret_cast<U*>(base + l.a);
  HPCS_CUDA(cudaMemcpyAsync(a, r.input, size_t(r.n) * w, cudaMemcpyHostToDevice, s));
  if (r.op == HPCS_OP_SORT) {
    int rc = enqueue_sort<U, KIND, NoValue>(c, a, nullptr, r.n, s);
    if (rc != HPCS_OK) return rc;
    HPCS_CUDA(cudaMemcpyAsync(r.output, a, size_t(r.n) * w, cudaMemcpyDeviceToHost, s));
  } else {
    U* out = reinterpret_cast<U*>(base + l.out);
    if (r.k > 0) {
      int rc = topk_largest_enqueue<U, U, KIND>(c, a, r.n, r.k, out, s);
      if (rc != HPCS_OK) return rc;
      HPCS_CUDA(cudaMemcpyAsync(r.output, out, size_t(r.k) * w, cudaMemcpyDeviceToHost, s));
    }
  }
  return HPCS_OK;
}

int dispatch_slot(hpcs_ctx* c, const hpcs_request& r, unsigned char* base, const SlotLayout& l, cudaStream_t s) {
  switch (r.dtype) {
    case HPCS_U32: return run_on_slot<uint32_t, KIND_UNSIGNED>(c, r, base, l, s);
    case HPCS_I32: return run_on_slot<uint32_t, KIND_SIGNED>(c, r, base, l, s);
    case HPCS_F32: return run_on_slot<uint32_t, KIND_FLOAT>(c, r, base, l, s);
    case HPCS_U64: return run_on_slot<uint64_t, KIND_UNSIGNED>(c, r, base, l, s);
    case HPCS_I64: return run_on_slot<uint64_t, KIND_SIGNED>(c, r, base, l, s);
    case HPCS_F64: return run_on_slot<uint64_t, KIND_FLOAT>(c, r, base, l, s);
    default: return fail(HPCS_ERR_UNSUPPORTED, "unknown dtype");
  }
}

void bind(DevBuf& b, unsigned char* p, size_t bytes) {
  b.ptr = p;
  b.bytes = bytes;
  b.borrowed = true;
}

void unbind(DevBuf& b) {
  b.ptr = nullptr;
  b.bytes = 0;
  b.borrowed = false;
}

}  // namespace
}  // namespace hpcs

using namespace hpcs;

struct hpcs_server {
  hpcs_server_config cfg{};
  unsigned char* arena_base = nullptr;
  Arena arena;
  struct Slot {
    hpcs_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    Req* busy = nullptr;
  };
  std::vector<Slot> slots;
  // coalesced batches
  hpcs_ctx* bctx = nullptr;
  cudaStream_t bstream = nullptr;
  cudaEvent_t bev = nullptr;
  std::vector<Req*> batch;
  size_t batch_meta_off = 0, batch_meta_bytes = 0;
  SegDesc* host_table = nullptr;  // pinned staging of the descriptor table
  uint32_t* host_err = nullptr;   // pinned: one error word per slot + one for batches
  // queues
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<Req*> pending;
  std::unordered_map<uint64_t, Req*> reqs;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread th;
  // stats
  int64_t completed = 0, keys_done = 0, batches = 0, coalesced = 0;
  size_t peak_arena = 0;
  std::string last_error;
};

namespace hpcs {
namespace {

void finish(hpcs_server* sv, Req* q, uint32_t err_bits) {
  q->t_done = now_ns();
  if (err_bits && q->status == HPCS_OK) q->status = HPCS_ERR_DEVICE_TIMEOUT;
  q->done = true;
  sv->arena.release(q->off, q->bytes);
  sv->completed++;
  sv->keys_done += q->r.n;
}

// Starts one large request on a free slot; returns false if it does not fit yet.
bool start_on_slot(hpcs_server* sv, hpcs_server::Slot& sl, int slot_idx, Req* q) {
  const SlotLayout l = slot_layout(q->r);
  size_t off = 0;
  if (!sv->arena.alloc(l.total, &off)) return false;
  q->off = off;
  q->bytes = l.total;
  q->t_admit = now_ns();
  unsigned char* base = sv->arena_base + off;
  hpcs_ctx* c = sl.ctx;
  bind(c->keys_b, base + l.b, l.keys_bytes);
  bind(c->status0, base + l.st0, l.status_bytes);
  bind(c->status1, base + l.st1, l.status_bytes);
  bind(c->plan, base + l.plan, up256(sizeof(SortPlan)));
  if (q->r.op == HPCS_OP_TOPK) {
    bind(c->aux0, base + l.cand, l.keys_bytes);
    bind(c->aux1, base + l.state, up256(sizeof(SelectState)));
  }
  c->last_stream = sl.stream;
  int rc = dispatch_slot(c, q->r, base, l, sl.stream);
  if (rc == HPCS_OK) {
    cudaMemcpyAsync(&sv->host_err[slot_idx], c->err_accum.ptr, 4, cudaMemcpyDeviceToHost, sl.stream);
    cudaMemsetAsync(c->err_accum.ptr, 0, 4, sl.stream);
  } else {
    q->status = rc;
  }
  cudaEventRecord(sl.ev, sl.stream);
  unbind(c->keys_b);
  unbind(c->status0);
  unbind(c->status1);
  unbind(c->plan);
  unbind(c->aux0);
  unbind(c->aux1);
  sl.busy = q;
  return true;
}

// Launches the gathered small requests as one segmented sort: the descriptors are ordered by
// tuned kernel variant (one persistent launch per variant, concurrent) and length.
void launch_batch(hpcs_server* sv) {
  const size_t n = sv->batch.size();
  hpcs_ctx* c = sv->bctx;
  cudaStream_t s = sv->bstream;
  SegDesc* d_table = reinterpret_cast<SegDesc*>(sv->arena_base + sv->batch_meta_off);
  uint32_t* d_queues = reinterpret_cast<uint32_t*>(sv->arena_base + sv->batch_meta_off + n * sizeof(SegDesc));
  std::vector<size_t> order(n);
  for (size_t i = 0; i < n; i++) order[i] = i;
  auto gid = [&](const hpcs_request& r) {
    return 2 * coalesced_variant(c->seg_tuning, r) + (coalesced_needs_scratch(c->seg_tuning, r) ? 1 : 0);
  };
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    const int va = gid(sv->batch[a]->r), vb = gid(sv->batch[b]->r);
    if (va != vb) return va < vb;
    return sv->batch[a]->r.n * dtype_bytes(sv->batch[a]->r.dtype) > sv->batch[b]->r.n * dtype_bytes(sv->batch[b]->r.dtype);
  });
  std::vector<SegGroup> groups;
  for (size_t j = 0; j < n; j++) {
    Req* q = sv->batch[order[j]];
    const int w = dtype_bytes(q->r.dtype);
    const int v = coalesced_variant(c->seg_tuning, q->r);
    const bool large = coalesced_needs_scratch(c->seg_tuning, q->r);
    if (groups.empty() || groups.back().variant != v || groups.back().large != large)
      groups.push_back({v, large, int(j), 0});
    groups.back().count++;
    unsigned char* keys = sv->arena_base + q->off;
    SegDesc& d = sv->host_table[j];
    d.keys = keys;
    d.n = q->r.n;
    d.dtype = q->r.dtype;
    d.pad = 0;
    d.scratch = coalesced_needs_scratch(c->seg_tuning, q->r) ? keys + up256(size_t(q->r.n) * w) : nullptr;
    cudaMemcpyAsync(keys, q->r.input, size_t(q->r.n) * w, cudaMemcpyHostToDevice, s);
  }
  cudaMemcpyAsync(d_table, sv->host_table, n * sizeof(SegDesc), cudaMemcpyHostToDevice, s);
  c->last_stream = s;
  int rc = seg_launch_groups(c, d_table, groups, d_queues, s);
  for (size_t i = 0; i < n; i++) {
    Req* q = sv->batch[i];
    const int w = dtype_bytes(q->r.dtype);
    unsigned char* keys = sv->arena_base + q->off;
    if (rc != HPCS_OK) {
      q->status = rc;
      continue;
    }
    if (q->r.op == HPCS_OP_SORT)
      cudaMemcpyAsync(q->r.output, keys, size_t(q->r.n) * w, cudaMemcpyDeviceToHost, s);
    else if (q->r.k > 0)  // the k largest = the tail of the sorted array, ascending
      cudaMemcpyAsync(q->r.output, keys + size_t(q->r.n - q->r.k) * w, size_t(q->r.k) * w,
                      cudaMemcpyDeviceToHost, s);
  }
  const size_t eidx = sv->slots.size();
  cudaMemcpyAsync(&sv->host_err[eidx], c->err_accum.ptr, 4, cudaMemcpyDeviceToHost, s);
  cudaMemsetAsync(c->err_accum.ptr, 0, 4, s);
  cudaEventRecord(sv->bev, s);
  sv->batches++;
  sv->coalesced += int64_t(n);
}

void scheduler(hpcs_server* sv) {
  cudaSetDevice(sv->cfg.device);
  std::unique_lock<std::mutex> lock(sv->mu);
  while (true) {
    bool progress = false;
    // retire
    for (size_t i = 0; i < sv->slots.size(); i++) {
      auto& sl = sv->slots[i];
      if (sl.busy && cudaEventQuery(sl.ev) == cudaSuccess) {
        finish(sv, sl.busy, sv->host_err[i]);
        sl.busy = nullptr;
        progress = true;
      }
    }
    if (!sv->batch.empty() && cudaEventQuery(sv->bev) == cudaSuccess) {
      const uint32_t e = sv->host_err[sv->slots.size()];
      for (Req* q : sv->batch) finish(sv, q, e);
      sv->arena.release(sv->batch_meta_off, sv->batch_meta_bytes);
      sv->batch.clear();
      progress = true;
    }
    if (progress) sv->cv_done.notify_all();
    // admit: small requests into the next batch (when none is in flight), large ones onto
    // free slots; each in arrival order among its kind while device memory allows
    if (sv->batch.empty()) {
      std::vector<Req*> take;
      for (Req* q : sv->pending) {
        if (q->r.n > sv->cfg.coalesce_max_keys) continue;
        if (int(take.size()) >= sv->cfg.coalesce_max_requests) break;
        size_t off = 0;
        if (!sv->arena.alloc(coalesced_bytes(sv->bctx->seg_tuning, q->r), &off)) break;
        q->off = off;
        q->bytes = coalesced_bytes(sv->bctx->seg_tuning, q->r);
        q->coalesced = true;
        q->t_admit = now_ns();
        take.push_back(q);
      }
      if (!take.empty()) {
        const size_t meta = take.size() * sizeof(SegDesc) + 256;
        size_t moff = 0;
        if (sv->arena.alloc(meta, &moff)) {
          sv->batch_meta_off = moff;
          sv->batch_meta_bytes = meta;
          sv->batch = take;
          for (Req* q : take) sv->pending.erase(std::find(sv->pending.begin(), sv->pending.end(), q));
          launch_batch(sv);
          progress = true;
        } else {
          for (Req* q : take) {
            sv->arena.release(q->off, q->bytes);
            q->coalesced = false;
          }
        }
      }
    }
    for (size_t i = 0; i < sv->slots.size(); i++) {
      auto& sl = sv->slots[i];
      if (sl.busy) continue;
      Req* next = nullptr;
      for (Req* q : sv->pending)
        if (q->r.n > sv->cfg.coalesce_max_keys) {
          next = q;
          break;
        }
      if (!next) break;
      if (!start_on_slot(sv, sl, int(i), next)) break;  // wait for memory
      sv->pending.erase(std::find(sv->pending.begin(), sv->pending.end(), next));
      progress = true;
    }
    if (sv->arena.used() > sv->peak_arena) sv->peak_arena = sv->arena.used();
    bool busy = !sv->batch.empty();
    for (auto& sl : sv->slots) busy = busy || sl.busy;
    if (sv->stop && !busy && sv->pending.empty()) break;
    if (!progress) {
      if (busy) sv->cv_sched.wait_for(lock, std::chrono::microseconds(20));
      else sv->cv_sched.wait_for(lock, std::chrono::milliseconds(5));
    }
  }
}

int check_request(hpcs_server* sv, const hpcs_request* r) {
  if (!r || !r->input || !r->output) return fail(HPCS_ERR_NULL, "request, input or output is NULL");
  if (r->op != HPCS_OP_SORT && r->op != HPCS_OP_TOPK) return fail(HPCS_ERR_UNSUPPORTED, "unknown op");
  if (r->dtype < HPCS_U32 || r->dtype > HPCS_F64) return fail(HPCS_ERR_UNSUPPORTED, "unknown dtype");
  if (r->n <= 0 || r->n > HPCS_MAX_SEGMENT_KEYS) return fail(HPCS_ERR_RANGE, "n out of range");
  if (r->op == HPCS_OP_TOPK && (r->k < 0 || r->k > r->n)) return fail(HPCS_ERR_RANGE, "k must be in [0, n]");
  const size_t need = r->n <= sv->cfg.coalesce_max_keys ? coalesced_bytes(sv->bctx->seg_tuning, *r) + 256 : slot_layout(*r).total;
  if (need > sv->arena.size()) return fail(HPCS_ERR_OOM, "request larger than the server's HBM budget");
  return HPCS_OK;
}

}  // namespace
}  // namespace hpcs

extern "C" {

void hpcs_server_config_default(hpcs_server_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->device = 0;
  c->slots = 4;
  c->hbm_budget_bytes = int64_t(64) << 30;
  c->coalesce_max_keys = 1 << 17;
  c->coalesce_max_requests = 4096;
}

int hpcs_server_create(const hpcs_server_config* cfg, hpcs_server** out) {
  if (!out) return fail(HPCS_ERR_NULL, "out is NULL");
  *out = nullptr;
  auto* sv = new hpcs_server();
  if (cfg) sv->cfg = *cfg;
  else hpcs_server_config_default(&sv->cfg);
  if (sv->cfg.slots < 1) sv->cfg.slots = 1;
  if (sv->cfg.coalesce_max_requests < 1) sv->cfg.coalesce_max_requests = 1;
  if (sv->cfg.hbm_budget_bytes <= 0) {
    delete sv;
    return fail(HPCS_ERR_RANGE, "hbm_budget_bytes must be positive");
  }
  int rc;
  auto undo = [&](int code) {
    hpcs_server_destroy(sv);
    return code;
  };
  cudaError_t e = cudaSetDevice(sv->cfg.device);
  if (e != cudaSuccess) {
    delete sv;
    return cuda_fail(e, "cudaSetDevice");
  }
  if ((e = cudaMalloc(&sv->arena_base, size_t(sv->cfg.hbm_budget_bytes))) != cudaSuccess) {
    sv->arena_base = nullptr;
    cudaGetLastError();
    return undo(cuda_fail(e, "cudaMalloc (server arena)"));
  }
  sv->arena.init(size_t(sv->cfg.hbm_budget_bytes));
  sv->slots.resize(size_t(sv->cfg.slots));
  for (auto& sl : sv->slots) {
    if ((rc = hpcs_ctx_create(sv->cfg.device, nullptr, &sl.ctx)) != HPCS_OK) return undo(rc);
    sl.stream = sl.ctx->stream;
    if ((e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming)) != cudaSuccess) return undo(cuda_fail(e, "event"));
  }
  if ((rc = hpcs_ctx_create(sv->cfg.device, nullptr, &sv->bctx)) != HPCS_OK) return undo(rc);
  sv->bstream = sv->bctx->stream;
  if ((e = cudaEventCreateWithFlags(&sv->bev, cudaEventDisableTiming)) != cudaSuccess) return undo(cuda_fail(e, "event"));
  if ((e = cudaMallocHost(&sv->host_table, size_t(sv->cfg.coalesce_max_requests) * sizeof(SegDesc))) != cudaSuccess)
    return undo(cuda_fail(e, "cudaMallocHost"));
  if ((e = cudaMallocHost(&sv->host_err, (sv->slots.size() + 1) * 4)) != cudaSuccess)
    return undo(cuda_fail(e, "cudaMallocHost"));
  std::memset(sv->host_err, 0, (sv->slots.size() + 1) * 4);
  sv->th = std::thread(scheduler, sv);
  *out = sv;
  return HPCS_OK;
}

int hpcs_server_submit(hpcs_server* sv, const hpcs_request* req, uint64_t* ticket) {
  if (!sv || !ticket) return fail(HPCS_ERR_NULL, "server or ticket is NULL");
  int rc = check_request(sv, req);
  if (rc != HPCS_OK) return rc;
  auto* q = new Req();
  q->r = *req;
  q->t_submit = now_ns();
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->stop) {
      delete q;
      return fail(HPCS_ERR_BUSY, "server is shutting down");
    }
    q->id = sv->next_id++;
    sv->reqs[q->id] = q;
    sv->pending.push_back(q);
  }
  sv->cv_sched.notify_one();
  *ticket = q->id;
  return HPCS_OK;
}

int hpcs_server_wait(hpcs_server* sv, uint64_t ticket, int64_t timeout_ns, hpcs_request_info* info) {
  if (!sv) return fail(HPCS_ERR_NULL, "server is NULL");
  std::unique_lock<std::mutex> lock(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return fail(HPCS_ERR_RANGE, "unknown ticket");
  Req* q = it->second;
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::nanoseconds(timeout_ns > 0 ? timeout_ns : 0);
  while (!q->done) {
    if (timeout_ns > 0) {
      if (sv->cv_done.wait_until(lock, deadline) == std::cv_status::timeout && !q->done)
        return fail(HPCS_ERR_BUSY, "request not finished before the timeout");
    } else {
      sv->cv_done.wait(lock);
    }
  }
  if (info) {
    info->status = q->status;
    info->coalesced = q->coalesced ? 1 : 0;
    info->submit_ns = q->t_submit;
    info->admit_ns = q->t_admit;
    info->done_ns = q->t_done;
  }
  const int status = q->status;
  sv->reqs.erase(it);
  delete q;
  return status;
}

int hpcs_server_stats(hpcs_server* sv, hpcs_server_counters* st) {
  if (!sv || !st) return fail(HPCS_ERR_NULL, "server or stats is NULL");
  std::lock_guard<std::mutex> lock(sv->mu);
  st->completed = sv->completed;
  st->keys = sv->keys_done;
  st->batches = sv->batches;
  st->coalesced = sv->coalesced;
  st->pending = int64_t(sv->pending.size());
  st->arena_bytes = int64_t(sv->arena.size());
  st->arena_used = int64_t(sv->arena.used());
  st->arena_peak = int64_t(sv->peak_arena);
  return HPCS_OK;
}

int hpcs_server_destroy(hpcs_server* sv) {
  if (!sv) return HPCS_OK;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->stop = true;
  }
  sv->cv_sched.notify_all();
  if (sv->th.joinable()) sv->th.join();
  for (auto& kv : sv->reqs) delete kv.second;
  for (auto& sl : sv->slots) {
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.ctx) hpcs_ctx_destroy(sl.ctx);
  }
  if (sv->bev) cudaEventDestroy(sv->bev);
  if (sv->bctx) hpcs_ctx_destroy(sv->bctx);
  if (sv->host_table) cudaFreeHost(sv->host_table);
  if (sv->host_err) cudaFreeHost(sv->host_err);
  if (sv->arena_base) cudaFree(sv->arena_base);
  delete sv;
  return HPCS_OK;
}

}  // extern "C"
