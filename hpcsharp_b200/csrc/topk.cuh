// Radix selection / top-k on the GPU.
//
// Restates the observable contract of HPCsharp's SelectTopK(this uint[] a, int k)
// (SelectionTopKRadix.cs:142-171): afterwards a[k] is the k-th smallest key (0-based) and
// a[k..n-1] holds exactly the multiset of the n-k largest.  The reference gets there with an
// in-place MSD radix select of 16-bit digits (RadixSelectionTopKWordInner, :96-133) whose
// movers clobber the prefix; here the prefix is defined too: a[0..k-1] holds the k smallest.
//
// Selection: an MSD radix select over the order-transformed key (the same transforms as the
// sort), 8 bits per level.  A strided sample of the keys first bounds where the selected key
// lies (a window around its rank; for the k largest, a threshold), and one read of all keys
// keeps the keys inside (the candidates) and counts those below.  The levels then histogram
// only candidates that match the prefix chosen so far.  When the sample misled (the rank falls
// outside the candidates), the select runs over all keys instead: level 0 histograms all n
// keys and the keys of the chosen bin are compacted into the candidate buffer.  The choice is
// made on the device.  A one-block "pick" kernel after each histogram advances the device-side
// SelectState, so nothing returns to the host between levels.  The passes over all n keys read
// them with 16-byte loads, several in flight per thread (visit_keys); compactions stage kept
// keys per warp in shared memory and take one global atomic per 1 KiB of them.
//
// Rearrangement: a stable three-way partition (keys < v, == v, > v around the selected key v)
// -- per-tile class counts, a two-level scan of them, a stable per-tile scatter.
// The k largest ("top-k" of a serving request) are the keys > v among the candidates plus
// copies of v up to k, sorted ascending (in one CTA for up to 8 Ki keys, else with the LSD
// sort) so the output bytes are deterministic.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace hpcs {

struct SelectState {
  uint64_t prefix;     // ordered-key bits chosen so far
  uint64_t mask;       // which bits of the prefix are fixed
  int64_t rank;        // rank still to find among keys matching the prefix
  int64_t less;        // keys strictly below the prefix range
  int64_t eq;          // keys equal to the selected key (valid after the last level)
  int64_t cand_count;  // candidates compacted after level 0
  unsigned long long gathered;  // keys > v written to the top-k output so far
  int64_t n_total;     // keys selected among
  uint64_t threshold;  // top-k: ordered keys at or above it are the filter's candidates;
                       // select: the window's lower end
  uint64_t threshold_hi;        // select: the window's upper end (inclusive)
  unsigned long long below;     // select: keys below the window
  int32_t mode;        // SEL_MODE_CAND (select among the candidates) or SEL_MODE_FULL
  int32_t pad;
  uint32_t hist[256];
};
enum : int32_t { SEL_MODE_ANY = -1, SEL_MODE_FULL = 0, SEL_MODE_CAND = 1 };

constexpr int SEL_NT = 512;
constexpr int SEL_COPIES = 32;
constexpr int SEL_VPT = 4;  // 16-byte vectors in flight per thread
constexpr int SEL_CTAS_PER_SM = 4;

// Per-warp staging of appended keys in shared memory: a warp scan places each lane's keys in
// the warp's CAP-key buffer, and a buffer that would overflow goes to dst with one atomic on
// the global counter, so a sparse compaction takes one atomic per CAP keys instead of one per
// warp and vector row.  Every lane of the warp makes the same calls; count is the same in all
// lanes.  Positions at or beyond `cap` are not written.
template <class U, int E, int CAP>
struct WarpStage {
  U* buf;
  uint32_t count;
  U* __restrict__ dst;
  unsigned long long* counter;
  int64_t cap;

  __device__ __forceinline__ void flush() {
    if (count == 0u) return;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, (unsigned long long)count);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    for (uint32_t j = lane; j < count; j += 32)
      if (int64_t(base + j) < cap) dst[base + j] = buf[j];
    __syncwarp();
    count = 0u;
  }

  __device__ __forceinline__ void add(const U* k, uint32_t take) {
    static_assert(32 * E <= CAP, "one call must fit an empty buffer");
    if (__ballot_sync(0xFFFFFFFFu, take != 0u) == 0u) return;  // nothing kept by the warp
    const int lane = threadIdx.x & 31;
    const uint32_t c = __popc(take);
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (total == 0u) return;  // uniform over the warp
    if (count + total > uint32_t(CAP)) flush();
    uint32_t pos = count + incl - c;
#pragma unroll
    for (int e = 0; e < E; e++)
      if ((take >> e) & 1u) buf[pos++] = k[e];
    count += total;
    __syncwarp();  // the keys are in the buffer before any lane flushes it
  }
};

// Histogram of the digit at `shift` over keys whose ordered bits match (prefix, mask).
template <class U, int KIND>
__global__ void __launch_bounds__(SEL_NT, SEL_CTAS_PER_SM) select_hist_kernel(const U* __restrict__ keys, const int64_t* n_ptr,
                                                             int64_t n_fixed, SelectState* st, int shift,
                                                             int only_mode = SEL_MODE_ANY) {
  using KO = KeyOrder<U, KIND>;
  constexpr int E = int(16 / sizeof(U));
  __shared__ uint32_t sh[256 * SEL_COPIES];
  if (only_mode != SEL_MODE_ANY && st->mode != only_mode) return;  // the other top-k path ran
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < 256 * SEL_COPIES; i += SEL_NT) sh[i] = 0;
  __syncthreads();
  const int64_t n = n_ptr ? *n_ptr : n_fixed;
  const U prefix = U(st->prefix), mask = U(st->mask);
  visit_keys<U, SEL_VPT>(keys, n, [&](const U* k, int nv) {
#pragma unroll
    for (int e = 0; e < E; e++) {
      const U o = KO::to_ordered(k[e]);
      if (e < nv && (o & mask) == prefix) atomicAdd(&sh[((uint32_t(o >> shift) & 0xFFu) * SEL_COPIES) + lane], 1u);
    }
  });
  __syncthreads();
  for (int b = tid; b < 256; b += SEL_NT) {
    uint32_t c = 0;
    for (int q = 0; q < SEL_COPIES; q++) c += sh[b * SEL_COPIES + ((q + lane) & (SEL_COPIES - 1))];
    if (c) atomicAdd(&st->hist[b], c);
  }
}

// One block of 256 threads: choose the bin holding st->rank (a scan of the 256 counts, the
// thread whose bin spans the rank records it), advance the prefix, clear the histogram.
// last != 0: record how many keys equal the selected key.
template <class U>
__global__ void __launch_bounds__(256) select_pick_kernel(SelectState* st, int shift, int last) {
  __shared__ int64_t s_w[8];
  __shared__ int s_bin;
  __shared__ int64_t s_excl, s_cnt;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t c = st->hist[tid];
  int64_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[warp] = incl;
  if (tid == 0) {
    s_bin = -1;
    s_excl = 0;
    s_cnt = 0;
  }
  __syncthreads();
  int64_t base = 0;
  for (int w = 0; w < warp; w++) base += s_w[w];
  const int64_t excl = base + incl - c;
  const int64_t r = st->rank;
  // the bins' ranges [excl, excl + c) are disjoint: at most one thread matches; a rank past
  // every key (not reachable through the entry points) falls to bin 255
  if ((c > 0 && r >= excl && r < excl + c) || (tid == 255 && r >= excl + c)) {
    s_bin = tid;
    s_excl = excl;
    s_cnt = c;
  }
  __syncthreads();
  if (tid == 0) {
    const int bin = s_bin < 0 ? 255 : s_bin;
    st->prefix |= uint64_t(bin) << shift;
    st->mask |= uint64_t(0xFF) << shift;
    st->rank = r - s_excl;
    st->less += s_excl;
    if (last) st->eq = s_cnt;
  }
  st->hist[tid] = 0;
}

// Copies the keys whose ordered top byte matches the level-0 prefix into `cand`.  With `out`
// (top-k): the keys above that bin, all among the k largest, go to out[0..) through
// st->gathered at once (fewer than k of them: the selected rank lies in the bin).
template <class U, int KIND>
__global__ void __launch_bounds__(SEL_NT, SEL_CTAS_PER_SM) select_compact_kernel(const U* __restrict__ keys, int64_t n,
                                                                U* __restrict__ cand, SelectState* st,
                                                                U* __restrict__ out, int64_t k_out,
                                                                int only_mode = SEL_MODE_ANY) {
  using KO = KeyOrder<U, KIND>;
  constexpr int E = int(16 / sizeof(U));
  constexpr int CAP = 1024 / int(sizeof(U));  // 1 KiB per warp and buffer
  __shared__ U s_buf[2][SEL_NT / 32][CAP];
  if (only_mode != SEL_MODE_ANY && st->mode != only_mode) return;  // the other top-k path ran
  const int warp = threadIdx.x >> 5;
  const U prefix = U(st->prefix), mask = U(st->mask);
  WarpStage<U, E, CAP> to_cand{s_buf[0][warp], 0u, cand, reinterpret_cast<unsigned long long*>(&st->cand_count),
                               INT64_MAX};
  WarpStage<U, E, CAP> to_out{s_buf[1][warp], 0u, out, &st->gathered, k_out};
  visit_keys<U, SEL_VPT>(keys, n, [&](const U* k, int nv) {
    uint32_t take = 0u, above = 0u;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const U top = KO::to_ordered(k[e]) & mask;
      if (e < nv && top == prefix) take |= 1u << e;
      if (e < nv && top > prefix) above |= 1u << e;
    }
    to_cand.add(k, take);
    if (out) to_out.add(k, above);
  });
  to_cand.flush();
  if (out) to_out.flush();
}

// ---- top-k with one read of the keys ---------------------------------------------------
// A strided sample of the keys gives a threshold T that about m sampled keys reach; one read of all keys then keeps the keys at or above T (the candidates).  When at
// least k keys were kept, every one of the k largest is among them and the radix select runs
// over the candidates only; otherwise (a sample far off, or tiny inputs) the select falls back
// to the two reads of the full path.  The choice is made on the device (SelectState::mode):
// the kernels of the path not taken return at their first instruction.
template <class U>
__host__ __device__ constexpr int topk_sample_size() {
  return 8192;  // 8 keys per thread in registers
}
// The select's window: its width shrinks as 1/sqrt(samples), and at the median it holds a few
// percent of the keys, so 32-bit keys take four times the samples (32 keys per thread; 64-bit
// keys stay at 8 per thread, where 16 would spill registers).
template <class U>
__host__ __device__ constexpr int select_sample_size() {
  return sizeof(U) == 4 ? 32768 : 8192;
}
constexpr int TOPK_SAMPLE_NT = 1024;

// The ordered value of 0-based ascending rank `rank` among the TOPK_SAMPLE_NT x PER samples o[]
// held by the CTA's threads: an MSD radix select in shared memory, per level a histogram of the
// samples matching the prefix and a scan of its 256 bins by 8 warps.  Every thread returns it.
template <class U, int PER>
__device__ __forceinline__ U sample_rank_value(const U (&o)[PER], uint32_t rank, uint32_t* hist, uint32_t* s_wsum,
                                               uint32_t* s_pick) {
  constexpr int BITS = int(sizeof(U) * 8);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  U prefix = 0, mask = 0;
  for (int shift = BITS - 8; shift >= 0; shift -= 8) {
    if (tid < 256) hist[tid] = 0;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; q++)
      if ((o[q] & mask) == prefix) atomicAdd(&hist[uint32_t(o[q] >> shift) & 0xFFu], 1u);
    __syncthreads();
    uint32_t c = 0, incl = 0;
    if (tid < 256) {
      c = hist[tid];
      incl = c;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, off);
        if (lane >= off) incl += y;
      }
      if (lane == 31) s_wsum[warp] = incl;
    }
    __syncthreads();
    if (tid < 256) {
      uint32_t base = 0;
      for (int w = 0; w < warp; w++) base += s_wsum[w];
      const uint32_t excl = base + incl - c;
      // the bins' ranges [excl, excl + c) are disjoint: exactly one thread matches
      if ((c > 0u && rank >= excl && rank < excl + c) || (tid == 255 && rank >= excl + c)) {
        s_pick[0] = uint32_t(tid);
        s_pick[1] = excl;
      }
    }
    __syncthreads();
    prefix |= U(s_pick[0]) << shift;
    mask |= U(0xFF) << shift;
    rank -= s_pick[1];
    __syncthreads();
  }
  return prefix;
}

// One CTA: the SelectState set up for the k largest of n keys (rank n - k), and the ordered
// sample value of rank (S - m) among S = topk_sample_size<U>() keys at stride n / S.  Writes
// st->threshold (0 = keep every key).
template <class U, int KIND>
__global__ void __launch_bounds__(TOPK_SAMPLE_NT) topk_sample_kernel(const U* __restrict__ keys, int64_t n,
                                                                     int64_t k, int64_t m, SelectState* st) {
  using KO = KeyOrder<U, KIND>;
  constexpr int S = topk_sample_size<U>();
  constexpr int PER = S / TOPK_SAMPLE_NT;
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_wsum[8];
  __shared__ uint32_t s_pick[2];
  const int tid = threadIdx.x;
  if (tid == 0) {
    st->n_total = n;
    st->prefix = 0;
    st->mask = 0;
    st->rank = n - k;
    st->less = 0;
    st->eq = 0;
    st->cand_count = 0;
    st->gathered = 0;
    st->below = 0;
    st->mode = SEL_MODE_FULL;
  }
  if (tid < 256) st->hist[tid] = 0;
  if (n < int64_t(4) * S || m >= S) {  // too few keys to sample: keep them all
    if (tid == 0) st->threshold = 0;
    return;
  }
  const int64_t stride = n / S;
  U o[PER];
#pragma unroll
  for (int q = 0; q < PER; q++) o[q] = KO::to_ordered(keys[int64_t(tid + q * TOPK_SAMPLE_NT) * stride]);
  const U t = sample_rank_value<U, PER>(o, uint32_t(S - m), hist, s_wsum, s_pick);
  if (tid == 0) st->threshold = uint64_t(t);
}

// ---- radix select with one read of the keys ---------------------------------------------
// The key of rank r among n: the same strided sample gives two values lo <= hi whose sample
// ranks lie m below and m above r's expected sample rank (r S / n); one read counts the keys
// below lo and keeps the keys in [lo, hi] (the candidates).  When r falls among the candidates
// (below <= r < below + candidates), the radix select runs over the candidates only, with
// `below` keys already counted under the prefix; otherwise over all keys (the two-read path).
// The choice is made on the device, as for the k largest.

// One CTA: the SelectState set up for rank `rank` among n keys, and the window [lo, hi].  An
// input too small to sample gets an empty window (lo > hi), which sends the select to the
// two-read path.
template <class U, int KIND>
__global__ void __launch_bounds__(TOPK_SAMPLE_NT) select_sample_kernel(const U* __restrict__ keys, int64_t n,
                                                                       int64_t rank, int64_t m, SelectState* st) {
  using KO = KeyOrder<U, KIND>;
  constexpr int S = select_sample_size<U>();
  constexpr int PER = S / TOPK_SAMPLE_NT;
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_wsum[8];
  __shared__ uint32_t s_pick[2];
  const int tid = threadIdx.x;
  if (tid == 0) {
    st->n_total = n;
    st->prefix = 0;
    st->mask = 0;
    st->rank = rank;
    st->less = 0;
    st->eq = 0;
    st->cand_count = 0;
    st->gathered = 0;
    st->below = 0;
    st->mode = SEL_MODE_FULL;
  }
  if (tid < 256) st->hist[tid] = 0;
  if (n < int64_t(4) * S) {
    if (tid == 0) {
      st->threshold = 1;
      st->threshold_hi = 0;
    }
    return;
  }
  const int64_t stride = n / S;
  U o[PER];
#pragma unroll
  for (int q = 0; q < PER; q++) o[q] = KO::to_ordered(keys[int64_t(tid + q * TOPK_SAMPLE_NT) * stride]);
  const int64_t rs = rank * S / n;  // expected sample rank of the selected key
  const int64_t rlo = rs - m, rhi = rs + m;
  // the window reaches the ends of the key range where the margin passes the sample's ends
  const U lo = rlo <= 0 ? U(0) : sample_rank_value<U, PER>(o, uint32_t(rlo), hist, s_wsum, s_pick);
  const U hi = rhi >= S - 1 ? U(~U(0)) : sample_rank_value<U, PER>(o, uint32_t(rhi), hist, s_wsum, s_pick);
  if (tid == 0) {
    st->threshold = uint64_t(lo);
    st->threshold_hi = uint64_t(hi);
  }
}

// One read of the keys: keys in [lo, hi] go to `cand`, keys below lo are counted.
template <class U, int KIND>
__global__ void __launch_bounds__(SEL_NT, SEL_CTAS_PER_SM) select_window_kernel(const U* __restrict__ keys, int64_t n,
                                                                               U* __restrict__ cand, SelectState* st) {
  using KO = KeyOrder<U, KIND>;
  constexpr int E = int(16 / sizeof(U));
  constexpr int CAP = 1024 / int(sizeof(U));
  __shared__ U s_buf[SEL_NT / 32][CAP];
  const U lo = U(st->threshold), hi = U(st->threshold_hi);
  WarpStage<U, E, CAP> to_cand{s_buf[threadIdx.x >> 5], 0u, cand,
                               reinterpret_cast<unsigned long long*>(&st->cand_count), INT64_MAX};
  uint32_t below = 0;
  visit_keys<U, SEL_VPT>(keys, n, [&](const U* k, int nv) {
    uint32_t take = 0u;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const U o = KO::to_ordered(k[e]);
      if (e < nv && o >= lo && o <= hi) take |= 1u << e;
      below += (e < nv && o < lo) ? 1u : 0u;
    }
    to_cand.add(k, take);
  });
  to_cand.flush();
  below = __reduce_add_sync(0xFFFFFFFFu, below);
  if ((threadIdx.x & 31) == 0 && below) atomicAdd(&st->below, (unsigned long long)below);
}

// One thread: select among the candidates when the rank falls among them, else over all keys.
static __global__ void select_decide_kernel(SelectState* st, int64_t n, int64_t rank) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int64_t c = st->cand_count, b = int64_t(st->below);
  if (b <= rank && rank < b + c) {
    st->mode = SEL_MODE_CAND;
    st->n_total = c;
    st->rank = rank - b;
    st->less = b;
  } else {
    st->mode = SEL_MODE_FULL;
    st->n_total = n;
    st->rank = rank;
    st->less = 0;
    st->cand_count = 0;
  }
}

// One read of the keys: the keys whose ordered value is at least the threshold go to `cand`.
template <class U, int KIND>
__global__ void __launch_bounds__(SEL_NT, SEL_CTAS_PER_SM) topk_filter_kernel(const U* __restrict__ keys, int64_t n,
                                                             U* __restrict__ cand, SelectState* st) {
  using KO = KeyOrder<U, KIND>;
  constexpr int E = int(16 / sizeof(U));
  constexpr int CAP = 1024 / int(sizeof(U));
  __shared__ U s_buf[SEL_NT / 32][CAP];
  const U t = U(st->threshold);
  WarpStage<U, E, CAP> to_cand{s_buf[threadIdx.x >> 5], 0u, cand,
                               reinterpret_cast<unsigned long long*>(&st->cand_count), INT64_MAX};
  visit_keys<U, SEL_VPT>(keys, n, [&](const U* k, int nv) {
    uint32_t take = 0u;
#pragma unroll
    for (int e = 0; e < E; e++)
      if (e < nv && KO::to_ordered(k[e]) >= t) take |= 1u << e;
    to_cand.add(k, take);
  });
  to_cand.flush();
}

// One thread: select among the candidates when there are at least k of them (rank cand - k),
// else fall back to the full path over all n keys (rank n - k, the candidates rebuilt).
static __global__ void topk_decide_kernel(SelectState* st, int64_t n, int64_t k) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int64_t c = st->cand_count;
  if (c >= k) {
    st->mode = SEL_MODE_CAND;
    st->n_total = c;
    st->rank = c - k;
  } else {
    st->mode = SEL_MODE_FULL;
    st->n_total = n;
    st->rank = n - k;
    st->cand_count = 0;
  }
}

// ---- stable three-way partition around the selected key -----------------------------
// Each warp owns a sub-tile of PART_SUB consecutive keys and partitions it on its own, with no
// CTA barrier: row j of the sub-tile is keys j * 32 + lane (coalesced loads), a key's stable
// slot among its class comes from the class ballots of its row and the rows before it, the
// warp stages the sub-tile in class order in its own shared memory and writes each class's run
// with consecutive lanes at consecutive positions.  The sub-tiles' class counts (one read) and
// a two-level scan of them give every sub-tile its output starts.
constexpr int PART_NT = 256, PART_KPT = 16;
constexpr int PART_SUB = 32 * PART_KPT;                  // keys per warp sub-tile
constexpr int PART_SUBS_PER_CTA = PART_NT / 32;

template <class U, int KIND>
__device__ __forceinline__ int part_class(U k, U v_ordered) {
  const U o = KeyOrder<U, KIND>::to_ordered(k);
  return o < v_ordered ? 0 : (o == v_ordered ? 1 : 2);
}

template <class U, int KIND>
__global__ void __launch_bounds__(PART_NT) partition_count_kernel(const U* __restrict__ keys, int64_t n,
                                                                  const SelectState* st, uint32_t* sub_counts) {
  const U v = U(st->prefix);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t sub = int64_t(blockIdx.x) * PART_SUBS_PER_CTA + warp;
  const int64_t base = sub * PART_SUB;
  if (base >= n) return;  // warp-uniform
  const int sub_n = int(n - base < PART_SUB ? n - base : PART_SUB);
  uint32_t l = 0, e = 0, g = 0;
#pragma unroll
  for (int j = 0; j < PART_KPT; j++) {
    const int i = j * 32 + lane;
    if (i < sub_n) {
      const int cl = part_class<U, KIND>(keys[base + i], v);
      l += cl == 0;
      e += cl == 1;
      g += cl == 2;
    }
  }
  l = __reduce_add_sync(0xFFFFFFFFu, l);
  e = __reduce_add_sync(0xFFFFFFFFu, e);
  g = __reduce_add_sync(0xFFFFFFFFu, g);
  if (lane < 3) sub_counts[sub * 3 + lane] = lane == 0 ? l : (lane == 1 ? e : g);
}

// Scan of the per-sub-tile class counts in two levels: partition_block_scan_kernel turns the
// counts of each run of PART_SCAN_RUN sub-tiles into starts within the run (a separate array:
// the scatter reads both) and records the run's totals; partition_top_scan_kernel (one CTA) turns the run totals into run starts, class
// c's run starting after all keys of the classes below it (st->less, st->eq).  A sub-tile's
// start is its run's start plus its start within the run.  (A single CTA stepping through all
// 4096-key tiles took 109-143 us for 65,536 tiles.)
constexpr int PART_SCAN_RUN = 1024;

template <int NT>
__device__ __forceinline__ void block_exclusive_scan3(const uint32_t (&v)[3], uint32_t (&excl)[3], uint32_t (&total)[3],
                                                      uint32_t (*wsum)[NT / 32]) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t incl[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    incl[c] = v[c];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl[c], o);
      if (lane >= o) incl[c] += y;
    }
    if (lane == 31) wsum[c][warp] = incl[c];
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 3; c++) {
    uint32_t before = 0, all = 0;
    for (int w = 0; w < NT / 32; w++) {
      const uint32_t x = wsum[c][w];
      before += w < warp ? x : 0u;
      all += x;
    }
    excl[c] = before + incl[c] - v[c];
    total[c] = all;
  }
  __syncthreads();  // wsum may be rewritten by a following call
}

static __global__ void __launch_bounds__(PART_SCAN_RUN) partition_block_scan_kernel(const uint32_t* sub_counts,
                                                                                   int64_t subs, uint32_t* sub_starts,
                                                                                   uint32_t* run_totals) {
  __shared__ uint32_t wsum[3][PART_SCAN_RUN / 32];
  const int64_t t = int64_t(blockIdx.x) * PART_SCAN_RUN + threadIdx.x;
  uint32_t v[3] = {0u, 0u, 0u}, excl[3], total[3];
  if (t < subs) {
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = sub_counts[t * 3 + c];
  }
  block_exclusive_scan3<PART_SCAN_RUN>(v, excl, total, wsum);
  if (t < subs) {
#pragma unroll
    for (int c = 0; c < 3; c++) sub_starts[t * 3 + c] = excl[c];
  }
  if (threadIdx.x < 3) run_totals[int64_t(blockIdx.x) * 3 + threadIdx.x] = total[threadIdx.x];
}

// One CTA over all runs, 1024 at a time with a carry.
static __global__ void __launch_bounds__(1024) partition_top_scan_kernel(uint32_t* run_totals, int64_t runs,
                                                                         const SelectState* st) {
  __shared__ uint32_t wsum[3][32];
  const uint32_t less = uint32_t(st->less), eq = uint32_t(st->eq);
  uint32_t carry[3] = {0u, less, less + eq};
  for (int64_t r0 = 0; r0 < runs; r0 += 1024) {
    const int64_t r = r0 + threadIdx.x;
    uint32_t v[3] = {0u, 0u, 0u}, excl[3], total[3];
    if (r < runs) {
#pragma unroll
      for (int c = 0; c < 3; c++) v[c] = run_totals[r * 3 + c];
    }
    block_exclusive_scan3<1024>(v, excl, total, wsum);
    if (r < runs) {
#pragma unroll
      for (int c = 0; c < 3; c++) run_totals[r * 3 + c] = carry[c] + excl[c];
    }
#pragma unroll
    for (int c = 0; c < 3; c++) carry[c] += total[c];
  }
}

template <class U, int KIND>
__global__ void __launch_bounds__(PART_NT) partition_scatter_kernel(const U* __restrict__ keys, int64_t n,
                                                                    const SelectState* st,
                                                                    const uint32_t* sub_counts,
                                                                    const uint32_t* sub_starts,
                                                                    const uint32_t* run_starts,
                                                                    U* __restrict__ out) {
  // staged slot j lives at j + j/32 of the warp's buffer
  __shared__ U s_k[PART_SUBS_PER_CTA][PART_SUB + PART_SUB / 32];
  const U v = U(st->prefix);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t sub = int64_t(blockIdx.x) * PART_SUBS_PER_CTA + warp;
  const int64_t base = sub * PART_SUB;
  if (base >= n) return;  // warp-uniform; nothing below waits on other warps
  const int sub_n = int(n - base < PART_SUB ? n - base : PART_SUB);
  const U* kin = keys + base;
  U k[PART_KPT];
  uint32_t cls[PART_KPT];
  if (sub_n == PART_SUB) {  // warp-uniform: full sub-tiles need no bounds
#pragma unroll
    for (int j = 0; j < PART_KPT; j++) {
      k[j] = kin[j * 32 + lane];
      cls[j] = uint32_t(part_class<U, KIND>(k[j], v));
    }
  } else {
#pragma unroll
    for (int j = 0; j < PART_KPT; j++) {
      const int i = j * 32 + lane;
      k[j] = i < sub_n ? kin[i] : U(0);
      cls[j] = i < sub_n ? uint32_t(part_class<U, KIND>(k[j], v)) : 3u;
    }
  }
  // the class runs of the staged sub-tile start at its class counts' prefix sums
  const uint32_t* sc = sub_counts + sub * 3;
  const uint32_t at1 = sc[0], at2 = sc[0] + sc[1];
  U* sw = s_k[warp];
  const uint32_t lt = lanemask_lt();
  uint32_t r0 = 0, r1 = at1, r2 = at2;  // next staged slot per class (uniform over the warp)
#pragma unroll
  for (int j = 0; j < PART_KPT; j++) {
    const uint32_t m0 = __ballot_sync(0xFFFFFFFFu, cls[j] == 0u);
    const uint32_t m1 = __ballot_sync(0xFFFFFFFFu, cls[j] == 1u);
    const uint32_t m2 = __ballot_sync(0xFFFFFFFFu, cls[j] == 2u);
    const uint32_t mine = cls[j] == 0u ? m0 : (cls[j] == 1u ? m1 : m2);
    const uint32_t run = cls[j] == 0u ? r0 : (cls[j] == 1u ? r1 : r2);
    const uint32_t slot = run + __popc(mine & lt);
    if (cls[j] < 3u) sw[slot + (slot >> 5)] = k[j];
    r0 += __popc(m0);
    r1 += __popc(m1);
    r2 += __popc(m2);
  }
  __syncwarp();
  // output positions fit 32 bits (n < 2^31)
  const uint32_t* ss = sub_starts + sub * 3;
  const uint32_t* rs = run_starts + (sub / PART_SCAN_RUN) * 3;
  const uint32_t o0 = rs[0] + ss[0], o1 = rs[1] + ss[1] - at1, o2 = rs[2] + ss[2] - at2;
  const uint32_t n32 = uint32_t(n);
  for (int j = lane; j < sub_n; j += 32) {
    const uint32_t uj = uint32_t(j);
    const uint32_t pos = (uj < at1 ? o0 : (uj < at2 ? o1 : o2)) + uj;
    if (pos < n32) out[pos] = sw[j + (j >> 5)];
  }
}

// ---- the k largest: keys > v compacted, then copies of v ------------------------------
// The keys above the level-0 bin are already in out (select_compact_kernel); this appends the
// candidates > v (the level-0 bin's keys) and fills the rest with copies of v.
template <class U, int KIND>
__global__ void __launch_bounds__(SEL_NT, SEL_CTAS_PER_SM) topk_gather_kernel(const U* __restrict__ cand, int64_t k,
                                                             SelectState* st, U* __restrict__ out) {
  using KO = KeyOrder<U, KIND>;
  constexpr int E = int(16 / sizeof(U));
  const U v = U(st->prefix);
  const int64_t n = st->n_total;
  int64_t greater = n - st->less - st->eq;
  greater = greater < 0 ? 0 : greater;  // never index below out[0]
  visit_keys<U, SEL_VPT>(cand, st->cand_count, [&](const U* kk, int nv) {
    uint32_t take = 0u;
#pragma unroll
    for (int e = 0; e < E; e++)
      if (e < nv && KO::to_ordered(kk[e]) > v) take |= 1u << e;
    warp_append<U, E>(kk, take, out, &st->gathered, k);
  });
  // copies of the selected key fill the rest (greater <= k by construction)
  const U vraw = KO::from_ordered(v);
  const int64_t stride = int64_t(gridDim.x) * SEL_NT;
  const int64_t gtid = int64_t(blockIdx.x) * SEL_NT + threadIdx.x;
  for (int64_t j = greater + gtid; j < k; j += stride) out[j] = vraw;
}

// ---- sort of a small top-k output in one CTA ------------------------------------------
// The k <= topk_small_sort_max<U>() outputs are sorted ascending by their ordered value in shared
// memory (a bitonic network over the next power of two, padded with the largest ordered value,
// so the padding sorts behind every key and only the first k slots are written back).  Keys
// with equal ordered values have equal bits, so the bytes equal the LSD sort's.
template <class U>
__host__ __device__ constexpr int topk_small_sort_max() {
  return sizeof(U) == 4 ? 8192 : 4096;  // 32 KiB of shared memory
}
constexpr int TOPK_SMALL_SORT_NT = 1024;

template <class U, int KIND>
__global__ void __launch_bounds__(TOPK_SMALL_SORT_NT) topk_small_sort_kernel(U* __restrict__ out, int k) {
  using KO = KeyOrder<U, KIND>;
  __shared__ U s[topk_small_sort_max<U>()];
  if (k <= 1) return;
  int N = 2;
  while (N < k) N <<= 1;
  for (int i = threadIdx.x; i < N; i += TOPK_SMALL_SORT_NT) s[i] = i < k ? KO::to_ordered(out[i]) : U(~U(0));
  __syncthreads();
  for (int size = 2; size <= N; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int p = threadIdx.x; p < (N >> 1); p += TOPK_SMALL_SORT_NT) {
        const int i = ((p & ~(stride - 1)) << 1) | (p & (stride - 1));  // lower element of the pair
        const int j = i + stride;
        const bool up = (i & size) == 0;
        const U a = s[i], b = s[j];
        if ((a > b) == up) {
          s[i] = b;
          s[j] = a;
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < k; i += TOPK_SMALL_SORT_NT) out[i] = KO::from_ordered(s[i]);
}

}  // namespace hpcs
