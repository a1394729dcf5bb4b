// Radix selection / top-k on the GPU.
//
// Restates the observable contract of HPCsharp's SelectTopK(this uint[] a, int k)
// (SelectionTopKRadix.cs:142-171): afterwards a[k] is the k-th smallest key (0-based) and
// a[k..n-1] holds exactly the multiset of the n-k largest.  The reference gets there with an
// in-place MSD radix select of 16-bit digits (RadixSelectionTopKWordInner, :96-133) whose
// movers clobber the prefix; here the prefix is defined too: a[0..k-1] holds the k smallest.
//
// Selection: an MSD radix select over the order-transformed key (the same transforms as the
// sort), 8 bits per level.  Level 0 histograms all n keys; the keys of the chosen bin are
// compacted into a candidate buffer (about n/256 of them for spread keys) and the remaining
// levels histogram only candidates that match the prefix chosen so far.  A one-block "pick"
// kernel after each histogram advances the device-side SelectState, so nothing returns to the
// host between levels.
//
// Rearrangement: a stable three-way partition (keys < v, == v, > v around the selected key v)
// in three kernels -- per-tile class counts, a one-block scan, a stable per-tile scatter.
// The k largest ("top-k" of a serving request) are the keys > v, compacted, plus copies of v
// up to k, then sorted ascending with the LSD sort so the output bytes are deterministic.
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
  unsigned long long gathered;  // keys > v written by topk_gather_kernel
  uint32_t hist[256];
};

static __global__ void select_init_kernel(SelectState* st, int64_t rank) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    st->prefix = 0;
    st->mask = 0;
    st->rank = rank;
    st->less = 0;
    st->eq = 0;
    st->cand_count = 0;
    st->gathered = 0;
  }
  if (tid < 256) st->hist[tid] = 0;
}

constexpr int SEL_NT = 512;
constexpr int SEL_COPIES = 32;

// Histogram of the digit at `shift` over keys whose ordered bits match (prefix, mask).
template <class U, int KIND>
__global__ void __launch_bounds__(SEL_NT) select_hist_kernel(const U* __restrict__ keys, const int64_t* n_ptr,
                                                             int64_t n_fixed, SelectState* st, int shift) {
  using KO = KeyOrder<U, KIND>;
  __shared__ uint32_t sh[256 * SEL_COPIES];
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < 256 * SEL_COPIES; i += SEL_NT) sh[i] = 0;
  __syncthreads();
  const int64_t n = n_ptr ? *n_ptr : n_fixed;
  const U prefix = U(st->prefix), mask = U(st->mask);
  const int64_t stride = int64_t(gridDim.x) * SEL_NT;
  for (int64_t i = int64_t(blockIdx.x) * SEL_NT + tid; i < n; i += stride) {
    const U o = KO::to_ordered(keys[i]);
    if ((o & mask) == prefix) atomicAdd(&sh[((uint32_t(o >> shift) & 0xFFu) * SEL_COPIES) + lane], 1u);
  }
  __syncthreads();
  for (int b = tid; b < 256; b += SEL_NT) {
    uint32_t c = 0;
    for (int q = 0; q < SEL_COPIES; q++) c += sh[b * SEL_COPIES + ((q + lane) & (SEL_COPIES - 1))];
    if (c) atomicAdd(&st->hist[b], c);
  }
}

// One block: choose the bin holding st->rank, advance the prefix, clear the histogram.
// last != 0: record how many keys equal the selected key.
template <class U>
__global__ void select_pick_kernel(SelectState* st, int shift, int last) {
  __shared__ uint32_t h[256];
  __shared__ int64_t cum[257];
  const int tid = threadIdx.x;
  if (tid < 256) h[tid] = st->hist[tid];
  __syncthreads();
  if (tid == 0) {
    int64_t run = 0;
    for (int b = 0; b < 256; b++) {
      cum[b] = run;
      run += h[b];
    }
    cum[256] = run;
    const int64_t r = st->rank;
    int bin = 255;
    for (int b = 0; b < 256; b++)
      if (r < cum[b + 1]) {
        bin = b;
        break;
      }
    st->prefix |= uint64_t(bin) << shift;
    st->mask |= uint64_t(0xFF) << shift;
    st->rank = r - cum[bin];
    st->less += cum[bin];
    if (last) st->eq = h[bin];
  }
  __syncthreads();
  if (tid < 256) st->hist[tid] = 0;
}

// Copies the keys whose ordered top byte matches the level-0 prefix into `cand`.
template <class U, int KIND>
__global__ void __launch_bounds__(SEL_NT) select_compact_kernel(const U* __restrict__ keys, int64_t n,
                                                                U* __restrict__ cand, SelectState* st) {
  using KO = KeyOrder<U, KIND>;
  const U prefix = U(st->prefix), mask = U(st->mask);
  const int lane = threadIdx.x & 31;
  const int64_t stride = int64_t(gridDim.x) * SEL_NT;
  // warp-uniform loop bounds: every lane reaches the ballot
  for (int64_t base = int64_t(blockIdx.x) * SEL_NT + (threadIdx.x - lane); base < n; base += stride) {
    const int64_t i = base + lane;
    U k = U(0);
    bool take = false;
    if (i < n) {
      k = keys[i];
      take = (KO::to_ordered(k) & mask) == prefix;
    }
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, take);
    if (bal == 0u) continue;
    unsigned long long slot = 0;
    if (lane == 0) slot = atomicAdd(reinterpret_cast<unsigned long long*>(&st->cand_count), (unsigned long long)__popc(bal));
    slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
    if (take) cand[slot + __popc(bal & lanemask_lt())] = k;
  }
}

// ---- stable three-way partition around the selected key -----------------------------
constexpr int PART_NT = 256, PART_KPT = 16, PART_TILE = PART_NT * PART_KPT;

template <class U, int KIND>
__device__ __forceinline__ int part_class(U k, U v_ordered) {
  const U o = KeyOrder<U, KIND>::to_ordered(k);
  return o < v_ordered ? 0 : (o == v_ordered ? 1 : 2);
}

template <class U, int KIND>
__global__ void __launch_bounds__(PART_NT) partition_count_kernel(const U* __restrict__ keys, int64_t n,
                                                                  const SelectState* st, uint32_t* tile_counts) {
  __shared__ uint32_t c[3];
  const U v = U(st->prefix);
  if (threadIdx.x < 3) c[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = int64_t(blockIdx.x) * PART_TILE;
  uint32_t l = 0, e = 0, g = 0;
  for (int i = threadIdx.x; i < PART_TILE; i += PART_NT) {
    const int64_t j = base + i;
    if (j < n) {
      const int cl = part_class<U, KIND>(keys[j], v);
      l += cl == 0;
      e += cl == 1;
      g += cl == 2;
    }
  }
  atomicAdd(&c[0], l);
  atomicAdd(&c[1], e);
  atomicAdd(&c[2], g);
  __syncthreads();
  if (threadIdx.x < 3) tile_counts[int64_t(blockIdx.x) * 3 + threadIdx.x] = c[threadIdx.x];
}

// One block: tile_counts[t][c] -> exclusive start of tile t's class-c keys in the output.
static __global__ void partition_scan_kernel(uint32_t* tile_counts, int64_t tiles, const SelectState* st, int64_t n) {
  __shared__ int64_t carry[3];
  __shared__ int64_t wsum[3][32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;  // 1024 threads
  if (tid < 3) {
    const int64_t less = st->less, eq = st->eq;
    carry[tid] = tid == 0 ? 0 : (tid == 1 ? less : less + eq);
  }
  __syncthreads();
  for (int64_t b0 = 0; b0 < tiles; b0 += 1024) {
    const int64_t t = b0 + tid;
    for (int c = 0; c < 3; c++) {
      const int64_t v = t < tiles ? int64_t(tile_counts[t * 3 + c]) : 0;
      int64_t incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) wsum[c][warp] = incl;
      __syncthreads();
      int64_t wb = 0;
      for (int w = 0; w < warp; w++) wb += wsum[c][w];
      if (t < tiles) tile_counts[t * 3 + c] = uint32_t(carry[c] + wb + incl - v);
      __syncthreads();
      if (tid == 1023) carry[c] += wb + incl;
      __syncthreads();
    }
  }
}

template <class U, int KIND>
__global__ void __launch_bounds__(PART_NT) partition_scatter_kernel(const U* __restrict__ keys, int64_t n,
                                                                    const SelectState* st,
                                                                    const uint32_t* tile_starts,
                                                                    U* __restrict__ out) {
  // Each thread takes PART_KPT consecutive keys (blocked), so a block scan of the per-thread
  // class counts gives stable positions.
  __shared__ uint32_t wsum[3][PART_NT / 32];
  const U v = U(st->prefix);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t base = int64_t(blockIdx.x) * PART_TILE + int64_t(tid) * PART_KPT;
  U k[PART_KPT];
  uint8_t cls[PART_KPT];
  uint32_t cnt[3] = {0, 0, 0};
#pragma unroll
  for (int i = 0; i < PART_KPT; i++) {
    const int64_t j = base + i;
    cls[i] = 3;
    if (j < n) {
      k[i] = keys[j];
      cls[i] = uint8_t(part_class<U, KIND>(k[i], v));
      cnt[cls[i]]++;
    }
  }
  uint32_t excl[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    uint32_t incl = cnt[c];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    excl[c] = incl - cnt[c];
    if (lane == 31) wsum[c][warp] = incl;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 3; c++) {
    uint32_t wb = 0;
    for (int w = 0; w < warp; w++) wb += wsum[c][w];
    excl[c] += wb + tile_starts[int64_t(blockIdx.x) * 3 + c];
  }
#pragma unroll
  for (int i = 0; i < PART_KPT; i++) {
    if (cls[i] < 3) {
      const uint32_t pos = excl[cls[i]]++;
      if (int64_t(pos) < n) out[pos] = k[i];
    }
  }
}

// ---- the k largest: keys > v compacted, then copies of v ------------------------------
template <class U, int KIND>
__global__ void __launch_bounds__(SEL_NT) topk_gather_kernel(const U* __restrict__ keys, int64_t n, int64_t k,
                                                             SelectState* st, U* __restrict__ out) {
  unsigned long long* counter = &st->gathered;
  using KO = KeyOrder<U, KIND>;
  const U v = U(st->prefix);
  int64_t greater = n - st->less - st->eq;
  greater = greater < 0 ? 0 : greater;  // never index below out[0]
  const int lane = threadIdx.x & 31;
  const int64_t stride = int64_t(gridDim.x) * SEL_NT;
  for (int64_t b = int64_t(blockIdx.x) * SEL_NT + (threadIdx.x - lane); b < n; b += stride) {
    const int64_t i = b + lane;
    U key = U(0);
    bool take = false;
    if (i < n) {
      key = keys[i];
      take = KO::to_ordered(key) > v;
    }
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, take);
    if (bal == 0u) continue;
    unsigned long long slot = 0;
    if (lane == 0) slot = atomicAdd(counter, (unsigned long long)__popc(bal));
    slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
    const unsigned long long pos = slot + __popc(bal & lanemask_lt());
    if (take && int64_t(pos) < k) out[pos] = key;
  }
  // copies of the selected key fill the rest (greater <= k by construction)
  const U vraw = KO::from_ordered(v);
  const int64_t gtid = int64_t(blockIdx.x) * SEL_NT + threadIdx.x;
  for (int64_t j = greater + gtid; j < k; j += stride) out[j] = vraw;
}

}  // namespace hpcs
