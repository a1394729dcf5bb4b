// Partition step of the sort of one array spread over ranks (one process per GPU).  HPCsharp
// sorts one array per process (RadixSortLsdParallel.cs:49-232 splits it across host threads,
// never across machines); the sharded form keeps its result: the concatenation of the ranks'
// outputs is the stable LSD sort of the concatenation of their inputs.
//
// Each rank partitions its shard by parts-1 splitters, sends part b to rank b (NCCL
// all-to-all over NVLink), and sorts what it received with the plain sort.  Element i of a
// shard has global position gpos0 + i; the splitters are (key, global position) pairs taken
// from the keys themselves, compared in (radix order of key, position) order, which is a
// total order.  Element (k, g) goes to part b = the number of splitters at or below (k, g),
// so a run of equal keys may be split between parts, and every part's size is set by the
// splitter positions alone, however many keys repeat.  The partition is stable (a part keeps
// its shard order), the exchange concatenates parts in rank order, and the local sort is
// stable, so equal keys leave in global position order.
//
// Two passes over the shard: a count of each CTA's contiguous range per part, an exclusive
// scan of the counts (part-major, CTA-minor), and a scatter that re-reads the range and
// writes each key to its part at the CTA's running offset.  Inside a tile the rank of a key
// among the same part's keys comes from __match_any_sync per warp and a scan of the
// per-(row, warp) counts per part.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace hpcs {

constexpr int SHARD_NT = 256;
constexpr int SHARD_KPT = 8;  // keys per thread per tile (rows of SHARD_NT keys)
constexpr int SHARD_NW = SHARD_NT / 32;
constexpr int SHARD_SUB = SHARD_KPT * SHARD_NW;  // (row, warp) sub-tiles per tile, in key order
constexpr int SHARD_TILE = SHARD_NT * SHARD_KPT;
constexpr int SHARD_MAX_PARTS = 64;

template <class U>
struct ShardSplit {
  U key[SHARD_MAX_PARTS];         // ordered keys of the splitters
  int64_t gpos[SHARD_MAX_PARTS];  // their global positions
};

template <class U, int KIND>
__device__ __forceinline__ void shard_load_splitters(ShardSplit<U>& sp, const U* split_keys,
                                                     const int64_t* split_gpos, int parts) {
  for (int j = threadIdx.x; j < parts - 1; j += blockDim.x) {
    sp.key[j] = KeyOrder<U, KIND>::to_ordered(split_keys[j]);
    sp.gpos[j] = split_gpos[j];
  }
}

// Number of splitters at or below (ok, g): the part of an element with ordered key ok.
template <class U>
__device__ __forceinline__ int shard_part_of(const ShardSplit<U>& sp, int m, U ok, int64_t g) {
  int lo = 0, hi = m;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const U sk = sp.key[mid];
    if (sk < ok || (sk == ok && sp.gpos[mid] <= g)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Pass 1: counts[cta][part] of the CTA's range [cta * per_cta, min(n, (cta + 1) * per_cta)).
template <class U, int KIND>
__global__ void __launch_bounds__(SHARD_NT) shard_count_kernel(const U* __restrict__ keys, int64_t n, int64_t per_cta,
                                                               int64_t gpos0, const U* __restrict__ split_keys,
                                                               const int64_t* __restrict__ split_gpos, int parts,
                                                               uint32_t* __restrict__ cta_counts) {
  __shared__ ShardSplit<U> sp;
  __shared__ uint32_t s_cnt[SHARD_MAX_PARTS];
  const int tid = threadIdx.x, lane = tid & 31;
  shard_load_splitters<U, KIND>(sp, split_keys, split_gpos, parts);
  if (tid < parts) s_cnt[tid] = 0u;
  __syncthreads();
  const int64_t begin = int64_t(blockIdx.x) * per_cta;
  const int64_t end = begin + per_cta < n ? begin + per_cta : n;
  for (int64_t t0 = begin; t0 < end; t0 += SHARD_TILE) {  // uniform trip count in the CTA
    U k[SHARD_KPT];
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      const int64_t i = t0 + int64_t(r) * SHARD_NT + tid;
      k[r] = i < end ? keys[i] : U(0);
    }
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      const int64_t i = t0 + int64_t(r) * SHARD_NT + tid;
      const int b = i < end ? shard_part_of<U>(sp, parts - 1, KeyOrder<U, KIND>::to_ordered(k[r]), gpos0 + i) : parts;
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
      if (b < parts && (__ffs(peers) - 1) == lane) atomicAdd(&s_cnt[b], uint32_t(__popc(peers)));
    }
  }
  __syncthreads();
  if (tid < parts) cta_counts[int64_t(blockIdx.x) * parts + tid] = s_cnt[tid];
}

// Exclusive offsets, part-major then CTA order: cta_offsets[c][b] = sum of all keys of parts
// below b + keys of part b in CTAs below c; counts_out[b] = keys of part b.  One CTA.
__global__ void __launch_bounds__(1024) shard_scan_kernel(const uint32_t* __restrict__ cta_counts, int grid, int parts,
                                                          int64_t* __restrict__ cta_offsets,
                                                          int64_t* __restrict__ counts_out) {
  __shared__ int64_t s_tot[SHARD_MAX_PARTS];
  __shared__ int64_t s_base[SHARD_MAX_PARTS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int b = warp; b < parts; b += nw) {
    int64_t run = 0;
    for (int c0 = 0; c0 < grid; c0 += 32) {
      const int c = c0 + lane;
      const int64_t v = c < grid ? int64_t(cta_counts[int64_t(c) * parts + b]) : 0;
      int64_t incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      if (c < grid) cta_offsets[int64_t(c) * parts + b] = run + incl - v;
      run += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    if (lane == 0) s_tot[b] = run;
  }
  __syncthreads();
  if (tid == 0) {
    int64_t base = 0;
    for (int b = 0; b < parts; b++) {
      s_base[b] = base;
      counts_out[b] = s_tot[b];
      base += s_tot[b];
    }
  }
  __syncthreads();
  for (int64_t i = tid; i < int64_t(grid) * parts; i += blockDim.x) cta_offsets[i] += s_base[i % parts];
}

// Pass 2: stable scatter of the CTA's range to its parts.  Per tile of SHARD_TILE keys (row r
// of SHARD_NT keys holds keys t0 + r*SHARD_NT + tid, so sub-tile (r, warp) = r*NW + warp is in
// key order):
//   count:   each key's part; its rank among the same part's keys of its warp (match_any);
//            the leader stores the (sub-tile, part) count;
//   scan:    warp w scans parts w, w + NW, ...: the (sub-tile, part) base inside the tile, the
//            tile's base of each part from the running offset, and clears the counts;
//   scatter: out[tile base + sub-tile base + rank] = key (and item).
// Dynamic shared memory: counts and bases, SHARD_SUB x parts u32 each.
template <class U, int KIND, bool ITEMS>
__global__ void __launch_bounds__(SHARD_NT) shard_scatter_kernel(
    const U* __restrict__ keys, const uint32_t* __restrict__ items, int64_t n, int64_t per_cta, int64_t gpos0,
    const U* __restrict__ split_keys, const int64_t* __restrict__ split_gpos, int parts,
    const int64_t* __restrict__ cta_offsets, U* __restrict__ keys_out, uint32_t* __restrict__ items_out) {
  __shared__ ShardSplit<U> sp;
  __shared__ int64_t s_run[SHARD_MAX_PARTS];
  __shared__ int64_t s_tile[SHARD_MAX_PARTS];
  extern __shared__ __align__(16) uint32_t s_dyn[];
  uint32_t* s_cnt = s_dyn;                      // [SHARD_SUB][parts]
  uint32_t* s_sub = s_dyn + SHARD_SUB * parts;  // [SHARD_SUB][parts]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  shard_load_splitters<U, KIND>(sp, split_keys, split_gpos, parts);
  if (tid < parts) s_run[tid] = cta_offsets[int64_t(blockIdx.x) * parts + tid];
  for (int i = tid; i < SHARD_SUB * parts; i += SHARD_NT) s_cnt[i] = 0u;
  __syncthreads();
  const int64_t begin = int64_t(blockIdx.x) * per_cta;
  const int64_t end = begin + per_cta < n ? begin + per_cta : n;
  constexpr int SPL = SHARD_SUB / 32;  // sub-tiles per lane in the scan
  static_assert(SHARD_SUB % 32 == 0, "sub-tiles must fill whole lanes");
  for (int64_t t0 = begin; t0 < end; t0 += SHARD_TILE) {
    U k[SHARD_KPT];
    uint32_t v[SHARD_KPT];
    int b[SHARD_KPT];
    int rk[SHARD_KPT];
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      const int64_t i = t0 + int64_t(r) * SHARD_NT + tid;
      k[r] = i < end ? keys[i] : U(0);
      if (ITEMS) v[r] = i < end ? items[i] : 0u;
    }
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      const int64_t i = t0 + int64_t(r) * SHARD_NT + tid;
      b[r] = i < end ? shard_part_of<U>(sp, parts - 1, KeyOrder<U, KIND>::to_ordered(k[r]), gpos0 + i) : parts;
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b[r]);
      rk[r] = __popc(peers & lanemask_lt());
      if (b[r] < parts && (__ffs(peers) - 1) == lane) s_cnt[(r * SHARD_NW + warp) * parts + b[r]] = __popc(peers);
    }
    __syncthreads();
    for (int p = warp; p < parts; p += SHARD_NW) {
      uint32_t c[SPL];
      uint32_t sum = 0;
#pragma unroll
      for (int j = 0; j < SPL; j++) {
        const int idx = (lane * SPL + j) * parts + p;
        c[j] = s_cnt[idx];
        s_cnt[idx] = 0u;
        sum += c[j];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      uint32_t run = incl - sum;
#pragma unroll
      for (int j = 0; j < SPL; j++) {
        s_sub[(lane * SPL + j) * parts + p] = run;
        run += c[j];
      }
      const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
      if (lane == 0) {
        s_tile[p] = s_run[p];
        s_run[p] += total;
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      if (b[r] < parts) {
        const int64_t pos = s_tile[b[r]] + s_sub[(r * SHARD_NW + warp) * parts + b[r]] + rk[r];
        keys_out[pos] = k[r];
        if (ITEMS) items_out[pos] = v[r];
      }
    }
    // s_tile and s_sub are rewritten by the next tile's scan only after the barrier that
    // follows its count step, which every thread reaches after this scatter
  }
}

}  // namespace hpcs
