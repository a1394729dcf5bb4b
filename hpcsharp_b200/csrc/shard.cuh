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
// among the same part's keys of its warp comes from one ballot per bit of the part index,
// and the tile-wide rank from a scan of the per-(row, warp) counts per part.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace hpcs {

constexpr int SHARD_NT = 256;
constexpr int SHARD_COUNT_NT = 256;
constexpr int SHARD_KPT = 8;  // keys per thread per tile (rows of SHARD_NT keys)
constexpr int SHARD_NW = SHARD_NT / 32;
constexpr int SHARD_SUB = SHARD_KPT * SHARD_NW;  // (row, warp) sub-tiles per tile, in key order
constexpr int SHARD_TILE = SHARD_NT * SHARD_KPT;
constexpr int SHARD_MAX_PARTS = 64;

// Resident CTAs per SM the scatter kernel is built for (its register budget); the grid is
// this many CTAs per SM, and the count kernel uses the same ranges.
template <class U, bool ITEMS>
__host__ __device__ constexpr int shard_ctas_per_sm() {
  return sizeof(U) == 4 && !ITEMS ? 4 : 3;
}

template <class U>
struct ShardSplit {
  U key[SHARD_MAX_PARTS];         // ordered keys of the splitters
  int64_t gpos[SHARD_MAX_PARTS];  // their global positions
};

// Splitters into shared memory, their keys ordered; entries from parts-1 up to the array's
// end hold the largest ordered key, so a search over 2^LOG - 1 entries never counts them.
template <class U, int KIND>
__device__ __forceinline__ void shard_load_splitters(ShardSplit<U>& sp, const U* split_keys,
                                                     const int64_t* split_gpos, int parts) {
  for (int j = threadIdx.x; j < SHARD_MAX_PARTS; j += blockDim.x) {
    sp.key[j] = j < parts - 1 ? KeyOrder<U, KIND>::to_ordered(split_keys[j]) : U(~U(0));
    sp.gpos[j] = j < parts - 1 ? split_gpos[j] : INT64_MAX;
  }
}

// Number of splitters at or below (ok, g): the part of an element with ordered key ok.  A
// branchless search over 2^LOG - 1 keys counts the splitters whose key is below ok; the
// splitters whose key equals ok follow in ascending position, and the (rarely entered) loop
// counts those at or below g = gbase + i (formed only there).  m = parts - 1 <= 2^LOG - 1.
template <class U, int LOG>
__device__ __forceinline__ int shard_part_of(const ShardSplit<U>& sp, int m, U ok, int64_t gbase, int i) {
  int pos = 0;
#pragma unroll
  for (int l = LOG - 1; l >= 0; l--)
    if (sp.key[pos + (1 << l) - 1] < ok) pos += 1 << l;
  if (pos < m && sp.key[pos] == ok) {
    const int64_t g = gbase + i;
    while (pos < m && sp.key[pos] == ok && sp.gpos[pos] <= g) pos++;
  }
  return pos;
}

// Lanes of the warp whose part equals b: one ballot per bit of the part index, NB bits
// (LOG for parts < 2^LOG only; LOG + 1 when the value parts marks an out-of-range key).
template <int NB>
__device__ __forceinline__ uint32_t shard_peers(int b) {
  uint32_t peers = 0xFFFFFFFFu;
#pragma unroll
  for (int j = 0; j < NB; j++) {
    const uint32_t bit = (uint32_t(b) >> j) & 1u;
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, bit);
    peers &= bit ? bal : ~bal;
  }
  return peers;
}

// Pass 1: counts[cta][part] of the CTA's range [cta * per_cta, min(n, (cta + 1) * per_cta)),
// indexed in 32 bits inside the range (per_cta < 2^31).  Up to 8 parts (LOG <= 3) each thread
// counts in bytes of two registers (part b in byte b % 4 of register b / 4) and the warp adds
// them up every 31 tiles (at most 248 keys per thread, so no byte overflows); more parts use
// one ballot per bit of the part index and the leader of each part's lanes adds their number.
template <class U, int KIND, int LOG>
__global__ void __launch_bounds__(SHARD_COUNT_NT, 4) shard_count_kernel(const U* __restrict__ keys, int64_t n,
                                                                     int64_t per_cta, int64_t gpos0,
                                                                     const U* __restrict__ split_keys,
                                                                     const int64_t* __restrict__ split_gpos,
                                                                     int parts, uint32_t* __restrict__ cta_counts) {
  constexpr int NT = SHARD_COUNT_NT, NW = NT / 32, TILE = NT * SHARD_KPT;
  constexpr bool PACKED = LOG <= 3;
  __shared__ ShardSplit<U> sp;
  __shared__ uint32_t s_cnt[NW][SHARD_MAX_PARTS];  // per warp, so warps never contend
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  shard_load_splitters<U, KIND>(sp, split_keys, split_gpos, parts);
  for (int i = tid; i < NW * SHARD_MAX_PARTS; i += NT) (&s_cnt[0][0])[i] = 0u;
  __syncthreads();
  const int64_t begin = int64_t(blockIdx.x) * per_cta;
  const int len = begin < n ? int((begin + per_cta < n ? begin + per_cta : n) - begin) : 0;
  const U* kr = keys + begin;
  const int64_t gbase = gpos0 + begin;
  uint32_t c0 = 0u, c1 = 0u;  // packed byte counters (PACKED)
  auto flush = [&]() {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if (j < parts) {
        const uint32_t v = ((j < 4 ? c0 : c1) >> (8 * (j & 3))) & 0xFFu;
        const uint32_t sum = __reduce_add_sync(0xFFFFFFFFu, v);
        if (lane == 0) s_cnt[warp][j] += sum;
      }
    }
    c0 = c1 = 0u;
  };
  int since = 0;
  for (int t = 0; t < len; t += TILE) {  // uniform trip count in the CTA
    const bool full = t + TILE <= len;
    U k[SHARD_KPT];
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      const int i = t + r * NT + tid;
      k[r] = full || i < len ? kr[i] : U(0);
    }
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      const int i = t + r * NT + tid;
      const bool valid = full || i < len;
      const int b = valid ? shard_part_of<U, LOG>(sp, parts - 1, KeyOrder<U, KIND>::to_ordered(k[r]), gbase, i)
                          : parts;
      if (PACKED) {
        const uint32_t inc = valid ? 1u << (8 * (b & 3)) : 0u;
        if (b < 4) c0 += inc;
        else c1 += inc;
      } else {
        const uint32_t peers = shard_peers<LOG + 1>(b);
        if (b < parts && (peers & lanemask_lt()) == 0u) atomicAdd(&s_cnt[warp][b], uint32_t(__popc(peers)));
      }
    }
    if (PACKED && ++since == 31) {
      flush();
      since = 0;
    }
  }
  if (PACKED) flush();
  __syncthreads();
  for (int p = tid; p < parts; p += NT) {
    uint32_t c = 0;
    for (int w = 0; w < NW; w++) c += s_cnt[w][p];
    cta_counts[int64_t(blockIdx.x) * parts + p] = c;
  }
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

// Pass 2: stable scatter of the CTA's range to its parts.  Per tile of SHARD_TILE keys at
// offset t of the range (row r of SHARD_NT keys holds keys t + r*SHARD_NT + tid, so sub-tile
// (r, warp) = r*NW + warp is in key order):
//   count:   each key's part; its rank among the same part's keys of its warp (ballots);
//            the leader stores the (sub-tile, part) count;
//   scan:    warp w scans parts w, w + NW, ...: the (sub-tile, part) base inside the part's
//            run of the tile, the run's length and its global base from the running offset,
//            and clears the counts; then warp 0 scans the run lengths over the parts;
//   stage:   each key (and item, and its part) goes to shared memory in part order;
//   write:   consecutive threads write consecutive staged keys, so each part's run of the
//            tile leaves as contiguous, coalesced stores.
// Dynamic shared memory (shard_scatter_smem): staged keys, counts and bases (SHARD_SUB x
// parts u32 each), staged items, staged parts.
template <class U, bool ITEMS>
__host__ __device__ constexpr size_t shard_scatter_smem(int parts) {
  return size_t(SHARD_TILE) * sizeof(U) + size_t(2) * SHARD_SUB * parts * 4 + (ITEMS ? size_t(SHARD_TILE) * 4 : 0) +
         size_t(SHARD_TILE);
}

template <class U, int KIND, bool ITEMS, int LOG>
__global__ void __launch_bounds__(SHARD_NT, (shard_ctas_per_sm<U, ITEMS>())) shard_scatter_kernel(
    const U* __restrict__ keys, const uint32_t* __restrict__ items, int64_t n, int64_t per_cta, int64_t gpos0,
    const U* __restrict__ split_keys, const int64_t* __restrict__ split_gpos, int parts,
    const int64_t* __restrict__ cta_offsets, U* __restrict__ keys_out, uint32_t* __restrict__ items_out) {
  __shared__ ShardSplit<U> sp;
  __shared__ int64_t s_run[SHARD_MAX_PARTS];   // global offset of each part's next key
  __shared__ int64_t s_tile[SHARD_MAX_PARTS];  // global base of each part's run in this tile
  __shared__ uint32_t s_len[SHARD_MAX_PARTS];  // length of each part's run in this tile
  __shared__ uint32_t s_at[SHARD_MAX_PARTS];   // start of each part's run in the staged tile
  __shared__ uint32_t s_out[SHARD_MAX_PARTS];  // s_tile - s_at (mod 2^32): output index of staged slot 0
  extern __shared__ __align__(16) unsigned char s_raw[];
  U* stage_k = reinterpret_cast<U*>(s_raw);
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(s_raw + size_t(SHARD_TILE) * sizeof(U));  // [SHARD_SUB][parts]
  uint32_t* s_sub = s_cnt + SHARD_SUB * parts;                                            // [SHARD_SUB][parts]
  uint32_t* stage_v = s_sub + SHARD_SUB * parts;
  uint8_t* stage_p = reinterpret_cast<uint8_t*>(stage_v + (ITEMS ? SHARD_TILE : 0));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  shard_load_splitters<U, KIND>(sp, split_keys, split_gpos, parts);
  if (tid < parts) s_run[tid] = cta_offsets[int64_t(blockIdx.x) * parts + tid];
  for (int i = tid; i < SHARD_SUB * parts; i += SHARD_NT) s_cnt[i] = 0u;
  __syncthreads();
  const int64_t begin = int64_t(blockIdx.x) * per_cta;
  const int len = begin < n ? int((begin + per_cta < n ? begin + per_cta : n) - begin) : 0;
  const U* kr = keys + begin;
  const uint32_t* vr = ITEMS ? items + begin : nullptr;
  const int64_t gbase = gpos0 + begin;
  constexpr int SPL = SHARD_SUB / 32;  // sub-tiles per lane in the scan
  static_assert(SHARD_SUB % 32 == 0, "sub-tiles must fill whole lanes");
  static_assert(SHARD_MAX_PARTS <= 64, "the run scan covers two parts per lane");
  // the keys (and items) of the next tile are loaded while this tile is ranked and written
  U k[SHARD_KPT];
  uint32_t v[SHARD_KPT];
#pragma unroll
  for (int r = 0; r < SHARD_KPT; r++) {
    const int i = r * SHARD_NT + tid;
    k[r] = i < len ? kr[i] : U(0);
    if (ITEMS) v[r] = i < len ? vr[i] : 0u;
  }
  for (int t = 0; t < len; t += SHARD_TILE) {
    const bool full = t + SHARD_TILE <= len;
    U kn[SHARD_KPT];
    uint32_t vn[SHARD_KPT];
    int b[SHARD_KPT];
    int rk[SHARD_KPT];
    if (t + 2 * SHARD_TILE <= len) {  // the next tile is whole (uniform over the CTA)
#pragma unroll
      for (int r = 0; r < SHARD_KPT; r++) {
        const int i = t + SHARD_TILE + r * SHARD_NT + tid;
        kn[r] = kr[i];
        if (ITEMS) vn[r] = vr[i];
      }
    } else {
#pragma unroll
      for (int r = 0; r < SHARD_KPT; r++) {
        const int i = t + SHARD_TILE + r * SHARD_NT + tid;
        kn[r] = i < len ? kr[i] : U(0);
        if (ITEMS) vn[r] = i < len ? vr[i] : 0u;
      }
    }
    if (full) {  // every key of the tile is in range: LOG ballots
#pragma unroll
      for (int r = 0; r < SHARD_KPT; r++) {
        const int i = t + r * SHARD_NT + tid;
        b[r] = shard_part_of<U, LOG>(sp, parts - 1, KeyOrder<U, KIND>::to_ordered(k[r]), gbase, i);
        const uint32_t peers = shard_peers<LOG>(b[r]);
        rk[r] = __popc(peers & lanemask_lt());
        if (rk[r] == 0) s_cnt[(r * SHARD_NW + warp) * parts + b[r]] = __popc(peers);
      }
    } else {
#pragma unroll
      for (int r = 0; r < SHARD_KPT; r++) {
        const int i = t + r * SHARD_NT + tid;
        b[r] = i < len ? shard_part_of<U, LOG>(sp, parts - 1, KeyOrder<U, KIND>::to_ordered(k[r]), gbase, i)
                       : parts;
        const uint32_t peers = shard_peers<LOG + 1>(b[r]);
        rk[r] = __popc(peers & lanemask_lt());
        if (b[r] < parts && rk[r] == 0) s_cnt[(r * SHARD_NW + warp) * parts + b[r]] = __popc(peers);
      }
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
        s_len[p] = total;
        s_tile[p] = s_run[p];
        s_run[p] += total;
      }
    }
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the run lengths over the parts (two parts per lane)
      const uint32_t a = lane < parts ? s_len[lane] : 0u;
      const uint32_t c = lane + 32 < parts ? s_len[lane + 32] : 0u;
      uint32_t ia = a, ic = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t ya = __shfl_up_sync(0xFFFFFFFFu, ia, o);
        const uint32_t yc = __shfl_up_sync(0xFFFFFFFFu, ic, o);
        if (lane >= o) {
          ia += ya;
          ic += yc;
        }
      }
      const uint32_t first_half = __shfl_sync(0xFFFFFFFFu, ia, 31);
      if (lane < parts) {
        s_at[lane] = ia - a;
        s_out[lane] = uint32_t(s_tile[lane]) - (ia - a);
      }
      if (lane + 32 < parts) {
        s_at[lane + 32] = first_half + ic - c;
        s_out[lane + 32] = uint32_t(s_tile[lane + 32]) - (first_half + ic - c);
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      if (b[r] < parts) {
        const uint32_t j = s_at[b[r]] + s_sub[(r * SHARD_NW + warp) * parts + b[r]] + uint32_t(rk[r]);
        stage_k[j] = k[r];
        if (ITEMS) stage_v[j] = v[r];
        stage_p[j] = uint8_t(b[r]);
      }
    }
    __syncthreads();
    const int cnt = len - t < SHARD_TILE ? len - t : SHARD_TILE;
    for (int j = tid; j < cnt; j += SHARD_NT) {
      const uint32_t pos = s_out[stage_p[j]] + uint32_t(j);  // shards hold fewer than 2^31 keys
      keys_out[pos] = stage_k[j];
      if (ITEMS) items_out[pos] = stage_v[j];
    }
#pragma unroll
    for (int r = 0; r < SHARD_KPT; r++) {
      k[r] = kn[r];
      if (ITEMS) v[r] = vn[r];
    }
    // everything the next tile rewrites (counts, bases, run starts, staged keys) is written
    // only after the barrier that follows its count step, which every thread reaches after
    // this write-out
  }
}

}  // namespace hpcs
