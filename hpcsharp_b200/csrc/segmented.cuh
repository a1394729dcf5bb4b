// Batched segmented LSD sort: thousands of independent arrays of mixed length and dtype in
// one persistent launch.
//
// No reference counterpart (HPCsharp sorts one array per call); it is the batched form of
// the same stable LSD sort, with identical per-array results.
//
// One CTA owns one segment at a time (segments are taken from a device-side queue, largest
// first, so the long ones start early).  Because a digit histogram does not depend on the
// order of the keys, the CTA reads its segment once to histogram every digit, then runs each
// 8-bit pass tile by tile with running per-digit offsets: tiles of one segment are processed
// in order by one CTA, so no look-back between CTAs is needed and every pass is one read and
// one write (the onesweep's 36 B/key for 32-bit keys).  Segments that fit in one tile are
// sorted entirely in shared memory: one global read, all passes in shared memory, one
// global write.  Ranking is the sort's in-warp ranking (ordered shared atomics after the
// lane-order probe, or the peer-mask ranking).
#pragma once
#include <cstdint>
#include <type_traits>

#include "common.cuh"
#include "radix_kernels.cuh"

namespace hpcs {

// Device-resident segment descriptor.
struct SegDesc {
  void* keys;     // device pointer, sorted in place
  void* scratch;  // device scratch of the same size (segments larger than one tile)
  int64_t n;
  int32_t dtype;  // hpcs_dtype
  int32_t pad;
};

struct SegParams {
  const SegDesc* segs;
  int nsegs;
  uint32_t* queue;  // next segment index (zeroed before each launch)
  uint32_t* err;    // device error bits
  uint64_t spin_limit_ns;  // bound on the bulk-copy waits
};

template <int NT, int KPT, int MODE>
struct SegSmem {
  static constexpr int NW = NT / 32;
  static constexpr int TILE_BYTES = NT * KPT * 4;  // u32 keys per tile = NT*KPT; u64 = half
  static constexpr size_t OFF_BUF = 0;             // [2][TILE_BYTES]
  static constexpr size_t OFF_CNT = OFF_BUF + 2 * size_t(TILE_BYTES);
  static constexpr size_t OFF_MSK = OFF_CNT + size_t(NW) * RADIX * 4;
  static constexpr size_t MSK_BYTES = MODE == RANK_PEER_MASK ? size_t(NW) * 2 * RADIX * 4 : 0;
  static constexpr size_t OFF_HIST = OFF_MSK + MSK_BYTES;  // [8][256]
  static constexpr size_t OFF_RUN = OFF_HIST + 8 * RADIX * 4;
  static constexpr size_t OFF_LOCAL = OFF_RUN + RADIX * 4;
  static constexpr size_t OFF_GBASE = OFF_LOCAL + RADIX * 4;
  static constexpr size_t OFF_WSUM = OFF_GBASE + RADIX * 4;
  static constexpr size_t OFF_SEG = OFF_WSUM + 32 * 4;
  static constexpr size_t OFF_MBAR = (OFF_SEG + 16 + 7) / 8 * 8;  // [2] bulk-copy barriers
  static constexpr size_t BYTES = OFF_MBAR + 16;
};

// Ranks one tile of keys held warp-striped in registers (key i of lane l = tile position
// w*32*KPT + i*32 + l) by digit `shift`, turns the warp counters into tile positions and
// leaves the tile-local digit starts in s_local and the per-digit totals computable as
// s_local[d+1]-s_local[d].  Returns each key's tile position in pos[].
template <class U, int KIND, int NT, int KPT, int MODE>
__device__ __forceinline__ void seg_rank_tile(const U (&key)[KPT], int tile_n, int shift, uint32_t* s_cnt,
                                              uint32_t* s_msk, uint32_t* s_local, uint32_t* s_wsum,
                                              uint32_t (&pos)[KPT]) {
  using KO = KeyOrder<U, KIND>;
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* cnt_w = s_cnt + warp * RADIX;
  for (int i = lane; i < RADIX; i += 32) cnt_w[i] = 0u;
  __syncwarp();
  const int wbase = warp * 32 * KPT;
#pragma unroll
  for (int i = 0; i < KPT; i++) {
    const bool valid = wbase + i * 32 + lane < tile_n;
    pos[i] = rank_in_warp<MODE>(cnt_w, s_msk + warp * 2 * RADIX, KO::digit(key[i], shift), valid, i & 1, lane);
  }
  __syncthreads();
  if (tid < RADIX) {
    const int dg = tid;
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) total += s_cnt[w * RADIX + dg];
    uint32_t incl = total;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    s_local[dg] = incl - total;
    if (lane == 31) s_wsum[warp] = incl;
  }
  __syncthreads();
  if (tid < RADIX) {
    const int dg = tid;
    uint32_t base = 0;
#pragma unroll
    for (int w = 0; w < RADIX / 32; w++) base += (w < warp) ? s_wsum[w] : 0u;
    const uint32_t local = base + s_local[dg];
    s_local[dg] = local;
    uint32_t run = local;
#pragma unroll
    for (int w = 0; w < NW; w++) {
      const uint32_t c = s_cnt[w * RADIX + dg];
      s_cnt[w * RADIX + dg] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < KPT; i++) {
    if (wbase + i * 32 + lane < tile_n) pos[i] += cnt_w[KO::digit(key[i], shift)];
  }
}

// A segment that fits in one tile: one global read, every pass in shared memory, one write.
template <class U, int KIND, int NT, int KPT, int MODE>
__device__ void seg_sort_small(U* keys, int n, unsigned char* smem) {
  using L = SegSmem<NT, KPT * int(sizeof(U)) / 4, MODE>;
  constexpr int P = int(sizeof(U));
  U* buf0 = reinterpret_cast<U*>(smem + L::OFF_BUF);
  U* buf1 = reinterpret_cast<U*>(smem + L::OFF_BUF + L::TILE_BYTES);
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + L::OFF_CNT);
  uint32_t* s_msk = reinterpret_cast<uint32_t*>(smem + L::OFF_MSK);
  uint32_t* s_local = reinterpret_cast<uint32_t*>(smem + L::OFF_LOCAL);
  uint32_t* s_wsum = reinterpret_cast<uint32_t*>(smem + L::OFF_WSUM);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wbase = warp * 32 * KPT;
  U key[KPT];
  uint32_t pos[KPT];
#pragma unroll
  for (int i = 0; i < KPT; i++) {
    const int idx = wbase + i * 32 + lane;
    key[i] = idx < n ? keys[idx] : U(0);
  }
  U* src = buf0;
  U* dst = buf1;
  for (int p = 0; p < P; p++) {
    if (p > 0) {
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int idx = wbase + i * 32 + lane;
        key[i] = idx < n ? src[idx] : U(0);
      }
    }
    seg_rank_tile<U, KIND, NT, KPT, MODE>(key, n, 8 * p, s_cnt, s_msk, s_local, s_wsum, pos);
#pragma unroll
    for (int i = 0; i < KPT; i++)
      if (wbase + i * 32 + lane < n) dst[pos[i]] = key[i];
    __syncthreads();
    U* t = src;
    src = dst;
    dst = t;
  }
  for (int i = tid; i < n; i += NT) keys[i] = src[i];
  __syncthreads();
}

// A segment larger than one tile: histogram every digit in one read, then per pass the
// tiles in order with running per-digit offsets (ping-pong with the segment's scratch).
// When the segment spans at least 8 tiles and its keys are 16-byte aligned, each tile is
// staged by a 1-D bulk async copy into one of the two tile buffers, issued two tiles ahead,
// so the next tile's load overlaps this tile's ranking and scatter; the ragged tail under 16
// bytes is read with plain loads.  (Shorter segments were measured faster with plain loads:
// the copies' barriers and proxy fences cost more than the latency they hide.)
// `phase` carries the two mbarriers' expected parities across the segments a CTA sorts.
template <class U, int KIND, int NT, int KPT, int MODE>
__device__ void seg_sort_large(U* keys, U* scratch, int64_t n, unsigned char* smem, uint32_t* err,
                               uint64_t spin_limit_ns, uint32_t& phase) {
  using KO = KeyOrder<U, KIND>;
  using L = SegSmem<NT, KPT * int(sizeof(U)) / 4, MODE>;
  constexpr int P = int(sizeof(U));
  constexpr int TILE = NT * KPT;
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + L::OFF_CNT);
  uint32_t* s_msk = reinterpret_cast<uint32_t*>(smem + L::OFF_MSK);
  uint32_t* s_hist = reinterpret_cast<uint32_t*>(smem + L::OFF_HIST);
  uint32_t* s_run = reinterpret_cast<uint32_t*>(smem + L::OFF_RUN);
  uint32_t* s_local = reinterpret_cast<uint32_t*>(smem + L::OFF_LOCAL);
  uint32_t* s_gbase = reinterpret_cast<uint32_t*>(smem + L::OFF_GBASE);
  uint32_t* s_wsum = reinterpret_cast<uint32_t*>(smem + L::OFF_WSUM);
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(smem + L::OFF_MBAR);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool staged = n >= 8 * int64_t(TILE) && (reinterpret_cast<uintptr_t>(keys) & 15) == 0 &&
                      (reinterpret_cast<uintptr_t>(scratch) & 15) == 0;

  // all-digit histogram of the segment (order-independent, so one read serves every pass)
  for (int i = tid; i < P * RADIX; i += NT) s_hist[i] = 0u;
  __syncthreads();
  for (int64_t i = tid; i < n; i += NT) {
    const U o = KO::to_ordered(keys[i]);
#pragma unroll
    for (int d = 0; d < P; d++) atomicAdd(&s_hist[d * RADIX + (uint32_t(o >> (8 * d)) & 0xFFu)], 1u);
  }
  __syncthreads();

  const int wbase = warp * 32 * KPT;
  const int ntiles = int((n + TILE - 1) / TILE);
  U* src = keys;
  U* dst = scratch;
  auto issue = [&](int t) {  // one thread: tile t of src into buffer t & 1
    const int64_t base = int64_t(t) * TILE;
    const int64_t cnt = n - base < TILE ? n - base : TILE;
    const uint32_t bytes = uint32_t((cnt * int64_t(sizeof(U))) & ~int64_t(15));
    unsigned char* buf = smem + L::OFF_BUF + size_t(t & 1) * L::TILE_BYTES;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&s_mbar[t & 1], bytes);
    if (bytes) bulk_copy_g2s(buf, src + base, bytes, &s_mbar[t & 1]);
  };
  for (int p = 0; p < P; p++) {
    // digit starts of this pass; a pass whose keys all share one digit is the identity
    bool trivial = false;
    if (tid < RADIX) {
      const uint32_t c = s_hist[p * RADIX + tid];
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      s_run[tid] = incl - c;
      if (lane == 31) s_wsum[warp] = incl;
    }
    __syncthreads();
    if (tid < RADIX) {
      uint32_t base = 0;
      for (int w = 0; w < (tid >> 5); w++) base += s_wsum[w];
      s_run[tid] += base;
    }
    trivial = __syncthreads_or(tid < RADIX && int64_t(s_hist[p * RADIX + tid]) == n) != 0;
    if (trivial) continue;
    if (staged && tid == 0) {
      issue(0);
      if (ntiles > 1) issue(1);
    }
    for (int t = 0; t < ntiles; t++) {
      const int64_t tb = int64_t(t) * TILE;
      const int tile_n = int((n - tb) < TILE ? (n - tb) : TILE);
      U* sk = reinterpret_cast<U*>(smem + L::OFF_BUF + size_t(staged ? (t & 1) : 0) * L::TILE_BYTES);
      U key[KPT];
      uint32_t pos[KPT];
      if (staged) {
        if (!mbar_wait_bounded(&s_mbar[t & 1], (phase >> (t & 1)) & 1u, spin_limit_ns)) {
          if (lane == 0) atomicOr(err, uint32_t(DERR_TMA_TIMEOUT));
        }
        phase ^= 1u << (t & 1);
        const int bulk_keys = int((int64_t(tile_n) * int64_t(sizeof(U))) & ~int64_t(15)) / int(sizeof(U));
#pragma unroll
        for (int i = 0; i < KPT; i++) {
          const int idx = wbase + i * 32 + lane;
          key[i] = idx < bulk_keys ? sk[idx] : (idx < tile_n ? src[tb + idx] : U(0));
        }
      } else {
#pragma unroll
        for (int i = 0; i < KPT; i++) {
          const int idx = wbase + i * 32 + lane;
          key[i] = idx < tile_n ? src[tb + idx] : U(0);
        }
      }
      seg_rank_tile<U, KIND, NT, KPT, MODE>(key, tile_n, 8 * p, s_cnt, s_msk, s_local, s_wsum, pos);
#pragma unroll
      for (int i = 0; i < KPT; i++)
        if (wbase + i * 32 + lane < tile_n) sk[pos[i]] = key[i];
      if (tid < RADIX) s_gbase[tid] = s_run[tid] - s_local[tid];
      __syncthreads();
      bool bad = false;
      for (int s = tid; s < tile_n; s += NT) {
        const U k = sk[s];
        const uint32_t dpos = s_gbase[KO::digit(k, 8 * p)] + uint32_t(s);
        if (int64_t(dpos) < n) dst[dpos] = k;
        else bad = true;
      }
      if (bad) atomicOr(err, uint32_t(DERR_BOUNDS));
      // the buffer was written through the generic proxy; a bulk copy refills it
      fence_proxy_async_smem();
      __syncthreads();
      if (staged && tid == 0 && t + 2 < ntiles) issue(t + 2);
      // advance the running offsets by this tile's digit counts
      if (tid < RADIX) {
        const uint32_t next = tid + 1 < RADIX ? s_local[tid + 1] : uint32_t(tile_n);
        s_run[tid] += next - s_local[tid];
      }
      __syncthreads();
    }
    // the next pass's bulk copies read what this pass wrote through the generic proxy
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
    U* tmp = src;
    src = dst;
    dst = tmp;
  }
  // an odd number of executed passes leaves the result in scratch
  if (src != keys) {
    for (int64_t i = tid; i < n; i += NT) keys[i] = src[i];
  }
  __syncthreads();
}

// ---- warp-level path: one warp sorts one small segment ----------------------------------
// Keys stay warp-striped in registers; every pass ranks them with the warp's 2^RB digit
// counters (RB-bit digits, so 32/RB or 64/RB passes), scans the counters across the lanes
// and reorders through the warp's own shared buffer.  No CTA barrier is involved, so the
// warps of a CTA sort different segments independently.
template <int KPT, int MODE>
struct WarpSegSmem {
  static constexpr int BUF_WORDS = 32 * KPT;  // one buffer of u32 words (u64 keys: half as many)
  static constexpr int CNT_WORDS = RADIX;
  static constexpr int MSK_WORDS = MODE == RANK_PEER_MASK ? 2 * RADIX : 0;
  static constexpr int WARP_WORDS = BUF_WORDS + CNT_WORDS + MSK_WORDS;
  static constexpr int WARPS = 8;  // 256 threads per CTA
  static constexpr size_t BYTES = size_t(WARPS) * WARP_WORDS * 4;
};

template <class U, int KIND, int KPTU, int RB, int MODE>
__device__ void warp_sort_small(U* keys, int n, U* buf, uint32_t* cnt, uint32_t* msk, int lane) {
  using KO = KeyOrder<U, KIND>;
  constexpr int RADIX_B = 1 << RB;
  constexpr int PASSES = (int(sizeof(U)) * 8 + RB - 1) / RB;
  U key[KPTU];
  uint32_t rank[KPTU];
#pragma unroll
  for (int i = 0; i < KPTU; i++) {
    const int idx = i * 32 + lane;
    key[i] = idx < n ? keys[idx] : U(0);
  }
  for (int p = 0; p < PASSES; p++) {
    const int shift = p * RB;
    for (int i = lane; i < RADIX_B; i += 32) cnt[i] = 0u;
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KPTU; i++) {
      const bool valid = i * 32 + lane < n;
      const uint32_t d = uint32_t(KO::to_ordered(key[i]) >> shift) & uint32_t(RADIX_B - 1);
      rank[i] = rank_in_warp<MODE>(cnt, msk, d, valid, i & 1, lane);
    }
    __syncwarp();
    // exclusive scan of the counters across the lanes
    if (RADIX_B >= 32) {
      constexpr int CPL = RADIX_B >= 32 ? RADIX_B / 32 : 1;
      uint32_t c[CPL];
      uint32_t sum = 0;
#pragma unroll
      for (int k = 0; k < CPL; k++) {
        c[k] = cnt[lane * CPL + k];
        sum += c[k];
      }
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      uint32_t run = incl - sum;
#pragma unroll
      for (int k = 0; k < CPL; k++) {
        cnt[lane * CPL + k] = run;
        run += c[k];
      }
    } else {
      const uint32_t c = lane < RADIX_B ? cnt[lane] : 0u;
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane < RADIX_B) cnt[lane] = incl - c;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KPTU; i++) {
      if (i * 32 + lane < n) {
        const uint32_t d = uint32_t(KO::to_ordered(key[i]) >> shift) & uint32_t(RADIX_B - 1);
        buf[cnt[d] + rank[i]] = key[i];
      }
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < KPTU; i++) {
      const int idx = i * 32 + lane;
      key[i] = idx < n ? buf[idx] : U(0);
    }
    __syncwarp();
  }
#pragma unroll
  for (int i = 0; i < KPTU; i++) {
    const int idx = i * 32 + lane;
    if (idx < n) keys[idx] = key[i];
  }
}

// Persistent warp-level kernel: each warp takes the next segment of its list (all of them at
// most 32 x KPT u32 / 16 x KPT u64 keys) and sorts it alone.
template <int KPT, int RB, int MODE>
__global__ void __launch_bounds__(256) seg_warp_kernel(SegParams prm) {
  using L = WarpSegSmem<KPT, MODE>;
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* base = reinterpret_cast<uint32_t*>(smem) + warp * L::WARP_WORDS;
  uint32_t* cnt = base + L::BUF_WORDS;
  uint32_t* msk = cnt + L::CNT_WORDS;
  if (MODE == RANK_PEER_MASK)
    for (int i = lane; i < L::MSK_WORDS; i += 32) msk[i] = 0u;
  __syncwarp();
  for (;;) {
    uint32_t sidx = 0;
    if (lane == 0) sidx = atomicAdd(prm.queue, 1u);
    sidx = __shfl_sync(0xFFFFFFFFu, sidx, 0);
    if (int(sidx) >= prm.nsegs) break;
    const SegDesc sd = prm.segs[sidx];
    const int n = int(sd.n);
    if (n <= 1) continue;
    const bool fits = sd.dtype >= 3 ? n <= 16 * KPT : n <= 32 * KPT;
    if (!fits) {  // the plan never routes such a segment here
      if (lane == 0) atomicOr(prm.err, uint32_t(DERR_BOUNDS));
      continue;
    }
    switch (sd.dtype) {
      case 0: warp_sort_small<uint32_t, KIND_UNSIGNED, KPT, RB, MODE>(static_cast<uint32_t*>(sd.keys), n, base, cnt, msk, lane); break;
      case 1: warp_sort_small<uint32_t, KIND_SIGNED, KPT, RB, MODE>(static_cast<uint32_t*>(sd.keys), n, base, cnt, msk, lane); break;
      case 2: warp_sort_small<uint32_t, KIND_FLOAT, KPT, RB, MODE>(static_cast<uint32_t*>(sd.keys), n, base, cnt, msk, lane); break;
      case 3: warp_sort_small<uint64_t, KIND_UNSIGNED, KPT / 2, RB, MODE>(static_cast<uint64_t*>(sd.keys), n, reinterpret_cast<uint64_t*>(base), cnt, msk, lane); break;
      case 4: warp_sort_small<uint64_t, KIND_SIGNED, KPT / 2, RB, MODE>(static_cast<uint64_t*>(sd.keys), n, reinterpret_cast<uint64_t*>(base), cnt, msk, lane); break;
      case 5: warp_sort_small<uint64_t, KIND_FLOAT, KPT / 2, RB, MODE>(static_cast<uint64_t*>(sd.keys), n, reinterpret_cast<uint64_t*>(base), cnt, msk, lane); break;
      default:
        if (lane == 0) atomicOr(prm.err, uint32_t(DERR_BOUNDS));
        break;
    }
  }
}

// ---- block-level path: one CTA sorts one segment ----------------------------------------
// LARGE = false: every array fits one tile and is sorted in shared memory; LARGE = true: every
// array is longer than a tile and is sorted tile by tile with scratch.  The plan routes each
// array to the right one, so each kernel carries one path only (and its register count).
template <int NT, int KPT, int MODE, bool LARGE>
__global__ void __launch_bounds__(NT, NT <= 256 ? 2 : 1) segmented_sort_kernel(SegParams prm) {
  static_assert(NT >= RADIX, "one thread per digit needed");
  using L = SegSmem<NT, KPT, MODE>;
  extern __shared__ __align__(128) unsigned char smem[];
  int* s_seg = reinterpret_cast<int*>(smem + L::OFF_SEG);
  uint32_t* s_msk = reinterpret_cast<uint32_t*>(smem + L::OFF_MSK);
  if (MODE == RANK_PEER_MASK)
    for (int i = threadIdx.x; i < L::NW * 2 * RADIX; i += NT) s_msk[i] = 0u;
  if (LARGE && threadIdx.x == 0) {
    uint64_t* s_mbar = reinterpret_cast<uint64_t*>(smem + L::OFF_MBAR);
    mbar_init(&s_mbar[0], 1);
    mbar_init(&s_mbar[1], 1);
    fence_mbar_init();
  }
  uint32_t phase = 0;  // expected parity of each bulk-copy barrier (bit s: buffer s)
  uint32_t* err = prm.err;
  for (;;) {
    if (threadIdx.x == 0) *s_seg = int(atomicAdd(prm.queue, 1u));
    __syncthreads();
    const int sidx = *s_seg;
    __syncthreads();
    if (sidx >= prm.nsegs) break;
    const SegDesc sd = prm.segs[sidx];
    if (sd.n <= 1) continue;
    const int64_t tile = sd.dtype >= 3 ? int64_t(NT) * (KPT / 2) : int64_t(NT) * KPT;
    if ((sd.n <= tile) == LARGE) {  // the plan never routes such an array here
      if (threadIdx.x == 0) atomicOr(err, uint32_t(DERR_BOUNDS));
      continue;
    }
    auto go32 = [&](auto kind) {
      constexpr int K = decltype(kind)::value;
      uint32_t* k = static_cast<uint32_t*>(sd.keys);
      if (LARGE) seg_sort_large<uint32_t, K, NT, KPT, MODE>(k, static_cast<uint32_t*>(sd.scratch), sd.n, smem, err, prm.spin_limit_ns, phase);
      else seg_sort_small<uint32_t, K, NT, KPT, MODE>(k, int(sd.n), smem);
    };
    auto go64 = [&](auto kind) {
      constexpr int K = decltype(kind)::value;
      uint64_t* k = static_cast<uint64_t*>(sd.keys);
      if (LARGE) seg_sort_large<uint64_t, K, NT, KPT / 2, MODE>(k, static_cast<uint64_t*>(sd.scratch), sd.n, smem, err, prm.spin_limit_ns, phase);
      else seg_sort_small<uint64_t, K, NT, KPT / 2, MODE>(k, int(sd.n), smem);
    };
    switch (sd.dtype) {
      case 0: go32(std::integral_constant<int, KIND_UNSIGNED>()); break;
      case 1: go32(std::integral_constant<int, KIND_SIGNED>()); break;
      case 2: go32(std::integral_constant<int, KIND_FLOAT>()); break;
      case 3: go64(std::integral_constant<int, KIND_UNSIGNED>()); break;
      case 4: go64(std::integral_constant<int, KIND_SIGNED>()); break;
      case 5: go64(std::integral_constant<int, KIND_FLOAT>()); break;
      default:
        if (threadIdx.x == 0) atomicOr(err, uint32_t(DERR_BOUNDS));
        break;
    }
  }
}

}  // namespace hpcs
