// LSD sort of a small array (keys, or keys with a 32-bit item each; at most SMALL_MAX_CTAS x
// SMALL_TILE keys) in one cooperative launch.
//
// A sort of ~10^5 keys through the large-array kernels is a chain of launches (histogram, one
// launch per digit pass, copy-back), each running on a handful of SMs with little to do, so its
// time is mostly launch gaps and per-launch set-up.  Here one launch of G = ceil(n / SMALL_TILE)
// CTAs runs every pass: CTA c owns keys [c * SMALL_TILE, (c + 1) * SMALL_TILE) of the pass's
// input.  Per pass:
//   rank     the keys are loaded warp-striped and ranked with the sort's own per-warp ranking
//            (ordered shared atomics or the peer-mask mode), stable within the CTA;
//   counts   the CTA's digit totals go to counts[c][256]; a grid barrier;
//   offsets  every CTA adds up all CTAs' totals (the global digit starts) and the totals of the
//            CTAs before it (the bin-major, CTA-minor offsets of RadixSortLsdParallel.cs:49-94
//            with one quantum per CTA);
//   scatter  each key (and its item) goes to its digit's start + its CTA's offset + its warp's
//            offset + its rank; a grid barrier before the next pass reads the output.
// The launch is cooperative, so all G CTAs are resident together; the grid barrier's wait is
// still bounded (spin_limit_ns) and records a timeout in the error word instead of hanging.
// Keys written by other CTAs are read through L2 (ld.global.cg), never from a stale L1 line.
// P passes (4 or 8) leave the result in the caller's buffer.
#pragma once
#include <cstdint>

#include "radix_kernels.cuh"

namespace hpcs {

constexpr int SMALL_NT = 256, SMALL_KPT = 16, SMALL_TILE = SMALL_NT * SMALL_KPT;
constexpr int SMALL_MAX_CTAS = 32;
constexpr int64_t SMALL_MAX_KEYS = int64_t(SMALL_MAX_CTAS) * SMALL_TILE;  // 131072

// Grid barrier over the launch's G CTAs: bar[0] counts arrivals, bar[1] is the generation.
// bar[0] is zero at launch; the last CTA to arrive resets it and advances the generation.
__device__ __forceinline__ void small_grid_barrier(uint32_t* bar, uint32_t G, uint32_t* err, uint64_t limit_ns) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t gen = ld_relaxed_gpu(bar + 1);  // GPU-scope loads: no stale L1 line
    __threadfence();  // this CTA's writes are visible before it arrives
    if (atomicAdd(bar, 1u) == G - 1u) {
      bar[0] = 0u;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const uint64_t t0 = global_timer_ns();
      while (ld_relaxed_gpu(bar + 1) == gen) {
        if (global_timer_ns() - t0 > limit_ns) {
          atomicOr(err, uint32_t(DERR_LOOKBACK_TIMEOUT));
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

template <class U>
__device__ __forceinline__ U ld_cg_key(const U* p) {
  if (sizeof(U) == 4) return U(__ldcg(reinterpret_cast<const unsigned int*>(p)));
  return U(__ldcg(reinterpret_cast<const unsigned long long*>(p)));
}

template <class U, int KIND, class V, int MODE>
__global__ void __launch_bounds__(SMALL_NT) small_sort_kernel(U* a, U* b, uint32_t* va, uint32_t* vb, int n,
                                                             uint32_t* counts, uint32_t* bar, uint32_t* err,
                                                             uint64_t spin_limit_ns) {
  using KO = KeyOrder<U, KIND>;
  constexpr bool PAIRS = !std::is_same<V, NoValue>::value;
  constexpr int P = int(sizeof(U));
  constexpr int NW = SMALL_NT / 32;
  __shared__ uint32_t s_cnt[NW][RADIX];  // per-warp digit counters, then per-(warp, digit) offsets
  __shared__ uint32_t s_msk[MODE == RANK_PEER_MASK ? NW * 2 * RADIX : 1];
  __shared__ uint32_t s_base[RADIX];
  __shared__ uint32_t s_wsum[RADIX / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t G = gridDim.x;
  const int lo = int(blockIdx.x) * SMALL_TILE;
  const int cnt_n = n - lo < SMALL_TILE ? n - lo : SMALL_TILE;
  uint32_t* cnt_w = s_cnt[warp];
  uint32_t* msk_w = s_msk + (MODE == RANK_PEER_MASK ? warp * 2 * RADIX : 0);
  const uint32_t n32 = uint32_t(n);
  bool out_of_range = false;
  for (int p = 0; p < P; p++) {
    const U* src = (p & 1) ? b : a;
    U* dst = (p & 1) ? a : b;
    const uint32_t* vsrc = (p & 1) ? vb : va;
    uint32_t* vdst = (p & 1) ? va : vb;
    const int shift = 8 * p;
    for (int i = tid; i < NW * RADIX; i += SMALL_NT) (&s_cnt[0][0])[i] = 0u;
    if (MODE == RANK_PEER_MASK)
      for (int i = tid; i < NW * 2 * RADIX; i += SMALL_NT) s_msk[i] = 0u;
    __syncthreads();
    U key[SMALL_KPT];
    uint32_t val[PAIRS ? SMALL_KPT : 1];
    uint32_t dg[SMALL_KPT], rank[SMALL_KPT];
    const int wbase = warp * 32 * SMALL_KPT;
#pragma unroll
    for (int i = 0; i < SMALL_KPT; i++) {  // all loads issued before the first is used
      const int idx = wbase + i * 32 + lane;
      key[i] = idx < cnt_n ? ld_cg_key(src + lo + idx) : U(0);
      if (PAIRS) val[PAIRS ? i : 0] = idx < cnt_n ? __ldcg(vsrc + lo + idx) : 0u;
    }
#pragma unroll
    for (int i = 0; i < SMALL_KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      dg[i] = KO::digit(key[i], shift);
      rank[i] = rank_in_warp<MODE>(cnt_w, msk_w, dg[i], idx < cnt_n, i & 1, lane);
    }
    __syncthreads();
    if (tid < RADIX) {  // per digit: the warps' exclusive offsets and the CTA's total
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < NW; w++) {
        const uint32_t c = s_cnt[w][tid];
        s_cnt[w][tid] = run;
        run += c;
      }
      counts[blockIdx.x * RADIX + tid] = run;
    }
    small_grid_barrier(bar, G, err, spin_limit_ns);
    if (tid < RADIX) {  // digit start over all CTAs + this digit's keys in the CTAs before this one
      uint32_t v[SMALL_MAX_CTAS];  // every CTA's total, all loads in flight together
#pragma unroll
      for (int c = 0; c < SMALL_MAX_CTAS; c++) v[c] = uint32_t(c) < G ? __ldcg(counts + c * RADIX + tid) : 0u;
      uint32_t tot = 0, pre = 0;
#pragma unroll
      for (int c = 0; c < SMALL_MAX_CTAS; c++) {
        tot += v[c];
        pre += uint32_t(c) < blockIdx.x ? v[c] : 0u;
      }
      uint32_t incl = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) s_wsum[warp] = incl;
      s_base[tid] = incl - tot + pre;  // the warps' sums are added below
    }
    __syncthreads();
    if (tid < RADIX) {
      uint32_t before = 0;
      for (int w = 0; w < warp; w++) before += s_wsum[w];
      s_base[tid] += before;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SMALL_KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      if (idx < cnt_n) {
        const uint32_t pos = s_base[dg[i]] + cnt_w[dg[i]] + rank[i];
        if (pos < n32) {
          dst[pos] = key[i];
          if (PAIRS) vdst[pos] = val[PAIRS ? i : 0];
        } else {
          out_of_range = true;
        }
      }
    }
    small_grid_barrier(bar, G, err, spin_limit_ns);  // the output is complete; counts may be reused
  }
  if (out_of_range) atomicOr(err, uint32_t(DERR_BOUNDS));
}

}  // namespace hpcs
