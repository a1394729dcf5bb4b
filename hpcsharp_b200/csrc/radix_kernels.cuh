// LSD radix sort kernels for sm_100a.
//
// Restates HPCsharp's LSD hot path (RadixSortLsd.cs, RadixSortLsdParallel.cs,
// Histogram.cs, HistogramParallel.cs) as three kernels per sort:
//
//   K1 hist_all_digits  One 128-bit vectorised read of every key builds the byte histogram
//                       of every digit at once (HistogramByteComponents[Par],
//                       Histogram.cs:261-296, HistogramParallel.cs:163-222).  The last CTA
//                       to finish turns the counts into the per-digit exclusive starts
//                       (ComputeStartOfBins, RadixSortLsd.cs:112-125), marks digit passes
//                       whose keys all share one digit value as skippable (the idea of
//                       RadixSortLsd.cs:2093-2117), and assigns ping-pong buffers.
//   K3 onesweep_pass    One launch per 8-bit digit.  Persistent CTAs take tile ids from a
//                       global counter; each tile is staged into shared memory by a bulk
//                       async copy (prefetched one tile ahead), ranked in-warp with
//                       __match_any_sync, chained to its predecessors by a single-pass
//                       decoupled look-back over per-(tile, digit) status words, reordered
//                       in shared memory by digit and written out as coalesced per-digit
//                       runs.  Ranking is stable (input order within a digit), so the pass
//                       equals the reference's stable scatter (RadixSortLsdParallel.cs:96-135
//                       with the bin-major / quantum-minor offsets of :49-94).
//   finalize            Copies the result back to the caller's buffer when an odd number of
//                       passes ran (only possible when passes were skipped).
#pragma once
#include <cstdint>
#include <type_traits>

#include "common.cuh"

namespace hpcs {

constexpr int RADIX = 256;
constexpr int MAX_PASSES = 8;

// Status word of the decoupled look-back: 2 flag bits + 30 value bits.
constexpr uint32_t ST_AGGREGATE = 1u << 30;  // tile-local count only
constexpr uint32_t ST_PREFIX = 2u << 30;     // inclusive prefix over tiles 0..t
constexpr uint32_t ST_FLAGS = 3u << 30;
constexpr uint32_t ST_VALUE = (1u << 30) - 1;
constexpr int64_t MAX_KEYS_PER_SORT = (int64_t(1) << 30) - 1;

struct NoValue {};

// Per-sort control block in device memory (zeroed before K1).
struct SortPlan {
  uint32_t hist[MAX_PASSES][RADIX];       // raw digit counts
  uint32_t bin_start[MAX_PASSES][RADIX];  // exclusive scan per digit
  int32_t src_sel[MAX_PASSES];            // 0: A->B, 1: B->A, -1: pass skipped
  int32_t status_sel[MAX_PASSES];         // which look-back buffer the pass uses
  uint32_t tile_counter[MAX_PASSES];
  int32_t final_sel;                      // buffer holding the result (0 = A)
  uint32_t done_blocks;
  uint32_t error;                         // DeviceError bits
  uint32_t pad;
};

struct SortArgs {
  void* keys_a;
  void* keys_b;
  void* vals_a;
  void* vals_b;
  int64_t n;
  SortPlan* plan;
  uint32_t* status[2];
  int num_tiles;
  int pass;
  int skip_trivial;
  int poison_tile;        // test hook: this tile never publishes (-1 = off)
  uint64_t spin_limit_ns; // bound on every device-side wait
};

// =====================================================================================
// K1: fused all-digit histogram (+ plan in the last CTA)
// =====================================================================================
template <class U, int KIND, int NT>
__global__ void __launch_bounds__(NT) hist_all_digits_kernel(const U* __restrict__ keys, int64_t n,
                                                              uint32_t* __restrict__ hist_out,
                                                              SortArgs args, int make_plan) {
  constexpr int P = int(sizeof(U));
  constexpr int VEC = 16 / int(sizeof(U));
  using KO = KeyOrder<U, KIND>;
  __shared__ uint32_t sh[P][RADIX];
  __shared__ uint32_t s_last;
  const int tid = threadIdx.x;
  for (int i = tid; i < P * RADIX; i += NT) (&sh[0][0])[i] = 0;
  __syncthreads();

  // Count the P digits of one key.  Every lane of the warp calls this together (the loop
  // bounds below are warp-uniform); lanes without a key pass valid = false.
  auto count_key = [&](U k, bool valid) {
    U o = KO::to_ordered(k);
#pragma unroll
    for (int d = 0; d < P; d++) {
      uint32_t dg = uint32_t(o >> (8 * d)) & 0xFFu;
      // Lane 0 holds a key whenever any lane does (indices grow with the lane).
      uint32_t first = __shfl_sync(0xFFFFFFFFu, dg, 0);
      if (__all_sync(0xFFFFFFFFu, !valid || dg == first)) {
        // constant or heavily skewed byte: one atomic for the warp
        uint32_t cnt = __popc(__ballot_sync(0xFFFFFFFFu, valid));
        if ((tid & 31) == 0 && cnt) atomicAdd(&sh[d][first], cnt);
      } else if (valid) {
        atomicAdd(&sh[d][dg], 1u);
      }
    }
  };

  const int64_t nvec = n / VEC;
  const uint4* vkeys = reinterpret_cast<const uint4*>(keys);
  const int64_t stride = int64_t(gridDim.x) * NT;
  const int lane = tid & 31;
  // Warp-uniform grid-stride loop, 4 vectors in flight per thread per iteration.
  for (int64_t wb = int64_t(blockIdx.x) * NT + (tid - lane); wb < nvec; wb += 4 * stride) {
    uint4 v[4];
    bool ok[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int64_t idx = wb + lane + int64_t(u) * stride;
      ok[u] = idx < nvec;
      v[u] = ok[u] ? ldg_stream_v4(vkeys + idx) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const U* e = reinterpret_cast<const U*>(&v[u]);
#pragma unroll
      for (int j = 0; j < VEC; j++) count_key(e[j], ok[u]);
    }
  }
  // Ragged tail (fewer than VEC keys): warp 0 of block 0.
  if (blockIdx.x == 0 && tid < 32) {
    const int64_t t = nvec * VEC + tid;
    const bool valid = t < n;
    count_key(valid ? keys[t] : U(0), valid);
  }
  __syncthreads();
  for (int j = tid; j < P * RADIX; j += NT) {
    uint32_t c = (&sh[0][0])[j];
    if (c) atomicAdd(hist_out + j, c);
  }
  if (!make_plan) return;

  // Zero the first look-back buffer for the first executed pass, and the tile counters.
  {
    uint32_t* s0 = args.status[0];
    const int64_t words = int64_t(args.num_tiles) * RADIX;
    for (int64_t w = int64_t(blockIdx.x) * NT + tid; w < words; w += stride) s0[w] = 0;
  }
  // Last-block-done: the final CTA builds the plan.
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = (atomicAdd(&args.plan->done_blocks, 1u) == gridDim.x - 1) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  SortPlan* plan = args.plan;
  __shared__ uint32_t s_trivial[P];
  __shared__ uint32_t s_wsum[RADIX / 32];
  for (int d = 0; d < P; d++) {
    uint32_t c = 0;
    if (tid < RADIX) {
      c = ld_volatile(&hist_out[d * RADIX + tid]);
    }
    if (tid == 0) s_trivial[d] = 0;
    __syncthreads();
    if (tid < RADIX && int64_t(c) == n) s_trivial[d] = 1;
    // exclusive scan of 256 counts (first 8 warps)
    uint32_t incl = c;
    if (tid < RADIX) {
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if ((tid & 31) >= o) incl += y;
      }
      if ((tid & 31) == 31) s_wsum[tid >> 5] = incl;
    }
    __syncthreads();
    if (tid < RADIX) {
      uint32_t base = 0;
      for (int w = 0; w < (tid >> 5); w++) base += s_wsum[w];
      plan->bin_start[d][tid] = base + incl - c;
    }
    __syncthreads();
  }
  if (tid == 0) {
    int sel = 0, executed = 0;
    for (int d = 0; d < MAX_PASSES; d++) {
      plan->tile_counter[d] = 0;
      if (d >= P) {
        plan->src_sel[d] = -1;
        plan->status_sel[d] = 0;
        continue;
      }
      bool skip = args.skip_trivial && s_trivial[d];
      if (skip) {
        plan->src_sel[d] = -1;
        plan->status_sel[d] = 0;
      } else {
        plan->src_sel[d] = sel;
        plan->status_sel[d] = executed & 1;
        sel ^= 1;
        executed++;
      }
    }
    plan->final_sel = sel;
    __threadfence();
  }
}

// =====================================================================================
// K3: one 8-bit digit pass (onesweep)
// =====================================================================================
template <class U, class V, int NT, int KPT, int STAGES>
struct OnesweepSmem {
  static constexpr bool PAIRS = !std::is_same<V, NoValue>::value;
  static constexpr int TILE = NT * KPT;
  static constexpr int NW = NT / 32;
  static constexpr size_t KEYS_BYTES = size_t(TILE) * sizeof(U);
  static constexpr size_t VALS_BYTES = PAIRS ? size_t(TILE) * 4 : 0;
  static constexpr size_t STAGE_BYTES = KEYS_BYTES + VALS_BYTES;
  static constexpr size_t OFF_STAGES = 0;
  static constexpr size_t OFF_WHIST = OFF_STAGES + STAGE_BYTES * STAGES;
  static constexpr size_t OFF_BINSTART = OFF_WHIST + size_t(NW) * RADIX * 4;
  static constexpr size_t OFF_TOTAL = OFF_BINSTART + RADIX * 4;
  static constexpr size_t OFF_LOCAL = OFF_TOTAL + RADIX * 4;
  static constexpr size_t OFF_GBASE = OFF_LOCAL + RADIX * 4;
  static constexpr size_t OFF_WSUM = OFF_GBASE + RADIX * 4;
  static constexpr size_t OFF_TILE = OFF_WSUM + 32 * 4;
  static constexpr size_t OFF_MBAR = (OFF_TILE + 16 + 7) / 8 * 8;
  static constexpr size_t BYTES = OFF_MBAR + 8 * STAGES;
};

// Issue the bulk copy of tile t into stage s (called by one thread).  The 16-byte-aligned
// body is copied by the TMA engine; the ragged tail (< 16 bytes) is read with plain loads
// by the consumers.  Stage buffers start at offset 0 of the dynamic shared memory.
template <class U, bool PAIRS, int TILE>
__device__ __forceinline__ void onesweep_issue_tile(unsigned char* smem, size_t stage_bytes, size_t keys_bytes,
                                                    uint64_t* mbar, const U* kin, const uint32_t* vin,
                                                    int64_t n, int t, int s) {
  const int64_t base = int64_t(t) * TILE;
  const int64_t cnt = (n - base) < TILE ? (n - base) : TILE;
  const uint32_t kbytes = uint32_t((cnt * int64_t(sizeof(U))) & ~int64_t(15));
  const uint32_t vbytes = PAIRS ? uint32_t((cnt * 4) & ~int64_t(15)) : 0u;
  unsigned char* dst = smem + size_t(s) * stage_bytes;
  fence_proxy_async_smem();
  mbar_arrive_expect_tx(&mbar[s], kbytes + vbytes);
  if (kbytes) bulk_copy_g2s(dst, kin + base, kbytes, &mbar[s]);
  if (PAIRS && vbytes) bulk_copy_g2s(dst + keys_bytes, vin + base, vbytes, &mbar[s]);
}

template <class U, int KIND, class V, int NT, int KPT, int STAGES, int MINB>
__global__ void __launch_bounds__(NT, MINB) onesweep_pass_kernel(SortArgs args) {
  using L = OnesweepSmem<U, V, NT, KPT, STAGES>;
  using KO = KeyOrder<U, KIND>;
  constexpr bool PAIRS = L::PAIRS;
  constexpr int TILE = L::TILE;
  constexpr int NW = L::NW;
  static_assert(NT >= RADIX && NT % 32 == 0, "one thread per digit needed");

  const SortPlan* plan = args.plan;
  const int pass = args.pass;
  const int sel = plan->src_sel[pass];
  if (sel < 0) return;  // every key has the same digit here: the pass is the identity
  const int shift = 8 * pass;
  const U* __restrict__ kin = static_cast<const U*>(sel ? args.keys_b : args.keys_a);
  U* __restrict__ kout = static_cast<U*>(sel ? args.keys_a : args.keys_b);
  const uint32_t* __restrict__ vin = static_cast<const uint32_t*>(sel ? args.vals_b : args.vals_a);
  uint32_t* __restrict__ vout = static_cast<uint32_t*>(sel ? args.vals_a : args.vals_b);
  const int ssel = plan->status_sel[pass];
  // selects, not args.status[ssel]: a dynamic index would copy the parameters to local memory
  uint32_t* __restrict__ status = ssel ? args.status[1] : args.status[0];
  uint32_t* __restrict__ status_next = ssel ? args.status[0] : args.status[1];
  uint32_t* tile_counter = const_cast<uint32_t*>(&plan->tile_counter[pass]);
  uint32_t* err = const_cast<uint32_t*>(&plan->error);
  const int64_t n = args.n;
  const int num_tiles = args.num_tiles;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* s_whist = reinterpret_cast<uint32_t*>(smem + L::OFF_WHIST);  // [NW][256]
  uint32_t* s_binstart = reinterpret_cast<uint32_t*>(smem + L::OFF_BINSTART);
  uint32_t* s_total = reinterpret_cast<uint32_t*>(smem + L::OFF_TOTAL);
  uint32_t* s_local = reinterpret_cast<uint32_t*>(smem + L::OFF_LOCAL);
  uint32_t* s_gbase = reinterpret_cast<uint32_t*>(smem + L::OFF_GBASE);
  uint32_t* s_wsum = reinterpret_cast<uint32_t*>(smem + L::OFF_WSUM);
  int* s_tile = reinterpret_cast<int*>(smem + L::OFF_TILE);
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(smem + L::OFF_MBAR);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) mbar_init(&s_mbar[s], 1);
    fence_mbar_init();
    fence_proxy_async_smem();
  }
  for (int i = tid; i < RADIX; i += NT) s_binstart[i] = plan->bin_start[pass][i];
  __syncthreads();
  if (tid == 0) {
    int t0 = int(atomicAdd(tile_counter, 1u));
    s_tile[0] = t0;
    if (t0 < num_tiles) onesweep_issue_tile<U, PAIRS, TILE>(smem, L::STAGE_BYTES, L::KEYS_BYTES, s_mbar, kin, vin, n, t0, 0);
  }
  __syncthreads();

  uint32_t phase_bits = 0;  // bit s = parity to wait for on stage s
  int stage = 0;
  for (;;) {
    const int t = s_tile[stage];
    if (t >= num_tiles) break;
    if (STAGES > 1 && tid == 0) {
      int tn = int(atomicAdd(tile_counter, 1u));
      s_tile[stage ^ 1] = tn;
      if (tn < num_tiles)
        onesweep_issue_tile<U, PAIRS, TILE>(smem, L::STAGE_BYTES, L::KEYS_BYTES, s_mbar, kin, vin, n, tn, stage ^ 1);
    }
    const int64_t tile_base = int64_t(t) * TILE;
    const int tile_n = int((n - tile_base) < TILE ? (n - tile_base) : TILE);
    const int bulk_keys = int((int64_t(tile_n) * int64_t(sizeof(U))) & ~int64_t(15)) / int(sizeof(U));
    const int bulk_vals = PAIRS ? int((int64_t(tile_n) * 4) & ~int64_t(15)) / 4 : 0;

    // zero this warp's digit counters
    for (int i = lane; i < RADIX; i += 32) s_whist[warp * RADIX + i] = 0;

    // wait for the staged tile (bounded)
    if (!mbar_wait_bounded(&s_mbar[stage], (phase_bits >> stage) & 1u, args.spin_limit_ns)) {
      if (lane == 0) atomicOr(err, uint32_t(DERR_TMA_TIMEOUT));
    }
    phase_bits ^= (1u << stage);
    __syncwarp();

    // ---- load keys (warp-striped) and rank them within the warp --------------------
    U* sk = reinterpret_cast<U*>(smem + L::OFF_STAGES + stage * L::STAGE_BYTES);
    U key[KPT];
    uint32_t rank[KPT];
    const int wbase = warp * 32 * KPT;
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      U k = U(0);
      if (idx < bulk_keys) k = sk[idx];
      else if (idx < tile_n) k = kin[tile_base + idx];
      key[i] = k;
    }
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      const bool valid = idx < tile_n;
      const uint32_t d = valid ? KO::digit(key[i], shift) : 0x100u;
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
      const int leader = __ffs(peers) - 1;
      uint32_t before = 0;
      if (lane == leader && valid) {
        before = s_whist[warp * RADIX + d];
        s_whist[warp * RADIX + d] = before + __popc(peers);
      }
      before = __shfl_sync(0xFFFFFFFFu, before, leader);
      rank[i] = before + __popc(peers & lanemask_lt());
      __syncwarp();
    }
    __syncthreads();  // (A) warp counts complete; stage buffer no longer read

    // ---- per digit: exclusive prefix over warps, tile total, publish aggregate -----
    if (tid < RADIX) {
      const int dg = tid;
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < NW; w++) {
        uint32_t c = s_whist[w * RADIX + dg];
        s_whist[w * RADIX + dg] = run;
        run += c;
      }
      s_total[dg] = run;
      if (t != args.poison_tile) {
        if (t == 0) st_relaxed_gpu(&status[dg], ST_PREFIX | run);
        else st_relaxed_gpu(&status[int64_t(t) * RADIX + dg], ST_AGGREGATE | run);
      }
      // warp-inclusive scan of the totals (digit order)
      uint32_t incl = run;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      s_local[dg] = incl;  // inclusive within the warp for now
      if (lane == 31) s_wsum[warp] = incl;
    }
    __syncthreads();  // (B)
    if (tid < RADIX) {
      const int dg = tid;
      uint32_t base = 0;
#pragma unroll
      for (int w = 0; w < RADIX / 32; w++) base += (w < warp) ? s_wsum[w] : 0u;
      s_local[dg] = base + s_local[dg] - s_total[dg];
    }
    __syncthreads();  // (B2) tile-local digit starts ready

    // ---- decoupled look-back (one thread per digit), overlapped with the reorder ----
    if (tid < RADIX) {
      const int dg = tid;
      uint32_t excl = 0;
      if (t > 0) {
        int j = t - 1;
        uint64_t t0 = 0;
        bool timed_out = false;
        while (j >= 0) {
          uint32_t s = ld_relaxed_gpu(&status[int64_t(j) * RADIX + dg]);
          if ((s & ST_FLAGS) == 0) {
            if (t0 == 0) t0 = global_timer_ns();
            else if (global_timer_ns() - t0 > args.spin_limit_ns || ld_volatile(err) != 0u) {
              timed_out = true;
              break;
            }
            continue;
          }
          t0 = 0;
          excl += s & ST_VALUE;
          if (s & ST_PREFIX) break;
          j--;
        }
        if (timed_out) atomicOr(err, uint32_t(DERR_LOOKBACK_TIMEOUT));
        if (t != args.poison_tile)
          st_relaxed_gpu(&status[int64_t(t) * RADIX + dg], ST_PREFIX | ((excl + s_total[dg]) & ST_VALUE));
      }
      s_gbase[dg] = s_binstart[dg] + excl - s_local[dg];
      // zero-ahead: clear this tile's words in the buffer the next executed pass uses
      status_next[int64_t(t) * RADIX + dg] = 0;
    }

    // ---- reorder the tile in shared memory by digit -----------------------------------
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      if (idx < tile_n) {
        const uint32_t d = KO::digit(key[i], shift);
        const uint32_t pos = s_local[d] + s_whist[warp * RADIX + d] + rank[i];
        rank[i] = pos;  // keep the tile position for the payload
        sk[pos] = key[i];
      }
    }
    __syncthreads();  // (C) reordered keys and global bases ready

    // ---- write coalesced per-digit runs ----------------------------------------------
    // Every destination is checked against n: after a timed-out look-back the offsets are
    // not trusted, and a bad one is recorded instead of written.
    uint8_t dsave[PAIRS ? KPT : 1];
    bool out_of_range = false;
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int s = i * NT + tid;
      if (s < tile_n) {
        const U k = sk[s];
        const uint32_t d = KO::digit(k, shift);
        if (PAIRS) dsave[i] = uint8_t(d);
        const uint32_t pos = s_gbase[d] + uint32_t(s);
        if (pos < uint32_t(n)) kout[pos] = k;
        else out_of_range = true;
      }
    }
    if (PAIRS) {
      uint32_t* sv = reinterpret_cast<uint32_t*>(smem + L::OFF_STAGES + stage * L::STAGE_BYTES + L::KEYS_BYTES);
      uint32_t val[KPT];
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int idx = wbase + i * 32 + lane;
        uint32_t v = 0;
        if (idx < bulk_vals) v = sv[idx];
        else if (idx < tile_n) v = vin[tile_base + idx];
        val[i] = v;
      }
      __syncthreads();  // (D) all payloads read before they are overwritten
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int idx = wbase + i * 32 + lane;
        if (idx < tile_n) sv[rank[i]] = val[i];
      }
      __syncthreads();  // (E)
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int s = i * NT + tid;
        if (s < tile_n) {
          const uint32_t pos = s_gbase[dsave[i]] + uint32_t(s);
          if (pos < uint32_t(n)) vout[pos] = sv[s];
        }
      }
    }
    if (out_of_range) atomicOr(err, uint32_t(DERR_BOUNDS));
    // The stage buffer was written through the generic proxy; a later bulk copy (async
    // proxy) refills it, so order the writes before the barrier.
    fence_proxy_async_smem();
    __syncthreads();  // (F) shared memory free for the next tile
    if (STAGES > 1) stage ^= 1;
    else if (tid == 0) {
      int tn = int(atomicAdd(tile_counter, 1u));
      s_tile[0] = tn;
      if (tn < num_tiles) onesweep_issue_tile<U, PAIRS, TILE>(smem, L::STAGE_BYTES, L::KEYS_BYTES, s_mbar, kin, vin, n, tn, 0);
    }
    if (STAGES == 1) __syncthreads();
  }
}

// Copy B -> A when the result ended in the scratch buffer, and fold this sort's device
// error bits into the context's accumulator.
template <class U>
__global__ void finalize_kernel(SortArgs args, int has_vals, uint32_t* err_accum) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    uint32_t e = ld_volatile(&args.plan->error);
    if (e) atomicOr(err_accum, e);
  }
  if (args.plan->final_sel != 1) return;
  const int64_t n = args.n;
  const U* src = static_cast<const U*>(args.keys_b);
  U* dst = static_cast<U*>(args.keys_a);
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[i];
  if (has_vals) {
    const uint32_t* vs = static_cast<const uint32_t*>(args.vals_b);
    uint32_t* vd = static_cast<uint32_t*>(args.vals_a);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) vd[i] = vs[i];
  }
}

}  // namespace hpcs
