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

#include <cooperative_groups.h>

#include "common.cuh"

namespace hpcs {

constexpr int RADIX = 256;
constexpr int MAX_PASSES = 8;

// Status word of the decoupled look-back: 2 flag bits + 30 value bits.
constexpr uint32_t ST_AGGREGATE = 1u << 30;  // tile-local count only
constexpr uint32_t ST_PREFIX = 2u << 30;     // inclusive prefix over tiles 0..t
constexpr uint32_t ST_FLAGS = 3u << 30;
constexpr uint32_t ST_VALUE = (1u << 30) - 1;
constexpr int64_t MAX_KEYS_PER_SORT = (int64_t(1) << 31) - 1;     // chunked passes: 32-bit positions
constexpr int64_t MAX_KEYS_LOOKBACK = (int64_t(1) << 30) - 1;     // look-back: 30-bit prefixes
// Predecessor status words read per look-back step.
#ifndef HPCS_LB_WINDOW
#define HPCS_LB_WINDOW 8
#endif
constexpr int LB_WINDOW = HPCS_LB_WINDOW;

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
  uint32_t idle_flag;                     // never written: the wait-timeout test hook spins on it
  int32_t exec_idx[MAX_PASSES];           // 0, 1, 2, ... over the executed passes
  int32_t next_shift[MAX_PASSES];         // bit shift of the next executed pass's digit, -1 if none
  int32_t heavy[MAX_PASSES];              // the most frequent value of each digit (lowest on ties)
  int32_t skewed[MAX_PASSES];             // 1 when that value holds more than 1/32 of the keys
  int32_t heavy2[MAX_PASSES];             // the second most frequent value
  int32_t grouped[MAX_PASSES];            // 1 when the two hold more than 3/4 of the keys
  int32_t use_lookback;                   // device-chosen scheme (SortArgs::choose_lookback)
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
  // Tile trace (debug): when non-null, thread 0 writes TRACE_WORDS stamps per tile of
  // pass `trace_pass`: tile id, SM id, then %globaltimer at start, data ready, ranked,
  // look-back done (digit 0), end of scatter.
  uint64_t* trace;
  int trace_pass;
  int trace_capacity;  // tiles
  // Chunked passes (chunk_hist != null): the keys are cut into `chunks` ranges of
  // chunk_keys keys (a whole number of tiles); CTA j of every kernel owns range j.
  uint32_t* chunk_hist;   // [chunks][P][256] digit counts of each input range (K1)
  uint32_t* ctab;         // [3][chunks][256] per-range counts of the next executed digit
  int chunks;
  uint32_t chunk_keys;
  uint32_t chunk_magic;   // ceil(2^32 / chunk_keys): range of position p = umulhi(p, magic) (-1)
  // 1: K1 chooses the scheme from the digit counts (plan->use_lookback); both the chunked and
  // the look-back passes are launched and the ones not chosen return at once.  The look-back
  // status buffers (status[]) are then separate from the chunked tables.
  int choose_lookback;
};
constexpr int TRACE_WORDS = 7;

__device__ __forceinline__ uint32_t sm_id() {
  uint32_t v;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(v));
  return v;
}

// =====================================================================================
// K1: fused all-digit histogram (+ plan in the last CTA)
// =====================================================================================
// Counters are privatised per lane: bin b of digit d for lane l lives at word
// (d*256 + b)*COPIES + l % COPIES, so the 32 shared atomics of one warp instruction fall in
// (nearly) distinct banks whatever the key values -- one shared-memory wavefront each
// instead of ~3.3 for random bins.  32-bit keys: 32 copies (4 x 256 x 32 words = 128 KiB);
// 64-bit keys: 16 copies (8 x 256 x 16 words = 128 KiB).
template <class U>
struct HistSmem {
  static constexpr int P = int(sizeof(U));
  static constexpr int COPIES = P == 4 ? 32 : 16;
  static constexpr size_t BYTES = size_t(P) * RADIX * COPIES * 4;
};

// 16-byte vectors in flight per thread in the histogram's read (8 x 16 B x 1024 threads = 128 KiB
// per SM).
#ifndef HPCS_HIST_VIF
#define HPCS_HIST_VIF 8
#endif

// cta / ncta: this CTA's index and the CTA count of this array's histogram (the grid of a
// single-array launch; the array's ranges in the batched sort's grid-level launch).
template <class U, int KIND, int NT>
__device__ __forceinline__ void hist_all_digits_body(const U* __restrict__ keys, int64_t n,
                                                     uint32_t* __restrict__ hist_out, const SortArgs& args,
                                                     int make_plan, const int cta, const int ncta) {
  constexpr int P = HistSmem<U>::P;
  constexpr int COPIES = HistSmem<U>::COPIES;
  constexpr int VEC = 16 / int(sizeof(U));
  using KO = KeyOrder<U, KIND>;
  extern __shared__ __align__(16) uint32_t sh[];  // [P][256][COPIES]
  __shared__ uint32_t s_last;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int copy = lane & (COPIES - 1);
  for (int i = tid; i < P * RADIX * COPIES; i += NT) sh[i] = 0;
  __syncthreads();

  auto count_key = [&](U k) {
    const U o = KO::to_ordered(k);
#pragma unroll
    for (int d = 0; d < P; d++) {
      const uint32_t dg = uint32_t(o >> (8 * d)) & 0xFFu;
      atomicAdd(&sh[(d * RADIX + dg) * COPIES + copy], 1u);
    }
  };

  // Grid-stride over all vectors, or (chunked) CTA j over the vectors of key range j.
  const bool chunked = args.chunk_hist != nullptr;
  const int64_t nvec = n / VEC;
  const uint4* vkeys = reinterpret_cast<const uint4*>(keys);
  int64_t vend = nvec, stride = int64_t(ncta) * NT;
  int64_t i = int64_t(cta) * NT + tid;
  bool owns_tail = cta == 0;
  if (chunked) {
    const int64_t lo = int64_t(cta) * args.chunk_keys;  // a multiple of VEC
    const int64_t hi = lo + args.chunk_keys < n ? lo + args.chunk_keys : n;
    i = lo / VEC + tid;
    vend = hi / VEC;
    stride = NT;
    owns_tail = hi == n;
  }
  // HPCS_HIST_VIF vectors in flight per thread per iteration
  for (; i + (HPCS_HIST_VIF - 1) * stride < vend; i += HPCS_HIST_VIF * stride) {
    uint4 v[HPCS_HIST_VIF];
#pragma unroll
    for (int u = 0; u < HPCS_HIST_VIF; u++) v[u] = ldg_stream_v4(vkeys + i + u * stride);
#pragma unroll
    for (int u = 0; u < HPCS_HIST_VIF; u++) {
      const U* e = reinterpret_cast<const U*>(&v[u]);
#pragma unroll
      for (int j = 0; j < VEC; j++) count_key(e[j]);
    }
  }
  for (; i < vend; i += stride) {
    const uint4 v = ldg_stream_v4(vkeys + i);
    const U* e = reinterpret_cast<const U*>(&v);
#pragma unroll
    for (int j = 0; j < VEC; j++) count_key(e[j]);
  }
  // ragged tail (fewer than VEC keys)
  if (owns_tail && tid < VEC) {
    const int64_t t = nvec * VEC + tid;
    if (t < n) count_key(keys[t]);
  }
  __syncthreads();
  // fold the copies (rotated start so a warp's reads hit distinct banks) into the output,
  // and (chunked) into this range's row of per-range counts
  uint32_t* crow = chunked ? args.chunk_hist + int64_t(cta) * P * RADIX : nullptr;
  for (int j = tid; j < P * RADIX; j += NT) {
    uint32_t c = 0;
#pragma unroll 8
    for (int q = 0; q < COPIES; q++) c += sh[j * COPIES + ((q + lane) & (COPIES - 1))];
    if (c) atomicAdd(hist_out + j, c);
    if (chunked) crow[j] = c;
  }

  if (!make_plan) return;

  if (chunked) {
    // the first executed pass adds its next-digit counts into table 1
    uint32_t* t1 = args.ctab + (int64_t(args.chunks) + cta) * RADIX;
    for (int j = tid; j < RADIX; j += NT) t1[j] = 0;
  } else {
    // Zero the first look-back buffer for the first executed pass.
    uint32_t* s0 = args.status[0];
    const int64_t words = int64_t(args.num_tiles) * RADIX;
    const int64_t gstride = int64_t(ncta) * NT;
    for (int64_t w = int64_t(cta) * NT + tid; w < words; w += gstride) s0[w] = 0;
  }
  // Last-block-done: the final CTA builds the plan.
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = (atomicAdd(&args.plan->done_blocks, 1u) == uint32_t(ncta) - 1u) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  SortPlan* plan = args.plan;
  __shared__ uint32_t s_trivial[P];
  __shared__ uint32_t s_wsum[RADIX / 32];
  __shared__ unsigned long long s_heavy[P];
  __shared__ unsigned long long s_heavy2[P];
  for (int d = 0; d < P; d++) {
    uint32_t c = 0;
    if (tid < RADIX) {
      c = ld_volatile(&hist_out[d * RADIX + tid]);
    }
    if (tid == 0) {
      s_trivial[d] = 0;
      s_heavy[d] = 0ull;
      s_heavy2[d] = 0ull;
    }
    __syncthreads();
    if (tid < RADIX && int64_t(c) == n) s_trivial[d] = 1;
    // most frequent value: max of (count, 255 - value); then the most frequent of the others
    const unsigned long long packed = (static_cast<unsigned long long>(c) << 8) | uint32_t(255 - tid);
    if (tid < RADIX && c) atomicMax(&s_heavy[d], packed);
    __syncthreads();
    if (tid < RADIX && c && packed != s_heavy[d]) atomicMax(&s_heavy2[d], packed);
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
    int sel = 0, executed = 0, prev = -1;
    for (int d = 0; d < MAX_PASSES; d++) {
      plan->tile_counter[d] = 0;
      plan->exec_idx[d] = -1;
      plan->next_shift[d] = -1;
      plan->heavy[d] = d < P ? int(255u - uint32_t(s_heavy[d] & 255ull)) : 0;
      plan->skewed[d] = d < P && int64_t(s_heavy[d] >> 8) > n / 32 ? 1 : 0;
      plan->heavy2[d] = d < P && s_heavy2[d] ? int(255u - uint32_t(s_heavy2[d] & 255ull)) : plan->heavy[d];
      plan->grouped[d] = d < P && int64_t(s_heavy[d] >> 8) + int64_t(s_heavy2[d] >> 8) > n / 4 * 3 ? 1 : 0;
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
        plan->exec_idx[d] = executed;
        if (prev >= 0) plan->next_shift[prev] = 8 * d;
        prev = d;
        sel ^= 1;
        executed++;
      }
    }
    plan->final_sel = sel;
    // Device-chosen passes: look-back when an executed digit has one value above 1/8 of the
    // keys but no two values holding 3/4 of them (several frequent values, as in the sign and
    // exponent byte of normally distributed floats): counting those for the next pass's
    // per-range tables costs the chunked passes more than the look-back.  Otherwise chunked.
    int lb = 0;
    if (args.choose_lookback)
      for (int d = 0; d < P; d++)
        if (plan->exec_idx[d] >= 0 && int64_t(s_heavy[d] >> 8) > n / 8 && !plan->grouped[d]) lb = 1;
    plan->use_lookback = lb;
    __threadfence();
  }
}

template <class U, int KIND, int NT>
__global__ void __launch_bounds__(NT, 1) hist_all_digits_kernel(const U* __restrict__ keys, int64_t n,
                                                                 uint32_t* __restrict__ hist_out,
                                                                 SortArgs args, int make_plan) {
  hist_all_digits_body<U, KIND, NT>(keys, n, hist_out, args, make_plan, int(blockIdx.x), int(gridDim.x));
}

// The fused histogram (and plan) of many arrays in one launch (the batched sort's grid-level
// path): CTA c counts range map[c].y of array map[c].x, whose sort arguments are args[map[c].x].
template <class U, int KIND, int NT>
__global__ void __launch_bounds__(NT, 1) seg_hist_all_digits_kernel(const SortArgs* __restrict__ args,
                                                                    const int2* __restrict__ map) {
  const int2 m = map[blockIdx.x];
  const SortArgs a = args[m.x];
  hist_all_digits_body<U, KIND, NT>(static_cast<const U*>(a.keys_a), a.n, &a.plan->hist[0][0], a, 1, m.y, a.chunks);
}

// =====================================================================================
// K3: one 8-bit digit pass (onesweep)
// =====================================================================================
//
// In-warp stable ranking.  Keys sit warp-striped (key i of lane l is tile position
// w*32*KPT + i*32 + l), so a warp's keys in (i, lane) order are in input order.  Each warp
// owns 256 digit counters in shared memory; the rank of a key among the warp's earlier
// keys with the same digit is
//   RANK_ORDERED_ATOMIC  the value returned by one shared-memory atomicAdd per key.  This
//                        relies on the hardware resolving same-address atomics of one warp
//                        instruction in ascending lane order.  PTX leaves that order
//                        undefined, so every context verifies it first with
//                        rank_probe_kernel (the same code path) and otherwise uses:
//   RANK_PEER_MASK       fully defined: each lane ORs its lane bit into a per-(warp, digit)
//                        mask; after __syncwarp the mask is the set of same-digit lanes
//                        (the peers), the rank is counter + popc(peers below me), and the
//                        lowest peer advances the counter and clears the mask.
// Both give identical ranks.  (__match_any_sync / ballots would also be defined but
// run 10-20x slower than one shared atomic on this part.)
enum RankMode : int { RANK_ORDERED_ATOMIC = 0, RANK_PEER_MASK = 1 };

template <int MODE>
__device__ __forceinline__ uint32_t rank_in_warp(uint32_t* cnt, uint32_t* msk, uint32_t d, bool valid, int parity,
                                                 int lane) {
  if (MODE == RANK_ORDERED_ATOMIC) {
    return valid ? atomicAdd(&cnt[d], 1u) : 0u;
  } else {
    uint32_t* m = msk + parity * RADIX + (valid ? d : 0u);
    if (valid) atomicOr(m, 1u << lane);
    __syncwarp();
    const uint32_t peers = valid ? *reinterpret_cast<volatile uint32_t*>(m) : 0u;
    const uint32_t before = valid ? cnt[d] : 0u;
    const uint32_t lt = peers & lanemask_lt();
    __syncwarp();
    if (valid && lt == 0u) {
      cnt[d] = before + __popc(peers);
      *m = 0u;
    }
    return before + __popc(lt);
  }
}

// Ordered-atomic ranking for a pass whose two most frequent digit values h1, h2 hold much of
// the keys: the lanes of a warp instruction holding h1 (or h2) take one atomicAdd of their
// count, made by the lowest of them, and rank among themselves by popcount, instead of
// serialising on one counter; other lanes rank with their own atomic.  Same ranks as
// rank_in_warp<RANK_ORDERED_ATOMIC>.  All lanes must call it (it uses warp votes).
__device__ __forceinline__ uint32_t rank_in_warp_top2(uint32_t* cnt, uint32_t d, bool valid, uint32_t h1,
                                                      uint32_t h2, int lane) {
  const bool is1 = valid && d == h1;
  const bool is2 = valid && d == h2 && h2 != h1;
  const uint32_t m1 = __ballot_sync(0xFFFFFFFFu, is1);
  const uint32_t m2 = __ballot_sync(0xFFFFFFFFu, is2);
  const int l1 = m1 ? __ffs(m1) - 1 : 0;
  const int l2 = m2 ? __ffs(m2) - 1 : 0;
  uint32_t b1 = 0, b2 = 0, r = 0;
  if (m1 && lane == l1) b1 = atomicAdd(&cnt[h1], uint32_t(__popc(m1)));
  if (m2 && lane == l2) b2 = atomicAdd(&cnt[h2], uint32_t(__popc(m2)));
  if (valid && !is1 && !is2) r = atomicAdd(&cnt[d], 1u);
  b1 = __shfl_sync(0xFFFFFFFFu, b1, l1);
  b2 = __shfl_sync(0xFFFFFFFFu, b2, l2);
  if (is1) r = b1 + uint32_t(__popc(m1 & lanemask_lt()));
  if (is2) r = b2 + uint32_t(__popc(m2 & lanemask_lt()));
  return r;
}

template <class U, class V, int NT, int KPT, int STAGES, int MODE>
struct OnesweepSmem {
  static constexpr bool PAIRS = !std::is_same<V, NoValue>::value;
  static constexpr int TILE = NT * KPT;
  static constexpr int NW = NT / 32;
  static constexpr size_t KEYS_BYTES = size_t(TILE) * sizeof(U);
  static constexpr size_t VALS_BYTES = PAIRS ? size_t(TILE) * 4 : 0;
  static constexpr size_t STAGE_BYTES = KEYS_BYTES + VALS_BYTES;
  static constexpr size_t OFF_STAGES = 0;
  static constexpr size_t OFF_CNT = OFF_STAGES + STAGE_BYTES * STAGES;      // [NW][256]
  static constexpr size_t OFF_MSK = OFF_CNT + size_t(NW) * RADIX * 4;        // [NW][2][256]
  static constexpr size_t MSK_BYTES = MODE == RANK_PEER_MASK ? size_t(NW) * 2 * RADIX * 4 : 0;
  static constexpr size_t OFF_BINSTART = OFF_MSK + MSK_BYTES;
  static constexpr size_t OFF_LOCAL = OFF_BINSTART + RADIX * 4;
  static constexpr size_t OFF_GBASE = OFF_LOCAL + RADIX * 4;
  static constexpr size_t OFF_TOT = OFF_GBASE + RADIX * 4;   // this CTA's digit totals
  static constexpr size_t OFF_CPRE = OFF_TOT + RADIX * 4;    // earlier CTAs of the unit
  static constexpr size_t OFF_EXCL = OFF_CPRE + RADIX * 4;   // unit exclusive prefix (rank 0)
  static constexpr size_t OFF_WSUM = OFF_EXCL + RADIX * 4;
  static constexpr size_t OFF_TILE = OFF_WSUM + 32 * 4;
  static constexpr size_t OFF_MBAR = (OFF_TILE + 16 + 7) / 8 * 8;
  static constexpr size_t BYTES = OFF_MBAR + 8 * STAGES;
};

// Issue the bulk copy of sub-tile `sub` into stage s (called by one thread).  The
// 16-byte-aligned body is copied by the TMA engine; the ragged tail (< 16 bytes) is read
// with plain loads by the consumers.  Stage buffers start at offset 0 of the dynamic
// shared memory.  A sub-tile past the end arrives with zero bytes.
template <class U, bool PAIRS, int TILE>
__device__ __forceinline__ void onesweep_issue_tile(unsigned char* smem, size_t stage_bytes, size_t keys_bytes,
                                                    uint64_t* mbar, const U* kin, const uint32_t* vin,
                                                    int64_t n, int64_t sub, int s) {
  const int64_t base = sub * TILE;
  int64_t cnt = n - base;
  cnt = cnt < 0 ? 0 : (cnt < TILE ? cnt : TILE);
  const uint32_t kbytes = uint32_t((cnt * int64_t(sizeof(U))) & ~int64_t(15));
  const uint32_t vbytes = PAIRS ? uint32_t((cnt * 4) & ~int64_t(15)) : 0u;
  unsigned char* dst = smem + size_t(s) * stage_bytes;
  fence_proxy_async_smem();
  mbar_arrive_expect_tx(&mbar[s], kbytes + vbytes);
  if (kbytes) bulk_copy_g2s(dst, kin + base, kbytes, &mbar[s]);
  if (PAIRS && vbytes) bulk_copy_g2s(dst + keys_bytes, vin + base, vbytes, &mbar[s]);
}

// Barrier over the CTAs of a cluster (all threads), or over the CTA when CL == 1.
template <int CL>
__device__ __forceinline__ void unit_sync() {
  if (CL > 1) {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
  } else {
    __syncthreads();
  }
}

// Address of `p` (a shared-memory location of this CTA) in the CTA of cluster rank `r`.
template <class T>
__device__ __forceinline__ T* cluster_peer(T* p, uint32_t r) {
  return cooperative_groups::this_cluster().map_shared_rank(p, r);
}

// One onesweep digit pass.  The look-back unit is a cluster of CL CTAs: the CTAs of a
// cluster each stage, rank and reorder their own TILE-key sub-tile, exchange their digit
// totals through distributed shared memory, and cluster rank 0 publishes one aggregate and
// runs one look-back for all CL x TILE keys.  This divides the rate at which look-back
// units are produced by CL: a decoupled look-back advances at most LB_WINDOW units per L2
// round trip, which otherwise caps a B200 pass well below its HBM bandwidth.
template <class U, int KIND, class V, int NT, int KPT, int STAGES, int MINB, int MODE, int CL>
__global__ void __launch_bounds__(NT, MINB) onesweep_pass_kernel(SortArgs args) {
  using L = OnesweepSmem<U, V, NT, KPT, STAGES, MODE>;
  using KO = KeyOrder<U, KIND>;
  constexpr bool PAIRS = L::PAIRS;
  constexpr int TILE = L::TILE;
  constexpr int NW = L::NW;
  static_assert(NT >= RADIX && NT % 32 == 0, "one thread per digit needed");
  static_assert(STAGES == 2, "two stages: one being processed, one being filled");

  const SortPlan* plan = args.plan;
  const int pass = args.pass;
  if (args.choose_lookback && !plan->use_lookback) return;  // the chunked passes were chosen
  const int sel = plan->src_sel[pass];
  if (sel < 0) return;  // every key has the same digit here: the pass is the identity (uniform)
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
  const int num_units = args.num_tiles;  // look-back units (clusters of CL sub-tiles)
  const uint32_t crank = CL > 1 ? cooperative_groups::this_cluster().block_rank() : 0u;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + L::OFF_CNT);  // [NW][256]
  uint32_t* s_msk = reinterpret_cast<uint32_t*>(smem + L::OFF_MSK);  // [NW][2][256] (peer-mask mode)
  uint32_t* s_binstart = reinterpret_cast<uint32_t*>(smem + L::OFF_BINSTART);
  uint32_t* s_local = reinterpret_cast<uint32_t*>(smem + L::OFF_LOCAL);
  uint32_t* s_gbase = reinterpret_cast<uint32_t*>(smem + L::OFF_GBASE);
  uint32_t* s_tot = reinterpret_cast<uint32_t*>(smem + L::OFF_TOT);
  uint32_t* s_cpre = reinterpret_cast<uint32_t*>(smem + L::OFF_CPRE);
  uint32_t* s_excl = reinterpret_cast<uint32_t*>(smem + L::OFF_EXCL);
  uint32_t* s_wsum = reinterpret_cast<uint32_t*>(smem + L::OFF_WSUM);
  int* s_tile = reinterpret_cast<int*>(smem + L::OFF_TILE);
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(smem + L::OFF_MBAR);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* cnt_w = s_cnt + warp * RADIX;
  uint32_t* msk_w = s_msk + warp * 2 * RADIX;

  // Rank 0 takes the next unit and writes its id into every CTA of the cluster.
  auto acquire_and_broadcast = [&](int slot) {
    const int u = int(atomicAdd(tile_counter, 1u));
    if (CL > 1) {
      for (uint32_t q = 0; q < uint32_t(CL); q++) *cluster_peer(&s_tile[slot], q) = u;
    } else {
      s_tile[slot] = u;
    }
  };

  if (tid == 0) {
    for (int st = 0; st < STAGES; st++) mbar_init(&s_mbar[st], 1);
    fence_mbar_init();
    fence_proxy_async_smem();
  }
  for (int i = tid; i < RADIX; i += NT) s_binstart[i] = plan->bin_start[pass][i];
  if (MODE == RANK_PEER_MASK)
    for (int i = lane; i < 2 * RADIX; i += 32) msk_w[i] = 0u;
  if (CL > 1) unit_sync<CL>();  // peers' shared memory is live before remote writes
  if (crank == 0 && tid == 0) acquire_and_broadcast(0);
  unit_sync<CL>();
  if (tid == 0 && s_tile[0] < num_units)
    onesweep_issue_tile<U, PAIRS, TILE>(smem, L::STAGE_BYTES, L::KEYS_BYTES, s_mbar, kin, vin, n,
                                        int64_t(s_tile[0]) * CL + crank, 0);

  uint32_t phase_bits = 0;  // bit s = parity to wait for on stage s
  int stage = 0;
  for (;;) {
    const int u = s_tile[stage];  // the same in every CTA of the cluster
    if (u >= num_units) break;
    // next unit: taken now (one iteration ahead), issued after the first cluster barrier
    if (crank == 0 && tid == 0) acquire_and_broadcast(stage ^ 1);
    const int64_t tile_base = (int64_t(u) * CL + crank) * TILE;
    int64_t tn64 = n - tile_base;
    const int tile_n = int(tn64 < 0 ? 0 : (tn64 < TILE ? tn64 : TILE));
    const int bulk_keys = int((int64_t(tile_n) * int64_t(sizeof(U))) & ~int64_t(15)) / int(sizeof(U));
    const int bulk_vals = PAIRS ? int((int64_t(tile_n) * 4) & ~int64_t(15)) / 4 : 0;
    uint64_t* trace = (args.trace && pass == args.trace_pass && u < args.trace_capacity && tid == 0 && crank == 0)
                          ? args.trace + int64_t(u) * TRACE_WORDS
                          : nullptr;
    if (trace) {
      trace[0] = uint64_t(u);
      trace[1] = sm_id();
      trace[2] = global_timer_ns();
    }

    // zero this warp's digit counters
    for (int i = lane; i < RADIX; i += 32) cnt_w[i] = 0u;

    // wait for the staged sub-tile (bounded)
    if (!mbar_wait_bounded(&s_mbar[stage], (phase_bits >> stage) & 1u, args.spin_limit_ns)) {
      if (lane == 0) atomicOr(err, uint32_t(DERR_TMA_TIMEOUT));
    }
    phase_bits ^= (1u << stage);
    __syncwarp();
    if (trace) trace[3] = global_timer_ns();

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
      rank[i] = rank_in_warp<MODE>(cnt_w, msk_w, KO::digit(key[i], shift), valid, i & 1, lane);
    }
    __syncthreads();  // (A) warp counts complete; stage buffer no longer read
    if (trace) trace[4] = global_timer_ns();

    // ---- per digit: sub-tile total and scan over digits -------------------------------
    if (tid < RADIX) {
      const int dg = tid;
      uint32_t total = 0;
#pragma unroll
      for (int w = 0; w < NW; w++) total += s_cnt[w * RADIX + dg];
      s_tot[dg] = total;
      uint32_t incl = total;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      s_local[dg] = incl - total;  // exclusive within this warp of digits for now
      if (lane == 31) s_wsum[warp] = incl;
    }
    __syncthreads();  // (B)
    // sub-tile start of each digit; counters become (digit start + earlier warps' count)
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
    unit_sync<CL>();  // (C1) offsets ready; every CTA's totals and the next unit id visible

    // prefetch the next sub-tile into the other stage (its previous contents are done)
    if (tid == 0) {
      const int un = s_tile[stage ^ 1];
      if (un < num_units)
        onesweep_issue_tile<U, PAIRS, TILE>(smem, L::STAGE_BYTES, L::KEYS_BYTES, s_mbar, kin, vin, n,
                                            int64_t(un) * CL + crank, stage ^ 1);
    }

    // ---- unit totals, aggregate, decoupled look-back (rank 0), overlapped with reorder ----
    if (tid < RADIX) {
      const int dg = tid;
      uint32_t utot = 0, cpre = 0;
      if (CL > 1) {
#pragma unroll
        for (int q = 0; q < CL; q++) {
          const uint32_t v = *cluster_peer(&s_tot[dg], uint32_t(q));
          utot += v;
          cpre += (q < int(crank)) ? v : 0u;
        }
      } else {
        utot = s_tot[dg];
      }
      s_cpre[dg] = cpre;
      if (crank == 0) {
        if (u != args.poison_tile) {
          if (u == 0) st_relaxed_gpu(&status[dg], ST_PREFIX | utot);
          else st_relaxed_gpu(&status[int64_t(u) * RADIX + dg], ST_AGGREGATE | utot);
        }
        uint32_t excl = 0;
        if (u > 0) {
          // Windowed walk: read LB_WINDOW predecessors' words at once (independent
          // loads), sum the ready ones from the nearest outward and stop at the first
          // inclusive prefix.
          int j = u - 1;
          uint64_t t0 = 0;
          bool timed_out = false;
          while (true) {
            uint32_t wv[LB_WINDOW];
#pragma unroll
            for (int q = 0; q < LB_WINDOW; q++)
              wv[q] = (j - q >= 0) ? ld_relaxed_gpu(&status[int64_t(j - q) * RADIX + dg]) : (ST_PREFIX | 0u);
            int used = 0;
            bool found = false;
#pragma unroll
            for (int q = 0; q < LB_WINDOW; q++) {
              if (used == q) {  // still contiguous from the nearest predecessor
                const uint32_t v = wv[q];
                if ((v & ST_FLAGS) != 0) {
                  excl += v & ST_VALUE;
                  used = q + 1;
                  if (v & ST_PREFIX) found = true;
                }
              }
              if (found) break;
            }
            if (found) break;
            j -= used;
            if (used == 0) {
              // nearest predecessor not published yet: spin on that one word with a short
              // back-off (frees issue slots for the reordering warps), bounded in time
              uint32_t v;
              while (((v = ld_relaxed_gpu(&status[int64_t(j) * RADIX + dg])) & ST_FLAGS) == 0) {
                __nanosleep(32);
                if (t0 == 0) t0 = global_timer_ns();
                else if (global_timer_ns() - t0 > args.spin_limit_ns || ld_volatile(err) != 0u) {
                  timed_out = true;
                  break;
                }
              }
              if (timed_out) break;
            }
          }
          if (timed_out) atomicOr(err, uint32_t(DERR_LOOKBACK_TIMEOUT));
          if (u != args.poison_tile)
            st_relaxed_gpu(&status[int64_t(u) * RADIX + dg], ST_PREFIX | ((excl + utot) & ST_VALUE));
        }
        s_excl[dg] = excl;
        // zero-ahead: clear this unit's words in the buffer the next executed pass uses
        status_next[int64_t(u) * RADIX + dg] = 0;
        if (trace) trace[5] = global_timer_ns();
      }
    }

    // ---- reorder the sub-tile in shared memory by digit -------------------------------
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      if (idx < tile_n) {
        const uint32_t d = KO::digit(key[i], shift);
        const uint32_t pos = cnt_w[d] + rank[i];
        rank[i] = pos;  // keep the tile position for the payload
        sk[pos] = key[i];
      }
    }
    unit_sync<CL>();  // (C2) rank 0's unit prefixes visible; reordered keys ready
    if (tid < RADIX) {
      const int dg = tid;
      const uint32_t excl = CL > 1 ? *cluster_peer(&s_excl[dg], 0u) : s_excl[dg];
      s_gbase[dg] = s_binstart[dg] + excl + s_cpre[dg] - s_local[dg];
    }
    __syncthreads();  // (D) global bases ready

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
      __syncthreads();  // (E1) all payloads read before they are overwritten
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int idx = wbase + i * 32 + lane;
        if (idx < tile_n) sv[rank[i]] = val[i];
      }
      __syncthreads();  // (E2)
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
    if (trace) trace[6] = global_timer_ns();
    // The stage buffer was written through the generic proxy; a later bulk copy (async
    // proxy) refills it, so order the writes before the barrier.
    fence_proxy_async_smem();
    __syncthreads();  // (F) shared memory free for the next sub-tile
    stage ^= 1;
  }
  // no CTA may exit while a peer can still read its shared memory
  if (CL > 1) unit_sync<CL>();
}

// Verifies, on this GPU, that the ordered-atomic ranking gives lane-ordered (stable) ranks:
// every warp ranks KPT x 32 digits with exactly the onesweep's code and compares each rank
// with a brute-force count of earlier equal digits.  Patterns: uniform bytes, 4 values,
// one value, and partial last rows.  Mismatches are added to *bad.
template <int NT, int KPT>
__global__ void __launch_bounds__(NT) rank_probe_kernel(uint32_t* bad, uint32_t seed) {
  constexpr int NW = NT / 32;
  __shared__ uint32_t cnt[NW][RADIX];
  __shared__ uint16_t dig[NW][32 * KPT];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t mism = 0;
  for (int pattern = 0; pattern < 4; pattern++) {
    for (int i = lane; i < RADIX; i += 32) cnt[warp][i] = 0u;
    const int valid_n = pattern == 3 ? (32 * KPT - 37) : 32 * KPT;
    __syncwarp();
    uint32_t x = seed ^ (blockIdx.x * 0x9E3779B9u) ^ (threadIdx.x * 0x85EBCA6Bu) ^ (pattern * 0xC2B2AE35u);
    uint32_t d[KPT], r[KPT];
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      x ^= x << 13;
      x ^= x >> 17;
      x ^= x << 5;
      d[i] = pattern == 0 ? (x & 255u) : pattern == 1 ? (x & 3u) : pattern == 2 ? 9u : ((x >> 3) & 7u);
      dig[warp][i * 32 + lane] = uint16_t(d[i]);
    }
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const bool valid = i * 32 + lane < valid_n;
      r[i] = rank_in_warp<RANK_ORDERED_ATOMIC>(cnt[warp], nullptr, d[i], valid, i & 1, lane);
    }
    __syncwarp();
    for (int i = 0; i < KPT; i++) {
      const int pos = i * 32 + lane;
      if (pos >= valid_n) continue;
      uint32_t want = 0;
      for (int q = 0; q < pos; q++) want += (dig[warp][q] == d[i]) ? 1u : 0u;
      if (want != r[i]) mism++;
    }
    __syncwarp();
  }
  if (mism) atomicAdd(bad, mism);
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

// The batched sort's grid-level path: CTA c copies range map[c].y of array map[c].x back into
// the caller's buffer when that array's result ended in its scratch buffer (an odd number of
// passes ran), and the array's first CTA folds its device error bits into the context's word.
template <class U>
__global__ void seg_finalize_kernel(const SortArgs* __restrict__ args, const int2* __restrict__ map,
                                    uint32_t* err_accum) {
  const int2 m = map[blockIdx.x];
  const SortArgs a = args[m.x];
  if (m.y == 0 && threadIdx.x == 0) {
    const uint32_t e = ld_volatile(&a.plan->error);
    if (e) atomicOr(err_accum, e);
  }
  if (a.plan->final_sel != 1) return;
  const int64_t lo = int64_t(m.y) * a.chunk_keys;
  const int64_t hi = lo + a.chunk_keys < a.n ? lo + a.chunk_keys : a.n;
  const U* src = static_cast<const U*>(a.keys_b);
  U* dst = static_cast<U*>(a.keys_a);
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) dst[i] = src[i];
}

}  // namespace hpcs
