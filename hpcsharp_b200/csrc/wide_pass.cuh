// Wide-digit LSD passes (sm_100a): digits of up to 11 bits, so a 32-bit key takes 3 passes
// instead of 4 (bits [0,11), [11,22), [22,32)).
//
// The digit order, the order transforms and the stability are those of the 8-bit passes, so the
// sorted result is the same: an LSD sort whose every pass is stable orders the keys by all their
// bits whatever the digit widths.  The reference's 8-bit digits (RadixSortLsd.cs:1136-1143) are a
// CPU choice; on this GPU a pass is bound by the shared-memory work per key (a ranking atomic, a
// counter lookup, a reorder store), which does not grow with the digit width, so fewer, wider
// passes do less of it.
//
// Each pass k runs three kernels over the same J key ranges (range j = CTA j, a whole number of
// tiles, as in the chunked 8-bit passes):
//   wide_count  per-range counts of digit k of the pass's input (one read of the keys; the
//               counters are spread over 16 lane copies so a warp's atomics rarely share a bank)
//   wide_plan   for every digit: the total over ranges and, per range, the sum over the ranges
//               before it; marks the pass as the identity when one digit value holds every key
//   wide_pass   per tile: rank each key within its warp (one shared atomic on 16-bit counters),
//               scan over (digit, warp), reorder the tile in shared memory by digit and write
//               coalesced per-digit runs.  The global start of digit d in range j is
//               bin_start[d] + (keys of digit d in ranges < j) + a running offset carried from
//               tile to tile, so no CTA waits for another.
// The first pass's counts come from the same count kernel run on the caller's keys.
#pragma once
#include "radix_kernels.cuh"

namespace hpcs {

constexpr int WIDE_MAX_BITS = 11;
constexpr int WIDE_MAX_BINS = 1 << WIDE_MAX_BITS;
constexpr int WIDE_MAX_PASSES = 6;  // 64-bit keys: 6 x 11 bits (the last two 10)

// Per-sort control block of the wide passes (device memory, zeroed before the first count).
struct WidePlan {
  int32_t in_sel[WIDE_MAX_PASSES];  // buffer the pass reads: 0 = A (caller), 1 = B (scratch)
  int32_t skip[WIDE_MAX_PASSES];    // 1: every key has the same digit value, the pass is the identity
  uint32_t error;                   // DeviceError bits
  uint32_t done_ctas;               // last-CTA-done counter of the plan kernel
};

struct WideArgs {
  void* keys_a;
  void* keys_b;
  void* vals_a;
  void* vals_b;
  int64_t n;
  WidePlan* plan;
  uint32_t* rcount;    // [J][bins]: counts of digit k per range (the count kernel's output)
  uint32_t* rprefix;   // [J][bins]: counts of digit k in the ranges before j
  uint32_t* totals;    // [bins]
  int pass;
  int shift;           // first bit of the digit
  int bits;            // digit width
  int ranges;          // J
  uint32_t range_keys; // L (a whole number of tiles of the pass kernel)
  uint64_t spin_limit_ns;
};

// Digit of a key with the order transform applied (signed: flip the top bit; float: sign 0
// flips the sign bit, sign 1 flips every bit; Histogram.cs:1210-1288).
template <class U, int KIND>
__device__ __forceinline__ uint32_t wide_digit(U x, int shift, uint32_t mask) {
  return uint32_t(KeyOrder<U, KIND>::to_ordered(x) >> shift) & mask;
}

// Buffer the input of pass `pass` lives in: the previous pass's input, flipped if it ran.
__device__ __forceinline__ int wide_src_sel(const WidePlan* plan, int pass) {
  if (pass == 0) return 0;
  return plan->in_sel[pass - 1] ^ (plan->skip[pass - 1] ? 0 : 1);
}

// Rank of a key among the earlier keys of its warp with the same digit, on 16-bit counters two
// to a word: the value an ordered shared atomic returns.  When a digit value is frequent (skewed
// digits: the top bits of small signed or float keys, low-entropy keys) the lanes of a warp
// instruction holding the two most frequent values h1, h2 take one atomic per value, made by the
// lowest of them, and rank among themselves by popcount instead of serialising on one counter;
// the other lanes rank with their own atomic.  All lanes call it when `grouped` (warp votes).
__device__ __forceinline__ uint32_t wide_rank(uint32_t* cnt_w, uint32_t d, bool valid, bool grouped, uint32_t h1,
                                              uint32_t h2, int lane) {
  if (!grouped) {
    if (!valid) return 0u;
    const uint32_t sh = (d & 1u) << 4;
    return (atomicAdd(cnt_w + (d >> 1), 1u << sh) >> sh) & 0xFFFFu;
  }
  const bool is1 = valid && d == h1;
  const bool is2 = valid && d == h2 && h2 != h1;
  const uint32_t m1 = __ballot_sync(0xFFFFFFFFu, is1);
  const uint32_t m2 = __ballot_sync(0xFFFFFFFFu, is2);
  const int l1 = m1 ? __ffs(m1) - 1 : 0;
  const int l2 = m2 ? __ffs(m2) - 1 : 0;
  uint32_t b1 = 0, b2 = 0, r = 0;
  if (m1 && lane == l1) {
    const uint32_t sh = (h1 & 1u) << 4;
    b1 = (atomicAdd(cnt_w + (h1 >> 1), uint32_t(__popc(m1)) << sh) >> sh) & 0xFFFFu;
  }
  if (m2 && lane == l2) {
    const uint32_t sh = (h2 & 1u) << 4;
    b2 = (atomicAdd(cnt_w + (h2 >> 1), uint32_t(__popc(m2)) << sh) >> sh) & 0xFFFFu;
  }
  if (valid && !is1 && !is2) {
    const uint32_t sh = (d & 1u) << 4;
    r = (atomicAdd(cnt_w + (d >> 1), 1u << sh) >> sh) & 0xFFFFu;
  }
  b1 = __shfl_sync(0xFFFFFFFFu, b1, l1);
  b2 = __shfl_sync(0xFFFFFFFFu, b2, l2);
  if (is1) r = b1 + uint32_t(__popc(m1 & lanemask_lt()));
  if (is2) r = b2 + uint32_t(__popc(m2 & lanemask_lt()));
  return r;
}

// ---------------------------------------------------------------------------------------
// wide_count: CTA j counts digit `pass` of the keys of range j.
// ---------------------------------------------------------------------------------------
constexpr int WIDE_COUNT_NT = 1024;
constexpr int WIDE_COUNT_COPIES = 16;
constexpr size_t WIDE_COUNT_SMEM = size_t(WIDE_MAX_BINS) * WIDE_COUNT_COPIES * 4;  // 128 KiB

template <class U, int KIND>
__global__ void __launch_bounds__(WIDE_COUNT_NT, 1) wide_count_kernel(WideArgs args) {
  constexpr int VEC = 16 / int(sizeof(U));
  extern __shared__ __align__(16) uint32_t cnt[];  // [bins][COPIES]
  const int tid = threadIdx.x, lane = tid & 31;
  const int bins = 1 << args.bits;
  const uint32_t mask = uint32_t(bins - 1);
  const int copy = lane & (WIDE_COUNT_COPIES - 1);
  const WidePlan* plan = args.plan;
  const int sel = wide_src_sel(plan, args.pass);
  if (tid == 0 && blockIdx.x == 0) args.plan->in_sel[args.pass] = sel;
  const U* __restrict__ keys = static_cast<const U*>(sel ? args.keys_b : args.keys_a);
  for (int i = tid; i < bins * WIDE_COUNT_COPIES; i += WIDE_COUNT_NT) cnt[i] = 0u;
  __syncthreads();
  const int64_t lo = int64_t(blockIdx.x) * args.range_keys;  // a multiple of VEC
  const int64_t hi = lo + args.range_keys < args.n ? lo + args.range_keys : args.n;
  auto count_key = [&](U k) {
    atomicAdd(&cnt[wide_digit<U, KIND>(k, args.shift, mask) * WIDE_COUNT_COPIES + copy], 1u);
  };
  if (lo < hi) {
    const uint4* v = reinterpret_cast<const uint4*>(keys + lo);
    const int64_t nvec = (hi - lo) / VEC;
    int64_t i = tid;
    for (; i + 3 * WIDE_COUNT_NT < nvec; i += 4 * WIDE_COUNT_NT) {
      uint4 w[4];
#pragma unroll
      for (int u = 0; u < 4; u++) w[u] = ldg_stream_v4(v + i + u * WIDE_COUNT_NT);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const U* e = reinterpret_cast<const U*>(&w[u]);
#pragma unroll
        for (int q = 0; q < VEC; q++) count_key(e[q]);
      }
    }
    for (; i < nvec; i += WIDE_COUNT_NT) {
      const uint4 w = ldg_stream_v4(v + i);
      const U* e = reinterpret_cast<const U*>(&w);
#pragma unroll
      for (int q = 0; q < VEC; q++) count_key(e[q]);
    }
    const int64_t tail = lo + nvec * VEC + tid;  // fewer than VEC keys at the end of the array
    if (tail < hi) count_key(keys[tail]);
  }
  __syncthreads();
  uint32_t* row = args.rcount + int64_t(blockIdx.x) * bins;
  for (int d = tid; d < bins; d += WIDE_COUNT_NT) {
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < WIDE_COUNT_COPIES; q++) c += cnt[d * WIDE_COUNT_COPIES + ((q + lane) & (WIDE_COUNT_COPIES - 1))];
    row[d] = c;
  }
}

// ---------------------------------------------------------------------------------------
// wide_plan: totals[d] and rprefix[j][d] = counts of digit d in the ranges before j; marks the
// pass as the identity when one digit value holds every key.  One CTA per 32 digits: thread
// (g, dl) owns digit dl of the CTA and the contiguous block g of the ranges.
// ---------------------------------------------------------------------------------------
constexpr int WIDE_PLAN_NT = 1024;

static __global__ void __launch_bounds__(WIDE_PLAN_NT) wide_plan_kernel(WideArgs args) {
  __shared__ uint32_t part[32][33];
  const int dl = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int bins = 1 << args.bits;
  const int d = blockIdx.x * 32 + dl;
  const int J = args.ranges;
  const int per = (J + 31) / 32;
  const int j0 = g * per < J ? g * per : J;
  const int j1 = j0 + per < J ? j0 + per : J;
  uint32_t bsum = 0;
  if (d < bins)
    for (int j = j0; j < j1; j++) bsum += args.rcount[int64_t(j) * bins + d];
  part[g][dl] = bsum;
  __syncthreads();
  if (g == 0) {
    uint32_t run = 0;
    for (int q = 0; q < 32; q++) {
      const uint32_t v = part[q][dl];
      part[q][dl] = run;
      run += v;
    }
    if (d < bins) {
      args.totals[d] = run;
      if (int64_t(run) == args.n) args.plan->skip[args.pass] = 1;
    }
  }
  __syncthreads();
  if (d < bins) {
    uint32_t run = part[g][dl];
    for (int j = j0; j < j1; j++) {
      args.rprefix[int64_t(j) * bins + d] = run;
      run += args.rcount[int64_t(j) * bins + d];
    }
  }
}

// ---------------------------------------------------------------------------------------
// wide_pass: one digit pass, CTA j over range j.
// ---------------------------------------------------------------------------------------
template <class U, class V, int NT, int KPT>
struct WideSmem {
  static constexpr bool PAIRS = !std::is_same<V, NoValue>::value;
  static constexpr int TILE = NT * KPT;
  static constexpr int NW = NT / 32;
  static constexpr int BINS = WIDE_MAX_BINS;
  static constexpr int DPT = BINS / NT;  // digits per thread in the scan
  static constexpr size_t KEYS_BYTES = size_t(TILE) * sizeof(U);
  static constexpr size_t VALS_BYTES = PAIRS ? size_t(TILE) * 4 : 0;
  static constexpr size_t STAGE_BYTES = KEYS_BYTES + VALS_BYTES;
  static constexpr size_t OFF_STAGES = 0;
  static constexpr size_t OFF_CNT = OFF_STAGES + 2 * STAGE_BYTES;  // [NW][BINS] 16-bit counters
  static constexpr size_t OFF_RUN = OFF_CNT + size_t(NW) * BINS * 2;  // running start per digit
  static constexpr size_t OFF_GBASE = OFF_RUN + size_t(BINS) * 4;     // this tile's base per digit
  static constexpr size_t OFF_WSUM = OFF_GBASE + size_t(BINS) * 4;
  static constexpr size_t OFF_TOP = OFF_WSUM + 32 * 4;  // the two most frequent digits
  static constexpr size_t OFF_MBAR = OFF_TOP + 16;
  static constexpr size_t BYTES = OFF_MBAR + 16;
  static_assert(DPT == 4, "the scan reads four 16-bit counters (8 bytes) per warp and thread");
  static_assert(TILE <= 32768, "tile offsets are 16-bit counters");
  static_assert(BYTES <= 232448, "227 KiB of shared memory per CTA");
};

template <class U, int KIND, class V, int NT, int KPT>
__global__ void __launch_bounds__(NT, 1) wide_pass_kernel(WideArgs args) {
  using L = WideSmem<U, V, NT, KPT>;
  constexpr bool PAIRS = L::PAIRS;
  constexpr int TILE = L::TILE, NW = L::NW, BINS = L::BINS, DPT = L::DPT;
  WidePlan* plan = args.plan;
  const int pass = args.pass;
  if (plan->skip[pass]) return;  // one digit value holds every key: the pass is the identity
  const int sel = plan->in_sel[pass];
  const U* __restrict__ kin = static_cast<const U*>(sel ? args.keys_b : args.keys_a);
  U* __restrict__ kout = static_cast<U*>(sel ? args.keys_a : args.keys_b);
  const uint32_t* __restrict__ vin = static_cast<const uint32_t*>(sel ? args.vals_b : args.vals_a);
  uint32_t* __restrict__ vout = static_cast<uint32_t*>(sel ? args.vals_a : args.vals_b);
  uint32_t* err = &plan->error;
  const int bins = 1 << args.bits;
  const uint32_t mask = uint32_t(bins - 1);
  const int shift = args.shift;
  const uint32_t n32 = uint32_t(args.n);
  const int j = blockIdx.x;
  const int64_t clo = int64_t(j) * args.range_keys;
  const int64_t chi = clo + args.range_keys < args.n ? clo + args.range_keys : args.n;
  const int ntiles = clo < chi ? int((chi - clo + TILE - 1) / TILE) : 0;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + L::OFF_CNT);  // words of two 16-bit counters
  uint32_t* s_run = reinterpret_cast<uint32_t*>(smem + L::OFF_RUN);
  uint32_t* s_gbase = reinterpret_cast<uint32_t*>(smem + L::OFF_GBASE);
  uint32_t* s_wsum = reinterpret_cast<uint32_t*>(smem + L::OFF_WSUM);
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(smem + L::OFF_MBAR);
  unsigned long long* s_top = reinterpret_cast<unsigned long long*>(smem + L::OFF_TOP);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* cnt_w = s_cnt + warp * (BINS / 2);
  const uint16_t* cnt16_w = reinterpret_cast<const uint16_t*>(cnt_w);
  const U* kin_c = kin + clo;

  auto issue = [&](int t) {
    onesweep_issue_tile<U, PAIRS, TILE>(smem, L::STAGE_BYTES, L::KEYS_BYTES, s_mbar, kin_c,
                                        vin ? vin + clo : nullptr, chi - clo, t, t & 1);
  };
  if (tid == 0) {
    mbar_init(&s_mbar[0], 1);
    mbar_init(&s_mbar[1], 1);
    fence_mbar_init();
    if (ntiles > 0) issue(0);
    if (ntiles > 1) issue(1);
  }

  // running start of each digit: bin start (exclusive scan of the totals) + ranges before j.
  // Thread t owns digits [t*DPT, t*DPT + DPT) here and in every tile's scan.
  {
    const int d0 = tid * DPT;
    uint32_t tot[DPT], sum = 0;
#pragma unroll
    for (int q = 0; q < DPT; q++) {
      tot[q] = d0 + q < bins ? args.totals[d0 + q] : 0u;
      sum += tot[q];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    uint32_t base = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) base += w < warp ? s_wsum[w] : 0u;
    uint32_t run = base + incl - sum;
    const uint32_t* pre = args.rprefix + int64_t(j) * bins;
#pragma unroll
    for (int q = 0; q < DPT; q++) {
      s_run[d0 + q] = run + (d0 + q < bins ? pre[d0 + q] : 0u);
      run += tot[q];
    }
    __syncthreads();
    // the two most frequent digit values (count, then the lower value, first)
    unsigned long long best = 0ull;
#pragma unroll
    for (int q = 0; q < DPT; q++) {
      const unsigned long long c = (static_cast<unsigned long long>(tot[q]) << 16) | uint32_t(0xFFFF - (d0 + q));
      best = c > best ? c : best;
    }
    s_top[0] = 0ull;
    s_top[1] = 0ull;
    __syncthreads();
    atomicMax(&s_top[0], best);
    __syncthreads();
    best = 0ull;
#pragma unroll
    for (int q = 0; q < DPT; q++) {
      const unsigned long long c = (static_cast<unsigned long long>(tot[q]) << 16) | uint32_t(0xFFFF - (d0 + q));
      if (c != s_top[0]) best = c > best ? c : best;
    }
    atomicMax(&s_top[1], best);
    __syncthreads();
  }
  const unsigned long long top1 = s_top[0], top2 = s_top[1];
  const uint32_t h1 = 0xFFFFu - uint32_t(top1 & 0xFFFFull);
  const uint32_t h2 = top2 ? 0xFFFFu - uint32_t(top2 & 0xFFFFull) : h1;
  // one value above 1/16 of the keys: many lanes of an instruction would share its counter
  const bool grouped = int64_t(top1 >> 16) > args.n / 16;

  bool out_of_range = false;
  auto tile_body = [&](auto full_tag, int t) {
    constexpr bool FULL = decltype(full_tag)::value;
    const int stage = t & 1;
    const int64_t tile_base = clo + int64_t(t) * TILE;
    const int tile_n = FULL ? TILE : int(chi - tile_base);
    const int bulk_keys = FULL ? TILE : int((int64_t(tile_n) * int64_t(sizeof(U))) & ~int64_t(15)) / int(sizeof(U));
    const int bulk_vals = FULL ? TILE : (PAIRS ? int((int64_t(tile_n) * 4) & ~int64_t(15)) / 4 : 0);

    {  // zero this warp's counters (BINS / 2 words, 16-byte stores)
      uint4* c4 = reinterpret_cast<uint4*>(cnt_w);
#pragma unroll
      for (int i = lane; i < BINS / 8; i += 32) c4[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (!mbar_wait_bounded(&s_mbar[stage], uint32_t(t >> 1) & 1u, args.spin_limit_ns)) {
      if (lane == 0) atomicOr(err, uint32_t(DERR_TMA_TIMEOUT));
    }
    __syncwarp();

    // ---- load keys (warp-striped) and rank them within the warp (ordered shared atomics) ----
    U* sk = reinterpret_cast<U*>(smem + L::OFF_STAGES + stage * L::STAGE_BYTES);
    U key[KPT];
    uint32_t rank[KPT];
    const int wbase = warp * 32 * KPT;
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      U k = U(0);
      if (FULL || idx < bulk_keys) k = sk[idx];
      else if (idx < tile_n) k = kin[tile_base + idx];
      key[i] = k;
    }
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      rank[i] = wide_rank(cnt_w, wide_digit<U, KIND>(key[i], shift, mask), FULL || idx < tile_n, grouped, h1, h2,
                          lane);
    }
    __syncthreads();  // (A) warp counts complete; the stage buffer is no longer read

    // ---- scan over (digit, warp): per-warp tile offsets and the global base per digit ----
    // Two reads of this thread's counters (totals, then running offsets) keep the registers
    // free for the keys and ranks.
    {
      const int d0 = tid * DPT;
      uint32_t tot[DPT] = {};
#pragma unroll
      for (int w = 0; w < NW; w++) {
        const uint2 v = *reinterpret_cast<const uint2*>(s_cnt + w * (BINS / 2) + d0 / 2);
        tot[0] += v.x & 0xFFFFu;
        tot[1] += v.x >> 16;
        tot[2] += v.y & 0xFFFFu;
        tot[3] += v.y >> 16;
      }
      const uint32_t sum = tot[0] + tot[1] + tot[2] + tot[3];
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) s_wsum[warp] = incl;
      __syncthreads();  // (B)
      uint32_t base = 0;
#pragma unroll
      for (int w = 0; w < NW; w++) base += w < warp ? s_wsum[w] : 0u;
      uint32_t local[DPT];
      local[0] = base + incl - sum;
      local[1] = local[0] + tot[0];
      local[2] = local[1] + tot[1];
      local[3] = local[2] + tot[2];
      uint32_t run01 = local[0] | (local[1] << 16), run23 = local[2] | (local[3] << 16);
#pragma unroll
      for (int w = 0; w < NW; w++) {
        uint2* p = reinterpret_cast<uint2*>(s_cnt + w * (BINS / 2) + d0 / 2);
        const uint2 v = *p;
        *p = make_uint2(run01, run23);
        run01 += v.x;  // both halves stay below 2^16: no carry between them
        run23 += v.y;
      }
#pragma unroll
      for (int q = 0; q < DPT; q++) {
        const uint32_t r = s_run[d0 + q];
        s_gbase[d0 + q] = r - local[q];
        s_run[d0 + q] = r + tot[q];
      }
    }
    __syncthreads();  // (C) offsets ready

    // ---- reorder the tile in shared memory by digit ----------------------------------
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      if (FULL || idx < tile_n) {
        const uint32_t pos = uint32_t(cnt16_w[wide_digit<U, KIND>(key[i], shift, mask)]) + rank[i];
        rank[i] = pos;  // the tile position, kept for the payload
        sk[pos] = key[i];
      }
    }
    __syncthreads();  // (D) reordered keys ready

    // ---- coalesced per-digit runs ------------------------------------------------------
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int s = i * NT + tid;
      key[i] = (FULL || s < tile_n) ? sk[s] : U(0);
    }
    if (!PAIRS) {
      fence_proxy_async_smem();
      __syncthreads();  // (F) the stage buffer is free
      if (tid == 0 && t + 2 < ntiles) issue(t + 2);
    }
    uint16_t dsave[PAIRS ? KPT : 1];
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int s = i * NT + tid;
      if (FULL || s < tile_n) {
        const uint32_t d = wide_digit<U, KIND>(key[i], shift, mask);
        if (PAIRS) dsave[i] = uint16_t(d);
        const uint32_t pos = s_gbase[d] + uint32_t(s);
        if (pos < n32) kout[pos] = key[i];
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
        if (FULL || idx < bulk_vals) v = sv[idx];
        else if (idx < tile_n) v = vin[tile_base + idx];
        val[i] = v;
      }
      __syncthreads();  // (E1) all payloads read before they are overwritten
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int idx = wbase + i * 32 + lane;
        if (FULL || idx < tile_n) sv[rank[i]] = val[i];
      }
      __syncthreads();  // (E2)
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int s = i * NT + tid;
        if (FULL || s < tile_n) {
          const uint32_t pos = s_gbase[dsave[i]] + uint32_t(s);
          if (pos < n32) vout[pos] = sv[s];
        }
      }
      fence_proxy_async_smem();
      __syncthreads();  // (F) the stage buffer is free
      if (tid == 0 && t + 2 < ntiles) issue(t + 2);
    }
  };

  for (int t = 0; t < ntiles; t++) {
    if (chi - (clo + int64_t(t) * TILE) >= TILE) tile_body(std::integral_constant<bool, true>(), t);
    else tile_body(std::integral_constant<bool, false>(), t);
  }
  if (out_of_range) atomicOr(err, uint32_t(DERR_BOUNDS));
}

// Copies the result back into the caller's buffer when it ended in the scratch buffer (an odd
// number of executed passes), and folds the device error bits into the context's word.
template <class U>
__global__ void wide_finalize_kernel(WideArgs args, int passes, int has_vals, uint32_t* err_accum) {
  const WidePlan* plan = args.plan;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t e = ld_volatile(&plan->error);
    if (e) atomicOr(err_accum, e);
  }
  if (wide_src_sel(plan, passes) != 1) return;
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
