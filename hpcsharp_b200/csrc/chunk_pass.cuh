// One LSD digit pass without inter-CTA waiting ("chunked" pass, sm_100a).
//
// The keys are cut into J ranges of L keys (a whole number of tiles), J <= number of SMs;
// CTA j of every kernel of the sort owns range j of the current input buffer.  The global
// position of a key with digit d read by CTA j is
//
//     bin_start[d] + (keys with digit d in ranges 0..j-1) + (keys with digit d before it in
//                                                           range j)
//
// which is the reference's bin-major / quantum-minor offset table (RadixSortLsdParallel.cs
// :49-94) with one quantum per range.  The middle term needs the per-range digit counts
// *before* the pass runs.  For the first executed pass K1 writes them (each K1 CTA counts
// its own range).  For every later pass they are produced by the pass before it: when a
// key is written to position p, the range that p falls in for the next pass (p / L) and
// the key's next digit are known, so the writing CTA adds one to count[p / L][next digit]
// in shared memory and adds its table into a global table at the end.  The last term is a
// running per-digit offset carried from tile to tile inside the CTA.  So no CTA ever waits
// for another: there is no look-back, no tile counter and no spin on another CTA's data.
//
// Per tile (TILE = NT x KPT keys, double-buffered by 1-D bulk async copies):
//   rank     one ordered shared atomic per key on per-warp digit counters (or the
//            peer-mask ranking), as in the onesweep pass;
//   scan     per-digit tile totals, tile-local digit starts, per-warp offsets; the
//            tile's global base per digit comes from the running offsets;
//   reorder  keys into shared memory in (digit, input order) order;
//   scatter  coalesced per-digit runs to global memory, and the next-digit count.
//
// Next-digit counters are 16 bits, J x 256 of them (74 KiB for J = 148), two per word: word
// (q / 2) * 256 + e holds range q's counter of next digit e in its low half for even q and in
// its high half for odd q.  The keys of a warp instruction mostly land in one range, so their
// random digits spread over 256 words (measured on B200: ~4 clocks per random warp atomic on 256
// words, ~6 on 128 words, where pairs of digits share a word).  A counter that reaches 0x8000 is moved to the global table by the thread whose increment
// reached it (it subtracts 0x8000 in shared memory and adds 0x8000 in global memory).  One
// increment per key, so exactly one thread sees each crossing, and between a crossing and
// its subtraction at most one tile of other increments can land (each thread's subtraction
// precedes the end-of-tile barrier): a counter stays below 0x8000 + TILE <= 0xC000 and never
// carries into its neighbour.
#pragma once
#include "radix_kernels.cuh"

namespace hpcs {

template <class U, class V, int NT, int KPT, int MODE>
struct ChunkSmem {
  static constexpr bool PAIRS = !std::is_same<V, NoValue>::value;
  static constexpr int TILE = NT * KPT;
  static constexpr int NW = NT / 32;
  static constexpr int G = NT / RADIX;        // threads per digit in the digit scan
  static constexpr int NWG = NW / G;          // warps summed by each of them
  static constexpr int RS = RADIX + 32 / NW;  // warp-counter row stride: conflict-free scan
  static constexpr size_t KEYS_BYTES = size_t(TILE) * sizeof(U);
  static constexpr size_t VALS_BYTES = PAIRS ? size_t(TILE) * 4 : 0;
  static constexpr size_t STAGE_BYTES = KEYS_BYTES + VALS_BYTES;
  static constexpr size_t OFF_STAGES = 0;
  static constexpr size_t OFF_CNT = OFF_STAGES + 2 * STAGE_BYTES;  // [NW][RS]
  static constexpr size_t OFF_MSK = OFF_CNT + size_t(NW) * RS * 4;
  static constexpr size_t MSK_BYTES = MODE == RANK_PEER_MASK ? size_t(NW) * 2 * RADIX * 4 : 0;
  static constexpr size_t OFF_RUN = (OFF_MSK + MSK_BYTES + 15) / 16 * 16;  // running start per digit
  // per digit for this tile: {global base, counter words of its first key's range q (word base
  // | half << 31), first position of range q + 1, counter words of range q + 1}
  static constexpr size_t OFF_META = OFF_RUN + RADIX * 4;
  static constexpr size_t OFF_WSUM = OFF_META + RADIX * 16;
  static constexpr size_t OFF_MBAR = (OFF_WSUM + 32 * 4 + 7) / 8 * 8;
  static constexpr size_t OFF_CTAB = (OFF_MBAR + 16 + 15) / 16 * 16;  // [(J + 1) / 2][256] words
  static constexpr size_t BASE_BYTES = OFF_CTAB;
  static constexpr size_t bytes(int chunks) { return BASE_BYTES + size_t((chunks + 1) / 2) * RADIX * 4; }
  static_assert(TILE <= 16384, "16-bit next-digit counters assume at most 16384 keys per tile");
  static_assert(G >= 1 && (G & (G - 1)) == 0 && NW % G == 0 && 32 % NW == 0, "digit-scan geometry");
  static_assert(size_t(NW) * RS >= size_t(G) * RADIX, "prologue partials fit in the counters");
};

// Counter words of range q in the next-digit table: word base (q / 2) * 256, half q % 2 in bit 31.
__device__ __forceinline__ uint32_t ctab_words(uint32_t q) { return (q >> 1) * uint32_t(RADIX) | ((q & 1u) << 31); }

// Ranks of one warp's keys are turned into tile offsets by a scan over (digit, warp) in
// which every thread takes part: thread t handles digit t / G and the NWG consecutive warps
// [q * NWG, (q + 1) * NWG), q = t % G.  With the row stride RS = 256 + 32 / NW the NWG x 32
// counters a warp instruction reads fall in 32 distinct banks.
template <class U, int KIND, class V, int NT, int KPT, int MODE>
__device__ __forceinline__ void chunk_pass_body(const SortArgs& args, const int j) {
  using L = ChunkSmem<U, V, NT, KPT, MODE>;
  using KO = KeyOrder<U, KIND>;
  constexpr bool PAIRS = L::PAIRS;
  constexpr int TILE = L::TILE;
  constexpr int G = L::G, NWG = L::NWG, RS = L::RS;
  constexpr int P = int(sizeof(U));
  static_assert(NT % RADIX == 0, "whole digit groups in the scan");

  const SortPlan* plan = args.plan;
  const int pass = args.pass;
  if (args.choose_lookback && plan->use_lookback) return;  // the look-back passes were chosen
  const int sel = plan->src_sel[pass];
  if (sel < 0) return;  // every key has the same digit here: the pass is the identity
  const int shift = 8 * pass;
  const int nshift = plan->next_shift[pass];  // uniform over the grid
  const int x = plan->exec_idx[pass];
  const U* __restrict__ kin = static_cast<const U*>(sel ? args.keys_b : args.keys_a);
  U* __restrict__ kout = static_cast<U*>(sel ? args.keys_a : args.keys_b);
  const uint32_t* __restrict__ vin = static_cast<const uint32_t*>(sel ? args.vals_b : args.vals_a);
  uint32_t* __restrict__ vout = static_cast<uint32_t*>(sel ? args.vals_a : args.vals_b);
  uint32_t* err = const_cast<uint32_t*>(&plan->error);
  const uint32_t n32 = uint32_t(args.n);
  const int J = args.chunks;
  const uint32_t LK = args.chunk_keys;
  const uint32_t magic = args.chunk_magic;
  const int64_t clo = int64_t(j) * LK;
  const int64_t chi = clo + LK < args.n ? clo + LK : args.n;
  const int ntiles = clo < chi ? int((chi - clo + TILE - 1) / TILE) : 0;

  // this pass's per-range counts, the table it fills, and the one it clears for later
  const uint32_t* cin;
  int64_t cin_stride;
  if (x == 0) {
    cin = args.chunk_hist + pass * RADIX;
    cin_stride = int64_t(P) * RADIX;
  } else {
    cin = args.ctab + int64_t(x % 3) * J * RADIX;
    cin_stride = RADIX;
  }
  uint32_t* __restrict__ cout = args.ctab + int64_t((x + 1) % 3) * J * RADIX;
  uint32_t* __restrict__ czero = args.ctab + int64_t((x + 2) % 3) * J * RADIX;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + L::OFF_CNT);
  uint32_t* s_msk = reinterpret_cast<uint32_t*>(smem + L::OFF_MSK);
  uint32_t* s_run = reinterpret_cast<uint32_t*>(smem + L::OFF_RUN);
  uint4* s_meta = reinterpret_cast<uint4*>(smem + L::OFF_META);
  uint32_t* s_wsum = reinterpret_cast<uint32_t*>(smem + L::OFF_WSUM);
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(smem + L::OFF_MBAR);
  uint32_t* s_ctab = reinterpret_cast<uint32_t*>(smem + L::OFF_CTAB);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* cnt_w = s_cnt + warp * RS;
  uint32_t* msk_w = s_msk + warp * 2 * RADIX;
  const U* kin_c = kin + clo;
  U* kout_base = kout;

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
  for (int i = tid; i < RADIX; i += NT) czero[int64_t(j) * RADIX + i] = 0u;
  if (nshift >= 0)
    for (int i = tid; i < (J + 1) / 2 * RADIX; i += NT) s_ctab[i] = 0u;
  if (MODE == RANK_PEER_MASK)
    for (int i = lane; i < 2 * RADIX; i += 32) msk_w[i] = 0u;

  // running start of each digit: bin start + counts of ranges 0..j-1 (G partial sums).
  // The pass before this one does not count this digit's most frequent value h (its
  // counters would be the most contended); ranges 0..j-1 hold j x L keys, so h's count
  // is j x L minus the other values' counts.
  const uint32_t heavy = uint32_t(plan->heavy[pass]);
  {
    // up to 16 independent loads in flight per thread: the sum's latency is a few L2
    // round trips even for the last range
    const int g = tid / RADIX, d = tid % RADIX;
    uint32_t acc[16];
#pragma unroll
    for (int u = 0; u < 16; u++) acc[u] = 0u;
    for (int q0 = g; q0 < j; q0 += 16 * G) {
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int q = q0 + u * G;
        if (q < j) acc[u] += __ldcg(cin + int64_t(q) * cin_stride + d);
      }
    }
    uint32_t sum = 0;
#pragma unroll
    for (int u = 0; u < 16; u++) sum += acc[u];
    s_cnt[g * RADIX + d] = sum;
  }
  __syncthreads();
  if (tid < RADIX) {
    uint32_t pre = 0;
#pragma unroll
    for (int g = 0; g < G; g++) pre += s_cnt[g * RADIX + tid];
    s_run[tid] = plan->bin_start[pass][tid] + pre;
    uint32_t w = pre;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) w += __shfl_xor_sync(0xFFFFFFFFu, w, o);
    if (lane == 0) s_wsum[warp] = w;
  }
  __syncthreads();
  if (x > 0 && tid == 0) {
    uint32_t others = 0;
#pragma unroll
    for (int w = 0; w < RADIX / 32; w++) others += s_wsum[w];
    s_run[heavy] = plan->bin_start[pass][heavy] + uint32_t(j) * LK - others;
  }
  __syncthreads();

  bool out_of_range = false;
  const int sd = tid / G, sq = tid % G;  // the digit and warp group this thread scans
  const Digit<U, KIND> dig(shift);
  const Digit<U, KIND> ndig(nshift < 0 ? 0 : nshift);
  // When the next digit has a frequent value, whole warp instructions of equal keys (runs
  // of one frequent key after the reorder) would serialise on one counter: such passes
  // test each instruction for a single (range, value) and add it once.
  const bool next_skewed = nshift >= 0 && plan->skewed[nshift >> 3] != 0;
  // When this pass's two most frequent values hold more than 3/4 of the keys (e.g. the top
  // byte of small signed values: 0x7F and 0x80), their lanes rank with one atomic per warp
  // instruction each (ordered-atomic mode only).  Measured on B200: +10% for normal(0, 2^20)
  // int32 keys; below 3/4 (floats' top byte, sparse-bit keys) the votes cost more than the
  // serialised atomics they replace.
  const bool grouped = MODE == RANK_ORDERED_ATOMIC && plan->grouped[pass] != 0;
  const uint32_t heavy2 = uint32_t(plan->heavy2[pass]);
  const uint32_t next_heavy = nshift < 0 ? 0u : uint32_t(plan->heavy[nshift >> 3]);

  auto tile_body = [&](auto full_tag, int t) {
    constexpr bool FULL = decltype(full_tag)::value;
    const int stage = t & 1;
    const int64_t tile_base = clo + int64_t(t) * TILE;
    const int tile_n = FULL ? TILE : int(chi - tile_base);
    const int bulk_keys = FULL ? TILE : int((int64_t(tile_n) * int64_t(sizeof(U))) & ~int64_t(15)) / int(sizeof(U));
    const int bulk_vals = FULL ? TILE : (PAIRS ? int((int64_t(tile_n) * 4) & ~int64_t(15)) / 4 : 0);
    const int64_t tile_id = int64_t(j) * (LK / TILE) + t;
    uint64_t* trace = (args.trace && pass == args.trace_pass && tile_id < args.trace_capacity && tid == 0)
                          ? args.trace + tile_id * TRACE_WORDS
                          : nullptr;
    if (trace) {
      trace[0] = uint64_t(tile_id);
      trace[1] = sm_id();
      trace[2] = global_timer_ns();
    }
    if (tile_id == args.poison_tile && tid == 0) {
      // test hook: a bounded wait on a flag that nothing sets, reported as a timeout
      const uint64_t t0 = global_timer_ns();
      while (ld_volatile(&plan->idle_flag) == 0u && global_timer_ns() - t0 < args.spin_limit_ns) __nanosleep(1000);
      atomicOr(err, uint32_t(DERR_LOOKBACK_TIMEOUT));
    }

    for (int i = lane; i < RADIX; i += 32) cnt_w[i] = 0u;

    // wait for the staged tile (bounded)
    if (!mbar_wait_bounded(&s_mbar[stage], uint32_t(t >> 1) & 1u, args.spin_limit_ns)) {
      if (lane == 0) atomicOr(err, uint32_t(DERR_TMA_TIMEOUT));
    }
    __syncwarp();
    if (trace) trace[3] = global_timer_ns();

    // ---- load keys (warp-striped) and rank them within the warp ----------------------
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
    if (grouped) {
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int idx = wbase + i * 32 + lane;
        rank[i] = rank_in_warp_top2(cnt_w, dig(key[i]), FULL || idx < tile_n, heavy, heavy2, lane);
      }
    } else {
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int idx = wbase + i * 32 + lane;
        rank[i] = rank_in_warp<MODE>(cnt_w, msk_w, dig(key[i]), FULL || idx < tile_n, i & 1, lane);
      }
    }
    __syncthreads();  // (A) warp counts complete; the stage buffer is no longer read
    if (trace) trace[4] = global_timer_ns();

    // ---- scan over (digit, warp): tile offsets per warp and global base per digit ----
    {
      uint32_t c[NWG];
      uint32_t gsum = 0;
#pragma unroll
      for (int m = 0; m < NWG; m++) {
        c[m] = s_cnt[(sq * NWG + m) * RS + sd];
        gsum += c[m];
      }
      uint32_t qi = gsum;  // inclusive over the digit's warp groups
#pragma unroll
      for (int o = 1; o < G; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, qi, o, G);
        if (sq >= o) qi += y;
      }
      const uint32_t total = __shfl_sync(0xFFFFFFFFu, qi, lane | (G - 1));
      uint32_t di = total;  // inclusive over this warp's digits (lanes G apart)
#pragma unroll
      for (int o = G; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, di, o);
        if (lane >= o) di += y;
      }
      if (lane == 31) s_wsum[warp] = di;
      __syncthreads();  // (B)
      uint32_t wv = lane < warp ? s_wsum[lane] : 0u;
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) wv += __shfl_xor_sync(0xFFFFFFFFu, wv, o);
      const uint32_t local = wv + di - total;  // tile-local start of digit sd
      uint32_t run = local + qi - gsum;
#pragma unroll
      for (int m = 0; m < NWG; m++) {
        s_cnt[(sq * NWG + m) * RS + sd] = run;
        run += c[m];
      }
      if (sq == 0) {
        // r: global position of this tile's first key of digit sd.  The digit's keys of the tile
        // (at most one tile, and a range holds whole tiles) fall in r's range q or the next one.
        const uint32_t r = s_run[sd];
        uint32_t q = __umulhi(r, magic);
        q -= (q * LK > r) ? 1u : 0u;
        s_meta[sd] = make_uint4(r - local, ctab_words(q), (q + 1u) * LK, ctab_words(q + 1u));
        s_run[sd] = r + total;
      }
    }
    __syncthreads();  // (C) offsets ready

    // ---- reorder the tile in shared memory by digit ----------------------------------
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int idx = wbase + i * 32 + lane;
      if (FULL || idx < tile_n) {
        const uint32_t pos = cnt_w[dig(key[i])] + rank[i];
        rank[i] = pos;  // the tile position, kept for the payload
        sk[pos] = key[i];
      }
    }
    __syncthreads();  // (D) reordered keys ready
    if (trace) trace[5] = global_timer_ns();

    // ---- coalesced per-digit runs, and the next pass's per-range digit counts -------
    // Keys-only tiles: every thread first takes its KPT reordered keys into registers, so
    // the stage buffer is released (and refilled) before the global writes.
    // Every destination is checked against n; a bad one is recorded instead of written.
    // Counter crossings are collected in a mask (no branch on an atomic's result inside
    // the loop) and moved to the global table afterwards.
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
    uint8_t dsave[PAIRS ? KPT : 1];
    uint32_t crossed = 0;
#pragma unroll
    for (int i = 0; i < KPT; i++) {
      const int s = i * NT + tid;
      if (FULL || s < tile_n) {
        const U k = key[i];
        const uint32_t d = dig(k);
        if (PAIRS) dsave[i] = uint8_t(d);
        const uint4 m = s_meta[d];
        const uint32_t pos = m.x + uint32_t(s);
        if (pos < n32) {
          kout_base[pos] = k;
          const uint32_t e = ndig(k);
          if (nshift >= 0 && !next_skewed && e != next_heavy) {
            const uint32_t cw = pos >= m.z ? m.w : m.y;
            const uint32_t inc = 1u << ((cw >> 31) << 4);
            const uint32_t old = atomicAdd(s_ctab + (cw & 0x7FFFFFFFu) + e, inc);
            // a half went from 0x7FFF to 0x8000 (the other half is unchanged)
            if ((old + inc) & ~old & 0x80008000u) crossed |= 1u << i;
          }
        } else {
          out_of_range = true;
        }
      }
    }
    if (next_skewed) {
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        const int s = i * NT + tid;
        const U k = key[i];
        const uint32_t e = ndig(k);
        const uint4 m = s_meta[dig(k)];
        const uint32_t pos = m.x + uint32_t(s);
        const uint32_t cw = pos >= m.z ? m.w : m.y;
        const bool counted = (FULL || s < tile_n) && pos < n32 && e != next_heavy;
        const uint32_t word = (cw & 0x7FFFFFFFu) + e;
        const uint32_t unit = 1u << ((cw >> 31) << 4);
        const uint32_t code = (word << 1) | (cw >> 31);
        const uint32_t lanes = __ballot_sync(0xFFFFFFFFu, counted);
        if (lanes == 0u) continue;
        const int leader = __ffs(lanes) - 1;
        const uint32_t lead = __shfl_sync(0xFFFFFFFFu, code, leader);
        const bool one_code = __all_sync(0xFFFFFFFFu, !counted || code == lead);
        uint32_t inc = counted ? unit : 0u;
        if (one_code) inc = lane == leader ? unit * uint32_t(__popc(lanes)) : 0u;
        if (inc) {
          const uint32_t old = atomicAdd(s_ctab + word, inc);
          // a half went below 0x8000 to at least 0x8000 (the other half is unchanged)
          if ((old + inc) & ~old & 0x80008000u) crossed |= 1u << i;
        }
      }
    }
    if (crossed) {
#pragma unroll
      for (int i = 0; i < KPT; i++) {
        if ((crossed >> i) & 1u) {
          const int s = i * NT + tid;
          const U k = key[i];
          const uint4 m = s_meta[dig(k)];
          const uint32_t pos = m.x + uint32_t(s);
          const uint32_t cw = pos >= m.z ? m.w : m.y;
          const uint32_t e = ndig(k);
          const uint32_t sh = (cw >> 31) << 4;
          const uint32_t q = ((cw & 0x7FFFFFFFu) / RADIX) * 2u + (cw >> 31);  // the range
          atomicSub(s_ctab + (cw & 0x7FFFFFFFu) + e, 0x8000u << sh);
          atomicAdd(cout + q * RADIX + e, 0x8000u);
        }
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
          const uint32_t pos = s_meta[dsave[i]].x + uint32_t(s);
          if (pos < n32) vout[pos] = sv[s];
        }
      }
    }
    if (trace) trace[6] = global_timer_ns();
    // The stage buffer was written through the generic proxy and is refilled by a bulk
    // copy (async proxy): order the writes before the barrier, then refill it.
    if (PAIRS) {
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

  // add this CTA's next-digit counts into the global table (nonzero counters only)
  if (nshift >= 0) {
    __syncthreads();
    for (int i = tid; i < (J + 1) / 2 * RADIX; i += NT) {
      const uint32_t v = s_ctab[i];
      const int e = i % RADIX, q0 = (i / RADIX) * 2;  // ranges q0 (low half) and q0 + 1
      if (v & 0xFFFFu) atomicAdd(cout + q0 * RADIX + e, v & 0xFFFFu);
      if (v >> 16) atomicAdd(cout + (q0 + 1) * RADIX + e, v >> 16);
    }
  }
}

// One digit pass of one array: CTA j owns range j.
template <class U, int KIND, class V, int NT, int KPT, int MODE>
__global__ void __launch_bounds__(NT, 1) chunk_pass_kernel(SortArgs args) {
  chunk_pass_body<U, KIND, V, NT, KPT, MODE>(args, int(blockIdx.x));
}

// One digit pass of many arrays in one launch (the batched sort's grid-level path): CTA c owns
// range map[c].y of array map[c].x, whose sort arguments are args[map[c].x].
template <class U, int KIND, class V, int NT, int KPT, int MODE>
__global__ void __launch_bounds__(NT, 1) seg_chunk_pass_kernel(const SortArgs* __restrict__ args,
                                                               const int2* __restrict__ map, int pass) {
  const int2 m = map[blockIdx.x];
  SortArgs a = args[m.x];
  a.pass = pass;
  chunk_pass_body<U, KIND, V, NT, KPT, MODE>(a, m.y);
}

}  // namespace hpcs
