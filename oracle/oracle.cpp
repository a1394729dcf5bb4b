// CPU oracle: a C++17 restatement of HPCsharp's LSD radix-sort hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the GPU library and the
// timed CPU baseline; nothing in the product links or calls it.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load liboracle.so.
//
// Parity status: the reference (C#, .NET 7-9) has no unit tests for radix sort,
// histogram or selection and cannot be compiled here (no .NET toolchain), so parity
// is pinned by (1) the reference's only known-answer case
// (HPCsharpExamples/HPCsharpExamples/Program.cs:15-34, {21,43,16,5,54,3}),
// (2) std::sort / std::stable_sort cross-checks on the order-transformed key, and
// (3) committed SHA-256 fixtures generated from this restatement
// (tests/golden/make_golden.py).
//
// Every function cites the reference file:line it restates (paths relative to the
// HPCsharp project root).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------------------------
// Digit extraction with the reference's order transforms.
//   unsigned: (x >> 8d) & 0xFF                      RadixSortLsd.cs:1136-1143 (ExtractDigit)
//   signed:   top digit ^ 128                       RadixSortLsd.cs:288-293 (i32), :464-469 (i64),
//                                                   Histogram.cs:1014, :1049
//   float:    sign 0 -> flip sign bit only,         Histogram.cs:1210-1248 (f32),
//             sign 1 -> flip every bit              Histogram.cs:1250-1288 (f64)
// ---------------------------------------------------------------------------------
enum Kind { UNSIGNED = 0, SIGNED = 1, FLOAT = 2 };

template <class U>
inline U order_bits(U x, int kind) {
  constexpr int W = sizeof(U) * 8;
  constexpr U top = U(1) << (W - 1);
  if (kind == SIGNED) return x ^ top;
  if (kind == FLOAT) return (x & top) ? U(~x) : U(x ^ top);
  return x;
}

template <class U>
inline U order_bits_inverse(U y, int kind) {
  constexpr int W = sizeof(U) * 8;
  constexpr U top = U(1) << (W - 1);
  if (kind == SIGNED) return y ^ top;
  if (kind == FLOAT) return (y & top) ? U(y ^ top) : U(~y);
  return y;
}

template <class U>
inline unsigned digit_of(U x, int d, int kind) {
  return unsigned((order_bits<U>(x, kind) >> (8 * d)) & 0xFF);
}

// Fused all-digit histogram: Histogram.cs:261-296 (u32), :957-990 (u64), :992-1017 (i32),
// :1019-1052 (i64).  One read of [l, r], counts[d][256] for every byte d.
template <class U>
void histogram_byte_components(const U* a, int64_t l, int64_t r, int kind, uint32_t* counts) {
  constexpr int P = sizeof(U);
  std::memset(counts, 0, sizeof(uint32_t) * P * 256);
  for (int64_t i = l; i <= r; i++) {
    U v = a[i];
    for (int d = 0; d < P; d++) counts[d * 256 + digit_of<U>(v, d, kind)]++;
  }
}

// ComputeStartOfBins: RadixSortLsd.cs:112-125 (exclusive scan per digit).
template <int P>
void compute_start_of_bins(const uint32_t* count, int64_t* start) {
  for (int d = 0; d < P; d++) {
    start[d * 256] = 0;
    for (int i = 1; i < 256; i++) start[d * 256 + i] = start[d * 256 + i - 1] + count[d * 256 + i - 1];
  }
}

// Serial LSD sort.  SortRadixLsdInner(uint[]) RadixSortLsd.cs:127-202 uses 128-deep
// per-bin write buffers ("de-randomized" writes) flushed with Array.Copy; the i32/u64/i64
// versions (:267-299, :359-384, :444-475) scatter directly.  Both give the same stable
// order; the buffered form is restated for u32 as in the reference.
template <class U>
void sort_radix_lsd(U* a, int64_t n, int kind, bool buffered) {
  constexpr int P = sizeof(U);
  if (n <= 0) return;
  std::vector<U> out(n);
  uint32_t count[P * 256];
  int64_t start[P * 256];
  histogram_byte_components<U>(a, 0, n - 1, kind, count);
  compute_start_of_bins<P>(count, start);
  U* in = a;
  U* o = out.data();
  const int64_t depth = 64 * 8 / int64_t(sizeof(uint32_t));  // BufferDepth = 128 (:138)
  std::vector<U> cache;
  std::vector<int64_t> cur(256);
  if (buffered) cache.resize(256 * depth);
  for (int d = 0; d < P; d++) {
    int64_t* sob = start + d * 256;
    if (!buffered) {
      for (int64_t i = 0; i < n; i++) o[sob[digit_of<U>(in[i], d, kind)]++] = in[i];
    } else {
      for (int b = 0; b < 256; b++) cur[b] = b * depth;
      for (int64_t i = 0; i < n; i++) {
        unsigned b = digit_of<U>(in[i], d, kind);
        if (cur[b] < b * depth + depth) {
          cache[cur[b]++] = in[i];
        } else {  // flush the full buffer (:166-177)
          std::memcpy(o + sob[b], cache.data() + b * depth, sizeof(U) * depth);
          sob[b] += depth;
          cur[b] = b * depth;
          cache[cur[b]++] = in[i];
        }
      }
      for (int b = 0; b < 256; b++) {  // final flush (:180-186)
        int64_t items = cur[b] - b * depth;
        std::memcpy(o + sob[b], cache.data() + b * depth, sizeof(U) * items);
        sob[b] += items;
      }
    }
    std::swap(in, o);
  }
  if (in != a) std::memcpy(a, in, sizeof(U) * n);  // P even: never taken for whole keys
}

// ---------------------------------------------------------------------------------
// Parallel restatements (RadixSortLsdParallel.cs)
// ---------------------------------------------------------------------------------
void parallel_for(int64_t count, int threads, const std::function<void(int64_t)>& fn) {
  if (threads <= 1 || count <= 1) {
    for (int64_t i = 0; i < count; i++) fn(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  int nt = int(std::min<int64_t>(threads, count));
  for (int t = 0; t < nt; t++)
    pool.emplace_back([&]() {
      for (int64_t i; (i = next.fetch_add(1)) < count;) fn(i);
    });
  for (auto& th : pool) th.join();
}

// HistogramByteComponentsPar: HistogramParallel.cs:163-222 (u32), :365-424 (i32),
// :487-555 (u64), :557-625 (i64).  Divide the range into leaves of at least
// parallelThreshold keys (raised to len/cores, :219-220), histogram each leaf serially,
// reduce by addition.  The reduction order does not change integer sums.
template <class U>
void histogram_byte_components_par(const U* a, int64_t l, int64_t r, int kind, uint32_t* counts,
                                   int threads, int64_t threshold) {
  constexpr int P = sizeof(U);
  int64_t len = r - l + 1;
  std::memset(counts, 0, sizeof(uint32_t) * P * 256);
  if (len <= 0) return;
  if (threads < 1) threads = 1;
  if (threshold * threads < len) threshold = len / threads;
  if (threshold < 1) threshold = 1;
  int64_t leaves = (len + threshold - 1) / threshold;
  std::vector<uint32_t> part(size_t(leaves) * P * 256);
  parallel_for(leaves, threads, [&](int64_t q) {
    int64_t lo = l + q * threshold, hi = std::min(r, lo + threshold - 1);
    histogram_byte_components<U>(a, lo, hi, kind, part.data() + q * P * 256);
  });
  for (int64_t q = 0; q < leaves; q++)
    for (int i = 0; i < P * 256; i++) counts[i] += part[q * P * 256 + i];
}

// Fully parallel u32 LSD: SortRadixPar(uint[], ParallelWorkQuantum = 64 Ki)
// RadixSortLsdParallel.cs:145-232.  Per digit pass:
//   ComputeStartOfBinsPar (:49-94): per-quantum histogram of this digit
//     (HistogramByteComponentsAcrossWorkQuantasQC, Histogram.cs:574-637), then start offsets
//     ordered bin-major, quantum-minor (stable);
//   one task per quantum runs SortRadixDeRandomizedInnerFunction (:96-135): scatter through
//     64-deep per-bin buffers, flush when full, final flush;
//   Task.WaitAll, swap buffers (:216-225).
// Scratch of one SortRadixPar call: the output array and, per work quantum, the 256 x 64-key
// de-randomisation buffers, the bin counts and the bin starts.  The reference allocates all of
// them once per call before its digit loop (RadixSortLsdParallel.cs:151-170); a caller that
// times repeated sorts allocates them once outside the timed region (RadixParWorkspace below).
template <class U>
struct RadixParScratch {
  U* out;            // n keys
  U* buffers;        // quanta x 256 x 64 keys
  uint32_t* count;   // quanta x 256
  int64_t* start;    // quanta x 256
};

// Fully parallel u32 LSD: SortRadixPar(uint[], ParallelWorkQuantum = 64 Ki)
// RadixSortLsdParallel.cs:145-232.  Per digit pass:
//   ComputeStartOfBinsPar (:49-94): per-quantum histogram of this digit
//     (HistogramByteComponentsAcrossWorkQuantasQC, Histogram.cs:574-637), then start offsets
//     ordered bin-major, quantum-minor (stable);
//   one task per quantum runs SortRadixDeRandomizedInnerFunction (:96-135): scatter through
//     64-deep per-bin buffers (one set per quantum, :159-161), flush when full, final flush;
//   Task.WaitAll, swap buffers (:216-225).
template <class U>
void sort_radix_par_full_ws(U* a, int64_t n, int kind, int64_t quantum, int threads, const RadixParScratch<U>& ws) {
  constexpr int P = sizeof(U);
  if (n <= 0) return;
  const int64_t quanta = (n + quantum - 1) / quantum;
  const int64_t depth = 64;  // BufferDepth (:158)
  U* in = a;
  U* out = ws.out;
  uint32_t* count = ws.count;
  int64_t* start = ws.start;
  for (int d = 0; d < P; d++) {
    parallel_for(quanta, threads, [&](int64_t q) {
      uint32_t* c = count + q * 256;
      std::memset(c, 0, 256 * sizeof(uint32_t));
      int64_t lo = q * quantum, hi = std::min(n, lo + quantum);
      for (int64_t i = lo; i < hi; i++) c[digit_of<U>(in[i], d, kind)]++;
    });
    // sizeOfBin and startOfBin (:66-91)
    int64_t run = 0;
    for (int b = 0; b < 256; b++)
      for (int64_t q = 0; q < quanta; q++) {
        start[q * 256 + b] = run;
        run += count[q * 256 + b];
      }
    parallel_for(quanta, threads, [&](int64_t q) {
      U* buf = ws.buffers + q * 256 * depth;
      int64_t idx[256];
      int64_t* sob = start + q * 256;
      for (int b = 0; b < 256; b++) idx[b] = b * depth;
      int64_t lo = q * quantum, hi = std::min(n, lo + quantum);
      for (int64_t i = lo; i < hi; i++) {
        unsigned b = digit_of<U>(in[i], d, kind);
        if (idx[b] < int64_t(b) * depth + depth) {
          buf[idx[b]++] = in[i];
        } else {
          std::memcpy(out + sob[b], buf + b * depth, sizeof(U) * depth);
          sob[b] += depth;
          buf[b * depth] = in[i];
          idx[b] = b * depth + 1;
        }
      }
      for (int b = 0; b < 256; b++) {
        int64_t items = idx[b] - int64_t(b) * depth;
        std::memcpy(out + sob[b], buf + b * depth, sizeof(U) * items);
        sob[b] += items;
      }
    });
    std::swap(in, out);
  }
  if (in != a) std::memcpy(a, in, sizeof(U) * n);
}

// Owns the scratch of sort_radix_par_full_ws for arrays of up to n keys.
struct RadixParWorkspace {
  int64_t n = 0, quantum = 0, width = 0;
  std::vector<unsigned char> out, buffers;
  std::vector<uint32_t> count;
  std::vector<int64_t> start;
  RadixParWorkspace(int64_t n_, int64_t quantum_, int64_t width_) : n(n_), quantum(quantum_), width(width_) {
    const int64_t quanta = (n + quantum - 1) / quantum;
    out.resize(size_t(n * width));
    buffers.resize(size_t(quanta * 256 * 64 * width));
    count.resize(size_t(quanta * 256));
    start.resize(size_t(quanta * 256));
  }
  template <class U>
  RadixParScratch<U> scratch() {
    return {reinterpret_cast<U*>(out.data()), reinterpret_cast<U*>(buffers.data()), count.data(), start.data()};
  }
};

template <class U>
void sort_radix_par_full(U* a, int64_t n, int kind, int64_t quantum, int threads) {
  if (n <= 0) return;
  if (quantum <= 0) quantum = 64 * 1024;
  RadixParWorkspace ws(n, quantum, int64_t(sizeof(U)));
  sort_radix_par_full_ws<U>(a, n, kind, quantum, threads, ws.scratch<U>());
}

// Partially parallel LSD: SortRadixPar(int[]) :446-495, (long[]) :560-609, (ulong[])
// :690-734.  Parallel fused histogram, serial prefix, serial per-digit scatter.
template <class U>
void sort_radix_par_partial(U* a, int64_t n, int kind, int threads) {
  constexpr int P = sizeof(U);
  if (n <= 0) return;
  uint32_t count[P * 256];
  int64_t start[P * 256];
  histogram_byte_components_par<U>(a, 0, n - 1, kind, count, threads, 16 * 1024);
  compute_start_of_bins<P>(count, start);
  std::vector<U> outv(n);
  U* in = a;
  U* out = outv.data();
  for (int d = 0; d < P; d++) {
    int64_t* sob = start + d * 256;
    for (int64_t i = 0; i < n; i++) out[sob[digit_of<U>(in[i], d, kind)]++] = in[i];
    std::swap(in, out);
  }
  if (in != a) std::memcpy(a, in, sizeof(U) * n);
}

// Key + item pairs: SortRadix<T>(T[] items, UInt32[] keys) RadixSortLsd.cs:1183-1237 and
// (T[] items, UInt64[] keys) :1245-1299.  Per pass: count this digit of the keys, exclusive
// scan, stable scatter of items and keys together, swap.  After an even number of passes
// the caller's arrays hold the result; that is the observable output restated here.  (The
// reference's returned Tuple.Item2 is its scratch array, which is not fully sorted; the
// caller's key array is.)
template <class U, class V>
void sort_pairs(U* keys, V* items, int64_t n, int kind) {
  constexpr int P = sizeof(U);
  if (n <= 0) return;
  std::vector<U> ko(n);
  std::vector<V> vo(n);
  U* kin = keys;
  U* kout = ko.data();
  V* vin = items;
  V* vout = vo.data();
  for (int d = 0; d < P; d++) {
    int64_t count[256] = {0};
    for (int64_t i = 0; i < n; i++) count[digit_of<U>(kin[i], d, kind)]++;
    int64_t end_of_bin[256];
    end_of_bin[0] = 0;
    for (int b = 1; b < 256; b++) end_of_bin[b] = end_of_bin[b - 1] + count[b - 1];
    for (int64_t i = 0; i < n; i++) {
      unsigned b = digit_of<U>(kin[i], d, kind);
      int64_t idx = end_of_bin[b]++;
      vout[idx] = vin[i];
      kout[idx] = kin[i];
    }
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  if (kin != keys) {
    std::memcpy(keys, kin, sizeof(U) * n);
    std::memcpy(items, vin, sizeof(V) * n);
  }
}

// ---------------------------------------------------------------------------------
// Radix top-k: SelectTopK(uint[] a, int k) SelectionTopKRadix.cs:142-171 with
// RadixSelectionTopKWordInner (:96-133) and the in-place movers (:19-94).  16-bit
// digits, MSD, in place.  Restated over the order-transformed unsigned key so the same
// routine serves u32 (the reference's only dtype) and the transformed i32/f32/u64 keys.
// Observable contract (what parity compares): a[k] is the k-th smallest (0-based) and
// a[k..n-1] holds exactly the multiset of the n-k largest values.  The prefix a[0..k-1]
// is clobbered by the movers in the reference and is not compared.
// ---------------------------------------------------------------------------------
template <class U>
inline unsigned word_of(U x, int shift) { return unsigned((x >> shift) & 0xFFFF); }

template <class U>
int64_t move_rob_into_kth_bin(U* a, int64_t sib, int64_t lib, int64_t srob, int64_t lrob, int shift,
                              unsigned kth) {  // :19-40
  int64_t eib = sib + lib - 1, erob = srob + lrob - 1;
  int64_t crob = srob, cib = sib;
  while (true) {
    for (; crob <= erob; crob++)
      if (word_of(a[crob], shift) == kth) break;
    if (crob <= erob)
      for (; cib <= eib; cib++)
        if (word_of(a[cib], shift) != kth) break;
    if (crob > erob || cib > eib) break;
    if (word_of(a[cib], shift) > kth) {
      std::swap(a[cib], a[crob]);
      cib++;
      crob++;
    } else {
      a[cib++] = a[crob++];
    }
  }
  return cib;
}

template <class U>
void move_rob_out_of_kth_bin(U* a, int64_t sib, int64_t lib, int64_t srob, int64_t lrob, int shift,
                             unsigned kth) {  // :43-62
  int64_t eib = sib + lib - 1, erob = srob + lrob - 1;
  int64_t crob = srob, cib = sib;
  while (true) {
    for (; cib <= eib; cib++)
      if (word_of(a[cib], shift) > kth) break;
    if (cib <= eib)
      for (; crob <= erob; crob++)
        if (word_of(a[crob], shift) < kth) break;
    if (crob > erob || cib > eib) break;
    a[crob++] = a[cib++];
  }
}

template <class U>
void move_lob_elements(U* a, int64_t slob, int64_t llob, int64_t sib, int64_t lib, int64_t skp1,
                       int64_t lrob, int shift, unsigned kth) {  // :66-94
  int64_t eib = sib + lib - 1, elob = slob + llob - 1, erob = skp1 + lrob - 1;
  int64_t clob = slob, cib = sib, crob = skp1;
  while (true) {
    int found_ib = 0, found_rob = 0;
    for (; clob <= elob; clob++) {
      if (word_of(a[clob], shift) == kth) { found_ib = 1; break; }
      if (word_of(a[clob], shift) > kth) { found_rob = 1; break; }
    }
    if (clob > elob) break;
    if (found_ib) {
      for (; cib <= eib; cib++)
        if (word_of(a[cib], shift) != kth) break;
      a[cib++] = a[clob++];
    }
    if (found_rob) {
      for (; crob <= erob; crob++)
        if (word_of(a[crob], shift) <= kth) break;
      a[crob++] = a[clob++];
    }
  }
}

// Returns 0 on success, -1 on the reference's "no elements in the k-th bin" exception
// (:131), which cannot happen for valid input.
template <class U>
int select_topk_word_inner(U* a, int64_t first, int64_t length, int shift, int64_t k) {  // :96-133
  int64_t last = first + length - 1;
  std::vector<int64_t> sob(65536 + 1);
  std::vector<int64_t> count(65536, 0);
  for (int64_t i = first; i <= last; i++) count[word_of(a[i], shift)]++;  // Histogram.cs:1129-1143
  sob[0] = first;
  sob[65536] = last + 1;
  for (int i = 1; i < 65536; i++) sob[i] = sob[i - 1] + count[i - 1];
  unsigned kth = 0;
  for (; kth < 65536; kth++) {
    int64_t bl = sob[kth + 1] - sob[kth];
    if (bl == 0) continue;
    if (k >= sob[kth] && k <= sob[kth + 1] - 1) break;
  }
  if (kth >= 65536) return -1;  // k == length: the reference reads past startOfBin here
  int64_t cib = move_rob_into_kth_bin(a, sob[kth], sob[kth + 1] - sob[kth], sob[kth + 1],
                                      last - sob[kth + 1] + 1, shift, kth);
  move_rob_out_of_kth_bin(a, cib, sob[kth + 1] - cib, sob[kth + 1], last - sob[kth + 1] + 1, shift,
                          kth);
  move_lob_elements(a, first, sob[kth] - first, sob[kth], sob[kth + 1] - sob[kth], sob[kth + 1],
                    last - sob[kth + 1] + 1, shift, kth);
  if (shift > 0) {
    shift = shift >= 16 ? shift - 16 : 0;
    int64_t bl = sob[kth + 1] - sob[kth];
    if (bl > 1) return select_topk_word_inner(a, sob[kth], bl, shift, k);
    if (bl == 1) return 0;
    return -1;
  }
  return 0;
}

template <class T, class U>
int select_topk(T* a, int64_t n, int64_t k, int kind) {
  if (n <= 0 || k < 0 || k >= n) return -2;
  U* u = reinterpret_cast<U*>(a);
  for (int64_t i = 0; i < n; i++) u[i] = order_bits<U>(u[i], kind);
  int rc = select_topk_word_inner<U>(u, 0, n, int(sizeof(U) * 8 - 16), k);
  for (int64_t i = 0; i < n; i++) u[i] = order_bits_inverse<U>(u[i], kind);
  return rc;
}

// ---------------------------------------------------------------------------------
// PartitionRadix(this uint[] a, int start, int length, int k / int[] k, int threshold = 1024)
// PartitionRadix.cs:135-210 with PartitionRadixMsdUIntInner (:15-63, the ulong twin :64-113).
// In place, MSD by 8-bit digits from the top: histogram of the current digit over
// [start, start + length) (HistogramOneByteComponent), bin starts, then the cycle-leader swap
// loop that moves every element into its bin (:32-41), then recursion into the bins that hold
// one of the k indices (:47-61).  A range shorter than `threshold` is sorted by the base case
// (Array.Sort, restated as std::sort on the order-transformed key).  Observable contract (what
// parity compares; the order inside each part is not): a[k_i] is the element the sorted
// subarray has at k_i, and every element between two consecutive k's (or a k and an end of the
// subarray) lies between their values.  k indexes the whole array; the k's ascend.
// ---------------------------------------------------------------------------------
template <class U>
void partition_radix_inner(U* a, int64_t start, int64_t length, int shift, const int64_t* k, int64_t kstart,
                           int64_t klength, int64_t threshold) {
  if (length < threshold) {
    std::sort(a + start, a + start + length);
    return;
  }
  const int64_t last = start + length - 1;
  int64_t count[256] = {0};
  for (int64_t i = start; i <= last; i++) count[(a[i] >> shift) & 0xFF]++;
  int64_t sob[257], eob[256];
  sob[0] = eob[0] = start;
  sob[256] = -1;  // sentinel (:28)
  for (int b = 1; b < 256; b++) sob[b] = eob[b] = sob[b - 1] + count[b - 1];
  int next_bin = 1;
  for (int64_t cur = start; cur <= last;) {
    U e = a[cur];
    unsigned d;
    while (eob[d = unsigned((e >> shift) & 0xFF)] != cur) std::swap(e, a[eob[d]++]);
    a[cur] = e;
    eob[d]++;
    while (next_bin < 256 && eob[next_bin - 1] == sob[next_bin]) next_bin++;
    cur = eob[next_bin - 1];
  }
  if (shift > 0) {
    const int nshift = shift >= 8 ? shift - 8 : 0;
    for (int b = 0, ki = int(kstart); b < 256 && ki < kstart + klength; b++) {
      if (sob[b] <= eob[b] && k[ki] >= sob[b] && k[ki] < eob[b]) {
        const int64_t ks = ki++;
        int64_t kl = 1;
        for (; ki < kstart + klength; ki++) {
          if (k[ki] >= sob[b] && k[ki] < eob[b]) kl++;
          else break;
        }
        partition_radix_inner<U>(a, sob[b], eob[b] - sob[b], nshift, k, ks, kl, threshold);
      }
    }
  }
}

template <class U>
void partition_radix(U* a, int64_t start, int64_t length, const int64_t* k, int64_t nk, int kind, int64_t threshold) {
  for (int64_t i = start; i < start + length; i++) a[i] = order_bits<U>(a[i], kind);
  if (nk > 0) partition_radix_inner<U>(a, start, length, int(sizeof(U) * 8 - 8), k, 0, nk, threshold);
  for (int64_t i = start; i < start + length; i++) a[i] = order_bits_inverse<U>(a[i], kind);
}

// std::sort stand-in for Array.Sort (introsort) on integer keys, and std::stable_sort on the
// transformed key for the cross-checks.
template <class U>
void stable_sort_transformed(U* a, int64_t n, int kind) {
  std::stable_sort(a, a + n, [kind](U x, U y) { return order_bits<U>(x, kind) < order_bits<U>(y, kind); });
}

}  // namespace

extern "C" {

// Serial SortRadixLsd: u32 (buffered), i32, u64, i64; f32/f64 via the float transform.
void orc_sort_radix_lsd_u32(uint32_t* a, int64_t n) { sort_radix_lsd<uint32_t>(a, n, UNSIGNED, true); }
void orc_sort_radix_lsd_i32(int32_t* a, int64_t n) {
  sort_radix_lsd<uint32_t>(reinterpret_cast<uint32_t*>(a), n, SIGNED, false);
}
void orc_sort_radix_lsd_f32(float* a, int64_t n) {
  sort_radix_lsd<uint32_t>(reinterpret_cast<uint32_t*>(a), n, FLOAT, false);
}
void orc_sort_radix_lsd_u64(uint64_t* a, int64_t n) { sort_radix_lsd<uint64_t>(a, n, UNSIGNED, false); }
void orc_sort_radix_lsd_i64(int64_t* a, int64_t n) {
  sort_radix_lsd<uint64_t>(reinterpret_cast<uint64_t*>(a), n, SIGNED, false);
}
void orc_sort_radix_lsd_f64(double* a, int64_t n) {
  sort_radix_lsd<uint64_t>(reinterpret_cast<uint64_t*>(a), n, FLOAT, false);
}

// Parallel SortRadixPar: fully parallel for u32 (:145-232); partially parallel for i32/u64/i64
// (:446-734); f32/f64 use the fully parallel structure with the float transform (the
// reference has no float LSD; the transform is Histogram.cs:1210-1288).
// SortRadixPar on a workspace made once (orc_radix_par_ws_create) for arrays of up to its n
// keys of `width` bytes: the timed CPU baseline allocates nothing inside the sort.
void* orc_radix_par_ws_create(int64_t n, int64_t quantum, int width) {
  if (n < 0 || (width != 4 && width != 8)) return nullptr;
  if (quantum <= 0) quantum = 64 * 1024;
  return new RadixParWorkspace(n, quantum, width);
}
void orc_radix_par_ws_destroy(void* ws) { delete static_cast<RadixParWorkspace*>(ws); }
int orc_sort_radix_par_ws_k32(void* wsp, uint32_t* a, int64_t n, int kind, int threads) {
  auto* ws = static_cast<RadixParWorkspace*>(wsp);
  if (!ws || ws->width != 4 || n > ws->n) return 1;
  sort_radix_par_full_ws<uint32_t>(a, n, kind, ws->quantum, threads, ws->scratch<uint32_t>());
  return 0;
}
int orc_sort_radix_par_ws_k64(void* wsp, uint64_t* a, int64_t n, int kind, int threads) {
  auto* ws = static_cast<RadixParWorkspace*>(wsp);
  if (!ws || ws->width != 8 || n > ws->n) return 1;
  sort_radix_par_full_ws<uint64_t>(a, n, kind, ws->quantum, threads, ws->scratch<uint64_t>());
  return 0;
}

// The benchmark's uniform uint32 keys, restated so that the CPU baseline needs no library of
// the product: element i belongs to chunk c = i / 65536 and chunk c draws from PCG32 (O'Neill's
// published minimal generator, pcg-random.org) seeded with (initstate = seed, initseq = c).
// tests/test_oracle.py checks it against the generator the GPU workloads use.
void orc_gen_u32_uniform(uint32_t* out, int64_t n, uint64_t seed, int threads) {
  const int64_t chunk = 65536;
  const int64_t chunks = (n + chunk - 1) / chunk;
  parallel_for(chunks, threads, [&](int64_t c) {
    uint64_t inc = (uint64_t(c) << 1u) | 1u;
    uint64_t state = 0u;
    auto step = [&]() {
      uint64_t old = state;
      state = old * 6364136223846793005ULL + inc;
      uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
      uint32_t rot = uint32_t(old >> 59u);
      return (xs >> rot) | (xs << ((32u - rot) & 31u));
    };
    step();
    state += seed;
    step();
    const int64_t lo = c * chunk, hi = std::min(n, lo + chunk);
    for (int64_t i = lo; i < hi; i++) out[i] = step();
  });
}

void orc_sort_radix_par_u32(uint32_t* a, int64_t n, int64_t quantum, int threads) {
  sort_radix_par_full<uint32_t>(a, n, UNSIGNED, quantum, threads);
}
void orc_sort_radix_par_f32(float* a, int64_t n, int64_t quantum, int threads) {
  sort_radix_par_full<uint32_t>(reinterpret_cast<uint32_t*>(a), n, FLOAT, quantum, threads);
}
void orc_sort_radix_par_f64(double* a, int64_t n, int64_t quantum, int threads) {
  sort_radix_par_full<uint64_t>(reinterpret_cast<uint64_t*>(a), n, FLOAT, quantum, threads);
}
void orc_sort_radix_par_u64_full(uint64_t* a, int64_t n, int64_t quantum, int threads) {
  sort_radix_par_full<uint64_t>(a, n, UNSIGNED, quantum, threads);
}
void orc_sort_radix_par_i32(int32_t* a, int64_t n, int threads) {
  sort_radix_par_partial<uint32_t>(reinterpret_cast<uint32_t*>(a), n, SIGNED, threads);
}
void orc_sort_radix_par_u64(uint64_t* a, int64_t n, int threads) {
  sort_radix_par_partial<uint64_t>(a, n, UNSIGNED, threads);
}
void orc_sort_radix_par_i64(int64_t* a, int64_t n, int threads) {
  sort_radix_par_partial<uint64_t>(reinterpret_cast<uint64_t*>(a), n, SIGNED, threads);
}

// Pairs (keys of 4 or 8 bytes; 4-byte items).  kind: 0 unsigned, 1 signed, 2 float.
void orc_sort_pairs_k32_v32(uint32_t* keys, uint32_t* items, int64_t n, int kind) {
  sort_pairs<uint32_t, uint32_t>(keys, items, n, kind);
}
void orc_sort_pairs_k64_v32(uint64_t* keys, uint32_t* items, int64_t n, int kind) {
  sort_pairs<uint64_t, uint32_t>(keys, items, n, kind);
}

// Histograms: counts[P][256]; signed kinds flip the top digit (Histogram.cs:1014, :1049;
// HistogramParallel.cs:397, :598); float kinds use the float transform.
void orc_histogram_byte_components_k32(const uint32_t* a, int64_t l, int64_t r, int kind, uint32_t* counts) {
  histogram_byte_components<uint32_t>(a, l, r, kind, counts);
}
void orc_histogram_byte_components_k64(const uint64_t* a, int64_t l, int64_t r, int kind, uint32_t* counts) {
  histogram_byte_components<uint64_t>(a, l, r, kind, counts);
}
void orc_histogram_byte_components_par_k32(const uint32_t* a, int64_t l, int64_t r, int kind, uint32_t* counts,
                                           int threads) {
  histogram_byte_components_par<uint32_t>(a, l, r, kind, counts, threads, 16 * 1024);
}
void orc_histogram_byte_components_par_k64(const uint64_t* a, int64_t l, int64_t r, int kind, uint32_t* counts,
                                           int threads) {
  histogram_byte_components_par<uint64_t>(a, l, r, kind, counts, threads, 16 * 1024);
}

// SelectTopK over 4- or 8-byte keys (kind as above).  Returns 0 on success.
int orc_select_topk_k32(uint32_t* a, int64_t n, int64_t k, int kind) {
  return select_topk<uint32_t, uint32_t>(a, n, k, kind);
}
int orc_select_topk_k64(uint64_t* a, int64_t n, int64_t k, int kind) {
  return select_topk<uint64_t, uint64_t>(a, n, k, kind);
}

// PartitionRadix over [start, start + length) by the ascending indices k[0..nk) (absolute).
void orc_partition_radix_k32(uint32_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk, int kind,
                             int64_t threshold) {
  partition_radix<uint32_t>(a, start, length, k, nk, kind, threshold);
}
void orc_partition_radix_k64(uint64_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk, int kind,
                             int64_t threshold) {
  partition_radix<uint64_t>(a, start, length, k, nk, kind, threshold);
}

// Cross-check helpers.
void orc_std_sort_u32(uint32_t* a, int64_t n) { std::sort(a, a + n); }
void orc_std_sort_i32(int32_t* a, int64_t n) { std::sort(a, a + n); }
void orc_std_sort_u64(uint64_t* a, int64_t n) { std::sort(a, a + n); }
void orc_std_sort_i64(int64_t* a, int64_t n) { std::sort(a, a + n); }
void orc_stable_sort_transformed_k32(uint32_t* a, int64_t n, int kind) { stable_sort_transformed<uint32_t>(a, n, kind); }
void orc_stable_sort_transformed_k64(uint64_t* a, int64_t n, int kind) { stable_sort_transformed<uint64_t>(a, n, kind); }
// Stable argsort by transformed key: perm[i] = original index of the i-th output element.
void orc_stable_argsort_k32(const uint32_t* a, int64_t n, int kind, uint32_t* perm) {
  for (int64_t i = 0; i < n; i++) perm[i] = uint32_t(i);
  std::stable_sort(perm, perm + n, [&](uint32_t x, uint32_t y) {
    return order_bits<uint32_t>(a[x], kind) < order_bits<uint32_t>(a[y], kind);
  });
}
void orc_stable_argsort_k64(const uint64_t* a, int64_t n, int kind, uint32_t* perm) {
  for (int64_t i = 0; i < n; i++) perm[i] = uint32_t(i);
  std::stable_sort(perm, perm + n, [&](uint32_t x, uint32_t y) {
    return order_bits<uint64_t>(a[x], kind) < order_bits<uint64_t>(a[y], kind);
  });
}
int orc_hardware_threads(void) {
  unsigned t = std::thread::hardware_concurrency();
  return t ? int(t) : 1;
}

}  // extern "C"
