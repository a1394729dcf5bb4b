// Counting sort of 8- and 16-bit keys (HPCsharp's SortCountingInPlace[Par], CountingSort.cs:41,
// :78, :115, :152 and CountingSortParallel.cs:22-99): one histogram read of the keys, an
// exclusive scan of the 2^8 or 2^16 counts, and one write that fills each value's run.  The
// result equals the radix sort's (equal keys are identical bit patterns).  Signed keys are
// counted by their order transform (top bit flipped) and written back as raw bits.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace hpcs {

template <class T>
struct CountTraits;
template <>
struct CountTraits<uint8_t> {
  static constexpr int BINS = 256;
};
template <>
struct CountTraits<uint16_t> {
  static constexpr int BINS = 65536;
};

constexpr int COUNT_NT = 1024;
constexpr int COUNT_ROUND = 16;  // keys per thread between barriers (16-bit counters)

// Per-CTA histogram.  8-bit keys: lane-private 32-bit counters ([256][32], conflict-free);
// 16-bit keys: 16-bit counters, two per word (128 KiB), a counter that reaches 0x8000 moved
// to the global counts by the thread whose increment reached it.  One increment per key, so
// exactly one thread sees each crossing; the keys go in rounds of COUNT_ROUND per thread
// with a barrier between rounds, so before a crossing thread's subtraction lands at most one
// round of the CTA's increments (16384) can reach the counter: it stays below 0xC000.
// The keys are read as 16-byte vectors (visit_keys for 8-bit keys; two vectors per thread and
// round for 16-bit keys), the unaligned head and ragged tail by the grid's first warp.
// `flip` is the signed transform's top-bit mask (0 for unsigned keys).
template <class T>
__global__ void __launch_bounds__(COUNT_NT) count_hist_kernel(const T* __restrict__ a, int64_t n, uint32_t flip,
                                                              uint32_t* __restrict__ counts) {
  constexpr int BINS = CountTraits<T>::BINS;
  constexpr int E = int(16 / sizeof(T));
  extern __shared__ __align__(16) uint32_t sh[];
  const int tid = threadIdx.x, lane = tid & 31;
  if (BINS == 256) {
    for (int i = tid; i < 256 * 32; i += COUNT_NT) sh[i] = 0u;
    __syncthreads();
    visit_keys<T, 4>(a, n, [&](const T* k, int nv) {
#pragma unroll
      for (int e = 0; e < E; e++)
        if (e < nv) atomicAdd(&sh[((uint32_t(k[e]) ^ flip) & 0xFFu) * 32 + lane], 1u);
    });
    __syncthreads();
    for (int b = tid; b < 256; b += COUNT_NT) {
      uint32_t c = 0;
#pragma unroll 8
      for (int q = 0; q < 32; q++) c += sh[b * 32 + ((q + lane) & 31)];
      if (c) atomicAdd(counts + b, c);
    }
  } else {
    for (int i = tid; i < BINS / 2; i += COUNT_NT) sh[i] = 0u;
    __syncthreads();
    auto bump = [&](uint32_t key) {
      const uint32_t b = (key ^ flip) & 0xFFFFu;
      const uint32_t sh16 = (b & 1u) << 4;
      const uint32_t inc = 1u << sh16;
      const uint32_t old = atomicAdd(&sh[b >> 1], inc);
      if ((old + inc) & ~old & 0x80008000u) {
        atomicSub(&sh[b >> 1], 0x8000u << sh16);
        atomicAdd(counts + b, 0x8000u);
      }
    };
    union Vec {
      uint4 v;
      T k[E];
    };
    constexpr int VPR = COUNT_ROUND / E;  // vectors per thread and round
    const uintptr_t addr = reinterpret_cast<uintptr_t>(a);
    int64_t head = int64_t(((16u - uint32_t(addr & 15u)) & 15u) / sizeof(T));
    if (head > n) head = n;
    const int64_t nvec = (n - head) / E;
    const int64_t rest = head + nvec * E;
    const uint4* vp = reinterpret_cast<const uint4*>(a + head);
    const int64_t G = int64_t(gridDim.x) * COUNT_NT;
    const int64_t gtid = int64_t(blockIdx.x) * COUNT_NT + tid;
    // the next round's vectors are loaded before this round's keys are counted, so two rounds
    // of loads are in flight (one round alone left the loop waiting on memory)
    Vec v[VPR], vn[VPR];
#pragma unroll
    for (int j = 0; j < VPR; j++) {
      const int64_t idx = j * G + gtid;
      v[j].v = idx < nvec ? __ldg(vp + idx) : make_uint4(0u, 0u, 0u, 0u);
    }
    for (int64_t base = 0; base < nvec; base += G * VPR) {  // the same number of rounds in every thread
#pragma unroll
      for (int j = 0; j < VPR; j++) {
        const int64_t idx = base + G * VPR + j * G + gtid;
        vn[j].v = idx < nvec ? __ldg(vp + idx) : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int j = 0; j < VPR; j++)
        if (base + j * G + gtid < nvec) {
#pragma unroll
          for (int e = 0; e < E; e++) bump(uint32_t(v[j].k[e]));
        }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < VPR; j++) v[j] = vn[j];
    }
    if (blockIdx.x == 0 && tid == 0) {  // fewer than 2E keys outside the vectors
      for (int64_t i = 0; i < head; i++) bump(uint32_t(a[i]));
      for (int64_t i = rest; i < n; i++) bump(uint32_t(a[i]));
    }
    __syncthreads();
    for (int w = tid; w < BINS / 2; w += COUNT_NT) {
      const uint32_t v = sh[w];
      if (v & 0xFFFFu) atomicAdd(counts + 2 * w, v & 0xFFFFu);
      if (v >> 16) atomicAdd(counts + 2 * w + 1, v >> 16);
    }
  }
}

// Exclusive scan of the counts into starts[0..BINS] (starts[BINS] = n), in CTAs of
// count_scan_nt<BINS>() bins: CTA j adds up the counts of the bins before its chunk (coalesced
// reads), then scans its own bins.  Each non-empty bin also records itself as the bin of every
// fill range's first and last output that it holds (range r = outputs [r*R, min(n, (r+1)*R))):
// range_lo[r] and range_hi[r], so the fill needs no search for its ranges' bounds.  A bin
// spanning many ranges records them in a loop of its own thread.
template <int BINS>
__host__ __device__ constexpr int count_scan_nt() {
  return BINS < 1024 ? BINS : 1024;
}

template <int BINS>
__global__ void __launch_bounds__(1024) count_scan_kernel(const uint32_t* __restrict__ counts, int64_t n, int64_t R,
                                                          int64_t* __restrict__ starts, int32_t* __restrict__ range_lo,
                                                          int32_t* __restrict__ range_hi) {
  constexpr int NT = count_scan_nt<BINS>();
  constexpr int NW = NT / 32;
  __shared__ int64_t s_w[NW];
  __shared__ int64_t s_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b0 = blockIdx.x * NT;
  int64_t pre = 0;
#pragma unroll 8
  for (int i = tid; i < b0; i += NT) pre += counts[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pre += __shfl_xor_sync(0xFFFFFFFFu, pre, o);
  if (lane == 0) s_w[warp] = pre;
  __syncthreads();
  if (tid == 0) {
    int64_t t = 0;
    for (int w = 0; w < NW; w++) t += s_w[w];
    s_base = t;
  }
  __syncthreads();
  const int b = b0 + tid;
  const int64_t c = counts[b];
  int64_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  __syncthreads();  // s_w is reused
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  int64_t excl = s_base + incl - c;
  for (int w = 0; w < warp; w++) excl += s_w[w];
  starts[b] = excl;
  if (b == BINS - 1) starts[BINS] = excl + c;
  if (c > 0) {
    const int64_t end = excl + c;  // this bin holds outputs [excl, end)
    for (int64_t r = (excl + R - 1) / R; r * R < end; r++) range_lo[r] = b;
    for (int64_t r = (excl + R) / R - 1; (r + 1) * R - 1 < end && (r + 1) * R - 1 < n; r++) range_hi[r] = b;
    if (n - 1 >= excl && n - 1 < end) range_hi[(n - 1) / R] = b;  // the last range ends at n - 1
  }
}

// Fills out[i] with the value v whose run [starts[v], starts[v+1]) holds i.  Each CTA takes
// ranges of count_fill_range outputs (grid-stride): the scan recorded the bins of the range's
// first and last output (range_lo, range_hi), and the CTA copies those bins' starts into shared memory
// (when there are at most COUNT_FILL_SMEM of them; otherwise the searches below stay in
// global memory).  When the range's runs average at least COUNT_FILL_RUN_VECS vectors, the CTA
// writes it run by run (replicated 16-byte vectors, single elements at the run's ends).
// Otherwise each thread writes 16-byte vectors: the bin of a vector's first element by binary
// search over the copied starts, then a walk across bin boundaries.  Unaligned
// outputs and the ragged end are written by scalar stores.  `flip` maps a bin back to its raw
// bits.
constexpr int COUNT_FILL_NT = 256;
constexpr int COUNT_FILL_VPT = 16;  // vectors per thread and range
constexpr int COUNT_FILL_SMEM = 2048;
// mean run length (vectors) from which a range is written bin by bin.  Measured on B200 (u16
// keys): runs of 512 vectors, bin by bin 0.366 ms per 2^28-key sort against 0.394 ms with the
// per-vector search; runs of 128 vectors, 97 us against 62 us for the fill of 2^26 keys.
constexpr int COUNT_FILL_RUN_VECS = 256;

template <class T>
__host__ __device__ constexpr int64_t count_fill_range() {
  return int64_t(COUNT_FILL_NT) * COUNT_FILL_VPT * (16 / int64_t(sizeof(T)));
}

template <class T>
__global__ void __launch_bounds__(COUNT_FILL_NT) count_fill_kernel(T* __restrict__ out, int64_t n,
                                                                   const int64_t* __restrict__ starts,
                                                                   const int32_t* __restrict__ range_lo,
                                                                   const int32_t* __restrict__ range_hi,
                                                                   uint32_t flip) {
  constexpr int BINS = CountTraits<T>::BINS;
  constexpr int VEC = 16 / int(sizeof(T));
  constexpr int64_t R = count_fill_range<T>();  // outputs per range
  __shared__ int64_t s_st[COUNT_FILL_SMEM + 1];
  __shared__ int s_lo, s_cnt;
  auto bin_of_global = [&](int64_t i) {  // largest v with starts[v] <= i (runs may be empty)
    int lo = 0, hi = BINS - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (starts[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  };
  const bool aligned = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
  const int tid = threadIdx.x;
  for (int64_t a = int64_t(blockIdx.x) * R; a < n; a += int64_t(gridDim.x) * R) {
    const int64_t e = a + R < n ? a + R : n;
    if (tid == 0) {
      const int lo = range_lo[a / R], hi = range_hi[a / R];  // the bins of outputs a and e - 1
      s_lo = lo;
      s_cnt = hi - lo + 2;  // starts[lo .. hi + 1]
    }
    __syncthreads();
    const int lo = s_lo, cnt = s_cnt;
    const bool local = cnt <= COUNT_FILL_SMEM + 1;
    if (local)
      for (int i = tid; i < cnt; i += COUNT_FILL_NT) s_st[i] = starts[lo + i];
    __syncthreads();
    // bin of output i in [a, e) and the start of the next bin
    auto find = [&](int64_t i, int& v, int64_t& next) {
      if (local) {
        int l = 0, h = cnt - 2;
        while (l < h) {
          const int mid = (l + h + 1) >> 1;
          if (s_st[mid] <= i) l = mid;
          else h = mid - 1;
        }
        v = lo + l;
        next = s_st[l + 1];
      } else {
        v = bin_of_global(i);
        next = starts[v + 1];
      }
    };
    auto advance = [&](int& v, int64_t& next) {
      v++;
      next = local ? s_st[v - lo + 1] : starts[v + 1];
    };
    if (aligned && local && (e - a) >= int64_t(cnt) * COUNT_FILL_RUN_VECS * VEC) {
      // long runs: the CTA writes the range bin by bin, each run's aligned body as replicated
      // vectors (no search per vector) and its ragged ends as single elements
      for (int bi = 0; bi + 1 < cnt; bi++) {
        const int64_t rs = s_st[bi] > a ? s_st[bi] : a;
        const int64_t re = s_st[bi + 1] < e ? s_st[bi + 1] : e;
        if (rs >= re) continue;
        const T val = T(uint32_t(lo + bi) ^ flip);
        const int64_t v0 = (rs + VEC - 1) / VEC, v1 = re / VEC;  // whole vectors [v0, v1)
        const int64_t head_end = v0 * VEC < re ? v0 * VEC : re;
        for (int64_t i = rs + tid; i < head_end; i += COUNT_FILL_NT) out[i] = val;
        if (v1 >= v0) {  // else the run lies inside one vector and the head loop wrote it
          const uint32_t w = sizeof(T) == 1 ? uint32_t(uint8_t(val)) * 0x01010101u : uint32_t(uint16_t(val)) * 0x00010001u;
          const uint4 rep = make_uint4(w, w, w, w);
          for (int64_t q = v0 + tid; q < v1; q += COUNT_FILL_NT) reinterpret_cast<uint4*>(out)[q] = rep;
          for (int64_t i = v1 * VEC + tid; i < re; i += COUNT_FILL_NT) out[i] = val;
        }
      }
    } else if (aligned) {
      const int64_t nvec = (e - a) / VEC;  // whole vectors of the range (a is a multiple of VEC)
      for (int64_t q = tid; q < nvec; q += COUNT_FILL_NT) {
        const int64_t first = a + q * VEC;
        int v;
        int64_t next;
        find(first, v, next);
        if (first + VEC <= next) {  // the whole vector is one value's run: the value replicated
          const uint32_t val = uint32_t(v) ^ flip;
          const uint32_t w = sizeof(T) == 1 ? (val & 0xFFu) * 0x01010101u : (val & 0xFFFFu) * 0x00010001u;
          reinterpret_cast<uint4*>(out)[first / VEC] = make_uint4(w, w, w, w);
          continue;
        }
        union {
          uint4 u;
          T e[VEC];
        } pack;
#pragma unroll
        for (int r = 0; r < VEC; r++) {
          while (first + r >= next && v < BINS - 1) advance(v, next);
          pack.e[r] = T(uint32_t(v) ^ flip);
        }
        reinterpret_cast<uint4*>(out)[first / VEC] = pack.u;
      }
      for (int64_t i = a + nvec * VEC + tid; i < e; i += COUNT_FILL_NT) {
        int v;
        int64_t next;
        find(i, v, next);
        out[i] = T(uint32_t(v) ^ flip);
      }
    } else {
      for (int64_t i = a + tid; i < e; i += COUNT_FILL_NT) {
        int v;
        int64_t next;
        find(i, v, next);
        out[i] = T(uint32_t(v) ^ flip);
      }
    }
    __syncthreads();  // the copied starts are read before the next range replaces them
  }
}

}  // namespace hpcs
