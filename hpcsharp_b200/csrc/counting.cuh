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
// `flip` is the signed transform's top-bit mask (0 for unsigned keys).
template <class T>
__global__ void __launch_bounds__(COUNT_NT, 1) count_hist_kernel(const T* __restrict__ a, int64_t n, uint32_t flip,
                                                                 uint32_t* __restrict__ counts) {
  constexpr int BINS = CountTraits<T>::BINS;
  extern __shared__ __align__(16) uint32_t sh[];
  const int tid = threadIdx.x, lane = tid & 31;
  const int64_t stride = int64_t(gridDim.x) * COUNT_NT;
  if (BINS == 256) {
    for (int i = tid; i < 256 * 32; i += COUNT_NT) sh[i] = 0u;
    __syncthreads();
    for (int64_t i = int64_t(blockIdx.x) * COUNT_NT + tid; i < n; i += stride) {
      const uint32_t b = (uint32_t(a[i]) ^ flip) & 0xFFu;
      atomicAdd(&sh[b * 32 + lane], 1u);
    }
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
    const int64_t per_round = stride * COUNT_ROUND;
    for (int64_t r0 = 0; r0 < n; r0 += per_round) {  // the same number of rounds in every thread
#pragma unroll 4
      for (int g = 0; g < COUNT_ROUND; g++) {
        const int64_t i = r0 + g * stride + int64_t(blockIdx.x) * COUNT_NT + tid;
        if (i < n) {
          const uint32_t b = (uint32_t(a[i]) ^ flip) & 0xFFFFu;
          const uint32_t sh16 = (b & 1u) << 4;
          const uint32_t inc = 1u << sh16;
          const uint32_t old = atomicAdd(&sh[b >> 1], inc);
          if ((old + inc) & ~old & 0x80008000u) {
            atomicSub(&sh[b >> 1], 0x8000u << sh16);
            atomicAdd(counts + b, 0x8000u);
          }
        }
      }
      __syncthreads();
    }
    for (int w = tid; w < BINS / 2; w += COUNT_NT) {
      const uint32_t v = sh[w];
      if (v & 0xFFFFu) atomicAdd(counts + 2 * w, v & 0xFFFFu);
      if (v >> 16) atomicAdd(counts + 2 * w + 1, v >> 16);
    }
  }
}

// Exclusive scan of the counts into starts[0..BINS] (starts[BINS] = n), one CTA.
template <int BINS>
__global__ void __launch_bounds__(COUNT_NT) count_scan_kernel(const uint32_t* __restrict__ counts,
                                                              int64_t* __restrict__ starts) {
  constexpr int PER = BINS / COUNT_NT > 0 ? BINS / COUNT_NT : 1;  // bins per thread
  __shared__ int64_t s_w[COUNT_NT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b0 = tid * PER;
  int64_t sum = 0;
  for (int q = 0; q < PER; q++)
    if (b0 + q < BINS) sum += counts[b0 + q];
  int64_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  int64_t base = 0;
  for (int w = 0; w < warp; w++) base += s_w[w];
  int64_t run = base + incl - sum;
  for (int q = 0; q < PER; q++) {
    if (b0 + q < BINS) {
      starts[b0 + q] = run;
      run += counts[b0 + q];
    }
  }
  if (tid == COUNT_NT - 1) starts[BINS] = base + incl;
}

// Fills out[i] with the value v whose run [starts[v], starts[v+1]) holds i.  Each thread
// writes 16-byte vectors: it finds the bin of the vector's first element by binary search over
// the starts, then walks forward across bin boundaries.  The ragged tail is written with
// scalar stores.  `flip` maps a bin back to its raw bits.
template <class T>
__global__ void __launch_bounds__(256) count_fill_kernel(T* __restrict__ out, int64_t n,
                                                         const int64_t* __restrict__ starts, uint32_t flip) {
  constexpr int BINS = CountTraits<T>::BINS;
  constexpr int VEC = 16 / int(sizeof(T));
  const int64_t nvec = n / VEC;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  auto bin_of = [&](int64_t i) {  // largest v with starts[v] <= i (runs may be empty)
    int lo = 0, hi = BINS - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (starts[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  };
  const bool aligned = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
  for (int64_t vi = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; vi < nvec + 1; vi += stride) {
    const int64_t first = vi * VEC;
    if (first >= n) break;
    int v = bin_of(first);
    int64_t next = starts[v + 1];
    if (vi < nvec && aligned) {
      union {
        uint4 u;
        T e[VEC];
      } pack;
#pragma unroll
      for (int q = 0; q < VEC; q++) {
        const int64_t i = first + q;
        while (i >= next && v < BINS - 1) {
          v++;
          next = starts[v + 1];
        }
        pack.e[q] = T(uint32_t(v) ^ flip);
      }
      reinterpret_cast<uint4*>(out)[vi] = pack.u;
    } else {
      const int64_t last = vi < nvec ? first + VEC : n;
      for (int64_t i = first; i < last; i++) {
        while (i >= next && v < BINS - 1) {
          v++;
          next = starts[v + 1];
        }
        out[i] = T(uint32_t(v) ^ flip);
      }
    }
  }
}

}  // namespace hpcs
