// Device-side building blocks shared by the radix kernels (sm_100a).
//
// * KeyOrder<U, KIND>: maps a key's bit pattern to an unsigned integer whose ascending
//   order is the key's order.  These are HPCsharp's own transforms:
//     signed   top byte ^ 0x80      RadixSortLsd.cs:288-293 (i32), :464-469 (i64)
//     float    sign 0: flip sign bit; sign 1: flip all bits
//                                   Histogram.cs:1210-1248 (f32), :1250-1288 (f64)
//   The transform is applied to the digit only; keys are moved as raw bits.
// * PTX wrappers for mbarriers and 1-D bulk async copies (cp.async.bulk, no multicast),
//   relaxed GPU-scope loads/stores for the decoupled look-back, and the global timer
//   used to bound every spin.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hpcs {

enum KeyKind : int { KIND_UNSIGNED = 0, KIND_SIGNED = 1, KIND_FLOAT = 2 };

// Device error word bits (the host maps them to status codes).
enum DeviceError : uint32_t {
  DERR_LOOKBACK_TIMEOUT = 1u << 0,
  DERR_TMA_TIMEOUT = 1u << 1,
  DERR_BOUNDS = 1u << 2,
  DERR_QUEUE_TIMEOUT = 1u << 3,
};

template <class U, int KIND>
struct KeyOrder {
  static constexpr int BITS = int(sizeof(U) * 8);
  static constexpr U TOP = U(1) << (BITS - 1);
  __host__ __device__ __forceinline__ static U to_ordered(U x) {
    if (KIND == KIND_SIGNED) return x ^ TOP;
    if (KIND == KIND_FLOAT) {
      // sign 1 -> ~x ; sign 0 -> x ^ TOP
      U mask = U(0) - U(x >> (BITS - 1));  // all ones when negative
      return x ^ (mask | TOP);
    }
    return x;
  }
  __host__ __device__ __forceinline__ static U from_ordered(U y) {
    if (KIND == KIND_SIGNED) return y ^ TOP;
    if (KIND == KIND_FLOAT) {
      U mask = U(0) - U((~y) >> (BITS - 1));  // all ones when the original was negative
      return y ^ (mask | TOP);
    }
    return y;
  }
  __device__ __forceinline__ static uint32_t digit(U x, int shift) {
    return uint32_t(to_ordered(x) >> shift) & 0xFFu;
  }
};

// Digit of one pass with the order transform folded in: one byte permute (plus the sign
// mask for floats) instead of the full to_ordered + shift + mask.  Only the byte the pass
// reads is transformed: signed keys flip bit 7 of the top byte, floats flip every bit of a
// negative key and the sign bit of a positive one.
template <class U, int KIND>
struct Digit;
template <int KIND>
struct Digit<uint32_t, KIND> {
  uint32_t sel;
  __device__ __forceinline__ explicit Digit(int shift) : sel(0x4440u | uint32_t(shift >> 3)) {}
  __device__ __forceinline__ uint32_t operator()(uint32_t x) const {
    if (KIND == KIND_SIGNED) x ^= 0x80000000u;
    if (KIND == KIND_FLOAT) x ^= uint32_t(int32_t(x) >> 31) | 0x80000000u;
    return __byte_perm(x, 0u, sel);
  }
};
template <int KIND>
struct Digit<uint64_t, KIND> {
  uint32_t sel, top;
  bool hi_word;
  __device__ __forceinline__ explicit Digit(int shift)
      : sel(0x4440u | uint32_t((shift >> 3) & 3)), top(shift >= 32 ? 0x80000000u : 0u), hi_word(shift >= 32) {}
  __device__ __forceinline__ uint32_t operator()(uint64_t x) const {
    const uint32_t hi = uint32_t(x >> 32);
    uint32_t w = hi_word ? hi : uint32_t(x);
    if (KIND == KIND_SIGNED) w ^= top;
    if (KIND == KIND_FLOAT) w ^= uint32_t(int32_t(hi) >> 31) | top;
    return __byte_perm(w, 0u, sel);
  }
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- mbarrier -------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and leaves the barrier alone) if `limit_ns` passes.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  uint64_t t0 = global_timer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// ---- 1-D bulk async copy global -> shared (TMA engine, no tensor map, no multicast) ----
// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ---- relaxed GPU-scope accesses for the look-back status words --------------------
__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}

// Streaming 128-bit read-only load.
__device__ __forceinline__ uint4 ldg_stream_v4(const void* p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// Calls f(k, nv) for the keys of keys[0..n) in groups of E = 16 / sizeof(U): k holds E keys,
// the first nv of them valid.  The 16-byte-aligned body goes as vectors, VPT per thread in
// flight (vector j of a round at base + j*G + global thread id, G = grid threads); the
// unaligned head (< E keys) and the ragged tail (< E keys) go to lanes 0 and 1 of the grid's
// first warp.  Every lane of a warp makes the same calls (nv = 0 pads), so f may use warp
// collectives.
template <class U, int VPT, class F>
__device__ __forceinline__ void visit_keys(const U* __restrict__ keys, int64_t n, F&& f) {
  constexpr int E = int(16 / sizeof(U));
  union Vec {
    uint4 v;
    U k[E];
  };
  const uintptr_t addr = reinterpret_cast<uintptr_t>(keys);
  int64_t head = int64_t(((16u - uint32_t(addr & 15u)) & 15u) / sizeof(U));
  if (head > n) head = n;
  const int64_t nvec = (n - head) / E;
  const int64_t rest = head + nvec * E;  // first key of the tail
  const uint4* vp = reinterpret_cast<const uint4*>(keys + head);
  const int64_t G = int64_t(gridDim.x) * blockDim.x;
  const int64_t gtid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int64_t base = 0; base < nvec; base += G * VPT) {  // uniform over the grid
    Vec v[VPT];
#pragma unroll
    for (int j = 0; j < VPT; j++) {
      const int64_t idx = base + j * G + gtid;
      v[j].v = idx < nvec ? __ldg(vp + idx) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int j = 0; j < VPT; j++) f(v[j].k, base + j * G + gtid < nvec ? E : 0);
  }
  if (blockIdx.x == 0 && threadIdx.x < 32) {
    const int lane = threadIdx.x;
    Vec v;
    v.v = make_uint4(0u, 0u, 0u, 0u);
    int nv = 0;
    if (lane == 0) {
      nv = int(head);
      for (int e = 0; e < nv; e++) v.k[e] = keys[e];
    } else if (lane == 1) {
      nv = int(n - rest);
      for (int e = 0; e < nv; e++) v.k[e] = keys[rest + e];
    }
    f(v.k, nv);
  }
}

// Appends the keys k[e] whose bit e of `take` is set to dst at a position drawn from *counter
// (one atomic per warp); positions at or beyond `cap` are not written.  All lanes call it.
template <class U, int E>
__device__ __forceinline__ void warp_append(const U* k, uint32_t take, U* __restrict__ dst,
                                            unsigned long long* counter, int64_t cap) {
  const int lane = threadIdx.x & 31;
  const uint32_t c = __popc(take);
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  if (total == 0u) return;  // uniform over the warp
  unsigned long long base = 0;
  if (lane == 31) base = atomicAdd(counter, (unsigned long long)total);
  base = __shfl_sync(0xFFFFFFFFu, base, 31);
  unsigned long long pos = base + incl - c;
#pragma unroll
  for (int e = 0; e < E; e++) {
    if ((take >> e) & 1u) {
      if (int64_t(pos) < cap) dst[pos] = k[e];
      pos++;
    }
  }
}

}  // namespace hpcs
