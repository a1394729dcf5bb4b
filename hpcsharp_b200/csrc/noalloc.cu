// hpcs_sort_u32_dev_noalloc: the uint32 device sort for callers that cannot allocate GPU
// memory -- code whose host framework owns every device allocation (a fixed-size arena or a
// caching allocator with a hard cap), or code on a path where cudaMalloc/cudaFree are not
// allowed (their implicit device synchronisation, or allocation failure, cannot be tolerated).
//
// Every byte of scratch the sort needs (the ping-pong key buffer, the two look-back status
// arrays, the per-sort plan and the device error word) lives in one file-scope __device__
// array of fixed size.  The module that holds it is loaded on every GPU that uses this
// library, so each such GPU keeps that array (about 4.3 MB) until the process exits.  The
// entry point itself calls no cudaMalloc, cudaFree or other allocating routine.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/hpcs_gpu.h"
#include "radix_kernels.cuh"
#include "sort_host.cuh"

namespace hpcs {
namespace {

// Ranking without the lane-order probe (which would need its own device memory): the fully
// defined peer-mask ranking, 512 threads x 16 keys per tile, one CTA per SM.
constexpr int NA_NT = 512, NA_KPT = 16, NA_TILE = NA_NT * NA_KPT;
using NaSmem = OnesweepSmem<uint32_t, NoValue, NA_NT, NA_KPT, 2, RANK_PEER_MASK>;
constexpr int64_t NA_UNITS = HPCS_NOALLOC_MAX_KEYS / NA_TILE;  // look-back units at the maximum

constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t NA_OFF_KEYS = 0;
constexpr size_t NA_OFF_STATUS0 = align256(NA_OFF_KEYS + size_t(HPCS_NOALLOC_MAX_KEYS) * 4);
constexpr size_t NA_OFF_STATUS1 = align256(NA_OFF_STATUS0 + size_t(NA_UNITS) * RADIX * 4);
constexpr size_t NA_OFF_PLAN = align256(NA_OFF_STATUS1 + size_t(NA_UNITS) * RADIX * 4);
constexpr size_t NA_OFF_ERR = align256(NA_OFF_PLAN + sizeof(SortPlan));
constexpr size_t NA_BYTES = align256(NA_OFF_ERR + 4);
static_assert(HPCS_NOALLOC_MAX_KEYS % NA_TILE == 0, "maximum must be whole tiles");

// The scratch.  In host code this name only stands for the symbol; its device address comes
// from cudaGetSymbolAddress (per device), never from taking the address here.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

struct NaDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int sms = 0;
  int onesweep_blocks = 1;
};
std::mutex g_na_mu;
NaDevice g_na[64];

#define NA_HIST_KERNEL hist_all_digits_kernel<uint32_t, KIND_UNSIGNED, HIST_NT>
#define NA_ONESWEEP_KERNEL \
  onesweep_pass_kernel<uint32_t, KIND_UNSIGNED, NoValue, NA_NT, NA_KPT, 2, 1, RANK_PEER_MASK, 1>

// Once per device, with that device current.  Resolves the scratch's device address and
// sizes the launches; clears the error word.  No allocation.
int na_setup(int dev, NaDevice** out) {
  std::lock_guard<std::mutex> lock(g_na_mu);
  NaDevice& d = g_na[dev & 63];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    d.scratch = static_cast<unsigned char*>(p);
    HPCS_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
    HPCS_CUDA(cudaFuncSetAttribute(NA_HIST_KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(HistSmem<uint32_t>::BYTES)));
    HPCS_CUDA(cudaFuncSetAttribute(NA_ONESWEEP_KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(NaSmem::BYTES)));
    HPCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.onesweep_blocks, NA_ONESWEEP_KERNEL, NA_NT,
                                                            NaSmem::BYTES));
    if (d.onesweep_blocks < 1) d.onesweep_blocks = 1;
    HPCS_CUDA(cudaMemset(d.scratch + NA_OFF_ERR, 0, 4));
    HPCS_CUDA(cudaDeviceSynchronize());
    d.ready = true;
  }
  *out = &d;
  return HPCS_OK;
}

}  // namespace
}  // namespace hpcs

using namespace hpcs;

extern "C" int hpcs_sort_u32_dev_noalloc(uint32_t* keys, int64_t n, void* stream) {
  if (!keys) return fail(HPCS_ERR_NULL, "keys is NULL");
  if (n < 0) return fail(HPCS_ERR_RANGE, "length is negative");
  if (n > HPCS_NOALLOC_MAX_KEYS) {
    char buf[128];
    std::snprintf(buf, sizeof buf, "n = %lld exceeds HPCS_NOALLOC_MAX_KEYS (%lld) of the no-allocation sort",
                  (long long)n, (long long)HPCS_NOALLOC_MAX_KEYS);
    return fail(HPCS_ERR_RANGE, buf);
  }
  if ((reinterpret_cast<uintptr_t>(keys) & 15) != 0)
    return fail(HPCS_ERR_UNSUPPORTED, "keys must be 16-byte aligned for the no-allocation sort");
  if (n <= 1) return HPCS_OK;
  int dev = 0;
  HPCS_CUDA(cudaGetDevice(&dev));
  NaDevice* d = nullptr;
  int rc = na_setup(dev, &d);
  if (rc != HPCS_OK) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the call waits for its stream and reads the error word back: it cannot be captured
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  HPCS_CUDA(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(HPCS_ERR_UNSUPPORTED, "the no-allocation sort cannot be called while its stream is being captured");
  const int64_t units = (n + NA_TILE - 1) / NA_TILE;

  SortArgs args{};
  args.keys_a = keys;
  args.keys_b = d->scratch + NA_OFF_KEYS;
  args.vals_a = nullptr;
  args.vals_b = nullptr;
  args.n = n;
  args.plan = reinterpret_cast<SortPlan*>(d->scratch + NA_OFF_PLAN);
  args.status[0] = reinterpret_cast<uint32_t*>(d->scratch + NA_OFF_STATUS0);
  args.status[1] = reinterpret_cast<uint32_t*>(d->scratch + NA_OFF_STATUS1);
  args.num_tiles = int(units);
  args.skip_trivial = 1;
  args.poison_tile = -1;
  args.spin_limit_ns = 2000000000ull;
  args.trace = nullptr;
  uint32_t* err = reinterpret_cast<uint32_t*>(d->scratch + NA_OFF_ERR);

  // The plan (counts, starts, tile counters, error bits) must start at zero on every call;
  // K1 clears the first look-back buffer and each pass clears the other ahead of use.
  HPCS_CUDA(cudaMemsetAsync(args.plan, 0, sizeof(SortPlan), s));
  {
    const int64_t want = (n / 4 + HIST_NT * 4 - 1) / (HIST_NT * 4);
    const int grid = int(want < 1 ? 1 : (want > d->sms ? d->sms : want));
    NA_HIST_KERNEL<<<grid, HIST_NT, HistSmem<uint32_t>::BYTES, s>>>(keys, n, &args.plan->hist[0][0], args, 1);
    HPCS_CUDA(cudaGetLastError());
  }
  {
    const int64_t cap = int64_t(d->sms) * d->onesweep_blocks;
    const int grid = int(units < cap ? units : cap);
    for (int p = 0; p < 4; p++) {
      args.pass = p;
      NA_ONESWEEP_KERNEL<<<grid, NA_NT, NaSmem::BYTES, s>>>(args);
      HPCS_CUDA(cudaGetLastError());
    }
  }
  {
    const int64_t want = (n + 255) / 256;
    const int grid = int(want > int64_t(d->sms) * 8 ? int64_t(d->sms) * 8 : want);
    finalize_kernel<uint32_t><<<grid, 256, 0, s>>>(args, 0, err);
    HPCS_CUDA(cudaGetLastError());
  }
  // Synchronous: report a device-side wait that ran out, then clear it for the next call.
  HPCS_CUDA(cudaStreamSynchronize(s));
  uint32_t bits = 0;
  HPCS_CUDA(cudaMemcpy(&bits, err, 4, cudaMemcpyDeviceToHost));
  if (bits) {
    HPCS_CUDA(cudaMemset(err, 0, 4));
    return fail(HPCS_ERR_DEVICE_TIMEOUT, "device-side wait ran out in the no-allocation sort");
  }
  return HPCS_OK;
}
