// Host-side launch of the batched segmented sort kernel (segmented.cuh), shared by the C ABI
// and the serving runtime's coalesced batches.
#pragma once
#include "segmented.cuh"
#include "sort_host.cuh"

namespace hpcs {

constexpr int SEG_NT = 512, SEG_KPT = 16;  // 8192 u32 / 4096 u64 keys per tile

// Keys per tile of the segmented kernel for a key width: arrays up to this size are sorted
// entirely in shared memory and need no scratch.
inline int64_t seg_tile_keys(int key_bytes) { return int64_t(SEG_NT) * SEG_KPT * 4 / key_bytes; }

template <int MODE>
inline int launch_segmented(hpcs_ctx* ctx, const SegDesc* d_desc, int nsegs, uint32_t* d_queue, cudaStream_t s) {
  using L = SegSmem<SEG_NT, SEG_KPT, MODE>;
  auto k = segmented_sort_kernel<SEG_NT, SEG_KPT, MODE>;
  static int blocks_by_dev[64] = {0};
  int& blocks = blocks_by_dev[ctx->device & 63];
  if (!blocks) {
    HPCS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::BYTES)));
    HPCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, SEG_NT, L::BYTES));
    if (blocks < 1) blocks = 1;
  }
  HPCS_CUDA(cudaMemsetAsync(d_queue, 0, 4, s));
  SegParams prm{d_desc, nsegs, d_queue, device_error_word(ctx)};
  const int64_t cap = int64_t(ctx->sms) * blocks;
  const int grid = int(nsegs < cap ? nsegs : cap);
  if (grid > 0) {
    KernelTimer kt(ctx, s, HPCS_K_SEGMENTED);
    k<<<grid, SEG_NT, L::BYTES, s>>>(prm);
    HPCS_CUDA(cudaGetLastError());
  }
  return HPCS_OK;
}

inline int enqueue_segmented(hpcs_ctx* ctx, const SegDesc* d_desc, int nsegs, uint32_t* d_queue, cudaStream_t s) {
  return ctx->rank_mode == RANK_ORDERED_ATOMIC ? launch_segmented<RANK_ORDERED_ATOMIC>(ctx, d_desc, nsegs, d_queue, s)
                                               : launch_segmented<RANK_PEER_MASK>(ctx, d_desc, nsegs, d_queue, s);
}

}  // namespace hpcs
