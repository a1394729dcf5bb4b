// Host-side launch of the batched segmented sort (segmented.cuh), shared by the C ABI and
// the serving runtime's coalesced batches.
//
// Arrays are classed by length; a tuning table names, per key width and class, one kernel
// variant (a warp-level or a block-level kernel with a given tile shape and digit width).
// Arrays of one variant are sorted by one persistent launch; the launches of different
// variants are forked onto helper streams so they run concurrently.
#pragma once
#include <algorithm>
#include <vector>

#include "segmented.cuh"
#include "sort_host.cuh"

namespace hpcs {

// Upper length limits of the length classes (the last is unbounded).
constexpr int64_t SEG_CLASS_LIMIT[HPCS_SEG_CLASSES] = {128, 256, 512, 2048, 4096, 8192, 65536, -1};

inline int seg_class_of(int64_t n) {
  for (int c = 0; c < HPCS_SEG_CLASSES - 1; c++)
    if (n <= SEG_CLASS_LIMIT[c]) return c;
  return HPCS_SEG_CLASSES - 1;
}

struct SegVariant {
  int kind;  // 0 warp level, 1 block level
  int nt;
  int kpt;   // 4-byte keys per thread
  int rbits;
};
constexpr SegVariant SEG_VARIANTS[] = {
    {0, 256, 4, 8}, {0, 256, 8, 8}, {0, 256, 16, 8}, {0, 256, 8, 4}, {0, 256, 16, 4},
    {1, 256, 8, 8}, {1, 256, 16, 8}, {1, 512, 8, 8}, {1, 512, 16, 8}, {1, 512, 32, 8}, {0, 256, 32, 8},
};
constexpr int SEG_NVARIANTS = int(sizeof(SEG_VARIANTS) / sizeof(SEG_VARIANTS[0]));

// Longest array a variant sorts for a key width (-1: any, block level with scratch beyond a tile).
inline int64_t seg_variant_max_keys(int v, int key_bytes) {
  const SegVariant& sv = SEG_VARIANTS[v];
  if (sv.kind == 1) return -1;
  return int64_t(32) * sv.kpt * 4 / key_bytes;
}
// Keys per tile of a block-level variant for a key width (arrays above it need scratch).
inline int64_t seg_variant_tile_keys(int v, int key_bytes) {
  const SegVariant& sv = SEG_VARIANTS[v];
  return int64_t(sv.nt) * sv.kpt * 4 / key_bytes;
}

inline bool seg_variant_fits(int v, int w_index, int c) {
  if (v < 0 || v >= SEG_NVARIANTS) return false;
  const int64_t cap = seg_variant_max_keys(v, w_index ? 8 : 4);
  if (cap < 0) return true;
  return SEG_CLASS_LIMIT[c] >= 0 && SEG_CLASS_LIMIT[c] <= cap;
}

// The built-in table (variant per [4-byte, 8-byte keys][length class]): the autotuner's
// choice on a B200 (148 SMs), recorded with its measurements in tune/b200_148sm.json.
inline hpcs_seg_tuning seg_default_tuning() {
  hpcs_seg_tuning t{};
  const int v4[HPCS_SEG_CLASSES] = {0, 1, 2, 5, 6, 8, 6, 8};
  const int v8[HPCS_SEG_CLASSES] = {1, 2, 10, 6, 8, 9, 9, 9};
  for (int c = 0; c < HPCS_SEG_CLASSES; c++) {
    t.variant[0][c] = v4[c];
    t.variant[1][c] = v8[c];
  }
  return t;
}

template <class Kernel>
inline int seg_setup_kernel(Kernel k, int nt, size_t smem, int& blocks) {
  if (blocks) return HPCS_OK;
  HPCS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  HPCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, nt, smem));
  if (blocks < 1) blocks = 1;
  return HPCS_OK;
}

// One persistent launch of variant v over `nsegs` descriptors (its queue already zeroed);
// `large` selects the block level's tiled path (arrays longer than the variant's tile).
template <int MODE>
inline int launch_seg_variant(hpcs_ctx* ctx, int v, bool large, const SegDesc* d_desc, int nsegs,
                              uint32_t* d_queue, cudaStream_t s) {
  static int blocks_by_dev[64][SEG_NVARIANTS][2] = {};
  int& blocks = blocks_by_dev[ctx->device & 63][v][large ? 1 : 0];
  SegParams prm{d_desc, nsegs, d_queue, device_error_word(ctx), uint64_t(ctx->cfg.spin_limit_ns)};
  auto go = [&](auto k, int nt, size_t smem, int per_block) -> int {
    int rc = seg_setup_kernel(k, nt, smem, blocks);
    if (rc != HPCS_OK) return rc;
    const int64_t want = (int64_t(nsegs) + per_block - 1) / per_block;
    const int64_t cap = int64_t(ctx->sms) * blocks;
    const int grid = int(want < cap ? want : cap);
    if (grid > 0) {
      k<<<grid, nt, smem, s>>>(prm);
      HPCS_CUDA(cudaGetLastError());
    }
    return HPCS_OK;
  };
#define HPCS_SEG_BLOCK(NTV, KPTV)                                                                          \
  (large ? go(segmented_sort_kernel<NTV, KPTV, MODE, true>, NTV, SegSmem<NTV, KPTV, MODE>::BYTES, 1)      \
         : go(segmented_sort_kernel<NTV, KPTV, MODE, false>, NTV, SegSmem<NTV, KPTV, MODE>::BYTES, 1))
  switch (v) {
    case 0: return go(seg_warp_kernel<4, 8, MODE>, 256, WarpSegSmem<4, MODE>::BYTES, 8);
    case 1: return go(seg_warp_kernel<8, 8, MODE>, 256, WarpSegSmem<8, MODE>::BYTES, 8);
    case 2: return go(seg_warp_kernel<16, 8, MODE>, 256, WarpSegSmem<16, MODE>::BYTES, 8);
    case 3: return go(seg_warp_kernel<8, 4, MODE>, 256, WarpSegSmem<8, MODE>::BYTES, 8);
    case 4: return go(seg_warp_kernel<16, 4, MODE>, 256, WarpSegSmem<16, MODE>::BYTES, 8);
    case 5: return HPCS_SEG_BLOCK(256, 8);
    case 6: return HPCS_SEG_BLOCK(256, 16);
    case 7: return HPCS_SEG_BLOCK(512, 8);
    case 8: return HPCS_SEG_BLOCK(512, 16);
    case 9: return HPCS_SEG_BLOCK(512, 32);
    case 10: return go(seg_warp_kernel<32, 8, MODE>, 256, WarpSegSmem<32, MODE>::BYTES, 8);
    default: return fail(HPCS_ERR_RANGE, "unknown segmented-sort variant");
  }
#undef HPCS_SEG_BLOCK
}

// A descriptor table grouped by (variant, path): group g covers [first, first + count) and
// uses queue g; `large` marks block-level arrays longer than the variant's tile.
struct SegGroup {
  int variant;
  bool large;
  int first;
  int count;
};

// Whether variant v sorts an array of n keys of width w with its tiled (scratch) path.
inline bool seg_variant_large(int v, int64_t n, int key_bytes) {
  return SEG_VARIANTS[v].kind == 1 && n > seg_variant_tile_keys(v, key_bytes);
}

// Orders the descriptors by (variant, bytes descending), fills `groups`, and returns through
// `scratch` the bytes of scratch the block-level arrays longer than one tile need (their
// scratch fields hold offsets until seg_relocate).
int seg_build_groups(const hpcs_seg_tuning& tuning, const hpcs_segment* segs, int64_t nsegs,
                     std::vector<SegDesc>& table, std::vector<SegGroup>& groups, size_t& scratch);
void seg_relocate(std::vector<SegDesc>& table, const std::vector<SegGroup>& groups, void* base);

// Launches every group: the first on `s`, the others forked onto the context's helper
// streams and joined back into `s`.  Zeroes the groups' queues first.
int seg_launch_groups(hpcs_ctx* ctx, const SegDesc* d_desc, const std::vector<SegGroup>& groups,
                      uint32_t* d_queues, cudaStream_t s);

}  // namespace hpcs
