// Grid-level path of the batched segmented sort: the longest arrays of a batch are spread over
// many CTAs each.
//
// An array of at least SEG_GRID_MIN_KEYS keys (16-byte aligned; both numbers are context settings)
// is cut into key ranges of at most SEG_GRID_TILES_PER_RANGE tiles of the plain sort's chunked
// pass, and every range becomes one
// CTA of the plain sort's own kernels: the fused histogram (which also builds the array's plan in
// its last CTA), one chunked digit pass per digit, and a copy back when an odd number of passes
// ran.  The arrays of one key type share each launch: CTA c reads (array, range) from a map and the
// array's sort arguments from a table, so a pass of thousands of arrays is one launch instead of a
// launch per array, and every array still gets exactly the plain sort's result (the same kernels
// on the same per-array ranges).  Each array has its own scratch: a ping-pong buffer, its
// per-range digit counts and next-digit tables, and its plan.
#pragma once
#include <vector>

#include "radix_kernels.cuh"
#include "sort_host.cuh"

namespace hpcs {

// Defaults, from a sweep on B200 over 65,536 arrays of log-uniform length on [32, 2^20] (4- and
// 8-byte keys): thresholds 8 Ki-256 Ki and 8-64 tiles per CTA were within 2% of each other
// from 32 Ki to 128 Ki keys and 32 tiles, and one CTA per array (no grid level) was 14% slower.
constexpr int64_t SEG_GRID_MIN_KEYS = int64_t(1) << 16;
constexpr int SEG_GRID_TILES_PER_RANGE = 32;

// The grid-level arrays of one key type: args[first, first + count) and map[map_first,
// map_first + ctas) (map entries index args relative to `first`).
struct SegGridSet {
  int dtype = 0;
  int first = 0, count = 0;
  int map_first = 0, ctas = 0;
  int max_ranges = 0;
  size_t plan_off = 0;  // the set's plans are contiguous in the scratch (zeroed before each sort)
  size_t plan_bytes = 0;
};

struct SegGrid {
  std::vector<SortArgs> args;  // device pointers are scratch offsets until seg_grid_relocate
  std::vector<int2> map;
  std::vector<SegGridSet> sets;
  size_t scratch = 0;  // bytes of scratch the arrays need
  int mode = RANK_ORDERED_ATOMIC;
};

// The context's length threshold (hpcs_config.seg_grid_min_keys; <0: none) and tiles per CTA.
inline int64_t seg_grid_min_keys(const hpcs_config& cfg) {
  return cfg.seg_grid_min_keys < 0 ? INT64_MAX : cfg.seg_grid_min_keys == 0 ? SEG_GRID_MIN_KEYS : cfg.seg_grid_min_keys;
}
inline int seg_grid_tiles(const hpcs_config& cfg) {
  return cfg.seg_grid_tiles > 0 ? cfg.seg_grid_tiles : SEG_GRID_TILES_PER_RANGE;
}

inline bool seg_grid_eligible(const hpcs_segment& sg, int64_t min_keys) {
  return sg.n >= min_keys && (reinterpret_cast<uintptr_t>(sg.keys) & 15) == 0;
}

// Builds the grid-level sets of the arrays `idx` (all eligible) for ranking mode `mode`, with
// ranges of at most `tiles_per_range` tiles.
int seg_grid_build(const hpcs_segment* segs, const std::vector<int64_t>& idx, int mode, int skip_trivial,
                   uint64_t spin_limit_ns, int tiles_per_range, SegGrid& grid);
// Turns the scratch offsets into device pointers.
void seg_grid_relocate(SegGrid& grid, void* base);
// Sets the kernels' shared-memory attributes (outside any stream capture).
int seg_grid_setup(hpcs_ctx* ctx, const SegGrid& grid);
// Enqueues every set on stream s: plan reset, histogram, digit passes, copy back.
int seg_grid_launch(hpcs_ctx* ctx, const SegGrid& grid, const SortArgs* d_args, const int2* d_map, cudaStream_t s);

}  // namespace hpcs
