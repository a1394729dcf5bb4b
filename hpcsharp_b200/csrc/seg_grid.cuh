// Grid-level path of the batched segmented sort: the longest arrays of a batch are spread over
// many CTAs each.
//
// An array of at least SEG_GRID_MIN_KEYS keys (16-byte aligned) is cut into key ranges of at most
// SEG_GRID_TILES_PER_RANGE tiles of the plain sort's chunked pass, and every range becomes one
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

constexpr int64_t SEG_GRID_MIN_KEYS = int64_t(1) << 18;
constexpr int SEG_GRID_TILES_PER_RANGE = 8;

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

inline bool seg_grid_eligible(const hpcs_segment& sg) {
  return sg.n >= SEG_GRID_MIN_KEYS && (reinterpret_cast<uintptr_t>(sg.keys) & 15) == 0;
}

// Builds the grid-level sets of the arrays `idx` (all eligible) for ranking mode `mode`.
int seg_grid_build(const hpcs_segment* segs, const std::vector<int64_t>& idx, int mode, int skip_trivial,
                   uint64_t spin_limit_ns, SegGrid& grid);
// Turns the scratch offsets into device pointers.
void seg_grid_relocate(SegGrid& grid, void* base);
// Sets the kernels' shared-memory attributes (outside any stream capture).
int seg_grid_setup(hpcs_ctx* ctx, const SegGrid& grid);
// Enqueues every set on stream s: plan reset, histogram, digit passes, copy back.
int seg_grid_launch(hpcs_ctx* ctx, const SegGrid& grid, const SortArgs* d_args, const int2* d_map, cudaStream_t s);

}  // namespace hpcs
