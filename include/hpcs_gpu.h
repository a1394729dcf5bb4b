/*
 * hpcs_gpu.h - C ABI of the B200 (sm_100a) LSD radix-sort library (libhpcs_gpu.so).
 *
 * This is the drop-in boundary for HPCsharp's radix-sort hot path.  A .NET caller binds
 * these functions with P/Invoke behind the same extension methods the reference exposes;
 * every entry point below names the reference method it replaces (paths relative to the
 * HPCsharp project root).
 *
 * Conventions
 *   - Every function returns an hpcs_status; nothing aborts, exits or traps.  The text of
 *     the last error on the calling thread is returned by hpcs_last_error_message().
 *   - NULL array          -> HPCS_ERR_NULL  (reference: ArgumentNullException,
 *                                            e.g. RadixSortLsd.cs:215-216)
 *   - bad length / k / l,r -> HPCS_ERR_RANGE (reference: ArgumentOutOfRangeException,
 *                                            SelectionTopKRadix.cs:146-149, :164-167)
 *   - n == 0 returns HPCS_OK at once (RadixSortLsdParallel.cs:175-176).
 *   - One sort, pairs sort or histogram call takes at most HPCS_MAX_KEYS keys; a segmented
 *     array, a served request or a select / top-k call at most HPCS_MAX_SEGMENT_KEYS.
 *   - Host-array functions (no suffix) are synchronous: they copy the caller's array to
 *     the GPU, sort, copy back into the same array and return.  The result is the
 *     reference's in-place result (the caller's array sorted, RadixSortLsdParallel.cs:227-231).
 *   - *_dev functions take device pointers and a cudaStream_t (passed as void*, NULL = the
 *     context's own stream, which does not synchronise with the legacy default stream; pass
 *     cudaStreamLegacy, (void*)1, to run on that one); they are asynchronous on that stream.
 *     Device-side failures (bounded waits that ran out) are reported by the next
 *     hpcs_ctx_synchronize().
 *   - A context is used by one host thread at a time.  Its scratch memory is reused
 *     across calls in stream order.
 *   - Sorting is stable and ascending.  Signed keys order by value; float keys order by
 *     the reference's bit transform (Histogram.cs:1210-1288): -NaN < -inf < ... < -0.0 <
 *     +0.0 < ... < +inf < +NaN.
 */
#ifndef HPCS_GPU_H
#define HPCS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPCS_ABI_VERSION 1
#define HPCS_MAX_KEYS ((int64_t)2147483647) /* 2^31 - 1 keys per sort, pairs sort or histogram
                                                call: the longest .NET array */
#define HPCS_MAX_SEGMENT_KEYS ((int64_t)1073741823) /* 2^30 - 1 keys per segmented array,
                                                       served request or select / top-k call */

typedef enum hpcs_status {
  HPCS_OK = 0,
  HPCS_ERR_NULL = 1,           /* ArgumentNullException */
  HPCS_ERR_RANGE = 2,          /* ArgumentOutOfRangeException */
  HPCS_ERR_OOM = 3,            /* device memory or the context's pool budget exhausted */
  HPCS_ERR_CUDA = 4,           /* a CUDA runtime call failed */
  HPCS_ERR_DEVICE_TIMEOUT = 5, /* a bounded device-side wait ran out */
  HPCS_ERR_UNSUPPORTED = 6,    /* dtype / option not supported */
  HPCS_ERR_NO_DEVICE = 7,      /* no CUDA device */
  HPCS_ERR_BUSY = 8            /* serving: admission refused */
} hpcs_status;

typedef enum hpcs_dtype {
  HPCS_U32 = 0,
  HPCS_I32 = 1,
  HPCS_F32 = 2,
  HPCS_U64 = 3,
  HPCS_I64 = 4,
  HPCS_F64 = 5
} hpcs_dtype;

typedef struct hpcs_ctx hpcs_ctx;

/* Digit-pass schemes (hpcs_config.pass_scheme). */
enum { HPCS_PASSES_AUTO = 0, HPCS_PASSES_LOOKBACK = 1, HPCS_PASSES_CHUNKED = 2 };

typedef struct hpcs_config {
  int64_t pool_bytes;          /* device scratch budget of the context; 0 = unlimited */
  int32_t skip_trivial_passes; /* 1: skip a digit pass whose keys all share that digit */
  int32_t rank_mode;           /* 0: one shared atomic per key, after this GPU passed the
                                  lane-order probe at context creation (else as 1);
                                  1: always the fully defined peer-mask ranking */
  int64_t spin_limit_ns;       /* bound on every device-side wait (default 2e9) */
  int32_t poison_tile;         /* test hook: tile whose device wait times out (-1 = off) */
  int32_t pass_scheme;         /* digit passes: HPCS_PASSES_AUTO (0, default) picks by key
                                  type and n (up to 131072 keys: every pass in one cooperative
                                  launch, outside stream capture); HPCS_PASSES_LOOKBACK (1):
                                  single-pass decoupled look-back; HPCS_PASSES_CHUNKED (2):
                                  per-range counts from the previous pass, no inter-CTA
                                  waiting */
  int32_t staged_host_copies;  /* host-array calls on pageable memory (default 1): copy through
                                  the context's pinned buffers in chunks, several host threads
                                  copying while the DMA engine moves earlier chunks; 0: one
                                  cudaMemcpyAsync per array (the driver stages it) */
  int32_t seg_grid_min_keys;   /* batched sort: arrays of at least this many keys (16-byte
                                  aligned) take the plain sort's kernels, spread over
                                  several CTAs each; 0 = 65536, negative = never */
  int32_t seg_grid_tiles;      /* batched sort: 16 Ki-key tiles per CTA of such an array
                                  (0 = 32) */
  int32_t reserved[3];
} hpcs_config;

/* ---- context ---------------------------------------------------------------------- */
void hpcs_config_default(hpcs_config* cfg);
int hpcs_ctx_create(int device, const hpcs_config* cfg, hpcs_ctx** out);
int hpcs_ctx_destroy(hpcs_ctx* ctx);
/* Wait for all work of the context; reports device-side timeouts of earlier *_dev calls. */
int hpcs_ctx_synchronize(hpcs_ctx* ctx);
/* The context's own stream (a cudaStream_t). */
void* hpcs_ctx_stream(hpcs_ctx* ctx);
/* Ranking used by this context: 0 = ordered shared atomics (probe passed), 1 = peer mask. */
int hpcs_ctx_rank_mode(hpcs_ctx* ctx);
const char* hpcs_last_error_message(void);
const char* hpcs_status_string(int status);
int hpcs_abi_version(void);

/* ---- per-kernel timing (tracing) ----------------------------------------------------
 * When enabled, the context records a CUDA event pair around every kernel it launches
 * (on the launching stream).  hpcs_ctx_profile_read waits for the context, sums the
 * durations per kernel class and clears the record.  No reference counterpart (the
 * reference has commented-out Stopwatch blocks in its hot loops, RadixSortLsd.cs:146-153). */
typedef enum hpcs_kernel_class {
  HPCS_K_HISTOGRAM = 0, /* fused all-digit histogram (+ plan) */
  HPCS_K_ONESWEEP = 1,  /* one 8-bit digit pass, chunked scheme */
  HPCS_K_FINALIZE = 2,  /* copy-back / error fold */
  HPCS_K_TOPK = 3,      /* radix select kernels */
  HPCS_K_SEGMENTED = 4, /* batched segmented sort kernels */
  HPCS_K_SHARD = 5,     /* sharded sort: partition of a shard (count, scan, scatter) */
  HPCS_K_LOOKBACK = 6,  /* one 8-bit digit pass, decoupled look-back scheme (a launch whose
                           scheme the histogram kernel did not choose returns at once) */
  HPCS_K_CLASSES = 8
} hpcs_kernel_class;

typedef struct hpcs_profile {
  int64_t launches[HPCS_K_CLASSES];
  double total_ms[HPCS_K_CLASSES];
} hpcs_profile;

int hpcs_ctx_profile_enable(hpcs_ctx* ctx, int enable);
/* Tile trace (debug): while set, each onesweep launch of digit pass `pass` writes 7 words
 * per tile t < capacity_tiles at trace[7*t]: tile id, SM id, and %globaltimer (ns) at
 * start, data ready, ranked, look-back done (digit 0), end of scatter.  trace is device
 * memory; NULL turns tracing off. */
int hpcs_ctx_trace_tiles(hpcs_ctx* ctx, uint64_t* trace, int capacity_tiles, int pass);
int hpcs_ctx_profile_read(hpcs_ctx* ctx, hpcs_profile* out);

/* ---- plain sort, host arrays, in place ----------------------------------------------
 * u32: ParallelAlgorithm.SortRadixPar(this uint[], int ParallelWorkQuantum)
 *        RadixSortLsdParallel.cs:145-232; Algorithm.SortRadixLsd(this uint[])
 *        RadixSortLsd.cs:255-260 (and SortRadixLsdFunc :238-243).  The work quantum is a
 *        CPU tuning knob with no meaning on the GPU.
 * i32: SortRadixPar(this int[]) RadixSortLsdParallel.cs:446-495; SortRadixLsd(this int[])
 *        RadixSortLsd.cs:352-357.
 * u64: SortRadixPar(this ulong[]) RadixSortLsdParallel.cs:690-734; SortRadixLsd(this
 *        ulong[]) RadixSortLsd.cs:437-442.
 * i64: SortRadixPar(this long[]) RadixSortLsdParallel.cs:560-609; SortRadixLsd(this
 *        long[]) RadixSortLsd.cs:527-532.
 * f32/f64: no LSD counterpart in the reference (its float radix sort is the unstable MSD
 *        SortRadixMsd(this float[]/double[]) RadixSortMsd.cs:1563-1610); the order is the
 *        reference's float transform, Histogram.cs:1210-1288. */
int hpcs_sort_u32(hpcs_ctx* ctx, uint32_t* keys, int64_t n);
int hpcs_sort_i32(hpcs_ctx* ctx, int32_t* keys, int64_t n);
int hpcs_sort_f32(hpcs_ctx* ctx, float* keys, int64_t n);
int hpcs_sort_u64(hpcs_ctx* ctx, uint64_t* keys, int64_t n);
int hpcs_sort_i64(hpcs_ctx* ctx, int64_t* keys, int64_t n);
int hpcs_sort_f64(hpcs_ctx* ctx, double* keys, int64_t n);

/* ---- plain sort, device pointers, asynchronous on `stream` -------------------------- */
int hpcs_sort_u32_dev(hpcs_ctx* ctx, uint32_t* keys, int64_t n, void* stream);
int hpcs_sort_i32_dev(hpcs_ctx* ctx, int32_t* keys, int64_t n, void* stream);
int hpcs_sort_f32_dev(hpcs_ctx* ctx, float* keys, int64_t n, void* stream);
int hpcs_sort_u64_dev(hpcs_ctx* ctx, uint64_t* keys, int64_t n, void* stream);
int hpcs_sort_i64_dev(hpcs_ctx* ctx, int64_t* keys, int64_t n, void* stream);
int hpcs_sort_f64_dev(hpcs_ctx* ctx, double* keys, int64_t n, void* stream);

/* ---- stable key + item pairs --------------------------------------------------------
 * Algorithm.SortRadix<T>(this T[] items, UInt32[] keys) RadixSortLsd.cs:1183-1237 and
 * SortRadix<T>(this T[] items, UInt64[] keys) :1245-1299, with T a 4-byte item (index).
 * Both arrays are permuted in place by the stable order of the keys.  (The reference's
 * returned Tuple.Item2 is its scratch buffer; the caller's key array is the sorted one.)
 * i32/f32/i64/f64 keys extend the same form with the signed / float transforms. */
int hpcs_sort_pairs_u32(hpcs_ctx* ctx, uint32_t* keys, uint32_t* items, int64_t n);
int hpcs_sort_pairs_i32(hpcs_ctx* ctx, int32_t* keys, uint32_t* items, int64_t n);
int hpcs_sort_pairs_f32(hpcs_ctx* ctx, float* keys, uint32_t* items, int64_t n);
int hpcs_sort_pairs_u64(hpcs_ctx* ctx, uint64_t* keys, uint32_t* items, int64_t n);
int hpcs_sort_pairs_i64(hpcs_ctx* ctx, int64_t* keys, uint32_t* items, int64_t n);
int hpcs_sort_pairs_f64(hpcs_ctx* ctx, double* keys, uint32_t* items, int64_t n);
int hpcs_sort_pairs_u32_dev(hpcs_ctx* ctx, uint32_t* keys, uint32_t* items, int64_t n, void* stream);
int hpcs_sort_pairs_i32_dev(hpcs_ctx* ctx, int32_t* keys, uint32_t* items, int64_t n, void* stream);
int hpcs_sort_pairs_f32_dev(hpcs_ctx* ctx, float* keys, uint32_t* items, int64_t n, void* stream);
int hpcs_sort_pairs_u64_dev(hpcs_ctx* ctx, uint64_t* keys, uint32_t* items, int64_t n, void* stream);
int hpcs_sort_pairs_i64_dev(hpcs_ctx* ctx, int64_t* keys, uint32_t* items, int64_t n, void* stream);
int hpcs_sort_pairs_f64_dev(hpcs_ctx* ctx, double* keys, uint32_t* items, int64_t n, void* stream);

/* ---- fused all-digit byte histogram -------------------------------------------------
 * ParallelAlgorithm.HistogramByteComponentsPar(uint[]/int[]/ulong[]/long[], int l, int r)
 * HistogramParallel.cs:214-222 (u32), :416-424 (i32), :547-555 (u64), :617-625 (i64), and
 * the serial Algorithm.HistogramByteComponents Histogram.cs:261-296, :957-1052.
 * Counts keys a[l..r] (inclusive, as the reference) into counts[P][256], P = key bytes,
 * digit d = byte d; signed keys flip the top byte (Histogram.cs:1014, :1049), float keys
 * use the float transform.  l > r yields all-zero counts. */
int hpcs_histogram_byte_components_u32(hpcs_ctx* ctx, const uint32_t* a, int64_t l, int64_t r, uint32_t* counts);
int hpcs_histogram_byte_components_i32(hpcs_ctx* ctx, const int32_t* a, int64_t l, int64_t r, uint32_t* counts);
int hpcs_histogram_byte_components_f32(hpcs_ctx* ctx, const float* a, int64_t l, int64_t r, uint32_t* counts);
int hpcs_histogram_byte_components_u64(hpcs_ctx* ctx, const uint64_t* a, int64_t l, int64_t r, uint32_t* counts);
int hpcs_histogram_byte_components_i64(hpcs_ctx* ctx, const int64_t* a, int64_t l, int64_t r, uint32_t* counts);
int hpcs_histogram_byte_components_f64(hpcs_ctx* ctx, const double* a, int64_t l, int64_t r, uint32_t* counts);
/* Device form: a is a device pointer to the n keys, counts a device buffer of P*256. */
int hpcs_histogram_byte_components_dev(hpcs_ctx* ctx, int dtype, const void* a, int64_t n, uint32_t* counts,
                                       void* stream);

/* ---- counting sort of 8- and 16-bit keys ----------------------------------------------
 * SortCountingInPlace(this byte[] / sbyte[] / ushort[] / short[]) CountingSort.cs:41, :78,
 * :115, :152 and SortCountingInPlacePar CountingSortParallel.cs:41: in place, ascending
 * (signed keys by value).  One histogram read, a scan of the 2^8 / 2^16 counts, one fill. */
int hpcs_sort_u8(hpcs_ctx* ctx, uint8_t* keys, int64_t n);
int hpcs_sort_i8(hpcs_ctx* ctx, int8_t* keys, int64_t n);
int hpcs_sort_u16(hpcs_ctx* ctx, uint16_t* keys, int64_t n);
int hpcs_sort_i16(hpcs_ctx* ctx, int16_t* keys, int64_t n);
int hpcs_sort_u8_dev(hpcs_ctx* ctx, uint8_t* keys, int64_t n, void* stream);
int hpcs_sort_i8_dev(hpcs_ctx* ctx, int8_t* keys, int64_t n, void* stream);
int hpcs_sort_u16_dev(hpcs_ctx* ctx, uint16_t* keys, int64_t n, void* stream);
int hpcs_sort_i16_dev(hpcs_ctx* ctx, int16_t* keys, int64_t n, void* stream);

/* ---- batched segmented sort ------------------------------------------------------------
 * No reference counterpart (HPCsharp sorts one array per call): many independent arrays of
 * mixed length and dtype sorted in one persistent launch, each with exactly the plain sort's
 * result (stable, ascending, same order transforms).  Keys are device pointers, sorted in
 * place; each array's n <= HPCS_MAX_SEGMENT_KEYS. */
typedef struct hpcs_segment {
  void* keys;      /* device pointer */
  int64_t n;
  int32_t dtype;   /* hpcs_dtype */
  int32_t reserved;
} hpcs_segment;

/* One-shot: uploads the descriptors and sorts on `stream`. */
int hpcs_sort_segmented_dev(hpcs_ctx* ctx, const hpcs_segment* segs, int64_t nsegs, void* stream);

/* Reusable plan: descriptors stay on the device (largest array first), scratch is reserved,
 * and the launch is captured in a CUDA graph; hpcs_segplan_execute replays it (sorting
 * whatever the same arrays hold at that time). */
typedef struct hpcs_segplan hpcs_segplan;
int hpcs_segplan_create(hpcs_ctx* ctx, const hpcs_segment* segs, int64_t nsegs, hpcs_segplan** out);
int hpcs_segplan_execute(hpcs_segplan* plan, void* stream);
int hpcs_segplan_destroy(hpcs_segplan* plan);

/* Segmented-sort tuning.  Arrays are classed by length: class c holds the arrays longer than
 * the limit of class c-1 and at most hpcs_seg_class_limit(c) keys (the last class is
 * unbounded).  For each key width (index 0: 4-byte keys, 1: 8-byte keys) and class the table
 * names one kernel variant of hpcs_seg_variants(): a warp-level one (one warp sorts one array
 * in registers and shared memory) or a block-level one (one CTA per array, in shared memory
 * when the array fits one tile, else tile by tile with scratch).  A context starts with the
 * built-in table, chosen on a B200 by the project's autotuner (hpcsharp_b200/autotune.py);
 * hpcs_ctx_set_seg_tuning replaces it.  A plan uses the table in force when it is created.
 * Arrays of one variant go to one persistent launch; the launches of different variants run
 * concurrently on forked streams (inside the plan's graph, as graph branches). */
#define HPCS_SEG_CLASSES 8
typedef struct hpcs_seg_tuning {
  int32_t variant[2][HPCS_SEG_CLASSES];
} hpcs_seg_tuning;
typedef struct hpcs_seg_variant_info {
  int32_t kind;            /* 0: warp level, 1: block level */
  int32_t threads;         /* threads per CTA */
  int32_t keys_per_thread; /* 4-byte keys per thread (8-byte keys: half) */
  int32_t digit_bits;      /* bits per pass */
  int64_t max_keys[2];     /* longest array it sorts for 4- / 8-byte keys; -1 = any length */
} hpcs_seg_variant_info;
/* Fills up to `capacity` entries and returns the number of variants. */
int hpcs_seg_variants(hpcs_seg_variant_info* out, int capacity);
/* Upper length limit of class c (-1 for the last, unbounded class; -2 if c is out of range). */
int64_t hpcs_seg_class_limit(int c);
int hpcs_ctx_get_seg_tuning(hpcs_ctx* ctx, hpcs_seg_tuning* out);
/* HPCS_ERR_RANGE if a variant index is unknown or cannot hold the longest array of its class. */
int hpcs_ctx_set_seg_tuning(hpcs_ctx* ctx, const hpcs_seg_tuning* tuning);

/* ---- radix top-k ---------------------------------------------------------------------
 * Algorithm.SelectTopK(this uint[] a, int k) SelectionTopKRadix.cs:160-171 (and the
 * (a, start, length, k) form :142-153 via a pointer offset): afterwards a[k] is the k-th
 * smallest key (0-based) and a[k..n-1] holds exactly the multiset of the n-k largest.  Here
 * a[0..k-1] also holds the k smallest (the reference clobbers that prefix).  n <= 0 or k
 * outside [0, n) -> HPCS_ERR_RANGE (the reference accepts k == n but then reads past its
 * bins).  The reference has uint only; the other dtypes use the sort's order transforms. */
int hpcs_select_topk_u32(hpcs_ctx* ctx, uint32_t* a, int64_t n, int64_t k);
int hpcs_select_topk_i32(hpcs_ctx* ctx, int32_t* a, int64_t n, int64_t k);
int hpcs_select_topk_f32(hpcs_ctx* ctx, float* a, int64_t n, int64_t k);
int hpcs_select_topk_u64(hpcs_ctx* ctx, uint64_t* a, int64_t n, int64_t k);
int hpcs_select_topk_i64(hpcs_ctx* ctx, int64_t* a, int64_t n, int64_t k);
int hpcs_select_topk_f64(hpcs_ctx* ctx, double* a, int64_t n, int64_t k);
int hpcs_select_topk_u32_dev(hpcs_ctx* ctx, uint32_t* a, int64_t n, int64_t k, void* stream);
int hpcs_select_topk_i32_dev(hpcs_ctx* ctx, int32_t* a, int64_t n, int64_t k, void* stream);
int hpcs_select_topk_f32_dev(hpcs_ctx* ctx, float* a, int64_t n, int64_t k, void* stream);
int hpcs_select_topk_u64_dev(hpcs_ctx* ctx, uint64_t* a, int64_t n, int64_t k, void* stream);
int hpcs_select_topk_i64_dev(hpcs_ctx* ctx, int64_t* a, int64_t n, int64_t k, void* stream);
int hpcs_select_topk_f64_dev(hpcs_ctx* ctx, double* a, int64_t n, int64_t k, void* stream);
/* The k largest of in[0..n) written to out[0..k) in ascending order (the top-k of a serving
 * request; equals the reference's a[n-k..n-1] after SelectTopK(a, n-k), sorted).  k in
 * [0, n]. */
int hpcs_topk_largest_u32(hpcs_ctx* ctx, const uint32_t* in, int64_t n, int64_t k, uint32_t* out);
int hpcs_topk_largest_i32(hpcs_ctx* ctx, const int32_t* in, int64_t n, int64_t k, int32_t* out);
int hpcs_topk_largest_f32(hpcs_ctx* ctx, const float* in, int64_t n, int64_t k, float* out);
int hpcs_topk_largest_u64(hpcs_ctx* ctx, const uint64_t* in, int64_t n, int64_t k, uint64_t* out);
int hpcs_topk_largest_i64(hpcs_ctx* ctx, const int64_t* in, int64_t n, int64_t k, int64_t* out);
int hpcs_topk_largest_f64(hpcs_ctx* ctx, const double* in, int64_t n, int64_t k, double* out);
int hpcs_topk_largest_u32_dev(hpcs_ctx* ctx, const uint32_t* in, int64_t n, int64_t k, uint32_t* out, void* stream);
int hpcs_topk_largest_i32_dev(hpcs_ctx* ctx, const int32_t* in, int64_t n, int64_t k, int32_t* out, void* stream);
int hpcs_topk_largest_f32_dev(hpcs_ctx* ctx, const float* in, int64_t n, int64_t k, float* out, void* stream);
int hpcs_topk_largest_u64_dev(hpcs_ctx* ctx, const uint64_t* in, int64_t n, int64_t k, uint64_t* out, void* stream);
int hpcs_topk_largest_i64_dev(hpcs_ctx* ctx, const int64_t* in, int64_t n, int64_t k, int64_t* out, void* stream);
int hpcs_topk_largest_f64_dev(hpcs_ctx* ctx, const double* in, int64_t n, int64_t k, double* out, void* stream);

/* ---- radix partition and selection by index --------------------------------------------
 * Algorithm.PartitionRadix(this uint[] a, int start, int length, int k, int threshold)
 * PartitionRadix.cs:135-147, (a, k) :155-164, and the k[] forms (a, start, length, int[] k)
 * :173-190, (a, int[] k) :198-210 (the ulong versions share them): in place, afterwards every
 * a[k_i] holds the key the sorted subarray a[start, start + length) has at index k_i, and the
 * keys between two consecutive indices (or an index and an end of the subarray) lie between
 * their keys, as C++'s nth_element does.  k indexes the whole array; the indices may come in any
 * order and repeat.  The threshold of the reference's base case is a CPU tuning knob with no
 * meaning here.  The order of keys inside each part is unspecified (the reference's is not
 * stable either).  start < 0, length <= 0, nk < 0 or an index outside the subarray ->
 * HPCS_ERR_RANGE; nk == 0 does nothing.  Up to 4 distinct indices are placed by radix selects
 * and three-way partitions; more sort the subarray. */
int hpcs_partition_radix_u32(hpcs_ctx* ctx, uint32_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk);
int hpcs_partition_radix_i32(hpcs_ctx* ctx, int32_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk);
int hpcs_partition_radix_f32(hpcs_ctx* ctx, float* a, int64_t start, int64_t length, const int64_t* k, int64_t nk);
int hpcs_partition_radix_u64(hpcs_ctx* ctx, uint64_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk);
int hpcs_partition_radix_i64(hpcs_ctx* ctx, int64_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk);
int hpcs_partition_radix_f64(hpcs_ctx* ctx, double* a, int64_t start, int64_t length, const int64_t* k, int64_t nk);
/* ParallelAlgorithm.SelectRadixPar(this uint[] a, int start, int length, int k, int
 * parallelThreshold) SelectionRadixParallel.cs:254-266 and (a, k) :271-283, and the serial
 * Algorithm.SelectRadix(this uint[], start, length, k) SelectionRadix.cs:236-250: *out = the
 * k-th smallest key of a[start, start + length) (k absolute), which is also left at a[k]; the
 * subarray is partitioned around it as by hpcs_partition_radix_<t> with one index. */
int hpcs_select_radix_u32(hpcs_ctx* ctx, uint32_t* a, int64_t start, int64_t length, int64_t k, uint32_t* out);
int hpcs_select_radix_i32(hpcs_ctx* ctx, int32_t* a, int64_t start, int64_t length, int64_t k, int32_t* out);
int hpcs_select_radix_f32(hpcs_ctx* ctx, float* a, int64_t start, int64_t length, int64_t k, float* out);
int hpcs_select_radix_u64(hpcs_ctx* ctx, uint64_t* a, int64_t start, int64_t length, int64_t k, uint64_t* out);
int hpcs_select_radix_i64(hpcs_ctx* ctx, int64_t* a, int64_t start, int64_t length, int64_t k, int64_t* out);
int hpcs_select_radix_f64(hpcs_ctx* ctx, double* a, int64_t start, int64_t length, int64_t k, double* out);

/* ---- serving: continuous batching of sort and top-k requests ---------------------------
 * No reference counterpart (HPCsharp is a synchronous library).  Requests of any size and
 * dtype are submitted at any time from any thread; a scheduler thread admits each one as
 * soon as its keys and scratch fit in the server's HBM budget (a device arena reserved at
 * creation) and an execution slot (a CUDA stream) is free, and runs admitted requests
 * concurrently; requests of at most coalesce_max_keys keys are gathered into one batched
 * segmented-sort launch.  Each result equals the plain entry point's result on the same input
 * (sort: hpcs_sort_<t>; top-k: hpcs_topk_largest_<t>).  Host buffers in pinned memory let
 * the copies overlap with other requests' kernels. */
typedef enum hpcs_op { HPCS_OP_SORT = 0, HPCS_OP_TOPK = 1 } hpcs_op;

typedef struct hpcs_request {
  int32_t op;          /* hpcs_op */
  int32_t dtype;       /* hpcs_dtype */
  const void* input;   /* host keys, n of them (read after submit, until the request is done) */
  void* output;        /* host: n sorted keys (sort) or the k largest ascending (top-k) */
  int64_t n;
  int64_t k;           /* top-k only, 0 <= k <= n */
} hpcs_request;

typedef struct hpcs_request_info {
  int32_t status;      /* hpcs_status of the request */
  int32_t coalesced;   /* 1 if it ran inside a batched segmented launch */
  int64_t submit_ns;   /* steady clock */
  int64_t admit_ns;
  int64_t done_ns;
} hpcs_request_info;

typedef struct hpcs_server_config {
  int32_t device;
  int32_t slots;                  /* concurrent large requests (CUDA streams), default 4 */
  int64_t hbm_budget_bytes;       /* device arena for keys and scratch, default 64 GiB */
  int64_t coalesce_max_keys;      /* requests up to this size are batched, default 131072 */
  int32_t coalesce_max_requests;  /* per batched launch, default 4096 */
  int32_t reserved[5];
} hpcs_server_config;

typedef struct hpcs_server_counters {
  int64_t completed, keys, batches, coalesced, pending;
  int64_t arena_bytes, arena_used, arena_peak;
} hpcs_server_counters;

typedef struct hpcs_server hpcs_server;
void hpcs_server_config_default(hpcs_server_config* cfg);
int hpcs_server_create(const hpcs_server_config* cfg, hpcs_server** out);
/* HPCS_ERR_OOM: the request can never fit the HBM budget. */
int hpcs_server_submit(hpcs_server* server, const hpcs_request* req, uint64_t* ticket);
/* Blocks until the request is done (timeout_ns <= 0: no limit; HPCS_ERR_BUSY on timeout),
 * fills info and returns the request's status; the ticket is then released. */
int hpcs_server_wait(hpcs_server* server, uint64_t ticket, int64_t timeout_ns, hpcs_request_info* info);
int hpcs_server_stats(hpcs_server* server, hpcs_server_counters* stats);
/* Finishes every submitted request, then frees the server. */
int hpcs_server_destroy(hpcs_server* server);

/* ---- uint32 device sort that allocates nothing --------------------------------------
 * No counterpart in the reference (HPCsharp allocates managed arrays per call).  For callers
 * that cannot allocate GPU memory: code whose framework owns every device allocation (a
 * fixed arena or a capped caching allocator), or code on a path where cudaMalloc/cudaFree and
 * their implicit device synchronisation are not allowed.  Sorts n <= HPCS_NOALLOC_MAX_KEYS
 * uint32 keys at `keys` (device memory, 16-byte aligned) in place, stable and ascending, with
 * all scratch taken from a fixed array compiled into the library; every GPU that loads the
 * library holds that array (about 4.3 MB) until the process exits.  No context is needed and
 * no cudaMalloc, cudaFree or other allocating routine is called.
 *   - Larger n returns HPCS_ERR_RANGE; an unaligned pointer HPCS_ERR_UNSUPPORTED.
 *   - Runs on `stream` (a cudaStream_t of the current device) and returns when the sort has
 *     finished, reporting a device-side wait that ran out as HPCS_ERR_DEVICE_TIMEOUT.  It
 *     synchronises with the stream, so it cannot be part of a CUDA graph: a call on a stream
 *     that is being captured returns HPCS_ERR_UNSUPPORTED and enqueues nothing.
 *   - The first call on a device also does a one-time set-up on the current device (it
 *     looks up the scratch array's device address and sets kernel attributes).
 *   - All calls on a device share the one scratch array, which keeps the last call's
 *     contents (each call clears what must start at zero).  Calls that overlap on the GPU --
 *     from several streams or host threads at once -- race and corrupt each other.
 *   - The set-up result is kept for the life of the process: a device reset
 *     (cudaDeviceReset) between calls is not supported. */
#define HPCS_NOALLOC_MAX_KEYS ((int64_t)1048576) /* 2^20 keys */
int hpcs_sort_u32_dev_noalloc(uint32_t* keys, int64_t n, void* stream);

/* ---- sort of one array spread over ranks: the per-rank partition step -----------------
 * No single reference call: HPCsharp sorts one array per process, splitting it across host
 * threads (SortRadixPar, RadixSortLsdParallel.cs:49-232).  The sharded sort (one process per
 * GPU) keeps its result -- the concatenation of the ranks' outputs is the stable sort of the
 * concatenation of their inputs -- by partitioning each rank's shard with parts-1 splitters,
 * exchanging the parts (NCCL all-to-all) and sorting what each rank received with the plain
 * sort (hpcs_sort_*_dev / hpcs_sort_pairs_*_dev).
 *
 * Element i of the shard has global position gpos0 + i.  It goes to part b = the number of
 * splitters (split_keys[j], split_gpos[j]) at or below (keys[i], gpos0 + i), comparing keys
 * in the sort's order (signed and float transforms) and then positions; so equal keys may be
 * split between parts.  The splitters must ascend in that order.  The partition is stable:
 * part b is keys_out[off_b .. off_b + counts_out[b]), off_b = counts of the parts below b, in
 * shard order.  All pointers are device pointers; items / items_out are both NULL (keys only)
 * or both set; keys_out must not overlap keys; counts_out receives parts int64 counts.
 *   - parts outside [1, HPCS_MAX_PARTS], n outside [0, HPCS_MAX_KEYS] or gpos0 < 0 ->
 *     HPCS_ERR_RANGE; a NULL array (splitters only when parts > 1) -> HPCS_ERR_NULL. */
#define HPCS_MAX_PARTS 64
int hpcs_shard_partition_dev(hpcs_ctx* ctx, int dtype, const void* keys, const uint32_t* items, int64_t n,
                             int64_t gpos0, const void* split_keys, const int64_t* split_gpos, int parts,
                             void* keys_out, uint32_t* items_out, int64_t* counts_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HPCS_GPU_H */
