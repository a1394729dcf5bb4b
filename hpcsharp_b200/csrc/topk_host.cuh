// Host-side enqueue sequences of the radix select / top-k kernels (topk.cuh), shared by the
// C ABI and the serving runtime.  Scratch comes from the context's buffers (aux0: candidate
// keys, aux1: SelectState, aux2: partition tile counts), which the serving runtime binds to
// slices of its arena.
#pragma once
#include <cmath>

#include "sort_host.cuh"
#include "topk.cuh"

namespace hpcs {

// Grid of the passes over the keys: SEL_CTAS_PER_SM CTAs per SM, fewer for small inputs.
inline int select_grid(hpcs_ctx* ctx, int64_t n, int key_bytes) {
  const int64_t per_cta = int64_t(SEL_NT) * SEL_VPT * (16 / key_bytes);
  const int64_t want = (n + per_cta - 1) / per_cta;
  const int64_t cap = int64_t(ctx->sms) * SEL_CTAS_PER_SM;
  return int(want < 1 ? 1 : (want > cap ? cap : want));
}

// Radix select of the key of 0-based rank `rank` among n keys at device pointer d.  Leaves
// the SelectState in ctx->aux1 (prefix = the ordered bits of the selected key, less/eq counts).
// One read of the keys in the common case: a sampled window around the rank, one read that
// counts the keys below it and keeps the keys inside (topk.cuh), the radix select over those;
// the two-read select over all keys when the rank falls outside the window.
template <class U, int KIND>
inline int enqueue_select(hpcs_ctx* ctx, const U* d, int64_t n, int64_t rank, cudaStream_t s, SelectState** out) {
  constexpr int BITS = int(sizeof(U) * 8);
  constexpr int LEVELS = BITS / 8;
  constexpr int S = select_sample_size<U>();
  int rc;
  if ((rc = ensure(ctx, ctx->aux1, sizeof(SelectState))) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->aux0, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  SelectState* st = static_cast<SelectState*>(ctx->aux1.ptr);
  U* cand = static_cast<U*>(ctx->aux0.ptr);
  // the sample rank of the selected key has standard deviation sqrt(S p (1 - p)), p = rank / n;
  // the window reaches 6 of them plus 9 samples to each side
  const double p = n > 0 ? double(rank) / double(n) : 0.0;
  const int64_t m = int64_t(6.0 * std::sqrt(double(S) * p * (1.0 - p)) + 9.0) + 1;
  const int grid = select_grid(ctx, n, int(sizeof(U)));
  const int64_t expect = n < int64_t(4) * S ? n : int64_t(double(2 * m + 1) / S * double(n));
  const int cgrid = select_grid(ctx, 2 * expect, int(sizeof(U)));
  KernelTimer kt(ctx, s, HPCS_K_TOPK);
  select_sample_kernel<U, KIND><<<1, TOPK_SAMPLE_NT, 0, s>>>(d, n, rank, m, st);
  select_window_kernel<U, KIND><<<grid, SEL_NT, 0, s>>>(d, n, cand, st);
  select_decide_kernel<<<1, 32, 0, s>>>(st, n, rank);
  // level 0: over the candidates, or (fallback) over all keys with the compaction
  select_hist_kernel<U, KIND><<<cgrid, SEL_NT, 0, s>>>(cand, &st->cand_count, 0, st, BITS - 8, SEL_MODE_CAND);
  select_hist_kernel<U, KIND><<<grid, SEL_NT, 0, s>>>(d, nullptr, n, st, BITS - 8, SEL_MODE_FULL);
  select_pick_kernel<U><<<1, 256, 0, s>>>(st, BITS - 8, LEVELS == 1);
  select_compact_kernel<U, KIND><<<grid, SEL_NT, 0, s>>>(d, n, cand, st, nullptr, 0, SEL_MODE_FULL);
  for (int l = 1; l < LEVELS; l++) {
    const int shift = BITS - 8 * (l + 1);
    select_hist_kernel<U, KIND><<<cgrid, SEL_NT, 0, s>>>(cand, &st->cand_count, 0, st, shift);
    select_pick_kernel<U><<<1, 256, 0, s>>>(st, shift, l == LEVELS - 1);
  }
  HPCS_CUDA(cudaGetLastError());
  *out = st;
  return HPCS_OK;
}

// Stable three-way partition of d[0..n) around the selected key into out.
template <class U, int KIND>
inline int enqueue_partition(hpcs_ctx* ctx, const U* d, int64_t n, SelectState* st, U* out, cudaStream_t s) {
  const int64_t subs = (n + PART_SUB - 1) / PART_SUB;
  const int64_t runs = (subs + PART_SCAN_RUN - 1) / PART_SCAN_RUN;
  const int64_t ctas = (subs + PART_SUBS_PER_CTA - 1) / PART_SUBS_PER_CTA;
  int rc;
  if ((rc = ensure(ctx, ctx->aux2, size_t(2 * subs + runs) * 3 * 4)) != HPCS_OK) return rc;
  uint32_t* sc = static_cast<uint32_t*>(ctx->aux2.ptr);  // per sub-tile: class counts
  uint32_t* ss = sc + subs * 3;                          // class starts within the run
  uint32_t* rt = ss + subs * 3;                          // per run: totals, then starts
  KernelTimer kt(ctx, s, HPCS_K_TOPK);
  partition_count_kernel<U, KIND><<<int(ctas), PART_NT, 0, s>>>(d, n, st, sc);
  partition_block_scan_kernel<<<int(runs), PART_SCAN_RUN, 0, s>>>(sc, subs, ss, rt);
  partition_top_scan_kernel<<<1, 1024, 0, s>>>(rt, runs, st);
  partition_scatter_kernel<U, KIND><<<int(ctas), PART_NT, 0, s>>>(d, n, st, sc, ss, rt, out);
  HPCS_CUDA(cudaGetLastError());
  return HPCS_OK;
}

// The k largest of in[0..n) into out[0..k), ascending (device pointers).  One read of the keys
// in the common case: a sampled threshold, one filtering read, the radix select over the
// candidates (topk.cuh); the two-read select over all keys when the candidates fall short.
template <class T, class U, int KIND>
inline int topk_largest_enqueue(hpcs_ctx* ctx, const U* d, int64_t n, int64_t k, U* out, cudaStream_t s) {
  constexpr int BITS = int(sizeof(U) * 8);
  constexpr int LEVELS = BITS / 8;
  int rc;
  if ((rc = ensure(ctx, ctx->aux1, sizeof(SelectState))) != HPCS_OK) return rc;
  if ((rc = ensure(ctx, ctx->aux0, size_t(n) * sizeof(U))) != HPCS_OK) return rc;
  SelectState* st = static_cast<SelectState*>(ctx->aux1.ptr);
  U* cand = static_cast<U*>(ctx->aux0.ptr);
  const int grid = select_grid(ctx, n, int(sizeof(U)));
  // sampled keys expected at or above the threshold: enough that fewer than k candidates
  // (k keys sampled at rate S/n, Poisson) is many standard deviations away
  constexpr int S = topk_sample_size<U>();
  const double ks = double(k) * S / double(n);
  const int64_t m = int64_t(1.5 * ks + 6.0 * std::sqrt(ks) + 8.0) + 1;
  // the passes over the candidates get a grid for about twice the expected number (m / S of
  // the keys; all of them below the sampling size); any number is correct, more take longer
  const int64_t expect = n < int64_t(4) * S || m >= S ? n : int64_t(double(m) / S * double(n)) + k;
  const int cgrid = select_grid(ctx, 2 * expect, int(sizeof(U)));
  {
    KernelTimer kt(ctx, s, HPCS_K_TOPK);
    topk_sample_kernel<U, KIND><<<1, TOPK_SAMPLE_NT, 0, s>>>(d, n, k, m, st);
    topk_filter_kernel<U, KIND><<<grid, SEL_NT, 0, s>>>(d, n, cand, st);
    topk_decide_kernel<<<1, 32, 0, s>>>(st, n, k);
    // level 0: over the candidates, or (fallback) over all keys with the compaction
    select_hist_kernel<U, KIND><<<cgrid, SEL_NT, 0, s>>>(cand, &st->cand_count, 0, st, BITS - 8, SEL_MODE_CAND);
    select_hist_kernel<U, KIND><<<grid, SEL_NT, 0, s>>>(d, nullptr, n, st, BITS - 8, SEL_MODE_FULL);
    select_pick_kernel<U><<<1, 256, 0, s>>>(st, BITS - 8, LEVELS == 1);
    select_compact_kernel<U, KIND><<<grid, SEL_NT, 0, s>>>(d, n, cand, st, out, k, SEL_MODE_FULL);
    for (int l = 1; l < LEVELS; l++) {
      const int shift = BITS - 8 * (l + 1);
      select_hist_kernel<U, KIND><<<cgrid, SEL_NT, 0, s>>>(cand, &st->cand_count, 0, st, shift);
      select_pick_kernel<U><<<1, 256, 0, s>>>(st, shift, l == LEVELS - 1);
    }
    topk_gather_kernel<U, KIND><<<cgrid, SEL_NT, 0, s>>>(cand, k, st, out);
    if (k <= topk_small_sort_max<U>()) topk_small_sort_kernel<U, KIND><<<1, TOPK_SMALL_SORT_NT, 0, s>>>(out, int(k));
    HPCS_CUDA(cudaGetLastError());
  }
  if (k <= topk_small_sort_max<U>()) return HPCS_OK;
  return enqueue_sort<U, KIND, NoValue>(ctx, out, nullptr, k, s);
}

}  // namespace hpcs
