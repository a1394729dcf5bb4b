// C++ usage of the HPCsharp mirror (include/hpcsharp_gpu.hpp): reads like the reference's
// examples (HPCsharpExamples/HPCsharpExamples/Program.cs) and checks against std::sort.
// Exit code 0 = all checks passed.
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <random>
#include <vector>

#include "hpcsharp_gpu.hpp"

using namespace HPCsharp;

static int failures = 0;
#define CHECK(c)                                                  \
  do {                                                            \
    if (!(c)) {                                                   \
      std::printf("FAILED %s at line %d\n", #c, __LINE__);        \
      failures++;                                                 \
    }                                                             \
  } while (0)

int main() {
  // Program.cs:15-34 known answer
  std::vector<uint32_t> four = {21, 43, 16, 5, 54, 3};
  Algorithm::SortRadix(four);
  CHECK((four == std::vector<uint32_t>{3, 5, 16, 21, 43, 54}));

  std::mt19937_64 rng(7);
  std::vector<uint32_t> u(3000017);
  for (auto& x : u) x = uint32_t(rng());
  std::vector<uint32_t> ref = u;
  std::sort(ref.begin(), ref.end());
  ParallelAlgorithm::SortRadixPar(u);
  CHECK(u == ref);

  std::vector<int64_t> l(1000003);
  for (auto& x : l) x = int64_t(rng());
  std::vector<int64_t> lref = l;
  std::sort(lref.begin(), lref.end());
  Algorithm::SortRadixLsd(l);
  CHECK(l == lref);

  // subrange sorted in place
  std::vector<int32_t> s(100000);
  for (auto& x : s) x = int32_t(rng());
  std::vector<int32_t> sref = s;
  std::sort(sref.begin() + 100, sref.begin() + 50100);
  Algorithm::SortRadixLsd(s, 100, 50000);
  CHECK(s == sref);

  // pairs: items follow the stable key order
  std::vector<uint64_t> keys(500009);
  for (auto& x : keys) x = rng() % 1000;
  std::vector<uint32_t> items(keys.size());
  std::iota(items.begin(), items.end(), 0u);
  std::vector<uint32_t> perm(keys.size());
  std::iota(perm.begin(), perm.end(), 0u);
  std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
  Algorithm::SortRadix(items, keys);
  CHECK(items == perm);
  CHECK(std::is_sorted(keys.begin(), keys.end()));

  // histogram of a[l..r]
  std::vector<uint32_t> h(100000);
  for (auto& x : h) x = uint32_t(rng());
  auto counts = ParallelAlgorithm::HistogramByteComponentsPar(h, 10, 99989);
  std::vector<uint32_t> want(256, 0);
  for (int64_t i = 10; i <= 99989; i++) want[h[i] & 0xFF]++;
  CHECK(counts.size() == 4 && counts[0] == want);

  // SortRadixLsd<T>(items, getKey): stable by the extracted key, new array
  struct Rec {
    uint32_t id;
    uint64_t score;
  };
  std::vector<Rec> recs(50000);
  for (size_t i = 0; i < recs.size(); i++) recs[i] = {uint32_t(i), uint64_t(rng() % 1000) << 40 | (rng() % 7)};
  auto by32 = Algorithm::SortRadixLsd(recs, [](const Rec& r) { return uint32_t(r.score >> 40); });
  auto by64 = Algorithm::SortRadixFaster(recs, [](const Rec& r) { return r.score; });
  std::vector<Rec> w32 = recs, w64 = recs;
  std::stable_sort(w32.begin(), w32.end(), [](const Rec& a, const Rec& b) { return (a.score >> 40) < (b.score >> 40); });
  std::stable_sort(w64.begin(), w64.end(), [](const Rec& a, const Rec& b) { return a.score < b.score; });
  bool same32 = by32.size() == w32.size(), same64 = by64.size() == w64.size();
  for (size_t i = 0; same32 && i < w32.size(); i++) same32 = by32[i].id == w32[i].id;
  for (size_t i = 0; same64 && i < w64.size(); i++) same64 = by64[i].id == w64[i].id;
  CHECK(same32);
  CHECK(same64);

  // exceptions mirror the reference's
  bool threw = false;
  try {
    ParallelAlgorithm::SortRadixPar<uint32_t>(nullptr, 5);
  } catch (const ArgumentNullException&) {
    threw = true;
  }
  CHECK(threw);
  threw = false;
  try {
    ParallelAlgorithm::HistogramByteComponentsPar(h, 0, int64_t(h.size()));
  } catch (const ArgumentOutOfRangeException&) {
    threw = true;
  }
  CHECK(threw);

  // PartitionRadix / SelectRadixPar: nth_element by each index, checked against std::sort
  {
    std::vector<uint32_t> p(500009);
    for (auto& x : p) x = uint32_t(rng()) & 0xFFFFu;  // many equal keys
    std::vector<uint32_t> sorted = p;
    std::sort(sorted.begin(), sorted.end());
    std::vector<int64_t> ks = {7, 250000, 499999};
    std::vector<uint32_t> q = p;
    Algorithm::PartitionRadix(q, ks);
    for (int64_t k : ks) CHECK(q[k] == sorted[k]);
    for (int64_t i = 0; i < 7; i++) CHECK(q[i] <= q[7]);
    for (int64_t i = 8; i < 250000; i++) CHECK(q[i] >= q[7] && q[i] <= q[250000]);
    std::vector<uint32_t> r = p;
    CHECK(ParallelAlgorithm::SelectRadixPar(r, 123456) == sorted[123456]);
    CHECK(r[123456] == sorted[123456]);
    CHECK(Algorithm::SelectRadix(p, 0) == sorted[0]);
  }

  std::printf(failures ? "mirror_test: %d failures\n" : "mirror_test: ok\n", failures);
  return failures ? 1 : 0;
}
