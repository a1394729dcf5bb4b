// Seeded synthetic key generators for the sort workloads (tests and benchmarks).
//
// Streams are deterministic for a given seed and independent of the thread count:
// element i belongs to chunk c = i / 65536, and chunk c draws from PCG32 seeded with
// (seed, stream = c).  PCG32 is O'Neill's published minimal generator (pcg-random.org);
// xorshift64* is Vigna's published generator; the mixing bijection used for Zipf values
// is the SplitMix64 finaliser.  Distributions:
//   u32 uniform over [0, 2^32)                       (plain sort, 10 M and 256 M keys)
//   i32 round(normal(0, sigma)) clamped to int32     (sigma = 2^20)
//   f32 normal(0,1) with a fraction of +0, -0, +inf, -inf, +/- subnormals spliced in
//   u64 uniform, and "low entropy" = AND of three independent uniform draws
//   u64 Zipf(s) over a fixed number of distinct values, each rank mapped to a random u64
//   f64 normal(0,1)
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

struct Pcg32 {
  uint64_t state, inc;
  Pcg32(uint64_t initstate, uint64_t initseq) {
    state = 0u;
    inc = (initseq << 1u) | 1u;
    next();
    state += initstate;
    next();
  }
  uint32_t next() {
    uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = uint32_t(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((-rot) & 31));
  }
  uint64_t next64() {
    uint64_t hi = next();
    return (hi << 32) | next();
  }
  // uniform double in (0, 1), 53 bits
  double unit_open() { return (double(next64() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
};

inline uint64_t splitmix_finalize(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

constexpr int64_t kChunk = 65536;

void for_chunks(int64_t n, int threads, const std::function<void(int64_t, int64_t, int64_t)>& fn) {
  int64_t chunks = (n + kChunk - 1) / kChunk;
  if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
  auto body = [&](int64_t c) { fn(c, c * kChunk, std::min(n, (c + 1) * kChunk)); };
  if (threads == 1 || chunks <= 1) {
    for (int64_t c = 0; c < chunks; c++) body(c);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < std::min<int64_t>(threads, chunks); t++)
    pool.emplace_back([&]() {
      for (int64_t c; (c = next.fetch_add(1)) < chunks;) body(c);
    });
  for (auto& th : pool) th.join();
}

inline double normal_draw(Pcg32& g) {  // Box-Muller, cosine branch
  double u1 = g.unit_open(), u2 = g.unit_open();
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

}  // namespace

extern "C" {

void hg_u32_uniform(uint32_t* out, int64_t n, uint64_t seed, int threads) {
  for_chunks(n, threads, [&](int64_t c, int64_t lo, int64_t hi) {
    Pcg32 g(seed, uint64_t(c));
    for (int64_t i = lo; i < hi; i++) out[i] = g.next();
  });
}

// One sequential PCG32 stream (seed, stream 0x5eed).
void hg_u32_pcg32_stream(uint32_t* out, int64_t n, uint64_t seed) {
  Pcg32 g(seed, 0x5eedULL);
  for (int64_t i = 0; i < n; i++) out[i] = g.next();
}

// One sequential xorshift64* stream; the high 32 bits of each output.
void hg_u32_xorshift64s(uint32_t* out, int64_t n, uint64_t seed) {
  uint64_t x = seed ? seed : 0x9E3779B97F4A7C15ULL;
  for (int64_t i = 0; i < n; i++) {
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    out[i] = uint32_t((x * 0x2545F4914F6CDD1DULL) >> 32);
  }
}

void hg_u64_uniform(uint64_t* out, int64_t n, uint64_t seed, int threads) {
  for_chunks(n, threads, [&](int64_t c, int64_t lo, int64_t hi) {
    Pcg32 g(seed, uint64_t(c));
    for (int64_t i = lo; i < hi; i++) out[i] = g.next64();
  });
}

void hg_u64_and3(uint64_t* out, int64_t n, uint64_t seed, int threads) {
  for_chunks(n, threads, [&](int64_t c, int64_t lo, int64_t hi) {
    Pcg32 g1(seed, uint64_t(c)), g2(seed + 1, uint64_t(c)), g3(seed + 2, uint64_t(c));
    for (int64_t i = lo; i < hi; i++) out[i] = g1.next64() & g2.next64() & g3.next64();
  });
}

void hg_i32_normal(int32_t* out, int64_t n, uint64_t seed, double sigma, int threads) {
  for_chunks(n, threads, [&](int64_t c, int64_t lo, int64_t hi) {
    Pcg32 g(seed, uint64_t(c));
    for (int64_t i = lo; i < hi; i++) {
      double v = std::nearbyint(normal_draw(g) * sigma);
      v = std::min(2147483647.0, std::max(-2147483648.0, v));
      out[i] = int32_t(v);
    }
  });
}

// normal(0,1) floats; each of the six specials (+0, -0, +inf, -inf, +subnormal, -subnormal)
// replaces an element with probability special_frac.  No NaN is produced.
void hg_f32_normal_special(float* out, int64_t n, uint64_t seed, double special_frac, int threads) {
  for_chunks(n, threads, [&](int64_t c, int64_t lo, int64_t hi) {
    Pcg32 g(seed, uint64_t(c));
    for (int64_t i = lo; i < hi; i++) {
      double u = g.unit_open();
      float v = float(normal_draw(g));
      uint32_t sub = 1u + (g.next() % 0x007FFFFFu);  // 0x00000001 .. 0x007FFFFF
      int which = int(u / special_frac);
      uint32_t bits;
      switch (which) {
        case 0: bits = 0x00000000u; break;          // +0
        case 1: bits = 0x80000000u; break;          // -0
        case 2: bits = 0x7F800000u; break;          // +inf
        case 3: bits = 0xFF800000u; break;          // -inf
        case 4: bits = sub; break;                  // +subnormal
        case 5: bits = 0x80000000u | sub; break;    // -subnormal
        default: std::memcpy(&bits, &v, 4); break;
      }
      std::memcpy(out + i, &bits, 4);
    }
  });
}

void hg_f64_normal(double* out, int64_t n, uint64_t seed, int threads) {
  for_chunks(n, threads, [&](int64_t c, int64_t lo, int64_t hi) {
    Pcg32 g(seed, uint64_t(c));
    for (int64_t i = lo; i < hi; i++) out[i] = normal_draw(g);
  });
}

void hg_f32_normal(float* out, int64_t n, uint64_t seed, int threads) {
  for_chunks(n, threads, [&](int64_t c, int64_t lo, int64_t hi) {
    Pcg32 g(seed, uint64_t(c));
    for (int64_t i = lo; i < hi; i++) out[i] = float(normal_draw(g));
  });
}

// Zipf(s) over ranks 1..nvalues (P(r) proportional to r^-s), rank r mapped to the u64
// splitmix_finalize(r + seed * 0x9E3779B97F4A7C15), a bijection, so distinct ranks give
// distinct keys.
void hg_u64_zipf(uint64_t* out, int64_t n, uint64_t seed, double s, int64_t nvalues, int threads) {
  std::vector<double> cdf(static_cast<size_t>(nvalues));
  double acc = 0;
  for (int64_t r = 0; r < nvalues; r++) {
    acc += std::pow(double(r + 1), -s);
    cdf[r] = acc;
  }
  for (auto& v : cdf) v /= acc;
  cdf.back() = 1.0;
  const uint64_t salt = seed * 0x9E3779B97F4A7C15ULL;
  for_chunks(n, threads, [&](int64_t c, int64_t lo, int64_t hi) {
    Pcg32 g(seed, uint64_t(c));
    for (int64_t i = lo; i < hi; i++) {
      double u = g.unit_open();
      int64_t r = int64_t(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
      out[i] = splitmix_finalize(uint64_t(r + 1) + salt);
    }
  });
}

void hg_iota_u32(uint32_t* out, int64_t n, int threads) {
  for_chunks(n, threads, [&](int64_t, int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi; i++) out[i] = uint32_t(i);
  });
}

}  // extern "C"
