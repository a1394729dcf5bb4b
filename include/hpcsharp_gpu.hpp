// hpcsharp_gpu.hpp - C++ host mirror of HPCsharp's radix-sort extension methods over the
// C ABI of libhpcs_gpu.so (include/hpcs_gpu.h).
//
// Same method names and argument meaning as the reference (paths relative to the HPCsharp
// project root); the .NET exceptions map to C++ ones:
//   ArgumentNullException        -> HPCsharp::ArgumentNullException   (std::invalid_argument)
//   ArgumentOutOfRangeException  -> HPCsharp::ArgumentOutOfRangeException (std::out_of_range)
//   other failures               -> HPCsharp::GpuException            (std::runtime_error)
// Arrays are sorted in place, as the reference's SortRadixPar returns the caller's array
// (RadixSortLsdParallel.cs:227-231).  A process-wide context on device 0 is created on first
// use; SetDevice() may select another device before the first call.
#pragma once

#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <type_traits>
#include <vector>

#include "hpcs_gpu.h"

namespace HPCsharp {

struct ArgumentNullException : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct ArgumentOutOfRangeException : std::out_of_range {
  using std::out_of_range::out_of_range;
};
struct GpuException : std::runtime_error {
  int status;
  GpuException(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

namespace detail {
inline void check(int status) {
  if (status == HPCS_OK) return;
  std::string msg = std::string(hpcs_status_string(status)) + ": " + hpcs_last_error_message();
  if (status == HPCS_ERR_NULL) throw ArgumentNullException(msg);
  if (status == HPCS_ERR_RANGE) throw ArgumentOutOfRangeException(msg);
  throw GpuException(status, msg);
}
struct Context {
  hpcs_ctx* ctx = nullptr;
  int device = 0;
  std::mutex mu;
  ~Context() {
    if (ctx) hpcs_ctx_destroy(ctx);
  }
  hpcs_ctx* get() {
    if (!ctx) check(hpcs_ctx_create(device, nullptr, &ctx));
    return ctx;
  }
};
inline Context& context() {
  static Context c;
  return c;
}
template <class T>
struct Fn;
template <>
struct Fn<uint32_t> {
  static int sort(hpcs_ctx* c, uint32_t* a, int64_t n) { return hpcs_sort_u32(c, a, n); }
  static int pairs(hpcs_ctx* c, uint32_t* k, uint32_t* v, int64_t n) { return hpcs_sort_pairs_u32(c, k, v, n); }
  static int hist(hpcs_ctx* c, const uint32_t* a, int64_t l, int64_t r, uint32_t* o) {
    return hpcs_histogram_byte_components_u32(c, a, l, r, o);
  }
  static int partition(hpcs_ctx* c, uint32_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk) {
    return hpcs_partition_radix_u32(c, a, start, length, k, nk);
  }
  static int select(hpcs_ctx* c, uint32_t* a, int64_t start, int64_t length, int64_t k, uint32_t* out) {
    return hpcs_select_radix_u32(c, a, start, length, k, out);
  }
};
template <>
struct Fn<int32_t> {
  static int sort(hpcs_ctx* c, int32_t* a, int64_t n) { return hpcs_sort_i32(c, a, n); }
  static int pairs(hpcs_ctx* c, int32_t* k, uint32_t* v, int64_t n) { return hpcs_sort_pairs_i32(c, k, v, n); }
  static int hist(hpcs_ctx* c, const int32_t* a, int64_t l, int64_t r, uint32_t* o) {
    return hpcs_histogram_byte_components_i32(c, a, l, r, o);
  }
  static int partition(hpcs_ctx* c, int32_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk) {
    return hpcs_partition_radix_i32(c, a, start, length, k, nk);
  }
  static int select(hpcs_ctx* c, int32_t* a, int64_t start, int64_t length, int64_t k, int32_t* out) {
    return hpcs_select_radix_i32(c, a, start, length, k, out);
  }
};
template <>
struct Fn<float> {
  static int sort(hpcs_ctx* c, float* a, int64_t n) { return hpcs_sort_f32(c, a, n); }
  static int pairs(hpcs_ctx* c, float* k, uint32_t* v, int64_t n) { return hpcs_sort_pairs_f32(c, k, v, n); }
  static int hist(hpcs_ctx* c, const float* a, int64_t l, int64_t r, uint32_t* o) {
    return hpcs_histogram_byte_components_f32(c, a, l, r, o);
  }
  static int partition(hpcs_ctx* c, float* a, int64_t start, int64_t length, const int64_t* k, int64_t nk) {
    return hpcs_partition_radix_f32(c, a, start, length, k, nk);
  }
  static int select(hpcs_ctx* c, float* a, int64_t start, int64_t length, int64_t k, float* out) {
    return hpcs_select_radix_f32(c, a, start, length, k, out);
  }
};
template <>
struct Fn<uint64_t> {
  static int sort(hpcs_ctx* c, uint64_t* a, int64_t n) { return hpcs_sort_u64(c, a, n); }
  static int pairs(hpcs_ctx* c, uint64_t* k, uint32_t* v, int64_t n) { return hpcs_sort_pairs_u64(c, k, v, n); }
  static int hist(hpcs_ctx* c, const uint64_t* a, int64_t l, int64_t r, uint32_t* o) {
    return hpcs_histogram_byte_components_u64(c, a, l, r, o);
  }
  static int partition(hpcs_ctx* c, uint64_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk) {
    return hpcs_partition_radix_u64(c, a, start, length, k, nk);
  }
  static int select(hpcs_ctx* c, uint64_t* a, int64_t start, int64_t length, int64_t k, uint64_t* out) {
    return hpcs_select_radix_u64(c, a, start, length, k, out);
  }
};
template <>
struct Fn<int64_t> {
  static int sort(hpcs_ctx* c, int64_t* a, int64_t n) { return hpcs_sort_i64(c, a, n); }
  static int pairs(hpcs_ctx* c, int64_t* k, uint32_t* v, int64_t n) { return hpcs_sort_pairs_i64(c, k, v, n); }
  static int hist(hpcs_ctx* c, const int64_t* a, int64_t l, int64_t r, uint32_t* o) {
    return hpcs_histogram_byte_components_i64(c, a, l, r, o);
  }
  static int partition(hpcs_ctx* c, int64_t* a, int64_t start, int64_t length, const int64_t* k, int64_t nk) {
    return hpcs_partition_radix_i64(c, a, start, length, k, nk);
  }
  static int select(hpcs_ctx* c, int64_t* a, int64_t start, int64_t length, int64_t k, int64_t* out) {
    return hpcs_select_radix_i64(c, a, start, length, k, out);
  }
};
template <>
struct Fn<double> {
  static int sort(hpcs_ctx* c, double* a, int64_t n) { return hpcs_sort_f64(c, a, n); }
  static int pairs(hpcs_ctx* c, double* k, uint32_t* v, int64_t n) { return hpcs_sort_pairs_f64(c, k, v, n); }
  static int hist(hpcs_ctx* c, const double* a, int64_t l, int64_t r, uint32_t* o) {
    return hpcs_histogram_byte_components_f64(c, a, l, r, o);
  }
  static int partition(hpcs_ctx* c, double* a, int64_t start, int64_t length, const int64_t* k, int64_t nk) {
    return hpcs_partition_radix_f64(c, a, start, length, k, nk);
  }
  static int select(hpcs_ctx* c, double* a, int64_t start, int64_t length, int64_t k, double* out) {
    return hpcs_select_radix_f64(c, a, start, length, k, out);
  }
};
template <class T>
void sort_in_place(T* a, int64_t n) {
  if (!a) throw ArgumentNullException("inputArray");
  Context& c = context();
  std::lock_guard<std::mutex> lock(c.mu);
  check(Fn<T>::sort(c.get(), a, n));
}
}  // namespace detail

// Selects the device of the process-wide context (before the first call only).
inline void SetDevice(int device) { detail::context().device = device; }

struct ParallelAlgorithm {
  // SortRadixPar(this uint[], int ParallelWorkQuantum) RadixSortLsdParallel.cs:145; the
  // work quantum is the reference's CPU task size and has no meaning on the GPU.
  template <class T>
  static std::vector<T>& SortRadixPar(std::vector<T>& inputArray, int ParallelWorkQuantum = 64 * 1024) {
    (void)ParallelWorkQuantum;
    if (!inputArray.empty()) detail::sort_in_place(inputArray.data(), int64_t(inputArray.size()));
    return inputArray;
  }
  template <class T>
  static T* SortRadixPar(T* inputArray, int64_t length) {
    detail::sort_in_place(inputArray, length);
    return inputArray;
  }
  // SortRadixInPlaceInterfacePar RadixSortLsdParallel.cs:240, :677, :743
  template <class T>
  static void SortRadixInPlaceInterfacePar(std::vector<T>& inputArray) {
    SortRadixPar(inputArray);
  }
  // HistogramByteComponentsPar(T[], int l, int r) HistogramParallel.cs:214, :416, :547, :617:
  // counts[digit][256] of a[l..r] inclusive.
  template <class T>
  static std::vector<std::vector<uint32_t>> HistogramByteComponentsPar(const std::vector<T>& inArray, int64_t l,
                                                                       int64_t r) {
    if (l < 0 || r >= int64_t(inArray.size())) throw ArgumentOutOfRangeException("l/r outside the array");
    std::vector<uint32_t> flat(sizeof(T) * 256);
    detail::Context& c = detail::context();
    std::lock_guard<std::mutex> lock(c.mu);
    detail::check(detail::Fn<T>::hist(c.get(), inArray.data(), l, r, flat.data()));
    std::vector<std::vector<uint32_t>> out(sizeof(T));
    for (size_t d = 0; d < sizeof(T); d++) out[d].assign(flat.begin() + d * 256, flat.begin() + (d + 1) * 256);
    return out;
  }
  // SelectRadixPar(this uint[], int start, int length, int k, int parallelThreshold)
  // SelectionRadixParallel.cs:254 and (a, k) :271: the k-th smallest of the (sub)array, k
  // absolute, also left at a[k].  The threshold is a CPU task size with no meaning on the GPU.
  template <class T>
  static T SelectRadixPar(std::vector<T>& a, int64_t start, int64_t length, int64_t k,
                          int parallelThreshold = 64 * 1024) {
    (void)parallelThreshold;
    if (start < 0 || length <= 0 || start + length > int64_t(a.size()))
      throw ArgumentOutOfRangeException("array length or length is invalid");
    T out{};
    detail::Context& c = detail::context();
    std::lock_guard<std::mutex> lock(c.mu);
    detail::check(detail::Fn<T>::select(c.get(), a.data(), start, length, k, &out));
    return out;
  }
  template <class T>
  static T SelectRadixPar(std::vector<T>& a, int64_t k, int parallelThreshold = 64 * 1024) {
    return SelectRadixPar(a, 0, int64_t(a.size()), k, parallelThreshold);
  }
};

struct Algorithm {
  // PartitionRadix(this uint[], int start, int length, int[] k, int threshold) PartitionRadix.cs:
  // 135-210 (and the one-k and whole-array forms): nth_element by every k (absolute indices).
  template <class T>
  static void PartitionRadix(std::vector<T>& a, int64_t start, int64_t length, const std::vector<int64_t>& k,
                             int threshold = 1024) {
    (void)threshold;
    if (start < 0 || length <= 0 || start + length > int64_t(a.size()))
      throw ArgumentOutOfRangeException("array length or length is invalid");
    if (k.size() > a.size()) throw ArgumentOutOfRangeException("k array length cannot be greater than the array length");
    if (k.empty()) return;
    detail::Context& c = detail::context();
    std::lock_guard<std::mutex> lock(c.mu);
    detail::check(detail::Fn<T>::partition(c.get(), a.data(), start, length, k.data(), int64_t(k.size())));
  }
  template <class T>
  static void PartitionRadix(std::vector<T>& a, int64_t k, int threshold = 1024) {
    PartitionRadix(a, 0, int64_t(a.size()), std::vector<int64_t>{k}, threshold);
  }
  template <class T>
  static void PartitionRadix(std::vector<T>& a, const std::vector<int64_t>& k, int threshold = 1024) {
    PartitionRadix(a, 0, int64_t(a.size()), k, threshold);
  }
  // SelectRadix(this uint[], int start, int length, int k) SelectionRadix.cs:236 and (a, k) :253
  template <class T>
  static T SelectRadix(std::vector<T>& a, int64_t start, int64_t length, int64_t k) {
    return ParallelAlgorithm::SelectRadixPar(a, start, length, k);
  }
  template <class T>
  static T SelectRadix(std::vector<T>& a, int64_t k) {
    return ParallelAlgorithm::SelectRadixPar(a, 0, int64_t(a.size()), k);
  }
  // SortRadixLsd(this T[]) RadixSortLsd.cs:255, :352, :437, :527 (in place)
  template <class T>
  static void SortRadixLsd(std::vector<T>& inOutArray) {
    if (!inOutArray.empty()) detail::sort_in_place(inOutArray.data(), int64_t(inOutArray.size()));
  }
  // SortRadixLsd(this T[], int startIndex, int length): sorts that subrange in place.
  template <class T>
  static void SortRadixLsd(std::vector<T>& inOutArray, int64_t startIndex, int64_t length) {
    if (startIndex < 0 || length < 0 || startIndex + length > int64_t(inOutArray.size()))
      throw ArgumentOutOfRangeException("startIndex/length outside the array");
    if (length == 0) return;
    detail::sort_in_place(inOutArray.data() + startIndex, length);
  }
  // SortRadixLsdFunc(this T[]) RadixSortLsd.cs:238, :315, :400, :490
  template <class T>
  static std::vector<T>& SortRadixLsdFunc(std::vector<T>& inOutArray) {
    SortRadixLsd(inOutArray);
    return inOutArray;
  }
  // SortRadix(this uint[]) -- the examples' spelling (Program.cs:26)
  template <class T>
  static std::vector<T>& SortRadix(std::vector<T>& inputArray) {
    SortRadixLsd(inputArray);
    return inputArray;
  }
  // SortRadix<T>(this T[] items, UInt32[]/UInt64[] keys) RadixSortLsd.cs:1183, :1245: both
  // arrays permuted in place by the stable key order; items are 4-byte payloads.
  template <class K, class V>
  static std::pair<std::vector<V>&, std::vector<K>&> SortRadix(std::vector<V>& items, std::vector<K>& keys) {
    static_assert(sizeof(V) == 4, "items must be a 4-byte type (index payload)");
    if (items.size() != keys.size()) throw ArgumentOutOfRangeException("items and keys differ in length");
    detail::Context& c = detail::context();
    std::lock_guard<std::mutex> lock(c.mu);
    if (!keys.empty())
      detail::check(detail::Fn<K>::pairs(c.get(), keys.data(), reinterpret_cast<uint32_t*>(items.data()),
                                         int64_t(keys.size())));
    return {items, keys};
  }
  // HistogramByteComponents(T[], int l, int r) Histogram.cs:261, :957, :992, :1019
  template <class T>
  static std::vector<std::vector<uint32_t>> HistogramByteComponents(const std::vector<T>& inArray, int64_t l,
                                                                    int64_t r) {
    return ParallelAlgorithm::HistogramByteComponentsPar(inArray, l, r);
  }
  // SortRadixLsd<T>(this T[] inputArray, Func<T, UInt32/UInt64> getKey) RadixSortLsd.cs:714,
  // :783 (and SortRadixFaster<T>, :861, :961): a new array of the elements in stable
  // ascending order of getKey.  The keys are extracted on the host, sorted on the GPU with
  // their indices as the payload, and the elements gathered by the sorted indices.
  template <class T, class F>
  static std::vector<T> SortRadixLsd(const std::vector<T>& inputArray, F getKey) {
    using K = typename std::decay<decltype(getKey(inputArray[0]))>::type;
    static_assert(std::is_same<K, uint32_t>::value || std::is_same<K, uint64_t>::value,
                  "getKey returns UInt32 or UInt64");
    const size_t n = inputArray.size();
    std::vector<K> keys(n);
    std::vector<uint32_t> index(n);
    for (size_t i = 0; i < n; i++) {
      keys[i] = getKey(inputArray[i]);
      index[i] = uint32_t(i);
    }
    SortRadix(index, keys);
    std::vector<T> out;
    out.reserve(n);
    for (size_t i = 0; i < n; i++) out.push_back(inputArray[index[i]]);
    return out;
  }
  template <class T, class F>
  static std::vector<T> SortRadixFaster(const std::vector<T>& inputArray, F getKey) {
    return SortRadixLsd(inputArray, getKey);
  }
};

}  // namespace HPCsharp
