// Host-only stand-in for the subset of the Kokkos Core API that BarytreeK's
// sources use, written from Kokkos' public documentation (View, resize,
// deep_copy, parallel_for over int / RangePolicy / MDRangePolicy<2>,
// atomic_add, fence, initialize/finalize, cos/sqrt/log/abs).
//
// TEST INFRASTRUCTURE ONLY. It exists so that the reference's own unmodified
// src/*.cpp can be compiled with g++ into the oracle library under
// oracle/_ref/ (the parity checker and the timed CPU baseline). Nothing in the
// product library includes it.
//
// Execution model: parallel_for runs as an OpenMP "parallel for" (static
// schedule) and atomic_add is an "omp atomic" update. With one OpenMP thread
// the loop runs in index order, which makes the reference bit-reproducible.
#ifndef BTK_ORACLE_KOKKOS_SHIM_HPP
#define BTK_ORACLE_KOKKOS_SHIM_HPP

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]

namespace Kokkos {

struct HostSpace {};
struct LayoutRight {};

namespace shim_detail {
template <class D> struct data_traits;
template <class T> struct data_traits<T*> { using value_type = T; static constexpr int rank = 1; };
template <class T> struct data_traits<T**> { using value_type = T; static constexpr int rank = 2; };

template <class I> inline std::ptrdiff_t as_index(const I& i) { return static_cast<std::ptrdiff_t>(i); }
}  // namespace shim_detail

// Reference-counted, row-major (LayoutRight) host array of rank 1 or 2.
// Copies are shallow, as in Kokkos; construction value-initialises.
template <class DataType, class... Props>
class View {
 public:
  using value_type = typename shim_detail::data_traits<DataType>::value_type;
  static constexpr int rank = shim_detail::data_traits<DataType>::rank;

  View() = default;
  explicit View(const std::string& label, std::size_t n0 = 0, std::size_t n1 = 1)
      : label_(label) { allocate(n0, rank == 2 ? n1 : 1); }

  template <class I0>
  value_type& operator()(const I0& i0) const { return ptr_.get()[shim_detail::as_index(i0)]; }
  template <class I0, class I1>
  value_type& operator()(const I0& i0, const I1& i1) const {
    return ptr_.get()[shim_detail::as_index(i0) * static_cast<std::ptrdiff_t>(n1_) + shim_detail::as_index(i1)];
  }

  value_type* data() const { return ptr_.get(); }
  std::size_t extent(int d) const { return d == 0 ? n0_ : (d == 1 ? n1_ : 1); }
  int extent_int(int d) const { return static_cast<int>(extent(d)); }
  std::size_t size() const { return n0_ * n1_; }
  const std::string& label() const { return label_; }

  // Used by resize(): new storage, value-initialised, overlap copied.
  void reshape(std::size_t n0, std::size_t n1) {
    std::shared_ptr<value_type> old = ptr_;
    std::size_t o0 = n0_, o1 = n1_;
    allocate(n0, n1);
    if (old) {
      std::size_t c0 = std::min(o0, n0), c1 = std::min(o1, n1);
      for (std::size_t i = 0; i < c0; ++i)
        for (std::size_t j = 0; j < c1; ++j) ptr_.get()[i * n1 + j] = old.get()[i * o1 + j];
    }
  }

 private:
  void allocate(std::size_t n0, std::size_t n1) {
    n0_ = n0;
    n1_ = n1;
    std::size_t n = n0 * n1;
    ptr_ = std::shared_ptr<value_type>(new value_type[n > 0 ? n : 1](), std::default_delete<value_type[]>());
  }
  std::shared_ptr<value_type> ptr_;
  std::size_t n0_ = 0, n1_ = 1;
  std::string label_;
};

template <class D, class... P>
inline void resize(View<D, P...>& v, std::size_t n0) { v.reshape(n0, 1); }
template <class D, class... P>
inline void resize(View<D, P...>& v, std::size_t n0, std::size_t n1) { v.reshape(n0, n1); }

template <class D1, class... P1, class D2, class... P2>
inline void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (dst.size() != src.size()) throw std::runtime_error("deep_copy: extent mismatch");
  if (src.size() == 0) return;
  std::copy(src.data(), src.data() + src.size(), dst.data());
}

struct RangePolicy {
  long long begin, end;
  RangePolicy(long long b, long long e) : begin(b), end(e) {}
};

template <int N>
struct MDRangePolicy {
  long long lo[N], hi[N];
  MDRangePolicy(const long long (&l)[N], const long long (&h)[N]) {
    for (int d = 0; d < N; ++d) { lo[d] = l[d]; hi[d] = h[d]; }
  }
};
template <int N>
MDRangePolicy(const long long (&)[N], const long long (&)[N]) -> MDRangePolicy<N>;

template <class F>
inline void parallel_for(const RangePolicy& p, const F& f) {
#pragma omp parallel for schedule(static)
  for (long long i = p.begin; i < p.end; ++i) f(static_cast<int>(i));
}

template <class F>
inline void parallel_for(long long n, const F& f) { parallel_for(RangePolicy(0, n), f); }

template <class F>
inline void parallel_for(const MDRangePolicy<2>& p, const F& f) {
  const long long n1 = p.hi[1] - p.lo[1];
  const long long total = (p.hi[0] - p.lo[0]) * n1;
#pragma omp parallel for schedule(static)
  for (long long t = 0; t < total; ++t)
    f(static_cast<int>(p.lo[0] + t / n1), static_cast<int>(p.lo[1] + t % n1));
}

template <class T>
inline void atomic_add(T* dst, const T& v) {
#pragma omp atomic
  *dst += v;
}

inline void fence() {}
inline void initialize(int&, char**) {}
inline void initialize() {}
inline void finalize() {}
inline int num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
inline int num_devices() { return 0; }

template <class T> inline T cos(T x) { return std::cos(x); }
template <class T> inline T sqrt(T x) { return std::sqrt(x); }
template <class T> inline T log(T x) { return std::log(x); }
template <class T> inline T abs(T x) { return std::abs(x); }

}  // namespace Kokkos

#endif
