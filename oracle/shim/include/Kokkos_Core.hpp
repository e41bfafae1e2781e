// Host-only stand-in for the subset of the Kokkos Core API that the frehg2
// groundwater sources use.  Test infrastructure: it exists so that the
// reference's own src/gw, src/core, src/bc and src/io translation units can
// be compiled unmodified on a machine without Kokkos, to pin the oracle
// restatement against the real reference step.
//
// Semantics follow the host (Serial/OpenMP) Kokkos backends:
//  - View<T*, T**, T***> are LayoutRight, reference-counted shallow handles;
//  - create_mirror_view of a host view returns the SAME allocation (as host
//    Kokkos does), so host staging code behaves exactly as in a CPU build;
//  - MDRangePolicy iterates row-major (last index fastest);
//  - parallel_reduce overwrites its result arguments with the reduction,
//    sum reducers start at 0, Max at lowest(), Min at max().
// Build with -DFREHG_SHIM_OPENMP to run parallel_for / parallel_reduce over
// OpenMP threads (timing lane); the default is serial (parity lane).
#ifndef FREHG_SHIM_KOKKOS_CORE_HPP
#define FREHG_SHIM_KOKKOS_CORE_HPP

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>
#ifdef FREHG_SHIM_OPENMP
#include <omp.h>
#endif

#define KOKKOS_LAMBDA [=]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_FORCEINLINE_FUNCTION inline

namespace Kokkos {

struct HostSpace;
struct Serial {
  using memory_space = HostSpace;
  using execution_space = Serial;
};
struct HostSpace {
  using memory_space = HostSpace;
  using execution_space = Serial;
};
using DefaultExecutionSpace = Serial;
using DefaultHostExecutionSpace = Serial;
struct LayoutRight {};
struct LayoutLeft {};

inline void initialize(int&, char**) {}
inline void initialize() {}
inline void finalize() {}
inline bool is_initialized() { return true; }
inline void fence() {}
inline void fence(const std::string&) {}

// ---------------------------------------------------------------- View
namespace impl {
template <class D> struct rank_of { static constexpr int value = 0; using type = D; };
template <class D> struct rank_of<D*> {
  static constexpr int value = rank_of<D>::value + 1;
  using type = typename rank_of<D>::type;
};
}  // namespace impl

template <class DataType, class... Props>
class View {
 public:
  static constexpr int Rank = impl::rank_of<DataType>::value;
  using value_type = typename impl::rank_of<DataType>::type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using memory_space = HostSpace;
  using execution_space = Serial;
  using HostMirror = View<DataType, Props...>;

  View() = default;
  explicit View(const std::string& label, std::size_t n0 = 0, std::size_t n1 = 0,
                std::size_t n2 = 0, std::size_t n3 = 0)
      : label_(label) {
    ext_[0] = n0; ext_[1] = n1; ext_[2] = n2; ext_[3] = n3;
    for (int r = Rank; r < 4; ++r) ext_[r] = 1;
    std::size_t n = 1;
    for (int r = 0; r < Rank; ++r) n *= ext_[r];
    owner_ = std::shared_ptr<non_const_value_type[]>(new non_const_value_type[n > 0 ? n : 1]());
    ptr_ = owner_.get();
    span_ = n;
    alloc_ = true;
  }
  // Subview/alias constructor.
  View(const View& base, value_type* ptr, std::size_t n)
      : owner_(base.owner_), ptr_(const_cast<non_const_value_type*>(ptr)), span_(n),
        label_(base.label_), alloc_(base.alloc_) {
    ext_[0] = n; ext_[1] = ext_[2] = ext_[3] = 1;
  }
  template <class D2, class... P2,
            class = std::enable_if_t<!std::is_same_v<View<D2, P2...>, View>>>
  View(const View<D2, P2...>& o)
      : owner_(o.owner_), ptr_(o.ptr_), span_(o.span_), label_(o.label_), alloc_(o.alloc_) {
    for (int r = 0; r < 4; ++r) ext_[r] = o.ext_[r];
  }

  std::size_t extent(int r) const { return r < Rank ? ext_[r] : 1; }
  int extent_int(int r) const { return static_cast<int>(extent(r)); }
  std::size_t size() const { return span_; }
  std::size_t span() const { return span_; }
  value_type* data() const { return ptr_; }
  bool is_allocated() const { return alloc_; }
  const std::string& label() const { return label_; }
  long use_count() const { return owner_.use_count(); }

  template <class I0>
  value_type& operator()(I0 i0) const {
    return ptr_[static_cast<std::size_t>(i0)];
  }
  template <class I0, class I1>
  value_type& operator()(I0 i0, I1 i1) const {
    return ptr_[static_cast<std::size_t>(i0) * ext_[1] + static_cast<std::size_t>(i1)];
  }
  template <class I0, class I1, class I2>
  value_type& operator()(I0 i0, I1 i1, I2 i2) const {
    return ptr_[(static_cast<std::size_t>(i0) * ext_[1] + static_cast<std::size_t>(i1)) *
                    ext_[2] +
                static_cast<std::size_t>(i2)];
  }
  template <class I0>
  value_type& operator[](I0 i0) const {
    return ptr_[static_cast<std::size_t>(i0)];
  }

  template <class D2, class... P2> friend class View;
  std::shared_ptr<non_const_value_type[]> owner_;
  non_const_value_type* ptr_ = nullptr;
  std::size_t span_ = 0;
  std::size_t ext_[4] = {0, 0, 0, 0};
  std::string label_;
  bool alloc_ = false;
};

template <class D, class... P>
View<D, P...> create_mirror_view(const View<D, P...>& v) {
  return v;
}
template <class Space, class D, class... P>
View<D, P...> create_mirror_view(const Space&, const View<D, P...>& v) {
  return v;
}
template <class D, class... P>
View<D, P...> create_mirror(const View<D, P...>& v) {
  View<D, P...> out(v.label(), v.extent(0), v.extent(1), v.extent(2));
  for (std::size_t n = 0; n < v.span(); ++n) out.data()[n] = v.data()[n];
  return out;
}
template <class D, class... P>
View<D, P...> create_mirror_view_and_copy(const HostSpace&, const View<D, P...>& v) {
  return v;
}

template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (static_cast<const void*>(dst.data()) == static_cast<const void*>(src.data())) return;
  const std::size_t n = std::min(dst.span(), src.span());
  for (std::size_t k = 0; k < n; ++k) dst.data()[k] = src.data()[k];
}
template <class D1, class... P1, class T,
          class = std::enable_if_t<std::is_arithmetic_v<T>>>
void deep_copy(const View<D1, P1...>& dst, const T& value) {
  using V = typename View<D1, P1...>::non_const_value_type;
  for (std::size_t k = 0; k < dst.span(); ++k) dst.data()[k] = static_cast<V>(value);
}
template <class Space, class D1, class... P1, class Src>
void deep_copy(const Space&, const View<D1, P1...>& dst, const Src& src) {
  deep_copy(dst, src);
}

struct ALL_t {};
constexpr ALL_t ALL{};
template <class A, class B> using pair = std::pair<A, B>;
template <class D, class... P, class A, class B>
View<D, P...> subview(const View<D, P...>& v, const std::pair<A, B>& range) {
  const std::size_t b = static_cast<std::size_t>(range.first);
  const std::size_t e = static_cast<std::size_t>(range.second);
  return View<D, P...>(v, v.data() + b, e - b);
}

// ---------------------------------------------------------------- policies
template <unsigned N> struct Rank { static constexpr unsigned value = N; };
template <class T> struct IndexType { using type = T; };

namespace impl {
template <class... Args> struct rank_in;
template <> struct rank_in<> { static constexpr int value = 0; };
template <unsigned N, class... Rest> struct rank_in<Rank<N>, Rest...> {
  static constexpr int value = static_cast<int>(N);
};
template <class A, class... Rest> struct rank_in<A, Rest...> {
  static constexpr int value = rank_in<Rest...>::value;
};
}  // namespace impl

template <class... Args>
struct MDRangePolicy {
  static constexpr int rank = impl::rank_in<Args...>::value;
  long long lo[3] = {0, 0, 0};
  long long hi[3] = {0, 0, 0};
  template <class LT, std::size_t LN, class UT, std::size_t UN>
  MDRangePolicy(const LT (&lower)[LN], const UT (&upper)[UN]) {
    static_assert(LN == UN, "MDRangePolicy bounds rank mismatch");
    for (std::size_t r = 0; r < LN; ++r) {
      lo[r] = static_cast<long long>(lower[r]);
      hi[r] = static_cast<long long>(upper[r]);
    }
  }
};

template <class... Args>
struct RangePolicy {
  long long lo = 0, hi = 0;
  template <class B, class E>
  RangePolicy(B b, E e) : lo(static_cast<long long>(b)), hi(static_cast<long long>(e)) {}
};

// ---------------------------------------------------------------- reducers
template <class T>
struct Max {
  using value_type = T;
  T& ref;
  explicit Max(T& r) : ref(r) {}
  static T init() { return std::numeric_limits<T>::lowest(); }
  static void join(T& a, const T& b) { if (b > a) a = b; }
};
template <class T>
struct Min {
  using value_type = T;
  T& ref;
  explicit Min(T& r) : ref(r) {}
  static T init() { return std::numeric_limits<T>::max(); }
  static void join(T& a, const T& b) { if (b < a) a = b; }
};
template <class T>
struct Sum {
  using value_type = T;
  T& ref;
  explicit Sum(T& r) : ref(r) {}
  static T init() { return T(0); }
  static void join(T& a, const T& b) { a += b; }
};

namespace impl {
template <class A> struct is_reducer : std::false_type {};
template <class T> struct is_reducer<Max<T>> : std::true_type {};
template <class T> struct is_reducer<Min<T>> : std::true_type {};
template <class T> struct is_reducer<Sum<T>> : std::true_type {};
template <class A> auto make_reducer(A& a) {
  using D = std::remove_cv_t<A>;
  if constexpr (is_reducer<D>::value) {
    return a;
  } else {
    return Sum<D>(a);
  }
}

template <class F>
void for_range(long long lo, long long hi, const F& body) {
#ifdef FREHG_SHIM_OPENMP
#pragma omp parallel for schedule(static)
  for (long long n = lo; n < hi; ++n) body(n);
#else
  for (long long n = lo; n < hi; ++n) body(n);
#endif
}

template <class Policy, class F>
void md_for(const Policy& p, const F& f) {
  constexpr int R = Policy::rank;
  if constexpr (R == 2) {
    const long long n0 = p.hi[0] - p.lo[0], n1 = p.hi[1] - p.lo[1];
    if (n0 <= 0 || n1 <= 0) return;
    for_range(0, n0 * n1, [&](long long n) { f(p.lo[0] + n / n1, p.lo[1] + n % n1); });
  } else {
    const long long n0 = p.hi[0] - p.lo[0], n1 = p.hi[1] - p.lo[1], n2 = p.hi[2] - p.lo[2];
    if (n0 <= 0 || n1 <= 0 || n2 <= 0) return;
    for_range(0, n0 * n1 * n2, [&](long long n) {
      f(p.lo[0] + n / (n1 * n2), p.lo[1] + (n / n2) % n1, p.lo[2] + n % n2);
    });
  }
}
}  // namespace impl

template <class... PA, class F>
void parallel_for(const std::string&, const MDRangePolicy<PA...>& p, const F& f) {
  constexpr int R = MDRangePolicy<PA...>::rank;
  if constexpr (R == 2) {
    impl::md_for(p, [&](long long a, long long b) { f(a, b); });
  } else {
    impl::md_for(p, [&](long long a, long long b, long long c) { f(a, b, c); });
  }
}
template <class... PA, class F>
void parallel_for(const MDRangePolicy<PA...>& p, const F& f) {
  parallel_for(std::string(), p, f);
}
template <class... PA, class F>
void parallel_for(const std::string&, const RangePolicy<PA...>& p, const F& f) {
  impl::for_range(p.lo, p.hi, [&](long long n) { f(n); });
}
template <class... PA, class F>
void parallel_for(const RangePolicy<PA...>& p, const F& f) {
  impl::for_range(p.lo, p.hi, [&](long long n) { f(n); });
}
template <class I, class F, class = std::enable_if_t<std::is_integral_v<I>>>
void parallel_for(const std::string&, I n, const F& f) {
  impl::for_range(0, static_cast<long long>(n), [&](long long k) { f(k); });
}

namespace impl {
template <class Tuple, std::size_t... Is>
auto init_accs(const Tuple& reds, std::index_sequence<Is...>) {
  return std::make_tuple(std::tuple_element_t<Is, Tuple>::init()...);
}
template <class Tuple, class Accs, std::size_t... Is>
void join_accs(Accs& into, const Accs& from, std::index_sequence<Is...>) {
  (std::tuple_element_t<Is, Tuple>::join(std::get<Is>(into), std::get<Is>(from)), ...);
}
template <class Tuple, class Accs, std::size_t... Is>
void store_accs(Tuple& reds, const Accs& accs, std::index_sequence<Is...>) {
  ((std::get<Is>(reds).ref = std::get<Is>(accs)), ...);
}

// Runs body(flat index, accs&) over [0, n) and joins the accumulators.
template <class Tuple, class Body>
void reduce_flat(long long n, Tuple& reds, const Body& body) {
  constexpr std::size_t NR = std::tuple_size_v<Tuple>;
  using Seq = std::make_index_sequence<NR>;
  auto total = init_accs(reds, Seq{});
#ifdef FREHG_SHIM_OPENMP
  const int nt = omp_get_max_threads();
  std::vector<decltype(total)> part(static_cast<std::size_t>(nt), total);
#pragma omp parallel num_threads(nt)
  {
    auto& mine = part[static_cast<std::size_t>(omp_get_thread_num())];
#pragma omp for schedule(static)
    for (long long k = 0; k < n; ++k) body(k, mine);
  }
  for (auto& p : part) join_accs<Tuple>(total, p, Seq{});
#else
  for (long long k = 0; k < n; ++k) body(k, total);
#endif
  store_accs(reds, total, Seq{});
}
}  // namespace impl

template <class... PA, class F, class... R>
void parallel_reduce(const std::string&, const MDRangePolicy<PA...>& p, const F& f,
                     R&&... results) {
  auto reds = std::make_tuple(impl::make_reducer(results)...);
  constexpr int RK = MDRangePolicy<PA...>::rank;
  const long long n0 = p.hi[0] - p.lo[0], n1 = p.hi[1] - p.lo[1];
  const long long n2 = (RK == 3) ? p.hi[2] - p.lo[2] : 1;
  const long long n = (n0 > 0 && n1 > 0 && n2 > 0) ? n0 * n1 * n2 : 0;
  impl::reduce_flat(n, reds, [&](long long k, auto& accs) {
    if constexpr (RK == 2) {
      std::apply([&](auto&... a) { f(p.lo[0] + k / n1, p.lo[1] + k % n1, a...); }, accs);
    } else {
      std::apply(
          [&](auto&... a) {
            f(p.lo[0] + k / (n1 * n2), p.lo[1] + (k / n2) % n1, p.lo[2] + k % n2, a...);
          },
          accs);
    }
  });
}
template <class... PA, class F, class... R>
void parallel_reduce(const std::string&, const RangePolicy<PA...>& p, const F& f,
                     R&&... results) {
  auto reds = std::make_tuple(impl::make_reducer(results)...);
  impl::reduce_flat(p.hi - p.lo, reds, [&](long long k, auto& accs) {
    std::apply([&](auto&... a) { f(p.lo + k, a...); }, accs);
  });
}

// ---------------------------------------------------------------- atomics, math
template <class T>
inline void atomic_add(T* p, T v) {
#ifdef FREHG_SHIM_OPENMP
#pragma omp atomic
#endif
  *p += v;
}

using std::abs;
using std::cbrt;
using std::cos;
using std::exp;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::isfinite;
using std::isnan;
using std::log;
using std::log10;
using std::pow;
using std::sin;
using std::sqrt;
using std::tanh;
using std::atan;
using std::atan2;
using std::ceil;
using std::min;
using std::max;

}  // namespace Kokkos

#endif  // FREHG_SHIM_KOKKOS_CORE_HPP
