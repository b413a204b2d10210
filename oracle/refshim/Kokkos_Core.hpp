// Single-rank, host-only stand-in for the subset of the Kokkos 4.0.01 API that
// the imexlb proxy apps use (tgv/src/lbm.hpp, lid_driven_cavity/src/lbm.hpp,
// sphere/src/lbm.hpp and their .cpp files).  It exists so that the reference's
// own solver sources compile with g++ on the CPU and can serve as the oracle
// that pins this project's restatement.  It is test infrastructure only.
//
// Semantics restated from Kokkos' published behaviour:
//   * View<T****, Space>: reference-counted, zero-initialised on allocation,
//     LayoutLeft (first index fastest) for CudaUVMSpace (the Cuda execution
//     space's layout) and LayoutRight for host spaces, unless a layout is given.
//   * subview(): strided alias; an integer argument drops that rank.
//   * deep_copy(dst, src): element-wise copy between equal extents.
//   * parallel_for(MDRangePolicy<Rank<N>>): every index tuple once; this shim
//     iterates with the first index fastest (the Cuda backend's default
//     Iterate::Left), OpenMP-parallel over the outermost index.
//   * TeamPolicy / TeamThreadRange / ThreadVectorRange: sequential loops, the
//     Serial backend's order; nested parallel_reduce sums in index order
//     starting from a value-initialised (zero) accumulator.
//   * parallel_reduce with Max/Min reducers: identity -DBL_MAX / +DBL_MAX.
#pragma once

#include <array>
#include <cfloat>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>

#define KOKKOS_CLASS_LAMBDA [=]
#define KOKKOS_LAMBDA [=]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION

namespace Kokkos {

struct HostSpace {};
struct CudaUVMSpace {};
struct CudaHostPinnedSpace {};
struct LayoutLeft {};
struct LayoutRight {};

struct ALL_t {};
inline constexpr ALL_t ALL{};

namespace shim {

[[noreturn]] inline void fail(const char* what) {
  std::fprintf(stderr, "refshim: %s\n", what);
  std::abort();
}

template <class D> struct data_traits {
  using value_type = D;
  static constexpr int rank = 0;
};
template <class D> struct data_traits<D*> {
  using value_type = typename data_traits<D>::value_type;
  static constexpr int rank = data_traits<D>::rank + 1;
};

// Layout selection: explicit layout wins; otherwise CudaUVMSpace -> Left.
template <class... P> struct is_left : std::false_type {};
template <class... P> struct is_left<LayoutLeft, P...> : std::true_type {};
template <class... P> struct is_left<LayoutRight, P...> : std::false_type {};
template <class... P> struct is_left<CudaUVMSpace, P...> : std::true_type {};
template <class H, class... P> struct is_left<H, P...> : is_left<P...> {};

template <class A> struct keeps_rank : std::true_type {};
template <> struct keeps_rank<int> : std::false_type {};
template <> struct keeps_rank<long> : std::false_type {};

}  // namespace shim

// Rank-R strided view over T.  All View<> types derive from this.
template <class T, int R>
class ViewBase {
 public:
  std::shared_ptr<T> mem_;
  T* ptr_ = nullptr;
  std::array<long, R> ext_{};
  std::array<long, R> str_{};
  std::string label_;

  template <class... I>
  T& operator()(I... idx) const {
    static_assert(sizeof...(I) == R, "wrong number of view indices");
    const long ix[R] = {static_cast<long>(idx)...};
    long off = 0;
    for (int d = 0; d < R; ++d) {
#ifndef REFSHIM_NO_BOUNDS_CHECK
      if (ix[d] < 0 || ix[d] >= ext_[d]) {
        std::fprintf(stderr, "refshim: view '%s' index %ld out of [0,%ld) in dim %d\n",
                     label_.c_str(), ix[d], ext_[d], d);
        std::abort();
      }
#endif
      off += ix[d] * str_[d];
    }
    return ptr_[off];
  }
  T* data() const { return ptr_; }
  size_t size() const {
    size_t n = 1;
    for (int d = 0; d < R; ++d) n *= static_cast<size_t>(ext_[d]);
    return n;
  }
  size_t extent(int d) const { return static_cast<size_t>(ext_[d]); }
  const std::string& label() const { return label_; }
};

template <class D, class... P>
class View : public ViewBase<typename shim::data_traits<D>::value_type, shim::data_traits<D>::rank> {
  using T = typename shim::data_traits<D>::value_type;
  static constexpr int R = shim::data_traits<D>::rank;
  using Base = ViewBase<T, R>;

 public:
  using value_type = T;
  View() = default;
  View(const Base& b) : Base(b) {}
  View& operator=(const Base& b) {
    Base::operator=(b);
    return *this;
  }
  template <class... N, typename = std::enable_if_t<sizeof...(N) == R>>
  View(const std::string& label, N... n) {
    const long e[R] = {static_cast<long>(n)...};
    long total = 1;
    for (int d = 0; d < R; ++d) {
      if (e[d] < 0) shim::fail("negative extent");
      this->ext_[d] = e[d];
      total *= e[d];
    }
    const bool left = shim::is_left<P...>::value;
    long s = 1;
    if (left) {
      for (int d = 0; d < R; ++d) { this->str_[d] = s; s *= e[d]; }
    } else {
      for (int d = R - 1; d >= 0; --d) { this->str_[d] = s; s *= e[d]; }
    }
    T* p = static_cast<T*>(std::calloc(total > 0 ? total : 1, sizeof(T)));
    if (!p) shim::fail("allocation failed");
    this->mem_ = std::shared_ptr<T>(p, [](T* q) { std::free(q); });
    this->ptr_ = p;
    this->label_ = label;
  }
};

// subview(view, ALL | pair<int,int> | int ...)
namespace shim {
template <class T, int R, int RO>
inline void sub_arg(const ViewBase<T, R>& v, ViewBase<T, RO>& o, int d, int& od, long& off, ALL_t) {
  o.ext_[od] = v.ext_[d];
  o.str_[od] = v.str_[d];
  ++od;
  (void)off;
}
template <class T, int R, int RO, class A, class B>
inline void sub_arg(const ViewBase<T, R>& v, ViewBase<T, RO>& o, int d, int& od, long& off,
                    const std::pair<A, B>& p) {
  if (p.first < 0 || p.second > v.ext_[d] || p.first > p.second) fail("subview range out of bounds");
  o.ext_[od] = static_cast<long>(p.second - p.first);
  o.str_[od] = v.str_[d];
  off += static_cast<long>(p.first) * v.str_[d];
  ++od;
}
template <class T, int R, int RO>
inline void sub_arg(const ViewBase<T, R>& v, ViewBase<T, RO>&, int d, int&, long& off, long i) {
  if (i < 0 || i >= v.ext_[d]) fail("subview index out of bounds");
  off += i * v.str_[d];
}
template <class A> struct arg_rank : std::integral_constant<int, 1> {};
template <> struct arg_rank<int> : std::integral_constant<int, 0> {};
template <> struct arg_rank<long> : std::integral_constant<int, 0> {};
}  // namespace shim

template <class T, int R, class... A>
auto subview(const ViewBase<T, R>& v, A... args) {
  static_assert(sizeof...(A) == R, "subview needs one argument per rank");
  constexpr int RO = (0 + ... + shim::arg_rank<std::decay_t<A>>::value);
  ViewBase<T, RO> o;
  o.mem_ = v.mem_;
  o.label_ = v.label_;
  long off = 0;
  int od = 0;
  int d = 0;
  (shim::sub_arg(v, o, d++, od, off, args), ...);
  o.ptr_ = v.ptr_ + off;
  return o;
}

template <class T, int R1, int R2>
void deep_copy(const ViewBase<T, R1>& dst, const ViewBase<T, R2>& src) {
  static_assert(R1 == R2, "deep_copy rank mismatch");
  for (int d = 0; d < R1; ++d)
    if (dst.ext_[d] != src.ext_[d]) shim::fail("deep_copy extent mismatch");
  const size_t n = dst.size();
  std::array<long, R1> ix{};
  for (size_t c = 0; c < n; ++c) {
    long od = 0, os = 0;
    for (int d = 0; d < R1; ++d) {
      od += ix[d] * dst.str_[d];
      os += ix[d] * src.str_[d];
    }
    dst.ptr_[od] = src.ptr_[os];
    for (int d = 0; d < R1; ++d) {
      if (++ix[d] < dst.ext_[d]) break;
      ix[d] = 0;
    }
  }
}

// ---------------------------------------------------------------- policies
template <int N> struct Rank {};
template <class... P> struct RangePolicy {
  long b = 0, e = 0;
  RangePolicy() = default;
  RangePolicy(long b_, long e_) : b(b_), e(e_) {}
};

template <class... P> struct MDRangePolicy;
template <int N> struct MDRangePolicy<Rank<N>> {
  std::array<long, N> lo{}, hi{};
  MDRangePolicy(std::initializer_list<long> l, std::initializer_list<long> h) {
    if (static_cast<int>(l.size()) != N || static_cast<int>(h.size()) != N) shim::fail("MDRange bounds");
    int d = 0;
    for (long x : l) lo[d++] = x;
    d = 0;
    for (long x : h) hi[d++] = x;
  }
};

struct AUTO_t {};
inline constexpr AUTO_t AUTO{};

struct TeamMember {
  long lr = 0, ls = 0;
  long league_rank() const { return lr; }
  long league_size() const { return ls; }
  int team_rank() const { return 0; }
  int team_size() const { return 1; }
};

template <class... P> struct TeamPolicy {
  using member_type = TeamMember;
  long league = 0;
  TeamPolicy(long l, AUTO_t) : league(l) {}
  TeamPolicy(long l, int) : league(l) {}
};

struct NestedRange {
  long b = 0, e = 0;
};
inline NestedRange TeamThreadRange(const TeamMember&, long n) { return {0, n}; }
inline NestedRange TeamThreadRange(const TeamMember&, long b, long e) { return {b, e}; }
inline NestedRange ThreadVectorRange(const TeamMember&, long n) { return {0, n}; }
inline NestedRange ThreadVectorRange(const TeamMember&, long b, long e) { return {b, e}; }

template <class T> struct Max {
  T& ref;
  explicit Max(T& r) : ref(r) {}
};
template <class T> struct Min {
  T& ref;
  explicit Min(T& r) : ref(r) {}
};

namespace shim {
template <int N, class F, class... X>
inline void md_call(const F& f, const std::array<long, N>& ix, X&... extra) {
  if constexpr (N == 1) f(static_cast<int>(ix[0]), extra...);
  if constexpr (N == 2) f(static_cast<int>(ix[0]), static_cast<int>(ix[1]), extra...);
  if constexpr (N == 3)
    f(static_cast<int>(ix[0]), static_cast<int>(ix[1]), static_cast<int>(ix[2]), extra...);
  if constexpr (N == 4)
    f(static_cast<int>(ix[0]), static_cast<int>(ix[1]), static_cast<int>(ix[2]),
      static_cast<int>(ix[3]), extra...);
}
// Visit every index tuple of the box for a fixed outermost index, first index fastest.
template <int N, class F>
inline void md_inner(const MDRangePolicy<Rank<N>>& p, long outer, const F& visit) {
  std::array<long, N> ix = p.lo;
  ix[N - 1] = outer;
  for (int d = 0; d < N - 1; ++d)
    if (p.lo[d] >= p.hi[d]) return;
  while (true) {
    visit(ix);
    int d = 0;
    for (; d < N - 1; ++d) {
      if (++ix[d] < p.hi[d]) break;
      ix[d] = p.lo[d];
    }
    if (d == N - 1) return;
  }
}
}  // namespace shim

template <int N, class F>
void parallel_for(const std::string&, const MDRangePolicy<Rank<N>>& p, const F& f) {
  const long lo = p.lo[N - 1], hi = p.hi[N - 1];
#pragma omp parallel for schedule(static)
  for (long o = lo; o < hi; ++o)
    shim::md_inner<N>(p, o, [&](const std::array<long, N>& ix) { shim::md_call<N>(f, ix); });
}

template <class F>
void parallel_for(const std::string&, const RangePolicy<>& p, const F& f) {
  for (long i = p.b; i < p.e; ++i) f(static_cast<int>(i));
}

template <class... P, class F>
void parallel_for(const std::string&, const TeamPolicy<P...>& p, const F& f) {
#pragma omp parallel for schedule(static)
  for (long l = 0; l < p.league; ++l) {
    TeamMember m;
    m.lr = l;
    m.ls = p.league;
    f(m);
  }
}

template <class F>
void parallel_for(const NestedRange& r, const F& f) {
  for (long i = r.b; i < r.e; ++i) f(static_cast<int>(i));
}

template <class F, class T>
void parallel_reduce(const NestedRange& r, const F& f, T& result) {
  T acc = T();
  for (long i = r.b; i < r.e; ++i) f(static_cast<int>(i), acc);
  result = acc;
}

template <int N, class F, class T>
void parallel_reduce(const std::string&, const MDRangePolicy<Rank<N>>& p, const F& f, Max<T> r) {
  T acc = -DBL_MAX;
  for (long o = p.lo[N - 1]; o < p.hi[N - 1]; ++o)
    shim::md_inner<N>(p, o, [&](const std::array<long, N>& ix) { shim::md_call<N>(f, ix, acc); });
  r.ref = acc;
}

template <int N, class F, class T>
void parallel_reduce(const std::string&, const MDRangePolicy<Rank<N>>& p, const F& f, Min<T> r) {
  T acc = DBL_MAX;
  for (long o = p.lo[N - 1]; o < p.hi[N - 1]; ++o)
    shim::md_inner<N>(p, o, [&](const std::array<long, N>& ix) { shim::md_call<N>(f, ix, acc); });
  r.ref = acc;
}

inline void fence() {}
inline void initialize(int&, char**) {}
inline void initialize() {}
inline void finalize() {}

}  // namespace Kokkos
