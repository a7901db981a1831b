// Kokkos_Core.hpp -- TEST INFRASTRUCTURE ONLY.
//
// A minimal host-only stand-in for the subset of the Kokkos programming model
// that the Jet reference sources use (reference src/*.hpp, src/jet*.cpp,
// app/*.cpp).  It exists so that the UNMODIFIED reference sources can be
// compiled here with g++ into the CPU checker and CPU baseline under
// oracle/_ref/ (oracle/ref.mk); Kokkos itself is not installed.
//
// Execution spaces:
//   * Serial  -- every parallel construct runs in index order on one thread,
//                atomics are plain read-modify-writes.  This is the reference's
//                own single-thread semantics (jet_serial).
//   * OpenMP  -- (when compiled with -fopenmp) range and team loops are split
//                over OpenMP threads, reductions and scans run as two passes,
//                atomics are GCC __atomic builtins (jet_host).
// Teams always have one thread (team_size() == 1): nested TeamThreadRange
// loops run in order inside the team, which is one of the executions Kokkos
// allows on a host back end.
//
// Randomness: Random_XorShift64_Pool is a pool of xorshift64* generators
// (S. Vigna, "An experimental exploration of Marsaglia's xorshift generators,
// scrambled", 2016), one state per thread, seeded by splitmix64.  The reference
// seeds its pool from the wall clock (src/contract.hpp:503); when the
// environment variable JET_SEED is set, that value replaces the constructor's
// seed so that a run can be repeated.
//
// pod_hash is MurmurHash3_x86_32 (Austin Appleby, public domain) over the
// key's bytes with seed 0, which is the hash Kokkos::pod_hash computes.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <limits>
#include <math.h>
#include <memory>
#include <stdlib.h>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION

namespace Kokkos {

// ------------------------------------------------------------------ spaces
struct HostSpace {
    using memory_space = HostSpace;
};
// Pinned host memory is ordinary host memory here.
using SharedHostPinnedSpace = HostSpace;

template <class Exec, class Mem>
struct Device {
    using execution_space = Exec;
    using memory_space = Mem;
    using device_type = Device<Exec, Mem>;
};

struct Serial {
    using execution_space = Serial;
    using memory_space = HostSpace;
    using device_type = Device<Serial, HostSpace>;
    static constexpr bool threaded = false;
    int concurrency() const { return 1; }
    void fence() const {}
};

#ifdef _OPENMP
struct OpenMP {
    using execution_space = OpenMP;
    using memory_space = HostSpace;
    using device_type = Device<OpenMP, HostSpace>;
    static constexpr bool threaded = true;
    int concurrency() const { return omp_get_max_threads(); }
    void fence() const {}
};
using DefaultHostExecutionSpace = OpenMP;
#else
using DefaultHostExecutionSpace = Serial;
#endif
using DefaultExecutionSpace = DefaultHostExecutionSpace;

inline void initialize() {}
inline void initialize(int&, char**) {}
inline void finalize() {}
inline void fence() {}
inline void fence(const std::string&) {}

namespace impl {
// Finds the execution space among a View's or policy's template arguments.
template <class T, class = void>
struct exec_of { using type = void; };
template <class T>
struct exec_of<T, std::void_t<typename T::execution_space>> { using type = typename T::execution_space; };

template <class... P>
struct first_exec;
template <>
struct first_exec<> { using type = DefaultExecutionSpace; };
template <class H, class... T>
struct first_exec<H, T...> {
    using h = typename exec_of<H>::type;
    using type = std::conditional_t<std::is_void_v<h>, typename first_exec<T...>::type, h>;
};

template <class... P>
inline constexpr bool threaded_v = first_exec<P...>::type::threaded;

inline int thread_id() {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}
inline int max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Argument types of a lambda's (non-template) call operator.
template <class F>
struct call_traits : call_traits<decltype(&F::operator())> {};
template <class C, class R, class... A>
struct call_traits<R (C::*)(A...) const> {
    template <size_t i>
    using arg = std::tuple_element_t<i, std::tuple<A...>>;
};
template <class C, class R, class... A>
struct call_traits<R (C::*)(A...)> {
    template <size_t i>
    using arg = std::tuple_element_t<i, std::tuple<A...>>;
};
template <class F, size_t i>
using arg_value_t = std::remove_cv_t<std::remove_reference_t<typename call_traits<F>::template arg<i>>>;
}  // namespace impl

// ------------------------------------------------------------------ views
struct ViewAllocateWithoutInitializing {
    std::string label;
    ViewAllocateWithoutInitializing(const std::string& l = "") : label(l) {}
};
struct WithoutInitializing_t {};
constexpr WithoutInitializing_t WithoutInitializing{};
inline ViewAllocateWithoutInitializing view_alloc(WithoutInitializing_t, const std::string& l) {
    return ViewAllocateWithoutInitializing(l);
}
inline ViewAllocateWithoutInitializing view_alloc(const std::string& l, WithoutInitializing_t) {
    return ViewAllocateWithoutInitializing(l);
}

struct ALL_t {};
constexpr ALL_t ALL{};

namespace impl {
template <class D>
struct data_traits {
    using value_type = D;
    static constexpr int rank = 0;
};
template <class D>
struct data_traits<D*> {
    using value_type = typename data_traits<D>::value_type;
    static constexpr int rank = 1 + data_traits<D>::rank;
};
template <class D>
struct data_traits<D[]> {
    using value_type = typename data_traits<D>::value_type;
    static constexpr int rank = 1 + data_traits<D>::rank;
};
}  // namespace impl

template <class DataType, class... Props>
class View {
public:
    using traits = impl::data_traits<DataType>;
    using value_type = typename traits::value_type;
    using non_const_value_type = std::remove_const_t<value_type>;
    using const_value_type = const non_const_value_type;
    using pointer_type = value_type*;
    using reference_type = value_type&;
    static constexpr int rank = traits::rank;
    using execution_space = typename impl::first_exec<Props...>::type;
    using memory_space = HostSpace;
    using device_type = Device<execution_space, memory_space>;
    using HostMirror = View<DataType, Props...>;
    using non_const_type = View<typename std::conditional_t<
        rank == 0, non_const_value_type,
        std::conditional_t<rank == 1, non_const_value_type*, non_const_value_type**>>, Props...>;
    using size_type = size_t;

    std::shared_ptr<void> owner_;
    value_type* ptr_ = nullptr;
    size_t n0_ = 0, n1_ = 1;
    std::string label_;

    View() = default;

    explicit View(const std::string& label, size_t n0 = 0, size_t n1 = 0) { alloc(label, n0, n1, true); }
    explicit View(const char* label, size_t n0 = 0, size_t n1 = 0) { alloc(label, n0, n1, true); }
    View(const ViewAllocateWithoutInitializing& a, size_t n0 = 0, size_t n1 = 0) { alloc(a.label, n0, n1, false); }
    // Unmanaged view over caller memory.
    View(value_type* p, size_t n0 = 1, size_t n1 = 1) : ptr_(p), n0_(rank >= 1 ? n0 : 1), n1_(rank >= 2 ? n1 : 1) {}

    // Shallow copies between views of the same element type and rank, whatever
    // their space arguments (everything lives in host memory here).
    template <class D2, class... P2,
              class = std::enable_if_t<(impl::data_traits<D2>::rank == rank) &&
                                       std::is_convertible_v<typename impl::data_traits<D2>::value_type*, value_type*>>>
    View(const View<D2, P2...>& o) : owner_(o.owner_), ptr_(o.ptr_), n0_(o.n0_), n1_(o.n1_), label_(o.label_) {}

    void alloc(const std::string& label, size_t n0, size_t n1, bool zero) {
        label_ = label;
        n0_ = rank >= 1 ? n0 : 1;
        n1_ = rank >= 2 ? n1 : 1;
        size_t cnt = n0_ * n1_;
        size_t bytes = std::max<size_t>(cnt, 1) * sizeof(non_const_value_type);
        void* p = std::malloc(bytes);
        if (!p) {
            std::cerr << "Kokkos shim: allocation of " << bytes << " bytes for '" << label << "' failed" << std::endl;
            std::abort();
        }
        if (zero) fill_bytes_zero(static_cast<char*>(p), bytes);
        owner_ = std::shared_ptr<void>(p, [](void* q) { std::free(q); });
        ptr_ = static_cast<value_type*>(p);
    }
    static void fill_bytes_zero(char* p, size_t bytes) {
#ifdef _OPENMP
        if (bytes >= (size_t(1) << 22)) {
            const int64_t chunk = 1 << 20;
            const int64_t nc = (int64_t)((bytes + chunk - 1) / chunk);
#pragma omp parallel for schedule(static)
            for (int64_t c = 0; c < nc; c++) {
                size_t b = (size_t)c * chunk, e = std::min(bytes, b + (size_t)chunk);
                std::memset(p + b, 0, e - b);
            }
            return;
        }
#endif
        std::memset(p, 0, bytes);
    }

    value_type* data() const { return ptr_; }
    size_t extent(int r) const { return r == 0 ? (rank >= 1 ? n0_ : 1) : (rank >= 2 ? n1_ : 1); }
    int64_t extent_int(int r) const { return (int64_t)extent(r); }
    size_t size() const { return rank == 0 ? 1 : n0_ * n1_; }
    size_t span() const { return size(); }
    bool is_allocated() const { return ptr_ != nullptr; }
    const std::string& label() const { return label_; }
    int use_count() const { return (int)owner_.use_count(); }

    value_type& operator()() const { return ptr_[0]; }
    template <class I>
    value_type& operator()(I i) const { return ptr_[(size_t)i]; }
    template <class I, class J>
    value_type& operator()(I i, J j) const { return ptr_[(size_t)i * n1_ + (size_t)j]; }
    template <class I>
    value_type& operator[](I i) const { return ptr_[(size_t)i]; }
};

template <class V>
inline std::enable_if_t<V::rank == 1, V> subview_range(const V& v, size_t b, size_t e) {
    V out(v);
    out.ptr_ = v.ptr_ + b;
    out.n0_ = e - b;
    return out;
}
template <class D, class... P, class A, class B>
View<D, P...> subview(const View<D, P...>& v, std::pair<A, B> r) {
    return subview_range(v, (size_t)r.first, (size_t)r.second);
}
// A single element of a rank-1 view as a rank-0 view.
template <class D, class... P, class I, class = std::enable_if_t<std::is_integral_v<I>>>
View<typename View<D, P...>::value_type, P...> subview(const View<D, P...>& v, I i) {
    View<typename View<D, P...>::value_type, P...> out;
    out.owner_ = v.owner_;
    out.ptr_ = v.ptr_ + (size_t)i;
    out.n0_ = 1;
    out.n1_ = 1;
    out.label_ = v.label_;
    return out;
}
// One row of a rank-2 view.
template <class D, class... P, class I, class = std::enable_if_t<std::is_integral_v<I>>>
View<typename View<D, P...>::value_type*, P...> subview(const View<D, P...>& v, I i, ALL_t) {
    View<typename View<D, P...>::value_type*, P...> out;
    out.owner_ = v.owner_;
    out.ptr_ = v.ptr_ + (size_t)i * v.n1_;
    out.n0_ = v.n1_;
    out.label_ = v.label_;
    return out;
}

// ------------------------------------------------------------------ deep_copy
namespace impl {
template <class T>
struct is_view : std::false_type {};
template <class D, class... P>
struct is_view<View<D, P...>> : std::true_type {};

template <class T, class U>
void fill(T* p, size_t n, const U& v) {
#ifdef _OPENMP
    if (n >= (size_t(1) << 16)) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) p[i] = (T)v;
        return;
    }
#endif
    for (size_t i = 0; i < n; i++) p[i] = (T)v;
}
template <class T>
void copy(T* d, const T* s, size_t n) {
    if (d == s || n == 0) return;
#ifdef _OPENMP
    if (n * sizeof(T) >= (size_t(1) << 22)) {
        const int64_t chunk = (1 << 20) / (int64_t)sizeof(T) + 1;
        const int64_t nc = ((int64_t)n + chunk - 1) / chunk;
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < nc; c++) {
            int64_t b = c * chunk, e = std::min<int64_t>((int64_t)n, b + chunk);
            std::memmove(d + b, s + b, (size_t)(e - b) * sizeof(T));
        }
        return;
    }
#endif
    std::memmove(d, s, n * sizeof(T));
}
}  // namespace impl

template <class D, class... P, class S, std::enable_if_t<!impl::is_view<S>::value, int> = 0>
void deep_copy(const View<D, P...>& dst, const S& value) {
    impl::fill(dst.data(), dst.size(), value);
}
template <class D, class... P, class D2, class... P2>
void deep_copy(const View<D, P...>& dst, const View<D2, P2...>& src) {
    if (dst.size() != src.size()) {
        std::cerr << "Kokkos shim: deep_copy extents differ (" << dst.size() << " vs " << src.size() << ")" << std::endl;
        std::abort();
    }
    impl::copy(dst.data(), (const typename View<D, P...>::non_const_value_type*)src.data(), dst.size());
}
// Scalar <- rank-0 view.
template <class S, class D, class... P, std::enable_if_t<!impl::is_view<S>::value, int> = 0>
void deep_copy(S& dst, const View<D, P...>& src) {
    dst = src();
}
template <class E, class A, class B,
          class = std::enable_if_t<!std::is_void_v<typename impl::exec_of<E>::type> && !impl::is_view<E>::value>>
void deep_copy(const E&, A&& a, const B& b) {
    deep_copy(std::forward<A>(a), b);
}

template <class V>
V create_mirror_view(const V& v) {
    return v;
}
template <class S, class V>
V create_mirror_view(const S&, const V& v) {
    return v;
}
template <class S, class V>
V create_mirror_view_and_copy(const S&, const V& v) {
    return v;
}
template <class V>
V create_mirror(const V& v) {
    V out(ViewAllocateWithoutInitializing(v.label()), v.extent(0), V::rank >= 2 ? v.extent(1) : 0);
    impl::copy(out.data(), v.data(), v.size());
    return out;
}

// ------------------------------------------------------------------ policies
struct Dynamic {};
struct Static {};
template <class S>
struct Schedule {
    using schedule = S;
};
struct AUTO_t {};
constexpr AUTO_t AUTO{};

namespace impl {
template <class... P>
struct is_dynamic : std::false_type {};
template <class H, class... T>
struct is_dynamic<H, T...> : is_dynamic<T...> {};
template <class... T>
struct is_dynamic<Schedule<Dynamic>, T...> : std::true_type {};
}  // namespace impl

template <class... Props>
struct RangePolicy {
    using execution_space = typename impl::first_exec<Props...>::type;
    static constexpr bool threaded = execution_space::threaded;
    static constexpr bool dynamic = impl::is_dynamic<Props...>::value;
    int64_t begin_ = 0, end_ = 0;
    RangePolicy() = default;
    template <class A, class B>
    RangePolicy(A b, B e) : begin_((int64_t)b), end_((int64_t)e) {}
    template <class E, class A, class B, class = std::enable_if_t<!std::is_integral_v<E>>>
    RangePolicy(const E&, A b, B e) : begin_((int64_t)b), end_((int64_t)e) {}
};

struct PerTeamValue {
    size_t bytes;
};
inline PerTeamValue PerTeam(size_t b) { return PerTeamValue{b}; }

// A team of one thread.  Scratch memory is a per-thread buffer handed out by a
// bump allocator that restarts for every league member.
class HostTeamMember {
public:
    struct Shmem {
        char* base = nullptr;
        size_t cap = 0;
        size_t used = 0;
        void* get_shmem(size_t bytes, int = 0) {
            size_t off = (used + 15) & ~size_t(15);
            if (off + bytes > cap) {
                std::cerr << "Kokkos shim: team scratch exhausted (" << off + bytes << " > " << cap << ")" << std::endl;
                std::abort();
            }
            used = off + bytes;
            return base + off;
        }
    };
    int64_t rank_ = 0, league_ = 0;
    mutable Shmem shmem_;
    explicit HostTeamMember(int64_t r, int64_t l, char* s, size_t cap) : rank_(r), league_(l) {
        shmem_.base = s;
        shmem_.cap = cap;
    }
    int64_t league_rank() const { return rank_; }
    int64_t league_size() const { return league_; }
    int team_rank() const { return 0; }
    int team_size() const { return 1; }
    void team_barrier() const {}
    Shmem& team_shmem() const { return shmem_; }
    Shmem& team_scratch(int) const { return shmem_; }
    Shmem& thread_scratch(int) const { return shmem_; }
};

template <class... Props>
struct TeamPolicy {
    using execution_space = typename impl::first_exec<Props...>::type;
    using member_type = HostTeamMember;
    static constexpr bool threaded = execution_space::threaded;
    int64_t league_ = 0;
    size_t scratch_ = 0;
    TeamPolicy() = default;
    template <class L>
    TeamPolicy(L league, AUTO_t) : league_((int64_t)league) {}
    template <class L, class T, class = std::enable_if_t<std::is_integral_v<T>>>
    TeamPolicy(L league, T) : league_((int64_t)league) {}
    template <class L>
    TeamPolicy(L league, AUTO_t, AUTO_t) : league_((int64_t)league) {}
    template <class L, class T, class V>
    TeamPolicy(L league, T, V) : league_((int64_t)league) {}
    TeamPolicy& set_scratch_size(int, PerTeamValue p) {
        scratch_ += p.bytes;
        return *this;
    }
    TeamPolicy& set_scratch_size(int, PerTeamValue p, PerTeamValue) {
        scratch_ += p.bytes;
        return *this;
    }
    int64_t league_size() const { return league_; }
    int team_size() const { return 1; }
};

template <class I>
struct TeamRange {
    const HostTeamMember* m;
    I begin, end;
};
template <class A, class B>
TeamRange<std::common_type_t<A, B>> TeamThreadRange(const HostTeamMember& m, A b, B e) {
    using I = std::common_type_t<A, B>;
    return TeamRange<I>{&m, (I)b, (I)e};
}
template <class A>
TeamRange<A> TeamThreadRange(const HostTeamMember& m, A e) {
    return TeamRange<A>{&m, (A)0, e};
}
template <class A, class B>
TeamRange<std::common_type_t<A, B>> TeamVectorRange(const HostTeamMember& m, A b, B e) {
    return TeamThreadRange(m, b, e);
}
template <class A, class B>
TeamRange<std::common_type_t<A, B>> ThreadVectorRange(const HostTeamMember& m, A b, B e) {
    return TeamThreadRange(m, b, e);
}

struct PerTeamTag {
    const HostTeamMember* m;
};
inline PerTeamTag PerTeam(const HostTeamMember& m) { return PerTeamTag{&m}; }
inline PerTeamTag PerThread(const HostTeamMember& m) { return PerTeamTag{&m}; }
template <class F>
void single(PerTeamTag, const F& f) {
    f();
}
template <class F, class T>
void single(PerTeamTag, const F& f, T& v) {
    f(v);
}

// ------------------------------------------------------------------ reducers
template <class T, class I>
struct ValLocScalar {
    T val;
    I loc;
};

namespace impl {
template <class T>
struct reducer_tag {};
template <class T>
struct result_ref {
    T* p;
    template <class D, class... P>
    result_ref(const View<D, P...>& v) : p(v.data()) {}
    result_ref(T& r) : p(&r) {}
};
}  // namespace impl

template <class T, class Space = HostSpace>
struct Max {
    using value_type = T;
    using reducer = Max;
    static constexpr bool is_reducer = true;
    impl::result_ref<T> r;
    template <class R>
    Max(R&& x) : r(std::forward<R>(x)) {}
    static void init(T& v) { v = std::numeric_limits<T>::lowest(); }
    static void join(T& d, const T& s) {
        if (s > d) d = s;
    }
    T& reference() const { return *r.p; }
};
template <class T, class Space = HostSpace>
struct Min {
    using value_type = T;
    using reducer = Min;
    static constexpr bool is_reducer = true;
    impl::result_ref<T> r;
    template <class R>
    Min(R&& x) : r(std::forward<R>(x)) {}
    static void init(T& v) { v = std::numeric_limits<T>::max(); }
    static void join(T& d, const T& s) {
        if (s < d) d = s;
    }
    T& reference() const { return *r.p; }
};
template <class T, class Space = HostSpace>
struct Sum {
    using value_type = T;
    using reducer = Sum;
    static constexpr bool is_reducer = true;
    impl::result_ref<T> r;
    template <class R>
    Sum(R&& x) : r(std::forward<R>(x)) {}
    static void init(T& v) { v = T(0); }
    static void join(T& d, const T& s) { d += s; }
    T& reference() const { return *r.p; }
};
// Location of the maximum value; the identity's location is the largest index.
template <class T, class I, class Space = HostSpace>
struct MaxLoc {
    using value_type = ValLocScalar<T, I>;
    using reducer = MaxLoc;
    static constexpr bool is_reducer = true;
    impl::result_ref<value_type> r;
    template <class R>
    MaxLoc(R&& x) : r(std::forward<R>(x)) {}
    static void init(value_type& v) {
        v.val = std::numeric_limits<T>::lowest();
        v.loc = std::numeric_limits<I>::max();
    }
    static void join(value_type& d, const value_type& s) {
        if (s.val > d.val) d = s;
    }
    value_type& reference() const { return *r.p; }
};
// As MaxLoc, but equal values keep the smallest location.
template <class T, class I, class Space = HostSpace>
struct MaxFirstLoc {
    using value_type = ValLocScalar<T, I>;
    using reducer = MaxFirstLoc;
    static constexpr bool is_reducer = true;
    impl::result_ref<value_type> r;
    template <class R>
    MaxFirstLoc(R&& x) : r(std::forward<R>(x)) {}
    static void init(value_type& v) {
        v.val = std::numeric_limits<T>::lowest();
        v.loc = std::numeric_limits<I>::max();
    }
    static void join(value_type& d, const value_type& s) {
        if (s.val > d.val || (s.val == d.val && s.loc < d.loc)) d = s;
    }
    value_type& reference() const { return *r.p; }
};

namespace impl {
template <class R, class = void>
struct is_reducer : std::false_type {};
template <class R>
struct is_reducer<R, std::enable_if_t<R::is_reducer>> : std::true_type {};

// Adapts a plain result (scalar reference or rank-0 view) into a sum reducer.
template <class T>
struct SumInto {
    using value_type = T;
    T* p;
    static void init(T& v) { v = T(0); }
    static void join(T& d, const T& s) { d += s; }
    T& reference() const { return *p; }
};
template <class T, class R>
SumInto<T> as_reducer(R& r, std::enable_if_t<!is_view<std::remove_cv_t<R>>::value, int> = 0) {
    return SumInto<T>{reinterpret_cast<T*>(&r)};
}
template <class T, class D, class... P>
SumInto<T> as_reducer(const View<D, P...>& v) {
    return SumInto<T>{reinterpret_cast<T*>(v.data())};
}
}  // namespace impl

template <class T>
constexpr T min(const T& a, const T& b) {
    return b < a ? b : a;
}
template <class T>
constexpr T max(const T& a, const T& b) {
    return a < b ? b : a;
}

// ------------------------------------------------------------------ atomics
#ifdef _OPENMP
template <class T, class U>
inline void atomic_add(T* p, U v) {
    if constexpr (std::is_integral_v<T>) {
        __atomic_fetch_add(p, (T)v, __ATOMIC_RELAXED);
    } else {
        T old, next;
        __atomic_load(p, &old, __ATOMIC_RELAXED);
        do {
            next = old + (T)v;
        } while (!__atomic_compare_exchange(p, &old, &next, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED));
    }
}
template <class T, class U>
inline T atomic_fetch_add(T* p, U v) {
    return __atomic_fetch_add(p, (T)v, __ATOMIC_RELAXED);
}
template <class T, class U, class V>
inline T atomic_compare_exchange(T* p, U expected, V desired) {
    T e = (T)expected;
    __atomic_compare_exchange_n(p, &e, (T)desired, false, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE);
    return e;
}
#else
template <class T, class U>
inline void atomic_add(T* p, U v) {
    *p += (T)v;
}
template <class T, class U>
inline T atomic_fetch_add(T* p, U v) {
    T old = *p;
    *p += (T)v;
    return old;
}
template <class T, class U, class V>
inline T atomic_compare_exchange(T* p, U expected, V desired) {
    T old = *p;
    if (old == (T)expected) *p = (T)desired;
    return old;
}
#endif
template <class T, class U>
inline void atomic_increment(T* p) {
    atomic_add(p, 1);
}

// ------------------------------------------------------------------ dispatch
namespace impl {
// Calls f(i) over [b, e).  Threaded spaces split the range over OpenMP threads.
template <bool threaded, bool dynamic, class F>
void range_for(int64_t b, int64_t e, const F& f) {
#ifdef _OPENMP
    if (threaded && e - b > 1) {
        if (dynamic) {
#pragma omp parallel for schedule(dynamic, 64)
            for (int64_t i = b; i < e; i++) f(i);
        } else {
#pragma omp parallel for schedule(static)
            for (int64_t i = b; i < e; i++) f(i);
        }
        return;
    }
#endif
    for (int64_t i = b; i < e; i++) f(i);
}

// Per-thread team scratch buffers.
inline std::vector<char>& team_buffer(size_t bytes) {
    static thread_local std::vector<char> buf;
    if (buf.size() < bytes) buf.resize(bytes);
    return buf;
}

// Reduction of f(i, v) over [b, e) with reducer r (init / join), result stored
// in r.reference().
template <bool threaded, class R, class F>
void range_reduce(int64_t b, int64_t e, const F& f, const R& r) {
    using T = typename R::value_type;
    T total;
    R::init(total);
#ifdef _OPENMP
    if (threaded && e - b > 1) {
        int nt = max_threads();
        std::vector<T> part(nt);
        for (auto& x : part) R::init(x);
#pragma omp parallel
        {
            int t = omp_get_thread_num();
            T local;
            R::init(local);
#pragma omp for schedule(static)
            for (int64_t i = b; i < e; i++) f(i, local);
            part[t] = local;
        }
        for (int t = 0; t < nt; t++) R::join(total, part[t]);
        r.reference() = total;
        return;
    }
#endif
    for (int64_t i = b; i < e; i++) f(i, total);
    r.reference() = total;
}

// Exclusive-style scan f(i, update, final) over [b, e); returns the total.
// The threaded version runs every chunk twice: once with final == false to
// sum it, once with final == true from its prefix.
template <bool threaded, class T, class F>
T range_scan(int64_t b, int64_t e, const F& f) {
#ifdef _OPENMP
    if (threaded && e - b >= 4096) {
        int nt = max_threads();
        std::vector<T> sums(nt + 1, T(0));
        int64_t len = e - b;
#pragma omp parallel num_threads(nt)
        {
            int t = omp_get_thread_num();
            int nth = omp_get_num_threads();
            int64_t lo = b + len * t / nth, hi = b + len * (t + 1) / nth;
            T local = T(0);
            for (int64_t i = lo; i < hi; i++) f(i, local, false);
            sums[t + 1] = local;
#pragma omp barrier
#pragma omp single
            {
                for (int x = 1; x <= nth; x++) sums[x] += sums[x - 1];
            }
            T run = sums[t];
            for (int64_t i = lo; i < hi; i++) f(i, run, true);
        }
        return sums[nt];
    }
#endif
    T update = T(0);
    for (int64_t i = b; i < e; i++) f(i, update, true);
    return update;
}
}  // namespace impl

// parallel_for over a range (policy or count).
template <class... P, class F>
void parallel_for(const RangePolicy<P...>& p, const F& f) {
    impl::range_for<RangePolicy<P...>::threaded, RangePolicy<P...>::dynamic>(p.begin_, p.end_, f);
}
template <class... P, class F>
void parallel_for(const std::string&, const RangePolicy<P...>& p, const F& f) {
    parallel_for(p, f);
}
template <class I, class F, class = std::enable_if_t<std::is_integral_v<I>>>
void parallel_for(I n, const F& f) {
    impl::range_for<DefaultExecutionSpace::threaded, false>(0, (int64_t)n, f);
}
template <class I, class F, class = std::enable_if_t<std::is_integral_v<I>>>
void parallel_for(const std::string&, I n, const F& f) {
    parallel_for(n, f);
}

// parallel_for over a league of one-thread teams.
template <class... P, class F>
void parallel_for(const TeamPolicy<P...>& p, const F& f) {
    const int64_t league = p.league_;
    const size_t scratch = p.scratch_;
    impl::range_for<TeamPolicy<P...>::threaded, true>(0, league, [&](int64_t r) {
        std::vector<char>& buf = impl::team_buffer(scratch);
        HostTeamMember m(r, league, buf.data(), buf.size());
        f(m);
    });
}
template <class... P, class F>
void parallel_for(const std::string&, const TeamPolicy<P...>& p, const F& f) {
    parallel_for(p, f);
}

// Nested loop inside a team.
template <class I, class F>
void parallel_for(const TeamRange<I>& r, const F& f) {
    for (I i = r.begin; i < r.end; i++) f(i);
}

// parallel_reduce over a range.
template <class... P, class F, class Res>
void parallel_reduce(const RangePolicy<P...>& p, const F& f, Res&& res) {
    using R = std::remove_cv_t<std::remove_reference_t<Res>>;
    if constexpr (impl::is_reducer<R>::value) {
        impl::range_reduce<RangePolicy<P...>::threaded>(p.begin_, p.end_, f, res);
    } else {
        using T = impl::arg_value_t<F, 1>;
        impl::range_reduce<RangePolicy<P...>::threaded>(p.begin_, p.end_, f, impl::as_reducer<T>(res));
    }
}
template <class... P, class F, class Res>
void parallel_reduce(const std::string&, const RangePolicy<P...>& p, const F& f, Res&& res) {
    parallel_reduce(p, f, std::forward<Res>(res));
}
template <class I, class F, class Res, class = std::enable_if_t<std::is_integral_v<I>>>
void parallel_reduce(I n, const F& f, Res&& res) {
    parallel_reduce(RangePolicy<DefaultExecutionSpace>(0, (int64_t)n), f, std::forward<Res>(res));
}
template <class I, class F, class Res, class = std::enable_if_t<std::is_integral_v<I>>>
void parallel_reduce(const std::string&, I n, const F& f, Res&& res) {
    parallel_reduce(n, f, std::forward<Res>(res));
}

// parallel_reduce over a league of one-thread teams.
template <class... P, class F, class Res>
void parallel_reduce(const TeamPolicy<P...>& p, const F& f, Res&& res) {
    const int64_t league = p.league_;
    const size_t scratch = p.scratch_;
    auto body = [&](int64_t r, auto& v) {
        std::vector<char>& buf = impl::team_buffer(scratch);
        HostTeamMember m(r, league, buf.data(), buf.size());
        f(m, v);
    };
    using R = std::remove_cv_t<std::remove_reference_t<Res>>;
    if constexpr (impl::is_reducer<R>::value) {
        impl::range_reduce<TeamPolicy<P...>::threaded>(0, league, body, res);
    } else {
        using T = impl::arg_value_t<F, 1>;
        impl::range_reduce<TeamPolicy<P...>::threaded>(0, league, body, impl::as_reducer<T>(res));
    }
}
template <class... P, class F, class Res>
void parallel_reduce(const std::string&, const TeamPolicy<P...>& p, const F& f, Res&& res) {
    parallel_reduce(p, f, std::forward<Res>(res));
}

// Nested reduction inside a team.
template <class I, class F, class Res>
void parallel_reduce(const TeamRange<I>& r, const F& f, Res&& res) {
    using R = std::remove_cv_t<std::remove_reference_t<Res>>;
    if constexpr (impl::is_reducer<R>::value) {
        typename R::value_type v;
        R::init(v);
        for (I i = r.begin; i < r.end; i++) f(i, v);
        res.reference() = v;
    } else {
        using T = impl::arg_value_t<F, 1>;
        T v = T(0);
        for (I i = r.begin; i < r.end; i++) f(i, v);
        res = v;
    }
}

// parallel_scan over a range; the total goes to the optional result.
template <class... P, class F>
void parallel_scan(const RangePolicy<P...>& p, const F& f) {
    using T = impl::arg_value_t<F, 1>;
    impl::range_scan<RangePolicy<P...>::threaded, T>(p.begin_, p.end_, f);
}
template <class... P, class F, class Res>
void parallel_scan(const RangePolicy<P...>& p, const F& f, Res&& res) {
    using T = impl::arg_value_t<F, 1>;
    T total = impl::range_scan<RangePolicy<P...>::threaded, T>(p.begin_, p.end_, f);
    using R = std::remove_cv_t<std::remove_reference_t<Res>>;
    if constexpr (impl::is_view<R>::value) {
        res() = total;
    } else {
        res = total;
    }
}
template <class... P, class F>
void parallel_scan(const std::string&, const RangePolicy<P...>& p, const F& f) {
    parallel_scan(p, f);
}
template <class... P, class F, class Res>
void parallel_scan(const std::string&, const RangePolicy<P...>& p, const F& f, Res&& res) {
    parallel_scan(p, f, std::forward<Res>(res));
}
// Nested scan inside a team (one thread: in order, final pass only).
template <class I, class F>
void parallel_scan(const TeamRange<I>& r, const F& f) {
    using T = impl::arg_value_t<F, 1>;
    T update = T(0);
    for (I i = r.begin; i < r.end; i++) f(i, update, true);
}
template <class I, class F, class Res>
void parallel_scan(const TeamRange<I>& r, const F& f, Res& res) {
    using T = impl::arg_value_t<F, 1>;
    T update = T(0);
    for (I i = r.begin; i < r.end; i++) f(i, update, true);
    res = update;
}

// ------------------------------------------------------------------ timer
class Timer {
    std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();

public:
    void reset() { t0_ = std::chrono::steady_clock::now(); }
    double seconds() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    }
};

// ------------------------------------------------------------------ hashing
namespace impl {
inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
// MurmurHash3_x86_32 over n bytes, seed 0.
inline uint32_t murmur3_32(const void* key, int len) {
    const uint8_t* data = static_cast<const uint8_t*>(key);
    const int nblocks = len / 4;
    const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    uint32_t h = 0;
    for (int i = 0; i < nblocks; i++) {
        uint32_t k;
        std::memcpy(&k, data + 4 * i, 4);
        k *= c1;
        k = rotl32(k, 15);
        k *= c2;
        h ^= k;
        h = rotl32(h, 13);
        h = h * 5 + 0xe6546b64u;
    }
    const uint8_t* tail = data + nblocks * 4;
    uint32_t k1 = 0;
    switch (len & 3) {
        case 3: k1 ^= uint32_t(tail[2]) << 16; [[fallthrough]];
        case 2: k1 ^= uint32_t(tail[1]) << 8; [[fallthrough]];
        case 1:
            k1 ^= tail[0];
            k1 *= c1;
            k1 = rotl32(k1, 15);
            k1 *= c2;
            h ^= k1;
    }
    h ^= (uint32_t)len;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}
}  // namespace impl

template <class T>
struct pod_hash {
    uint32_t operator()(const T& t) const { return impl::murmur3_32(&t, (int)sizeof(T)); }
};

// ------------------------------------------------------------------ random
namespace impl {
inline uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
}  // namespace impl

template <class Dev>
class Random_XorShift64;

template <class Dev>
class Random_XorShift64_Pool {
public:
    using generator_type = Random_XorShift64<Dev>;
    std::shared_ptr<std::vector<uint64_t>> states_;

    Random_XorShift64_Pool() = default;
    explicit Random_XorShift64_Pool(uint64_t seed) {
        const char* env = std::getenv("JET_SEED");
        if (env && *env) seed = std::strtoull(env, nullptr, 10);
        int n = impl::max_threads();
        states_ = std::make_shared<std::vector<uint64_t>>(n);
        uint64_t x = seed;
        for (int i = 0; i < n; i++) {
            uint64_t s = impl::splitmix64(x);
            (*states_)[i] = s ? s : 0x2545F4914F6CDD1Dull;
        }
    }
    generator_type get_state() const {
        return generator_type((*states_)[impl::thread_id()], impl::thread_id());
    }
    void free_state(const generator_type& g) const { (*states_)[g.slot_] = g.state_; }
};

template <class Dev>
class Random_XorShift64 {
public:
    uint64_t state_;
    int slot_;
    Random_XorShift64(uint64_t s, int slot) : state_(s), slot_(slot) {}
    // xorshift64*: three xorshifts of the state, output scrambled by a multiply.
    uint64_t urand64() {
        state_ ^= state_ >> 12;
        state_ ^= state_ << 25;
        state_ ^= state_ >> 27;
        return state_ * 0x2545F4914F6CDD1Dull;
    }
    uint32_t urand() { return (uint32_t)(urand64() >> 32); }
    uint64_t urand64(uint64_t range) { return urand64() % range; }
    template <class A>
    A urand(A start, A end) {
        uint64_t range = (uint64_t)(end - start);
        return (A)(start + (A)(urand64() % range));
    }
};

}  // namespace Kokkos
