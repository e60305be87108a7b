// Open multimethods for the C++ layer of the B200 engine.
//
// FRANK dispatches every operation on the dynamic types of its matrix
// arguments through yomm2's open multimethods (e.g. gemm_omm,
// operations/BLAS/gemm.cpp; getrf_omm, operations/LAPACK/getrf.cpp), written
// with the macros declare_method / define_method / register_class and the
// parameter marker virtual_<T>.  This header provides the same surface, so
// that the layer above the C ABI reads like FRANK's operations:
//
//   register_class(Matrix)
//   register_class(Dense, Matrix)
//   declare_method(void, gemm_omm, (virtual_<const Matrix&>, virtual_<const Matrix&>,
//                                   virtual_<Matrix&>, double, double, bool, bool))
//   define_method(void, gemm_omm, (const Dense& A, const Dense& B, Dense& C,
//                                  double alpha, double beta, bool ta, bool tb)) { ... }
//   gemm_omm(A, B, C, 1, 1, false, false);   // A, B, C: const Matrix& / Matrix&
//
// Resolution rule (the one yomm2 documents): among the overloads whose
// virtual parameter types are each a base of (or equal to) the dynamic type of
// the corresponding argument, the unique most specific one is called; an
// overload is more specific than another when each of its virtual parameter
// types derives from (or equals) the other's.  No applicable overload, or
// several equally specific ones, throws frank_mm::dispatch_error naming the
// method and the dynamic types.  The resolved overload is cached per tuple of
// dynamic types.
//
// Requirements: classes that take part in dispatch are polymorphic and
// registered with their direct bases; inheritance is single and non-virtual
// (virtual arguments are down-cast with static_cast after the type check).
// Method declarations must not contain a top-level comma inside the return
// type (use an alias, as FRANK does with MatrixPair).
#ifndef FRANK_B200_MULTIMETHOD_HPP
#define FRANK_B200_MULTIMETHOD_HPP

#include <array>
#include <cstddef>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <typeindex>
#include <typeinfo>
#include <unordered_map>
#include <utility>
#include <vector>

namespace frank_mm {

// Marks a parameter of declare_method that takes part in dispatch.
template <class T>
struct virtual_;

// Thrown when a call has no applicable overload or an ambiguous one.
struct dispatch_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

namespace detail {

template <class T> struct strip { using type = T; };
template <class T> struct strip<virtual_<T>> { using type = T; };
template <class T> using strip_t = typename strip<T>::type;

template <class T> struct is_virtual : std::false_type {};
template <class T> struct is_virtual<virtual_<T>> : std::true_type {};

template <class... A>
constexpr std::size_t count_virtual() { return (std::size_t(0) + ... + (is_virtual<A>::value ? 1u : 0u)); }

// Registered classes: type -> direct bases.
struct ClassTable {
  std::mutex mu;
  std::unordered_map<std::type_index, std::vector<std::type_index>> bases;
};

inline ClassTable& classes() {
  static ClassTable t;
  return t;
}

inline void add_class(std::type_index c, std::vector<std::type_index> b) {
  ClassTable& t = classes();
  std::lock_guard<std::mutex> lock(t.mu);
  t.bases[c] = std::move(b);
}

// d is b, or derives from b through registered classes (caller holds no lock).
inline bool is_a_locked(const ClassTable& t, std::type_index d, std::type_index b) {
  if (d == b) return true;
  auto it = t.bases.find(d);
  if (it == t.bases.end()) return false;
  for (const auto& p : it->second)
    if (is_a_locked(t, p, b)) return true;
  return false;
}

inline bool is_a(std::type_index d, std::type_index b) {
  ClassTable& t = classes();
  std::lock_guard<std::mutex> lock(t.mu);
  return is_a_locked(t, d, b);
}

// Converts a method argument to the overload's parameter type: a down-cast
// for virtual parameters (checked by the resolution), an ordinary
// conversion for the others.
template <class P, class T>
inline P cast_arg(T&& a) {
  return static_cast<P>(std::forward<T>(a));
}

template <class A, class P>
inline void push_type(std::vector<std::type_index>& out) {
  if constexpr (is_virtual<A>::value) out.emplace_back(typeid(std::remove_cv_t<std::remove_reference_t<P>>));
}

template <class A, class T>
inline void push_dynamic(std::array<const std::type_info*, 16>& out, std::size_t& n, const T& a) {
  if constexpr (is_virtual<A>::value) out[n++] = &typeid(a);
}

}  // namespace detail

template <class C, class... Bases>
struct class_registrar {
  class_registrar() { detail::add_class(typeid(C), {std::type_index(typeid(Bases))...}); }
};

// Finishes registration.  Dispatch tables are built lazily, so this only
// exists for the FRANK::initialize() call sequence (initialize.cpp:14-16).
inline void update_methods() {}

template <class Tag, class Sig>
class method;

template <class Tag, class R, class... A>
class method<Tag, R(A...)> {
 public:
  static constexpr std::size_t n_virtual = detail::count_virtual<A...>();
  static_assert(n_virtual >= 1 && n_virtual <= 16, "a method needs 1..16 virtual parameters");
  using raw_fn = void (*)();
  using thunk_fn = R (*)(raw_fn, detail::strip_t<A>...);
  using call_type = R (*)(detail::strip_t<A>...);
  // Argument types T... can be passed to this method.
  template <class... T>
  static constexpr bool accepts = std::is_invocable_v<call_type, T...>;

  struct Overload {
    std::vector<std::type_index> types;  // decayed types of the virtual parameters
    raw_fn fn;
    thunk_fn thunk;
    const char* where;
  };

  // Adds an overload; P... are the overload's parameter types.
  template <class... P>
  static bool add(R (*fn)(P...), const char* where) {
    static_assert(sizeof...(P) == sizeof...(A), "define_method: parameter count differs from declare_method");
    Overload o;
    (detail::push_type<A, P>(o.types), ...);
    o.fn = reinterpret_cast<raw_fn>(fn);
    o.thunk = &thunk<P...>;
    o.where = where;
    State& s = state();
    std::lock_guard<std::mutex> lock(s.mu);
    s.overloads.push_back(std::move(o));
    s.cache.clear();
    return true;
  }

  R operator()(detail::strip_t<A>... args) const {
    std::array<const std::type_info*, 16> dyn{};
    std::size_t n = 0;
    (detail::push_dynamic<A>(dyn, n, args), ...);
    const Overload& o = resolve(dyn);
    return o.thunk(o.fn, std::forward<detail::strip_t<A>>(args)...);
  }

  static const char* name() { return state().name.c_str(); }

  static bool set_name(const char* n) {
    State& s = state();
    std::lock_guard<std::mutex> lock(s.mu);
    s.name = n;
    return true;
  }

 private:
  struct State {
    std::mutex mu;
    std::string name = "method";
    std::vector<Overload> overloads;
    std::map<std::vector<std::type_index>, std::size_t> cache;
  };

  static State& state() {
    static State s;
    return s;
  }

  template <class... P>
  static R thunk(raw_fn f, detail::strip_t<A>... args) {
    auto fn = reinterpret_cast<R (*)(P...)>(f);
    return fn(detail::cast_arg<P>(std::forward<detail::strip_t<A>>(args))...);
  }

  static std::string type_list(const std::vector<std::type_index>& k) {
    std::string s;
    for (std::size_t j = 0; j < k.size(); ++j) s += (j ? ", " : "") + std::string(k[j].name());
    return s;
  }

  static const Overload& resolve(const std::array<const std::type_info*, 16>& dyn) {
    std::vector<std::type_index> key;
    key.reserve(n_virtual);
    for (std::size_t j = 0; j < n_virtual; ++j) key.emplace_back(*dyn[j]);
    State& s = state();
    std::lock_guard<std::mutex> lock(s.mu);
    auto hit = s.cache.find(key);
    if (hit != s.cache.end()) return s.overloads[hit->second];
    detail::ClassTable& ct = detail::classes();
    std::lock_guard<std::mutex> lock2(ct.mu);
    auto applies = [&](const std::vector<std::type_index>& from, const std::vector<std::type_index>& to) {
      for (std::size_t j = 0; j < n_virtual; ++j)
        if (!detail::is_a_locked(ct, from[j], to[j])) return false;
      return true;
    };
    std::vector<std::size_t> cand;
    for (std::size_t q = 0; q < s.overloads.size(); ++q)
      if (applies(key, s.overloads[q].types)) cand.push_back(q);
    std::vector<std::size_t> best;
    for (std::size_t c : cand) {
      bool dominated = false;
      for (std::size_t d : cand)
        if (d != c && s.overloads[d].types != s.overloads[c].types &&
            applies(s.overloads[d].types, s.overloads[c].types)) {
          dominated = true;
          break;
        }
      if (!dominated) best.push_back(c);
    }
    if (best.size() != 1)
      throw dispatch_error(s.name + "(" + type_list(key) + "): " +
                           (best.empty() ? "no applicable overload" : "ambiguous overloads"));
    s.cache.emplace(std::move(key), best[0]);
    return s.overloads[best[0]];
  }
};

// Registers fn as an overload of the method that `select` names: select is
// called (unevaluated) with fn's parameter types and returns the method type
// chosen by ordinary C++ overload resolution among the methods of that name.
template <class R, class... P, class Select>
bool add_overload(R (*fn)(P...), Select, const char* where) {
  using M = decltype(std::declval<Select&>()(std::declval<P>()...));
  return M::add(fn, where);
}

}  // namespace frank_mm

#define FRANK_MM_CAT_(a, b) a##b
#define FRANK_MM_CAT(a, b) FRANK_MM_CAT_(a, b)
#define FRANK_MM_STR_(a) #a
#define FRANK_MM_STR(a) FRANK_MM_STR_(a)

// register_class(C) or register_class(C, Base): C takes part in dispatch.
#define register_class(...) \
  static const ::frank_mm::class_registrar<__VA_ARGS__> FRANK_MM_CAT(frank_mm_class_, __COUNTER__);

// Argument counting and per-parameter expansion over a parenthesised list
// of up to 12 parameter types (no top-level commas inside a type).
#define FRANK_MM_NARG(...) FRANK_MM_NARG_(__VA_ARGS__, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1, 0)
#define FRANK_MM_NARG_(_1, _2, _3, _4, _5, _6, _7, _8, _9, _10, _11, _12, n, ...) n
#define FRANK_MM_T(T) ::frank_mm::detail::strip_t<T>
#define FRANK_MM_P_1(T1) FRANK_MM_T(T1) frank_mm_a1
#define FRANK_MM_F_1(T1) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1)
#define FRANK_MM_U_1(T1) FRANK_MM_T(T1)
#define FRANK_MM_P_2(T1, T2) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2
#define FRANK_MM_F_2(T1, T2) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2)
#define FRANK_MM_U_2(T1, T2) FRANK_MM_T(T1), FRANK_MM_T(T2)
#define FRANK_MM_P_3(T1, T2, T3) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3
#define FRANK_MM_F_3(T1, T2, T3) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3)
#define FRANK_MM_U_3(T1, T2, T3) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3)
#define FRANK_MM_P_4(T1, T2, T3, T4) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4
#define FRANK_MM_F_4(T1, T2, T3, T4) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4)
#define FRANK_MM_U_4(T1, T2, T3, T4) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4)
#define FRANK_MM_P_5(T1, T2, T3, T4, T5) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4, FRANK_MM_T(T5) frank_mm_a5
#define FRANK_MM_F_5(T1, T2, T3, T4, T5) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4), static_cast<FRANK_MM_T(T5)&&>(frank_mm_a5)
#define FRANK_MM_U_5(T1, T2, T3, T4, T5) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4), FRANK_MM_T(T5)
#define FRANK_MM_P_6(T1, T2, T3, T4, T5, T6) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4, FRANK_MM_T(T5) frank_mm_a5, FRANK_MM_T(T6) frank_mm_a6
#define FRANK_MM_F_6(T1, T2, T3, T4, T5, T6) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4), static_cast<FRANK_MM_T(T5)&&>(frank_mm_a5), static_cast<FRANK_MM_T(T6)&&>(frank_mm_a6)
#define FRANK_MM_U_6(T1, T2, T3, T4, T5, T6) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4), FRANK_MM_T(T5), FRANK_MM_T(T6)
#define FRANK_MM_P_7(T1, T2, T3, T4, T5, T6, T7) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4, FRANK_MM_T(T5) frank_mm_a5, FRANK_MM_T(T6) frank_mm_a6, FRANK_MM_T(T7) frank_mm_a7
#define FRANK_MM_F_7(T1, T2, T3, T4, T5, T6, T7) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4), static_cast<FRANK_MM_T(T5)&&>(frank_mm_a5), static_cast<FRANK_MM_T(T6)&&>(frank_mm_a6), static_cast<FRANK_MM_T(T7)&&>(frank_mm_a7)
#define FRANK_MM_U_7(T1, T2, T3, T4, T5, T6, T7) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4), FRANK_MM_T(T5), FRANK_MM_T(T6), FRANK_MM_T(T7)
#define FRANK_MM_P_8(T1, T2, T3, T4, T5, T6, T7, T8) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4, FRANK_MM_T(T5) frank_mm_a5, FRANK_MM_T(T6) frank_mm_a6, FRANK_MM_T(T7) frank_mm_a7, FRANK_MM_T(T8) frank_mm_a8
#define FRANK_MM_F_8(T1, T2, T3, T4, T5, T6, T7, T8) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4), static_cast<FRANK_MM_T(T5)&&>(frank_mm_a5), static_cast<FRANK_MM_T(T6)&&>(frank_mm_a6), static_cast<FRANK_MM_T(T7)&&>(frank_mm_a7), static_cast<FRANK_MM_T(T8)&&>(frank_mm_a8)
#define FRANK_MM_U_8(T1, T2, T3, T4, T5, T6, T7, T8) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4), FRANK_MM_T(T5), FRANK_MM_T(T6), FRANK_MM_T(T7), FRANK_MM_T(T8)
#define FRANK_MM_P_9(T1, T2, T3, T4, T5, T6, T7, T8, T9) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4, FRANK_MM_T(T5) frank_mm_a5, FRANK_MM_T(T6) frank_mm_a6, FRANK_MM_T(T7) frank_mm_a7, FRANK_MM_T(T8) frank_mm_a8, FRANK_MM_T(T9) frank_mm_a9
#define FRANK_MM_F_9(T1, T2, T3, T4, T5, T6, T7, T8, T9) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4), static_cast<FRANK_MM_T(T5)&&>(frank_mm_a5), static_cast<FRANK_MM_T(T6)&&>(frank_mm_a6), static_cast<FRANK_MM_T(T7)&&>(frank_mm_a7), static_cast<FRANK_MM_T(T8)&&>(frank_mm_a8), static_cast<FRANK_MM_T(T9)&&>(frank_mm_a9)
#define FRANK_MM_U_9(T1, T2, T3, T4, T5, T6, T7, T8, T9) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4), FRANK_MM_T(T5), FRANK_MM_T(T6), FRANK_MM_T(T7), FRANK_MM_T(T8), FRANK_MM_T(T9)
#define FRANK_MM_P_10(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4, FRANK_MM_T(T5) frank_mm_a5, FRANK_MM_T(T6) frank_mm_a6, FRANK_MM_T(T7) frank_mm_a7, FRANK_MM_T(T8) frank_mm_a8, FRANK_MM_T(T9) frank_mm_a9, FRANK_MM_T(T10) frank_mm_a10
#define FRANK_MM_F_10(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4), static_cast<FRANK_MM_T(T5)&&>(frank_mm_a5), static_cast<FRANK_MM_T(T6)&&>(frank_mm_a6), static_cast<FRANK_MM_T(T7)&&>(frank_mm_a7), static_cast<FRANK_MM_T(T8)&&>(frank_mm_a8), static_cast<FRANK_MM_T(T9)&&>(frank_mm_a9), static_cast<FRANK_MM_T(T10)&&>(frank_mm_a10)
#define FRANK_MM_U_10(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4), FRANK_MM_T(T5), FRANK_MM_T(T6), FRANK_MM_T(T7), FRANK_MM_T(T8), FRANK_MM_T(T9), FRANK_MM_T(T10)
#define FRANK_MM_P_11(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4, FRANK_MM_T(T5) frank_mm_a5, FRANK_MM_T(T6) frank_mm_a6, FRANK_MM_T(T7) frank_mm_a7, FRANK_MM_T(T8) frank_mm_a8, FRANK_MM_T(T9) frank_mm_a9, FRANK_MM_T(T10) frank_mm_a10, FRANK_MM_T(T11) frank_mm_a11
#define FRANK_MM_F_11(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4), static_cast<FRANK_MM_T(T5)&&>(frank_mm_a5), static_cast<FRANK_MM_T(T6)&&>(frank_mm_a6), static_cast<FRANK_MM_T(T7)&&>(frank_mm_a7), static_cast<FRANK_MM_T(T8)&&>(frank_mm_a8), static_cast<FRANK_MM_T(T9)&&>(frank_mm_a9), static_cast<FRANK_MM_T(T10)&&>(frank_mm_a10), static_cast<FRANK_MM_T(T11)&&>(frank_mm_a11)
#define FRANK_MM_U_11(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4), FRANK_MM_T(T5), FRANK_MM_T(T6), FRANK_MM_T(T7), FRANK_MM_T(T8), FRANK_MM_T(T9), FRANK_MM_T(T10), FRANK_MM_T(T11)
#define FRANK_MM_P_12(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12) FRANK_MM_T(T1) frank_mm_a1, FRANK_MM_T(T2) frank_mm_a2, FRANK_MM_T(T3) frank_mm_a3, FRANK_MM_T(T4) frank_mm_a4, FRANK_MM_T(T5) frank_mm_a5, FRANK_MM_T(T6) frank_mm_a6, FRANK_MM_T(T7) frank_mm_a7, FRANK_MM_T(T8) frank_mm_a8, FRANK_MM_T(T9) frank_mm_a9, FRANK_MM_T(T10) frank_mm_a10, FRANK_MM_T(T11) frank_mm_a11, FRANK_MM_T(T12) frank_mm_a12
#define FRANK_MM_F_12(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12) static_cast<FRANK_MM_T(T1)&&>(frank_mm_a1), static_cast<FRANK_MM_T(T2)&&>(frank_mm_a2), static_cast<FRANK_MM_T(T3)&&>(frank_mm_a3), static_cast<FRANK_MM_T(T4)&&>(frank_mm_a4), static_cast<FRANK_MM_T(T5)&&>(frank_mm_a5), static_cast<FRANK_MM_T(T6)&&>(frank_mm_a6), static_cast<FRANK_MM_T(T7)&&>(frank_mm_a7), static_cast<FRANK_MM_T(T8)&&>(frank_mm_a8), static_cast<FRANK_MM_T(T9)&&>(frank_mm_a9), static_cast<FRANK_MM_T(T10)&&>(frank_mm_a10), static_cast<FRANK_MM_T(T11)&&>(frank_mm_a11), static_cast<FRANK_MM_T(T12)&&>(frank_mm_a12)
#define FRANK_MM_U_12(T1, T2, T3, T4, T5, T6, T7, T8, T9, T10, T11, T12) FRANK_MM_T(T1), FRANK_MM_T(T2), FRANK_MM_T(T3), FRANK_MM_T(T4), FRANK_MM_T(T5), FRANK_MM_T(T6), FRANK_MM_T(T7), FRANK_MM_T(T8), FRANK_MM_T(T9), FRANK_MM_T(T10), FRANK_MM_T(T11), FRANK_MM_T(T12)
#define FRANK_MM_EXPAND(x) x
#define FRANK_MM_APPLY_(kind, n, ARGS) FRANK_MM_CAT(FRANK_MM_CAT(FRANK_MM_, kind), FRANK_MM_CAT(_, n)) ARGS
#define FRANK_MM_APPLY(kind, ARGS) FRANK_MM_APPLY_(kind, FRANK_MM_EXPAND(FRANK_MM_NARG ARGS), ARGS)

// declare_method(R, name, (params)): `name` becomes an inline function taking
// the declared parameters (an overload set when several methods share the
// name, e.g. FRANK's two gemm_omm), virtual_<T> ones taking part in
// dispatch.  A method is identified by its name and signature, so declaring
// the same method in several translation units yields one method.
#define declare_method(R, NAME, ARGS)                                                                     \
  struct FRANK_MM_CAT(NAME, _frank_mm_tag);                                                               \
  [[maybe_unused]] static const bool FRANK_MM_CAT(frank_mm_named_, __COUNTER__) =                         \
      ::frank_mm::method<FRANK_MM_CAT(NAME, _frank_mm_tag), R ARGS>::set_name(#NAME);                     \
  inline R NAME(FRANK_MM_APPLY(P, ARGS)) {                                                                \
    return ::frank_mm::method<FRANK_MM_CAT(NAME, _frank_mm_tag), R ARGS>{}(FRANK_MM_APPLY(F, ARGS));      \
  }                                                                                                       \
  ::frank_mm::method<FRANK_MM_CAT(NAME, _frank_mm_tag), R ARGS> FRANK_MM_CAT(NAME, _frank_mm_select)(    \
      FRANK_MM_APPLY(U, ARGS));

// define_method(R, name, (typed params)) { body }: one overload of the method
// `name` whose declared parameters accept these parameter types.
#define define_method(R, NAME, ARGS) FRANK_MM_DEFINE_(R, NAME, ARGS, FRANK_MM_CAT(frank_mm_fn_, __COUNTER__))
#define FRANK_MM_DEFINE_(R, NAME, ARGS, FN)                                                                \
  static R FN ARGS;                                                                                        \
  [[maybe_unused]] static const bool FRANK_MM_CAT(FN, _added) = ::frank_mm::add_overload(                 \
      &FN,                                                                                                 \
      [](auto&&... frank_mm_a) -> decltype(FRANK_MM_CAT(NAME, _frank_mm_select)(                         \
                                   ::std::forward<decltype(frank_mm_a)>(frank_mm_a)...)) { return {}; }, \
      __FILE__ ":" FRANK_MM_STR(__LINE__));                                                                \
  static R FN ARGS

#endif  // FRANK_B200_MULTIMETHOD_HPP
