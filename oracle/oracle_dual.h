// oracle_dual.h -- forward-mode automatic differentiation types for the
// oracle's gradient checks.
//
// TEST INFRASTRUCTURE ONLY (see oracle_math.h): used by the WARDiffPathTracer
// restatement to compute reference derivatives; never part of the product.
//
//   Dual<N>   value + N tangents in FP64.  Branches and comparisons use the
//             value, as Slang's differentiable code does; detach() drops the
//             tangents (Slang `detach` / `no_diff`).
//   Shadow    (base, perturbed) pair: every operation is applied to both
//             members, comparisons use the base and detach() copies the base
//             into the perturbed member.  Evaluating a path with the seeded
//             parameters offset by +-eps in the perturbed member gives a
//             central finite difference that honours exactly the same
//             non-differentiable points as Dual, which checks Dual's rules.
#pragma once

#include <cmath>
#include <cstring>

namespace orc {

template <int N>
struct Dual {
    double v;
    double d[N];
    constexpr Dual() : v(0), d{} {}
    constexpr Dual(double x) : v(x), d{} {}  // NOLINT: implicit like a real
    explicit operator float() const { return float(v); }
    explicit operator double() const { return v; }
};

template <int N> inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v + b.v);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v - b.v);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> inline Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r(-a.v);
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
template <int N> inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v * b.v);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v / b.v);
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v);
    return r;
}
template <int N> inline Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) { return a = a + b; }
template <int N> inline Dual<N>& operator-=(Dual<N>& a, const Dual<N>& b) { return a = a - b; }
template <int N> inline Dual<N>& operator*=(Dual<N>& a, const Dual<N>& b) { return a = a * b; }
template <int N> inline Dual<N>& operator/=(Dual<N>& a, const Dual<N>& b) { return a = a / b; }
#define ORC_DUAL_CMP(op) \
    template <int N> inline bool operator op(const Dual<N>& a, const Dual<N>& b) { return a.v op b.v; }
ORC_DUAL_CMP(<)
ORC_DUAL_CMP(>)
ORC_DUAL_CMP(<=)
ORC_DUAL_CMP(>=)
ORC_DUAL_CMP(==)
ORC_DUAL_CMP(!=)
#undef ORC_DUAL_CMP

// Chain rule helper: r = f(a) with f'(a) = fp.
template <int N> inline Dual<N> chain(const Dual<N>& a, double fa, double fp) {
    Dual<N> r(fa);
    for (int i = 0; i < N; i++) r.d[i] = fp * a.d[i];
    return r;
}
template <int N> inline Dual<N> detach(const Dual<N>& a) { return Dual<N>(a.v); }
template <int N> inline double value_of(const Dual<N>& a) { return a.v; }

struct Shadow {
    double b, p;  // base, perturbed
    constexpr Shadow() : b(0), p(0) {}
    constexpr Shadow(double x) : b(x), p(x) {}  // NOLINT
    constexpr Shadow(double x, double y) : b(x), p(y) {}
    explicit operator float() const { return float(b); }
    explicit operator double() const { return b; }
};
inline Shadow operator+(const Shadow& a, const Shadow& c) { return Shadow(a.b + c.b, a.p + c.p); }
inline Shadow operator-(const Shadow& a, const Shadow& c) { return Shadow(a.b - c.b, a.p - c.p); }
inline Shadow operator-(const Shadow& a) { return Shadow(-a.b, -a.p); }
inline Shadow operator*(const Shadow& a, const Shadow& c) { return Shadow(a.b * c.b, a.p * c.p); }
inline Shadow operator/(const Shadow& a, const Shadow& c) { return Shadow(a.b / c.b, a.p / c.p); }
inline Shadow& operator+=(Shadow& a, const Shadow& c) { return a = a + c; }
inline Shadow& operator-=(Shadow& a, const Shadow& c) { return a = a - c; }
inline Shadow& operator*=(Shadow& a, const Shadow& c) { return a = a * c; }
inline Shadow& operator/=(Shadow& a, const Shadow& c) { return a = a / c; }
inline bool operator<(const Shadow& a, const Shadow& c) { return a.b < c.b; }
inline bool operator>(const Shadow& a, const Shadow& c) { return a.b > c.b; }
inline bool operator<=(const Shadow& a, const Shadow& c) { return a.b <= c.b; }
inline bool operator>=(const Shadow& a, const Shadow& c) { return a.b >= c.b; }
inline bool operator==(const Shadow& a, const Shadow& c) { return a.b == c.b; }
inline bool operator!=(const Shadow& a, const Shadow& c) { return a.b != c.b; }
inline Shadow detach(const Shadow& a) { return Shadow(a.b, a.b); }
inline double value_of(const Shadow& a) { return a.b; }

inline float detach(float a) { return a; }
inline double detach(double a) { return a; }
inline double value_of(float a) { return a; }
inline double value_of(double a) { return a; }

// The value type a real type's non-differentiable code runs in.
template <class R> struct ValueType { using type = R; };
template <int N> struct ValueType<Dual<N>> { using type = double; };
template <> struct ValueType<Shadow> { using type = double; };

}  // namespace orc

// Elementary functions for the AD types (the oracle's templated code calls
// them std::-qualified, like the float and double instantiations).
namespace std {
template <int N> inline orc::Dual<N> sqrt(const orc::Dual<N>& a) {
    const double s = std::sqrt(a.v);
    return orc::chain(a, s, 0.5 / s);
}
template <int N> inline orc::Dual<N> fabs(const orc::Dual<N>& a) { return a.v < 0 ? -a : a; }
template <int N> inline orc::Dual<N> exp(const orc::Dual<N>& a) {
    const double e = std::exp(a.v);
    return orc::chain(a, e, e);
}
template <int N> inline orc::Dual<N> log(const orc::Dual<N>& a) { return orc::chain(a, std::log(a.v), 1.0 / a.v); }
template <int N> inline orc::Dual<N> cos(const orc::Dual<N>& a) { return orc::chain(a, std::cos(a.v), -std::sin(a.v)); }
template <int N> inline orc::Dual<N> sin(const orc::Dual<N>& a) { return orc::chain(a, std::sin(a.v), std::cos(a.v)); }
template <int N> inline orc::Dual<N> pow(const orc::Dual<N>& a, const orc::Dual<N>& b) {
    // Only constant exponents occur on differentiable paths (Schlick's 5).
    const double r = std::pow(a.v, b.v);
    return orc::chain(a, r, b.v == 0 ? 0.0 : b.v * std::pow(a.v, b.v - 1.0));
}
template <int N> inline orc::Dual<N> fma(const orc::Dual<N>& a, const orc::Dual<N>& b, const orc::Dual<N>& c) { return a * b + c; }
template <int N> inline bool isnan(const orc::Dual<N>& a) { return std::isnan(a.v); }
template <int N> inline bool isinf(const orc::Dual<N>& a) { return std::isinf(a.v); }

inline orc::Shadow sqrt(const orc::Shadow& a) { return orc::Shadow(std::sqrt(a.b), std::sqrt(a.p)); }
inline orc::Shadow fabs(const orc::Shadow& a) { return a.b < 0 ? -a : a; }
inline orc::Shadow exp(const orc::Shadow& a) { return orc::Shadow(std::exp(a.b), std::exp(a.p)); }
inline orc::Shadow log(const orc::Shadow& a) { return orc::Shadow(std::log(a.b), std::log(a.p)); }
inline orc::Shadow cos(const orc::Shadow& a) { return orc::Shadow(std::cos(a.b), std::cos(a.p)); }
inline orc::Shadow sin(const orc::Shadow& a) { return orc::Shadow(std::sin(a.b), std::sin(a.p)); }
inline orc::Shadow pow(const orc::Shadow& a, const orc::Shadow& c) { return orc::Shadow(std::pow(a.b, c.b), std::pow(a.p, c.p)); }
inline orc::Shadow fma(const orc::Shadow& a, const orc::Shadow& b, const orc::Shadow& c) { return a * b + c; }
inline bool isnan(const orc::Shadow& a) { return std::isnan(a.b); }
inline bool isinf(const orc::Shadow& a) { return std::isinf(a.b); }
}  // namespace std
