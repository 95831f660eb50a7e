// running_error.hpp -- test infrastructure for the oracle: a bound on the
// rounding error of an f32 evaluation of a variation body.
//
// RE carries a double value and a first-order bound on the absolute error an
// f32 evaluation of the same expression accumulates, in units of the f32
// epsilon 2^-23 (Wilkinson's running error analysis).  Each basic operation
// propagates its operands' bounds through its derivative and adds half an
// ulp of its result; each library function adds three ulps of its result
// (the device's and the host's libm each within two).  Comparisons,
// floor and the like act on the value: a result on the far side of a
// branch or a step from its f32 twin is outside what the bound covers, so
// each one taken within its operands' bounds (the values closer than the
// bounds' sum, or an integer step inside [v - e, v + e]) marks the
// evaluation undecided (re_undecided()): an f32 twin may have taken the
// other side, and the caller treats the point's result as arbitrary.
//
// The variation bodies are templates over their arithmetic type; the
// std:: overloads below let the same source run over RE, so each body's
// bound follows its own operation order.
#pragma once

#include <algorithm>
#include <cmath>

struct RE {
    double v = 0, e = 0;
    RE() = default;
    RE(double value, double err) : v(value), e(err) {}
    RE(double value) : v(value), e(0) {}   // NOLINT: exact constants and inputs
    RE(float value) : v(value), e(0) {}    // NOLINT
    RE(int value) : v(value), e(0) {}      // NOLINT
    explicit operator double() const { return v; }
    explicit operator float() const { return (float)v; }
    RE& operator+=(const RE& o);
    RE& operator-=(const RE& o);
    RE& operator*=(const RE& o);
    RE& operator/=(const RE& o);
};

constexpr double kF32Eps = 1.0 / 8388608.0;

// Set by a comparison or an integer step taken within the bounds; the
// caller clears it before an evaluation and reads it after.
inline bool& re_undecided() {
    static thread_local bool flag = false;
    return flag;
}
// (The bounds are in units of the f32 epsilon.)
inline void re_compare(const RE& a, const RE& b) {
    const double e = (a.e + b.e) * kF32Eps;
    if (e > 0 && std::fabs(a.v - b.v) <= e) re_undecided() = true;
}
// An integer step (floor, ceil, trunc, rounding) between v - e and v + e.
template <class F> inline void re_step(const RE& a, F f) {
    const double e = a.e * kF32Eps;
    if (e > 0 && f(a.v - e) != f(a.v + e)) re_undecided() = true;
}

inline RE re_round(double v, double e, double ulps) { return {v, e + ulps * std::fabs(v)}; }
inline RE operator+(const RE& a, const RE& b) { return re_round(a.v + b.v, a.e + b.e, 0.5); }
inline RE operator-(const RE& a, const RE& b) { return re_round(a.v - b.v, a.e + b.e, 0.5); }
inline RE operator-(const RE& a) { return {-a.v, a.e}; }
inline RE operator*(const RE& a, const RE& b) {
    return re_round(a.v * b.v, std::fabs(a.v) * b.e + std::fabs(b.v) * a.e, 0.5);
}
inline RE operator/(const RE& a, const RE& b) {
    const double d = b.v == 0 ? 0.0 : b.v, v = a.v / d;
    if (d == 0 || !std::isfinite(v)) return {v, 0.0};
    return re_round(v, (a.e + std::fabs(v) * b.e) / std::fabs(d), 0.5);
}
inline RE& RE::operator+=(const RE& o) { return *this = *this + o; }
inline RE& RE::operator-=(const RE& o) { return *this = *this - o; }
inline RE& RE::operator*=(const RE& o) { return *this = *this * o; }
inline RE& RE::operator/=(const RE& o) { return *this = *this / o; }
inline bool operator<(const RE& a, const RE& b) { re_compare(a, b); return a.v < b.v; }
inline bool operator>(const RE& a, const RE& b) { re_compare(a, b); return a.v > b.v; }
inline bool operator<=(const RE& a, const RE& b) { re_compare(a, b); return a.v <= b.v; }
inline bool operator>=(const RE& a, const RE& b) { re_compare(a, b); return a.v >= b.v; }
inline bool operator==(const RE& a, const RE& b) { re_compare(a, b); return a.v == b.v; }
inline bool operator!=(const RE& a, const RE& b) { re_compare(a, b); return a.v != b.v; }

// f(a) with derivative d at a: the propagated bound plus three ulps.
inline RE re_fn(double v, double d, const RE& a) { return re_round(v, std::fabs(d) * a.e, 3.0); }
// A root-like function whose derivative is unbounded where its argument's
// error reaches the singularity: bounded by the function of the error.
inline double re_cap(double lin, double e, double k) { return std::min(lin, std::sqrt(k * e / kF32Eps)); }

namespace std {
inline RE sin(const RE& a) { return re_fn(std::sin(a.v), std::cos(a.v), a); }
inline RE cos(const RE& a) { return re_fn(std::cos(a.v), std::sin(a.v), a); }
inline RE tan(const RE& a) { const double t = std::tan(a.v); return re_fn(t, 1 + t * t, a); }
inline RE sinh(const RE& a) { return re_fn(std::sinh(a.v), std::cosh(a.v), a); }
inline RE cosh(const RE& a) { return re_fn(std::cosh(a.v), std::sinh(a.v), a); }
inline RE tanh(const RE& a) { const double t = std::tanh(a.v); return re_fn(t, 1 - t * t, a); }
inline RE exp(const RE& a) { const double v = std::exp(a.v); return re_fn(v, v, a); }
inline RE exp2(const RE& a) { const double v = std::exp2(a.v); return re_fn(v, v * 0.6931471805599453, a); }
inline RE log(const RE& a) { return re_fn(std::log(a.v), a.v != 0 ? 1 / a.v : 0.0, a); }
inline RE atan(const RE& a) { return re_fn(std::atan(a.v), 1 / (1 + a.v * a.v), a); }
inline RE atan2(const RE& y, const RE& x) {
    const double v = std::atan2(y.v, x.v), r2 = x.v * x.v + y.v * y.v;
    return re_round(v, r2 > 0 ? (std::fabs(x.v) * y.e + std::fabs(y.v) * x.e) / r2 : 0.0, 3.0);
}
inline RE sqrt(const RE& a) {
    const double v = std::sqrt(a.v);
    return re_round(v, re_cap(v > 0 ? a.e / (2 * v) : 1e300, a.e, 1.0), 0.5);
}
inline RE acos(const RE& a) {
    const double s = std::sqrt(std::max(1 - a.v * a.v, 0.0));
    return re_round(std::acos(a.v), re_cap(s > 0 ? a.e / s : 1e300, a.e, 2.0), 3.0);
}
inline RE asin(const RE& a) {
    const double s = std::sqrt(std::max(1 - a.v * a.v, 0.0));
    return re_round(std::asin(a.v), re_cap(s > 0 ? a.e / s : 1e300, a.e, 2.0), 3.0);
}
inline RE acosh(const RE& a) {
    const double s = std::sqrt(std::max(a.v * a.v - 1, 0.0));
    return re_round(std::acosh(a.v), re_cap(s > 0 ? a.e / s : 1e300, a.e, 2.0), 3.0);
}
inline RE pow(const RE& a, const RE& b) {
    const double v = std::pow(a.v, b.v);
    if (!std::isfinite(v)) return {v, 0.0};
    const double da = a.v != 0 ? b.v * v / a.v : 0.0, db = a.v > 0 ? v * std::log(a.v) : 0.0;
    return re_round(v, std::fabs(da) * a.e + std::fabs(db) * b.e, 3.0);
}
inline RE fabs(const RE& a) { return {std::fabs(a.v), a.e}; }
inline RE abs(const RE& a) { return {std::fabs(a.v), a.e}; }
inline RE fmax(const RE& a, const RE& b) { return a.v >= b.v || std::isnan(b.v) ? a : b; }
inline RE fmin(const RE& a, const RE& b) { return a.v <= b.v || std::isnan(b.v) ? a : b; }
inline RE floor(const RE& a) { re_step(a, [](double t) { return std::floor(t); }); return {std::floor(a.v), 0.0}; }
inline RE ceil(const RE& a) { re_step(a, [](double t) { return std::ceil(t); }); return {std::ceil(a.v), 0.0}; }
inline RE trunc(const RE& a) { re_step(a, [](double t) { return std::trunc(t); }); return {std::trunc(a.v), 0.0}; }
inline RE nearbyint(const RE& a) { re_step(a, [](double t) { return std::nearbyint(t); }); return {std::nearbyint(a.v), 0.0}; }
inline RE fmod(const RE& a, const RE& b) {
    const double v = std::fmod(a.v, b.v), n = b.v != 0 ? std::trunc(a.v / b.v) : 0.0;
    if (b.v != 0 && a.e > 0 && std::trunc((a.v - a.e * kF32Eps) / b.v) != std::trunc((a.v + a.e * kF32Eps) / b.v))
        re_undecided() = true;
    return re_round(v, a.e + std::fabs(n) * b.e, 0.5);
}
inline bool signbit(const RE& a) { return std::signbit(a.v); }
inline bool isnan(const RE& a) { return std::isnan(a.v); }
inline bool isfinite(const RE& a) { return std::isfinite(a.v); }
}  // namespace std
