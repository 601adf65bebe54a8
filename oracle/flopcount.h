// flopcount.h -- operation counting for the CPU oracle (test and measurement
// infrastructure only; never part of the product).
//
// `make -C oracle count` compiles hosono_oracle.cpp a third time with this
// header included first and `double` defined as fc::CD: a one-double struct
// whose arithmetic performs the same IEEE double operation and increments a
// counter.  The struct is trivially copyable and 8 bytes, so the library's
// C functions keep their ABI (double arrays, double arguments and results
// pass and return in the same registers), and oracle.py loads it like the
// strict build.  Counters are plain globals: run the counting library with
// one OpenMP thread.
//
// Classes: add (+ and -), mul, div, sqrt; cmp (comparisons, min/max, fmin,
// fmax); other (fabs, negation, sin, classification).  Flops in the usual
// convention: add + mul + div + sqrt (an FMA would count 2; the strict build
// has none).
#pragma once

#include <omp.h>
#include <quadmath.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

namespace fc {

struct Counts {
    unsigned long long add, mul, div, sqrt, cmp, other;
};
// counts by phase of the time step, set by FC_PHASE markers in the oracle:
// 0 RK combines, boundary fills, CFL and the rest; 1 MOOD pass 1
// reconstruct + fluxes; 2 later passes' reconstruct + fluxes; 3 FLICD,
// update, detect and the MOOD flag sync
constexpr int NPHASE = 4;
inline Counts g_all[NPHASE] = {};
inline int g_phase = 0;
#define g_counts g_all[fc::g_phase]

struct CD {
    double v;
    CD() = default;
    constexpr CD(double x) : v(x) {}
    template <class T, class = typename std::enable_if<std::is_integral<T>::value>::type>
    constexpr CD(T x) : v((double)x) {}
    CD(__float128 q) : v((double)q) {}
    explicit operator double() const { return v; }
    explicit operator __float128() const { return (__float128)v; }
    template <class T, class = typename std::enable_if<std::is_integral<T>::value>::type>
    explicit operator T() const { return (T)v; }
    CD& operator+=(CD o) { g_counts.add++; v += o.v; return *this; }
    CD& operator-=(CD o) { g_counts.add++; v -= o.v; return *this; }
    CD& operator*=(CD o) { g_counts.mul++; v *= o.v; return *this; }
    CD& operator/=(CD o) { g_counts.div++; v /= o.v; return *this; }
};
static_assert(sizeof(CD) == sizeof(double) && std::is_trivially_copyable<CD>::value, "CD must be a plain double");

inline CD operator+(CD a, CD b) { g_counts.add++; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { g_counts.add++; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { g_counts.mul++; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { g_counts.div++; return CD(a.v / b.v); }
inline CD operator-(CD a) { g_counts.other++; return CD(-a.v); }
inline CD operator+(CD a) { return a; }
inline bool operator<(CD a, CD b) { g_counts.cmp++; return a.v < b.v; }
inline bool operator<=(CD a, CD b) { g_counts.cmp++; return a.v <= b.v; }
inline bool operator>(CD a, CD b) { g_counts.cmp++; return a.v > b.v; }
inline bool operator>=(CD a, CD b) { g_counts.cmp++; return a.v >= b.v; }
inline bool operator==(CD a, CD b) { g_counts.cmp++; return a.v == b.v; }
inline bool operator!=(CD a, CD b) { g_counts.cmp++; return a.v != b.v; }

// mixed operands: the other operand is a double or an integer, converted as
// the built-in operator would
#define FC_MIXED(OP)                                                                            \
    template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>     \
    inline auto operator OP(CD a, T b) -> decltype(a OP CD((double)b)) { return a OP CD((double)b); } \
    template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>     \
    inline auto operator OP(T a, CD b) -> decltype(CD((double)a) OP b) { return CD((double)a) OP b; }
FC_MIXED(+)
FC_MIXED(-)
FC_MIXED(*)
FC_MIXED(/)
FC_MIXED(<)
FC_MIXED(<=)
FC_MIXED(>)
FC_MIXED(>=)
FC_MIXED(==)
FC_MIXED(!=)
#undef FC_MIXED

}  // namespace fc

// the math functions the oracle calls as std::f(x)
namespace std {
inline fc::CD sqrt(fc::CD x) { fc::g_counts.sqrt++; return fc::CD(::sqrt(x.v)); }
inline fc::CD fabs(fc::CD x) { fc::g_counts.other++; return fc::CD(::fabs(x.v)); }
inline fc::CD copysign(fc::CD a, fc::CD b) { fc::g_counts.other++; return fc::CD(::copysign(a.v, b.v)); }
inline fc::CD copysign(double a, fc::CD b) { return std::copysign(fc::CD(a), b); }
inline fc::CD abs(fc::CD x) { fc::g_counts.other++; return fc::CD(::fabs(x.v)); }
inline fc::CD sin(fc::CD x) { fc::g_counts.other++; return fc::CD(::sin(x.v)); }
inline fc::CD fmax(fc::CD a, fc::CD b) { fc::g_counts.cmp++; return fc::CD(::fmax(a.v, b.v)); }
inline fc::CD fmin(fc::CD a, fc::CD b) { fc::g_counts.cmp++; return fc::CD(::fmin(a.v, b.v)); }
inline fc::CD fmax(fc::CD a, double b) { return std::fmax(a, fc::CD(b)); }
inline fc::CD fmax(double a, fc::CD b) { return std::fmax(fc::CD(a), b); }
inline fc::CD fmin(fc::CD a, double b) { return std::fmin(a, fc::CD(b)); }
inline fc::CD fmin(double a, fc::CD b) { return std::fmin(fc::CD(a), b); }
inline fc::CD max(fc::CD a, fc::CD b) { return (a < b) ? b : a; }
inline fc::CD min(fc::CD a, fc::CD b) { return (b < a) ? b : a; }
inline bool isnan(fc::CD x) { fc::g_counts.other++; return std::isnan(x.v); }
inline bool isfinite(fc::CD x) { fc::g_counts.other++; return std::isfinite(x.v); }
}  // namespace std

// the CFL loop's OpenMP max reduction over the counted type
#pragma omp declare reduction(max : fc::CD : omp_out = std::fmax(omp_out, omp_in)) initializer(omp_priv = omp_orig)

extern "C" {
// counters of the operations executed in one phase since the last reset
__attribute__((used, visibility("default"))) void orc_count_get(int phase, unsigned long long* c) {
    const fc::Counts& k = fc::g_all[phase < 0 || phase >= fc::NPHASE ? 0 : phase];
    c[0] = k.add;
    c[1] = k.mul;
    c[2] = k.div;
    c[3] = k.sqrt;
    c[4] = k.cmp;
    c[5] = k.other;
}
__attribute__((used, visibility("default"))) void orc_count_reset() {
    for (auto& k : fc::g_all) k = fc::Counts{0, 0, 0, 0, 0, 0};
    fc::g_phase = 0;
}
}

#define FC_PHASE(p) (fc::g_phase = (p))

#define double fc::CD
