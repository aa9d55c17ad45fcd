// opcount.hpp -- an arithmetic type that counts operations (test and measurement infrastructure only).
//
// orc::CR wraps a double and counts every floating-point operation the oracle's statements perform on
// it.  Instantiating the restatement (rrtm_lw.hpp, rrtm_sw.hpp) with R = CR gives the operation-count
// table of the reference algorithm, which fixes the algorithmic FLOPs per column used for the roofline.
// Counting rule: + - * / one FLOP each (the reference statements carry no explicit fma); exp, log, sqrt
// and pow one FLOP each (counted apart as well); negation, comparisons, min/max/abs are not FLOPs and are
// counted apart.  Table lookups and integer index arithmetic are not counted.
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>

namespace orc {

struct OpCounts {
    uint64_t add = 0, mul = 0, div = 0, func = 0, other = 0;
    uint64_t flops() const { return add + mul + div + func; }
};
extern OpCounts g_ops;

struct CR {
    double v = 0;
    CR() = default;
    CR(double x) : v(x) {}
    explicit operator double() const { return v; }
    explicit operator float() const { return (float)v; }
    explicit operator int() const { return (int)v; }
    CR& operator+=(CR b) { ++g_ops.add; v += b.v; return *this; }
    CR& operator-=(CR b) { ++g_ops.add; v -= b.v; return *this; }
    CR& operator*=(CR b) { ++g_ops.mul; v *= b.v; return *this; }
    CR& operator/=(CR b) { ++g_ops.div; v /= b.v; return *this; }
};
inline CR operator+(CR a, CR b) { ++g_ops.add; return CR(a.v + b.v); }
inline CR operator-(CR a, CR b) { ++g_ops.add; return CR(a.v - b.v); }
inline CR operator*(CR a, CR b) { ++g_ops.mul; return CR(a.v * b.v); }
inline CR operator/(CR a, CR b) { ++g_ops.div; return CR(a.v / b.v); }
inline CR operator-(CR a) { return CR(-a.v); }
inline bool operator<(CR a, CR b) { ++g_ops.other; return a.v < b.v; }
inline bool operator>(CR a, CR b) { ++g_ops.other; return a.v > b.v; }
inline bool operator<=(CR a, CR b) { ++g_ops.other; return a.v <= b.v; }
inline bool operator>=(CR a, CR b) { ++g_ops.other; return a.v >= b.v; }
inline bool operator==(CR a, CR b) { ++g_ops.other; return a.v == b.v; }
inline bool operator!=(CR a, CR b) { ++g_ops.other; return a.v != b.v; }

template <> inline CR fminR<CR>(CR a, CR b) { ++g_ops.other; return CR(std::fmin(a.v, b.v)); }
template <> inline CR fmaxR<CR>(CR a, CR b) { ++g_ops.other; return CR(std::fmax(a.v, b.v)); }
template <> inline CR fmod1<CR>(CR a) { ++g_ops.add; return CR(std::fmod(a.v, 1.0)); }
template <> inline CR mexp<CR>(CR a) { ++g_ops.func; return CR(std::exp(a.v)); }
template <> inline CR mlog<CR>(CR a) { ++g_ops.func; return CR(std::log(a.v)); }
template <> inline CR msqrt<CR>(CR a) { ++g_ops.func; return CR(std::sqrt(a.v)); }
template <> inline CR mfabs<CR>(CR a) { ++g_ops.other; return CR(std::fabs(a.v)); }
template <> inline CR mpow<CR>(CR a, CR b) { ++g_ops.func; return CR(std::pow(a.v, b.v)); }

}  // namespace orc

namespace std {
template <>
struct numeric_limits<orc::CR> : numeric_limits<double> {
    static orc::CR min() noexcept { return orc::CR(numeric_limits<double>::min()); }
};
}  // namespace std
