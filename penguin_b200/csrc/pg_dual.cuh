// First-order dual numbers (value, derivative along one seeded direction) for
// the adjoint kernels.  The hydro building blocks are templates on their scalar
// type; evaluated with Dual they give the exact derivative of the FP64 step
// along the branch its comparisons take (limiters, upwinding, HLLC wave signs,
// floors), which is the derivative a discrete adjoint must transpose.
//
// Comparisons and the selection functions (fmin, fmax, fabs, copysign,
// signbit) act on the value; the derivative follows the selected operand.
// The functions live in pg::ad, found by argument-dependent lookup, so plain
// double arithmetic elsewhere keeps resolving to the CUDA math library.
#pragma once

#include <cmath>

namespace pg {
namespace ad {

struct Dual {
    double v, d;
    Dual() = default;
    __host__ __device__ constexpr Dual(double a) : v(a), d(0.0) {}
    __host__ __device__ constexpr Dual(double a, double b) : v(a), d(b) {}
};

#define PG_AD __host__ __device__ __forceinline__

PG_AD Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
PG_AD Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
PG_AD Dual operator-(Dual a) { return {-a.v, -a.d}; }
PG_AD Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
PG_AD Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
PG_AD Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
PG_AD Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
PG_AD Dual& operator*=(Dual& a, Dual b) { return a = a * b; }
PG_AD Dual& operator/=(Dual& a, Dual b) { return a = a / b; }
PG_AD bool operator<(Dual a, Dual b) { return a.v < b.v; }
PG_AD bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
PG_AD bool operator>(Dual a, Dual b) { return a.v > b.v; }
PG_AD bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
PG_AD bool operator==(Dual a, Dual b) { return a.v == b.v; }
PG_AD bool operator!=(Dual a, Dual b) { return a.v != b.v; }

PG_AD Dual fmin(Dual a, Dual b) { return (b.v < a.v) ? b : a; }
PG_AD Dual fmax(Dual a, Dual b) { return (b.v > a.v) ? b : a; }
PG_AD Dual fabs(Dual a) { return std::signbit(a.v) ? Dual{-a.v, -a.d} : a; }
PG_AD Dual copysign(Dual a, Dual b) {
    const double r = std::copysign(a.v, b.v);
    return {r, (std::signbit(r) == std::signbit(a.v)) ? a.d : -a.d};
}
PG_AD bool signbit(Dual a) { return std::signbit(a.v); }
PG_AD Dual sqrt(Dual a) {
    const double s = std::sqrt(a.v);
    return {s, a.d == 0.0 ? 0.0 : 0.5 * a.d / s};
}
PG_AD Dual exp(Dual a) {
    const double e = std::exp(a.v);
    return {e, a.d * e};
}
PG_AD Dual pow(Dual a, double b) {
    const double p = std::pow(a.v, b);
    return {p, a.d == 0.0 ? 0.0 : a.d * b * std::pow(a.v, b - 1.0)};
}

#undef PG_AD

}  // namespace ad

// value part of a scalar of either type
__host__ __device__ __forceinline__ double val(double a) { return a; }
__host__ __device__ __forceinline__ double val(const ad::Dual& a) { return a.v; }

}  // namespace pg
