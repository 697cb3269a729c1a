// Forward-mode dual numbers for the discrete adjoint: Dual<N> carries a value
// and N tangents.  The adjoint kernels evaluate each element function (Roe
// flux of one face, gradient + limiter of one cell, boundary state of one
// ghost, time step of one cell) on Dual<4> inputs seeded with the identity on
// the 4 conserved variables of one stencil cell, which gives that cell's
// 4-column block of the element Jacobian; its transpose times the incoming
// adjoint is the cell's contribution.  Branches (min, max, abs, limiter
// regions, boundary regimes) follow the primal values, as the discrete
// derivative of the primal code path.
#pragma once
#include <math.h>

#ifndef FV_HD
#define FV_HD __host__ __device__ __forceinline__
#endif

namespace fvgpu {

// the double overloads stay visible next to the Dual templates below
using ::fabs;
using ::sqrt;

template <int N>
struct Dual {
    double v;
    double d[N];
    FV_HD Dual() : v(0.0) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    FV_HD Dual(double x) : v(x) {  // a constant
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0.0;
    }
    FV_HD Dual& operator+=(const Dual& b) {
        v += b.v;
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] += b.d[i];
        return *this;
    }
    FV_HD Dual& operator-=(const Dual& b) {
        v -= b.v;
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] -= b.d[i];
        return *this;
    }
    FV_HD Dual& operator*=(double s) {
        v *= s;
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] *= s;
        return *this;
    }
    FV_HD Dual& operator*=(const Dual& b) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = d[i] * b.v + v * b.d[i];
        v *= b.v;
        return *this;
    }
};

template <int N> FV_HD Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r; r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N> FV_HD Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> FV_HD Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> FV_HD Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> FV_HD Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N> FV_HD Dual<N> operator+(const Dual<N>& a, double b) { Dual<N> r = a; r.v += b; return r; }
template <int N> FV_HD Dual<N> operator+(double a, const Dual<N>& b) { Dual<N> r = b; r.v += a; return r; }
template <int N> FV_HD Dual<N> operator-(const Dual<N>& a, double b) { Dual<N> r = a; r.v -= b; return r; }
template <int N> FV_HD Dual<N> operator-(double a, const Dual<N>& b) { Dual<N> r = -b; r.v += a; return r; }
template <int N> FV_HD Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r; r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int N> FV_HD Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N> FV_HD Dual<N> operator/(const Dual<N>& a, double b) {
    Dual<N> r; r.v = a.v / b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / b;
    return r;
}
template <int N> FV_HD Dual<N> operator/(double a, const Dual<N>& b) {
    Dual<N> r; r.v = a / b.v;
    const double s = -r.v / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = s * b.d[i];
    return r;
}
template <int N> FV_HD bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N> FV_HD bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N> FV_HD bool operator<=(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v; }
template <int N> FV_HD bool operator>=(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v; }
template <int N> FV_HD bool operator<(const Dual<N>& a, double b) { return a.v < b; }
template <int N> FV_HD bool operator>(const Dual<N>& a, double b) { return a.v > b; }
template <int N> FV_HD bool operator<=(const Dual<N>& a, double b) { return a.v <= b; }
template <int N> FV_HD bool operator>=(const Dual<N>& a, double b) { return a.v >= b; }
template <int N> FV_HD bool operator<(double a, const Dual<N>& b) { return a < b.v; }
template <int N> FV_HD bool operator>(double a, const Dual<N>& b) { return a > b.v; }

template <int N> FV_HD Dual<N> sqrt(const Dual<N>& a) {
    Dual<N> r; r.v = ::sqrt(a.v);
    const double s = 0.5 / r.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
    return r;
}
template <int N> FV_HD Dual<N> fabs(const Dual<N>& a) { return a.v < 0.0 ? -a : a; }
// std::min / std::max semantics of the primal (ties keep the first argument)
template <int N> FV_HD Dual<N> dmin(const Dual<N>& a, const Dual<N>& b) { return (b.v < a.v) ? b : a; }
template <int N> FV_HD Dual<N> dmax(const Dual<N>& a, const Dual<N>& b) { return (a.v < b.v) ? b : a; }

FV_HD double value(double x) { return x; }
template <int N> FV_HD double value(const Dual<N>& x) { return x.v; }

}  // namespace fvgpu
