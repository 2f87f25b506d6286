// fv_dual.cuh -- forward-mode dual numbers for the tangent (JVP) kernels.
//
// A Dual carries a value and one directional derivative. Arithmetic and the elementary functions
// propagate the derivative by the chain rule; comparisons, min/max and branch decisions use the
// value only, so a Dual evaluation follows exactly the branches of the primal evaluation (the
// derivative is that of the active branch: subgradient convention at the limiter's min and at the
// flux splittings' |M| = 1 switches).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace abl {

struct Dual {
    double v, d;
    __host__ __device__ constexpr Dual() : v(0), d(0) {}
    __host__ __device__ constexpr Dual(double x) : v(x), d(0) {}
    __host__ __device__ constexpr Dual(double x, double dx) : v(x), d(dx) {}
    __host__ __device__ explicit operator double() const { return v; }
    __host__ __device__ Dual& operator+=(const Dual& o) {
        v += o.v;
        d += o.d;
        return *this;
    }
    __host__ __device__ Dual& operator-=(const Dual& o) {
        v -= o.v;
        d -= o.d;
        return *this;
    }
    __host__ __device__ Dual& operator*=(const Dual& o) {
        d = d * o.v + v * o.d;
        v *= o.v;
        return *this;
    }
    __host__ __device__ Dual& operator/=(const Dual& o) {
        const double q = v / o.v;
        d = (d - q * o.d) / o.v;
        v = q;
        return *this;
    }
};

#define ABL_DD __host__ __device__ __forceinline__

ABL_DD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
ABL_DD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
ABL_DD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
ABL_DD Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
ABL_DD Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
ABL_DD Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
ABL_DD Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
ABL_DD Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
ABL_DD Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
ABL_DD Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
ABL_DD Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
ABL_DD Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
ABL_DD Dual operator/(double a, Dual b) {
    const double q = a / b.v;
    return Dual(q, -q * b.d / b.v);
}
ABL_DD bool operator<(Dual a, Dual b) { return a.v < b.v; }
ABL_DD bool operator>(Dual a, Dual b) { return a.v > b.v; }
ABL_DD bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
ABL_DD bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
ABL_DD bool operator==(Dual a, Dual b) { return a.v == b.v; }
ABL_DD bool operator!=(Dual a, Dual b) { return a.v != b.v; }
ABL_DD bool operator<(Dual a, double b) { return a.v < b; }
ABL_DD bool operator>(Dual a, double b) { return a.v > b; }
ABL_DD bool operator<=(Dual a, double b) { return a.v <= b; }
ABL_DD bool operator>=(Dual a, double b) { return a.v >= b; }
ABL_DD bool operator==(Dual a, double b) { return a.v == b; }
ABL_DD bool operator!=(Dual a, double b) { return a.v != b; }
ABL_DD bool operator<(double a, Dual b) { return a < b.v; }
ABL_DD bool operator>(double a, Dual b) { return a > b.v; }
ABL_DD bool operator<=(double a, Dual b) { return a <= b.v; }
ABL_DD bool operator>=(double a, Dual b) { return a >= b.v; }

// Elementary functions under the d-prefixed names the generic physics code calls (plain names such as
// sqrt would hide the double overloads inside namespace abl).
ABL_DD Dual dsqrt(Dual a) {
    const double s = ::sqrt(a.v);
    return Dual(s, a.v > 0 ? 0.5 * a.d / s : 0.0);
}
ABL_DD Dual dabs(Dual a) { return a.v < 0 ? -a : a; }
ABL_DD Dual dpow(Dual a, Dual b) {
    // b is a constant exponent everywhere this is used (gamma ratios)
    const double p = ::pow(a.v, b.v);
    return Dual(p, a.v != 0 ? b.v * p / a.v * a.d : 0.0);
}
ABL_DD Dual dsin(Dual a) { return Dual(::sin(a.v), ::cos(a.v) * a.d); }
ABL_DD Dual rcp64(Dual a) { return 1.0 / a; }
ABL_DD bool dfinite(Dual a) { return ::isfinite(a.v) && ::isfinite(a.d); }

// value / tangent accessors that also work on plain doubles
ABL_DD double dval(double a) { return a; }
ABL_DD double dval(Dual a) { return a.v; }
ABL_DD double dtangent(double) { return 0.0; }
ABL_DD double dtangent(Dual a) { return a.d; }

}  // namespace abl

namespace abl {

// N-direction forward dual: value + gradient with respect to N seeded inputs. Used to obtain the full
// local Jacobian of a flux calculator (8 scalar inputs -> mass flux, interface pressure) in one pass
// for the adjoint kernels; like Dual, every branch follows the value.
template <int N>
struct DualN {
    double v;
    double d[N];
    __host__ __device__ DualN() : v(0) {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0;
    }
    __host__ __device__ DualN(double x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0;
    }
    __host__ __device__ static DualN seed(double x, int i) {
        DualN r(x);
        r.d[i] = 1.0;
        return r;
    }
    __host__ __device__ explicit operator double() const { return v; }
};

template <int N>
ABL_DD DualN<N> lin(double a, const DualN<N>& x, double b, const DualN<N>& y, double value) {
    DualN<N> r(value);
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a * x.d[i] + b * y.d[i];
    return r;
}
template <int N>
ABL_DD DualN<N> scale(double a, const DualN<N>& x, double value) {
    DualN<N> r(value);
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a * x.d[i];
    return r;
}
template <int N>
ABL_DD DualN<N> operator+(const DualN<N>& a, const DualN<N>& b) { return lin(1.0, a, 1.0, b, a.v + b.v); }
template <int N>
ABL_DD DualN<N> operator-(const DualN<N>& a, const DualN<N>& b) { return lin(1.0, a, -1.0, b, a.v - b.v); }
template <int N>
ABL_DD DualN<N> operator*(const DualN<N>& a, const DualN<N>& b) { return lin(b.v, a, a.v, b, a.v * b.v); }
template <int N>
ABL_DD DualN<N> operator/(const DualN<N>& a, const DualN<N>& b) {
    const double q = a.v / b.v;
    return lin(1.0 / b.v, a, -q / b.v, b, q);
}
template <int N>
ABL_DD DualN<N> operator-(const DualN<N>& a) { return scale(-1.0, a, -a.v); }
template <int N>
ABL_DD DualN<N> operator+(const DualN<N>& a, double b) { return scale(1.0, a, a.v + b); }
template <int N>
ABL_DD DualN<N> operator+(double a, const DualN<N>& b) { return scale(1.0, b, a + b.v); }
template <int N>
ABL_DD DualN<N> operator-(const DualN<N>& a, double b) { return scale(1.0, a, a.v - b); }
template <int N>
ABL_DD DualN<N> operator-(double a, const DualN<N>& b) { return scale(-1.0, b, a - b.v); }
template <int N>
ABL_DD DualN<N> operator*(const DualN<N>& a, double b) { return scale(b, a, a.v * b); }
template <int N>
ABL_DD DualN<N> operator*(double a, const DualN<N>& b) { return scale(a, b, a * b.v); }
template <int N>
ABL_DD DualN<N> operator/(const DualN<N>& a, double b) { return scale(1.0 / b, a, a.v / b); }
template <int N>
ABL_DD DualN<N> operator/(double a, const DualN<N>& b) {
    const double q = a / b.v;
    return scale(-q / b.v, b, q);
}
template <int N>
ABL_DD DualN<N>& operator+=(DualN<N>& a, const DualN<N>& b) { return a = a + b; }
template <int N>
ABL_DD DualN<N>& operator-=(DualN<N>& a, const DualN<N>& b) { return a = a - b; }
template <int N>
ABL_DD DualN<N>& operator*=(DualN<N>& a, const DualN<N>& b) { return a = a * b; }
template <int N>
ABL_DD DualN<N>& operator/=(DualN<N>& a, const DualN<N>& b) { return a = a / b; }
template <int N>
ABL_DD bool operator<(const DualN<N>& a, const DualN<N>& b) { return a.v < b.v; }
template <int N>
ABL_DD bool operator>(const DualN<N>& a, const DualN<N>& b) { return a.v > b.v; }
template <int N>
ABL_DD bool operator<=(const DualN<N>& a, const DualN<N>& b) { return a.v <= b.v; }
template <int N>
ABL_DD bool operator>=(const DualN<N>& a, const DualN<N>& b) { return a.v >= b.v; }
template <int N>
ABL_DD bool operator<(const DualN<N>& a, double b) { return a.v < b; }
template <int N>
ABL_DD bool operator>(const DualN<N>& a, double b) { return a.v > b; }
template <int N>
ABL_DD bool operator<=(const DualN<N>& a, double b) { return a.v <= b; }
template <int N>
ABL_DD bool operator>=(const DualN<N>& a, double b) { return a.v >= b; }
template <int N>
ABL_DD DualN<N> dsqrt(const DualN<N>& a) {
    const double s = ::sqrt(a.v);
    return scale(a.v > 0 ? 0.5 / s : 0.0, a, s);
}
template <int N>
ABL_DD DualN<N> dabs(const DualN<N>& a) { return a.v < 0 ? -a : a; }
template <int N>
ABL_DD DualN<N> dpow(const DualN<N>& a, const DualN<N>& b) {
    const double p = ::pow(a.v, b.v);  // constant exponent
    return scale(a.v != 0 ? b.v * p / a.v : 0.0, a, p);
}
template <int N>
ABL_DD DualN<N> rcp64(const DualN<N>& a) { return 1.0 / a; }

}  // namespace abl
