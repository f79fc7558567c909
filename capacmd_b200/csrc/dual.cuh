// Forward-mode dual numbers for the gradient kernels.
//
// A Dual carries a value and its derivative along one direction of the
// positions.  The gradient kernels are templates over the scalar type: with
// double they evaluate a quantity, with Dual they also give its directional
// derivative, which the force-matching gradient needs (a Hessian-vector
// product of the energy, computed exactly instead of by differences).
#pragma once

#include <cmath>
#include <type_traits>

#include "device.cuh"

namespace capac {

using ::erf;
using ::erfc;
using ::exp;
using ::log;
using ::pow;
using ::sqrt;

struct Dual {
    double v, d;
};

__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b)
{
    const double q = a / b.v;
    return {q, -q * b.d / b.v};
}
__device__ __forceinline__ Dual &operator+=(Dual &a, Dual b)
{
    a.v += b.v;
    a.d += b.d;
    return a;
}
__device__ __forceinline__ Dual &operator-=(Dual &a, Dual b)
{
    a.v -= b.v;
    a.d -= b.d;
    return a;
}

__device__ __forceinline__ Dual sqrt(Dual a)
{
    const double s = ::sqrt(a.v);
    return {s, a.d / (2.0 * s)};
}
__device__ __forceinline__ Dual exp(Dual a)
{
    const double e = ::exp(a.v);
    return {e, e * a.d};
}
__device__ __forceinline__ Dual log(Dual a) { return {::log(a.v), a.d / a.v}; }
__device__ __forceinline__ Dual erf(Dual a) { return {::erf(a.v), 2.0 * kInvSqrtPi * ::exp(-a.v * a.v) * a.d}; }
__device__ __forceinline__ Dual erfc(Dual a) { return {::erfc(a.v), -2.0 * kInvSqrtPi * ::exp(-a.v * a.v) * a.d}; }
// x^p for a real exponent p (x > 0)
__device__ __forceinline__ Dual pow(Dual a, double p)
{
    const double y = ::pow(a.v, p);
    return {y, p * y / a.v * a.d};
}

__device__ __forceinline__ double val(double a) { return a; }
__device__ __forceinline__ double val(Dual a) { return a.v; }
__device__ __forceinline__ double der(double) { return 0.0; }
__device__ __forceinline__ double der(Dual a) { return a.d; }

template <class T>
__device__ __forceinline__ T lift(double v, double d)
{
    if constexpr (std::is_same<T, Dual>::value) return Dual{v, d};
    else return v;
}

// Number of doubles a T occupies in a reduction.
template <class T>
__host__ __device__ constexpr int width() { return std::is_same<T, Dual>::value ? 2 : 1; }

// Minimum image of a difference: the shift is decided on the values, as in
// the force kernels, and does not change the derivative.
template <class T>
__device__ __forceinline__ T zero() { return lift<T>(0.0, 0.0); }

template <class T>
__device__ __forceinline__ T warp_sum_t(T v)
{
    if constexpr (std::is_same<T, Dual>::value) return Dual{warp_sum(v.v), warp_sum(v.d)};
    else return warp_sum(v);
}

// Position of atom a; for Dual, with derivative wdir[3a .. 3a+2].
template <class T>
__device__ __forceinline__ void load_pos(const double4 *__restrict__ pos4, const double *__restrict__ wdir, int a,
                                         T (&r)[3])
{
    const double4 p = pos4[a];
    if constexpr (std::is_same<T, Dual>::value) {
        r[0] = Dual{p.x, wdir[3 * a]};
        r[1] = Dual{p.y, wdir[3 * a + 1]};
        r[2] = Dual{p.z, wdir[3 * a + 2]};
    } else {
        r[0] = p.x;
        r[1] = p.y;
        r[2] = p.z;
    }
}

__device__ __forceinline__ void set_val(double &a, double v) { a = v; }
__device__ __forceinline__ void set_val(Dual &a, double v) { a.v = v; }

template <class T>
__device__ __forceinline__ void image_t(T &x, T &y, T &z, const Box &b)
{
    double vx = val(x), vy = val(y), vz = val(z);
    image(vx, vy, vz, b);
    set_val(x, vx);
    set_val(y, vy);
    set_val(z, vz);
}

}  // namespace capac
