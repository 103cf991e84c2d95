// qem_dual.cuh -- forward-mode dual numbers (value + NT tangents) in FP64 for
// the adjoint kernels.
//
// A Dual<NT> carries a value and its derivatives with respect to NT chosen
// inputs.  Running a pair or self evaluation on Duals seeded with unit
// tangents gives that evaluation's exact local Jacobian (quadrature limits
// that move with the image distance included), which the adjoint kernels
// contract with the incoming cotangents.
#pragma once

#include <cuda_runtime.h>

template <int NT>
struct Dual {
    double v;
    double d[NT];
};

template <int NT>
__device__ __forceinline__ Dual<NT> dconst(double v)
{
    Dual<NT> r;
    r.v = v;
#pragma unroll
    for (int t = 0; t < NT; t++) r.d[t] = 0.0;
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> dvar(double v, int t0)
{
    Dual<NT> r = dconst<NT>(v);
    r.d[t0] = 1.0;
    return r;
}
// r = f(x) with f'(x) = df
template <int NT>
__device__ __forceinline__ Dual<NT> dchain(const Dual<NT> &x, double f, double df)
{
    Dual<NT> r;
    r.v = f;
#pragma unroll
    for (int t = 0; t < NT; t++) r.d[t] = df * x.d[t];
    return r;
}

template <int NT>
__device__ __forceinline__ Dual<NT> operator+(const Dual<NT> &a, const Dual<NT> &b)
{
    Dual<NT> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int t = 0; t < NT; t++) r.d[t] = a.d[t] + b.d[t];
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> operator-(const Dual<NT> &a, const Dual<NT> &b)
{
    Dual<NT> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int t = 0; t < NT; t++) r.d[t] = a.d[t] - b.d[t];
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> operator-(const Dual<NT> &a)
{
    Dual<NT> r;
    r.v = -a.v;
#pragma unroll
    for (int t = 0; t < NT; t++) r.d[t] = -a.d[t];
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> operator*(const Dual<NT> &a, const Dual<NT> &b)
{
    Dual<NT> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int t = 0; t < NT; t++) r.d[t] = a.d[t] * b.v + a.v * b.d[t];
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> operator/(const Dual<NT> &a, const Dual<NT> &b)
{
    Dual<NT> r;
    const double ib = 1.0 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int t = 0; t < NT; t++) r.d[t] = (a.d[t] - r.v * b.d[t]) * ib;
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> operator+(const Dual<NT> &a, double b)
{
    Dual<NT> r = a;
    r.v += b;
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> operator+(double b, const Dual<NT> &a) { return a + b; }
template <int NT>
__device__ __forceinline__ Dual<NT> operator-(const Dual<NT> &a, double b)
{
    Dual<NT> r = a;
    r.v -= b;
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> operator-(double b, const Dual<NT> &a) { return -a + b; }
template <int NT>
__device__ __forceinline__ Dual<NT> operator*(const Dual<NT> &a, double b)
{
    Dual<NT> r;
    r.v = a.v * b;
#pragma unroll
    for (int t = 0; t < NT; t++) r.d[t] = a.d[t] * b;
    return r;
}
template <int NT>
__device__ __forceinline__ Dual<NT> operator*(double b, const Dual<NT> &a) { return a * b; }
template <int NT>
__device__ __forceinline__ Dual<NT> operator/(const Dual<NT> &a, double b) { return a * (1.0 / b); }
template <int NT>
__device__ __forceinline__ Dual<NT> operator/(double a, const Dual<NT> &b)
{
    const double ib = 1.0 / b.v;
    return dchain(b, a * ib, -a * ib * ib);
}
template <int NT>
__device__ __forceinline__ Dual<NT> &operator+=(Dual<NT> &a, const Dual<NT> &b)
{
    a = a + b;
    return a;
}
template <int NT>
__device__ __forceinline__ Dual<NT> &operator-=(Dual<NT> &a, const Dual<NT> &b)
{
    a = a - b;
    return a;
}

template <int NT>
__device__ __forceinline__ Dual<NT> exp(const Dual<NT> &x)
{
    const double e = ::exp(x.v);
    return dchain(x, e, e);
}
template <int NT>
__device__ __forceinline__ Dual<NT> sqrt(const Dual<NT> &x)
{
    const double s = ::sqrt(x.v);
    return dchain(x, s, s > 0.0 ? 0.5 / s : 0.0);
}
template <int NT>
__device__ __forceinline__ Dual<NT> fabs(const Dual<NT> &x)
{
    return dchain(x, ::fabs(x.v), (double)((x.v > 0) - (x.v < 0)));
}
// J0 and J1 together: J0' = -J1, J1' = J0 - J1 / x (1/2 at x = 0)
template <int NT>
__device__ __forceinline__ void bessel01(const Dual<NT> &x, Dual<NT> &J0, Dual<NT> &J1)
{
    const double j0v = ::j0(x.v), j1v = ::j1(x.v);
    J0 = dchain(x, j0v, -j1v);
    J1 = dchain(x, j1v, x.v != 0.0 ? j0v - j1v / x.v : 0.5);
}
__device__ __forceinline__ void bessel01(double x, double &J0, double &J1)
{
    J0 = ::j0(x);
    J1 = ::j1(x);
}

__device__ __forceinline__ double dval(double x) { return x; }
template <int NT>
__device__ __forceinline__ double dval(const Dual<NT> &x) { return x.v; }
