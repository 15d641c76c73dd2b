/*
 * Forward-mode dual numbers for the adjoint (ipg_adjoint): a value and its
 * derivatives along D directions, carried through the thermal fits (the
 * directions ne, Theta_e, |B|) and through the polarized transfer step (the
 * Stokes vector and the coefficients).  Each operation applies the chain
 * rule exactly; the values are computed with the same operations as the
 * FP64 functions they shadow.
 */
#pragma once

#include <math.h>

template <int D>
struct Dual {
  double v;
  double d[D];
};

template <int D>
__device__ __forceinline__ Dual<D> dconst(double v)
{
  Dual<D> r;
  r.v = v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = 0.;
  return r;
}

template <int D>
__device__ __forceinline__ Dual<D> dvar(double v, int dir)
{
  Dual<D> r = dconst<D>(v);
  r.d[dir] = 1.;
  return r;
}

/* value and derivative of a function of one variable at x.v */
template <int D>
__device__ __forceinline__ Dual<D> dchain(const Dual<D> &x, double fv, double dfdx)
{
  Dual<D> r;
  r.v = fv;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = dfdx * x.d[k];
  return r;
}

template <int D>
__device__ __forceinline__ Dual<D> operator+(const Dual<D> &a, const Dual<D> &b)
{
  Dual<D> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator-(const Dual<D> &a, const Dual<D> &b)
{
  Dual<D> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator-(const Dual<D> &a)
{
  Dual<D> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = -a.d[k];
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator*(const Dual<D> &a, const Dual<D> &b)
{
  Dual<D> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
/* by division, not by a reciprocal: 1/b overflows for a subnormal b (the
 * Bessel functions of cold electrons), a/b does not */
template <int D>
__device__ __forceinline__ Dual<D> operator/(const Dual<D> &a, const Dual<D> &b)
{
  Dual<D> r;
  r.v = a.v / b.v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator+(const Dual<D> &a, double b)
{
  Dual<D> r = a;
  r.v = a.v + b;
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator+(double a, const Dual<D> &b)
{
  return b + a;
}
template <int D>
__device__ __forceinline__ Dual<D> operator-(const Dual<D> &a, double b)
{
  Dual<D> r = a;
  r.v = a.v - b;
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator-(double a, const Dual<D> &b)
{
  Dual<D> r;
  r.v = a - b.v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = -b.d[k];
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator*(const Dual<D> &a, double b)
{
  Dual<D> r;
  r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = a.d[k] * b;
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator*(double a, const Dual<D> &b)
{
  Dual<D> r;
  r.v = a * b.v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = a * b.d[k];
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator/(const Dual<D> &a, double b)
{
  Dual<D> r;
  r.v = a.v / b;
  const double ib = 1. / b;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = a.d[k] * ib;
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> operator/(double a, const Dual<D> &b)
{
  Dual<D> r;
  r.v = a / b.v;
  const double f = -r.v / b.v;
#pragma unroll
  for (int k = 0; k < D; k++) r.d[k] = f * b.d[k];
  return r;
}
template <int D>
__device__ __forceinline__ Dual<D> &operator+=(Dual<D> &a, const Dual<D> &b)
{
  a = a + b;
  return a;
}
template <int D>
__device__ __forceinline__ Dual<D> &operator-=(Dual<D> &a, const Dual<D> &b)
{
  a = a - b;
  return a;
}
template <int D>
__device__ __forceinline__ Dual<D> &operator*=(Dual<D> &a, const Dual<D> &b)
{
  a = a * b;
  return a;
}
template <int D>
__device__ __forceinline__ Dual<D> &operator*=(Dual<D> &a, double b)
{
  a = a * b;
  return a;
}
template <int D>
__device__ __forceinline__ Dual<D> &operator/=(Dual<D> &a, double b)
{
  a = a / b;
  return a;
}
template <int D>
__device__ __forceinline__ Dual<D> &operator/=(Dual<D> &a, const Dual<D> &b)
{
  a = a / b;
  return a;
}

/* comparisons act on the value: the branches of the fits follow the value */
template <int D> __device__ __forceinline__ bool operator<(const Dual<D> &a, double b) { return a.v < b; }
template <int D> __device__ __forceinline__ bool operator>(const Dual<D> &a, double b) { return a.v > b; }
template <int D> __device__ __forceinline__ bool operator<=(const Dual<D> &a, double b) { return a.v <= b; }
template <int D> __device__ __forceinline__ bool operator>=(const Dual<D> &a, double b) { return a.v >= b; }
template <int D> __device__ __forceinline__ bool operator<(const Dual<D> &a, const Dual<D> &b) { return a.v < b.v; }
template <int D> __device__ __forceinline__ bool operator>(const Dual<D> &a, const Dual<D> &b) { return a.v > b.v; }

template <int D>
__device__ __forceinline__ Dual<D> exp(const Dual<D> &x)
{
  const double e = exp(x.v);
  return dchain(x, e, e);
}
template <int D>
__device__ __forceinline__ Dual<D> log(const Dual<D> &x)
{
  return dchain(x, log(x.v), 1. / x.v);
}
/* At a zero argument (the k-B angle's sine along the field) the functions
 * below with an infinite slope there take the derivative 0: the argument is
 * then identically zero in every direction that occurs (sin theta = 0 does
 * not move with ne, Theta_e or |B|), and inf * 0 would poison the result. */
template <int D>
__device__ __forceinline__ Dual<D> sqrt(const Dual<D> &x)
{
  const double s = sqrt(x.v);
  return dchain(x, s, x.v == 0. ? 0. : 0.5 / s);
}
template <int D>
__device__ __forceinline__ Dual<D> rsqrt(const Dual<D> &x)
{
  const double s = rsqrt(x.v);
  return dchain(x, s, -0.5 * s / x.v);
}
template <int D>
__device__ __forceinline__ Dual<D> cbrt(const Dual<D> &x)
{
  const double c = cbrt(x.v);
  return dchain(x, c, x.v == 0. ? 0. : c / (3. * x.v));
}
template <int D>
__device__ __forceinline__ Dual<D> pow(const Dual<D> &x, double p)
{
  const double v = pow(x.v, p);
  return dchain(x, v, x.v == 0. ? 0. : p * v / x.v);
}
template <int D>
__device__ __forceinline__ Dual<D> tanh(const Dual<D> &x)
{
  const double t = tanh(x.v);
  return dchain(x, t, 1. - t * t);
}
template <int D>
__device__ __forceinline__ Dual<D> cos(const Dual<D> &x)
{
  return dchain(x, cos(x.v), -sin(x.v));
}
template <int D>
__device__ __forceinline__ Dual<D> sin(const Dual<D> &x)
{
  return dchain(x, sin(x.v), cos(x.v));
}
template <int D>
__device__ __forceinline__ Dual<D> fabs(const Dual<D> &x)
{
  return x.v < 0. ? -x : x;
}
template <int D>
__device__ __forceinline__ Dual<D> fmax(const Dual<D> &x, double b)
{
  return x.v >= b ? x : dconst<D>(b);
}
template <int D>
__device__ __forceinline__ void sincos(const Dual<D> &x, Dual<D> *s, Dual<D> *c)
{
  double sv, cv;
  sincos(x.v, &sv, &cv);
  *s = dchain(x, sv, cv);
  *c = dchain(x, cv, -sv);
}

/* value of a number of either kind */
__device__ __forceinline__ double val(double x) { return x; }
template <int D>
__device__ __forceinline__ double val(const Dual<D> &x)
{
  return x.v;
}
