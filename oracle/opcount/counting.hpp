/*
 * Operation counting for the oracle's restatement of the reference
 * (TEST INFRASTRUCTURE ONLY): a double that counts every arithmetic
 * operation done on it, and a complex type over it, so that compiling
 * oracle.c against them (make_counting_source.py) counts the reference
 * algorithm's own operations per ray step.
 *
 * Counted per scope (the innermost function scope, see ORC_SCOPE): adds and
 * subtracts, multiplies, divides, square roots, and calls of transcendental
 * functions (exp, log, pow, sin, cos, tan, atan2, tanh, acos, cbrt and the
 * Bessel K_n of the fits).  Comparisons, fabs/fmin/fmax and conversions are
 * not counted.
 */
#pragma once

#include <cmath>
#include <cstring>

enum { OC_ADD = 0, OC_MUL, OC_DIV, OC_SQRT, OC_TRANS, OC_N };
enum { SC_GEO = 0, SC_PUSH, SC_COEF, SC_STEP, SC_EVOLVE, SC_PROJ, SC_OTHER, SC_N };

struct OpCounts {
  long long c[SC_N][OC_N];
  long long calls[SC_N];
};
static OpCounts g_oc;
static int g_scope = SC_OTHER;

struct ScopeGuard {
  int prev;
  explicit ScopeGuard(int s) : prev(g_scope)
  {
    g_scope = s;
    g_oc.calls[s]++;
  }
  ~ScopeGuard() { g_scope = prev; }
};
#define ORC_SCOPE(s) ScopeGuard orc_scope_guard_(s)

static inline void oc_count(int op) { g_oc.c[g_scope][op]++; }

struct oreal {
  double v;
  oreal() : v(0.) {}
  oreal(double x) : v(x) {}
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
  explicit operator long() const { return (long)v; }
  oreal &operator+=(const oreal &b) { oc_count(OC_ADD); v += b.v; return *this; }
  oreal &operator-=(const oreal &b) { oc_count(OC_ADD); v -= b.v; return *this; }
  oreal &operator*=(const oreal &b) { oc_count(OC_MUL); v *= b.v; return *this; }
  oreal &operator/=(const oreal &b) { oc_count(OC_DIV); v /= b.v; return *this; }
  oreal operator-() const { return oreal(-v); }
  oreal operator+() const { return *this; }
};
static inline oreal operator+(oreal a, oreal b) { oc_count(OC_ADD); return oreal(a.v + b.v); }
static inline oreal operator-(oreal a, oreal b) { oc_count(OC_ADD); return oreal(a.v - b.v); }
static inline oreal operator*(oreal a, oreal b) { oc_count(OC_MUL); return oreal(a.v * b.v); }
static inline oreal operator/(oreal a, oreal b) { oc_count(OC_DIV); return oreal(a.v / b.v); }
static inline oreal operator+(oreal a, double b) { return a + oreal(b); }
static inline oreal operator+(double a, oreal b) { return oreal(a) + b; }
static inline oreal operator-(oreal a, double b) { return a - oreal(b); }
static inline oreal operator-(double a, oreal b) { return oreal(a) - b; }
static inline oreal operator*(oreal a, double b) { return a * oreal(b); }
static inline oreal operator*(double a, oreal b) { return oreal(a) * b; }
static inline oreal operator/(oreal a, double b) { return a / oreal(b); }
static inline oreal operator/(double a, oreal b) { return oreal(a) / b; }
static inline oreal operator+(oreal a, int b) { return a + oreal(b); }
static inline oreal operator+(int a, oreal b) { return oreal(a) + b; }
static inline oreal operator-(oreal a, int b) { return a - oreal(b); }
static inline oreal operator-(int a, oreal b) { return oreal(a) - b; }
static inline oreal operator*(oreal a, int b) { return a * oreal(b); }
static inline oreal operator*(int a, oreal b) { return oreal(a) * b; }
static inline oreal operator/(oreal a, int b) { return a / oreal(b); }
static inline oreal operator/(int a, oreal b) { return oreal(a) / b; }
#define OC_CMP(op)                                                                 \
  static inline bool operator op(oreal a, oreal b) { return a.v op b.v; }          \
  static inline bool operator op(oreal a, double b) { return a.v op b; }           \
  static inline bool operator op(double a, oreal b) { return a op b.v; }           \
  static inline bool operator op(oreal a, int b) { return a.v op (double)b; }      \
  static inline bool operator op(int a, oreal b) { return (double)a op b.v; }
OC_CMP(<)
OC_CMP(>)
OC_CMP(<=)
OC_CMP(>=)
OC_CMP(==)
OC_CMP(!=)
#undef OC_CMP

#define OC_T1(f)                                                                   \
  static inline oreal f(oreal x) { oc_count(OC_TRANS); return oreal(std::f(x.v)); }
OC_T1(exp)
OC_T1(log)
OC_T1(sin)
OC_T1(cos)
OC_T1(tan)
OC_T1(tanh)
OC_T1(acos)
OC_T1(asin)
OC_T1(atan)
OC_T1(cbrt)
OC_T1(log10)
#undef OC_T1
static inline oreal pow(oreal x, oreal y) { oc_count(OC_TRANS); return oreal(std::pow(x.v, y.v)); }
static inline oreal pow(oreal x, double y) { return pow(x, oreal(y)); }
static inline oreal pow(double x, oreal y) { return pow(oreal(x), y); }
static inline oreal atan2(oreal y, oreal x) { oc_count(OC_TRANS); return oreal(std::atan2(y.v, x.v)); }
static inline oreal sqrt(oreal x) { oc_count(OC_SQRT); return oreal(std::sqrt(x.v)); }
static inline oreal fabs(oreal x) { return oreal(std::fabs(x.v)); }
static inline oreal fmin(oreal a, oreal b) { return oreal(std::fmin(a.v, b.v)); }
static inline oreal fmax(oreal a, oreal b) { return oreal(std::fmax(a.v, b.v)); }
static inline oreal fmin(oreal a, double b) { return oreal(std::fmin(a.v, b)); }
static inline oreal fmax(oreal a, double b) { return oreal(std::fmax(a.v, b)); }
static inline oreal fmin(double a, oreal b) { return oreal(std::fmin(a, b.v)); }
static inline oreal fmax(double a, oreal b) { return oreal(std::fmax(a, b.v)); }
static inline oreal fmod(oreal a, oreal b) { oc_count(OC_DIV); return oreal(std::fmod(a.v, b.v)); }
static inline bool isnan(oreal x) { return std::isnan(x.v); }
static inline bool isinf(oreal x) { return std::isinf(x.v); }
static inline bool isfinite(oreal x) { return std::isfinite(x.v); }
static inline void sincos(oreal x, oreal *s, oreal *c)
{
  oc_count(OC_TRANS);
  *s = oreal(std::sin(x.v));
  *c = oreal(std::cos(x.v));
}

/* the complex numbers of the coherency tensor */
struct ocplx {
  oreal re, im;
  ocplx() {}
  ocplx(oreal r) : re(r), im(0.) {}
  ocplx(double r) : re(r), im(0.) {}
  ocplx(int r) : re((double)r), im(0.) {}
  ocplx(oreal r, oreal i) : re(r), im(i) {}
  ocplx &operator+=(const ocplx &b) { re += b.re; im += b.im; return *this; }
  ocplx &operator-=(const ocplx &b) { re -= b.re; im -= b.im; return *this; }
};
static inline ocplx operator+(ocplx a, ocplx b) { return ocplx(a.re + b.re, a.im + b.im); }
static inline ocplx operator-(ocplx a, ocplx b) { return ocplx(a.re - b.re, a.im - b.im); }
static inline ocplx operator-(ocplx a) { return ocplx(-a.re, -a.im); }
static inline ocplx operator*(ocplx a, ocplx b)
{
  return ocplx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline ocplx operator*(oreal a, ocplx b) { return ocplx(a * b.re, a * b.im); }
static inline ocplx operator*(ocplx a, oreal b) { return ocplx(a.re * b, a.im * b); }
static inline ocplx operator*(double a, ocplx b) { return oreal(a) * b; }
static inline ocplx operator*(ocplx a, double b) { return a * oreal(b); }
static inline ocplx operator+(ocplx a, oreal b) { return ocplx(a.re + b, a.im); }
static inline ocplx operator+(oreal a, ocplx b) { return ocplx(a + b.re, b.im); }
static inline ocplx operator-(ocplx a, oreal b) { return ocplx(a.re - b, a.im); }
static inline ocplx operator-(oreal a, ocplx b) { return ocplx(a - b.re, -b.im); }
static inline ocplx operator+(ocplx a, double b) { return a + oreal(b); }
static inline ocplx operator+(double a, ocplx b) { return oreal(a) + b; }
static inline ocplx operator-(ocplx a, double b) { return a - oreal(b); }
static inline ocplx operator-(double a, ocplx b) { return oreal(a) - b; }
static inline ocplx operator/(ocplx a, oreal b) { return ocplx(a.re / b, a.im / b); }
static inline ocplx operator/(ocplx a, double b) { return a / oreal(b); }
static inline oreal ocreal(ocplx z) { return z.re; }
static inline oreal ocimag(ocplx z) { return z.im; }
static inline ocplx oconj(ocplx z) { return ocplx(z.re, -z.im); }
static const ocplx OC_I(oreal(0.), oreal(1.));
static inline bool isnan(ocplx z) { return isnan(z.re) || isnan(z.im); }

/* the Bessel K_n of the thermal fits (gsl_sf_bessel_Kn, the shim's) */
static inline oreal gsl_sf_bessel_Kn(int n, oreal x)
{
  oc_count(OC_TRANS);
  return oreal(::gsl_sf_bessel_Kn(n, (double)x));
}
