/*
 * Test infrastructure for the golden noise floor (oracle/Makefile target
 * `noise`, build _ref/ipole_ulp).  The reference calls the C library's
 * transcendental functions; IEEE 754 does not require them to be correctly
 * rounded, and two faithful implementations (glibc on the CPU, CUDA's libm on
 * the GPU) may return neighbouring doubles for the same argument.  This file
 * wraps the ones on the reference's path (linked with -Wl,--wrap=...) and moves
 * each result by -1, 0 or +1 ulp, chosen by a hash of the argument bits, so
 * that the reference can be run "with another equally accurate libm".  The
 * spread of that build around the reference's own is part of the noise floor
 * recorded with each golden image.  The environment variable IPG_ULP_SALT (an
 * integer, default 0) selects another hash, i.e. another such libm, so that
 * several independent ones can be sampled.  Never linked into the product.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline uint64_t bits(double x)
{
  uint64_t u;
  memcpy(&u, &x, sizeof(u));
  return u;
}

/* splitmix64 finaliser: a fixed, well-mixed function of the argument bits */
static inline uint64_t mix(uint64_t z)
{
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

/* read once at start-up, before the OpenMP threads exist */
static uint64_t g_salt = 0;
__attribute__((constructor)) static void read_salt(void)
{
  const char *e = getenv("IPG_ULP_SALT");
  const unsigned long long v = e ? strtoull(e, NULL, 10) : 0;
  g_salt = v ? mix(v + 0x5bd1e995ULL) : 0;
}
static inline uint64_t salt(void) { return g_salt; }

static inline double nudge(double r, uint64_t key)
{
  if (!isfinite(r) || r == 0.) return r;
  switch (mix(key ^ salt()) % 3) {
    case 0: return nextafter(r, -INFINITY);
    case 1: return nextafter(r, INFINITY);
    default: return r;
  }
}

#define WRAP1(f, salt)                                           \
  double __real_##f(double);                                     \
  double __wrap_##f(double x) { return nudge(__real_##f(x), bits(x) ^ (salt)); }

/* functions whose values lie in [-1, 1]: a faithful libm never leaves that
 * range, so neither does the nudge */
static inline double nudge_unit(double r, uint64_t key)
{
  const double v = nudge(r, key);
  return v > 1. ? 1. : (v < -1. ? -1. : v);
}

#define WRAP1U(f, salt)                                          \
  double __real_##f(double);                                     \
  double __wrap_##f(double x) { return nudge_unit(__real_##f(x), bits(x) ^ (salt)); }

WRAP1U(sin, 0x11)
WRAP1U(cos, 0x22)
WRAP1(tan, 0x33)
WRAP1(exp, 0x44)
WRAP1(log, 0x55)
WRAP1(log10, 0x66)
WRAP1(atan, 0x77)
WRAP1U(tanh, 0x88)
/* and the inverse functions stay in their ranges [-pi/2, pi/2], [0, pi] */
double __real_asin(double);
double __wrap_asin(double x)
{
  const double v = nudge(__real_asin(x), bits(x) ^ 0x99);
  return fmax(-M_PI_2, fmin(M_PI_2, v));
}
double __real_acos(double);
double __wrap_acos(double x)
{
  const double v = nudge(__real_acos(x), bits(x) ^ 0xaa);
  return fmax(0., fmin(M_PI, v));
}
WRAP1(cbrt, 0xbb)

double __real_pow(double, double);
double __wrap_pow(double x, double y)
{
  double r = __real_pow(x, y);
  /* integer powers small enough to be exact stay exact, as they are in any
   * careful libm */
  if (y == floor(y) && fabs(y) <= 3.) return r;
  return nudge(r, bits(x) * 31 ^ bits(y) ^ 0xcc);
}

double __real_atan2(double, double);
double __wrap_atan2(double y, double x) { return nudge(__real_atan2(y, x), bits(y) * 17 ^ bits(x) ^ 0xdd); }

void __real_sincos(double, double *, double *);
void __wrap_sincos(double x, double *s, double *c)
{
  __real_sincos(x, s, c);
  *s = nudge_unit(*s, bits(x) ^ 0x11);
  *c = nudge_unit(*c, bits(x) ^ 0x22);
}
