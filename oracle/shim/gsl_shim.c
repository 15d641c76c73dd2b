/*
 * GSL replacements for the CPU oracle build of the reference (test
 * infrastructure; never part of the product library).
 *
 * The reference's thermal path calls gsl_sf_bessel_Kn(n, 1/Theta_e) for
 * n = 0, 1, 2 only (src/symphony/maxwell_juettner_fits.c:227,228,263,264,376).
 * GNU GSL is not vendored in the reference (makefile:76 links the system
 * -lgsl) and is absent here, so K_n is restated from published methods:
 *
 *   x <= 2 : the ascending series of Abramowitz & Stegun 9.6.11 (n = 0, 1);
 *   x >  2 : Temme's method / Steed's continued fraction CF2 for K_0 and K_1
 *            (N. M. Temme, J. Comput. Phys. 19, 324 (1975));
 *   n = 2  : upward recurrence K_2 = K_0 + (2/x) K_1 (stable for K).
 *
 * Accuracy is checked against scipy.special.kn (tests/test_oracle_bessel.py).
 * Where exp(-x) underflows (x > ~745) GSL would report an underflow error;
 * here the value is returned as 0.  The reference treats K2 <= 0 with its
 * own fallbacks (maxwell_juettner_fits.c:229,276,376).
 *
 * The remaining GSL symbols the reference links against are reachable only
 * for kappa, power-law or bremsstrahlung emission; they abort if called.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "gsl/gsl_sf_bessel.h"
#include "gsl/gsl_sf_expint.h"
#include "gsl/gsl_sf_hyperg.h"
#include "gsl/gsl_spline2d.h"

#define EULER_GAMMA 0.57721566490153286061

/* K0(x), K1(x) multiplied by exp(x), for x > 2 (Temme/Steed CF2, nu = 0). */
static void k01_scaled_cf2(double x, double *k0s, double *k1s)
{
  const double a1 = 0.25; /* 1/4 - nu^2 with nu = 0 */
  double b = 2.0 * (1.0 + x);
  double d = 1.0 / b;
  double delh = d, h = d;
  double q1 = 0.0, q2 = 1.0;
  double q = a1, c = a1;
  double a = -a1;
  double s = 1.0 + q * delh;
  for (int i = 2; i < 10000; i++) {
    a -= 2.0 * (i - 1);
    c = -a * c / i;
    double qnew = (q1 - b * q2) / a;
    q1 = q2;
    q2 = qnew;
    q += c * qnew;
    b += 2.0;
    d = 1.0 / (b + a * d);
    delh = (b * d - 1.0) * delh;
    h += delh;
    double dels = q * delh;
    s += dels;
    if (fabs(dels / s) < 1.0e-17) break;
  }
  h = a1 * h;
  double k0 = sqrt(M_PI / (2.0 * x)) / s;
  *k0s = k0;
  *k1s = k0 * (x + 0.5 - h) / x;
}

/* K0(x), K1(x) for 0 < x <= 2 by the ascending series (A&S 9.6.11). */
static void k01_series(double x, double *k0, double *k1)
{
  double y = 0.25 * x * x;
  double lg = log(0.5 * x);
  /* K0 = -(ln(x/2) + gamma) I0 + sum_k y^k/(k!)^2 H_k */
  double t = 1.0, i0 = 1.0, sum0 = 0.0, hk = 0.0;
  /* K1 = 1/x + ln(x/2) I1 - (x/4) sum_k y^k/(k!(k+1)!) (psi(k+1)+psi(k+2)) */
  double u = 1.0, i1s = 1.0, sum1 = 0.0;
  double psi1 = -EULER_GAMMA;       /* psi(k+1) at k = 0 */
  double psi2 = 1.0 - EULER_GAMMA;  /* psi(k+2) at k = 0 */
  sum1 = psi1 + psi2;
  for (int k = 1; k < 60; k++) {
    t *= y / ((double)k * k);
    hk += 1.0 / k;
    i0 += t;
    sum0 += t * hk;
    u *= y / ((double)k * (k + 1));
    psi1 += 1.0 / k;
    psi2 += 1.0 / (k + 1);
    i1s += u;
    sum1 += u * (psi1 + psi2);
    if (t < 1e-18 * i0 && u < 1e-18 * i1s) break;
  }
  *k0 = -(lg + EULER_GAMMA) * i0 + sum0;
  double i1 = 0.5 * x * i1s;
  *k1 = 1.0 / x + lg * i1 - 0.25 * x * sum1;
}

double gsl_sf_bessel_Kn(const int n, const double x)
{
  if (!(x > 0.0)) {
    fprintf(stderr, "gsl_sf_bessel_Kn shim: domain error x=%g\n", x);
    abort();
  }
  double k0, k1;
  if (x <= 2.0) {
    k01_series(x, &k0, &k1);
  } else {
    double k0s, k1s;
    k01_scaled_cf2(x, &k0s, &k1s);
    double ex = exp(-x);
    if (n == 2) {
      /* recurrence on the scaled values, then unscale */
      return (k0s + 2.0 / x * k1s) * ex;
    }
    k0 = k0s * ex;
    k1 = k1s * ex;
  }
  switch (n) {
    case 0: return k0;
    case 1: return k1;
    case 2: return k0 + 2.0 / x * k1;
    default:
      fprintf(stderr, "gsl_sf_bessel_Kn shim: order %d not provided\n", n);
      abort();
  }
}

double gsl_sf_hyperg_2F1(double a, double b, double c, double x)
{
  (void)a; (void)b; (void)c; (void)x;
  fprintf(stderr, "gsl_sf_hyperg_2F1 is not provided by the oracle shim (kappa fits)\n");
  abort();
}

double gsl_sf_expint_Ei(const double x)
{
  (void)x;
  fprintf(stderr, "gsl_sf_expint_Ei is not provided by the oracle shim (bremsstrahlung)\n");
  abort();
}

static const gsl_interp2d_type ipg_bilinear_stub = {0};
const gsl_interp2d_type *gsl_interp2d_bilinear = &ipg_bilinear_stub;

static void spline_abort(void)
{
  fprintf(stderr, "gsl spline2d is not provided by the oracle shim (bremsstrahlung)\n");
  abort();
}
gsl_interp_accel *gsl_interp_accel_alloc(void) { spline_abort(); return NULL; }
gsl_spline2d *gsl_spline2d_alloc(const gsl_interp2d_type *T, size_t xsize, size_t ysize)
{
  (void)T; (void)xsize; (void)ysize; spline_abort(); return NULL;
}
int gsl_spline2d_set(const gsl_spline2d *interp, double zarr[], const size_t i, const size_t j, const double z)
{
  (void)interp; (void)zarr; (void)i; (void)j; (void)z; spline_abort(); return 0;
}
int gsl_spline2d_init(gsl_spline2d *interp, const double xa[], const double ya[], const double za[],
                      size_t xsize, size_t ysize)
{
  (void)interp; (void)xa; (void)ya; (void)za; (void)xsize; (void)ysize; spline_abort(); return 0;
}
double gsl_spline2d_eval(const gsl_spline2d *interp, const double x, const double y,
                         gsl_interp_accel *xa, gsl_interp_accel *ya)
{
  (void)interp; (void)x; (void)y; (void)xa; (void)ya; spline_abort(); return 0.0;
}
