/* Stand-in for GSL's <gsl/gsl_sf_bessel.h> for the CPU oracle build.
 * gsl_sf_bessel_Kn is implemented in oracle/shim/gsl_shim.c (n = 0, 1, 2). */
#ifndef IPG_ORACLE_GSL_SF_BESSEL_H
#define IPG_ORACLE_GSL_SF_BESSEL_H
double gsl_sf_bessel_Kn(const int n, const double x);
#endif
