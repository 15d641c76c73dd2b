/* Stand-in for GSL's <gsl/gsl_sf_hyperg.h> for the CPU oracle build (kappa fits only;
 * not reachable for emission_type 1 or 4).  The symbol aborts if called. */
#ifndef IPG_ORACLE_GSL_SF_HYPERG_H
#define IPG_ORACLE_GSL_SF_HYPERG_H
double gsl_sf_hyperg_2F1(double a, double b, double c, double x);
#endif
