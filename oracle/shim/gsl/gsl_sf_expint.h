/* Stand-in for GSL's <gsl/gsl_sf_expint.h> for the CPU oracle build (bremsstrahlung
 * only; not reachable with bremss=0).  The symbol aborts if called. */
#ifndef IPG_ORACLE_GSL_SF_EXPINT_H
#define IPG_ORACLE_GSL_SF_EXPINT_H
double gsl_sf_expint_Ei(const double x);
#endif
