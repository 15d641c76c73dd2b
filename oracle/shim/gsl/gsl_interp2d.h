/* Stand-in for GSL's <gsl/gsl_interp2d.h> for the CPU oracle build (bremsstrahlung
 * spline only; src/symphony/bremss_fits.c init body is compiled out). */
#ifndef IPG_ORACLE_GSL_INTERP2D_H
#define IPG_ORACLE_GSL_INTERP2D_H
#include <stddef.h>
typedef struct { int unused; } gsl_interp2d_type;
typedef struct { int unused; } gsl_interp_accel;
extern const gsl_interp2d_type *gsl_interp2d_bilinear;
gsl_interp_accel *gsl_interp_accel_alloc(void);
#endif
