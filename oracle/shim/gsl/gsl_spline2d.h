/* Stand-in for GSL's <gsl/gsl_spline2d.h> for the CPU oracle build.  Every symbol
 * aborts if called; the bremsstrahlung path is off (bremss=0). */
#ifndef IPG_ORACLE_GSL_SPLINE2D_H
#define IPG_ORACLE_GSL_SPLINE2D_H
#include "gsl_interp2d.h"
typedef struct { int unused; } gsl_spline2d;
gsl_spline2d *gsl_spline2d_alloc(const gsl_interp2d_type *T, size_t xsize, size_t ysize);
int gsl_spline2d_set(const gsl_spline2d *interp, double zarr[], const size_t i, const size_t j, const double z);
int gsl_spline2d_init(gsl_spline2d *interp, const double xa[], const double ya[], const double za[],
                      size_t xsize, size_t ysize);
double gsl_spline2d_eval(const gsl_spline2d *interp, const double x, const double y,
                         gsl_interp_accel *xa, gsl_interp_accel *ya);
#endif
