/* Host-side FMKS geometry for set-up code (camera, dump loading).
 *
 * These follow the reference's operation order (loops included) so that,
 * compiled without FMA contraction, the camera tetrad and the derived fluid
 * fields are bit-identical to the reference's on the same host.  The per-step
 * device versions live in ipg_device.cuh. */
#ifndef IPG_HOST_COORDS_H
#define IPG_HOST_COORDS_H
#include "ipole_b200.h"

#define NDIM 4

void hc_bl_coord(const ipg_grid *g, const double X[NDIM], double *r, double *th);
void hc_gcov_ks(const ipg_grid *g, double r, double th, double gcov[NDIM][NDIM]);
void hc_set_dxdX(const ipg_grid *g, const double X[NDIM], double dxdX[NDIM][NDIM]);
void hc_gcov_func(const ipg_grid *g, const double X[NDIM], double gcov[NDIM][NDIM]);
int hc_invert_matrix(const double Am[NDIM][NDIM], double Aminv[NDIM][NDIM]);
double hc_gdet_func(const double gcov[NDIM][NDIM]);
void hc_flip_index(const double ucon[NDIM], const double Gcov[NDIM][NDIM], double ucov[NDIM]);
int hc_make_plasma_tetrad(const double Ucon[NDIM], const double Kcon[NDIM], const double Bcon[NDIM],
                          const double Gcov[NDIM][NDIM], double Econ[NDIM][NDIM], double Ecov[NDIM][NDIM]);
int hc_make_camera_tetrad(const ipg_grid *g, const double X[NDIM], double Econ[NDIM][NDIM],
                          double Ecov[NDIM][NDIM]);
int hc_make_camera_tetrad_old(const ipg_grid *g, const double X[NDIM], double Econ[NDIM][NDIM],
                              double Ecov[NDIM][NDIM]);
void hc_native_coord(const ipg_grid *g, double r, double th_deg, double phi_deg, double X[NDIM]);
void hc_ijktoX(const ipg_grid *g, int i, int j, int k, double X[NDIM]);
double hc_gdet_zone(const ipg_grid *g, int i, int j, int k);
#endif
