/* Camera set-up of src/main.c:125-168 (frequency normalisation, native
 * camera coordinates, field of view, flux scale) plus the camera tetrad that
 * init_XK builds for every pixel (src/model_geodesics.c:186-190); it is
 * pixel independent, so it is built once here. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "../ipg_constants.h"
#include "coords.h"
#include "ipole_b200.h"

int ipg_camera_setup(const ipg_grid *grid, double rcam, double thetacam_deg, double phicam_deg, double rotcam_deg,
                     double fovx_muas, double fovy_muas, double dx_rg, double dy_rg, double dsource_pc, int nx, int ny,
                     double freqcgs, int old_centering, ipg_camera *cam, double *scale, double *DXo, double *DYo)
{
  if (!grid || !cam || nx <= 0 || ny <= 0 || !(rcam > 0)) return IPG_E_ARG;
  double freq = freqcgs * IPG_HPL / (IPG_ME * IPG_CL * IPG_CL);
  if (freq == 0) {
    fprintf(stderr, "Frequency cannot be zero. Quitting!\n");
    return IPG_E_ARG;
  }
  memset(cam, 0, sizeof(*cam));
  cam->rotcam = rotcam_deg * (M_PI / 180.);
  hc_native_coord(grid, rcam, thetacam_deg, phicam_deg, cam->Xcam);
  double Dsource = dsource_pc * IPG_PC;
  double fov_to_d = Dsource / grid->L_unit / IPG_MUAS_PER_RAD;
  if (fovx_muas != 0.0) {
    /* FOV given in muas */
  } else if (dx_rg != 0.0) {
    fovx_muas = dx_rg / fov_to_d;
    fovy_muas = dy_rg / fov_to_d;
  } else {
    fprintf(stderr, "No FOV was specified. Using default 160muas!\n");
    fovx_muas = 160.;
    fovy_muas = 160.;
  }
  double DX = fovx_muas * fov_to_d;
  double DY = fovy_muas * fov_to_d;
  cam->fovx = DX / rcam;
  cam->fovy = DY / rcam;
  if (scale) *scale = (DX * grid->L_unit / nx) * (DY * grid->L_unit / ny) / (Dsource * Dsource) / IPG_JY;
  if (DXo) *DXo = DX;
  if (DYo) *DYo = DY;
  cam->freq = freq;
  cam->freqcgs = freqcgs;
  cam->nx = nx;
  cam->ny = ny;
  cam->eps = 0.01;
  cam->maxnstep = 50000;
  cam->emission_type = 4;
  cam->target_nturns = -1;
  if (old_centering) hc_make_camera_tetrad_old(grid, cam->Xcam, cam->Econ, cam->Ecov);
  else hc_make_camera_tetrad(grid, cam->Xcam, cam->Econ, cam->Ecov);
  return IPG_OK;
}
