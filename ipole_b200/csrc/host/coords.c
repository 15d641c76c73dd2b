/* Host-side geometry (FMKS, and the MKS / flat metrics of the known-answer
 * models) for set-up code.  Each function follows the
 * operation order of the reference function it names (cited), so that the
 * camera tetrad and derived fluid fields match the reference bit for bit when
 * both are compiled without FMA contraction. */
#include "coords.h"

#include <math.h>
#include <string.h>

#define SMALL 1.e-40

/* src/coordinates.c:46-97 (METRIC_MINKOWSKI, EMINKOWSKI, MKS, FMKS branches) */
void hc_bl_coord(const ipg_grid *g, const double X[NDIM], double *r, double *th)
{
  if (g->metric == IPG_METRIC_MINKOWSKI) {
    *r = X[1];
    *th = X[2];
    return;
  } else if (g->metric == IPG_METRIC_EMINKOWSKI) {
    *r = exp(X[1]);
    *th = X[2];
    return;
  }
  *r = exp(X[1]);
  if (g->metric == IPG_METRIC_MKS) {
    *th = M_PI * X[2] + ((1. - g->hslope) / 2.) * sin(2. * M_PI * X[2]);
    return;
  }
  double thG = M_PI * X[2] + ((1. - g->hslope) / 2.) * sin(2. * M_PI * X[2]);
  double y = 2 * X[2] - 1.;
  double thJ = g->poly_norm * y * (1. + pow(y / g->poly_xt, g->poly_alpha) / (g->poly_alpha + 1.)) + 0.5 * M_PI;
  *th = thG + exp(g->mks_smooth * (g->startx[1] - X[1])) * (thJ - thG);
}

/* src/coordinates.c:216-239 */
void hc_gcov_ks(const ipg_grid *g, double r, double th, double gcov[NDIM][NDIM])
{
  const double a = g->a;
  double cth = cos(th);
  double sth = sin(th);
  double s2 = sth * sth;
  double rho2 = r * r + a * a * cth * cth;
  memset(gcov, 0, sizeof(double) * 16);
  gcov[0][0] = -1. + 2. * r / rho2;
  gcov[0][1] = 2. * r / rho2;
  gcov[0][3] = -2. * a * r * s2 / rho2;
  gcov[1][0] = gcov[0][1];
  gcov[1][1] = 1. + 2. * r / rho2;
  gcov[1][3] = -a * s2 * (1. + 2. * r / rho2);
  gcov[2][2] = rho2;
  gcov[3][0] = gcov[0][3];
  gcov[3][1] = gcov[1][3];
  gcov[3][3] = s2 * (rho2 + a * a * s2 * (1. + 2. * r / rho2));
}

/* src/coordinates.c:263-348 (METRIC_FMKS, MKS, MINKOWSKI, EMINKOWSKI branches) */
void hc_set_dxdX(const ipg_grid *g, const double X[NDIM], double dxdX[NDIM][NDIM])
{
  const double hslope = g->hslope, poly_xt = g->poly_xt, poly_alpha = g->poly_alpha;
  const double mks_smooth = g->mks_smooth, poly_norm = g->poly_norm;
  for (int mu = 0; mu < NDIM; mu++)
    for (int nu = 0; nu < NDIM; nu++) dxdX[mu][nu] = (mu == nu);
  dxdX[1][1] = exp(X[1]);
  if (g->metric == IPG_METRIC_MKS) {
    dxdX[2][2] = M_PI + (1 - hslope) * M_PI * cos(2. * M_PI * X[2]);
    return;
  } else if (g->metric == IPG_METRIC_MINKOWSKI) {
    dxdX[1][1] = 1.;
    return;
  } else if (g->metric == IPG_METRIC_EMINKOWSKI) {
    return;
  }
  dxdX[2][1] = -exp(mks_smooth * (g->startx[1] - X[1])) * mks_smooth *
               (M_PI / 2. - M_PI * X[2] +
                poly_norm * (2. * X[2] - 1.) * (1 + (pow((-1. + 2 * X[2]) / poly_xt, poly_alpha)) / (1 + poly_alpha)) -
                1. / 2. * (1. - hslope) * sin(2. * M_PI * X[2]));
  dxdX[2][2] = M_PI + (1. - hslope) * M_PI * cos(2. * M_PI * X[2]) +
               exp(mks_smooth * (g->startx[1] - X[1])) *
                   (-M_PI + 2. * poly_norm * (1. + pow((2. * X[2] - 1.) / poly_xt, poly_alpha) / (poly_alpha + 1.)) +
                    (2. * poly_alpha * poly_norm * (2. * X[2] - 1.) * pow((2. * X[2] - 1.) / poly_xt, poly_alpha - 1.)) /
                        ((1. + poly_alpha) * poly_xt) -
                    (1. - hslope) * M_PI * cos(2. * M_PI * X[2]));
}

/* src/coordinates.c:175-213 */
void hc_gcov_func(const ipg_grid *g, const double X[NDIM], double gcov[NDIM][NDIM])
{
  double r, th;
  hc_bl_coord(g, X, &r, &th);
  if (g->metric == IPG_METRIC_MINKOWSKI || g->metric == IPG_METRIC_EMINKOWSKI) {
    memset(gcov, 0, sizeof(double) * 16);
    gcov[0][0] = -1;
    gcov[1][1] = (g->metric == IPG_METRIC_MINKOWSKI) ? 1 : r * r;
    gcov[2][2] = r * r;
    gcov[3][3] = r * r * sin(th) * sin(th);
    return;
  }
  double Gcov_ks[NDIM][NDIM];
  hc_gcov_ks(g, r, th, Gcov_ks);
  double dxdX[NDIM][NDIM];
  hc_set_dxdX(g, X, dxdX);
  for (int mu = 0; mu < NDIM; mu++)
    for (int nu = 0; nu < NDIM; nu++) {
      gcov[mu][nu] = 0;
      for (int lam = 0; lam < NDIM; ++lam)
        for (int kap = 0; kap < NDIM; ++kap) gcov[mu][nu] += Gcov_ks[lam][kap] * dxdX[lam][mu] * dxdX[kap][nu];
    }
}

/* Crout LU with implicit partial pivoting, src/geometry.c:304-457 */
static int lu_decompose(double A[NDIM][NDIM], int permute[NDIM])
{
  const double absmin = 1.e-30;
  double row_norm[NDIM];
  double absmax, maxtemp;
  int max_row = 0;
  const int n = NDIM;
  for (int i = 0; i < n; i++) {
    absmax = 0.;
    for (int j = 0; j < n; j++) {
      maxtemp = fabs(A[i][j]);
      if (maxtemp > absmax) absmax = maxtemp;
    }
    if (absmax == 0.) return 1;
    row_norm[i] = 1. / absmax;
  }
  for (int j = 0; j < n; j++) {
    for (int i = 0; i < j; i++)
      for (int k = 0; k < i; k++) A[i][j] -= A[i][k] * A[k][j];
    absmax = 0.0;
    for (int i = j; i < n; i++) {
      for (int k = 0; k < j; k++) A[i][j] -= A[i][k] * A[k][j];
      maxtemp = fabs(A[i][j]) * row_norm[i];
      if (maxtemp >= absmax) {
        absmax = maxtemp;
        max_row = i;
      }
    }
    if (max_row != j) {
      if ((j == (n - 2)) && (A[j][j + 1] == 0.)) {
        max_row = j;
      } else {
        for (int k = 0; k < n; k++) {
          maxtemp = A[j][k];
          A[j][k] = A[max_row][k];
          A[max_row][k] = maxtemp;
        }
        row_norm[max_row] = row_norm[j];
      }
    }
    permute[j] = max_row;
    if (A[j][j] == 0.) A[j][j] = absmin;
    if (j != (n - 1)) {
      maxtemp = 1. / A[j][j];
      for (int i = (j + 1); i < n; i++) A[i][j] *= maxtemp;
    }
  }
  return 0;
}

/* src/geometry.c:471-504 */
static void lu_substitution(double A[NDIM][NDIM], double B[NDIM], const int permute[NDIM])
{
  const int n = NDIM;
  double tmpvar;
  for (int i = 0; i < n; i++) {
    tmpvar = B[permute[i]];
    B[permute[i]] = B[i];
    for (int j = (i - 1); j >= 0; j--) tmpvar -= A[i][j] * B[j];
    B[i] = tmpvar;
  }
  for (int i = (n - 1); i >= 0; i--) {
    for (int j = (i + 1); j < n; j++) B[i] -= A[i][j] * B[j];
    B[i] /= A[i][i];
  }
}

/* src/geometry.c:252-287 */
int hc_invert_matrix(const double Am[NDIM][NDIM], double Aminv[NDIM][NDIM])
{
  int permute[NDIM];
  double dxm[NDIM], Amtmp[NDIM][NDIM];
  memcpy(Amtmp, Am, sizeof(Amtmp));
  if (lu_decompose(Amtmp, permute) != 0) return 1;
  for (int i = 0; i < NDIM; i++) {
    for (int j = 0; j < NDIM; j++) dxm[j] = 0.;
    dxm[i] = 1.;
    lu_substitution(Amtmp, dxm, permute);
    for (int j = 0; j < NDIM; j++) Aminv[j][i] = dxm[j];
  }
  return 0;
}

/* src/geometry.c:26-51 */
double hc_gdet_func(const double gcov[NDIM][NDIM])
{
  int permute[NDIM];
  double t[NDIM][NDIM];
  memcpy(t, gcov, sizeof(t));
  if (lu_decompose(t, permute) != 0) return -1;
  double gdet = 1.;
  for (int i = 0; i < NDIM; i++) gdet *= t[i][i];
  return sqrt(fabs(gdet));
}

/* src/geometry.c:66-87 */
void hc_flip_index(const double ucon[NDIM], const double Gcov[NDIM][NDIM], double ucov[NDIM])
{
  for (int m = 0; m < NDIM; m++)
    ucov[m] = Gcov[m][0] * ucon[0] + Gcov[m][1] * ucon[1] + Gcov[m][2] * ucon[2] + Gcov[m][3] * ucon[3];
}

/* src/geometry.c:151-166 */
static void normalize(double vcon[NDIM], const double Gcov[NDIM][NDIM])
{
  double norm = 0.;
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++) norm += vcon[k] * vcon[l] * Gcov[k][l];
  norm = sqrt(fabs(norm));
  for (int k = 0; k < 4; k++) vcon[k] /= norm;
}

/* src/tetrads.c:95-115 */
static void project_out(double vcona[NDIM], const double vconb[NDIM], const double Gcov[NDIM][NDIM])
{
  double vconb_sq = 0., adotb = 0.;
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++) vconb_sq += vconb[k] * vconb[l] * Gcov[k][l];
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++) adotb += vcona[k] * vconb[l] * Gcov[k][l];
  for (int k = 0; k < 4; k++) vcona[k] -= vconb[k] * adotb / vconb_sq;
}

/* src/tetrads.c:40-54 */
static void set_Econ_from_trial(double Econ[4], int defdir, const double trial[4])
{
  double norm = 0.;
  for (int k = 1; k < 4; k++) norm += fabs(trial[k]);
  for (int k = 0; k < 4; k++) Econ[k] = (norm <= SMALL) ? (double)(k == defdir) : trial[k];
}

/* src/geometry.c:205-232 */
static int levi_civita(int i, int j, int k, int l)
{
  if (i == j || i == k || i == l || j == k || j == l || k == l) return 0;
  int idx[4] = {i, j, k, l}, n_perm = 0, swapped = 1;
  while (swapped) {
    swapped = 0;
    for (int n = 0; n < 3; n++)
      if (idx[n] > idx[n + 1]) {
        int t = idx[n];
        idx[n] = idx[n + 1];
        idx[n + 1] = t;
        n_perm++;
        swapped++;
      }
  }
  return (n_perm % 2) ? -1 : 1;
}

/* src/tetrads.c:64-87 */
static int check_handedness(const double Econ[NDIM][NDIM], const double Gcov[NDIM][NDIM], double *dot)
{
  double g = hc_gdet_func(Gcov);
  if (g < 0.) return 1;
  *dot = 0.;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int l = 0; l < 4; l++)
        for (int k = 0; k < 4; k++)
          *dot += g * levi_civita(i, j, k, l) * Econ[0][i] * Econ[1][j] * Econ[2][k] * Econ[3][l];
  return 0;
}

/* src/model_tetrads.c:35-127 */
int hc_make_plasma_tetrad(const double Ucon[NDIM], const double Kcon[NDIM], const double Bcon[NDIM],
                          const double Gcov[NDIM][NDIM], double Econ[NDIM][NDIM], double Ecov[NDIM][NDIM])
{
  const double ones[NDIM] = {1., 1., 1., 1.};
  set_Econ_from_trial(Econ[0], 0, Ucon);
  set_Econ_from_trial(Econ[1], 3, ones);
  set_Econ_from_trial(Econ[2], 2, Bcon);
  set_Econ_from_trial(Econ[3], 3, Kcon);
  normalize(Econ[0], Gcov);
  project_out(Econ[3], Econ[0], Gcov);
  project_out(Econ[3], Econ[0], Gcov);
  normalize(Econ[3], Gcov);
  project_out(Econ[2], Econ[0], Gcov);
  project_out(Econ[2], Econ[3], Gcov);
  project_out(Econ[2], Econ[0], Gcov);
  project_out(Econ[2], Econ[3], Gcov);
  normalize(Econ[2], Gcov);
  project_out(Econ[1], Econ[0], Gcov);
  project_out(Econ[1], Econ[2], Gcov);
  project_out(Econ[1], Econ[3], Gcov);
  project_out(Econ[1], Econ[0], Gcov);
  project_out(Econ[1], Econ[2], Gcov);
  project_out(Econ[1], Econ[3], Gcov);
  normalize(Econ[1], Gcov);
  int oddflag = 0;
  double dot = 0.;
  if (check_handedness(Econ, Gcov, &dot)) oddflag |= 16;
  if (fabs(fabs(dot) - 1.) > 1.e-10) oddflag |= 1;
  if (dot < 0.)
    for (int k = 0; k < 4; k++) Econ[1][k] *= -1.;
  for (int k = 0; k < 4; k++) hc_flip_index(Econ[k], Gcov, Ecov[k]);
  for (int l = 0; l < 4; l++) Ecov[0][l] *= -1.;
  return oddflag;
}

/* src/model_tetrads.c:143-193 */
int hc_make_camera_tetrad(const ipg_grid *g, const double X[NDIM], double Econ[NDIM][NDIM],
                          double Ecov[NDIM][NDIM])
{
  double Gcov[NDIM][NDIM], Gcon[NDIM][NDIM];
  hc_gcov_func(g, X, Gcov);
  hc_invert_matrix(Gcov, Gcon);
  double Ucam[NDIM], Kcon[NDIM], trial[NDIM];
  trial[0] = -1.; trial[1] = 0.; trial[2] = 0.; trial[3] = 0.;
  hc_flip_index(trial, Gcon, Ucam);
  trial[0] = 1.; trial[1] = 1.; trial[2] = 0.; trial[3] = 0.;
  hc_flip_index(trial, Gcon, Kcon);
  trial[0] = 0.; trial[1] = 0.; trial[2] = 1.; trial[3] = 0.;
  return hc_make_plasma_tetrad(Ucam, Kcon, trial, Gcov, Econ, Ecov);
}

/* src/model_tetrads.c:209-241 (old_centering) */
int hc_make_camera_tetrad_old(const ipg_grid *g, const double X[NDIM], double Econ[NDIM][NDIM],
                              double Ecov[NDIM][NDIM])
{
  double Gcov[NDIM][NDIM], Gcon[NDIM][NDIM];
  hc_gcov_func(g, X, Gcov);
  hc_invert_matrix(Gcov, Gcon);
  double Ucam[NDIM] = {1., 0., 0., 0.}, Kcon[NDIM], trial[NDIM] = {1., 1., 0., 0.};
  hc_flip_index(trial, Gcon, Kcon);
  trial[0] = 0.; trial[1] = 0.; trial[2] = 1.; trial[3] = 0.;
  return hc_make_plasma_tetrad(Ucam, Kcon, trial, Gcov, Econ, Ecov);
}

static double theta_func(const ipg_grid *g, const double X[NDIM])
{
  double r, th;
  hc_bl_coord(g, X, &r, &th);
  return th;
}

/* src/coordinates.c:394-442 */
static double root_find(const ipg_grid *g, const double X[NDIM])
{
  double th = X[2];
  double tha, thb, thc;
  double Xa[NDIM] = {0}, Xb[NDIM] = {0}, Xc[NDIM] = {0};
  Xa[1] = log(X[1]);
  Xa[3] = X[3];
  Xb[1] = Xa[1];
  Xb[3] = Xa[3];
  Xc[1] = Xa[1];
  Xc[3] = Xa[3];
  if (X[2] < M_PI / 2.) {
    Xa[2] = g->cstartx[2];
    Xb[2] = (g->cstopx[2] - g->cstartx[2]) / 2 + SMALL;
  } else {
    Xa[2] = (g->cstopx[2] - g->cstartx[2]) / 2 - SMALL;
    Xb[2] = g->cstopx[2];
  }
  double tol = 1.e-9;
  tha = theta_func(g, Xa);
  thb = theta_func(g, Xb);
  if (fabs(tha - th) < tol) return Xa[2];
  else if (fabs(thb - th) < tol) return Xb[2];
  for (int i = 0; i < 1000; i++) {
    Xc[2] = 0.5 * (Xa[2] + Xb[2]);
    thc = theta_func(g, Xc);
    if ((thc - th) * (thb - th) < 0.) Xa[2] = Xc[2];
    else Xb[2] = Xc[2];
    double err = theta_func(g, Xc) - th;
    if (fabs(err) < tol) break;
  }
  return Xc[2];
}

/* src/coordinates.c:375-387 */
void hc_native_coord(const ipg_grid *g, double r, double th_deg, double phi_deg, double X[NDIM])
{
  if (g->metric == IPG_METRIC_MINKOWSKI || g->metric == IPG_METRIC_EMINKOWSKI) {
    X[0] = 1;
    X[1] = (g->metric == IPG_METRIC_MINKOWSKI) ? r : log(r);
    X[2] = th_deg / 180 * M_PI;
    X[3] = phi_deg / 180 * M_PI;
    return;
  }
  double x[NDIM] = {0., r, th_deg / 180. * M_PI, phi_deg / 180. * M_PI};
  X[0] = 0.0;
  X[1] = log(r);
  X[2] = root_find(g, x);
  X[3] = phi_deg / 180. * M_PI;
}

/* src/grid.c:62-74 */
void hc_ijktoX(const ipg_grid *g, int i, int j, int k, double X[NDIM])
{
  X[0] = 0.;
  X[1] = g->startx[1] + (i + 0.5) * g->dx[1];
  X[2] = g->startx[2] + (j + 0.5) * g->dx[2];
  X[3] = g->startx[3] + (k + 0.5) * g->dx[3];
}

/* src/grid.c:339-379 */
double hc_gdet_zone(const ipg_grid *g, int i, int j, int k)
{
  double X[NDIM], Xzone[NDIM];
  hc_ijktoX(g, i, j, k, X);
  Xzone[0] = 0.;
  Xzone[1] = g->startx[1] + (i + 0.5) * g->dx[1];
  Xzone[2] = g->startx[2] + (j + 0.5) * g->dx[2];
  Xzone[3] = g->startx[3] + (k + 0.5) * g->dx[3];
  double gcovKS[NDIM][NDIM], gcov[NDIM][NDIM], dxdX[NDIM][NDIM];
  double r, th;
  memset(gcov, 0, sizeof(gcov));
  hc_bl_coord(g, X, &r, &th);
  hc_gcov_ks(g, r, th, gcovKS);
  hc_set_dxdX(g, Xzone, dxdX);
  for (int mu = 0; mu < NDIM; mu++)
    for (int nu = 0; nu < NDIM; nu++)
      for (int lam = 0; lam < NDIM; ++lam)
        for (int kap = 0; kap < NDIM; ++kap) gcov[mu][nu] += gcovKS[lam][kap] * dxdX[lam][mu] * dxdX[kap][nu];
  return hc_gdet_func(gcov);
}
