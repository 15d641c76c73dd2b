/*
 * CPU oracle: plain-C restatement of the reference's per-pixel ray pipeline
 * (iharm FMKS grid, thermal synchrotron, polarized transfer).  TEST
 * INFRASTRUCTURE ONLY -- see oracle.h.  Each function names the reference
 * routine it restates; operation order follows the reference so that a
 * -ffp-contract=off build matches the reference's own -ffp-contract=off build
 * bit for bit.  GSL's Bessel K_n comes from shim/gsl_shim.c.
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_sf_bessel.h"

#define NDIM 4
#define SMALL 1.e-40
#define DEL 1.e-7
#define EE (4.80320680e-10)
#define CL (2.99792458e10)
#define ME (9.1093826e-28)
#define HPL (6.6260693e-27)
#define PC (3.085678e18)
#define JY (1.e-23)
#define MUAS_PER_RAD (2.06265e11)
#define CUT_SMALL_OPTICAL_DEPTH 1e-5
#define CUT_PREVENT_NAN 1e-80

typedef struct {
  int nturns;
  double dl;
  double X[NDIM], Kcon[NDIM], Xhalf[NDIM], Kconhalf[NDIM];
} traj_t;

/* ---------------- coordinates.c ---------------- */
static void bl_coord(const orc_model *m, const double X[NDIM], double *r, double *th)
{
  *r = exp(X[1]);
  double thG = M_PI * X[2] + ((1. - m->hslope) / 2.) * sin(2. * M_PI * X[2]);
  double y = 2 * X[2] - 1.;
  double thJ = m->poly_norm * y * (1. + pow(y / m->poly_xt, m->poly_alpha) / (m->poly_alpha + 1.)) + 0.5 * M_PI;
  *th = thG + exp(m->mks_smooth * (m->startx[1] - X[1])) * (thJ - thG);
}

static void gcov_ks(const orc_model *m, double r, double th, double gcov[NDIM][NDIM])
{
  double a = m->a;
  double cth = cos(th), sth = sin(th);
  double s2 = sth * sth;
  double rho2 = r * r + a * a * cth * cth;
  memset(gcov, 0, 16 * sizeof(double));
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

static void set_dxdX(const orc_model *m, const double X[NDIM], double dxdX[NDIM][NDIM])
{
  double hslope = m->hslope, poly_xt = m->poly_xt, poly_alpha = m->poly_alpha, mks_smooth = m->mks_smooth,
         poly_norm = m->poly_norm;
  for (int mu = 0; mu < NDIM; mu++)
    for (int nu = 0; nu < NDIM; nu++) dxdX[mu][nu] = (mu == nu);
  dxdX[1][1] = exp(X[1]);
  dxdX[2][1] = -exp(mks_smooth * (m->startx[1] - X[1])) * mks_smooth *
               (M_PI / 2. - M_PI * X[2] +
                poly_norm * (2. * X[2] - 1.) * (1 + (pow((-1. + 2 * X[2]) / poly_xt, poly_alpha)) / (1 + poly_alpha)) -
                1. / 2. * (1. - hslope) * sin(2. * M_PI * X[2]));
  dxdX[2][2] = M_PI + (1. - hslope) * M_PI * cos(2. * M_PI * X[2]) +
               exp(mks_smooth * (m->startx[1] - X[1])) *
                   (-M_PI + 2. * poly_norm * (1. + pow((2. * X[2] - 1.) / poly_xt, poly_alpha) / (poly_alpha + 1.)) +
                    (2. * poly_alpha * poly_norm * (2. * X[2] - 1.) * pow((2. * X[2] - 1.) / poly_xt, poly_alpha - 1.)) /
                        ((1. + poly_alpha) * poly_xt) -
                    (1. - hslope) * M_PI * cos(2. * M_PI * X[2]));
}

static void gcov_func(const orc_model *m, const double X[NDIM], double gcov[NDIM][NDIM])
{
  double r, th;
  bl_coord(m, X, &r, &th);
  double G[NDIM][NDIM], J[NDIM][NDIM];
  gcov_ks(m, r, th, G);
  set_dxdX(m, X, J);
  for (int mu = 0; mu < NDIM; mu++)
    for (int nu = 0; nu < NDIM; nu++) {
      gcov[mu][nu] = 0;
      for (int lam = 0; lam < NDIM; ++lam)
        for (int kap = 0; kap < NDIM; ++kap) gcov[mu][nu] += G[lam][kap] * J[lam][mu] * J[kap][nu];
    }
}

/* ---------------- geometry.c ---------------- */
static int LU_decompose(double A[NDIM][NDIM], int permute[NDIM])
{
  const double absmin = 1.e-30;
  double row_norm[NDIM], absmax, maxtemp;
  int max_row = 0, n = NDIM;
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

static void LU_substitution(double A[NDIM][NDIM], double B[NDIM], int permute[NDIM])
{
  int n = NDIM;
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

static int invert_matrix(double Am[NDIM][NDIM], double Aminv[NDIM][NDIM])
{
  int permute[NDIM];
  double dxm[NDIM], Amtmp[NDIM][NDIM];
  for (int i = 0; i < NDIM; i++)
    for (int j = 0; j < NDIM; j++) Amtmp[i][j] = Am[i][j];
  if (LU_decompose(Amtmp, permute) != 0) return 1;
  for (int i = 0; i < NDIM; i++) {
    for (int j = 0; j < NDIM; j++) dxm[j] = 0.;
    dxm[i] = 1.;
    LU_substitution(Amtmp, dxm, permute);
    for (int j = 0; j < NDIM; j++) Aminv[j][i] = dxm[j];
  }
  return 0;
}

static double gdet_func(double gcov[NDIM][NDIM])
{
  int permute[NDIM];
  double t[NDIM][NDIM];
  for (int i = 0; i < NDIM; i++)
    for (int j = 0; j < NDIM; j++) t[i][j] = gcov[i][j];
  if (LU_decompose(t, permute) != 0) return -1;
  double gdet = 1.;
  for (int i = 0; i < NDIM; i++) gdet *= t[i][i];
  return sqrt(fabs(gdet));
}

static void flip_index(const double ucon[NDIM], double G[NDIM][NDIM], double ucov[NDIM])
{
  for (int m = 0; m < NDIM; m++) ucov[m] = G[m][0] * ucon[0] + G[m][1] * ucon[1] + G[m][2] * ucon[2] + G[m][3] * ucon[3];
}

static void get_connection(const orc_model *m, const double X[NDIM], double conn[NDIM][NDIM][NDIM])
{
  double tmp[NDIM][NDIM][NDIM], Xh[NDIM], Xl[NDIM], gcon[NDIM][NDIM], gcov[NDIM][NDIM], gh[NDIM][NDIM],
      gl[NDIM][NDIM];
  gcov_func(m, X, gcov);
  invert_matrix(gcov, gcon);
  for (int k = 0; k < NDIM; k++) {
    for (int l = 0; l < NDIM; l++) Xh[l] = X[l];
    for (int l = 0; l < NDIM; l++) Xl[l] = X[l];
    Xh[k] += DEL;
    Xl[k] -= DEL;
    gcov_func(m, Xh, gh);
    gcov_func(m, Xl, gl);
    for (int i = 0; i < NDIM; i++)
      for (int j = 0; j < NDIM; j++) conn[i][j][k] = (gh[i][j] - gl[i][j]) / (Xh[k] - Xl[k]);
  }
  for (int i = 0; i < NDIM; i++)
    for (int j = 0; j < NDIM; j++)
      for (int k = 0; k < NDIM; k++) tmp[i][j][k] = 0.5 * (conn[j][i][k] + conn[k][i][j] - conn[k][j][i]);
  for (int i = 0; i < NDIM; i++)
    for (int j = 0; j < NDIM; j++)
      for (int k = 0; k < NDIM; k++) {
        conn[i][j][k] = 0.;
        for (int l = 0; l < NDIM; l++) conn[i][j][k] += gcon[i][l] * tmp[l][j][k];
      }
}

static void normalize(double v[NDIM], double G[NDIM][NDIM])
{
  double norm = 0.;
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++) norm += v[k] * v[l] * G[k][l];
  norm = sqrt(fabs(norm));
  for (int k = 0; k < 4; k++) v[k] /= norm;
}

static void null_normalize(double K[NDIM], double fnorm)
{
  double inorm = sqrt(K[1] * K[1] + K[2] * K[2] + K[3] * K[3]);
  K[0] = fnorm;
  K[1] *= fnorm / inorm;
  K[2] *= fnorm / inorm;
  K[3] *= fnorm / inorm;
}

static int levi_civita(int i, int j, int k, int l)
{
  if (i == j || i == k || i == l || j == k || j == l || k == l) return 0;
  int idx[4] = {i, j, k, l}, n_perm = 0, do_sort = 1;
  while (do_sort) {
    int n_swap = 0;
    for (int n = 0; n < 3; n++)
      if (idx[n] > idx[n + 1]) {
        n_perm++;
        n_swap++;
        int v = idx[n];
        idx[n] = idx[n + 1];
        idx[n + 1] = v;
      }
    do_sort = n_swap;
  }
  return (n_perm % 2) ? -1 : 1;
}

/* ---------------- tetrads.c, model_tetrads.c ---------------- */
static void set_Econ_from_trial(double E[4], int defdir, const double trial[4])
{
  double norm = 0.;
  for (int k = 1; k < 4; k++) norm += fabs(trial[k]);
  for (int k = 0; k < 4; k++)
    if (norm <= SMALL) E[k] = (k == defdir);
    else E[k] = trial[k];
}

static void project_out(double a[NDIM], const double b[NDIM], double G[4][4])
{
  double bsq = 0., adb = 0.;
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++) bsq += b[k] * b[l] * G[k][l];
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++) adb += a[k] * b[l] * G[k][l];
  for (int k = 0; k < 4; k++) a[k] -= b[k] * adb / bsq;
}

static int check_handedness(double E[NDIM][NDIM], double G[NDIM][NDIM], double *dot)
{
  double g = gdet_func(G);
  if (g < 0.) return 1;
  *dot = 0.;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int l = 0; l < 4; l++)
        for (int k = 0; k < 4; k++) *dot += g * levi_civita(i, j, k, l) * E[0][i] * E[1][j] * E[2][k] * E[3][l];
  return 0;
}

static int make_plasma_tetrad(const double Ucon[NDIM], const double Kcon[NDIM], const double Bcon[NDIM],
                              double G[NDIM][NDIM], double Econ[NDIM][NDIM], double Ecov[NDIM][NDIM])
{
  double ones[NDIM] = {1., 1., 1., 1.};
  set_Econ_from_trial(Econ[0], 0, Ucon);
  set_Econ_from_trial(Econ[1], 3, ones);
  set_Econ_from_trial(Econ[2], 2, Bcon);
  set_Econ_from_trial(Econ[3], 3, Kcon);
  normalize(Econ[0], G);
  project_out(Econ[3], Econ[0], G);
  project_out(Econ[3], Econ[0], G);
  normalize(Econ[3], G);
  project_out(Econ[2], Econ[0], G);
  project_out(Econ[2], Econ[3], G);
  project_out(Econ[2], Econ[0], G);
  project_out(Econ[2], Econ[3], G);
  normalize(Econ[2], G);
  project_out(Econ[1], Econ[0], G);
  project_out(Econ[1], Econ[2], G);
  project_out(Econ[1], Econ[3], G);
  project_out(Econ[1], Econ[0], G);
  project_out(Econ[1], Econ[2], G);
  project_out(Econ[1], Econ[3], G);
  normalize(Econ[1], G);
  int oddflag = 0;
  double dot;
  if (check_handedness(Econ, G, &dot)) oddflag |= 16;
  if (fabs(fabs(dot) - 1.) > 1.e-10) oddflag |= 1;
  if (dot < 0.)
    for (int k = 0; k < 4; k++) Econ[1][k] *= -1.;
  for (int k = 0; k < 4; k++) flip_index(Econ[k], G, Ecov[k]);
  for (int l = 0; l < 4; l++) Ecov[0][l] *= -1.;
  return oddflag;
}

static void make_camera_tetrad(const orc_model *m, const double X[NDIM], double Econ[NDIM][NDIM],
                               double Ecov[NDIM][NDIM])
{
  double Gcov[NDIM][NDIM], Gcon[NDIM][NDIM], Ucam[NDIM], Kcon[NDIM], trial[NDIM];
  gcov_func(m, X, Gcov);
  invert_matrix(Gcov, Gcon);
  trial[0] = -1.; trial[1] = 0.; trial[2] = 0.; trial[3] = 0.;
  flip_index(trial, Gcon, Ucam);
  trial[0] = 1.; trial[1] = 1.; trial[2] = 0.; trial[3] = 0.;
  flip_index(trial, Gcon, Kcon);
  trial[0] = 0.; trial[1] = 0.; trial[2] = 1.; trial[3] = 0.;
  make_plasma_tetrad(Ucam, Kcon, trial, Gcov, Econ, Ecov);
}

/* ---------------- geodesics ---------------- */
static void push_photon(const orc_model *m, double X[NDIM], double Kcon[NDIM], double dl, double Xhalf[NDIM],
                        double Kconhalf[NDIM])
{
  double lconn[NDIM][NDIM][NDIM], dKcon[NDIM], Xh[NDIM], Kconh[NDIM];
  get_connection(m, X, lconn);
  for (int k = 0; k < 4; k++) dKcon[k] = 0.;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) dKcon[k] -= 0.5 * dl * lconn[k][i][j] * Kcon[i] * Kcon[j];
  for (int k = 0; k < 4; k++) Kconh[k] = Kcon[k] + dKcon[k];
  for (int i = 0; i < 4; i++) Xh[i] = X[i] + 0.5 * dl * Kcon[i];
  for (int i = 0; i < 4; i++) Xhalf[i] = Xh[i];
  for (int i = 0; i < 4; i++) Kconhalf[i] = Kconh[i];
  get_connection(m, Xh, lconn);
  for (int k = 0; k < 4; k++) dKcon[k] = 0.;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) dKcon[k] -= dl * lconn[k][i][j] * Kconh[i] * Kconh[j];
  for (int k = 0; k < 4; k++) Kcon[k] += dKcon[k];
  for (int k = 0; k < 4; k++) X[k] += dl * Kconh[k];
}

static double stepsize(const orc_model *m, const double X[NDIM], const double Kcon[NDIM], double eps)
{
  double deh = fmin(fabs(X[1] - m->cstartx[1]), 0.1);
  double dlx1 = eps * (10 * deh) / (fabs(Kcon[1]) + SMALL * SMALL);
  double cut = 0.02;
  double lx2 = m->cstopx[2] - m->cstartx[2];
  double dpole = fmin(fabs(X[2] / lx2), fabs((m->cstopx[2] - X[2]) / lx2));
  double d2fac = (dpole < cut) ? dpole / 3 : fmin(cut / 3 + (dpole - cut) * 10., 1);
  double dlx2 = eps * d2fac / (fabs(Kcon[2]) + SMALL * SMALL);
  double dlx3 = eps / (fabs(Kcon[3]) + SMALL * SMALL);
  double idlx1 = 1. / (fabs(dlx1) + SMALL * SMALL);
  double idlx2 = 1. / (fabs(dlx2) + SMALL * SMALL);
  double idlx3 = 1. / (fabs(dlx3) + SMALL * SMALL);
  return 1. / (idlx1 + idlx2 + idlx3);
}

static int stop_backward_integration(const orc_model *m, const double X[NDIM], const double Kcon[NDIM])
{
  double r, th;
  bl_coord(m, X, &r, &th);
  return (r > m->rmax_geo && Kcon[1] < 0.) || r < (m->Rh + 0.0001);
}

static int trace_geodesic(const orc_model *m, const orc_camera *c, const double Xi[NDIM], const double Kconi[NDIM],
                          traj_t *traj, int step_max)
{
  double X[NDIM], Kcon[NDIM], Xhalf[NDIM], Kconhalf[NDIM];
  for (int mu = 0; mu < NDIM; mu++) {
    X[mu] = Xi[mu];
    Xhalf[mu] = Xi[mu];
    Kcon[mu] = Kconi[mu];
    Kconhalf[mu] = Kconi[mu];
    traj[0].X[mu] = Xi[mu];
    traj[0].Kcon[mu] = Kconi[mu];
  }
  int nstep = 0, nturns = 0;
  int passed = (c->Xcam[2] < 0.5) ? 1 : ((c->Xcam[2] > 0.5) ? -1 : 0);
  while (!stop_backward_integration(m, X, Kcon) && (nstep < step_max - 1)) {
    nstep++;
    double dl = stepsize(m, X, Kcon, c->eps);
    traj[nstep].dl = dl * m->L_unit * HPL / (ME * CL * CL);
    push_photon(m, X, Kcon, -dl, Xhalf, Kconhalf);
    for (int mu = 0; mu < NDIM; mu++) {
      traj[nstep].X[mu] = X[mu];
      traj[nstep].Kcon[mu] = Kcon[mu];
      traj[nstep].Xhalf[mu] = Xhalf[mu];
      traj[nstep].Kconhalf[mu] = Kconhalf[mu];
    }
    if (passed != 0) {
      if (passed > 0) {
        if (traj[nstep].X[2] > 0.5) passed = 0;
      } else {
        if (traj[nstep].X[2] < 0.5) passed = 0;
      }
    } else if (nstep > 3) {
      if (c->subring_dtheta == 1) {
        double a_ = traj[nstep - 1].X[2] - traj[nstep - 2].X[2];
        double b_ = traj[nstep].X[2] - traj[nstep - 1].X[2];
        if (a_ * b_ < 0) nturns++;
      } else {
        double ra, rb, rc, ha, hb, hc;
        bl_coord(m, traj[nstep - 2].X, &ra, &ha);
        bl_coord(m, traj[nstep - 1].X, &rb, &hb);
        bl_coord(m, traj[nstep - 0].X, &rc, &hc);
        double dz_1 = rb * cos(hb) - ra * cos(ha);
        double dz_2 = rc * cos(hc) - rb * cos(hb);
        if (dz_1 * dz_2 < 0) nturns++;
      }
    }
    traj[nstep].nturns = nturns;
  }
  return nstep;
}

/* ---------------- grid.c and the iharm model ---------------- */
static size_t cidx(const orc_model *m, int i, int j, int k)
{
  return ((size_t)i * (m->n2 + 2) + j) * (m->n3 + 2) + k;
}

static void Xtoijk_ghost(const orc_model *m, const double X[NDIM], int *i, int *j, int *k, double del[NDIM])
{
  double phi = fmod(X[3], m->cstopx[3]);
  if (phi < 0.0) phi = m->cstopx[3] + phi;
  *i = (int)((X[1] - m->startx[1]) / m->dx[1] - 0.5 + 1000) - 1000;
  *j = (int)((X[2] - m->startx[2]) / m->dx[2] - 0.5 + 1000) - 1000;
  *k = (int)((phi - m->startx[3]) / m->dx[3] - 0.5 + 1000) - 1000;
  if (*i < -1) *i = -1;
  if (*j < -1) *j = -1;
  if (*k < -1) *k = -1;
  if (*i >= m->n1) *i = m->n1 - 1;
  if (*j >= m->n2) *j = m->n2 - 1;
  if (*k >= m->n3) *k = m->n3 - 1;
  del[1] = (X[1] - ((*i + 0.5) * m->dx[1] + m->startx[1])) / m->dx[1];
  del[2] = (X[2] - ((*j + 0.5) * m->dx[2] + m->startx[2])) / m->dx[2];
  del[3] = (phi - ((*k + 0.5) * m->dx[3] + m->startx[3])) / m->dx[3];
  for (int q = 0; q < 4; ++q) {
    if (del[q] < 0.) del[q] = 0.;
    if (del[q] >= 1.) del[q] = 1.;
  }
  *i += 1;
  *j += 1;
  *k += 1;
}

static double interp_scalar(const orc_model *m, const double X[NDIM], const double *var)
{
  double del[NDIM] = {0};
  int i, j, k;
  Xtoijk_ghost(m, X, &i, &j, &k, del);
  int ip1 = i + 1, jp1 = j + 1, kp1 = k + 1;
  double b1 = 1. - del[1], b2 = 1. - del[2];
  double interp = var[cidx(m, i, j, k)] * b1 * b2 + var[cidx(m, i, jp1, k)] * b1 * del[2] +
                  var[cidx(m, ip1, j, k)] * del[1] * b2 + var[cidx(m, ip1, jp1, k)] * del[1] * del[2];
  interp = (1. - del[3]) * interp +
           del[3] * (var[cidx(m, i, j, kp1)] * b1 * b2 + var[cidx(m, i, jp1, kp1)] * del[2] * b1 +
                     var[cidx(m, ip1, j, kp1)] * del[1] * b2 + var[cidx(m, ip1, jp1, kp1)] * del[1] * del[2]);
  return interp;
}

static int X_in_domain(const orc_model *m, const double X[NDIM])
{
  return !(X[1] < m->startx[1] || X[1] >= m->stopx[1] || X[2] < m->startx[2] || X[2] >= m->stopx[2]);
}

static void get_model_fourv(const orc_model *m, const double X[NDIM], double Ucon[NDIM], double Ucov[NDIM],
                            double Bcon[NDIM], double Bcov[NDIM])
{
  double gcov[NDIM][NDIM], gcon[NDIM][NDIM];
  gcov_func(m, X, gcov);
  invert_matrix(gcov, gcon);
  if (X_in_domain(m, X) == 0) {
    Ucov[0] = -1. / sqrt(-gcon[0][0]);
    Ucov[1] = 0.; Ucov[2] = 0.; Ucov[3] = 0.;
    Ucon[0] = 0.; Ucon[1] = 0.; Ucon[2] = 0.; Ucon[3] = 0.;
    for (int mu = 0; mu < NDIM; ++mu) {
      Ucon[0] += Ucov[mu] * gcon[0][mu];
      Ucon[1] += Ucov[mu] * gcon[1][mu];
      Ucon[2] += Ucov[mu] * gcon[2][mu];
      Ucon[3] += Ucov[mu] * gcon[3][mu];
      Bcon[mu] = 0.;
      Bcov[mu] = 0.;
    }
    return;
  }
  double Vcon[NDIM];
  Vcon[1] = interp_scalar(m, X, m->f[0]);
  Vcon[2] = interp_scalar(m, X, m->f[1]);
  Vcon[3] = interp_scalar(m, X, m->f[2]);
  double VdotV = 0.;
  for (int i = 1; i < NDIM; i++)
    for (int j = 1; j < NDIM; j++) VdotV += gcov[i][j] * Vcon[i] * Vcon[j];
  double Vfac = sqrt(-1. / gcon[0][0] * (1. + fabs(VdotV)));
  Ucon[0] = -Vfac * gcon[0][0];
  for (int i = 1; i < NDIM; i++) Ucon[i] = Vcon[i] - Vfac * gcon[0][i];
  flip_index(Ucon, gcov, Ucov);
  double Bcon1 = interp_scalar(m, X, m->f[3]);
  double Bcon2 = interp_scalar(m, X, m->f[4]);
  double Bcon3 = interp_scalar(m, X, m->f[5]);
  Bcon[0] = Bcon1 * Ucov[1] + Bcon2 * Ucov[2] + Bcon3 * Ucov[3];
  Bcon[1] = (Bcon1 + Ucon[1] * Bcon[0]) / Ucon[0];
  Bcon[2] = (Bcon2 + Ucon[2] * Bcon[0]) / Ucon[0];
  Bcon[3] = (Bcon3 + Ucon[3] * Bcon[0]) / Ucon[0];
  flip_index(Bcon, gcov, Bcov);
}

static double get_model_ne(const orc_model *m, const double X[NDIM])
{
  if (X_in_domain(m, X) == 0) return 0.;
  double sigma = interp_scalar(m, X, m->f[9]);
  if (sigma > m->sigma_cut) return 0.;
  double sigma_above = m->sigma_cut;
  if (m->sigma_cut_high > 0) sigma_above = m->sigma_cut_high;
  double fac;
  if (sigma < m->sigma_cut) fac = 1;
  else if (sigma >= sigma_above) fac = 0;
  else fac = cos(M_PI / 2. / (sigma_above - m->sigma_cut) * (sigma - m->sigma_cut));
  return interp_scalar(m, X, m->f[6]) * fac;
}

static double get_model_thetae(const orc_model *m, const double X[NDIM])
{
  if (X_in_domain(m, X) == 0) return 0.;
  return interp_scalar(m, X, m->f[7]);
}

static double get_model_b(const orc_model *m, const double X[NDIM])
{
  if (X_in_domain(m, X) == 0) return 0.;
  return interp_scalar(m, X, m->f[8]);
}

static int radiating_region(const orc_model *m, const double X[NDIM])
{
  double r, th;
  bl_coord(m, X, &r, &th);
  return (r > m->rmin_geo && r < m->rmax_geo && th > m->th_beg && th < (M_PI - m->th_beg));
}

/* ---------------- radiation.c, symphony thermal fits ---------------- */
static double Bnu_inv(double nu, double Thetae)
{
  double x = HPL * nu / (ME * CL * CL * Thetae);
  if (x < 2.e-3) return ((2. * HPL / (CL * CL)) / (x / 24. * (24. + x * (12. + x * (4. + x)))));
  return ((2. * HPL / (CL * CL)) / (exp(x) - 1.));
}

static double get_fluid_nu(const double Kcon[NDIM], const double Ucov[NDIM])
{
  return -(Kcon[0] * Ucov[0] + Kcon[1] * Ucov[1] + Kcon[2] * Ucov[2] + Kcon[3] * Ucov[3]) * ME * CL * CL / HPL;
}

static double get_bk_angle(const double Kcon[NDIM], const double Ucov[NDIM], const double Bcon[NDIM],
                           const double Bcov[NDIM])
{
  double B = sqrt(fabs(Bcon[0] * Bcov[0] + Bcon[1] * Bcov[1] + Bcon[2] * Bcov[2] + Bcon[3] * Bcov[3]));
  if (B == 0.) return (M_PI / 2.);
  double k = fabs(Kcon[0] * Ucov[0] + Kcon[1] * Ucov[1] + Kcon[2] * Ucov[2] + Kcon[3] * Ucov[3]);
  double mu = (Kcon[0] * Bcov[0] + Kcon[1] * Bcov[1] + Kcon[2] * Bcov[2] + Kcon[3] * Bcov[3]) / (k * B);
  if (fabs(mu) > 1.) mu /= fabs(mu);
  return (acos(mu));
}

/* symphony constants (src/symphony/params.c:15-19) */
#define S_PI 3.1415926535897932384
#define S_ME 9.1093826e-28
#define S_CL 2.99792458e10
#define S_EE 4.80320680e-10

typedef struct {
  double nu, B, Ne, theta, Thetae;
} fitp;

static double get_nu_c(const fitp *p) { return (S_EE * p->B) / (2. * S_PI * S_ME * S_CL); }

static double I_I(double x)
{
  return 2.5651 * (1 + 1.92 * pow(x, -1. / 3.) + 0.9977 * pow(x, -2. / 3.)) * exp(-1.8899 * pow(x, 1. / 3.));
}
static double I_Q(double x)
{
  return 2.5651 * (1 + 0.93193 * pow(x, -1. / 3.) + 0.499873 * pow(x, -2. / 3.)) * exp(-1.8899 * pow(x, 1. / 3.));
}
static double I_V(double x)
{
  return (1.81384 / x + 3.42319 * pow(x, -2. / 3.) + 0.0292545 * pow(x, -0.5) + 2.03773 * pow(x, -1. / 3.)) *
         exp(-1.8899 * pow(x, 1. / 3.));
}

static double dexter_I(const fitp *p)
{
  double nus = 3.0 * EE * p->B * sin(p->theta) / 4.0 / M_PI / ME / CL * p->Thetae * p->Thetae + 1.0;
  double x = p->nu / nus;
  return p->Ne * EE * EE * p->nu / 2. / sqrt(3) / CL / p->Thetae / p->Thetae * I_I(x);
}
static double dexter_Q(const fitp *p)
{
  double nus = 3.0 * EE * p->B * sin(p->theta) / 4.0 / M_PI / ME / CL * p->Thetae * p->Thetae + 1.0;
  double x = p->nu / nus;
  return -p->Ne * EE * EE * p->nu / 2. / sqrt(3) / CL / p->Thetae / p->Thetae * I_Q(x);
}
static double dexter_V(const fitp *p)
{
  double nus = 3.0 * EE * p->B * sin(p->theta) / 4.0 / M_PI / ME / CL * p->Thetae * p->Thetae + 1.0;
  double x = p->nu / nus;
  return 2. * p->Ne * EE * EE * p->nu / tan(p->theta) / 3. / sqrt(3) / CL / p->Thetae / p->Thetae / p->Thetae * I_V(x);
}

static double leung_I(const fitp *p)
{
  double K2 = fmax(gsl_sf_bessel_Kn(2, 1. / p->Thetae), SMALL);
  double nuc = EE * p->B / (2. * M_PI * ME * CL);
  double nus = (2. / 9.) * nuc * p->Thetae * p->Thetae * sin(p->theta);
  if (p->nu > 1.e12 * nus) return 0.;
  double x = p->nu / nus;
  double f = pow(pow(x, 1. / 2.) + pow(2., 11. / 12.) * pow(x, 1. / 6.), 2);
  return (sqrt(2.) * M_PI * EE * EE * p->Ne * nus / (3. * CL * K2)) * f * exp(-pow(x, 1. / 3.));
}

static double pandya_I(const fitp *p)
{
  double nu_c = get_nu_c(p);
  double nu_s = (2. / 9.) * nu_c * sin(p->theta) * p->Thetae * p->Thetae;
  double X = p->nu / nu_s;
  double prefactor = (p->Ne * pow(S_EE, 2.) * nu_c) / S_CL;
  double term1 = sqrt(2.) * S_PI / 27. * sin(p->theta);
  double term2 = pow(pow(X, 0.5) + pow(2., 11. / 12.) * pow(X, 1. / 6.), 2.);
  double term3 = exp(-pow(X, 1. / 3.));
  return prefactor * term1 * term2 * term3;
}
static double pandya_Q(const fitp *p)
{
  double nu_c = get_nu_c(p);
  double nu_s = (2. / 9.) * nu_c * sin(p->theta) * p->Thetae * p->Thetae;
  double X = p->nu / nu_s;
  double prefactor = (p->Ne * pow(S_EE, 2.) * nu_c) / S_CL;
  double term1 = sqrt(2.) * S_PI / 27. * sin(p->theta);
  double term2 = (7. * pow(p->Thetae, 24. / 25.) + 35.) / (10. * pow(p->Thetae, 24. / 25.) + 75.);
  double term3 = pow(pow(X, 0.5) + term2 * pow(2., 11. / 12.) * pow(X, 1. / 6.), 2.);
  double ans = prefactor * term1 * term3 * exp(-pow(X, 1. / 3.));
  return -ans;
}
static double pandya_V(const fitp *p)
{
  double nu_c = get_nu_c(p);
  double nu_s = (2. / 9.) * nu_c * sin(p->theta) * p->Thetae * p->Thetae;
  double X = p->nu / nu_s;
  double prefactor = (p->Ne * pow(S_EE, 2.) * nu_c) / S_CL;
  double term1 = (37. - 87. * sin(p->theta - 28. / 25.)) / (100. * (p->Thetae + 1.));
  double term2 = pow(1. + (pow(p->Thetae, 3. / 5.) / 25. + 7. / 10.) * pow(X, 9. / 25.), 5. / 3.);
  return prefactor * term1 * term2 * exp(-pow(X, 1. / 3.));
}

static double rho_Q(const fitp *p)
{
  double omega0 = S_EE * p->B / (S_ME * S_CL);
  double wp2 = 4. * S_PI * p->Ne * pow(S_EE, 2.) / S_ME;
  double x = p->Thetae * sqrt(sqrt(2.) * sin(p->theta) * (1.e3 * omega0 / (2. * S_PI * p->nu)));
  double extraterm = (.011 * exp(-x / 47.2) - pow(2., (-1. / 3.)) / pow(3., (23. / 6.)) * S_PI * 1.e4 *
                                                 pow((x + 1.e-16), (-8. / 3.))) *
                     (0.5 + 0.5 * tanh((log(x) - log(120.)) / 0.1));
  double jffunc = 2.011 * exp(-pow(x, 1.035) / 4.7) - cos(x / 2.) * exp(-pow(x, 1.2) / 2.73) - .011 * exp(-x / 47.2) +
                  extraterm;
  double k1 = gsl_sf_bessel_Kn(1, 1. / p->Thetae);
  double k2 = gsl_sf_bessel_Kn(2, 1. / p->Thetae);
  double k_ratio = (k2 > 0) ? k1 / k2 : 1;
  double eps11m22 = jffunc * wp2 * pow(omega0, 2.) / pow(2. * S_PI * p->nu, 4.) * (k_ratio + 6. * p->Thetae) *
                    pow(sin(p->theta), 2.);
  return 2. * S_PI * p->nu / (2. * S_CL) * eps11m22;
}

static double rho_V(const fitp *p, int dexter)
{
  double omega0 = S_EE * p->B / (S_ME * S_CL);
  double wp2 = 4. * S_PI * p->Ne * pow(S_EE, 2.) / S_ME;
  double x = p->Thetae * sqrt(sqrt(2.) * sin(p->theta) * (1.e3 * omega0 / (2. * S_PI * p->nu)));
  double k0 = gsl_sf_bessel_Kn(0, 1. / p->Thetae);
  double k2 = gsl_sf_bessel_Kn(2, 1. / p->Thetae);
  double fit_factor;
  if (dexter && k2 > 0) {
    /* Dexter (2016) g(X), src/symphony/maxwell_juettner_fits.c:269-272 */
    double shgmfunc = 0.43793091 * log(1. + 0.00185777 * pow(x, 1.50316886));
    fit_factor = (k0 - shgmfunc) / k2;
  } else {
    double shgmfunc = 1 - 0.11 * log(1 + 0.035 * x);
    double k_ratio = (k2 > 0) ? k0 / k2 : 1;
    fit_factor = k_ratio * shgmfunc;
  }
  double eps12 = wp2 * omega0 / pow((2. * S_PI * p->nu), 3.) * fit_factor * cos(p->theta);
  return 2. * S_PI * p->nu / S_CL * eps12;
}

static void jar_fits_at(const fitp *pp, int dist, int pol, double *jI, double *jQ, double *jU, double *jV,
                        double *aI, double *aQ, double *aU, double *aV, double *rQ, double *rU, double *rV);

/* jar_calc_dist, src/model_radiation.c:145-332 (thermal types 1, 4) */
static void jar_calc_dist(const orc_model *m, int dist, int pol, const double X[NDIM], const double Kcon[NDIM],
                          double *jI, double *jQ, double *jU, double *jV, double *aI, double *aQ, double *aU,
                          double *aV, double *rQ, double *rU, double *rV)
{
  double Ne = get_model_ne(m, X);
  if (Ne <= 0.) {
    *jI = 0.0; *jQ = 0.0; *jU = 0.0; *jV = 0.0;
    *aI = 0.0; *aQ = 0.0; *aU = 0.0; *aV = 0.0;
    *rQ = 0; *rU = 0; *rV = 0;
    return;
  }
  double Ucon[NDIM], Ucov[NDIM], Bcon[NDIM], Bcov[NDIM];
  get_model_fourv(m, X, Ucon, Ucov, Bcon, Bcov);
  double nu = get_fluid_nu(Kcon, Ucov);
  double theta = get_bk_angle(Kcon, Ucov, Bcon, Bcov);
  fitp p = {nu, get_model_b(m, X), Ne, theta, get_model_thetae(m, X)};
  jar_fits_at(&p, dist, pol, jI, jQ, jU, jV, aI, aQ, aU, aV, rQ, rU, rV);
}

/* the thermal fits of jar_calc_dist at given (nu, B, Ne, theta, Thetae),
 * Ne > 0: src/model_radiation.c:182-332 after the model lookup */
static void jar_fits_at(const fitp *pp, int dist, int pol, double *jI, double *jQ, double *jU, double *jV,
                        double *aI, double *aQ, double *aU, double *aV, double *rQ, double *rU, double *rV)
{
  fitp p = *pp;
  double nu = p.nu, theta = p.theta;
  double nusq = nu * nu;
  if (theta <= 0.0 || theta >= M_PI) {
    *jI = 0.0; *jQ = 0.0; *jU = 0.0; *jV = 0.0;
    *aI = 0.0; *aQ = 0.0; *aU = 0.0; *aV = 0.0;
    *rQ = 0.0; *rU = 0.0;
    /* the reference leaves paramsM.dexter_fit = 1 on this early return for
     * the Dexter emission type (src/model_radiation.c:202-207, 212-221), so
     * its rho_V takes Dexter's g(X) here, Shcherbakov's elsewhere */
    *rV = pol ? rho_V(&p, dist == 4) * nu : 0.0;
    return;
  }
  if (!pol) {
    *jI = leung_I(&p);
    *jI /= nusq;
    double Bnuinv = Bnu_inv(nu, p.Thetae);
    *aI = (Bnuinv > 0) ? *jI / Bnuinv : 0;
    return;
  }
  if (dist == 1) {
    *jI = pandya_I(&p);
    *jI /= nusq;
    *jQ = -pandya_Q(&p) / nusq;
    *jU = -0. / nusq;
    *jV = pandya_V(&p) / nusq;
  } else {
    *jI = dexter_I(&p);
    *jI /= nusq;
    *jQ = -dexter_Q(&p) / nusq;
    *jU = -0. / nusq;
    *jV = dexter_V(&p) / nusq;
  }
  double jP = sqrt(*jQ * *jQ + *jU * *jU + *jV * *jV);
  if (*jI < jP / 0.99) {
    double pol_frac_e = *jI / jP * 0.99;
    *jQ *= pol_frac_e;
    *jU *= pol_frac_e;
    *jV *= pol_frac_e;
  }
  double Bnuinv = Bnu_inv(nu, p.Thetae);
  if (Bnuinv > 0) {
    *aI = *jI / Bnuinv;
    *aQ = *jQ / Bnuinv;
    *aU = *jU / Bnuinv;
    *aV = *jV / Bnuinv;
  } else {
    *aI = 0.; *aQ = 0.; *aU = 0.; *aV = 0.;
  }
  *rQ = rho_Q(&p) * nu;
  *rU = 0. * nu;
  *rV = rho_V(&p, 0) * nu;
}

static void get_jkinv(const orc_model *m, const orc_camera *c, const double X[NDIM], const double K[NDIM], double *j,
                      double *k)
{
  double a, b, d, e, f, g, h, q, r;
  jar_calc_dist(m, c->emission_type, 0, X, K, j, &a, &b, &d, k, &e, &f, &g, &h, &q, &r);
}

/* Both calls of jar_calc_dist at given plasma parameters: in = (nu, Ne,
 * Thetae, B, theta) per point, out = (jI/nu^2 and aI of pol = 0, then jI jQ
 * jU jV aI aQ aU aV rQ rV of pol = 1) per point; zeros where Ne <= 0. */
void orc_thermal_coefficients(const double *in, int n, int dist, double *out)
{
  for (int i = 0; i < n; i++) {
    const double *q = in + 5 * (size_t)i;
    double *o = out + 12 * (size_t)i;
    for (int k = 0; k < 12; k++) o[k] = 0.;
    if (q[1] <= 0.) continue;
    fitp p = {q[0], q[3], q[1], q[4], q[2]};
    double a, b, d, e, f, g, h, r, t;
    jar_fits_at(&p, dist, 0, &o[0], &a, &b, &d, &o[1], &e, &f, &g, &h, &r, &t);
    double rU;
    jar_fits_at(&p, dist, 1, &o[2], &o[3], &o[4], &o[5], &o[6], &o[7], &o[8], &o[9], &o[10], &rU, &o[11]);
  }
}

/* ---------------- ipolarray.c ---------------- */
static void push_polar(const orc_model *m, const double Xm[NDIM], const double Km[NDIM], double complex Ni[NDIM][NDIM],
                       double complex Nm[NDIM][NDIM], double complex Nf[NDIM][NDIM], double dlam)
{
  double dl = dlam / (m->L_unit * HPL / (ME * CL * CL));
  double lconn[NDIM][NDIM][NDIM];
  get_connection(m, Xm, lconn);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) Nf[i][j] = Ni[i][j];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++)
        for (int l = 0; l < 4; l++)
          Nf[i][j] += -(lconn[i][k][l] * Nm[k][j] * Km[l] + lconn[j][k][l] * Nm[i][k] * Km[l]) * dl;
}

static double approximate_solve(double Ii, double ji, double ki, double jf, double kf, double dl, double *tau)
{
  double javg = (ji + jf) / 2., kavg = (ki + kf) / 2.;
  double dtau = dl * kavg;
  *tau += dtau;
  if (dtau < 1.e-3) return Ii + (javg - Ii * kavg) * dl * (1. - (dtau / 2.) * (1. - dtau / 3.));
  double efac = exp(-dtau);
  return Ii * efac + (javg / kavg) * (1. - efac);
}

static void coord_to_tetrad2(double complex T[NDIM][NDIM], double E[NDIM][NDIM], double complex Tt[NDIM][NDIM])
{
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) Tt[i][j] = 0. + I * 0.;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++)
        for (int l = 0; l < 4; l++) Tt[i][j] += T[k][l] * E[i][k] * E[j][l];
}

static void tetrad_to_coord2(double complex Tt[NDIM][NDIM], double E[NDIM][NDIM], double complex T[NDIM][NDIM])
{
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) T[i][j] = 0. + I * 0.;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++)
        for (int l = 0; l < 4; l++) T[i][j] += Tt[k][l] * E[k][i] * E[l][j];
}

static void tensor_to_stokes(double complex f[NDIM][NDIM], double *fI, double *fQ, double *fU, double *fV)
{
  *fI = creal(f[1][1] + f[2][2]) / 2;
  *fQ = creal(f[1][1] - f[2][2]) / 2;
  *fU = creal(f[1][2] + f[2][1]) / 2;
  *fV = cimag(f[2][1] - f[1][2]) / 2;
}

static void stokes_to_tensor(double fI, double fQ, double fU, double fV, double complex f[NDIM][NDIM])
{
  f[1][1] = (fI + fQ + 0. * I);
  f[1][2] = (fU - I * fV);
  f[2][1] = (fU + I * fV);
  f[2][2] = (fI - fQ + 0. * I);
}

static int evolve_N(const orc_model *m, const orc_camera *c, const double Xf[NDIM], const double Kconf[NDIM],
                    double dlam, double complex N_coord[NDIM][NDIM], double *tauF, int zero_emission)
{
  double gcov[NDIM][NDIM], Ucon[NDIM], Bcon[NDIM], Ucov[NDIM], Bcov[NDIM], Ecov[NDIM][NDIM], Econ[NDIM][NDIM];
  double complex N_tetrad[NDIM][NDIM];
  double jI, jQ, jU, jV, aI, aQ, aU, aV, rV, rU, rQ;
  double SI0, SQ0, SU0, SV0, SI1, SQ1, SU1, SV1, SI2, SQ2, SU2, SV2, SI, SQ, SU, SV;
  int oddflag = 0;
  jar_calc_dist(m, c->emission_type, 1, Xf, Kconf, &jI, &jQ, &jU, &jV, &aI, &aQ, &aU, &aV, &rQ, &rU, &rV);
  if (zero_emission) {
    jI = 0.; jQ = 0.; jU = 0.; jV = 0.;
  }
  get_model_fourv(m, Xf, Ucon, Ucov, Bcon, Bcov);
  double bsq = 0.;
  for (int mu = 0; mu < NDIM; mu++) bsq += Bcon[mu] * Bcov[mu];
  if (bsq <= 0.) {
    Bcon[0] = 0.; Bcon[1] = 1.; Bcon[2] = 1.; Bcon[3] = 1.;
  }
  gcov_func(m, Xf, gcov);
  oddflag |= make_plasma_tetrad(Ucon, Kconf, Bcon, gcov, Econ, Ecov);
  coord_to_tetrad2(N_coord, Ecov, N_tetrad);
  tensor_to_stokes(N_tetrad, &SI0, &SQ0, &SU0, &SV0);
  double x = dlam * 0.5;
  double rho2 = rQ * rQ + rU * rU + rV * rV;
  if (rho2 > CUT_PREVENT_NAN) {
    double rho = sqrt(rho2);
    double rdS = rQ * SQ0 + rU * SU0 + rV * SV0;
    double cc = cos(rho * x), s = sin(rho * x), sh = sin(0.5 * rho * x);
    SI1 = SI0;
    SQ1 = SQ0 * cc + 2 * rQ * rdS / rho2 * sh * sh + (rU * SV0 - rV * SU0) / rho * s;
    SU1 = SU0 * cc + 2 * rU * rdS / rho2 * sh * sh + (rV * SQ0 - rQ * SV0) / rho * s;
    SV1 = SV0 * cc + 2 * rV * rdS / rho2 * sh * sh + (rQ * SU0 - rU * SQ0) / rho * s;
  } else {
    SI1 = SI0;
    SQ1 = SQ0 + (-rV * SU0 + rU * SV0) * x;
    SU1 = SU0 + (rV * SQ0 - rQ * SV0) * x;
    SV1 = SV0 + (-rU * SQ0 + rQ * SU0) * x;
  }
  x = dlam;
  double aP2 = aQ * aQ + aU * aU + aV * aV;
  if (aP2 > CUT_PREVENT_NAN) {
    double aP = sqrt(aP2);
    double tauP = aP * x, tauI = aI * x;
    double ads0 = aQ * SQ1 + aU * SU1 + aV * SV1;
    double adj = aQ * jQ + aU * jU + aV * jV;
    double efacm = exp(-tauI + tauP), efacp = exp(-tauI - tauP), efac = exp(-tauI);
    SI2 = efacm * (SI1 / 2. - ads0 / (2. * aP)) + efacp * (SI1 / 2. + ads0 / (2. * aP));
    SQ2 = efacm * (-SI1 * aQ * aP + ads0 * aQ) / (2. * aP2) + efacp * (SI1 * aQ * aP + ads0 * aQ) / (2. * aP2) +
          efac * (SQ1 - ads0 * aQ / (aP2));
    SU2 = efacm * (-SI1 * aU * aP + ads0 * aU) / (2. * aP2) + efacp * (SI1 * aU * aP + ads0 * aU) / (2. * aP2) +
          efac * (SU1 - ads0 * aU / (aP2));
    SV2 = efacm * (-SI1 * aV * aP + ads0 * aV) / (2. * aP2) + efacp * (SI1 * aV * aP + ads0 * aV) / (2. * aP2) +
          efac * (SV1 - ads0 * aV / (aP2));
    double afacm = 1. - efacm, afac = 1. - efac, afacp = 1. - efacp;
    if (tauI - tauP <= CUT_SMALL_OPTICAL_DEPTH) {
      double e = tauI - tauP;
      afacm = e * (1. - (e / 2.) * (1. - e / 3.));
      if (tauI <= CUT_SMALL_OPTICAL_DEPTH) {
        e = tauI;
        afac = e * (1. - (e / 2.) * (1. - e / 3.));
        if (tauI + tauP <= CUT_SMALL_OPTICAL_DEPTH) {
          e = tauI + tauP;
          afacp = e * (1. - (e / 2.) * (1. - e / 3.));
        }
      }
    }
    SQ2 += afac * (jQ / aI - aQ * adj / (aI * aP2));
    SU2 += afac * (jU / aI - aU * adj / (aI * aP2));
    SV2 += afac * (jV / aI - aV * adj / (aI * aP2));
    SI2 += afacm * (aP * jI - adj) / (2. * aP * (aI - aP));
    SQ2 += afacm * aQ * (-aP * jI + adj) / (2. * aP2 * (aI - aP));
    SU2 += afacm * aU * (-aP * jI + adj) / (2. * aP2 * (aI - aP));
    SV2 += afacm * aV * (-aP * jI + adj) / (2. * aP2 * (aI - aP));
    SI2 += afacp * (aP * jI + adj) / (2. * aP * (aI + aP));
    SQ2 += afacp * aQ * (aP * jI + adj) / (2. * aP2 * (aI + aP));
    SU2 += afacp * aU * (aP * jI + adj) / (2. * aP2 * (aI + aP));
    SV2 += afacp * aV * (aP * jI + adj) / (2. * aP2 * (aI + aP));
  } else {
    double tau_fake = 0;
    SI2 = approximate_solve(SI1, jI, aI, jI, aI, x, &tau_fake);
    SQ2 = approximate_solve(SQ1, jQ, aI, jQ, aI, x, &tau_fake);
    SU2 = approximate_solve(SU1, jU, aI, jU, aI, x, &tau_fake);
    SV2 = approximate_solve(SV1, jV, aI, jV, aI, x, &tau_fake);
  }
  x = dlam * 0.5;
  rho2 = rQ * rQ + rU * rU + rV * rV;
  if (rho2 > CUT_PREVENT_NAN) {
    double rdS = rQ * SQ2 + rU * SU2 + rV * SV2;
    double rho = sqrt(rho2);
    double cc = cos(rho * x), s = sin(rho * x), sh = sin(0.5 * rho * x);
    SI = SI2;
    SQ = SQ2 * cc + 2 * rQ * rdS / rho2 * sh * sh + (rU * SV2 - rV * SU2) / rho * s;
    SU = SU2 * cc + 2 * rU * rdS / rho2 * sh * sh + (rV * SQ2 - rQ * SV2) / rho * s;
    SV = SV2 * cc + 2 * rV * rdS / rho2 * sh * sh + (rQ * SU2 - rU * SQ2) / rho * s;
  } else {
    SI = SI2;
    SQ = SQ2 + (-rV * SU2 + rU * SV2) * x;
    SU = SU2 + (rV * SQ2 - rQ * SV2) * x;
    SV = SV2 + (-rU * SQ2 + rQ * SU2) * x;
  }
  *tauF += dlam * fabs(rV);
  if (c->stokes_floors) {
    if (SI < 0) {
      SI = 0; SQ = 0; SU = 0; SV = 0;
    } else {
      double pol_frac = sqrt(SQ * SQ + SU * SU + SV * SV) / SI;
      if (pol_frac > 1.) {
        SQ /= pol_frac;
        SU /= pol_frac;
        SV /= pol_frac;
      }
    }
  }
  stokes_to_tensor(SI, SQ, SU, SV, N_tetrad);
  tetrad_to_coord2(N_tetrad, Econ, N_coord);
  if (*tauF > 1.e100 || *tauF < -1.e100 || isnan(*tauF)) oddflag |= 2;
  if (isnan(creal(N_tetrad[0][0])) || isnan(creal(N_coord[0][0]))) oddflag |= 4;
  if (isnan(Ucov[0])) oddflag |= 8;
  return oddflag;
}

static int integrate_emission(const orc_model *m, const orc_camera *c, traj_t *traj, int nsteps, double *Intensity,
                              double *Tau, double *tauF, double complex N_coord[NDIM][NDIM])
{
  *tauF = 0.;
  *Intensity = 0.;
  *Tau = 0.;
  double js = 0., ks;
  int oddflag = 0;
  get_jkinv(m, c, traj[nsteps].X, traj[nsteps].Kcon, &js, &ks);
  for (int nstep = nsteps; nstep > 0; --nstep) {
    int sflag = 0;
    traj_t ti = traj[nstep], tf = traj[nstep - 1];
    if (!c->only_unpolarized) {
      double complex Nh[NDIM][NDIM];
      push_polar(m, ti.X, ti.Kcon, N_coord, N_coord, Nh, 0.5 * ti.dl);
      push_polar(m, ti.Xhalf, ti.Kconhalf, N_coord, Nh, N_coord, ti.dl);
    }
    if (radiating_region(m, tf.X)) {
      int zero_emission = 0;
      if (c->target_nturns >= 0 && ti.nturns != c->target_nturns) zero_emission = 1;
      if (c->counterjet == 1) {
        if (tf.X[2] < (m->cstopx[2] - m->cstartx[2]) / 2) zero_emission = 1;
      } else if (c->counterjet == 2) {
        if (tf.X[2] > (m->cstopx[2] - m->cstartx[2]) / 2) zero_emission = 1;
      }
      double ji = js, ki = ks, jf, kf;
      get_jkinv(m, c, tf.X, tf.Kcon, &jf, &kf);
      js = jf;
      ks = kf;
      if (zero_emission) *Intensity = approximate_solve(*Intensity, 0, ki, 0, kf, ti.dl, Tau);
      else *Intensity = approximate_solve(*Intensity, ji, ki, jf, kf, ti.dl, Tau);
      if (!c->only_unpolarized) sflag |= evolve_N(m, c, tf.X, tf.Kcon, ti.dl, N_coord, tauF, zero_emission);
    }
    oddflag |= sflag;
  }
  return oddflag;
}

static void project_N(const orc_camera *c, double complex N_coord[NDIM][NDIM], double *I_, double *Q_, double *U_,
                      double *V_)
{
  double complex N_tetrad[NDIM][NDIM];
  double Ecov[NDIM][NDIM], Q, U;
  memcpy(Ecov, c->Ecov, sizeof(Ecov));
  coord_to_tetrad2(N_coord, Ecov, N_tetrad);
  tensor_to_stokes(N_tetrad, I_, &Q, &U, V_);
  double rotcam = c->rotcam * -2.;
  *Q_ = Q * cos(rotcam) - U * sin(rotcam);
  *U_ = Q * sin(rotcam) + U * cos(rotcam);
}

/* init_XK, src/model_geodesics.c:178-212 */
static void init_XK(const orc_camera *c, long i, long j, double X[NDIM], double Kcon[NDIM])
{
  double Kt[NDIM];
  double dxoff = (i + 0.5 + c->xoff - 0.01) / c->nx - 0.5;
  double dyoff = (j + 0.5 + c->yoff) / c->ny - 0.5;
  Kt[0] = 0.;
  Kt[1] = (dxoff * cos(c->rotcam) - dyoff * sin(c->rotcam)) * c->fovx;
  Kt[2] = (dxoff * sin(c->rotcam) + dyoff * cos(c->rotcam)) * c->fovy;
  Kt[3] = 1.;
  null_normalize(Kt, 1.);
  for (int l = 0; l < 4; l++)
    Kcon[l] = c->Econ[0][l] * Kt[0] + c->Econ[1][l] * Kt[1] + c->Econ[2][l] * Kt[2] + c->Econ[3][l] * Kt[3];
  for (int mu = 0; mu < NDIM; mu++) X[mu] = c->Xcam[mu];
}

int orc_trace_pixel(const orc_model *m, const orc_camera *c, int i, int j, double out[9])
{
  double X[NDIM] = {0.}, Kcon[NDIM] = {0.};
  double complex N_coord[NDIM][NDIM];
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) N_coord[a][b] = 0.;
  double Intensity = 0., Tau = 0., tauF = 0., Is = 0., Qs = 0., Us = 0., Vs = 0.;
  init_XK(c, i, j, X, Kcon);
  traj_t *traj = (traj_t *)calloc(c->maxnstep, sizeof(traj_t));
  for (int mu = 0; mu < NDIM; mu++) Kcon[mu] *= c->freq;
  int nstep = trace_geodesic(m, c, X, Kcon, traj, c->maxnstep);
  int oddflag = 0;
  if (nstep >= c->maxnstep - 1) {
    free(traj);
    for (int q = 0; q < 9; q++) out[q] = 0.;
    out[7] = nstep;
    return 1;
  }
  oddflag = integrate_emission(m, c, traj, nstep, &Intensity, &Tau, &tauF, N_coord);
  if (!c->only_unpolarized) project_N(c, N_coord, &Is, &Qs, &Us, &Vs);
  free(traj);
  out[0] = Intensity;
  out[1] = Tau;
  out[2] = tauF;
  out[3] = Is;
  out[4] = Qs;
  out[5] = Us;
  out[6] = Vs;
  out[7] = nstep;
  out[8] = oddflag;
  return 0;
}

static long long g_last_steps = 0;

void orc_trace_pixels(const orc_model *m, const orc_camera *c, const int *ij, int n, double *out, int threads)
{
  long long steps = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : steps) num_threads(threads > 0 ? threads : 1) if (threads != 1)
  for (int q = 0; q < n; q++) {
    orc_trace_pixel(m, c, ij[2 * q], ij[2 * q + 1], out + 9 * q);
    steps += (long long)out[9 * q + 7];
  }
  g_last_steps = steps;
}

long long orc_last_steps(void) { return g_last_steps; }

/* root_find / native_coord, src/coordinates.c:375-442 */
static double theta_func(const orc_model *m, const double X[NDIM])
{
  double r, th;
  bl_coord(m, X, &r, &th);
  return th;
}

static double root_find(const orc_model *m, const double X[NDIM])
{
  double th = X[2], tha, thb, thc;
  double Xa[NDIM] = {0}, Xb[NDIM] = {0}, Xc[NDIM] = {0};
  Xa[1] = log(X[1]);
  Xa[3] = X[3];
  Xb[1] = Xa[1];
  Xb[3] = Xa[3];
  Xc[1] = Xa[1];
  Xc[3] = Xa[3];
  if (X[2] < M_PI / 2.) {
    Xa[2] = m->cstartx[2];
    Xb[2] = (m->cstopx[2] - m->cstartx[2]) / 2 + SMALL;
  } else {
    Xa[2] = (m->cstopx[2] - m->cstartx[2]) / 2 - SMALL;
    Xb[2] = m->cstopx[2];
  }
  double tol = 1.e-9;
  tha = theta_func(m, Xa);
  thb = theta_func(m, Xb);
  if (fabs(tha - th) < tol) return Xa[2];
  else if (fabs(thb - th) < tol) return Xb[2];
  for (int q = 0; q < 1000; q++) {
    Xc[2] = 0.5 * (Xa[2] + Xb[2]);
    thc = theta_func(m, Xc);
    if ((thc - th) * (thb - th) < 0.) Xa[2] = Xc[2];
    else Xb[2] = Xc[2];
    double err = theta_func(m, Xc) - th;
    if (fabs(err) < tol) break;
  }
  return Xc[2];
}

double orc_camera_setup(const orc_model *m, double rcam, double thetacam, double phicam, double rotcam_deg,
                        double fov_muas, double dsource_pc, int nx, int ny, double freqcgs, orc_camera *c)
{
  memset(c, 0, sizeof(*c));
  double x[NDIM] = {0., rcam, thetacam / 180. * M_PI, phicam / 180. * M_PI};
  c->Xcam[0] = 0.0;
  c->Xcam[1] = log(rcam);
  c->Xcam[2] = root_find(m, x);
  c->Xcam[3] = phicam / 180. * M_PI;
  c->rotcam = rotcam_deg * (M_PI / 180.);
  double Dsource = dsource_pc * PC;
  double fov_to_d = Dsource / m->L_unit / MUAS_PER_RAD;
  double DX = fov_muas * fov_to_d, DY = fov_muas * fov_to_d;
  c->fovx = DX / rcam;
  c->fovy = DY / rcam;
  c->freq = freqcgs * HPL / (ME * CL * CL);
  c->nx = nx;
  c->ny = ny;
  c->eps = 0.01;
  c->maxnstep = 50000;
  c->emission_type = 4;
  c->target_nturns = -1;
  make_camera_tetrad(m, c->Xcam, c->Econ, c->Ecov);
  return (DX * m->L_unit / nx) * (DY * m->L_unit / ny) / (Dsource * Dsource) / JY;
}
