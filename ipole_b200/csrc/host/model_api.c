/* The reference's model plugin interface (src/model.h:9-44) with its own
 * names and signatures, over the iharm model the library loads: code
 * written against ipole's model.h links to this library instead of
 * model/iharm/model.c.
 *
 * As in the reference, the interface keeps one model in library-global
 * state: try_set_model_parameter collects the keys, init_model loads the
 * dump they name (ipg_iharm_load, the derived fields of
 * init_physical_quantities) and sets the unit globals, and the point
 * queries read it.  They evaluate on the host, at one point per call, what
 * the ray kernels evaluate on the device at every step: Xtoijk_ghost and
 * interp_scalar (src/grid.c:15-44, 216-334) and get_model_fourv/ne/thetae/
 * b/sigma/beta/primitives (model/iharm/model.c:420-593).  They are for
 * callers of the reference's interface (plotting along a geodesic, set-up
 * code); the images come from the device (ipg_render_image).
 *
 * Where the reference calls exit(), init_model leaves the model unloaded
 * and ipg_model_status() returns the error code. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "coords.h"
#include "ipole_host.h"

double M_unit, L_unit, T_unit, RHO_unit, U_unit, B_unit, Te_unit;

static ipg_params g_par;
static int g_par_ready;
static ipg_iharm_model g_model;
static int g_loaded;
static int g_status = IPG_E_STATE;

static ipg_params *params(void)
{
  if (!g_par_ready) {
    ipg_params_default(&g_par);
    g_par_ready = 1;
  }
  return &g_par;
}

ipg_params *ipg_model_params(void) { return params(); }
const ipg_iharm_model *ipg_model_loaded(void) { return g_loaded ? &g_model : NULL; }
int ipg_model_status(void) { return g_status; }

void try_set_model_parameter(const char *word, const char *value) { ipg_params_set(params(), word, value); }

void init_model(double *tA, double *tB)
{
  if (g_loaded) {
    ipg_iharm_free(&g_model);
    g_loaded = 0;
  }
  g_status = ipg_iharm_load(params(), &g_model);
  if (g_status != IPG_OK) {
    fprintf(stderr, "init_model: %s\n", ipg_strerror(g_status));
    return;
  }
  g_loaded = 1;
  M_unit = g_model.M_unit;
  L_unit = g_model.L_unit;
  T_unit = g_model.T_unit;
  RHO_unit = g_model.RHO_unit;
  U_unit = g_model.U_unit;
  B_unit = g_model.B_unit;
  Te_unit = g_model.Te_unit;
  if (tA) *tA = g_model.t;
  if (tB) *tB = g_model.t;
}

/* X_in_domain (src/grid.c:285-334) for native coordinates */
static int in_domain(const ipg_grid *g, const double X[NDIM])
{
  return !(X[1] < g->startx[1] || X[1] >= g->stopx[1] || X[2] < g->startx[2] || X[2] >= g->stopx[2]);
}

/* Xtoijk_ghost (src/grid.c:216-283): zone of X (ghost-padded indices) and
 * the offsets within it */
static void zone_of(const ipg_grid *g, const double X[NDIM], int *i, int *j, int *k, double del[NDIM])
{
  double phi = fmod(X[3], g->cstopx[3]);
  if (phi < 0.0) phi = g->cstopx[3] + phi;
  *i = (int)((X[1] - g->startx[1]) / g->dx[1] - 0.5 + 1000) - 1000;
  *j = (int)((X[2] - g->startx[2]) / g->dx[2] - 0.5 + 1000) - 1000;
  *k = (int)((phi - g->startx[3]) / g->dx[3] - 0.5 + 1000) - 1000;
  if (*i < -1) *i = -1;
  if (*j < -1) *j = -1;
  if (*k < -1) *k = -1;
  if (*i >= g->n1) *i = g->n1 - 1;
  if (*j >= g->n2) *j = g->n2 - 1;
  if (*k >= g->n3) *k = g->n3 - 1;
  del[0] = 0.;
  del[1] = (X[1] - ((*i + 0.5) * g->dx[1] + g->startx[1])) / g->dx[1];
  del[2] = (X[2] - ((*j + 0.5) * g->dx[2] + g->startx[2])) / g->dx[2];
  del[3] = (phi - ((*k + 0.5) * g->dx[3] + g->startx[3])) / g->dx[3];
  for (int d = 1; d < NDIM; d++) {
    if (del[d] < 0.) del[d] = 0.;
    if (del[d] >= 1.) del[d] = 1.;
  }
  *i += 1;
  *j += 1;
  *k += 1;
}

/* interp_scalar (src/grid.c:15-44): bilinear in x1, x2 on the k and k+1
 * planes, then linear in x3 */
static double interp(const ipg_grid *g, const double X[NDIM], const double *f)
{
  int i, j, k;
  double d[NDIM];
  zone_of(g, X, &i, &j, &k, d);
  const size_t sj = (size_t)g->n3 + 2, si = ((size_t)g->n2 + 2) * sj;
#define F(a, b, c) f[(size_t)(a) * si + (size_t)(b) * sj + (size_t)(c)]
  const double b1 = 1. - d[1], b2 = 1. - d[2];
  double lo = F(i, j, k) * b1 * b2 + F(i, j + 1, k) * b1 * d[2] + F(i + 1, j, k) * d[1] * b2 +
              F(i + 1, j + 1, k) * d[1] * d[2];
  double hi = F(i, j, k + 1) * b1 * b2 + F(i, j + 1, k + 1) * d[2] * b1 + F(i + 1, j, k + 1) * d[1] * b2 +
              F(i + 1, j + 1, k + 1) * d[1] * d[2];
#undef F
  return (1. - d[3]) * lo + d[3] * hi;
}

static int ready(void) { return g_loaded && g_model.plugin.kind == IPG_PLUGIN_IHARM; }

/* radiating_region, model/iharm/model.c:2093-2098 */
int radiating_region(double X[NDIM])
{
  if (!g_loaded) return 0;
  double r, th;
  hc_bl_coord(&g_model.grid, X, &r, &th);
  const ipg_grid *g = &g_model.grid;
  return r > g->rmin_geo && r < g->rmax_geo && th > g->th_beg && th < (M_PI - g->th_beg);
}

double get_model_thetae(double X[NDIM])
{
  if (!ready() || !in_domain(&g_model.grid, X)) return 0.;
  return interp(&g_model.grid, X, g_model.fields[IPG_F_THETAE]);
}

double get_model_b(double X[NDIM])
{
  if (!ready() || !in_domain(&g_model.grid, X)) return 0.;
  return interp(&g_model.grid, X, g_model.fields[IPG_F_B]);
}

double get_model_sigma(double X[NDIM])
{
  if (!ready() || !in_domain(&g_model.grid, X)) return 0.;
  return interp(&g_model.grid, X, g_model.fields[IPG_F_SIGMA]);
}

double get_model_beta(double X[NDIM])
{
  if (!ready() || !in_domain(&g_model.grid, X) || !g_model.trace_fields[2]) return 0.;
  return interp(&g_model.grid, X, g_model.trace_fields[2]);
}

/* get_model_ne with the geodesic sigma cut (model/iharm/model.c:567-593):
 * no electrons above sigma_cut, and a cosine taper up to sigma_cut_high
 * when that is set */
double get_model_ne(double X[NDIM])
{
  if (!ready() || !in_domain(&g_model.grid, X)) return 0.;
  const ipg_grid *g = &g_model.grid;
  const double sigma = get_model_sigma(X);
  if (sigma > g->sigma_cut) return 0.;
  const double above = g->sigma_cut_high > 0 ? g->sigma_cut_high : g->sigma_cut;
  double fac = 1.;
  if (!(sigma < g->sigma_cut)) fac = (sigma >= above) ? 0. : cos(M_PI / 2. / (above - g->sigma_cut) * (sigma - g->sigma_cut));
  return interp(g, X, g_model.fields[IPG_F_NE]) * fac;
}

/* get_model_fourv, model/iharm/model.c:420-493 */
void get_model_fourv(double X[NDIM], double Kcon[NDIM], double Ucon[NDIM], double Ucov[NDIM], double Bcon[NDIM],
                     double Bcov[NDIM])
{
  (void)Kcon;
  for (int m = 0; m < NDIM; m++) Ucon[m] = Ucov[m] = Bcon[m] = Bcov[m] = 0.;
  if (!ready()) return;
  const ipg_grid *g = &g_model.grid;
  double gcov[NDIM][NDIM], gcon[NDIM][NDIM];
  hc_gcov_func(g, X, gcov);
  hc_invert_matrix(gcov, gcon);
  if (!in_domain(g, X)) {
    /* the normal observer, no field */
    Ucov[0] = -1. / sqrt(-gcon[0][0]);
    for (int m = 0; m < NDIM; m++) Ucon[m] = Ucov[0] * gcon[m][0];
    return;
  }
  double V[NDIM] = {0., interp(g, X, g_model.fields[IPG_F_U1]), interp(g, X, g_model.fields[IPG_F_U2]),
                    interp(g, X, g_model.fields[IPG_F_U3])};
  double VdotV = 0.;
  for (int a = 1; a < NDIM; a++)
    for (int b = 1; b < NDIM; b++) VdotV += gcov[a][b] * V[a] * V[b];
  const double Vfac = sqrt(-1. / gcon[0][0] * (1. + fabs(VdotV)));
  Ucon[0] = -Vfac * gcon[0][0];
  for (int a = 1; a < NDIM; a++) Ucon[a] = V[a] - Vfac * gcon[0][a];
  hc_flip_index(Ucon, gcov, Ucov);
  const double B1 = interp(g, X, g_model.fields[IPG_F_B1]), B2 = interp(g, X, g_model.fields[IPG_F_B2]),
               B3 = interp(g, X, g_model.fields[IPG_F_B3]);
  Bcon[0] = B1 * Ucov[1] + B2 * Ucov[2] + B3 * Ucov[3];
  Bcon[1] = (B1 + Ucon[1] * Bcon[0]) / Ucon[0];
  Bcon[2] = (B2 + Ucon[2] * Bcon[0]) / Ucon[0];
  Bcon[3] = (B3 + Ucon[3] * Bcon[0]) / Ucon[0];
  hc_flip_index(Bcon, gcov, Bcov);
}

/* get_model_primitives (model/iharm/model.c): rho, u, U1..3, B1..3 at X */
void get_model_primitives(double X[NDIM], double *p)
{
  if (!ready() || !in_domain(&g_model.grid, X) || !g_model.trace_fields[0]) return;
  const ipg_grid *g = &g_model.grid;
  p[0] = interp(g, X, g_model.trace_fields[0]);
  p[1] = interp(g, X, g_model.trace_fields[1]);
  for (int q = 0; q < 6; q++) p[2 + q] = interp(g, X, g_model.fields[IPG_F_U1 + q]);
}

/* the iharm model has no custom emissivities (emission_type 10): the
 * reference's get_model_jar for it returns zeros */
void get_model_jar(double X[NDIM], double Kcon[NDIM], double *jI, double *jQ, double *jU, double *jV, double *aI,
                   double *aQ, double *aU, double *aV, double *rQ, double *rU, double *rV)
{
  (void)X;
  (void)Kcon;
  *jI = *jQ = *jU = *jV = *aI = *aQ = *aU = *aV = *rQ = *rU = *rV = 0.;
}

/* one dump, fast light: the data never changes between the times */
void update_data(double *tA, double *tB)
{
  (void)tA;
  (void)tB;
}

void update_data_until(double *tA, double *tB, double tgt)
{
  (void)tA;
  (void)tB;
  (void)tgt;
}
