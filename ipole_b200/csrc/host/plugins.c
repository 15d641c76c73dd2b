/* Host side of the known-answer models: their init_model (geometry, units,
 * constants), the model-specific image header, and the upload dispatch.
 *
 *   analytic  model/analytic/model.c:79-187 (init_model, set_units,
 *             output_hdf5): the five GRRT test problems of Gold et al. 2020
 *   sphere    model/sphere/model.c:53-110, 199-204: an isothermal,
 *             optically thin sphere with a poloidal field in eMinkowski
 *
 * The device side is ipole_b200/csrc/ipg_plugins.cuh. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "../ipg_constants.h"
#include "ipgc.h"
#include "ipole_host.h"

static void analytic_init(const ipg_params *p, ipg_iharm_model *m)
{
  ipg_plugin *pl = &m->plugin;
  ipg_grid *g = &m->grid;
  memset(pl, 0, sizeof(*pl));
  pl->kind = IPG_PLUGIN_ANALYTIC;
  pl->model = p->analytic_model;
  double a = 0.;
  /* init_model, model/analytic/model.c:86-117 */
  switch (pl->model) {
    case 1: pl->A = 0; pl->alpha = -3; pl->height = 0; pl->l0 = 0; a = 0.9; break;
    case 2: pl->A = 0; pl->alpha = -2; pl->height = 0; pl->l0 = 1; a = 0; break;
    case 3: pl->A = 0; pl->alpha = 0; pl->height = 10. / 3; pl->l0 = 1; a = 0.9; break;
    case 4: pl->A = 1.e5; pl->alpha = 0; pl->height = 10. / 3; pl->l0 = 1; a = 0.9; break;
    case 5: pl->A = 1.e6; pl->alpha = 0; pl->height = 100. / 3; pl->l0 = 1; a = 0.9; break;
  }
  pl->freqcgs = p->freqcgs;
  /* set_units, model/analytic/model.c:126-160 */
  double MBH_solar = p->MBH_set ? p->MBH_solar : 4.e6;
  m->MBH = MBH_solar * IPG_MSUN;
  m->L_unit = IPG_GNEWT * m->MBH / (IPG_CL * IPG_CL);
  m->T_unit = m->L_unit / IPG_CL;
  m->RHO_unit = (p->rho_unit > 0) ? p->rho_unit : 3.e-18;
  m->B_unit = IPG_CL * sqrt(4. * M_PI * m->RHO_unit);
  m->M_unit = 0.;
  pl->rho_unit = m->RHO_unit;
  pl->B_unit = m->B_unit;
  memset(g, 0, sizeof(*g));
  g->metric = IPG_METRIC_MKS;
  g->hslope = 1.0;
  g->a = a;
  g->Rh = 1 + sqrt(1. - a * a);
  g->Rin = g->Rh;
  g->Rout = 1000.0;
  g->rmin_geo = 1.;
  g->rmax_geo = 10000.;
  g->startx[1] = log(g->Rin);
  g->stopx[1] = log(g->Rout);
  g->stopx[2] = 1.0;
  g->stopx[3] = 2 * M_PI;
  for (int mu = 0; mu < 4; mu++) {
    g->cstartx[mu] = g->startx[mu];
    g->cstopx[mu] = g->stopx[mu];
  }
  g->L_unit = m->L_unit;
  double z1 = 1. + pow(1. - a * a, 1. / 3.) * (pow(1. + a, 1. / 3.) + pow(1. - a, 1. / 3.));
  double z2 = sqrt(3. * a * a + z1 * z1);
  double r_isco = 3. + z2 - copysign(sqrt((3. - z1) * (3. + z1 + 2. * z2)), a);
  printf("Running analytic model %d:\nMBH: %g\na: %g\nRh: %g\nR_isco: %g\n\n", pl->model, m->MBH, a, g->Rh, r_isco);
  printf("A: %g\nalpha: %g\nh: %g\nl0: %g\n\n", pl->A, pl->alpha, pl->height, pl->l0);
}

static void sphere_init(const ipg_params *p, ipg_iharm_model *m)
{
  ipg_plugin *pl = &m->plugin;
  ipg_grid *g = &m->grid;
  memset(pl, 0, sizeof(*pl));
  pl->kind = IPG_PLUGIN_SPHERE;
  /* init_model, model/sphere/model.c:53-110 */
  double MBH = (p->MBH_set ? p->MBH_solar : 4.1e6) * IPG_MSUN;
  m->MBH = MBH;
  m->L_unit = IPG_GNEWT * MBH / (IPG_CL * IPG_CL);
  pl->R0 = p->sphere_R0;
  pl->Thetae0 = p->sphere_Thetae0;
  pl->Ne0 = p->sphere_tau0 / IPG_SIGMA_THOMSON / pl->R0 / m->L_unit;
  double gam = p->sphere_gam;
  /* the RAPTOR / kmonty convention, the one the reference keeps */
  double THETAE_UNIT = IPG_MP / IPG_ME * (gam - 1.) / (1. + p->tp_over_te);
  pl->B0 = IPG_CL * sqrt(8 * M_PI * (gam - 1.) * (IPG_MP + IPG_ME) / p->sphere_beta0) * sqrt(pl->Ne0 * pl->Thetae0) /
           sqrt(THETAE_UNIT);
  pl->sigma0 = pl->Thetae0 * p->tp_over_te / p->sphere_beta0;
  pl->beta0 = p->sphere_beta0;
  fprintf(stderr, "Running with isothermal sphere model.\n");
  fprintf(stderr, "MBH, L_unit: %g [Msun], %g\n", MBH / IPG_MSUN, m->L_unit);
  fprintf(stderr, "Ne, Thetae, B: %g %g %g\n", pl->Ne0, pl->Thetae0, pl->B0);
  fprintf(stderr, "Rout: %g\n", pl->R0 * m->L_unit);
  memset(g, 0, sizeof(*g));
  g->metric = IPG_METRIC_EMINKOWSKI;
  g->n1 = 300;
  g->n2 = 100;
  g->n3 = 1;
  g->dx[0] = 0.1;
  g->dx[1] = (pl->R0 - 0) / g->n1;
  g->dx[2] = M_PI / g->n2;
  g->dx[3] = 2. * M_PI / g->n3;
  g->stopx[0] = 1.;
  g->stopx[1] = g->startx[1] + g->n1 * g->dx[1];
  g->stopx[2] = g->startx[2] + g->n2 * g->dx[2];
  g->stopx[3] = g->startx[3] + g->n3 * g->dx[3];
  for (int mu = 0; mu < 4; mu++) {
    g->cstartx[mu] = g->startx[mu];
    g->cstopx[mu] = g->stopx[mu];
  }
  g->rmin_geo = 0;
  g->rmax_geo = fmax(100., pl->R0);
  g->Rh = 0.; /* never set by the sphere model: the global's zero */
  g->L_unit = m->L_unit;
  fprintf(stderr, "Native coordinate start: %g %g %g stop: %g %g %g\n", g->startx[1], g->startx[2], g->startx[3],
          g->stopx[1], g->stopx[2], g->stopx[3]);
}

/* called by ipg_iharm_load for a non-iharm plugin name; 1 if it handled it */
int ipg__plugin_load(const ipg_params *p, ipg_iharm_model *m, int *rc)
{
  if (strcmp(p->plugin, "iharm") == 0) return 0;
  memset(m, 0, sizeof(*m));
  if (strcmp(p->plugin, "analytic") == 0) {
    analytic_init(p, m);
    *rc = IPG_OK;
  } else if (strcmp(p->plugin, "sphere") == 0) {
    sphere_init(p, m);
    *rc = IPG_OK;
  } else {
    fprintf(stderr, "unknown model plugin '%s' (iharm, analytic, sphere)\n", p->plugin);
    *rc = IPG_E_ARG;
  }
  return 1;
}

int ipg_upload_model(ipg_ctx *ctx, const ipg_iharm_model *m)
{
  if (!ctx || !m) return IPG_E_ARG;
  if (m->plugin.kind != IPG_PLUGIN_IHARM) return ipg_upload_plugin(ctx, &m->grid, &m->plugin);
  return ipg_upload_iharm(ctx, &m->grid, (const double *const *)m->fields);
}

/* output_hdf5 of the known-answer models (model/analytic/model.c:162-187,
 * model/sphere/model.c:199-212) */
void ipg__plugin_write_header(void *fp, const ipg_iharm_model *m)
{
  ipgc_file *f = (ipgc_file *)fp;
  const ipg_plugin *pl = &m->plugin;
  if (pl->kind == IPG_PLUGIN_ANALYTIC) {
    ipgc_put_f64(f, "/header/t", 0.);
    ipgc_put_f64(f, "/header/a", m->grid.a);
    ipgc_put_i32(f, "/header/model", pl->model);
    ipgc_put_f64(f, "/header/A", pl->A);
    ipgc_put_f64(f, "/header/alpha", pl->alpha);
    ipgc_put_f64(f, "/header/height", pl->height);
    ipgc_put_f64(f, "/header/l0", pl->l0);
    ipgc_put_group(f, "/header/units");
    ipgc_put_f64(f, "/header/units/M_unit", 0.);
    ipgc_put_f64(f, "/header/units/L_unit", m->L_unit);
    ipgc_put_f64(f, "/header/units/T_unit", m->T_unit);
  } else if (pl->kind == IPG_PLUGIN_SPHERE) {
    ipgc_put_group(f, "/header/units");
    ipgc_put_f64(f, "/header/units/L_unit", m->L_unit);
  }
}
