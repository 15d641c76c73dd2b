/* iharm fluid model set-up on the host: grid header, units, primitive load,
 * magnetic-field magnitude, ghost zones and derived fields, following
 * model/iharm/model.c (init_iharm_grid :848-1074, set_units :595-608,
 * load_iharm_data :1876-2090, populate_boundary_conditions :1314-1370,
 * init_physical_quantities :610-717).  The per-point queries of the model
 * (get_model_fourv, get_model_ne, ...) run on the device. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../ipg_constants.h"
#include "coords.h"
#include "ipgc.h"
#include "../ipg_internal.h"
#include "ipole_host.h"

#define KRHO 0
#define UU 1
#define U1 2
#define U2 3
#define U3 4
#define B1 5
#define B2 6
#define B3 7
#define NPRIM_STORE 8

typedef struct {
  int n1, n2, n3;
  double *p[NPRIM_STORE];
  double *b;
} fluid_t;

static inline size_t IDX(const fluid_t *f, int i, int j, int k)
{
  return ((size_t)i * (f->n2 + 2) + j) * (f->n3 + 2) + k;
}

/* the mass-unit part of set_units: RHO_unit and B_unit of M_unit at L_unit */
void ipg__units(double M_unit, double L_unit, double *RHO_unit, double *B_unit)
{
  *RHO_unit = M_unit / pow(L_unit, 3);
  *B_unit = IPG_CL * sqrt(4. * M_PI * *RHO_unit);
}

/* set_units, model/iharm/model.c:595-608 */
static void set_units(ipg_iharm_model *m, double MBH_solar, double *Mdotedd)
{
  m->MBH = MBH_solar * IPG_MSUN;
  m->L_unit = IPG_GNEWT * m->MBH / (IPG_CL * IPG_CL);
  m->T_unit = m->L_unit / IPG_CL;
  ipg__units(m->M_unit, m->L_unit, &m->RHO_unit, &m->B_unit);
  m->U_unit = m->RHO_unit * IPG_CL * IPG_CL;
  *Mdotedd = 4. * M_PI * IPG_GNEWT * m->MBH * IPG_MP / IPG_CL / 0.1 / IPG_SIGMA_THOMSON;
  fprintf(stderr, "MBH: %g [Msun]\n", m->MBH / IPG_MSUN);
  fprintf(stderr, "L,T,M units: %g [cm] %g [s] %g [g]\n", m->L_unit, m->T_unit, m->M_unit);
  fprintf(stderr, "rho,u,B units: %g [g cm^-3] %g [g cm^-1 s^-2] %g [G] \n", m->RHO_unit, m->U_unit, m->B_unit);
}

/* populate_boundary_conditions, model/iharm/model.c:1314-1370 */
static void boundary_conditions(fluid_t *f)
{
  const int N1 = f->n1, N2 = f->n2, N3 = f->n3;
  for (int j = 1; j < N2 + 1; ++j)
    for (int k = 1; k < N3 + 1; ++k) {
      for (int l = 0; l < NPRIM_STORE; ++l) {
        f->p[l][IDX(f, 0, j, k)] = f->p[l][IDX(f, 1, j, k)];
        f->p[l][IDX(f, N1 + 1, j, k)] = f->p[l][IDX(f, N1, j, k)];
      }
      f->b[IDX(f, 0, j, k)] = f->b[IDX(f, 1, j, k)];
      f->b[IDX(f, N1 + 1, j, k)] = f->b[IDX(f, N1, j, k)];
    }
  for (int i = 0; i < N1 + 2; ++i)
    for (int k = 1; k < N3 + 1; ++k) {
      if (N3 % 2 == 0) {
        int kflip = ((k - 1) + (N3 / 2)) % N3 + 1;
        for (int l = 0; l < NPRIM_STORE; ++l) {
          f->p[l][IDX(f, i, 0, k)] = f->p[l][IDX(f, i, 1, kflip)];
          f->p[l][IDX(f, i, N2 + 1, k)] = f->p[l][IDX(f, i, N2, kflip)];
        }
        f->b[IDX(f, i, 0, k)] = f->b[IDX(f, i, 1, kflip)];
        f->b[IDX(f, i, N2 + 1, k)] = f->b[IDX(f, i, N2, kflip)];
      } else {
        int kflip1 = (k + (N3 / 2)) % N3;
        int kflip2 = (k + (N3 / 2) + 1) % N3;
        for (int l = 0; l < NPRIM_STORE; ++l) {
          f->p[l][IDX(f, i, 0, k)] = (f->p[l][IDX(f, i, 1, kflip1)] + f->p[l][IDX(f, i, 1, kflip2)]) / 2.;
          f->p[l][IDX(f, i, N2 + 1, k)] = (f->p[l][IDX(f, i, N2, kflip1)] + f->p[l][IDX(f, i, N2, kflip2)]) / 2.;
        }
        f->b[IDX(f, i, 0, k)] = (f->b[IDX(f, i, 1, kflip1)] + f->b[IDX(f, i, 1, kflip2)]) / 2.;
        f->b[IDX(f, i, N2 + 1, k)] = (f->b[IDX(f, i, N2, kflip1)] + f->b[IDX(f, i, N2, kflip2)]) / 2.;
      }
    }
  for (int i = 0; i < N1 + 2; ++i)
    for (int j = 0; j < N2 + 2; ++j) {
      for (int l = 0; l < NPRIM_STORE; ++l) {
        f->p[l][IDX(f, i, j, 0)] = f->p[l][IDX(f, i, j, N3)];
        f->p[l][IDX(f, i, j, N3 + 1)] = f->p[l][IDX(f, i, j, 1)];
      }
      f->b[IDX(f, i, j, 0)] = f->b[IDX(f, i, j, N3)];
      f->b[IDX(f, i, j, N3 + 1)] = f->b[IDX(f, i, j, 1)];
    }
}

void ipg_iharm_free(ipg_iharm_model *m)
{
  for (int f = 0; f < IPG_NFIELD; f++) {
    free(m->fields[f]);
    m->fields[f] = NULL;
  }
  for (int f = 0; f < 3; f++) {
    free(m->trace_fields[f]);
    m->trace_fields[f] = NULL;
  }
  free(m->bmag_code);
  m->bmag_code = NULL;
  if (m->fluid_header) {
    ipgc_free((ipgc_file *)m->fluid_header);
    free(m->fluid_header);
    m->fluid_header = NULL;
  }
}

int ipg_iharm_load(const ipg_params *p, ipg_iharm_model *m)
{
  int prc;
  if (ipg__plugin_load(p, m, &prc)) return prc;
  memset(m, 0, sizeof(*m));
  ipg_grid *g = &m->grid;
  ipgc_file file;
  char fname[IPG_STRLEN];
  snprintf(fname, sizeof(fname), p->dump, p->dump_min);
  fprintf(stderr, "Determining dump file type... ");
  int lrc = ipgc_load(fname, &file);
  if (lrc != 0) {
    fprintf(stderr, "! unable to open file %s. Exiting!\n  (%s)\n", fname, ipgc_error());
    return lrc == -2 ? IPG_E_FORMAT : IPG_E_IO;
  }
  fprintf(stderr, "iharm!\n");

  /* --- init_iharm_grid --- */
  if (ipgc_find(&file, "/header/has_derefine_poles")) {
    fprintf(stderr, "Dump includes flag 'has_derefine_poles' and is therefore non-standard and not well-defined");
    ipgc_free(&file);
    return IPG_E_FORMAT;
  }
  if (ipgc_find(&file, "/header/weights")) {
    fprintf(stderr, "! dumps with /header/weights (fluid-temperature electrons) are not supported\n");
    ipgc_free(&file);
    return IPG_E_FORMAT;
  }
  char metric_name[32] = {0};
  if (ipgc_get_str(&file, "/header/metric", metric_name, sizeof(metric_name)) != 0 ||
      (strncmp(metric_name, "MMKS", 19) != 0 && strncmp(metric_name, "FMKS", 19) != 0)) {
    fprintf(stderr, "File is in metric '%s'; this program supports FMKS/MMKS only.\n", metric_name);
    ipgc_free(&file);
    return IPG_E_FORMAT;
  }
  m->gam = 1.444444444444444;
  m->game = 1.333333333333333;
  m->gamp = 1.666666666666667;
  if (ipgc_get_i32(&file, "/header/n1", &g->n1) || ipgc_get_i32(&file, "/header/n2", &g->n2) ||
      ipgc_get_i32(&file, "/header/n3", &g->n3) || ipgc_get_f64(&file, "/header/gam", &m->gam)) {
    ipgc_free(&file);
    return IPG_E_FORMAT;
  }
  if (ipgc_find(&file, "/header/gam_e")) {
    fprintf(stderr, "custom electron model loaded from dump file...\n");
    ipgc_get_f64(&file, "/header/gam_e", &m->game);
    ipgc_get_f64(&file, "/header/gam_p", &m->gamp);
  }
  m->electrons = 2; /* USE_MIXED_TPTE, model/iharm/model.c:952-956 */
  fprintf(stderr, "Using mixed tp_over_te with trat_small = %g, trat_large = %g, and beta_crit = %g\n", p->trat_small,
          p->trat_large, p->beta_crit);
  fprintf(stderr, "sigma_cut = %g\n", p->sigma_cut);
  m->Te_unit = 0.; /* Thetae_unit is still zero when init_iharm_grid copies it */

  int bad = 0;
  bad |= ipgc_get_f64(&file, "/header/geom/startx1", &g->startx[1]);
  bad |= ipgc_get_f64(&file, "/header/geom/startx2", &g->startx[2]);
  bad |= ipgc_get_f64(&file, "/header/geom/startx3", &g->startx[3]);
  bad |= ipgc_get_f64(&file, "/header/geom/dx1", &g->dx[1]);
  bad |= ipgc_get_f64(&file, "/header/geom/dx2", &g->dx[2]);
  bad |= ipgc_get_f64(&file, "/header/geom/dx3", &g->dx[3]);
  bad |= ipgc_get_f64(&file, "/header/geom/mmks/a", &g->a);
  bad |= ipgc_get_f64(&file, "/header/geom/mmks/hslope", &g->hslope);
  if (ipgc_find(&file, "/header/geom/mmks/Rin")) {
    bad |= ipgc_get_f64(&file, "/header/geom/mmks/Rin", &g->Rin);
    bad |= ipgc_get_f64(&file, "/header/geom/mmks/Rout", &g->Rout);
  } else {
    bad |= ipgc_get_f64(&file, "/header/geom/mmks/r_in", &g->Rin);
    bad |= ipgc_get_f64(&file, "/header/geom/mmks/r_out", &g->Rout);
  }
  bad |= ipgc_get_f64(&file, "/header/geom/mmks/poly_xt", &g->poly_xt);
  bad |= ipgc_get_f64(&file, "/header/geom/mmks/poly_alpha", &g->poly_alpha);
  bad |= ipgc_get_f64(&file, "/header/geom/mmks/mks_smooth", &g->mks_smooth);
  bad |= ipgc_get_f64(&file, "/dump_cadence", &m->DTd);
  if (bad) {
    fprintf(stderr, "! dump header incomplete\n");
    ipgc_free(&file);
    return IPG_E_FORMAT;
  }
  fprintf(stderr, "MKS parameters a: %f hslope: %f Rin: %f Rout: %f\n", g->a, g->hslope, g->Rin, g->Rout);
  g->poly_norm = 0.5 * M_PI * 1. / (1. + 1. / (g->poly_alpha + 1.) * 1. / pow(g->poly_xt, g->poly_alpha));
  fprintf(stderr, "MKS parameters poly_xt: %f poly_alpha: %f mks_smooth: %f poly_norm: %f\n", g->poly_xt,
          g->poly_alpha, g->mks_smooth, g->poly_norm);
  g->rmax_geo = fmin(p->rmax_geo, g->Rout);
  g->rmin_geo = fmax(p->rmin_geo, g->Rin);
  g->stopx[0] = 1.;
  g->stopx[1] = g->startx[1] + g->n1 * g->dx[1];
  g->stopx[2] = g->startx[2] + g->n2 * g->dx[2];
  g->stopx[3] = g->startx[3] + g->n3 * g->dx[3];
  for (int i = 0; i < 4; i++) g->cstartx[i] = 0;
  g->cstopx[0] = 0;
  g->cstopx[1] = log(g->Rout);
  g->cstopx[2] = 1.0;
  g->cstopx[3] = 2 * M_PI;
  g->sigma_cut = p->sigma_cut;
  g->sigma_cut_high = p->sigma_cut_high;
  fprintf(stderr, "Native coordinate start: %g %g %g stop: %g %g %g\n", g->cstartx[1], g->cstartx[2], g->cstartx[3],
          g->cstopx[1], g->cstopx[2], g->cstopx[3]);
  fprintf(stderr, "Grid start: %g %g %g stop: %g %g %g\n", g->startx[1], g->startx[2], g->startx[3], g->stopx[1],
          g->stopx[2], g->stopx[3]);

  /* copy of /header for the output's /fluid_header */
  ipgc_file *hdr = (ipgc_file *)calloc(1, sizeof(ipgc_file));
  ipgc_copy_subtree(&file, "/header", hdr, "");
  m->fluid_header = hdr;

  /* --- set_units --- */
  m->M_unit = p->M_unit;
  double Mdotedd;
  set_units(m, p->MBH_solar, &Mdotedd);
  g->L_unit = m->L_unit;

  /* --- load_iharm_data --- */
  fprintf(stderr, "Reading data...\n");
  const int N1 = g->n1, N2 = g->n2, N3 = g->n3;
  fluid_t f = {N1, N2, N3, {0}, NULL};
  size_t ncell = (size_t)(N1 + 2) * (N2 + 2) * (N3 + 2);
  for (int l = 0; l < NPRIM_STORE; l++) f.p[l] = (double *)calloc(ncell, sizeof(double));
  f.b = (double *)calloc(ncell, sizeof(double));
  /* sqrt(b^2) in code units, kept for batched instances, whose b field the
   * device derives per mass unit (interior cells; ghost cells stay zero) */
  m->bmag_code = (double *)calloc(ncell, sizeof(double));
  int n_prims = 0;
  const ipgc_entry *pe = ipgc_find(&file, "/prims");
  if (ipgc_get_i32(&file, "/header/n_prim", &n_prims) || !pe || pe->rank != 4 || pe->kind != IPGC_F64 ||
      (int)pe->dims[0] != N1 || (int)pe->dims[1] != N2 || (int)pe->dims[2] != N3 || (int)pe->dims[3] != n_prims ||
      n_prims < 8) {
    fprintf(stderr, "! /prims missing or not [n1][n2][n3][n_prim]\n");
    for (int l = 0; l < NPRIM_STORE; l++) free(f.p[l]);
    free(f.b);
    ipgc_free(&file);
    return IPG_E_FORMAT;
  }
  const double *prims = (const double *)pe->data;
  for (int i = 0; i < N1; i++)
    for (int j = 0; j < N2; j++)
      for (int k = 0; k < N3; k++)
        for (int l = 0; l < NPRIM_STORE; l++)
          f.p[l][IDX(&f, i + 1, j + 1, k + 1)] = prims[(((size_t)i * N2 + j) * N3 + k) * n_prims + l];
  if (p->reverse_field) {
    for (size_t c = 0; c < ncell; c++) {
      f.p[B1][c] = -1.0 * f.p[B1][c];
      f.p[B2][c] = -1.0 * f.p[B2][c];
      f.p[B3][c] = -1.0 * f.p[B3][c];
    }
  }
  ipgc_get_f64(&file, "/t", &m->t);
  ipgc_free(&file);

  double dMact = 0., Ladv = 0.;
  for (int i = 1; i < N1 + 1; i++) {
    for (int j = 1; j < N2 + 1; j++) {
      double X[NDIM] = {0.};
      double gcov[NDIM][NDIM], gcon[NDIM][NDIM];
      hc_ijktoX(g, i - 1, j - 1, 0, X);
      hc_gcov_func(g, X, gcov);
      hc_invert_matrix(gcov, gcon);
      double gd = hc_gdet_zone(g, i - 1, j - 1, 0);
      for (int k = 1; k < N3 + 1; k++) {
        size_t c = IDX(&f, i, j, k);
        double UdotU = 0.;
        for (int l = 1; l < NDIM; l++)
          for (int mm = 1; mm < NDIM; mm++) UdotU += gcov[l][mm] * f.p[U1 + l - 1][c] * f.p[U1 + mm - 1][c];
        double ufac = sqrt(-1. / gcon[0][0] * (1 + fabs(UdotU)));
        double ucon[NDIM] = {0.};
        ucon[0] = -ufac * gcon[0][0];
        for (int l = 1; l < NDIM; l++) ucon[l] = f.p[U1 + l - 1][c] - ufac * gcon[0][l];
        double ucov[NDIM] = {0.};
        hc_flip_index(ucon, gcov, ucov);
        double udotB = 0.;
        for (int l = 1; l < NDIM; l++) udotB += ucov[l] * f.p[B1 + l - 1][c];
        double bcon[NDIM] = {0.}, bcov[NDIM] = {0.};
        bcon[0] = udotB;
        for (int l = 1; l < NDIM; l++) bcon[l] = (f.p[B1 + l - 1][c] + ucon[l] * udotB) / ucon[0];
        hc_flip_index(bcon, gcov, bcov);
        double bsq = 0.;
        for (int l = 0; l < NDIM; ++l) bsq += bcon[l] * bcov[l];
        const double bcode = sqrt(bsq);
        m->bmag_code[c] = bcode;
        f.b[c] = bcode * m->B_unit;
        if (i <= 21) dMact += gd * f.p[KRHO][c] * ucon[1];
        if (i <= 21) Ladv += gd * f.p[UU][c] * ucon[1] * ucov[0];
      }
    }
  }
  {
    double r_eh = 1. + sqrt(1. - g->a * g->a);
    double X[NDIM] = {0.}, r, th;
    hc_ijktoX(g, 20, N2 / 2, 0, X);
    hc_bl_coord(g, X, &r, &th);
    if (r < r_eh) fprintf(stderr, "warning: zone 21 lies inside r_eh; Mdot in the output header is approximate\n");
  }
  boundary_conditions(&f);
  dMact *= g->dx[3] * g->dx[2];
  dMact /= 21.;
  Ladv *= g->dx[3] * g->dx[2];
  Ladv /= 21.;
  m->Mdot_dump = -dMact * m->M_unit / m->T_unit;
  m->MdotEdd_dump = Mdotedd;
  m->Ladv_dump = Ladv;
  double rescale_factor = 1.;
  if (p->target_mdot > 0) {
    fprintf(stderr, "Resetting M_unit to match target_mdot = %g ", p->target_mdot);
    double current_mdot = m->Mdot_dump / m->MdotEdd_dump;
    fprintf(stderr, "... is now %g\n", m->M_unit * fabs(p->target_mdot / current_mdot));
    rescale_factor = fabs(p->target_mdot / current_mdot);
    m->M_unit *= rescale_factor;
    set_units(m, p->MBH_solar, &Mdotedd);
    g->L_unit = m->L_unit;
  }
  m->Mdot_dump = -dMact * m->M_unit / m->T_unit;
  m->MdotEdd_dump = Mdotedd;
  m->Ladv_dump = Ladv;
  fprintf(stderr, "dMact: %g [code]\n", dMact);
  fprintf(stderr, "Ladv: %g [code]\n", m->Ladv_dump);
  fprintf(stderr, "Mdot: %g [g/s] \n", m->Mdot_dump);
  fprintf(stderr, "Mdot: %g [MSUN/YR] \n", m->Mdot_dump / (IPG_MSUN / IPG_YEAR));
  fprintf(stderr, "Mdot: %g [Mdotedd]\n", m->Mdot_dump / m->MdotEdd_dump);
  fprintf(stderr, "Mdotedd: %g [g/s]\n", m->MdotEdd_dump);
  fprintf(stderr, "Mdotedd: %g [MSUN/YR]\n", m->MdotEdd_dump / (IPG_MSUN / IPG_YEAR));

  /* --- init_physical_quantities (ELECTRONS == 2) --- */
  for (int q = 0; q < IPG_NFIELD; q++) m->fields[q] = (double *)malloc(ncell * sizeof(double));
  memcpy(m->fields[IPG_F_U1], f.p[U1], ncell * sizeof(double));
  memcpy(m->fields[IPG_F_U2], f.p[U2], ncell * sizeof(double));
  memcpy(m->fields[IPG_F_U3], f.p[U3], ncell * sizeof(double));
  memcpy(m->fields[IPG_F_B1], f.p[B1], ncell * sizeof(double));
  memcpy(m->fields[IPG_F_B2], f.p[B2], ncell * sizeof(double));
  memcpy(m->fields[IPG_F_B3], f.p[B3], ncell * sizeof(double));
  double rf = sqrt(rescale_factor);
  const double game = m->game, gamp = m->gamp, gam = m->gam;
  for (size_t c = 0; c < ncell; c++) {
    double rho = f.p[KRHO][c], uu = f.p[UU][c];
    double ne = rho * m->RHO_unit / (IPG_MP + IPG_ME) * 1.;
    double bb = f.b[c] * rf;
    double bsq = bb / m->B_unit;
    bsq = bsq * bsq;
    double sigma_m = bsq / rho;
    double beta_m = uu * (gam - 1.) / 0.5 / bsq;
    double betasq = beta_m * beta_m / p->beta_crit / p->beta_crit;
    double trat = p->trat_large * betasq / (1. + betasq) + p->trat_small / (1. + betasq);
    double lcl_Thetae_u = (IPG_MP / IPG_ME) * (game - 1.) * (gamp - 1.) / ((gamp - 1.) + (game - 1.) * trat);
    double thetae = lcl_Thetae_u * uu / rho;
    if (p->cooling_dynamical_times > 1e-20) {
      int i = (int)(c / ((size_t)(N2 + 2) * (N3 + 2)));
      int j = (int)((c / (N3 + 2)) % (N2 + 2));
      int k = (int)(c % (N3 + 2));
      double X[NDIM], r, th;
      hc_ijktoX(g, i, j, k, X);
      hc_bl_coord(g, X, &r, &th);
      double Thetae_max_dynamical = 1 / p->cooling_dynamical_times * 7.71232e46 / 2 / m->MBH * pow(bb, -2) *
                                    pow(r * sin(th), -1.5);
      thetae = fmin(thetae, Thetae_max_dynamical);
    }
    thetae = fmax(thetae, 1.e-3);
    m->fields[IPG_F_NE][c] = ne;
    m->fields[IPG_F_B][c] = bb;
    m->fields[IPG_F_THETAE][c] = thetae;
    m->fields[IPG_F_SIGMA][c] = fmax(sigma_m, IPG_SMALL);
  }
  /* rho, u and beta for the trace output (fmax(beta, SMALL), model/iharm/model.c:700) */
  m->trace_fields[0] = f.p[KRHO];
  m->trace_fields[1] = f.p[UU];
  f.p[KRHO] = f.p[UU] = NULL;
  m->trace_fields[2] = (double *)malloc(ncell * sizeof(double));
  for (size_t c = 0; c < ncell; c++) {
    double bsq = f.b[c] * rf / m->B_unit;
    bsq = bsq * bsq;
    m->trace_fields[2][c] = fmax(m->trace_fields[1][c] * (gam - 1.) / 0.5 / bsq, IPG_SMALL);
  }
  for (int l = 0; l < NPRIM_STORE; l++) free(f.p[l]);
  free(f.b);

  g->Rh = 1 + sqrt(1. - g->a * g->a);
  g->th_beg = (p->polar_cut >= 0) ? 0.0174 * p->polar_cut : 0.0174;
  return IPG_OK;
}
