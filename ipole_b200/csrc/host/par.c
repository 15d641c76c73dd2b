/* Parameters: defaults, par-file and command-line parsing with the reference
 * semantics (src/par.c:43-253, model/iharm/model.c:130-167,
 * src/model_radiation.c:77-96). */
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ipole_host.h"

#define TYPE_INT 1
#define TYPE_DBL 2
#define TYPE_STR 3

#define DM87_PC (16.9e6)

/* src/par.c:235-253 */
static void set_by_word_val(const char *word, const char *value, const char *key, void *val, int type)
{
  if (strcmp(word, key) != 0) return;
  switch (type) {
    case TYPE_INT: sscanf(value, "%d", (int *)val); break;
    case TYPE_DBL: sscanf(value, "%lf", (double *)val); break;
    case TYPE_STR: sscanf(value, "%2047s", (char *)val); break;
  }
}

void ipg_params_default(ipg_params *p)
{
  memset(p, 0, sizeof(*p));
  p->add_ppm = 0;
  p->qu_conv = 0;
  p->quench_output = 0;
  p->only_unpolarized = 0;
  p->perform_check = 0;
  p->old_centering = 0;
  p->emission_type = 4;
  strcpy(p->plugin, "iharm");
  p->sphere_R0 = 100.;
  p->sphere_tau0 = 1.e-5;
  p->sphere_Thetae0 = 10.;
  p->sphere_beta0 = 20.;
  p->sphere_gam = 13. / 9;
  p->stokes_floors = 0;
  p->isolate_counterjet = 0;
  p->rcam = 1000.;
  p->thetacam = 90.;
  p->phicam = 0.;
  p->rotcam = 0.;
  p->nx = 160;
  p->ny = 160;
  p->eps = 0.01;
  p->maxnstep = 50000;
  p->dsource = DM87_PC;
  p->restart_int = -1.;
  p->target_nturns = -1;
  p->subring_dtheta = 0;
  p->nx_min = -1;
  p->ny_min = -1;
  p->refine_rel = 1.e-1;
  p->refine_abs = 1.e-5;
  p->refine_cut = 0.0;
  p->nearest_neighbor = 0;
  p->xoff = 0.0;
  p->yoff = 0.0;
  p->trace = 0;
  p->trace_stride = 1;
  p->trace_i = -1;
  p->trace_j = -1;
  strcpy(p->trace_outf, "trace.h5");
  p->histo = 0;
  p->histo_polar = 0;
  strcpy(p->histo_outf, "histo.h5");
  /* iharm statics, model/iharm/model.c:33-95 */
  p->MBH_solar = 6.2e9;
  p->M_unit = 0.;
  p->target_mdot = 0.0;
  strcpy(p->dump, "dump.h5");
  p->tp_over_te = 3.;
  p->trat_small = 1.;
  p->trat_large = 40.;
  p->sigma_cut = 1.;
  p->sigma_cut_high = -1.0;
  p->beta_crit = 1.0;
  p->cooling_dynamical_times = 1.e-20;
  p->rmax_geo = 100.;
  p->rmin_geo = 1.;
  p->reverse_field = 0;
  p->polar_cut = -1;
  p->dump_min = 0;
  p->dump_max = 0;
  p->dump_skip = 1;
  /* radiation statics, src/model_radiation.c:62-75 */
  p->model_kappa = 3.5;
  p->powerlaw_gamma_cut = 1e10;
  p->powerlaw_gamma_min = 1e2;
  p->powerlaw_gamma_max = 1e5;
  p->powerlaw_p = 3.25;
  p->powerlaw_eta = 0.02;
  p->variable_kappa = 0;
  p->variable_kappa_min = 3.1;
  p->variable_kappa_interp_start = 1e20;
  p->variable_kappa_max = 7.0;
  p->bremss = 0;
  p->bremss_type = 2;
}

/* model/iharm/model.c:130-167 */
static void set_model_parameter(ipg_params *p, const char *word, const char *value)
{
  set_by_word_val(word, value, "MBH", &p->MBH_solar, TYPE_DBL);
  if (strcmp(word, "MBH") == 0) p->MBH_set = 1;
  /* model selection and the known-answer models' keys */
  set_by_word_val(word, value, "plugin", p->plugin, TYPE_STR);
  set_by_word_val(word, value, "model", &p->analytic_model, TYPE_INT);
  set_by_word_val(word, value, "rho_unit", &p->rho_unit, TYPE_DBL);
  set_by_word_val(word, value, "Thetae0", &p->sphere_Thetae0, TYPE_DBL);
  set_by_word_val(word, value, "R0", &p->sphere_R0, TYPE_DBL);
  set_by_word_val(word, value, "tau0", &p->sphere_tau0, TYPE_DBL);
  set_by_word_val(word, value, "beta0", &p->sphere_beta0, TYPE_DBL);
  set_by_word_val(word, value, "gam", &p->sphere_gam, TYPE_DBL);
  set_by_word_val(word, value, "M_unit", &p->M_unit, TYPE_DBL);
  set_by_word_val(word, value, "mdot", &p->target_mdot, TYPE_DBL);
  set_by_word_val(word, value, "dump", p->dump, TYPE_STR);
  set_by_word_val(word, value, "tp_over_te", &p->tp_over_te, TYPE_DBL);
  set_by_word_val(word, value, "trat_small", &p->trat_small, TYPE_DBL);
  set_by_word_val(word, value, "trat_large", &p->trat_large, TYPE_DBL);
  set_by_word_val(word, value, "sigma_cut", &p->sigma_cut, TYPE_DBL);
  set_by_word_val(word, value, "sigma_cut_high", &p->sigma_cut_high, TYPE_DBL);
  set_by_word_val(word, value, "beta_crit", &p->beta_crit, TYPE_DBL);
  set_by_word_val(word, value, "cooling_dynamical_times", &p->cooling_dynamical_times, TYPE_DBL);
  set_by_word_val(word, value, "rmax_geo", &p->rmax_geo, TYPE_DBL);
  set_by_word_val(word, value, "rmin_geo", &p->rmin_geo, TYPE_DBL);
  set_by_word_val(word, value, "reverse_field", &p->reverse_field, TYPE_INT);
  set_by_word_val(word, value, "polar_cut_deg", &p->polar_cut, TYPE_DBL);
  set_by_word_val(word, value, "dump_min", &p->dump_min, TYPE_INT);
  set_by_word_val(word, value, "dump_max", &p->dump_max, TYPE_INT);
  set_by_word_val(word, value, "dump_skip", &p->dump_skip, TYPE_INT);
  if (p->target_mdot > 0.) p->M_unit = 1.;
}

/* src/model_radiation.c:77-96, including its quirk that max_pol_frac_e/a
 * write into powerlaw_p (model_radiation.c:94-95) */
static void set_radiation_parameter(ipg_params *p, const char *word, const char *value)
{
  set_by_word_val(word, value, "kappa", &p->model_kappa, TYPE_DBL);
  set_by_word_val(word, value, "variable_kappa", &p->variable_kappa, TYPE_INT);
  set_by_word_val(word, value, "variable_kappa_min", &p->variable_kappa_min, TYPE_DBL);
  set_by_word_val(word, value, "variable_kappa_interp_start", &p->variable_kappa_interp_start, TYPE_DBL);
  set_by_word_val(word, value, "variable_kappa_max", &p->variable_kappa_max, TYPE_DBL);
  set_by_word_val(word, value, "powerlaw_gamma_cut", &p->powerlaw_gamma_cut, TYPE_DBL);
  set_by_word_val(word, value, "powerlaw_gamma_min", &p->powerlaw_gamma_min, TYPE_DBL);
  set_by_word_val(word, value, "powerlaw_gamma_max", &p->powerlaw_gamma_max, TYPE_DBL);
  set_by_word_val(word, value, "powerlaw_p", &p->powerlaw_p, TYPE_DBL);
  set_by_word_val(word, value, "powerlaw_eta", &p->powerlaw_eta, TYPE_DBL);
  set_by_word_val(word, value, "bremss", &p->bremss, TYPE_INT);
  set_by_word_val(word, value, "bremss_type", &p->bremss_type, TYPE_INT);
  set_by_word_val(word, value, "max_pol_frac_e", &p->powerlaw_p, TYPE_DBL);
  set_by_word_val(word, value, "max_pol_frac_a", &p->powerlaw_p, TYPE_DBL);
}

/* src/par.c:139-210 */
void ipg_params_set(ipg_params *p, const char *word, const char *value)
{
  set_by_word_val(word, value, "freqcgs", &p->freqcgs, TYPE_DBL);
  set_by_word_val(word, value, "add_ppm", &p->add_ppm, TYPE_INT);
  set_by_word_val(word, value, "qu_conv", &p->qu_conv, TYPE_INT);
  set_by_word_val(word, value, "quench_output", &p->quench_output, TYPE_INT);
  set_by_word_val(word, value, "only_unpolarized", &p->only_unpolarized, TYPE_INT);
  set_by_word_val(word, value, "emission_type", &p->emission_type, TYPE_INT);
  set_by_word_val(word, value, "stokes_floors", &p->stokes_floors, TYPE_INT);
  set_by_word_val(word, value, "counterjet", &p->isolate_counterjet, TYPE_INT);
  set_by_word_val(word, value, "old_centering", &p->old_centering, TYPE_INT);
  set_by_word_val(word, value, "rcam", &p->rcam, TYPE_DBL);
  set_by_word_val(word, value, "thetacam", &p->thetacam, TYPE_DBL);
  set_by_word_val(word, value, "phicam", &p->phicam, TYPE_DBL);
  set_by_word_val(word, value, "rotcam", &p->rotcam, TYPE_DBL);
  set_by_word_val(word, value, "dsource", &p->dsource, TYPE_DBL);
  set_by_word_val(word, value, "fovx", &p->fovx_dsource, TYPE_DBL);
  set_by_word_val(word, value, "fovy", &p->fovy_dsource, TYPE_DBL);
  set_by_word_val(word, value, "fovx_dsource", &p->fovx_dsource, TYPE_DBL);
  set_by_word_val(word, value, "fovy_dsource", &p->fovy_dsource, TYPE_DBL);
  set_by_word_val(word, value, "fov", &p->fovx_dsource, TYPE_DBL);
  set_by_word_val(word, value, "fov", &p->fovy_dsource, TYPE_DBL);
  set_by_word_val(word, value, "dx", &p->dx, TYPE_DBL);
  set_by_word_val(word, value, "dy", &p->dy, TYPE_DBL);
  set_by_word_val(word, value, "nx", &p->nx, TYPE_INT);
  set_by_word_val(word, value, "ny", &p->ny, TYPE_INT);
  set_by_word_val(word, value, "nx_min", &p->nx_min, TYPE_INT);
  set_by_word_val(word, value, "ny_min", &p->ny_min, TYPE_INT);
  set_by_word_val(word, value, "refine_abs", &p->refine_abs, TYPE_DBL);
  set_by_word_val(word, value, "refine_rel", &p->refine_rel, TYPE_DBL);
  set_by_word_val(word, value, "refine_cut", &p->refine_cut, TYPE_DBL);
  set_by_word_val(word, value, "use_nearest_neighbor", &p->nearest_neighbor, TYPE_INT);
  set_by_word_val(word, value, "target_nturns", &p->target_nturns, TYPE_INT);
  set_by_word_val(word, value, "subring_dtheta", &p->subring_dtheta, TYPE_INT);
  set_by_word_val(word, value, "eps", &p->eps, TYPE_DBL);
  set_by_word_val(word, value, "maxnstep", &p->maxnstep, TYPE_INT);
  set_by_word_val(word, value, "xoff", &p->xoff, TYPE_DBL);
  set_by_word_val(word, value, "yoff", &p->yoff, TYPE_DBL);
  set_by_word_val(word, value, "outfile", p->outf, TYPE_STR);
  set_by_word_val(word, value, "img_cadence", &p->img_cadence, TYPE_DBL);
  set_by_word_val(word, value, "restart_int", &p->restart_int, TYPE_DBL);
  set_by_word_val(word, value, "trace", &p->trace, TYPE_INT);
  set_by_word_val(word, value, "trace_stride", &p->trace_stride, TYPE_INT);
  set_by_word_val(word, value, "trace_i", &p->trace_i, TYPE_INT);
  set_by_word_val(word, value, "trace_j", &p->trace_j, TYPE_INT);
  set_by_word_val(word, value, "trace_outf", p->trace_outf, TYPE_STR);
  set_by_word_val(word, value, "mixed_records", &p->mixed_records, TYPE_INT);
  set_by_word_val(word, value, "fp32_step", &p->fp32_step, TYPE_INT);
  set_by_word_val(word, value, "fp32_fits", &p->fp32_fits, TYPE_INT);
  set_by_word_val(word, value, "histo", &p->histo, TYPE_INT);
  set_by_word_val(word, value, "histo_polar", &p->histo_polar, TYPE_INT);
  set_by_word_val(word, value, "histo_outf", p->histo_outf, TYPE_STR);
  set_model_parameter(p, word, value);
  set_radiation_parameter(p, word, value);
}

/* src/par.c:213-232 */
int ipg_params_load_file(ipg_params *p, const char *fname)
{
  char line[256] = {0}, word[256] = {0}, value[256] = {0};
  FILE *fp = fopen(fname, "r");
  if (fp == NULL) {
    fprintf(stderr, "! unable to load parameter file '%s'. (%d: %s)\n", fname, errno, strerror(errno));
    return IPG_E_IO;
  }
  while (fgets(line, 255, fp) != NULL) {
    if (line[0] == '#') continue;
    sscanf(line, "%255s %255s", word, value);
    ipg_params_set(p, word, value);
  }
  fclose(fp);
  return IPG_OK;
}

/* src/par.c:43-136 */
int ipg_params_from_argv(ipg_params *p, int argc, char **argv)
{
  ipg_params_default(p);
  for (int i = 0; i < argc; ++i) {
    if (strcmp(argv[i], "-quench") == 0) p->quench_output = 1;
    else if (strcmp(argv[i], "-unpol") == 0) p->only_unpolarized = 1;
    else if (strcmp(argv[i], "-check") == 0) p->perform_check = 1;

    if (strlen(argv[i]) > 2 && argv[i][0] == '-' && argv[i][1] == '-') {
      char buf[IPG_STRLEN];
      snprintf(buf, sizeof(buf), "%s", argv[i] + 2);
      char *saveptr = NULL;
      char *word = strtok_r(buf, "=", &saveptr);
      char *value = strtok_r(NULL, "=", &saveptr);
      if (word == NULL) continue;
      if (value != NULL) ipg_params_set(p, word, value);
      else if (i == argc - 1 || (argv[i + 1][0] == '-' && argv[i + 1][1] == '-')) ipg_params_set(p, word, "1");
      else ipg_params_set(p, word, argv[i + 1]);
    }

    if (strcmp(argv[i], "-par") == 0) {
      if (i == argc - 1) {
        fprintf(stderr, "! parameter filename must follow -par argument\n");
        return IPG_E_ARG;
      }
      int rc = ipg_params_load_file(p, argv[i + 1]);
      if (rc != IPG_OK) return rc;
    }
  }
  if (p->histo != 0 || p->histo_polar != 0) {
    fprintf(stderr,
            "histogramming emission is nuanced. please either use the trace feature or uncomment this exit() at your "
            "own risk.\n");
    return IPG_E_ARG;
  }
  return IPG_OK;
}
