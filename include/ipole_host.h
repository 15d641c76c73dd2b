/*
 * ipole_host.h -- host-side C API that mirrors the reference program around
 * the ray pipeline: parameters (src/par.h, src/par.c), the iharm fluid model
 * set-up (model/iharm/model.c), the fast-light image driver with adaptive
 * refinement (src/main.c:506-811) and the image writer (src/io.c:140-273).
 *
 * All functions are plain C, return IPG_OK / IPG_E_* and never exit().
 */
#ifndef IPOLE_HOST_H
#define IPOLE_HOST_H

#include "ipole_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define IPG_STRLEN 2048

/* Params (src/par.h:14-73) plus the iharm model keys
 * (model/iharm/model.c:130-167) and the radiation keys
 * (src/model_radiation.c:77-96). */
typedef struct ipg_params {
  double rcam, thetacam, phicam, rotcam;
  double dx, dy;
  double fovx_dsource, fovy_dsource;
  int nx, ny;
  double dsource;
  double freqcgs;
  int old_centering;
  double eps;
  int maxnstep;
  int add_ppm, qu_conv, quench_output, only_unpolarized, perform_check;
  int emission_type, stokes_floors, isolate_counterjet;
  char dump[IPG_STRLEN];
  char outf[IPG_STRLEN];
  int target_nturns, subring_dtheta;
  int nx_min, ny_min;
  double refine_abs, refine_rel, refine_cut;
  int nearest_neighbor;
  double xoff, yoff;
  double img_cadence, restart_int;
  int trace, trace_stride, trace_i, trace_j;
  char trace_outf[IPG_STRLEN];
  int histo, histo_polar;
  char histo_outf[IPG_STRLEN];
  /* iharm model keys */
  double MBH_solar, M_unit, target_mdot;
  double tp_over_te, trat_small, trat_large, sigma_cut, sigma_cut_high, beta_crit;
  double cooling_dynamical_times;
  double rmax_geo, rmin_geo;
  int reverse_field;
  double polar_cut;
  int dump_min, dump_max, dump_skip;
  /* radiation keys (thermal path ignores the non-thermal ones) */
  double model_kappa, powerlaw_gamma_cut, powerlaw_gamma_min, powerlaw_gamma_max, powerlaw_p, powerlaw_eta;
  int variable_kappa;
  double variable_kappa_min, variable_kappa_interp_start, variable_kappa_max;
  int bremss, bremss_type;
  /* Model selection (the reference selects at build time, makefile:2
   * MODEL=...): key "plugin" = iharm (default), analytic or sphere. */
  char plugin[IPG_STRLEN];
  int MBH_set;              /* 1 once the "MBH" key was given (each model has its own default) */
  /* analytic keys (model/analytic/model.c:56-72) */
  int analytic_model;       /* "model": problem 1..5 of Gold et al. 2020 */
  double rho_unit;          /* "rho_unit" (<= 0: 3e-18) */
  /* sphere keys (model/sphere/model.c:37-46); tp_over_te is shared with iharm */
  double sphere_Thetae0, sphere_R0, sphere_tau0, sphere_beta0, sphere_gam;
  /* "mixed_records" (no reference counterpart): 1 stores the step records
   * compactly between the kernels (ipg_set_record_precision,
   * IPG_RECORDS_MIXED); 0, the default, keeps them in FP64 */
  int mixed_records;
  /* "fp32_step" (no reference counterpart): 1 evaluates the polarized step
   * in FP32 (ipg_set_step_precision, IPG_STEP_FP32); 0, the default, FP64 */
  int fp32_step;
  /* "fp32_fits" (no reference counterpart): 1 evaluates the thermal fits
   * with FP32 shapes (ipg_set_fit_precision, IPG_FITS_FP32); 0, the default,
   * FP64 */
  int fp32_fits;
} ipg_params;

/* Defaults of load_par_from_argv (src/par.c:48-100) and the model/radiation
 * statics. */
void ipg_params_default(ipg_params *p);
/* try_set_parameter chain (src/par.c:139-210): sets any matching key; unknown
 * keys are ignored, as in the reference. */
void ipg_params_set(ipg_params *p, const char *word, const char *value);
/* load_par (src/par.c:213-232): returns IPG_E_IO if the file cannot be opened. */
int ipg_params_load_file(ipg_params *p, const char *fname);
/* load_par_from_argv (src/par.c:43-136): -par, --k=v, --k v, bare --flag,
 * -unpol, -quench, -check.  Returns IPG_E_ARG for histogram requests (the
 * reference exits 42) or a missing -par file name. */
int ipg_params_from_argv(ipg_params *p, int argc, char **argv);

/* The iharm model after init_model (model/iharm/model.c:295-389). */
typedef struct ipg_iharm_model {
  ipg_grid grid;
  double *fields[IPG_NFIELD];  /* ghost-padded, [i][j][k], k fastest */
  double M_unit, L_unit, T_unit, RHO_unit, U_unit, B_unit, Te_unit, MBH;
  double Mdot_dump, MdotEdd_dump, Ladv_dump, t, DTd;
  int electrons;
  double gam, game, gamp;
  void *fluid_header;          /* copy of the dump's /header group (for /fluid_header) */
  ipg_plugin plugin;           /* kind IPG_PLUGIN_IHARM, or a known-answer model (no fields) */
  double *trace_fields[3];     /* rho, u, beta per ghost-padded cell (trace output; NULL for plugins) */
  double *bmag_code;           /* sqrt(b^2) per cell in code units, interior cells (batched instances; NULL for plugins) */
} ipg_iharm_model;

/* init_model: read the dump named in p->dump (an iharm v1 HDF5 dump, or the
 * same schema in an IPGC container), build ghost zones and derived fields.  Returns
 * IPG_E_IO / IPG_E_FORMAT on a bad dump (reference: exit(-1) / exit(-3)).
 * With p->plugin "analytic" or "sphere", the known-answer model's init_model
 * instead (model/analytic/model.c:79-160, model/sphere/model.c:53-110):
 * geometry, units and model constants, no dump.  Returns IPG_E_ARG for an
 * unknown plugin name. */
int ipg_iharm_load(const ipg_params *p, ipg_iharm_model *m);
void ipg_iharm_free(ipg_iharm_model *m);
/* Upload the loaded model to a context: ipg_upload_iharm for a dump,
 * ipg_upload_plugin for a known-answer model. */
int ipg_upload_model(ipg_ctx *ctx, const ipg_iharm_model *m);

/* A rendered image, internal size nx x ny (params.nx + 1 when refining an
 * even size, main.c:107-123), arrays as in main.c:184-197. */
typedef struct ipg_image {
  size_t nx, ny;           /* internal (memory) size */
  double *image;           /* [nx*ny] unpolarized I nu^3 */
  double *imageS;          /* [nx*ny*5] I, Q, U, V (nu^3, qu_conv sign), tauF; NULL if unpolarized */
  double *taus;            /* [nx*ny] */
  int *interp_flag;        /* [nx*ny] 1 where refinement interpolated */
  double scale;            /* intensity -> Jy per pixel */
  double Xcam[4];
  double fovx, fovy;
  ipg_camera cam;
  int32_t *oddflag;        /* [nx*ny] oddflag of traced pixels */
  int32_t *nstep;          /* [nx*ny] steps of traced pixels, 0 if interpolated */
  size_t traced;           /* pixels traced */
} ipg_image;

/* Fast-light image of main.c:506-792: base image at nx_min, then the
 * refinement levels, each level traced with one ipg_trace_pixels call.
 * Progress lines go to `log` (stderr in the CLI) when non-NULL. */
int ipg_render_image(ipg_ctx *ctx, ipg_params *p, const ipg_iharm_model *m, ipg_image *img, void *log);

/* The same driver with the per-level tracing supplied by the caller: the
 * tracer fills out[0..n) for the pixel list ij (get_pixel semantics) and
 * returns IPG_OK or an IPG_E_* code.  ipg_render_image passes
 * ipg_trace_pixels on its context. */
typedef int (*ipg_tracer_fn)(void *user, const ipg_camera *cam, const int32_t *ij, size_t n, ipg_pixel_out *out);
int ipg_render_image_with(ipg_tracer_fn tracer, void *user, ipg_params *p, const ipg_iharm_model *m, ipg_image *img,
                          void *log);
void ipg_image_free(ipg_image *img);

/* ---- batches of images (no counterpart in the reference, which renders
 * one image per run) ----
 * Upload the loaded dump's primitives for batches (ipg_upload_iharm_batch:
 * rho and u with their ghost zones, the velocity and field primitives, and
 * sqrt(b^2) in code units). */
int ipg_upload_model_batch(ipg_ctx *ctx, const ipg_iharm_model *m);
/* Render n images of the batch-uploaded dump in one ipg_render_batch call,
 * image i with the parameters *ps[i] (modified as ipg_render_image modifies
 * its parameters).  Each image equals the one ipg_render_image renders from
 * the same dump loaded with ps[i]'s M_unit and electron keys, bit for bit.
 * Instances share emission_type and -unpol; check mode, target_mdot,
 * cooling_dynamical_times and a black-hole mass other than the model's
 * return IPG_E_ARG.  imgs[0..n) are filled (free each with ipg_image_free,
 * also after an error).  step_budget as for ipg_render_batch. */
int ipg_render_batch_params(ipg_ctx *ctx, ipg_params *const *ps, size_t n, const ipg_iharm_model *m,
                            ipg_image *imgs, uint64_t step_budget, void *log);

/* ---- adjoint of an image (no counterpart in the reference) ----
 * Gradients of a loss L of the polarized image rendered with *p (no
 * refinement: every pixel is traced) from dL/dpol, the derivative with
 * respect to the image's pol[nx][ny][0..3] (I, Q, U, V as the image file
 * holds them).  Per cell: dL/dne, dL/dTheta_e, dL/d|B| of the model's fields
 * (ipg_adjoint; dL/drho with Theta_e held is dL/dne RHO_unit / (MP + ME));
 * and, through init_physical_quantities (model/iharm/model.c:610-717), the
 * derivatives with respect to M_unit, R_high (trat_large) and R_low
 * (trat_small).  The model must be loaded with p's electron keys.  pol_out
 * (nx*ny*4, may be NULL) receives the image the adjoint traced. */
typedef struct ipg_grad {
  double *d_ne, *d_thetae, *d_b; /* per ghost-padded cell (caller-owned, may be NULL) */
  double d_M_unit, d_R_high, d_R_low;
} ipg_grad;
int ipg_adjoint_params(ipg_ctx *ctx, ipg_params *p, const ipg_iharm_model *m, const double *dL_dpol,
                       int ckpt_interval, ipg_grad *g, double *pol_out);

/* print_image_stats (src/main.c:1001-1042) to `log` (a FILE*), same lines;
 * the "Ftot" line format is kept verbatim for scripts that scrape it. */
void ipg_print_image_stats(const ipg_image *img, const ipg_params *p, void *log);
/* Totals of print_image_stats: Ftot, Ftot_unpol, Qtot, Utot, Vtot (Jy). */
void ipg_image_totals(const ipg_image *img, const ipg_params *p, double tot[5]);

/* dump() (src/io.c:229-273) with write_header (:140-191) and the iharm
 * output_hdf5 (model/iharm/model.c:1254-1301): an HDF5 file with the
 * reference's datasets and attributes, or an IPGC container when fname ends
 * in ".ipgc". */
int ipg_write_image(const char *fname, const ipg_image *img, const ipg_params *p, const ipg_iharm_model *m);

/* Check mode (-check, src/main.c:538-575): ipg_render_image traces every
 * IPG_CHECK_SKIP-th pixel (i, j) and its mirror (nx - i - offset, j) and
 * saves them at reduced indices; ipg_write_check then appends them to an
 * existing image file as unpol/tau/pol _check and _recheck (dump_check,
 * src/io.c:193-227).  Check mode needs nx_min = nx. */
#define IPG_CHECK_SKIP 10
int ipg_write_check(const char *fname, const ipg_image *img, const ipg_params *p);

/* Trace output (dump_var_along, src/io.c:279-543, for the pixels that
 * src/main.c:865-879 selects): with p->trace set, every traced pixel (i, j)
 * of the image with i and j multiples of trace_stride, or only (trace_i,
 * trace_j) when both are >= 0, is traced again step by step
 * (ipg_trace_ray) and written to p->trace_outf: the image header, "nstep"
 * [nx'][ny'] and the per-step datasets [nx'][ny'][L](4)(4) of the
 * reference (nx' = nx / trace_stride, or 1).  The step axis L is the longest
 * traced ray's nstep + 1, where the reference's chunked datasets run to
 * maxnstep (their entries past a ray's end are zero, as here).  An existing
 * file keeps the pixels it holds.  "Flagged integration when tracing" lines
 * go to stdout as in the reference. */
int ipg_write_traces(ipg_ctx *ctx, const ipg_image *img, const ipg_params *p, const ipg_iharm_model *m);

/* Copy a dump or image between the two file formats the library reads: HDF5
 * (the reference's format, src/hdf5_utils.c over libhdf5; this library reads
 * and writes the subset those files use without libhdf5) and the flat IPGC
 * container.  The source format is detected from its signature; the
 * destination is IPGC when its name ends in ".ipgc", HDF5 otherwise.  Returns
 * IPG_E_IO on a missing or malformed file and IPG_E_FORMAT on HDF5 features
 * outside the subset (dense groups, chunk indexes other than the version 1
 * B-tree, filters other than deflate and shuffle). */
int ipg_container_convert(const char *src, const char *dst);

/* ---- the reference's model plugin interface (src/model.h:9-44) ----
 * The same names and signatures, over one library-global iharm model:
 * try_set_model_parameter collects par keys (ipg_params_set on the
 * interface's own parameters, ipg_model_params), init_model loads the dump
 * they name (ipg_iharm_load) and sets the unit globals, the point queries
 * read the loaded fields on the host.  Where the reference exits, init_model
 * leaves no model loaded and ipg_model_status() returns the IPG_E_* code.
 * update_data and update_data_until do nothing (one dump, fast light).  The
 * image file's model header (the reference's output_hdf5) is written by
 * ipg_write_image. */
extern double M_unit, L_unit, T_unit, RHO_unit, U_unit, B_unit, Te_unit;
void try_set_model_parameter(const char *word, const char *value);
void init_model(double *tA, double *tB);
int radiating_region(double X[4]);
double get_model_thetae(double X[4]);
double get_model_b(double X[4]);
double get_model_sigma(double X[4]);
double get_model_beta(double X[4]);
double get_model_ne(double X[4]);
void get_model_jar(double X[4], double Kcon[4], double *jI, double *jQ, double *jU, double *jV, double *aI,
                   double *aQ, double *aU, double *aV, double *rQ, double *rU, double *rV);
void get_model_fourv(double X[4], double Kcon[4], double Ucon[4], double Ucov[4], double Bcon[4], double Bcov[4]);
void update_data(double *tA, double *tB);
void update_data_until(double *tA, double *tB, double tgt);
void get_model_primitives(double X[4], double *p);
/* the interface's parameters, its loaded model (NULL before init_model) and
 * the status of the last init_model */
ipg_params *ipg_model_params(void);
const ipg_iharm_model *ipg_model_loaded(void);
int ipg_model_status(void);

#ifdef __cplusplus
}
#endif
#endif /* IPOLE_HOST_H */
