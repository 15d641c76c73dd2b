/*
 * ipole_b200.h -- C-ABI of the B200 (sm_100a) ray pipeline of ipole.
 *
 * The library replaces ipole's per-pixel OpenMP loop (src/main.c:536-615 and
 * :640-777, each iteration calling get_pixel, src/main.c:822-883) with GPU
 * kernels: backward geodesic integration in Kerr FMKS coordinates
 * (src/model_geodesics.c:38-171, src/geodesics.c:9-70), the iharm grid gather
 * (src/grid.c:15-44, model/iharm/model.c:420-593), the plasma tetrad
 * (src/model_tetrads.c:35-127), thermal synchrotron coefficients
 * (src/model_radiation.c:145-332, src/symphony/maxwell_juettner_fits.c) and
 * the polarized transfer step (src/ipolarray.c:59-628).
 *
 * Conventions: every call is synchronous unless it says otherwise, the
 * caller owns every host buffer, functions return IPG_OK or an IPG_E_* code
 * and never call exit().  Arrays are plain C arrays; no framework types cross
 * this boundary.  One context per host thread.
 */
#ifndef IPOLE_B200_H
#define IPOLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the CLI maps them to the reference's exit codes) ---- */
#define IPG_OK 0
#define IPG_E_ARG 1       /* invalid argument */
#define IPG_E_CUDA 2      /* CUDA runtime error or no device */
#define IPG_E_MAXNSTEP 3  /* a geodesic hit maxnstep (reference: exit(-10), src/main.c:841-845) */
#define IPG_E_NAN 4       /* NaN in the image (reference: exit(-1), src/main.c:905-908) */
#define IPG_E_TIMEOUT 5   /* a batch's step budget ran out (ipg_render_batch) */
#define IPG_E_NOMEM 6     /* device or trajectory-pool memory exhausted */
#define IPG_E_IO 7        /* file read/write error */
#define IPG_E_STATE 8     /* call order error (e.g. tracing before a model upload) */
#define IPG_E_FORMAT 9    /* unsupported dump content (metric, schema) */

/* ---- grid / coordinate description (coordinates.h:25-33, grid.h:6) ----
 * Native coordinates: FMKS ("funky" modified Kerr-Schild) for iharm dumps;
 * the known-answer models use MKS (hslope = 1) and eMinkowski. */
#define IPG_METRIC_FMKS 0        /* METRIC_FMKS (coordinates.h) */
#define IPG_METRIC_MKS 1         /* METRIC_MKS */
#define IPG_METRIC_MINKOWSKI 2   /* METRIC_MINKOWSKI: r = X1 */
#define IPG_METRIC_EMINKOWSKI 3  /* METRIC_EMINKOWSKI: r = exp(X1) */
typedef struct ipg_grid {
  int n1, n2, n3;                 /* physical zones (ghost zones excluded) */
  double startx[4], stopx[4], dx[4];
  double cstartx[4], cstopx[4];   /* coordinate-system limits (step control) */
  double a, hslope;               /* spin, MKS hslope */
  double poly_xt, poly_alpha, mks_smooth, poly_norm;
  double Rin, Rout, Rh;           /* Rh = 1 + sqrt(1 - a^2) */
  double rmin_geo, rmax_geo;      /* radiating region in r */
  double th_beg;                  /* radiating region cut around the poles */
  double sigma_cut;               /* emission cut: ne = 0 where sigma > sigma_cut */
  double sigma_cut_high;          /* model key sigma_cut_high (<= 0: off), only decides sigma == sigma_cut */
  double L_unit;                  /* GM/c^2 in cm */
  int metric;                     /* IPG_METRIC_*; 0 (FMKS) for iharm dumps */
} ipg_grid;

/* Field order of ipg_upload_iharm: primitives U1..3, B1..3 (native FMKS
 * components as in the dump), then the derived cgs fields of
 * init_physical_quantities (model/iharm/model.c:610-717). */
enum {
  IPG_F_U1 = 0, IPG_F_U2, IPG_F_U3, IPG_F_B1, IPG_F_B2, IPG_F_B3,
  IPG_F_NE, IPG_F_THETAE, IPG_F_B, IPG_F_SIGMA, IPG_NFIELD
};

/* ---- camera + run parameters of one image (main.c:125-168, par.h) ---- */
typedef struct ipg_camera {
  double Xcam[4];                 /* native_coord(rcam, thetacam, phicam) */
  double Econ[4][4], Ecov[4][4];  /* make_camera_tetrad(Xcam) (or the old centering) */
  double fovx, fovy;              /* camera FOV: DX / rcam, DY / rcam */
  double rotcam;                  /* radians */
  double xoff, yoff;              /* pixel offsets (par keys xoff, yoff) */
  double freq;                    /* freqcgs * HPL / (ME CL^2) */
  double freqcgs;
  double eps;                     /* geodesic accuracy (par key eps) */
  int nx, ny;                     /* params.nx, params.ny (image size, not the padded internal size) */
  int maxnstep;
  int only_unpolarized;           /* -unpol */
  int emission_type;              /* 4 (Dexter thermal, default) or 1 (Pandya thermal) */
  int stokes_floors;
  int target_nturns;              /* -1: off */
  int subring_dtheta;
  int counterjet;                 /* isolate_counterjet: 0, 1 or 2 */
} ipg_camera;

/* ---- per-ray result, the outputs of get_pixel (main.c:822-883) ---- */
typedef struct ipg_pixel_out {
  double I_unpol;     /* *Intensity  (invariant, before the nu^3 of save_pixel) */
  double tau;         /* *Tau */
  double tauF;        /* *tauF */
  double I, Q, U, V;  /* project_N outputs (before nu^3 and the qu_conv sign) */
  int32_t nstep;      /* geodesic steps */
  int32_t flag;       /* oddflag bits: 1 tetrad, 2 tauF, 4 NaN N, 8 NaN Ucov, 16 singular gcov */
} ipg_pixel_out;

typedef struct ipg_ctx ipg_ctx;

/* Create a context on CUDA device `device`.  The trajectory pool is sized
 * from free device memory unless pool_bytes > 0. */
int ipg_create(ipg_ctx **ctx, int device, size_t pool_bytes);
void ipg_destroy(ipg_ctx *ctx);
const char *ipg_strerror(int code);
/* Text of the last error recorded on the context (CUDA message, pixel id). */
const char *ipg_last_error(const ipg_ctx *ctx);

/* Upload one iharm FMKS model: grid constants plus IPG_NFIELD ghost-padded
 * fields, each (n1+2)*(n2+2)*(n3+2) doubles indexed [i][j][k], k fastest,
 * exactly the arrays model/iharm/model.c keeps in data[0] (p[U1..B3], ne,
 * thetae, b, sigma).  Replaces the model's static field storage as the source
 * of get_model_fourv / get_model_ne / get_model_thetae / get_model_b /
 * get_model_sigma point queries.  Returns IPG_E_ARG unless grid->metric is
 * IPG_METRIC_FMKS. */
int ipg_upload_iharm(ipg_ctx *ctx, const ipg_grid *grid, const double *const fields[IPG_NFIELD]);

/* ---- known-answer models (model/analytic/model.c, model/sphere/model.c) ----
 * The reference builds one binary per model (makefile:2, MODEL=...); here the
 * context is switched to a model by uploading it, and the ray kernels run
 * their instantiation for it.  The grid carries the model's geometry
 * (startx/stopx/cstartx/cstopx, a, Rh, rmin_geo, rmax_geo, L_unit) and its
 * metric: IPG_METRIC_MKS for the analytic models, IPG_METRIC_EMINKOWSKI for
 * the sphere. */
#define IPG_PLUGIN_IHARM 0
#define IPG_PLUGIN_ANALYTIC 1  /* Gold et al. 2020 GRRT problems, emission_type 10 */
#define IPG_PLUGIN_SPHERE 2    /* isothermal sphere, thermal emission_type 4 or 1 */
typedef struct ipg_plugin {
  int kind;                       /* IPG_PLUGIN_* */
  int model;                      /* analytic problem number 1..5 */
  /* analytic: init_model's problem constants and units (model/analytic/model.c:79-140) */
  double A, alpha, height, l0, freqcgs, rho_unit;
  /* sphere: derived density, temperature and field (model/sphere/model.c:53-85) */
  double R0, Ne0, Thetae0, B0;
  /* read by the trace output only: analytic B_unit; sphere get_model_sigma
   * and get_model_beta inside the sphere (model/sphere/model.c:161-185) */
  double B_unit, sigma0, beta0;
} ipg_plugin;
/* Upload a known-answer model; replaces any model of the context.  Returns
 * IPG_E_ARG for an unknown kind or a grid whose metric does not match it. */
int ipg_upload_plugin(ipg_ctx *ctx, const ipg_grid *grid, const ipg_plugin *plugin);

/* Trace n pixels (ij[2*m] = i, ij[2*m+1] = j) and return get_pixel's
 * outputs for each.  Host buffers; the call copies in, runs, copies out.
 * Returns IPG_E_MAXNSTEP if any ray hit maxnstep (its out[].nstep is
 * maxnstep-1); the other rays are still filled in. */
int ipg_trace_pixels(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *ij, size_t n, ipg_pixel_out *out);

/* Same, on device-resident buffers (d_ij: int32[2n], d_out: ipg_pixel_out[n]),
 * enqueued on `stream` (a cudaStream_t, 0 = legacy default) and
 * synchronised before return.  No host<->device copies. */
int ipg_trace_pixels_device(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *d_ij, size_t n,
                            ipg_pixel_out *d_out, void *stream);

/* Trace n pixels without allocating any device memory.  This entry point has
 * no counterpart in the reference.
 *
 * It is for callers that cannot call cudaMalloc: applications that give the
 * library a fixed share of device memory through their own allocator or pool
 * and treat any allocation made behind their back as a budget violation, and
 * latency-sensitive pipelines in which cudaMalloc/cudaFree, which can
 * synchronise the whole device, would stall their other streams.  Everything
 * the call needs beyond its inputs and outputs lives in one statically sized
 * scratch array per device (IPG_NOALLOC_SCRATCH_BYTES, 26.5 MiB) that every
 * process loading the library holds on each GPU it uses until it exits.
 *
 * Inputs and outputs, all on the current device: d_fields holds the model in
 * the library's layout, cell-major with the IPG_NFIELD fields of a zone
 * contiguous: d_fields[((i*(n2+2) + j)*(n3+2) + k)*IPG_NFIELD + f] for the
 * ghost-padded zone (i, j, k) and field f; d_ij is int32[2n], d_out is
 * ipg_pixel_out[n].  grid and cam are host structs as for the other calls.
 * Work is enqueued on `stream` (a cudaStream_t, 0 = legacy default stream),
 * which is synchronised before the call returns.
 *
 * Limits: n <= IPG_NOALLOC_MAX_RAYS and cam->maxnstep <= IPG_NOALLOC_MAX_STEPS,
 * otherwise IPG_E_ARG; grid->metric must be IPG_METRIC_FMKS (an iharm dump),
 * otherwise IPG_E_ARG.  The scratch holds IPG_NOALLOC_MAX_STEPS trajectory
 * steps at a time, so a batch runs in as many waves as it needs and is much
 * slower than ipg_trace_pixels_device.  Returns IPG_E_MAXNSTEP like
 * ipg_trace_pixels_device.
 *
 * The first call on a device sets the call up: it looks up the device address
 * of the scratch array, which may load the library's device code.  The
 * address is kept for the life of the process, so resetting the device
 * (cudaDeviceReset) between calls is not supported.  Every call synchronises
 * `stream` and copies a few status words back to the host before it returns,
 * so no call can be captured into a CUDA graph.  All calls share the
 * scratch array and the kernels' constant parameters, which keep what the last
 * call wrote: calls whose work overlaps on the GPU (from other streams or host
 * threads, or a context's ipg_trace_pixels* calls) race and give wrong
 * results, so serialise them.  Per ray, the results are the bits that
 * ipg_trace_pixels_device gives with FP64 step records. */
#define IPG_NOALLOC_MAX_RAYS 65536
#define IPG_NOALLOC_MAX_STEPS 51200
#define IPG_NOALLOC_SCRATCH_BYTES 27806720
int ipg_trace_pixels_noalloc(const ipg_grid *grid, const double *d_fields, const ipg_camera *cam,
                             const int32_t *d_ij, size_t n, ipg_pixel_out *d_out, void *stream);

/* ---- batches of image instances ----
 * No counterpart in the reference, which renders one image per run
 * (src/main.c:506-811).  A batch renders many images of one iharm dump in
 * one call: instances may differ in camera (inclination, frequency,
 * resolution, refinement keys) and electron model (M_unit, R_high, R_low,
 * beta_crit).  Instances whose cameras coincide share their geodesics, the
 * four-vectors and the plasma tetrads of every step; each instance's image
 * is the image ipg_render_image gives for the same parameters, bit for bit.
 *
 * The dump is uploaded once, as primitives: rho, u, U1..3, B1..3 with their
 * ghost zones filled (populate_boundary_conditions, model/iharm/model.c:
 * 1314-1370), and sqrt(b^2) in code units at the interior cells; gam, game,
 * gamp are the model's adiabatic indices.  The derived fields of each
 * electron model are computed on the device as init_physical_quantities
 * computes them (model/iharm/model.c:610-717, ELECTRONS == 2). */
enum {
  IPG_BP_RHO = 0, IPG_BP_UU, IPG_BP_U1, IPG_BP_U2, IPG_BP_U3, IPG_BP_B1, IPG_BP_B2, IPG_BP_B3, IPG_BP_BMAG,
  IPG_NBPRIM
};
int ipg_upload_iharm_batch(ipg_ctx *ctx, const ipg_grid *grid, const double *const prims[IPG_NBPRIM], double gam,
                           double game, double gamp);

/* electron model of an instance: set_units (model/iharm/model.c:595-608)
 * for its M_unit, and the R_high/R_low temperature ratio */
typedef struct ipg_electrons {
  double RHO_unit, B_unit;                /* M_unit / L_unit^3, CL sqrt(4 pi RHO_unit) */
  double trat_large, trat_small, beta_crit;
} ipg_electrons;

/* one image of a batch: its camera (as for ipg_trace_pixels), electron
 * model and the image driver's sizes and keys (src/main.c:102-123,
 * 520-792): internal size nx, ny (params.nx + 1 when refining an even size),
 * internal base size nx_min, ny_min, refinement levels (1: none), and
 * save_pixel's freqcgs^3 and qu_conv */
typedef struct ipg_instance {
  ipg_camera cam;
  ipg_electrons el;
  int nx, ny, nx_min, ny_min, refine_level;
  double f3;
  int qu_conv, nearest_neighbor;
  double refine_abs, refine_rel, refine_cut;
} ipg_instance;

/* caller-owned host arrays of one instance's image, internal size nx * ny,
 * as ipg_image holds them (imageS may be NULL for -unpol) */
typedef struct ipg_instance_image {
  double *image, *imageS, *taus;
  int32_t *interp_flag, *oddflag, *nstep;
  size_t traced; /* set by the call: pixels traced */
} ipg_instance_image;

/* Render n instances (needs ipg_upload_iharm_batch).  All instances share
 * emission_type (4 or 1) and -unpol; at most IPG_BATCH_MAX_CAMERAS distinct
 * cameras and IPG_BATCH_MAX_PER_CAMERA instances per camera.  The images
 * come back in out[0..n).  step_budget > 0 caps the geodesic plus transfer
 * steps of the whole call: once they are spent no further ray starts and
 * the call returns IPG_E_TIMEOUT.  Returns IPG_E_MAXNSTEP / IPG_E_NAN as
 * ipg_render_image does for any instance (ipg_last_error names it). */
#define IPG_BATCH_MAX_CAMERAS 64
#define IPG_BATCH_MAX_PER_CAMERA 32
int ipg_render_batch(ipg_ctx *ctx, const ipg_instance *inst, size_t n, ipg_instance_image *out,
                     uint64_t step_budget);

/* ---- adjoint of the polarized image ----
 * No counterpart in the reference, which only renders.  Given dL/d(I, Q,
 * U, V) of the n pixels ij (the get_pixel outputs of ipg_pixel_out, before
 * save_pixel's nu^3 and qu_conv sign), returns dL/dne, dL/dTheta_e and
 * dL/d|B| for every ghost-padded cell of the uploaded iharm fields (the
 * cell values the trilinear gather reads, layout of ipg_upload_iharm).  The
 * call traces the pixels again (the forward outputs come back in out, when
 * non-NULL), keeps N every ckpt_interval steps (16, 32 or 64) and walks each
 * ray back to front, recomputing the coherency tensor between checkpoints
 * and the fits with their derivatives at every radiating step.  Geodesics
 * do not depend on the fluid and are not differentiated; neither are the
 * sigma cut and the host's Theta_e floor (zero derivative almost
 * everywhere).  Needs a polarized image without Stokes floors (IPG_E_ARG
 * otherwise).  grad_* may be NULL. */
int ipg_adjoint(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *ij, size_t n, const double *dL_dIQUV,
                int ckpt_interval, double *grad_ne, double *grad_thetae, double *grad_b, ipg_pixel_out *out);

/* ---- per-step trace of one ray (dump_var_along, src/io.c:279-543) ----
 * Traces pixel (i, j) with the same kernels as the image and returns, for
 * steps s = 0..nstep, one row of IPG_TRACE_DOUBLES doubles: the quantities
 * the reference records along the ray, with its index conventions (rows 1
 * .. nstep-1 filled, e2Transported one row down, I_unpol the intensity of
 * the one step from s+1 to s).  steps holds max_steps rows (zero-filled by
 * the call); returns IPG_E_ARG when the ray has more than max_steps - 1
 * steps, IPG_E_MAXNSTEP when it hits maxnstep.  For an iharm model the
 * primitives rho, u and beta come from ipg_upload_trace_fields (zero until
 * it is called).  Columns: */
#define IPG_TRACE_B 0           /* get_model_b */
#define IPG_TRACE_NE 1          /* get_model_ne */
#define IPG_TRACE_THETAE 2      /* get_model_thetae */
#define IPG_TRACE_NU 3          /* get_fluid_nu */
#define IPG_TRACE_BK_ANGLE 4    /* get_bk_angle */
#define IPG_TRACE_SIGMA 5       /* get_model_sigma */
#define IPG_TRACE_BETA 6        /* get_model_beta */
#define IPG_TRACE_DL 7          /* traj[s].dl */
#define IPG_TRACE_R 8           /* bl_coord r, th; X[3] */
#define IPG_TRACE_TH 9
#define IPG_TRACE_PHI 10
#define IPG_TRACE_J_UNPOL 11    /* get_jkinv */
#define IPG_TRACE_K_UNPOL 12
#define IPG_TRACE_I_UNPOL 13
#define IPG_TRACE_X 14          /* [4] X, Kcon */
#define IPG_TRACE_KCON 18
#define IPG_TRACE_J_INV 22      /* [4] jar_calc jI..jV, aI..aV, (0, rQ, rU, rV) */
#define IPG_TRACE_ALPHA_INV 26
#define IPG_TRACE_RHO_INV 30
#define IPG_TRACE_STOKES 34     /* [4] I, Q, U, V of N in the plasma tetrad */
#define IPG_TRACE_E2C 38        /* [4] e2Constructed, e2ConstructedCov, e2Transported, e2TransportedCov */
#define IPG_TRACE_E2C_COV 42
#define IPG_TRACE_E2T 46
#define IPG_TRACE_E2T_COV 50
#define IPG_TRACE_PRIMS 54      /* [8] get_model_primitives */
#define IPG_TRACE_NTETRAD 62    /* [16] real parts of N_tetrad, N_coord; Econ, Ecov */
#define IPG_TRACE_NCOORD 78
#define IPG_TRACE_ECON 94
#define IPG_TRACE_ECOV 110
#define IPG_TRACE_FLAG 126      /* integrate_emission's flag of the step */
#define IPG_TRACE_DOUBLES 127
int ipg_trace_ray(ipg_ctx *ctx, const ipg_camera *cam, int i, int j, size_t max_steps, double *steps,
                  int32_t *nstep);
/* rho, u and beta per ghost-padded cell ([i][j][k], k fastest, as the
 * fields of ipg_upload_iharm) for the trace's primitives and beta */
int ipg_upload_trace_fields(ipg_ctx *ctx, const double *const extra[3]);

/* Kernel statistics of the last trace call: total ray-steps of the geodesic
 * pass, steps inside the radiating region, number of kernel launches and
 * pool waves, the device time (ms, CUDA events) of the geodesic, coefficient
 * and transfer kernels, summed over the batches of a wave (batches run
 * concurrently, so these can add up to more than the call), the time of the
 * ray-length prediction, and the device time of the whole call. */
typedef struct ipg_stats {
  uint64_t ray_steps;
  uint64_t radiating_steps;
  int32_t launches;
  int32_t waves;
  double geodesic_ms;
  double transfer_ms;
  double coeffs_ms;
  double predict_ms;
  double wall_ms;
  /* each kernel's wall time per wave: from the first length class's start
   * of that kernel to the last class's end (the *_ms above sum the classes'
   * concurrent launches) */
  double geodesic_span_ms;
  double coeffs_span_ms;
  double transfer_span_ms;
  /* ipg_adjoint: the reverse walk (link pass and adjoint kernel) and the
   * scatter of the cells' gradients; its forward pass is in geodesic_ms,
   * coeffs_ms and transfer_ms */
  double adjoint_ms;
  double adj_scatter_ms;
  /* ipg_render_batch: geodesic items of the longest predicted class traced
   * beside the waves (batches that take more than one wave) */
  uint64_t long_class_items;
  /* waves whose longest length class's blocks did not all report resident
   * within the host's bounded wait before the other classes were launched */
  uint64_t start_waits_timed_out;
} ipg_stats;
int ipg_get_stats(const ipg_ctx *ctx, ipg_stats *stats);

/* Storage precision of the step records between the three kernels (no
 * counterpart in the reference, whose integrate_emission holds one step in
 * registers).  IPG_RECORDS_FP64 (the default) keeps every value in FP64: the
 * plain tier.  IPG_RECORDS_MIXED stores the transport matrices and the plasma
 * tetrad rows (order-one values) in FP32 and the emission, absorption and
 * rotation coefficients in FP64; all arithmetic stays FP64, and the walk back
 * reads 320 bytes per step instead of 512.  Its images differ from the FP64
 * records' by the FP32 rounding of those values (the test of this mode states
 * the errors).  Batches (ipg_render_batch) store their shared records in the
 * same compact layout, the instances' coefficient blocks in FP64;
 * ipg_trace_ray, ipg_trace_pixels_noalloc and ipg_adjoint always use FP64.
 * Returns IPG_E_ARG for another value. */
#define IPG_RECORDS_FP64 0
#define IPG_RECORDS_MIXED 1
int ipg_set_record_precision(ipg_ctx *ctx, int precision);

/* Arithmetic of the polarized transfer step (no counterpart in the
 * reference).  IPG_STEP_FP64 (the default) is evolve_N of
 * src/ipolarray.c:332-575 in FP64.  IPG_STEP_FP32 evaluates its Faraday
 * rotation and absorption/emission in FP32, written in optical depths with
 * the Stokes vector and emission scaled by a power of two per step; the
 * projection of N and its update stay FP64.  The test of this mode states
 * its errors against the FP64 step.  Returns IPG_E_ARG for another value. */
#define IPG_STEP_FP64 0
#define IPG_STEP_FP32 1
int ipg_set_step_precision(ipg_ctx *ctx, int precision);

/* Arithmetic of the thermal synchrotron fits (no counterpart in the
 * reference).  IPG_FITS_FP64 (the default) evaluates get_jkinv and jar_calc
 * (src/model_radiation.c:145-332) in FP64.  IPG_FITS_FP32 evaluates the
 * shape of each fit (its transcendental functions and the Bessel functions
 * K_n(1/Theta_e), kept as mantissa and exponent) in FP32 and the
 * prefactors and exponents in FP64, so that no coefficient leaves FP32's
 * range; the coefficients keep FP64 storage.  Applies to ipg_render_* and
 * ipg_render_batch; ipg_trace_ray, ipg_trace_pixels_noalloc and ipg_adjoint
 * always use the FP64 fits.  The test of this mode states its errors.
 * Returns IPG_E_ARG for another value. */
#define IPG_FITS_FP64 0
#define IPG_FITS_FP32 1
int ipg_set_fit_precision(ipg_ctx *ctx, int precision);

/* The thermal fits at given plasma parameters (the fits of jar_calc,
 * src/model_radiation.c:182-332, for emission_type 4 or 1, without the
 * model lookup): in[5n] = (nu, Ne, Thetae, B, theta) per point, host memory;
 * out[12n] = (j_I/nu^2 and a_I of get_jkinv, then jI jQ jU jV aI aQ aU aV rQ
 * rV of jar_calc) per point, zeros where Ne <= 0.  precision is
 * IPG_FITS_FP64 or IPG_FITS_FP32 (the kernels' two forms). */
int ipg_thermal_coefficients(ipg_ctx *ctx, const double *in, size_t n, int emission_type, int precision,
                             double *out);

/* The context's CUDA stream (a cudaStream_t), on which every kernel of the
 * context is launched; lets a caller bracket calls with its own events. */
int ipg_get_stream(const ipg_ctx *ctx, void **stream);

/* ---- host-side helpers mirroring the reference's setup code ---- */

/* Camera setup of main.c:125-168 and init_XK's tetrad (model_geodesics.c:
 * 178-190): native_coord/root_find (coordinates.c:375-442), FOV from
 * fov (muas) or dx/dy, make_camera_tetrad (model_tetrads.c:143-193) or the
 * old centering.  Fills cam->Xcam/Econ/Ecov/fovx/fovy/freq/freqcgs and
 * returns the intensity-to-Jy `scale` and DX, DY (GM/c^2) through pointers. */
int ipg_camera_setup(const ipg_grid *grid, double rcam, double thetacam_deg, double phicam_deg,
                     double rotcam_deg, double fovx_muas, double fovy_muas, double dx_rg, double dy_rg,
                     double dsource_pc, int nx, int ny, double freqcgs, int old_centering,
                     ipg_camera *cam, double *scale, double *DX, double *DY);

/* Peak FP64 FMA throughput of the device in TFLOP/s (2 flops per FMA),
 * measured with a register-resident FMA loop for `ms` milliseconds. */
int ipg_measure_fp64_peak(int device, double ms, double *tflops);
/* The same probe with FP32 FMA chains: the FP32 CUDA-core peak. */
int ipg_measure_fp32_peak(int device, double ms, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* IPOLE_B200_H */
