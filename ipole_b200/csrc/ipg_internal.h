/* Internal interface between the library's translation units (not installed,
 * not part of the C-ABI).
 *
 * ipg_kernels.cu owns the context and the ray kernels; ipg_refine.cu holds
 * the on-device image driver (base image and refinement levels of
 * src/main.c:520-792); host/render.c calls that driver and shares its
 * oddity report with it.  Everything here is plain C so that render.c can
 * include it. */
#ifndef IPG_INTERNAL_H
#define IPG_INTERNAL_H

#include <stdio.h>

#include "ipole_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- provided by ipg_kernels.cu ---- */
/* trace n pixels from the device list d_ij into d_out on the context's
 * stream (no host copies, no MaxNStep check: the caller inspects d_out) */
int ipg__trace_core(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *d_ij, size_t n, ipg_pixel_out *d_out);
/* the context's cudaStream_t */
void *ipg__stream(const ipg_ctx *ctx);
/* records `msg` as the context's last error (ipg_last_error) */
void ipg__set_error(ipg_ctx *ctx, const char *msg);
/* per-context storage owned by ipg_refine.cu; ipg_destroy releases it with
 * ipg__refine_release */
void **ipg__refine_slot(ipg_ctx *ctx);

/* the step arithmetic of the context (ipg_set_step_precision): 1 for FP32 */
int ipg__step32(const ipg_ctx *ctx);
int ipg__fits32(const ipg_ctx *ctx);
/* self-check of the adjoint's reverse-mode transfer step against forward
 * dual numbers on n seeded cases; *max_err the largest relative difference */
int ipg__check_step_vjp(int device, int n, unsigned long long seed, double max_err[4], double worst[96]);
/* per-context storage of the batch driver (ipg_refine.cu); ipg_destroy
 * releases it with ipg__batch_arena_release */
void **ipg__batch_arena_slot(ipg_ctx *ctx);
/* set-up of a batch: one camera per camera group, the derived-field set of
 * each (group, instance slot) as slot_set[g * G + k], the electron models */
int ipg__batch_begin(ipg_ctx *ctx, const ipg_camera *grp_cam, int ngrp, const int *slot_set, int G,
                     const ipg_electrons *sets, int nsets, int step32);
/* the items of one traced level of a batch (device arrays) */
typedef struct ipg_batch_items {
  size_t n_geo;             /* geodesic items: one per (camera group, pixel) some instance traces */
  const int32_t *geo_ij;    /* [2 n_geo] pixel */
  const int32_t *geo_grp;   /* [n_geo] camera group */
  const uint32_t *geo_mask; /* [n_geo] instance slots of the group that trace it */
  size_t n_xf;              /* transfer items: one per (instance, traced pixel) */
  const int32_t *xf_geo;    /* [n_xf] geodesic item */
  const int32_t *xf_slot;   /* [n_xf] instance slot in its group */
  ipg_pixel_out *xf_out;    /* [n_xf] get_pixel's outputs */
  const int32_t *xf_order;  /* [n_xf] the order in which the transfer takes the items (NULL: 0..n_xf-1) */
  const int32_t *geo_order; /* [n_geo] the order in which the geodesics start (NULL: 0..n_geo-1) */
  size_t n_long;            /* the first n_long of geo_order are the longest class (0: none) */
  double long_steps;        /* their predicted steps at the full step size */
  double pred_steps;        /* the predicted steps of all the items */
} ipg_batch_items;
/* the geodesic items in *sorted, longest predicted first (pred: n scratch);
 * *n_long of them, with *long_steps predicted steps, form the longest length
 * class (predicted at least the single image's first class factor times the
 * mean); *pred_steps is the predicted steps of all n */
int ipg__batch_sort_geo(ipg_ctx *ctx, const int32_t *geo_ij, const int32_t *geo_grp, size_t n, int maxnstep,
                        int32_t *pred, int32_t *sorted, size_t *n_long, double *long_steps, double *pred_steps);
/* trace one level; *steps_left (NULL: no budget) is the remaining step
 * budget, decreased by the steps taken */
int ipg__batch_trace(ipg_ctx *ctx, const ipg_batch_items *items, unsigned long long *steps_left);

/* ---- provided by host/model_iharm.c ---- */
/* RHO_unit and B_unit of a mass unit (set_units, model/iharm/model.c:595-608) */
void ipg__units(double M_unit, double L_unit, double *RHO_unit, double *B_unit);

/* ---- provided by ipg_refine.cu ---- */
void ipg__refine_release(void *bufs);
void ipg__batch_arena_release(void *arena);

/* what the image driver needs beyond the camera: the sizes and keys of
 * src/main.c:102-123 and the save_pixel/refinement parameters */
typedef struct ipg_refine_args {
  size_t nx, ny;       /* internal image size */
  size_t nxmin, nymin; /* internal size of the base image */
  int refine_level;    /* 1: no refinement */
  int params_nx, params_ny;
  double f3;           /* freqcgs^3 (save_pixel) */
  int only_unpolarized, qu_conv, nearest_neighbor;
  double refine_abs, refine_rel, refine_cut;
} ipg_refine_args;

/* Base image and refinement levels on the device, with the host driver's
 * results, log lines and error codes; fills img->image, taus, imageS (when
 * polarized), interp_flag, oddflag, nstep and traced (arrays allocated by
 * the caller, nx*ny). */
int ipg__render_levels_device(ipg_ctx *ctx, const ipg_camera *cam, const ipg_refine_args *a, void *img, FILE *log);

/* ---- provided by host/plugins.c ---- */
struct ipg_params;
struct ipg_iharm_model;
struct ipg_image;
/* the known-answer models' init_model; returns 1 (and *rc) when p->plugin
 * names one of them (or an unknown plugin), 0 for iharm */
int ipg__plugin_load(const struct ipg_params *p, struct ipg_iharm_model *m, int *rc);
/* their output_hdf5 into an ipgc_file */
void ipg__plugin_write_header(void *ipgc_file_ptr, const struct ipg_iharm_model *m);

/* ---- provided by host/render.c ---- */
/* write_header (src/io.c:140-191) into an ipgc_file */
void ipg__write_header(void *ipgc_file_ptr, const struct ipg_image *img, const struct ipg_params *p);
/* the oddity lines of get_pixel (src/main.c:852-869) for a traced list */
void ipg__report_oddities(int only_unpolarized, const int32_t *ij, const ipg_pixel_out *o, size_t n, FILE *log);

#ifdef __cplusplus
}
#endif
#endif
