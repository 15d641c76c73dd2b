/* Fast-light image driver (src/main.c:98-123, 184-197, 506-811): base image at
 * nx_min, adaptive refinement levels, save_pixel / lininterp bookkeeping,
 * image statistics and the image writer (src/io.c:140-273 with the iharm
 * output_hdf5, model/iharm/model.c:1254-1301).  Every level's pixels are
 * traced with one ipg_trace_pixels call. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../ipg_constants.h"
#include "../ipg_internal.h"
#include "ipgc.h"
#include "ipole_host.h"

#define NIMG 5
#define IPG_VERSION_STRING "ipole-b200-1"

void ipg_image_free(ipg_image *img)
{
  free(img->image);
  free(img->imageS);
  free(img->taus);
  free(img->interp_flag);
  free(img->oddflag);
  free(img->nstep);
  memset(img, 0, sizeof(*img));
}

/* save_pixel, src/main.c:885-910 */
static int save_pixel(ipg_image *img, const ipg_params *p, size_t i, size_t j, const ipg_pixel_out *o)
{
  const size_t ny = img->ny;
  double f3 = pow(p->freqcgs, 3);
  img->image[i * ny + j] = o->I_unpol * f3;
  img->taus[i * ny + j] = o->tau;
  img->oddflag[i * ny + j] = o->flag;
  img->nstep[i * ny + j] = o->nstep;
  if (!p->only_unpolarized) {
    double *s = img->imageS + (i * ny + j) * NIMG;
    s[0] = o->I * f3;
    if (p->qu_conv == 0) {
      s[1] = -o->Q * f3;
      s[2] = -o->U * f3;
    } else {
      s[1] = o->Q * f3;
      s[2] = o->U * f3;
    }
    s[3] = o->V * f3;
    s[4] = o->tauF;
    if (isnan(s[0])) {
      fprintf(stderr, "NaN in image! Exiting.\n");
      return IPG_E_NAN;
    }
  }
  return IPG_OK;
}

/* save_pixelTransfer, src/main.c:912-939 */
static int copy_pixel(ipg_image *img, int unpol, size_t io, size_t jo, size_t in, size_t jn)
{
  const size_t ny = img->ny;
  img->image[in * ny + jn] = img->image[io * ny + jo];
  if (!unpol) {
    img->taus[in * ny + jn] = img->taus[io * ny + jo];
    for (int c = 0; c < NIMG; c++) img->imageS[(in * ny + jn) * NIMG + c] = img->imageS[(io * ny + jo) * NIMG + c];
    if (isnan(img->imageS[(io * ny + jo) * NIMG])) return IPG_E_NAN;
  }
  return IPG_OK;
}

/* lininterp2, src/main.c:941-968 */
static int lininterp2(ipg_image *img, int unpol, size_t i1, size_t j1, size_t i2, size_t j2, size_t in, size_t jn)
{
  const size_t ny = img->ny;
  img->image[in * ny + jn] = .5 * (img->image[i1 * ny + j1] + img->image[i2 * ny + j2]);
  img->taus[in * ny + jn] = .5 * (img->taus[i1 * ny + j1] + img->taus[i2 * ny + j2]);
  if (!unpol) {
    for (int c = 0; c < NIMG; c++)
      img->imageS[(in * ny + jn) * NIMG + c] =
          .5 * (img->imageS[(i1 * ny + j1) * NIMG + c] + img->imageS[(i2 * ny + j2) * NIMG + c]);
    if (isnan(img->imageS[(i1 * ny + j1) * NIMG]) || isnan(img->imageS[(i2 * ny + j2) * NIMG])) return IPG_E_NAN;
  }
  return IPG_OK;
}

/* lininterp4, src/main.c:971-999 */
static int lininterp4(ipg_image *img, int unpol, size_t i1, size_t j1, size_t i2, size_t j2, size_t i3, size_t j3,
                      size_t i4, size_t j4, size_t in, size_t jn)
{
  const size_t ny = img->ny;
  img->image[in * ny + jn] = .25 * (img->image[i1 * ny + j1] + img->image[i2 * ny + j2] + img->image[i3 * ny + j3] +
                                    img->image[i4 * ny + j4]);
  img->taus[in * ny + jn] =
      .25 * (img->taus[i1 * ny + j1] + img->taus[i2 * ny + j2] + img->taus[i3 * ny + j3] + img->taus[i4 * ny + j4]);
  if (!unpol) {
    for (int c = 0; c < NIMG; c++)
      img->imageS[(in * ny + jn) * NIMG + c] =
          .25 * (img->imageS[(i1 * ny + j1) * NIMG + c] + img->imageS[(i2 * ny + j2) * NIMG + c] +
                 img->imageS[(i3 * ny + j3) * NIMG + c] + img->imageS[(i4 * ny + j4) * NIMG + c]);
    if (isnan(img->imageS[(i1 * ny + j1) * NIMG]) || isnan(img->imageS[(i2 * ny + j2) * NIMG]) ||
        isnan(img->imageS[(i3 * ny + j3) * NIMG]) || isnan(img->imageS[(i4 * ny + j4) * NIMG]))
      return IPG_E_NAN;
  }
  return IPG_OK;
}

void ipg__report_oddities(int only_unpolarized, const int32_t *ij, const ipg_pixel_out *o, size_t n, FILE *log)
{
  if (!log) return;
  for (size_t m = 0; m < n; m++) {
    if (o[m].flag != 0 || (!only_unpolarized && o[m].I < -1.e-10)) {
      fprintf(log, "\nOddity in pixel %d %d (flag %d):\n", ij[2 * m], ij[2 * m + 1], o[m].flag);
      fprintf(log, "nstep: %d\n", o[m].nstep);
      fprintf(log, "Final Stokes parameters: [%g %g %g %g]\n", o[m].I, o[m].Q, o[m].U, o[m].V);
    }
  }
}

typedef struct {
  ipg_tracer_fn fn;
  void *user;
} tracer_t;

static int ctx_tracer(void *user, const ipg_camera *cam, const int32_t *ij, size_t n, ipg_pixel_out *out)
{
  return ipg_trace_pixels((ipg_ctx *)user, cam, ij, n, out);
}

static int trace_list(const tracer_t *tr, const ipg_camera *cam, const int32_t *ij, size_t n, ipg_pixel_out *out,
                      FILE *log)
{
  int rc = tr->fn(tr->user, cam, ij, n, out);
  if (rc == IPG_E_MAXNSTEP) {
    for (size_t m = 0; m < n; m++)
      if (out[m].nstep >= cam->maxnstep - 1) {
        if (log) fprintf(log, "\nMaxNStep exceeded in pixel %d %d!\n", ij[2 * m], ij[2 * m + 1]);
        break;
      }
  } else if (rc != IPG_OK && log) {
    fprintf(log, "trace failed: %s\n", ipg_strerror(rc));
  }
  return rc;
}

static int render(ipg_tracer_fn tracer, void *user, ipg_ctx *dev, ipg_params *p, const ipg_iharm_model *m,
                  ipg_image *img, FILE *log);

/* With a context, the levels run on the device (ipg_refine.cu); the host
 * loop below serves caller-supplied tracers and check mode, and is the
 * device driver's bit-for-bit reference. */
int ipg_render_image(ipg_ctx *ctx, ipg_params *p, const ipg_iharm_model *m, ipg_image *img, void *logp)
{
  if (!ctx) return IPG_E_ARG;
  return render(ctx_tracer, ctx, p->perform_check ? NULL : ctx, p, m, img, (FILE *)logp);
}

int ipg_render_image_with(ipg_tracer_fn tracer, void *user, ipg_params *p, const ipg_iharm_model *m, ipg_image *img,
                          void *logp)
{
  return render(tracer, user, NULL, p, m, img, (FILE *)logp);
}

/* The set-up of one image (main.c:102-168): the refinement geometry, the
 * camera, the unit conversions of the parameters, and the image arrays
 * (calloc'ed, internal size).  Fills ra with the image driver's sizes and
 * keys.  Shared by the image driver and the batch driver. */
static int image_setup(ipg_params *p, const ipg_iharm_model *m, ipg_image *img, ipg_refine_args *ra, FILE *log)
{
  memset(img, 0, sizeof(*img));
  if (p->nx_min < 0) {
    p->nx_min = p->nx;
    p->ny_min = p->ny;
  }
  int refine_level = (int)(log2((double)((p->nx - p->nx % 2) / (p->nx_min - p->nx_min % 2))) + 1);
  size_t nx, ny, nxmin, nymin;
  if (refine_level > 1 && p->nx % 2 == 0) {
    nx = p->nx + 1;
    nxmin = p->nx_min + 1;
  } else {
    nx = p->nx;
    nxmin = p->nx_min;
  }
  if (refine_level > 1 && p->ny % 2 == 0) {
    ny = p->ny + 1;
    nymin = p->ny_min + 1;
  } else {
    ny = p->ny;
    nymin = p->ny_min;
  }
  if (nxmin < 2 || nymin < 2 || nx < 2 || ny < 2) {
    if (log) fprintf(log, "image sizes below 2 pixels are not supported\n");
    return IPG_E_ARG;
  }

  /* camera, main.c:125-168 */
  ipg_camera *cam = &img->cam;
  double scale, DX, DY;
  int rc = ipg_camera_setup(&m->grid, p->rcam, p->thetacam, p->phicam, p->rotcam, p->fovx_dsource, p->fovy_dsource,
                            p->dx, p->dy, p->dsource, p->nx, p->ny, p->freqcgs, p->old_centering, cam, &scale, &DX, &DY);
  if (rc) return rc;
  double fov_to_d = p->dsource * IPG_PC / m->grid.L_unit / IPG_MUAS_PER_RAD;
  if (p->fovx_dsource != 0.0) {
  } else if (p->dx != 0.0) {
    p->fovx_dsource = p->dx / fov_to_d;
    p->fovy_dsource = p->dy / fov_to_d;
  } else {
    p->fovx_dsource = 160.;
    p->fovy_dsource = 160.;
  }
  p->rotcam *= M_PI / 180.;
  p->dsource *= IPG_PC;
  p->dx = DX;
  p->dy = DY;
  cam->xoff = p->xoff;
  cam->yoff = p->yoff;
  cam->eps = p->eps;
  cam->maxnstep = p->maxnstep;
  cam->only_unpolarized = p->only_unpolarized;
  cam->emission_type = p->emission_type;
  cam->stokes_floors = p->stokes_floors;
  cam->target_nturns = p->target_nturns;
  cam->subring_dtheta = p->subring_dtheta;
  cam->counterjet = p->isolate_counterjet;
  img->scale = scale;
  memcpy(img->Xcam, cam->Xcam, sizeof(img->Xcam));
  img->fovx = cam->fovx;
  img->fovy = cam->fovy;
  if (log) {
    fprintf(log, "Xcam[] = %e %e %e %e\n", cam->Xcam[0], cam->Xcam[1], cam->Xcam[2], cam->Xcam[3]);
    fprintf(log, "intensity [cgs] to flux per pixel [Jy] conversion: %g\n", scale);
    fprintf(log, "Dsource: %g [cm]\n", p->dsource);
    fprintf(log, "Dsource: %g [kpc]\n", p->dsource / (1.e3 * IPG_PC));
    fprintf(log, "FOVx, FOVy: %g %g [GM/c^2]\n", DX, DY);
    fprintf(log, "FOVx, FOVy: %g %g [rad]\n", DX * m->grid.L_unit / p->dsource, DY * m->grid.L_unit / p->dsource);
    fprintf(log, "FOVx, FOVy: %g %g [muas]\n", DX * m->grid.L_unit / p->dsource * IPG_MUAS_PER_RAD,
            DY * m->grid.L_unit / p->dsource * IPG_MUAS_PER_RAD);
    if (refine_level > 1) {
      fprintf(log, "Resolution: %dx%d, refined up to %dx%d (%d levels)\n", p->nx_min, p->ny_min, p->nx, p->ny,
              refine_level);
      fprintf(log,
              "Refinement when relative error is >%g%% or absolute error is >%g%% of estimated total flux, for pixel "
              "brightness > %f%% of average\n",
              p->refine_rel * 100, p->refine_abs * 100, p->refine_cut * 100);
    } else {
      fprintf(log, "Resolution: %dx%d\n", p->nx, p->ny);
    }
  }

  img->nx = nx;
  img->ny = ny;
  img->image = (double *)calloc(nx * ny, sizeof(double));
  img->taus = (double *)calloc(nx * ny, sizeof(double));
  img->interp_flag = (int *)calloc(nx * ny, sizeof(int));
  img->oddflag = (int32_t *)calloc(nx * ny, sizeof(int32_t));
  img->nstep = (int32_t *)calloc(nx * ny, sizeof(int32_t));
  if (!p->only_unpolarized) img->imageS = (double *)calloc(nx * ny * NIMG, sizeof(double));
  if (!img->image || !img->taus || !img->interp_flag || !img->oddflag || !img->nstep ||
      (!p->only_unpolarized && !img->imageS))
    return IPG_E_NOMEM;
  ra->nx = nx;
  ra->ny = ny;
  ra->nxmin = nxmin;
  ra->nymin = nymin;
  ra->refine_level = refine_level;
  ra->params_nx = p->nx;
  ra->params_ny = p->ny;
  ra->f3 = pow(p->freqcgs, 3);
  ra->only_unpolarized = p->only_unpolarized;
  ra->qu_conv = p->qu_conv;
  ra->nearest_neighbor = p->nearest_neighbor;
  ra->refine_abs = p->refine_abs;
  ra->refine_rel = p->refine_rel;
  ra->refine_cut = p->refine_cut;
  return IPG_OK;
}

static int render(ipg_tracer_fn tracer, void *user, ipg_ctx *dev, ipg_params *p, const ipg_iharm_model *m,
                  ipg_image *img, FILE *log)
{
  if (!tracer || !p || !m || !img) return IPG_E_ARG;
  tracer_t tr = {tracer, user};
  if (p->perform_check && log) fprintf(log, "Running in check mode...\n");
  ipg_refine_args ra;
  int rc = image_setup(p, m, img, &ra, log);
  if (rc) return rc;
  const size_t nx = ra.nx, ny = ra.ny, nxmin = ra.nxmin, nymin = ra.nymin;
  const int refine_level = ra.refine_level;
  ipg_camera *cam = &img->cam;
  int32_t *ij = (int32_t *)malloc(2 * nx * ny * sizeof(int32_t));
  ipg_pixel_out *out = (ipg_pixel_out *)malloc(nx * ny * sizeof(ipg_pixel_out));
  if (!ij || !out) {
    free(ij);
    free(out);
    return IPG_E_NOMEM;
  }

  if (p->perform_check) {
    /* check mode, main.c:538-575: every CHECK_SKIP-th pixel and its mirror
     * in i, saved side by side at reduced indices (check, then recheck) */
    if (refine_level > 1) {
      if (log) fprintf(log, "check mode needs an unrefined image (nx_min = nx)\n");
      free(ij);
      free(out);
      return IPG_E_ARG;
    }
    const size_t skip = IPG_CHECK_SKIP;
    size_t offset = nx % skip;
    if (offset == 0) offset = skip;
    size_t n = 0;
    for (size_t i = 0; i < nx; i++)
      for (size_t j = 0; j < ny; j++) {
        if (i % skip != 0 || j % skip != 0) continue;
        ij[2 * n] = (int32_t)i;
        ij[2 * n + 1] = (int32_t)j;
        n++;
        ij[2 * n] = (int32_t)(nx - i - offset);
        ij[2 * n + 1] = (int32_t)j;
        n++;
      }
    rc = trace_list(&tr, cam, ij, n, out, log);
    if (rc == IPG_OK) ipg__report_oddities(p->only_unpolarized, ij, out, n, log);
    for (size_t q = 0; rc == IPG_OK && q < n; q += 2) {
      size_t i = (size_t)ij[2 * q], j = (size_t)ij[2 * q + 1], i2 = (size_t)ij[2 * q + 2];
      rc = save_pixel(img, p, i / skip, j / skip, &out[q]);
      if (rc == IPG_OK) rc = save_pixel(img, p, (nx / skip) + i2 / skip, j / skip, &out[q + 1]);
    }
    img->traced = n;
    free(ij);
    free(out);
    return rc;
  }

  if (dev) {
    free(ij);
    free(out);
    return ipg__render_levels_device(dev, cam, &ra, img, log);
  }

  /* base image, main.c:535-615 */
  size_t sx = (nx - 1) / (nxmin - 1);
  size_t sy = (ny - 1) / (nymin - 1);
  double *prelim = refine_level > 1 ? (double *)calloc(nxmin * nymin, sizeof(double)) : NULL;
  size_t n = 0;
  for (size_t i = 0; i < nx; i += sx)
    for (size_t j = 0; j < ny; j += sy) {
      ij[2 * n] = (int32_t)i;
      ij[2 * n + 1] = (int32_t)j;
      n++;
    }
  rc = trace_list(&tr, cam, ij, n, out, log);
  if (rc) goto done;
  ipg__report_oddities(p->only_unpolarized, ij, out, n, log);
  for (size_t q = 0; q < n; q++) {
    size_t i = (size_t)ij[2 * q], j = (size_t)ij[2 * q + 1];
    rc = save_pixel(img, p, i, j, &out[q]);
    if (rc) goto done;
    img->interp_flag[i * ny + j] = 0;
    if (refine_level > 1) {
      double Intensity = out[q].I_unpol;
      size_t loc = i / sy * nymin + j / sx;
      if (loc >= nxmin * nymin) continue; /* only when sx != sy */
      if (i % (nx - 1) != 0 && j % (ny - 1) != 0) prelim[loc] = Intensity * sx * sx;
      else if ((i == 0 && j % (ny - 1) != 0) || (i % (nx - 1) != 0 && j == 0))
        prelim[loc] = Intensity * (sx / 2 + 1) * sx;
      else if (i % (nx - 1) != 0 || j % (ny - 1) != 0) prelim[loc] = Intensity * (sx / 2) * sx;
      else if (i == 0 && j == 0) prelim[loc] = Intensity * (sx / 2 + 1) * (sx / 2 + 1);
      else if (i == 0 || j == 0) prelim[loc] = Intensity * (sx / 2 + 1) * sx / 2;
      else prelim[loc] = Intensity * (sx * sx) / 4;
    }
  }
  img->traced = n;

  double Iavg = 0;
  if (refine_level > 1) {
    double interp_tot = 0;
    for (size_t q = 0; q < nxmin * nymin; q++) interp_tot += prelim[q];
    Iavg = interp_tot * pow(p->freqcgs, 3) / (nx * ny);
  }

  /* refinement levels, main.c:635-792 */
  for (int lvl = 1; lvl < refine_level; lvl++) {
    size_t nsx = sx / pow(2, lvl);
    size_t nsy = sy / pow(2, lvl);
    size_t psx = nsx * 2, psy = nsy * 2;
    if (nsx < 1 || nsy < 1) { /* the reference loops forever here */
      if (log) fprintf(log, "refinement spacing below one pixel at level %d: nx_min/ny_min too small\n", lvl + 1);
      rc = IPG_E_ARG;
      goto done;
    }
    if (log) fprintf(log, "Refining level %d of %d, spacing %zu,%zu\n", lvl + 1, refine_level, nsx, nsy);
    n = 0;
    for (size_t i = 0; i < nx; i += nsx)
      for (size_t j = 0; j < ny; j += nsy) {
        if (i % psx == 0 && j % psy == 0) continue;
        double I1 = 0, I2, I3, err_abs = 0, err_rel = 0;
        int trace;
        /* the +ns neighbours exist unless the spacing does not divide the
         * image (a base-to-final ratio that is not a power of two), where the
         * reference reads past the image: such a pixel is traced */
        int inside = (i % psx == 0 || i + nsx <= nx - 1) && (j % psy == 0 || j + nsy <= ny - 1);
        if (!inside) {
        } else if (i % psx == 0) {
          I1 = img->image[i * ny + j - nsy];
          I2 = img->image[i * ny + j + nsy];
          err_abs = (I2 - I1) / 2 / Iavg;
          err_rel = (I2 - I1) / 2 / I1;
        } else if (j % psy == 0) {
          I1 = img->image[(i - nsx) * ny + j];
          I2 = img->image[(i + nsx) * ny + j];
          err_abs = (I2 - I1) / 2 / Iavg;
          err_rel = (I2 - I1) / 2 / I1;
        } else {
          I1 = img->image[(i - nsx) * ny + j - nsy];
          I2 = img->image[(i + nsx) * ny + j - nsy];
          I3 = img->image[(i - nsx) * ny + j + nsy];
          err_abs = ((I2 + I3) / 2 - I1) / Iavg;
          err_rel = (I2 + I3) / (2 * I1) - 1.;
        }
        trace = !inside || ((fabs(err_abs) > p->refine_abs && fabs(err_rel) > p->refine_rel) && fabs(I1) > p->refine_cut);
        if (trace) {
          ij[2 * n] = (int32_t)i;
          ij[2 * n + 1] = (int32_t)j;
          n++;
          img->interp_flag[i * ny + j] = 0;
          continue;
        }
        img->interp_flag[i * ny + j] = 1;
        int unpol = p->only_unpolarized;
        if (i % psx == 0) {
          rc = p->nearest_neighbor ? copy_pixel(img, unpol, i, j - nsy, i, j)
                                   : lininterp2(img, unpol, i, j - nsy, i, j + nsy, i, j);
        } else if (j % psy == 0) {
          rc = p->nearest_neighbor ? copy_pixel(img, unpol, i - nsx, j, i, j)
                                   : lininterp2(img, unpol, i - nsx, j, i + nsx, j, i, j);
        } else {
          rc = p->nearest_neighbor
                   ? copy_pixel(img, unpol, i - nsx, j - nsy, i, j)
                   : lininterp4(img, unpol, i - nsx, j - nsy, i + nsx, j - nsy, i - nsx, j + nsy, i + nsx, j + nsy, i,
                                j);
        }
        if (rc) {
          if (log) fprintf(log, "NaN in image! Exiting.\n");
          goto done;
        }
      }
    if (n) {
      rc = trace_list(&tr, cam, ij, n, out, log);
      if (rc) goto done;
      ipg__report_oddities(p->only_unpolarized, ij, out, n, log);
      for (size_t q = 0; q < n; q++) {
        rc = save_pixel(img, p, (size_t)ij[2 * q], (size_t)ij[2 * q + 1], &out[q]);
        if (rc) goto done;
      }
      img->traced += n;
    }
    size_t total_interpolated = 0;
    for (size_t q = 0; q < nx * ny; q++) total_interpolated += img->interp_flag[q];
    size_t nxl = p->nx / nsx, nyl = p->ny / nsy;
    if (log)
      fprintf(log, "\n%zu of %zu (%f%%) of computed pixels at %zux%zu were interpolated\n\n", total_interpolated,
              nxl * nyl, ((double)total_interpolated) / (nxl * nyl) * 100, nxl, nyl);
  }
done:
  free(prelim);
  free(ij);
  free(out);
  return rc;
}

/* ---- batches (ipg_render_batch) ---- */
int ipg_upload_model_batch(ipg_ctx *ctx, const ipg_iharm_model *m)
{
  if (!ctx || !m || m->plugin.kind != IPG_PLUGIN_IHARM || !m->bmag_code || !m->trace_fields[0] ||
      !m->trace_fields[1])
    return IPG_E_ARG;
  const double *prims[IPG_NBPRIM] = {m->trace_fields[0],  m->trace_fields[1],  m->fields[IPG_F_U1],
                                     m->fields[IPG_F_U2], m->fields[IPG_F_U3], m->fields[IPG_F_B1],
                                     m->fields[IPG_F_B2], m->fields[IPG_F_B3], m->bmag_code};
  return ipg_upload_iharm_batch(ctx, &m->grid, prims, m->gam, m->game, m->gamp);
}

int ipg_render_batch_params(ipg_ctx *ctx, ipg_params *const *ps, size_t n, const ipg_iharm_model *m,
                            ipg_image *imgs, uint64_t step_budget, void *logp)
{
  FILE *log = (FILE *)logp;
  if (!ctx || !ps || !m || !imgs || n == 0) return IPG_E_ARG;
  for (size_t i = 0; i < n; i++) memset(&imgs[i], 0, sizeof(imgs[i]));
  if (m->plugin.kind != IPG_PLUGIN_IHARM) return IPG_E_ARG;
  ipg_instance *inst = (ipg_instance *)calloc(n, sizeof(ipg_instance));
  ipg_instance_image *outs = (ipg_instance_image *)calloc(n, sizeof(ipg_instance_image));
  int rc = (inst && outs) ? IPG_OK : IPG_E_NOMEM;
  for (size_t i = 0; rc == IPG_OK && i < n; i++) {
    ipg_params *p = ps[i];
    /* the keys a batch does not serve: check mode, the accretion-rate
     * rescaling of M_unit and the cooling cap of Theta_e; the black-hole
     * mass fixes L_unit, which the dump's geometry carries */
    const double L_unit = IPG_GNEWT * (p->MBH_solar * IPG_MSUN) / (IPG_CL * IPG_CL);
    if (p->perform_check || p->target_mdot > 0 || p->cooling_dynamical_times > 1e-20 ||
        L_unit != m->grid.L_unit) {
      if (log)
        fprintf(log, "batch instance %zu: check mode, target_mdot, cooling_dynamical_times and a black-hole "
                     "mass other than the model's are not supported in a batch\n", i);
      rc = IPG_E_ARG;
      break;
    }
    ipg_refine_args ra;
    rc = image_setup(p, m, &imgs[i], &ra, log);
    if (rc) break;
    ipg_instance *a = &inst[i];
    a->cam = imgs[i].cam;
    ipg__units(p->M_unit, m->grid.L_unit, &a->el.RHO_unit, &a->el.B_unit);
    a->el.trat_large = p->trat_large;
    a->el.trat_small = p->trat_small;
    a->el.beta_crit = p->beta_crit;
    a->nx = (int)ra.nx;
    a->ny = (int)ra.ny;
    a->nx_min = (int)ra.nxmin;
    a->ny_min = (int)ra.nymin;
    a->refine_level = ra.refine_level;
    a->f3 = ra.f3;
    a->qu_conv = ra.qu_conv;
    a->nearest_neighbor = ra.nearest_neighbor;
    a->refine_abs = ra.refine_abs;
    a->refine_rel = ra.refine_rel;
    a->refine_cut = ra.refine_cut;
    outs[i].image = imgs[i].image;
    outs[i].imageS = imgs[i].imageS;
    outs[i].taus = imgs[i].taus;
    outs[i].interp_flag = imgs[i].interp_flag;
    outs[i].oddflag = imgs[i].oddflag;
    outs[i].nstep = imgs[i].nstep;
  }
  if (rc == IPG_OK) rc = ipg_render_batch(ctx, inst, n, outs, step_budget);
  if (rc == IPG_OK)
    for (size_t i = 0; i < n; i++) imgs[i].traced = outs[i].traced;
  free(inst);
  free(outs);
  return rc;
}

/* ---- adjoint of an image ---- */
int ipg_adjoint_params(ipg_ctx *ctx, ipg_params *p, const ipg_iharm_model *m, const double *dL_dpol,
                       int ckpt_interval, ipg_grad *g, double *pol_out)
{
  if (!ctx || !p || !m || !dL_dpol || !g) return IPG_E_ARG;
  if (m->plugin.kind != IPG_PLUGIN_IHARM || !m->trace_fields[0] || !m->trace_fields[1] || !m->bmag_code ||
      p->only_unpolarized || p->perform_check || p->target_mdot > 0 || p->cooling_dynamical_times > 1e-20)
    return IPG_E_ARG;
  ipg_image img;
  ipg_refine_args ra;
  int rc = image_setup(p, m, &img, &ra, NULL);
  if (rc == IPG_OK && ra.refine_level != 1) rc = IPG_E_ARG; /* the adjoint traces every pixel */
  const size_t nx = ra.nx, ny = ra.ny, npix = nx * ny;
  const ipg_grid *gr = &m->grid;
  const size_t ncell = (size_t)(gr->n1 + 2) * (gr->n2 + 2) * (gr->n3 + 2);
  int32_t *ij = NULL;
  double *dL = NULL, *gbuf = NULL;
  double *gne = g->d_ne, *gth = g->d_thetae, *gb = g->d_b; /* the cells' gradients land in the caller's arrays */
  ipg_pixel_out *out = NULL;
  if (rc == IPG_OK) {
    ij = (int32_t *)malloc(2 * npix * sizeof(int32_t));
    dL = (double *)malloc(4 * npix * sizeof(double));
    out = (ipg_pixel_out *)malloc(npix * sizeof(ipg_pixel_out));
    /* scratch only for the arrays the caller does not take */
    const size_t nmiss = (gne ? 0 : 1) + (gth ? 0 : 1) + (gb ? 0 : 1);
    if (nmiss) gbuf = (double *)malloc(nmiss * ncell * sizeof(double));
    if (!ij || !dL || !out || (nmiss && !gbuf)) rc = IPG_E_NOMEM;
    double *q = gbuf;
    if (!gne) gne = q, q += ncell;
    if (!gth) gth = q, q += ncell;
    if (!gb) gb = q;
  }
  if (rc == IPG_OK) {
    /* save_pixel (main.c:885-910): pol = (I, Q, U, V) nu^3, Q and U negated
     * for qu_conv = 0 */
    const double sq = p->qu_conv ? 1. : -1.;
    for (size_t i = 0; i < nx; i++)
      for (size_t j = 0; j < ny; j++) {
        const size_t q = i * ny + j;
        ij[2 * q] = (int32_t)i;
        ij[2 * q + 1] = (int32_t)j;
        dL[4 * q] = dL_dpol[4 * q] * ra.f3;
        dL[4 * q + 1] = dL_dpol[4 * q + 1] * sq * ra.f3;
        dL[4 * q + 2] = dL_dpol[4 * q + 2] * sq * ra.f3;
        dL[4 * q + 3] = dL_dpol[4 * q + 3] * ra.f3;
      }
    rc = ipg_adjoint(ctx, &img.cam, ij, npix, dL, ckpt_interval, gne, gth, gb, out);
  }
  if (rc == IPG_OK) {
    if (pol_out) {
      const double sq = p->qu_conv ? 1. : -1.;
      for (size_t q = 0; q < npix; q++) {
        pol_out[4 * q] = out[q].I * ra.f3;
        pol_out[4 * q + 1] = sq * out[q].Q * ra.f3;
        pol_out[4 * q + 2] = sq * out[q].U * ra.f3;
        pol_out[4 * q + 3] = out[q].V * ra.f3;
      }
    }
    /* the electron model's parameters through init_physical_quantities
     * (model/iharm/model.c:610-717): ne is proportional to M_unit and |B|
     * to its square root; Theta_e = Th_u(trat) u / rho with
     * trat = (R_high betasq + R_low) / (1 + betasq), floored at 1e-3 */
    const double *ne = m->fields[IPG_F_NE], *th = m->fields[IPG_F_THETAE], *bb = m->fields[IPG_F_B];
    const double *rho = m->trace_fields[0], *uu = m->trace_fields[1];
    const double gam = m->gam, game = m->game, gamp = m->gamp;
    const double gem1 = game - 1., gpm1 = gamp - 1.;
    double dM = 0., dRh = 0., dRl = 0.;
    /* over the host's cores: ~5e6 cells of a production dump */
#pragma omp parallel for reduction(+ : dM, dRh, dRl) schedule(static)
    for (size_t c = 0; c < ncell; c++) {
      const double gn = gne[c], gt = gth[c], gbc = gb[c];
      dM += gn * ne[c] + 0.5 * gbc * bb[c];
      if (gt == 0.) continue;
      double bsq = bb[c] / m->B_unit;
      bsq = bsq * bsq;
      const double beta = uu[c] * (gam - 1.) / 0.5 / bsq;
      const double betasq = beta * beta / p->beta_crit / p->beta_crit;
      const double trat = p->trat_large * betasq / (1. + betasq) + p->trat_small / (1. + betasq);
      const double den = gpm1 + gem1 * trat;
      const double th_raw = (IPG_MP / IPG_ME) * gem1 * gpm1 / den * uu[c] / rho[c];
      if (!(th_raw >= 1.e-3) || th[c] != th_raw) continue; /* floored */
      const double dth_dtrat = -th_raw * gem1 / den;
      dRh += gt * dth_dtrat * betasq / (1. + betasq);
      dRl += gt * dth_dtrat / (1. + betasq);
    }
    g->d_M_unit = dM / m->M_unit;
    g->d_R_high = dRh;
    g->d_R_low = dRl;
  }
  free(ij);
  free(dL);
  free(out);
  free(gbuf);
  ipg_image_free(&img);
  return rc;
}

void ipg_image_totals(const ipg_image *img, const ipg_params *p, double tot[5])
{
  double Ftot = 0., Ftot_unpol = 0., Qtot = 0., Utot = 0., Vtot = 0.;
  const size_t ny = img->ny;
  for (size_t i = 0; i < (size_t)p->nx; i++)
    for (size_t j = 0; j < (size_t)p->ny; j++) {
      Ftot_unpol += img->image[i * ny + j] * img->scale;
      if (!p->only_unpolarized) {
        Ftot += img->imageS[(i * ny + j) * NIMG + 0] * img->scale;
        Qtot += img->imageS[(i * ny + j) * NIMG + 1] * img->scale;
        Utot += img->imageS[(i * ny + j) * NIMG + 2] * img->scale;
        Vtot += img->imageS[(i * ny + j) * NIMG + 3] * img->scale;
      }
    }
  tot[0] = Ftot;
  tot[1] = Ftot_unpol;
  tot[2] = Qtot;
  tot[3] = Utot;
  tot[4] = Vtot;
}

/* src/main.c:1001-1042 */
void ipg_print_image_stats(const ipg_image *img, const ipg_params *p, void *logp)
{
  FILE *log = (FILE *)logp;
  if (!log) return;
  double Imax = 0.0, Iavg = 0.0;
  size_t imax = 0, jmax = 0;
  const size_t ny = img->ny;
  double t[5];
  ipg_image_totals(img, p, t);
  if (!p->only_unpolarized)
    for (size_t i = 0; i < (size_t)p->nx; i++)
      for (size_t j = 0; j < (size_t)p->ny; j++) {
        double v = img->imageS[(i * ny + j) * NIMG + 0];
        Iavg += v;
        if (v > Imax) {
          imax = i;
          jmax = j;
          Imax = v;
        }
      }
  fprintf(log, "\nscale = %e\n", img->scale);
  fprintf(log, "imax=%zu jmax=%zu Imax=%g Iavg=%g\n", imax, jmax, Imax, Iavg / (p->nx * p->ny));
  fprintf(log, "freq: %g Ftot: %g Jy (%g Jy unpol xfer) scale=%g\n", p->freqcgs, t[0], t[1], img->scale);
  fprintf(log, "nuLnu = %g erg/s\n", 4. * M_PI * t[0] * p->dsource * p->dsource * IPG_JY * p->freqcgs);
  double LPfrac = 100. * sqrt(t[2] * t[2] + t[3] * t[3]) / t[0];
  double CPfrac = 100. * t[4] / t[0];
  fprintf(log, "I,Q,U,V [Jy]: %g %g %g %g\n", t[0], t[2], t[3], t[4]);
  fprintf(log, "LP,CP [%%]: %g %g\n", LPfrac, CPfrac);
}

/* dump (src/io.c:229-273) + write_header (:140-191) + output_hdf5
 * (model/iharm/model.c:1254-1301) */
/* write_header, src/io.c:140-191 (the image file and the trace file) */
void ipg__write_header(void *fp, const ipg_image *img, const ipg_params *p)
{
  ipgc_file *fh = (ipgc_file *)fp;
#define f (*fh)
  ipgc_put_str(&f, "/@githash", "b200", 20);
  ipgc_put_group(&f, "/header");
  ipgc_put_str(&f, "/header/version", IPG_VERSION_STRING, 20);
  ipgc_put_str(&f, "/header/githash", "b200", 20);
  ipgc_put_f64(&f, "/header/freqcgs", p->freqcgs);
  ipgc_put_f64(&f, "/header/scale", img->scale);
  ipgc_put_f64(&f, "/header/dsource", p->dsource);
  ipgc_put_str(&f, "/header/evpa_0", p->qu_conv == 0 ? "N" : "W", 2);
  ipgc_put_group(&f, "/header/camera");
  ipgc_put_i32(&f, "/header/camera/nx", p->nx);
  ipgc_put_i32(&f, "/header/camera/ny", p->ny);
  ipgc_put_f64(&f, "/header/camera/dx", p->dx);
  ipgc_put_f64(&f, "/header/camera/dy", p->dy);
  ipgc_put_f64(&f, "/header/camera/fovx_dsource", p->fovx_dsource);
  ipgc_put_f64(&f, "/header/camera/fovy_dsource", p->fovy_dsource);
  ipgc_put_f64(&f, "/header/camera/rcam", p->rcam);
  ipgc_put_f64(&f, "/header/camera/thetacam", p->thetacam);
  ipgc_put_f64(&f, "/header/camera/phicam", p->phicam);
  ipgc_put_f64(&f, "/header/camera/rotcam", p->rotcam);
  ipgc_put_f64(&f, "/header/camera/fovx", img->fovx);
  ipgc_put_f64(&f, "/header/camera/fovy", img->fovy);
  ipgc_put_f64(&f, "/header/camera/xoff", p->xoff);
  ipgc_put_f64(&f, "/header/camera/yoff", p->yoff);
  uint64_t d4 = 4;
  ipgc_put_array_f64(&f, "/header/camera/x", 1, &d4, img->Xcam);
#undef f
}

int ipg_write_image(const char *fname, const ipg_image *img, const ipg_params *p, const ipg_iharm_model *m)
{
  ipgc_file f = {0};
  ipg__write_header(&f, img, p);
  if (m && m->plugin.kind != IPG_PLUGIN_IHARM) {
    ipg__plugin_write_header(&f, m);
  } else if (m) {
    if (m->fluid_header) ipgc_copy_subtree((const ipgc_file *)m->fluid_header, "", &f, "/fluid_header");
    ipgc_put_f64(&f, "/Mdot", m->Mdot_dump);
    ipgc_put_f64(&f, "/MdotEdd", m->MdotEdd_dump);
    ipgc_put_f64(&f, "/Ladv", m->Ladv_dump);
    ipgc_put_f64(&f, "/header/t", m->t);
    ipgc_put_f64(&f, "/header/sigma_cut", p->sigma_cut);
    ipgc_put_group(&f, "/header/electrons");
    ipgc_put_f64(&f, "/header/electrons/rlow", p->trat_small);
    ipgc_put_f64(&f, "/header/electrons/rhigh", p->trat_large);
    ipgc_put_f64(&f, "/header/electrons/beta_crit", p->beta_crit);
    ipgc_put_i32(&f, "/header/electrons/type", m->electrons);
    ipgc_put_i32(&f, "/header/field_config", p->reverse_field);
    ipgc_put_group(&f, "/header/units");
    ipgc_put_f64(&f, "/header/units/L_unit", m->L_unit);
    ipgc_put_f64(&f, "/header/units/M_unit", m->M_unit);
    ipgc_put_f64(&f, "/header/units/T_unit", m->T_unit);
    ipgc_put_f64(&f, "/header/units/Thetae_unit", m->Te_unit);
  }
  double t[5];
  ipg_image_totals(img, p, t);
  ipgc_put_f64(&f, "/Ftot_unpol", t[1]);
  if (!p->only_unpolarized) ipgc_put_f64(&f, "/Ftot", t[0]);
  ipgc_put_f64(&f, "/nuLnu", 4. * M_PI * t[0] * p->dsource * p->dsource * IPG_JY * p->freqcgs);
  ipgc_put_f64(&f, "/nuLnu_unpol", 4. * M_PI * t[1] * p->dsource * p->dsource * IPG_JY * p->freqcgs);
  size_t nx = (size_t)p->nx, ny = (size_t)p->ny;
  double *buf = (double *)malloc(nx * ny * NIMG * sizeof(double));
  uint64_t d2[2] = {nx, ny}, d3[3] = {nx, ny, NIMG};
  for (size_t i = 0; i < nx; i++) memcpy(buf + i * ny, img->image + i * img->ny, ny * sizeof(double));
  ipgc_put_array_f64(&f, "/unpol", 2, d2, buf);
  for (size_t i = 0; i < nx; i++) memcpy(buf + i * ny, img->taus + i * img->ny, ny * sizeof(double));
  ipgc_put_array_f64(&f, "/tau", 2, d2, buf);
  if (!p->only_unpolarized) {
    for (size_t i = 0; i < nx; i++)
      memcpy(buf + i * ny * NIMG, img->imageS + i * img->ny * NIMG, ny * NIMG * sizeof(double));
    ipgc_put_array_f64(&f, "/pol", 3, d3, buf);
  }
  free(buf);
  int rc = ipgc_save(fname, &f) == 0 ? IPG_OK : IPG_E_IO;
  if (rc) fprintf(stderr, "! %s\n", ipgc_error());
  ipgc_free(&f);
  return rc;
}

/* dump_check, src/io.c:193-227: appends the check and recheck blocks of a
 * check-mode image (rows [0, nx/skip) and [nx/skip, 2 nx/skip), columns
 * [0, ny/skip)) to an existing image file; without one it only says so. */
int ipg_write_check(const char *fname, const ipg_image *img, const ipg_params *p)
{
  ipgc_file f;
  if (ipgc_load(fname, &f) != 0) {
    fprintf(stderr, "oh no :(\nno file to check.\n\n");
    return IPG_OK;
  }
  const size_t skip = IPG_CHECK_SKIP, nx = (size_t)p->nx, ny = (size_t)p->ny, ld = img->ny;
  const size_t fx = nx / skip, fy = ny / skip;
  const int unpol = p->only_unpolarized;
  double *buf = (double *)malloc((fx * fy * NIMG + 1) * sizeof(double));
  uint64_t d2[2] = {fx, fy}, d3[3] = {fx, fy, NIMG};
  for (int pass = 0; pass < 2; pass++) {
    const size_t r0 = pass ? fx : 0;
    const char *sfx = pass ? "recheck" : "check";
    char name[32];
    for (size_t i = 0; i < fx; i++)
      for (size_t j = 0; j < fy; j++) buf[i * fy + j] = img->image[(r0 + i) * ld + j];
    snprintf(name, sizeof(name), "/unpol_%s", sfx);
    ipgc_put_array_f64(&f, name, 2, d2, buf);
    for (size_t i = 0; i < fx; i++)
      for (size_t j = 0; j < fy; j++) buf[i * fy + j] = img->taus[(r0 + i) * ld + j];
    snprintf(name, sizeof(name), "/tau_%s", sfx);
    ipgc_put_array_f64(&f, name, 2, d2, buf);
    if (!unpol) {
      for (size_t i = 0; i < fx; i++)
        for (size_t j = 0; j < fy; j++)
          for (int c = 0; c < NIMG; c++) buf[(i * fy + j) * NIMG + c] = img->imageS[((r0 + i) * ld + j) * NIMG + c];
      snprintf(name, sizeof(name), "/pol_%s", sfx);
      ipgc_put_array_f64(&f, name, 3, d3, buf);
    }
  }
  free(buf);
  int rc = ipgc_save(fname, &f) == 0 ? IPG_OK : IPG_E_IO;
  if (rc) fprintf(stderr, "! %s\n", ipgc_error());
  ipgc_free(&f);
  return rc;
}

int ipg_container_convert(const char *src, const char *dst)
{
  if (!src || !dst) return IPG_E_ARG;
  ipgc_file f;
  int rc = ipgc_load(src, &f);
  if (rc) {
    fprintf(stderr, "! %s\n", ipgc_error());
    return rc == -2 ? IPG_E_FORMAT : IPG_E_IO;
  }
  rc = ipgc_save(dst, &f) == 0 ? IPG_OK : IPG_E_IO;
  if (rc) fprintf(stderr, "! %s\n", ipgc_error());
  ipgc_free(&f);
  return rc;
}
