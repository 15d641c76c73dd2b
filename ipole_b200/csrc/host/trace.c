/* Trace output of the traced pixels (dump_var_along, src/io.c:279-543, with
 * the pixel selection of src/main.c:865-879), from the device's per-step
 * trace of each ray (ipg_trace_ray). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../ipg_internal.h"
#include "ipgc.h"
#include "ipole_host.h"

/* dataset name, first column of the trace row, values per step */
typedef struct {
  const char *name;
  int col, width;
} tr_set;

static const tr_set SETS[] = {
    {"b", IPG_TRACE_B, 1},          {"ne", IPG_TRACE_NE, 1},
    {"thetae", IPG_TRACE_THETAE, 1}, {"nu", IPG_TRACE_NU, 1},
    {"b_k_angle", IPG_TRACE_BK_ANGLE, 1}, {"sigma", IPG_TRACE_SIGMA, 1},
    {"beta", IPG_TRACE_BETA, 1},    {"dl", IPG_TRACE_DL, 1},
    {"r", IPG_TRACE_R, 1},          {"th", IPG_TRACE_TH, 1},
    {"phi", IPG_TRACE_PHI, 1},      {"j_unpol", IPG_TRACE_J_UNPOL, 1},
    {"k_unpol", IPG_TRACE_K_UNPOL, 1}, {"I_unpol", IPG_TRACE_I_UNPOL, 1},
    {"X", IPG_TRACE_X, 4},          {"Kcon", IPG_TRACE_KCON, 4},
    {"j_inv", IPG_TRACE_J_INV, 4},  {"alpha_inv", IPG_TRACE_ALPHA_INV, 4},
    {"rho_inv", IPG_TRACE_RHO_INV, 4}, {"stokes", IPG_TRACE_STOKES, 4},
    {"e2Constructed", IPG_TRACE_E2C, 4}, {"e2ConstructedCov", IPG_TRACE_E2C_COV, 4},
    {"e2Transported", IPG_TRACE_E2T, 4}, {"e2TransportedCov", IPG_TRACE_E2T_COV, 4},
    {"prims", IPG_TRACE_PRIMS, 8},  {"ntetrad", IPG_TRACE_NTETRAD, 16},
    {"ncoord", IPG_TRACE_NCOORD, 16}, {"Econ", IPG_TRACE_ECON, 16},
    {"Ecov", IPG_TRACE_ECOV, 16},
};
#define NSETS ((int)(sizeof(SETS) / sizeof(SETS[0])))

typedef struct {
  int ti, tj;     /* position in the trace file */
  int32_t nstep;
  double *rows;   /* (nstep + 1) x IPG_TRACE_DOUBLES */
} tr_pix;

static int set_rank(const tr_set *s) { return s->width == 1 ? 3 : (s->width == 16 ? 5 : 4); }

static void set_dims(const tr_set *s, uint64_t nxt, uint64_t nyt, uint64_t L, uint64_t d[5])
{
  d[0] = nxt;
  d[1] = nyt;
  d[2] = L;
  if (s->width == 16) {
    d[3] = d[4] = 4;
  } else if (s->width > 1) {
    d[3] = (uint64_t)s->width;
  }
}

int ipg_write_traces(ipg_ctx *ctx, const ipg_image *img, const ipg_params *p, const ipg_iharm_model *m)
{
  if (!ctx || !img || !p || !m || !p->trace) return IPG_E_ARG;
  const int single = p->trace_i >= 0 && p->trace_j >= 0;
  const int stride = p->trace_stride > 0 ? p->trace_stride : 1;
  const size_t nxt = single ? 1 : (size_t)p->nx / stride, nyt = single ? 1 : (size_t)p->ny / stride;
  if (nxt == 0 || nyt == 0) return IPG_E_ARG;
  int rc = IPG_OK;
  if (m->plugin.kind == IPG_PLUGIN_IHARM && m->trace_fields[0]) {
    rc = ipg_upload_trace_fields(ctx, (const double *const *)m->trace_fields);
    if (rc) return rc;
  }
  /* the traced pixels (traced, not interpolated) that main.c:865-879 picks */
  size_t cap = 16, np = 0;
  tr_pix *pix = (tr_pix *)calloc(cap, sizeof(tr_pix));
  const size_t max_rows = (size_t)p->maxnstep + 1;
  double *buf = (double *)malloc(max_rows * IPG_TRACE_DOUBLES * sizeof(double));
  if (!pix || !buf) {
    free(pix);
    free(buf);
    return IPG_E_NOMEM;
  }
  for (size_t i = 0; i < img->nx && rc == IPG_OK; i++)
    for (size_t j = 0; j < img->ny && rc == IPG_OK; j++) {
      if (img->interp_flag[i * img->ny + j]) continue;
      int ti, tj;
      if (single) {
        if ((int)i != p->trace_i || (int)j != p->trace_j) continue;
        ti = tj = 0;
      } else {
        if (i % stride || j % stride) continue;
        ti = (int)(i / stride);
        tj = (int)(j / stride);
        if ((size_t)ti >= nxt || (size_t)tj >= nyt) continue;
      }
      int32_t nstep = 0;
      rc = ipg_trace_ray(ctx, &img->cam, (int)i, (int)j, max_rows, buf, &nstep);
      if (rc) break;
      for (int s = nstep - 1; s > 0; --s) {
        int fl = (int)buf[(size_t)s * IPG_TRACE_DOUBLES + IPG_TRACE_FLAG];
        if (fl) printf("Flagged integration when tracing: %d\n", fl);
      }
      if (np == cap) {
        cap *= 2;
        pix = (tr_pix *)realloc(pix, cap * sizeof(tr_pix));
      }
      tr_pix *t = &pix[np++];
      t->ti = ti;
      t->tj = tj;
      t->nstep = nstep;
      t->rows = (double *)malloc(((size_t)nstep + 1) * IPG_TRACE_DOUBLES * sizeof(double));
      memcpy(t->rows, buf, ((size_t)nstep + 1) * IPG_TRACE_DOUBLES * sizeof(double));
    }
  free(buf);
  if (rc == IPG_OK && np) {
    /* an existing trace file keeps its pixels (hdf5_append) */
    ipgc_file f = {0};
    int have = ipgc_load(p->trace_outf, &f) == 0;
    if (!have) {
      memset(&f, 0, sizeof(f));
      ipg__write_header(&f, img, p);
    }
    size_t L = 0;
    for (size_t k = 0; k < np; k++)
      if ((size_t)pix[k].nstep + 1 > L) L = (size_t)pix[k].nstep + 1;
    const ipgc_entry *old = ipgc_find(&f, "/dl");
    size_t Lold = 0;
    if (old && old->rank == 3 && old->dims[0] == nxt && old->dims[1] == nyt) Lold = (size_t)old->dims[2];
    if (Lold > L) L = Lold;
    /* nstep */
    {
      int32_t *ns = (int32_t *)calloc(nxt * nyt, sizeof(int32_t));
      const ipgc_entry *e = ipgc_find(&f, "/nstep");
      if (e && e->kind == IPGC_I32 && e->rank == 2 && e->dims[0] == nxt && e->dims[1] == nyt)
        memcpy(ns, e->data, nxt * nyt * sizeof(int32_t));
      for (size_t k = 0; k < np; k++) ns[(size_t)pix[k].ti * nyt + pix[k].tj] = pix[k].nstep;
      uint64_t d2[2] = {nxt, nyt};
      ipgc_put(&f, "/nstep", IPGC_I32, 2, d2, ns, nxt * nyt * sizeof(int32_t));
      free(ns);
    }
    for (int q = 0; q < NSETS; q++) {
      const tr_set *s = &SETS[q];
      const size_t w = (size_t)s->width, per_pix = L * w;
      double *a = (double *)calloc(nxt * nyt * per_pix, sizeof(double));
      if (!a) {
        rc = IPG_E_NOMEM;
        break;
      }
      char path[64];
      snprintf(path, sizeof(path), "/%s", s->name);
      const ipgc_entry *e = ipgc_find(&f, path);
      if (e && e->kind == IPGC_F64 && e->rank == set_rank(s) && e->dims[0] == nxt && e->dims[1] == nyt &&
          Lold && e->dims[2] == Lold) {
        const double *src = (const double *)e->data;
        for (size_t c = 0; c < nxt * nyt; c++) memcpy(a + c * per_pix, src + c * Lold * w, Lold * w * sizeof(double));
      }
      for (size_t k = 0; k < np; k++) {
        double *dst = a + ((size_t)pix[k].ti * nyt + pix[k].tj) * per_pix;
        memset(dst, 0, per_pix * sizeof(double));
        for (size_t r = 0; r <= (size_t)pix[k].nstep; r++)
          memcpy(dst + r * w, pix[k].rows + r * IPG_TRACE_DOUBLES + s->col, w * sizeof(double));
      }
      uint64_t d[5];
      set_dims(s, nxt, nyt, L, d);
      ipgc_put(&f, path, IPGC_F64, set_rank(s), d, a, nxt * nyt * per_pix * sizeof(double));
      free(a);
    }
    if (rc == IPG_OK && ipgc_save(p->trace_outf, &f) != 0) {
      fprintf(stderr, "! %s\n", ipgc_error());
      rc = IPG_E_IO;
    }
    ipgc_free(&f);
  }
  for (size_t k = 0; k < np; k++) free(pix[k].rows);
  free(pix);
  return rc;
}
