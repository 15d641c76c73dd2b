/*
 * Batched image instances (ipg_render_batch): many images of one iharm dump
 * that differ in camera (inclination, frequency, resolution) and in the
 * electron model (M_unit, R_high, R_low, beta_crit), traced together.
 *
 * The reference renders one image per process (src/main.c:506-811); a set
 * of images is a set of runs.  Here the images of a batch share work where
 * the physics lets them:
 *
 *   - Instances whose cameras coincide (same position, tetrad, field of
 *     view, frequency, resolution and step control) form a camera group.
 *     Their geodesics are the same bits, so each pixel that any of them
 *     traces is integrated once (k_geodesic, CamTable: the group's camera is
 *     read from a constant table).  The fluid does not enter the geodesic.
 *   - The four-vectors (get_model_fourv: velocity and field primitives in
 *     code units), the k-B geometry, the fluid frequency and the plasma
 *     tetrad at a step depend only on the camera group, so the coefficient
 *     pass evaluates them once per step record; only the thermal fits, which
 *     read ne, Theta_e and |B|, run once per instance of the group that
 *     traces the pixel (k_coef_batch).
 *   - ne, Theta_e, |B| and sigma are derived on the device once per electron
 *     model, bit for bit as init_physical_quantities derives them on the
 *     host (model/iharm/model.c:610-717), and gathered like the single-image
 *     fields.
 *   - The transfer walks one lane per (instance, ray) over the shared
 *     records and the instance's coefficient block (k_xfer_batch).
 *
 * Each instance's image is therefore the single-image path's image, bit for
 * bit.  Included by ipg_kernels.cu (one translation unit holds the constant
 * banks).
 */

/* doubles of an instance's coefficient block: ju ku jI jQ jV aI aQ aV rQ rV */
#define IPG_BCOEF 10
/* instance slots of a camera group (a 32-bit mask per geodesic item) */
#define IPG_BATCH_MAX_SLOTS 32
static_assert(IPG_BATCH_MAX_SLOTS == IPG_BATCH_MAX_PER_CAMERA && IPG_BATCH_MAX_GROUPS == IPG_BATCH_MAX_CAMERAS,
              "the published batch limits are the constant tables' sizes");
/* derived-field set of each (camera group, instance slot) */
__constant__ int c_bslot_set[IPG_BATCH_MAX_GROUPS][IPG_BATCH_MAX_SLOTS];

/* ===================================================================== */
/* derived fields per electron model                                      */
/* ===================================================================== */
/* set_units (model/iharm/model.c:595-608) and the electron model
 * (ELECTRONS == 2, :647-654) of one instance */
struct DeriveSet {
  double RHO_unit, B_unit;
  double trat_large, trat_small, beta_crit;
  double gam, game, gamp;
};

/* |B| in G at interior cells: sqrt(b^2) (code units) times B_unit, the
 * product the host loader forms (f.b = sqrt(bsq) * B_unit) */
__global__ void k_bfield(const double *__restrict__ bcode, int n1, int n2, int n3, double B_unit, double *__restrict__ bb)
{
  const long long n = (long long)n1 * n2 * n3;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t / ((long long)n2 * n3)) + 1, j = (int)((t / n3) % n2) + 1, k = (int)(t % n3) + 1;
    size_t c = ((size_t)i * (n2 + 2) + j) * (n3 + 2) + k;
    bb[c] = __dmul_rn(bcode[c], B_unit);
  }
}

/* ghost zones of one field (populate_boundary_conditions,
 * model/iharm/model.c:1314-1370): radial copy, polar reflection across the
 * axis with a half turn in phi (the average of two cells for odd n3), then
 * periodic phi.  Three launches, in that order, as the passes read each
 * other's ghosts. */
__global__ void k_bc_radial(double *f, int n1, int n2, int n3)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n2 * n3) return;
  const int j = t / n3 + 1, k = t % n3 + 1;
  const size_t sj = n3 + 2, si = (size_t)(n2 + 2) * (n3 + 2);
  f[0 * si + j * sj + k] = f[1 * si + j * sj + k];
  f[(size_t)(n1 + 1) * si + j * sj + k] = f[(size_t)n1 * si + j * sj + k];
}

__global__ void k_bc_polar(double *f, int n1, int n2, int n3)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (n1 + 2) * n3) return;
  const int i = t / n3, k = t % n3 + 1;
  const size_t sj = n3 + 2, si = (size_t)(n2 + 2) * (n3 + 2);
  const size_t b = (size_t)i * si;
  if (n3 % 2 == 0) {
    const int kflip = ((k - 1) + (n3 / 2)) % n3 + 1;
    f[b + 0 * sj + k] = f[b + 1 * sj + kflip];
    f[b + (size_t)(n2 + 1) * sj + k] = f[b + (size_t)n2 * sj + kflip];
  } else {
    const int k1 = (k + (n3 / 2)) % n3, k2 = (k + (n3 / 2) + 1) % n3;
    f[b + 0 * sj + k] = __ddiv_rn(__dadd_rn(f[b + 1 * sj + k1], f[b + 1 * sj + k2]), 2.);
    f[b + (size_t)(n2 + 1) * sj + k] =
        __ddiv_rn(__dadd_rn(f[b + (size_t)n2 * sj + k1], f[b + (size_t)n2 * sj + k2]), 2.);
  }
}

__global__ void k_bc_phi(double *f, int n1, int n2, int n3)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (n1 + 2) * (n2 + 2)) return;
  const size_t row = (size_t)t * (n3 + 2);
  f[row + 0] = f[row + n3];
  f[row + n3 + 1] = f[row + 1];
}

/* ne, Theta_e, |B|, sigma per cell, cell-major (4 per cell), with the host
 * loader's operations in its order and rounding (no contraction):
 *   ne = rho RHO_unit / (MP + ME); bsq = (bb / B_unit)^2; sigma = bsq / rho;
 *   beta = u (gam - 1) / 0.5 / bsq; betasq = beta^2 / beta_crit^2;
 *   trat = R_high betasq / (1 + betasq) + R_low / (1 + betasq);
 *   Theta_e = (MP/ME) (game - 1) (gamp - 1) / ((gamp - 1) + (game - 1) trat) u / rho,
 *   floored at 1e-3; sigma floored at SMALL. */
__global__ void k_derive(const double *__restrict__ rho, const double *__restrict__ uu,
                         const double *__restrict__ bb, long long ncell, DeriveSet S, double *__restrict__ out)
{
  const double mpme = IPG_MP + IPG_ME, mp_me = IPG_MP / IPG_ME;
  const double gm1 = __dsub_rn(S.gam, 1.), gem1 = __dsub_rn(S.game, 1.), gpm1 = __dsub_rn(S.gamp, 1.);
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
       c += (long long)gridDim.x * blockDim.x) {
    const double r = rho[c], u = uu[c], b = bb[c];
    const double ne = __dmul_rn(__ddiv_rn(__dmul_rn(r, S.RHO_unit), mpme), 1.);
    double bsq = __ddiv_rn(b, S.B_unit);
    bsq = __dmul_rn(bsq, bsq);
    const double sigma_m = __ddiv_rn(bsq, r);
    const double beta_m = __ddiv_rn(__ddiv_rn(__dmul_rn(u, gm1), 0.5), bsq);
    const double betasq = __ddiv_rn(__ddiv_rn(__dmul_rn(beta_m, beta_m), S.beta_crit), S.beta_crit);
    const double opb = __dadd_rn(1., betasq);
    const double trat = __dadd_rn(__ddiv_rn(__dmul_rn(S.trat_large, betasq), opb), __ddiv_rn(S.trat_small, opb));
    const double th_u =
        __ddiv_rn(__dmul_rn(__dmul_rn(mp_me, gem1), gpm1), __dadd_rn(gpm1, __dmul_rn(gem1, trat)));
    double thetae = __ddiv_rn(__dmul_rn(th_u, u), r);
    thetae = fmax(thetae, 1.e-3);
    double2 *o = reinterpret_cast<double2 *>(out + 4 * c);
    o[0] = make_double2(ne, thetae);
    o[1] = make_double2(b, fmax(sigma_m, IPG_SMALL));
  }
}

/* ===================================================================== */
/* coefficient pass                                                       */
/* ===================================================================== */
/* One thread per stored step of a finished geodesic item: the radiating
 * test, the four-vectors and the plasma tetrad once (shared by the camera
 * group), then the thermal coefficients for every instance slot of the
 * group that traces the pixel, each from its own derived fields.  The
 * shared part goes into the record in place (flags, tetrad rows; dl and
 * nturns keep their slots), the instances' coefficients into their blocks
 * of the side pool: side[((chunk * 32 + slot) * G + k) * IPG_BCOEF]. */
/* the shared part of a record in the compact layout (IPG_RECORDS_MIXED):
 * flags, dl and nturns in the coefficient block, the tetrad rows in FP32
 * over the geodesic state (read before) */
__device__ __forceinline__ void store_shared_m(double *p, int flags, double dl, double nturns, const double e1[4],
                                               const double e2[4], const double a[4], const double b[4])
{
  double *q = p + RECM_COEF;
  store4(q, (double)flags, 0., 0., dl);
  store4(q + 4, 0., 0., 0., 0.);
  store4(q + 8, 0., 0., nturns, 0.);
  store4(q + 12, 0., 0., 0., 0.);
  float4 *t = reinterpret_cast<float4 *>(reinterpret_cast<float *>(p) + RECM_TETF);
  t[0] = make_float4((float)e1[0], (float)e1[1], (float)e1[2], (float)e1[3]);
  t[1] = make_float4((float)e2[0], (float)e2[1], (float)e2[2], (float)e2[3]);
  t[2] = make_float4((float)a[0], (float)a[1], (float)a[2], (float)a[3]);
  t[3] = make_float4((float)b[0], (float)b[1], (float)b[2], (float)b[3]);
}

#ifndef IPG_BCOEF_MINB
#define IPG_BCOEF_MINB IPG_COEF_MINB /* blocks of 128 per SM the batch's coefficient pass is compiled for */
#endif
template <int EM, bool F32 = false, bool RM = false>
__global__ void __launch_bounds__(128, IPG_BCOEF_MINB)
    k_coef_batch(double *__restrict__ pool, double *__restrict__ side, int G, const int2 *__restrict__ chunk_meta,
                 const unsigned long long *__restrict__ counters, long long n_chunks, const RayRec *__restrict__ rays,
                 const int32_t *__restrict__ geo_grp, const uint32_t *__restrict__ geo_mask,
                 const double *__restrict__ fourv, const double *__restrict__ sets, long long ncell,
                 long long c_first)
{
  const DevGrid &Gd = c_grid;
  long long used = (long long)counters[CNT_POOL];
  if (used > n_chunks) used = n_chunks;
  const long long total = used * IPG_CHUNK_STEPS;
  for (long long t = c_first * IPG_CHUNK_STEPS + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int c = (int)(t / IPG_CHUNK_STEPS), slot = (int)(t % IPG_CHUNK_STEPS);
    int2 meta = chunk_meta[c];
    if (meta.x < 0) continue;
    RayRec rec = rays[meta.x];
    int s = meta.y + slot;
    if (rec.status != IPG_RAY_OK || s > rec.nstep) continue;
    const int g = geo_grp[meta.x];
    const DevCam &C = c_cams[g];
    const int pol = !C.unpol;
    double *p = step_ptr(pool, c, slot);
    double X1 = p[REC_X1], X2 = p[REC_X2], X3 = p[REC_X3];
    double K[4];
    load4(p + REC_K, K);
    /* RM: dl and nturns move out of the geodesic state, which the compact
     * tetrad rows overwrite */
    const double dl_rec = RM ? p[REC_DL] : 0., nturns_rec = RM ? p[REC_NTURNS] : 0.;
    PointGeo pg;
    point_geo<IPG_MET_FMKS>(X1, X2, &pg);
    int flags = radiating_t<IPG_PLUG_IHARM>(pg) ? 1 : 0;
    /* isolate_counterjet, src/ipolarray.c:128-136 */
    if (C.counterjet == 1) {
      if (X2 < (Gd.cstopx[2] - Gd.cstartx[2]) / 2) flags |= 2;
    } else if (C.counterjet == 2) {
      if (X2 > (Gd.cstopx[2] - Gd.cstartx[2]) / 2) flags |= 2;
    }
    if (!((flags & 1) || s == rec.nstep)) {
      /* no coefficients here: the transfer reads only the flags */
      if constexpr (RM) {
        const double z[4] = {0., 0., 0., 0.};
        store_shared_m(p, flags, dl_rec, nturns_rec, z, z, z, z);
        continue;
      }
      p[REC_FLAGS] = (double)flags;
      store4(p + REC_E1COV, 0., 0., 0., 0.);
      store4(p + REC_E2COV, 0., 0., 0., 0.);
      store4(p + REC_E1CON, 0., 0., 0., 0.);
      store4(p + REC_E2CON, 0., 0., 0., 0.);
      continue;
    }
    ModelPt mp;
    mp.geo = pg;
    mp.gu = gcon_from(pg.r, pg.sth, pg.cth, pg.J21, pg.J22);
    mp.in_domain = in_grid(X1, X2);
    GridLoc gl;
    if (!mp.in_domain) {
      outside_point(&mp);
    } else {
      grid_locate(X1, X2, X3, &gl);
      double a6[6];
      gather_cells<6>(fourv, gl, a6);
      fourv_from(a6[0], a6[1], a6[2], a6[3], a6[4], a6[5], &mp);
    }
    const int want_pol = pol && (flags & 1);
    {
      double e1[4] = {0., 0., 0., 0.}, e2[4] = {0., 0., 0., 0.}, Econ[4][4];
#pragma unroll
      for (int q = 0; q < 4; q++) Econ[1][q] = Econ[2][q] = 0.;
      if (want_pol) {
        double Bcon[4] = {mp.Bcon[0], mp.Bcon[1], mp.Bcon[2], mp.Bcon[3]};
        double bsq = Bcon[0] * mp.Bcov[0] + Bcon[1] * mp.Bcov[1] + Bcon[2] * mp.Bcov[2] + Bcon[3] * mp.Bcov[3];
        if (bsq <= 0.) {
          Bcon[0] = 0.;
          Bcon[1] = 1.;
          Bcon[2] = 1.;
          Bcon[3] = 1.;
        }
        int tf = plasma_tetrad<IPG_MET_FMKS>(mp.Ucon, K, Bcon, mp.geo.g, mp.geo, Econ, e1, e2);
        if (isnan(mp.Ucov[0])) tf |= 8;
        flags |= tf << 2;
      }
      /* the shared part first: the tetrad is dead before the slot loop */
      if constexpr (RM) {
        store_shared_m(p, flags, dl_rec, nturns_rec, e1, e2, Econ[1], Econ[2]);
      } else {
        p[REC_FLAGS] = (double)flags;
        store4(p + REC_E1COV, e1[0], e1[1], e1[2], e1[3]);
        store4(p + REC_E2COV, e2[0], e2[1], e2[2], e2[3]);
        store4(p + REC_E1CON, Econ[1][0], Econ[1][1], Econ[1][2], Econ[1][3]);
        store4(p + REC_E2CON, Econ[2][0], Econ[2][1], Econ[2][2], Econ[2][3]);
      }
    }
    double *q0 = side + ((size_t)c * IPG_CHUNK_STEPS + slot) * G * IPG_BCOEF;
    for (uint32_t m = geo_mask[meta.x]; m; m &= m - 1) {
      const int k = __ffs(m) - 1;
      if (mp.in_domain) {
        const double *fs = sets + (size_t)c_bslot_set[g][k] * ncell * 4;
        double d4[4];
        gather_cells<4>(fs, gl, d4);
        mp.ne = sigma_cut_ne(d4[0], d4[3]);
        mp.thetae = d4[1];
        mp.bmag = d4[2];
      }
      double ju = 0., ku = 0.;
      Jar jar;
      coeffs_t<IPG_PLUG_IHARM, F32>(mp, K, want_pol, EM, &ju, &ku, &jar);
      double2 *q2 = reinterpret_cast<double2 *>(q0 + (size_t)k * IPG_BCOEF);
      q2[0] = make_double2(ju, ku);
      q2[1] = make_double2(jar.jI, jar.jQ);
      q2[2] = make_double2(jar.jV, jar.aI);
      q2[3] = make_double2(jar.aQ, jar.aV);
      q2[4] = make_double2(jar.rQ, jar.rV);
    }
  }
}

/* ===================================================================== */
/* transfer                                                               */
/* ===================================================================== */
/* the coefficient block of one step: the shared record's flags, dl,
 * nturns and tetrad rows with the instance's coefficients */
__device__ __forceinline__ void load_coef_b(const double *__restrict__ p, const double *__restrict__ q, CoefBlock &c)
{
  const double2 *r = reinterpret_cast<const double2 *>(p + REC_FLAGS);
  double2 h0 = r[0], h1 = r[1];
  c.flags = h0.x;
  c.dl = h1.y;
  c.nturns = p[REC_NTURNS];
  const double2 *te = reinterpret_cast<const double2 *>(p + REC_E1COV);
  double2 v[8];
#pragma unroll
  for (int k = 0; k < 8; k++) v[k] = te[k];
  c.e1[0] = v[0].x; c.e1[1] = v[0].y; c.e1[2] = v[1].x; c.e1[3] = v[1].y;
  c.e2[0] = v[2].x; c.e2[1] = v[2].y; c.e2[2] = v[3].x; c.e2[3] = v[3].y;
  c.a[0] = v[4].x; c.a[1] = v[4].y; c.a[2] = v[5].x; c.a[3] = v[5].y;
  c.b[0] = v[6].x; c.b[1] = v[6].y; c.b[2] = v[7].x; c.b[3] = v[7].y;
  const double2 *b2 = reinterpret_cast<const double2 *>(q);
  double2 w[5];
#pragma unroll
  for (int k = 0; k < 5; k++) w[k] = b2[k];
  c.ju = w[0].x;
  c.ku = w[0].y;
  c.jI = w[1].x;
  c.jQ = w[1].y;
  c.jV = w[2].x;
  c.aI = w[2].y;
  c.aQ = w[3].x;
  c.aV = w[3].y;
  c.rQ = w[4].x;
  c.rV = w[4].y;
}
static_assert(REC_FLAGS % 2 == 0 && REC_DL == REC_FLAGS + 3 && REC_E1COV % 2 == 0 && REC_E2CON == REC_E1COV + 12,
              "load_coef_b follows the record layout");

/* the same from a compact shared record (store_shared_m) */
__device__ __forceinline__ void load_coef_bm(const double *__restrict__ p, const double *__restrict__ q, CoefBlock &c)
{
  const double2 *r = reinterpret_cast<const double2 *>(p + RECM_COEF);
  const double2 h0 = r[0], h1 = r[1], h5 = r[5];
  c.flags = h0.x;
  c.dl = h1.y;
  c.nturns = h5.x;
  const float4 *t = reinterpret_cast<const float4 *>(reinterpret_cast<const float *>(p) + RECM_TETF);
  float4 w[4];
#pragma unroll
  for (int k = 0; k < 4; k++) w[k] = t[k];
  c.e1[0] = w[0].x; c.e1[1] = w[0].y; c.e1[2] = w[0].z; c.e1[3] = w[0].w;
  c.e2[0] = w[1].x; c.e2[1] = w[1].y; c.e2[2] = w[1].z; c.e2[3] = w[1].w;
  c.a[0] = w[2].x; c.a[1] = w[2].y; c.a[2] = w[2].z; c.a[3] = w[2].w;
  c.b[0] = w[3].x; c.b[1] = w[3].y; c.b[2] = w[3].z; c.b[3] = w[3].w;
  const double2 *b2 = reinterpret_cast<const double2 *>(q);
  double2 v[5];
#pragma unroll
  for (int k = 0; k < 5; k++) v[k] = b2[k];
  c.ju = v[0].x;
  c.ku = v[0].y;
  c.jI = v[1].x;
  c.jQ = v[1].y;
  c.jV = v[2].x;
  c.aI = v[2].y;
  c.aQ = v[3].x;
  c.aV = v[3].y;
  c.rQ = v[4].x;
  c.rV = v[4].y;
}

struct XbLane {
  HermN N;
  const double *rec_i;
  double dl_i, nturns_i;
  double I, tau, tauF, js, ks;
  int item, geo, grp, kslot, n, chunk, flag, nrad, cprev;
};

__device__ __forceinline__ const double *side_ptr(const double *side, int G, int chunk, int slot, int k)
{
  return side + (((size_t)chunk * IPG_CHUNK_STEPS + slot) * G + k) * IPG_BCOEF;
}

/* next (instance, ray) item whose geodesic is complete; items whose
 * geodesic was deferred go to the next wave's list; after the step budget
 * is spent no new item starts */
template <bool RM>
__device__ __forceinline__ bool xb_fetch(XbLane &L, const int32_t *__restrict__ list, int n_list,
                                         const double *__restrict__ pool, const double *__restrict__ side, int G,
                                         const int *__restrict__ chunk_prev, const RayRec *__restrict__ rays,
                                         const int32_t *__restrict__ xf_geo, const int32_t *__restrict__ xf_slot,
                                         const int32_t *__restrict__ geo_grp, ipg_pixel_out *__restrict__ out,
                                         unsigned long long *__restrict__ counters, int32_t *__restrict__ xdeferred)
{
  while (true) {
    const unsigned long long budget = counters[CNT_BUDGET];
    if (budget && *(volatile unsigned long long *)&counters[CNT_XSTEPS] +
                          *(volatile unsigned long long *)&counters[CNT_STEPS] >=
                      budget) {
      counters[CNT_TIMEOUT] = 1;
      return false;
    }
    unsigned long long t = atomicAdd(&counters[CNT_NEXT_T], 1ULL);
    if (t >= (unsigned long long)n_list) return false;
    const int item = list ? list[t] : (int)t;
    const int geo = xf_geo[item];
    RayRec rec = rays[geo];
    if (rec.status == IPG_RAY_POOL_FULL) {
      xdeferred[atomicAdd(&counters[CNT_XDEFER], 1ULL)] = item;
      continue;
    }
    if (rec.status == IPG_RAY_MAXNSTEP) {
      ipg_pixel_out o;
      o.I_unpol = o.tau = o.tauF = o.I = o.Q = o.U = o.V = 0.;
      o.nstep = rec.nstep;
      o.flag = 0;
      out[item] = o;
      continue;
    }
    L.item = item;
    L.geo = geo;
    L.grp = geo_grp[geo];
    L.kslot = xf_slot[item];
    L.n = rec.nstep;
    L.chunk = rec.last_chunk;
    L.rec_i = step_ptr(const_cast<double *>(pool), L.chunk, L.n % IPG_CHUNK_STEPS);
    L.cprev = chunk_prev[L.chunk];
    prefetch_rec<RM>(L.rec_i);
    /* get_jkinv at the far end of the ray, src/ipolarray.c:74 */
    const double *q = side_ptr(side, G, L.chunk, L.n % IPG_CHUNK_STEPS, L.kslot);
    L.js = q[0];
    L.ks = q[1];
    L.dl_i = L.rec_i[RM ? RECM_COEF + 3 : REC_DL];
    L.nturns_i = L.rec_i[RM ? RECM_COEF + 10 : REC_NTURNS];
    L.I = L.tau = L.tauF = 0.;
    hn_zero(&L.N);
    L.flag = 0;
    L.nrad = 0;
    return true;
  }
}

template <int TPB, bool S32, bool RM = false>
__global__ void __launch_bounds__(TPB, 1)
    k_xfer_batch(const int32_t *__restrict__ list, int n_list, const double *__restrict__ pool,
                 const double *__restrict__ side, int G, const int *__restrict__ chunk_prev,
                 const RayRec *__restrict__ rays, const int32_t *__restrict__ xf_geo,
                 const int32_t *__restrict__ xf_slot, const int32_t *__restrict__ geo_grp,
                 ipg_pixel_out *__restrict__ out, unsigned long long *__restrict__ counters,
                 int32_t *__restrict__ xdeferred)
{
  XbLane L;
  bool has = xb_fetch<RM>(L, list, n_list, pool, side, G, chunk_prev, rays, xf_geo, xf_slot, geo_grp, out, counters,
                      xdeferred);
  while (__any_sync(0xffffffffu, has)) {
    if (!has) continue;
    const DevCam &C = c_cams[L.grp];
    const int unpol = C.unpol;
    if (L.n == 0) {
      ipg_pixel_out o;
      const int nstep = rays[L.geo].nstep;
      xfer_result(C, L, unpol, nstep, &o);
      out[L.item] = o;
      atomicAdd(&counters[CNT_RAD], (unsigned long long)L.nrad);
      atomicAdd(&counters[CNT_XSTEPS], (unsigned long long)nstep);
      has = xb_fetch<RM>(L, list, n_list, pool, side, G, chunk_prev, rays, xf_geo, xf_slot, geo_grp, out, counters,
                     xdeferred);
      continue;
    }
    /* step n -> n-1 of integrate_emission's loop, src/ipolarray.c:78-244 */
    int s = L.n - 1;
    if (s % IPG_CHUNK_STEPS == IPG_CHUNK_STEPS - 1) {
      L.chunk = L.cprev;
      L.cprev = chunk_prev[L.chunk];
    }
    const double *rec_f = step_ptr(const_cast<double *>(pool), L.chunk, s % IPG_CHUNK_STEPS);
    if (s >= 1) {
      if ((s - 1) % IPG_CHUNK_STEPS != IPG_CHUNK_STEPS - 1) prefetch_rec<RM>(rec_f - IPG_STEP_DOUBLES);
      else if (L.cprev >= 0) prefetch_rec<RM>(step_ptr(const_cast<double *>(pool), L.cprev, IPG_CHUNK_STEPS - 1));
    }
    CoefBlock cb;
    if constexpr (RM)
      load_coef_bm(rec_f, side_ptr(side, G, L.chunk, s % IPG_CHUNK_STEPS, L.kslot), cb);
    else
      load_coef_b(rec_f, side_ptr(side, G, L.chunk, s % IPG_CHUNK_STEPS, L.kslot), cb);
    xfer_step<S32, RM ? 1 : 0>(C, L, cb, unpol);
    L.dl_i = cb.dl;
    L.nturns_i = cb.nturns;
    L.rec_i = rec_f;
    L.n--;
  }
}

/* all pending geodesic items start the wave marked deferred: items past the
 * wave's share of the list then read as deferred to the transfer */
__global__ void k_mark_pending(const int32_t *__restrict__ list, int n, RayRec *__restrict__ rays)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) {
    RayRec r = {-1, 0, IPG_RAY_POOL_FULL, 0};
    rays[list ? list[t] : t] = r;
  }
}

__global__ void k_iota(int32_t *list, int n, int first)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) list[t] = first + t;
}

/* chunks [0, n) of the pool have no owner: the coefficient pass skips them
 * (the longest class's range, of which its geodesics use a part) */
__global__ void k_meta_clear(int2 *__restrict__ chunk_meta, long long n)
{
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    chunk_meta[c] = make_int2(-1, 0);
}

/* the longest class's geodesic records become visible to the coefficient
 * and transfer passes */
__global__ void k_rider_merge(const int32_t *__restrict__ items, int n, const RayRec *__restrict__ from,
                              RayRec *__restrict__ to)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) to[items[t]] = from[items[t]];
}

/* ===================================================================== */
/* host side                                                              */
/* ===================================================================== */
/* device copy of a batch model: the velocity and field primitives
 * cell-major for the shared gather, rho and u for the derivation */
struct BatchModel {
  double *fourv;    /* 6 per cell: U1 U2 U3 B1 B2 B3 */
  double *rho, *uu; /* per cell (ghost zones filled) */
  double *bcode;    /* sqrt(b^2) in code units (interior cells) */
  double *bb;       /* scratch: |B| of one set */
  double *sets;     /* derived fields, 4 per cell per set */
  int nsets_cap;
  size_t ncell;
  int n1, n2, n3;
  double gam, game, gamp;
  DevGrid dg;
  int have;
};

/* work arrays of one traced batch level (sized by its item counts) */
struct BatchWs {
  size_t cap_geo, cap_xf;
  RayRec *rays;      /* per geodesic item */
  int32_t *glist[2]; /* wave lists of geodesic items */
  int32_t *xlist[2]; /* wave lists of transfer items */
  unsigned long long *cnt;
  /* the longest class's own queue and counters (first wave) and its
   * deferred items */
  unsigned long long *cnt_long;
  int32_t *gdef_long;
  RayRec *rays_long; /* per geodesic item, written by the longest class's geodesics */
};

struct BatchState {
  BatchModel m;
  BatchWs w;
  int G; /* instance slots per group of the current batch */
  int emission_type, step32, unpol, rec_mixed;
  int xfer_threads; /* transfer block size (128 or 256) */
  /* the transfer block size is tuned per batch shape (slots per group,
   * groups): the first call of a shape runs 128 threads, the second 256,
   * and later calls keep the one whose transfer took less time per
   * transfer item (the images do not depend on it: one lane per item) */
  int tune_G, tune_ngrp, tune_calls;
  double tune_ms[2], tune_items[2], call_xfer_ms, call_items;
};

static void batch_ws_free(BatchWs *w)
{
  cudaFree(w->rays);
  cudaFree(w->glist[0]);
  cudaFree(w->glist[1]);
  cudaFree(w->xlist[0]);
  cudaFree(w->xlist[1]);
  cudaFree(w->cnt);
  cudaFree(w->cnt_long);
  cudaFree(w->gdef_long);
  cudaFree(w->rays_long);
  memset(w, 0, sizeof(*w));
}

static void batch_model_free(BatchModel *m)
{
  cudaFree(m->fourv);
  cudaFree(m->rho);
  cudaFree(m->uu);
  cudaFree(m->bcode);
  cudaFree(m->bb);
  cudaFree(m->sets);
  memset(m, 0, sizeof(*m));
}

static BatchState *batch_state(ipg_ctx *ctx)
{
  if (!ctx->batch) ctx->batch = (BatchState *)calloc(1, sizeof(BatchState));
  return ctx->batch;
}

static void batch_release(ipg_ctx *ctx)
{
  if (!ctx->batch) return;
  batch_model_free(&ctx->batch->m);
  batch_ws_free(&ctx->batch->w);
  free(ctx->batch);
  ctx->batch = NULL;
}

extern "C" int ipg_upload_iharm_batch(ipg_ctx *ctx, const ipg_grid *g, const double *const prims[IPG_NBPRIM],
                                      double gam, double game, double gamp)
{
  if (!ctx || !g || !prims || g->n1 <= 0 || g->n2 <= 0 || g->n3 <= 0) return IPG_E_ARG;
  for (int f = 0; f < IPG_NBPRIM; f++)
    if (!prims[f]) return IPG_E_ARG;
  if (g->metric != IPG_METRIC_FMKS) {
    snprintf(ctx->err, sizeof(ctx->err), "an iharm dump needs the FMKS metric (%d), grid has %d", IPG_METRIC_FMKS,
             g->metric);
    return IPG_E_ARG;
  }
  BatchState *B = batch_state(ctx);
  if (!B) return IPG_E_NOMEM;
  CK(cudaSetDevice(ctx->device));
  BatchModel &M = B->m;
  const size_t ncell = (size_t)(g->n1 + 2) * (g->n2 + 2) * (g->n3 + 2);
  if (M.ncell != ncell) {
    batch_model_free(&M);
    CK(cudaMalloc(&M.fourv, ncell * 6 * sizeof(double)));
    CK(cudaMalloc(&M.rho, ncell * sizeof(double)));
    CK(cudaMalloc(&M.uu, ncell * sizeof(double)));
    CK(cudaMalloc(&M.bcode, ncell * sizeof(double)));
    CK(cudaMalloc(&M.bb, ncell * sizeof(double)));
    M.ncell = ncell;
  }
  /* velocity and field primitives cell-major, as the single-image fields */
  std::vector<double> aos(ncell * 6);
  for (size_t c = 0; c < ncell; c++)
    for (int f = 0; f < 6; f++) aos[c * 6 + f] = prims[IPG_BP_U1 + f][c];
  CK(cudaMemcpy(M.fourv, aos.data(), ncell * 6 * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(M.rho, prims[IPG_BP_RHO], ncell * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(M.uu, prims[IPG_BP_UU], ncell * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(M.bcode, prims[IPG_BP_BMAG], ncell * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemset(M.bb, 0, ncell * sizeof(double)));
  M.n1 = g->n1;
  M.n2 = g->n2;
  M.n3 = g->n3;
  M.gam = gam;
  M.game = game;
  M.gamp = gamp;
  devgrid_from(g, &M.dg);
  M.have = 1;
  return IPG_OK;
}

/* Set-up of a batch: the camera table, the slot -> derived-set table and the
 * derived fields of every electron model.  Enqueued on the context's
 * stream. */
extern "C" int ipg__batch_begin(ipg_ctx *ctx, const ipg_camera *grp_cam, int ngrp, const int *slot_set, int G,
                                const ipg_electrons *sets, int nsets, int step32)
{
  BatchState *B = ctx->batch;
  if (!B || !B->m.have) return IPG_E_STATE;
  if (ngrp < 1 || ngrp > IPG_BATCH_MAX_GROUPS || G < 1 || G > IPG_BATCH_MAX_SLOTS || nsets < 1) return IPG_E_ARG;
  BatchModel &M = B->m;
  CK(cudaSetDevice(ctx->device));
  int em = grp_cam[0].emission_type, unpol = grp_cam[0].only_unpolarized;
  if (em != 4 && em != 1) {
    snprintf(ctx->err, sizeof(ctx->err), "emission_type %d not supported by batches (thermal types 1 and 4)", em);
    return IPG_E_ARG;
  }
  std::vector<DevCam> dcs(ngrp);
  for (int g = 0; g < ngrp; g++) {
    if (grp_cam[g].emission_type != em || grp_cam[g].only_unpolarized != unpol) {
      snprintf(ctx->err, sizeof(ctx->err), "the instances of a batch share emission_type and -unpol");
      return IPG_E_ARG;
    }
    if (grp_cam[g].maxnstep < 2 || grp_cam[g].nx <= 0 || grp_cam[g].ny <= 0) return IPG_E_ARG;
    make_devcam(&grp_cam[g], &dcs[g]);
    dcs[g].mixed = ctx->rec_mixed; /* the shared records' layout (the coefficient blocks stay FP64) */
  }
  int rc = ensure_pool(ctx);
  if (rc) return rc;
  /* derived fields, one set per electron model */
  if (M.nsets_cap < nsets) {
    cudaFree(M.sets);
    M.sets = NULL;
    M.nsets_cap = 0;
    CK(cudaMalloc(&M.sets, (size_t)nsets * M.ncell * 4 * sizeof(double)));
    M.nsets_cap = nsets;
  }
  cudaStream_t st = ctx->stream;
  const int n1 = M.n1, n2 = M.n2, n3 = M.n3;
  const int gridN = 4 * ctx->n_sm;
  for (int s = 0; s < nsets; s++) {
    k_bfield<<<gridN, 256, 0, st>>>(M.bcode, n1, n2, n3, sets[s].B_unit, M.bb);
    k_bc_radial<<<(n2 * n3 + 255) / 256, 256, 0, st>>>(M.bb, n1, n2, n3);
    k_bc_polar<<<((n1 + 2) * n3 + 255) / 256, 256, 0, st>>>(M.bb, n1, n2, n3);
    k_bc_phi<<<((n1 + 2) * (n2 + 2) + 255) / 256, 256, 0, st>>>(M.bb, n1, n2, n3);
    DeriveSet S = {sets[s].RHO_unit, sets[s].B_unit, sets[s].trat_large, sets[s].trat_small, sets[s].beta_crit,
                   M.gam, M.game, M.gamp};
    k_derive<<<gridN, 256, 0, st>>>(M.rho, M.uu, M.bb, (long long)M.ncell, S, M.sets + (size_t)s * M.ncell * 4);
    CK(cudaGetLastError());
  }
  std::vector<int> tab((size_t)IPG_BATCH_MAX_GROUPS * IPG_BATCH_MAX_SLOTS, 0);
  for (int g = 0; g < ngrp; g++)
    for (int k = 0; k < G; k++) tab[(size_t)g * IPG_BATCH_MAX_SLOTS + k] = slot_set[g * G + k];
  CK(cudaMemcpyToSymbolAsync(c_grid, &M.dg, sizeof(DevGrid), 0, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyToSymbolAsync(c_cams, dcs.data(), ngrp * sizeof(DevCam), 0, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyToSymbolAsync(c_bslot_set, tab.data(), tab.size() * sizeof(int), 0, cudaMemcpyHostToDevice, st));
  B->G = G;
  B->emission_type = em;
  B->unpol = unpol;
  B->step32 = step32;
  B->rec_mixed = ctx->rec_mixed;
  /* block-size tuning: close the previous call's sample, pick this call's */
  if (B->tune_calls > 0 && B->tune_calls <= 2 && B->call_items > 0) {
    B->tune_ms[B->tune_calls - 1] = B->call_xfer_ms;
    B->tune_items[B->tune_calls - 1] = B->call_items;
  }
  if (G != B->tune_G || ngrp != B->tune_ngrp) {
    B->tune_G = G;
    B->tune_ngrp = ngrp;
    B->tune_calls = 0;
  }
  if (B->tune_calls < 2) {
    B->xfer_threads = B->tune_calls == 0 ? 128 : 256;
  } else if (B->tune_calls == 2) {
    const double r128 = B->tune_ms[0] / fmax(B->tune_items[0], 1.), r256 = B->tune_ms[1] / fmax(B->tune_items[1], 1.);
    B->xfer_threads = r256 < r128 ? 256 : 128;
  }
  if (B->tune_calls <= 2) B->tune_calls++;
  B->call_xfer_ms = 0.;
  B->call_items = 0.;
  memset(&ctx->stats, 0, sizeof(ctx->stats));
  return IPG_OK;
}

static int batch_ws_reserve(ipg_ctx *ctx, BatchWs &w, size_t n_geo, size_t n_xf)
{
  if (!w.cnt) CK(cudaMalloc(&w.cnt, CNT_NB * sizeof(unsigned long long)));
  if (!w.cnt_long) CK(cudaMalloc(&w.cnt_long, CNT_NB * sizeof(unsigned long long)));
  if (w.cap_geo < n_geo) {
    cudaFree(w.rays);
    cudaFree(w.glist[0]);
    cudaFree(w.glist[1]);
    cudaFree(w.gdef_long);
    cudaFree(w.rays_long);
    w.gdef_long = nullptr;
    w.rays_long = nullptr;
    w.cap_geo = 0;
    CK(cudaMalloc(&w.rays, n_geo * sizeof(RayRec)));
    CK(cudaMalloc(&w.glist[0], n_geo * sizeof(int32_t)));
    CK(cudaMalloc(&w.glist[1], n_geo * sizeof(int32_t)));
    CK(cudaMalloc(&w.gdef_long, n_geo * sizeof(int32_t)));
    CK(cudaMalloc(&w.rays_long, n_geo * sizeof(RayRec)));
    w.cap_geo = n_geo;
  }
  if (w.cap_xf < n_xf) {
    cudaFree(w.xlist[0]);
    cudaFree(w.xlist[1]);
    w.cap_xf = 0;
    CK(cudaMalloc(&w.xlist[0], n_xf * sizeof(int32_t)));
    CK(cudaMalloc(&w.xlist[1], n_xf * sizeof(int32_t)));
    w.cap_xf = n_xf;
  }
  return IPG_OK;
}

#define IPG_LAUNCH_XB(TPB, S32, RMC)                                                                                  \
  do {                                                                                                          \
    int tb = grid_blocks(ctx, (const void *)k_xfer_batch<TPB, S32, RMC>, TPB, pend_x);                               \
    k_xfer_batch<TPB, S32, RMC><<<tb, TPB, 0, st>>>(xl, (int)pend_x, pool, side, G, ctx->d_chunk_prev, W.rays,      \
                                                it->xf_geo, it->xf_slot, it->geo_grp, it->xf_out, W.cnt, xnext); \
  } while (0)

/* Trace one level of a batch: every geodesic item once, then its step
 * records' coefficients for the instance slots that trace it, then every
 * (instance, ray) transfer item.  Waves as in the single-image trace: items
 * whose geodesic finds the pool full are deferred with their transfer
 * items.  The pool is shared out per chunk of 32 steps as the 32 shared
 * records (512 B each) and the G instance blocks of each (80 B each).
 *
 * The longest predicted class (items->n_long, the head of the sorted order)
 * rides beside the waves.  Started in a wave with the others, its rays, in
 * flight the longest, are the ones the full pool defers, and their walks,
 * at a lone ray's step latency, then set the last wave's geodesic time.
 * Instead its geodesics start at once on the context's stream, in a pool
 * range [0, cl) reserved for them and in blocks of 256 lanes (their
 * registers fill an SM, so these rays get SMs of their own).  The waves run
 * the other items on a second stream, allocating from cl up.  The class
 * joins the first wave that starts after its geodesics end (or the wave that
 * has no other geodesics left, which waits for them): that wave's
 * coefficient pass covers the range too, and its transfer takes the class's
 * transfer items, which read as deferred until then. */
struct BatchRider {
  size_t nl;     /* items in the class (0: none) */
  long long cl;  /* its pool range [0, cl) */
  bool launched, merged;
};

static int batch_waves(ipg_ctx *ctx, const ipg_batch_items *it, unsigned long long *steps_left, BatchRider &R)
{
  BatchState *B = ctx->batch;
  BatchWs &W = B->w;
  const int G = B->G;
  const size_t rec_bytes = (size_t)IPG_CHUNK_STEPS * IPG_STEP_DOUBLES * sizeof(double);
  const size_t side_bytes = (size_t)IPG_CHUNK_STEPS * G * IPG_BCOEF * sizeof(double);
  const long long n_chunks = (long long)(((size_t)ctx->n_chunks * rec_bytes) / (rec_bytes + side_bytes));
  if (n_chunks < 16) return IPG_E_NOMEM;
  double *pool = ctx->d_pool;
  double *side = ctx->d_pool + (size_t)n_chunks * IPG_CHUNK_STEPS * IPG_STEP_DOUBLES;
  const int threads = 128;
  const void *geo_fn = (const void *)k_geodesic<IPG_PLUG_IHARM, 256, IPG_GEO_MINB, false, CamTable>;
  cudaStream_t st = ctx->stream; /* the waves */
  size_t pend_g = it->n_geo, pend_x = it->n_xf;
  const int32_t *gl = it->geo_order, *xl = it->xf_order;
  /* only where the items take more than one wave: in a wave that holds them
   * all, the class's transfer overlaps the others' instead of following it */
  if (ctx->split && it->geo_order && it->n_long > 0 && it->n_long < it->n_geo &&
      it->pred_steps > (double)n_chunks * IPG_CHUNK_STEPS) {
    /* its predicted steps with the single image's 15% margin */
    const long long cl = (long long)(it->long_steps * 1.15 / IPG_CHUNK_STEPS) + (long long)it->n_long + 16;
    if (cl <= n_chunks / 2) {
      R.nl = it->n_long;
      R.cl = cl;
    }
  }
  if (R.nl) {
    cudaStream_t sr = ctx->stream;
    const int nl = (int)R.nl;
    unsigned long long hl0[CNT_NB];
    memset(hl0, 0, sizeof(hl0));
    hl0[CNT_BUDGET] = steps_left ? *steps_left : 0;
    CK(cudaMemcpyAsync(W.cnt_long, hl0, sizeof(hl0), cudaMemcpyHostToDevice, sr));
    k_meta_clear<<<4 * ctx->n_sm, 256, 0, sr>>>(ctx->d_chunk_meta, R.cl);
    k_mark_pending<<<(nl + 255) / 256, 256, 0, sr>>>(it->geo_order, nl, W.rays);
    k_mark_pending<<<(nl + 255) / 256, 256, 0, sr>>>(it->geo_order, nl, W.rays_long);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->bev[0][2], sr));
    int lb = grid_blocks(ctx, geo_fn, 256, R.nl);
    if (lb > IPG_STARTED_MAX) lb = IPG_STARTED_MAX;
    memset(ctx->h_started, 0, IPG_STARTED_MAX * sizeof(int));
    k_geodesic<IPG_PLUG_IHARM, 256, IPG_GEO_MINB, false, CamTable><<<lb, 256, 0, sr>>>(
        it->geo_ij, it->geo_order, nl, pool, ctx->d_chunk_prev, ctx->d_chunk_meta, R.cl, W.cnt_long, W.rays_long,
        W.gdef_long, it->geo_grp, ctx->d_started);
    CK(cudaGetLastError());
    /* the waves' blocks are launched once the class's SM-filling blocks are
     * resident (bounded host wait), so these find whole SMs */
    wait_started(ctx, lb);
    R.launched = true;
    CK(cudaEventRecord(ctx->ev_join[0], sr)); /* the class's geodesics are done */
    st = ctx->bstream[0];
    CK(cudaStreamWaitEvent(st, ctx->bev[0][2], 0));
    gl = it->geo_order + R.nl;
    pend_g -= R.nl;
  }
  const long long c0 = R.cl; /* the waves allocate from here */
  size_t wave = pend_g;
  int cur = 0;
  bool first = true;
  while (pend_g > 0 || pend_x > 0) {
    /* the class joins this wave: its records and its rays that found its
     * range full (continued as ordinary items) */
    long long c_first = c0;
    if (R.launched && !R.merged && !first && (pend_g == 0 || cudaEventQuery(ctx->ev_join[0]) == cudaSuccess)) {
      CK(cudaStreamWaitEvent(st, ctx->ev_join[0], 0));
      k_rider_merge<<<(int)((R.nl + 255) / 256), 256, 0, st>>>(it->geo_order, (int)R.nl, W.rays_long, W.rays);
      CK(cudaGetLastError());
      unsigned long long hl[CNT_NB];
      CK(cudaMemcpyAsync(hl, W.cnt_long, sizeof(hl), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      R.merged = true;
      ctx->stats.ray_steps += hl[CNT_STEPS];
      ctx->stats.long_class_items += R.nl;
      if (steps_left) *steps_left = hl[CNT_STEPS] >= *steps_left ? 0 : *steps_left - hl[CNT_STEPS];
      if (hl[CNT_TIMEOUT]) {
        snprintf(ctx->err, sizeof(ctx->err), "the batch's step budget ran out");
        return IPG_E_TIMEOUT;
      }
      if (hl[CNT_DEFER]) {
        CK(cudaMemcpyAsync(W.glist[cur] + pend_g, W.gdef_long, hl[CNT_DEFER] * sizeof(int32_t),
                           cudaMemcpyDeviceToDevice, st));
        pend_g += (size_t)hl[CNT_DEFER];
        gl = W.glist[cur];
      }
      c_first = 0;
#ifdef IPG_DEBUG_TIMING
      fprintf(stderr, "batch: the longest class (%zu items, range %lld, used %llu, deferred %llu) joins wave %d\n",
              R.nl, R.cl, hl[CNT_POOL], hl[CNT_DEFER], ctx->stats.waves + 1);
#endif
    }
    size_t run = pend_g < wave ? pend_g : wave;
    size_t carry = pend_g - run;
    int32_t *gnext = W.glist[cur ^ 1], *xnext = W.xlist[cur ^ 1];
    if (steps_left && *steps_left == 0) return IPG_E_TIMEOUT;
    unsigned long long h0[CNT_NB];
    memset(h0, 0, sizeof(h0));
    h0[CNT_POOL] = (unsigned long long)c0;
    h0[CNT_DEFER] = carry;
    h0[CNT_BUDGET] = steps_left ? *steps_left : 0;
    CK(cudaMemcpyAsync(W.cnt, h0, sizeof(h0), cudaMemcpyHostToDevice, st));
    if (pend_g) k_mark_pending<<<(int)((pend_g + 255) / 256), 256, 0, st>>>(gl, (int)pend_g, W.rays);
    if (carry) {
      if (gl) CK(cudaMemcpyAsync(gnext, gl + run, carry * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
      else k_iota<<<(int)((carry + 255) / 256), 256, 0, st>>>(gnext, (int)carry, (int)run);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[0], st));
    int gb = grid_blocks(ctx, geo_fn, threads, run);
    k_geodesic<IPG_PLUG_IHARM, 256, IPG_GEO_MINB, false, CamTable><<<gb, threads, 0, st>>>(
        it->geo_ij, gl, (int)run, pool, ctx->d_chunk_prev, ctx->d_chunk_meta, n_chunks, W.cnt, W.rays, gnext,
        it->geo_grp);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[1], st));
#define IPG_LAUNCH_BCOEF(EMT, F, RMC)                                                                              \
  do {                                                                                                       \
    int cb = grid_blocks(ctx, (const void *)k_coef_batch<EMT, F, RMC>, threads, (size_t)n_chunks * IPG_CHUNK_STEPS); \
    k_coef_batch<EMT, F, RMC><<<cb, threads, 0, st>>>(pool, side, G, ctx->d_chunk_meta, W.cnt, n_chunks, W.rays,  \
                                                 it->geo_grp, it->geo_mask, B->m.fourv, B->m.sets,          \
                                                 (long long)B->m.ncell, c_first);                             \
  } while (0)
    if (B->emission_type == 1) {
      if (ctx->fits32) {
        if (B->rec_mixed) IPG_LAUNCH_BCOEF(1, true, true);
        else IPG_LAUNCH_BCOEF(1, true, false);
      } else {
        if (B->rec_mixed) IPG_LAUNCH_BCOEF(1, false, true);
        else IPG_LAUNCH_BCOEF(1, false, false);
      }
    } else {
      if (ctx->fits32) {
        if (B->rec_mixed) IPG_LAUNCH_BCOEF(4, true, true);
        else IPG_LAUNCH_BCOEF(4, true, false);
      } else {
        if (B->rec_mixed) IPG_LAUNCH_BCOEF(4, false, true);
        else IPG_LAUNCH_BCOEF(4, false, false);
      }
    }
#undef IPG_LAUNCH_BCOEF
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[2], st));
    if (B->rec_mixed) {
      if (B->step32) {
        if (B->xfer_threads == 256) IPG_LAUNCH_XB(256, true, true);
        else IPG_LAUNCH_XB(128, true, true);
      } else {
        if (B->xfer_threads == 256) IPG_LAUNCH_XB(256, false, true);
        else IPG_LAUNCH_XB(128, false, true);
      }
    } else if (B->step32) {
      if (B->xfer_threads == 256) IPG_LAUNCH_XB(256, true, false);
      else IPG_LAUNCH_XB(128, true, false);
    } else {
      if (B->xfer_threads == 256) IPG_LAUNCH_XB(256, false, false);
      else IPG_LAUNCH_XB(128, false, false);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[3], st));
    unsigned long long h[CNT_NB];
    CK(cudaMemcpyAsync(h, W.cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float a = 0.f, b = 0.f, c = 0.f;
    cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&c, ctx->ev[2], ctx->ev[3]);
    ctx->stats.geodesic_ms += a;
    ctx->stats.coeffs_ms += b;
    ctx->stats.transfer_ms += c;
    ctx->stats.wall_ms += a + b + c;
    B->call_xfer_ms += c;
    B->call_items += (double)pend_x;
    ctx->stats.ray_steps += h[CNT_STEPS];
    ctx->stats.radiating_steps += h[CNT_RAD];
    ctx->stats.launches += 3;
    ctx->stats.waves += 1;
    if (steps_left) {
      const unsigned long long used = h[CNT_STEPS] + h[CNT_XSTEPS];
      *steps_left = used >= *steps_left ? 0 : *steps_left - used;
    }
    if (h[CNT_TIMEOUT]) {
      snprintf(ctx->err, sizeof(ctx->err), "the batch's step budget ran out");
      return IPG_E_TIMEOUT;
    }
#ifdef IPG_DEBUG_TIMING
    fprintf(stderr, "batch wave: run %zu used %llu deferred %llu; geo %.1f coef %.1f xfer %.1f ms\n", run,
            h[CNT_POOL] - (unsigned long long)c0, h[CNT_DEFER], a, b, c);
#endif
    const size_t dg = (size_t)h[CNT_DEFER], dx = (size_t)h[CNT_XDEFER];
    if (dg == pend_g && pend_g > 0) {
      /* nothing fitted: fewer rays share the pool next time */
      if (run == 1) {
        snprintf(ctx->err, sizeof(ctx->err), "trajectory pool (%lld chunks) too small for a single ray",
                 (long long)n_chunks);
        return IPG_E_NOMEM;
      }
      wave = run / 2;
    }
    pend_g = dg;
    pend_x = dx;
    first = false;
    cur ^= 1;
    gl = W.glist[cur];
    xl = W.xlist[cur];
  }
  return IPG_OK;
}

extern "C" int ipg__batch_trace(ipg_ctx *ctx, const ipg_batch_items *it, unsigned long long *steps_left)
{
  BatchState *B = ctx->batch;
  if (!B || !B->m.have || !B->G) return IPG_E_STATE;
  if (it->n_geo == 0) return IPG_OK;
  if (it->n_geo > 0x7fffffff || it->n_xf > 0x7fffffff) return IPG_E_ARG;
  int rc = batch_ws_reserve(ctx, B->w, it->n_geo, it->n_xf);
  if (rc) return rc;
  BatchRider R = {0, 0, false, false};
  rc = batch_waves(ctx, it, steps_left, R);
  if (R.launched) {
    /* the context's stream continues after the waves; on an early return
     * the class's geodesics, which write into the pool, end before it */
    cudaEventRecord(ctx->ev_join[1], ctx->bstream[0]);
    cudaStreamWaitEvent(ctx->stream, ctx->ev_join[1], 0);
    if (rc || !R.merged) cudaStreamSynchronize(ctx->stream);
  }
  return rc;
}
#undef IPG_LAUNCH_XB
