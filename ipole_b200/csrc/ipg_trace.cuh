/* Per-step trace of one ray: the quantities dump_var_along records along a
 * traced geodesic (src/io.c:279-543).
 *
 * The ray is integrated by k_geodesic (the same kernel and arithmetic as the
 * image), its step records are gathered before the coefficient pass reuses
 * them, and two kernels fill one row of IPG_TRACE_DOUBLES per step:
 *
 *   k_trace_local  one thread per step: the model's point queries
 *                  (primitives, b, ne, Theta_e, sigma, beta), the fluid
 *                  frequency and k-B angle, jar_calc and get_jkinv, the
 *                  plasma tetrad, the two parallel-transport pushes of its
 *                  e2 vector; and the coefficient block integrate_emission
 *                  uses at that step.
 *   k_trace_walk   the one sequential part: the coherency tensor N carried
 *                  from step to step, recorded (in the coordinate and plasma
 *                  frames, and as Stokes parameters) before each one-step
 *                  integrate_emission call, as dump_var_along does.
 *
 * Index conventions are the reference's: rows 1..nstep-1 are filled,
 * e2Transported is written one row down (row i-1 at step i), and every
 * integrate_emission call starts from I = 0 (it resets its outputs), so
 * I_unpol is the one-step intensity.  Included by ipg_kernels.cu. */
#ifndef IPG_TRACE_CUH
#define IPG_TRACE_CUH

#define TR_GEO 48 /* record slots 0..47: A1, A2, geodesic state */

/* gather the records of the ray traced into `pool` (ray 0 of the wave)
 * into G[s][TR_GEO], s = 0..nstep */
__global__ void k_trace_gather(const double *__restrict__ pool, const int2 *__restrict__ chunk_meta,
                               const unsigned long long *__restrict__ counters, long long n_chunks, int nstep,
                               double *__restrict__ G)
{
  long long used = (long long)counters[CNT_POOL];
  if (used > n_chunks) used = n_chunks;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < used * IPG_CHUNK_STEPS;
       t += (long long)gridDim.x * blockDim.x) {
    int c = (int)(t / IPG_CHUNK_STEPS), slot = (int)(t % IPG_CHUNK_STEPS);
    int2 meta = chunk_meta[c];
    int s = meta.y + slot;
    if (meta.x != 0 || s > nstep) continue;
    const double *p = pool + ((size_t)c * IPG_CHUNK_STEPS + slot) * IPG_STEP_DOUBLES;
    for (int k = 0; k < TR_GEO; k++) G[(size_t)s * TR_GEO + k] = p[k];
  }
}

/* get_bk_angle, src/radiation.c:47-72 */
__device__ __forceinline__ double bk_angle(const double K[4], const double Ucov[4], const double Bcon[4],
                                           const double Bcov[4])
{
  double B = sqrt(fabs(Bcon[0] * Bcov[0] + Bcon[1] * Bcov[1] + Bcon[2] * Bcov[2] + Bcon[3] * Bcov[3]));
  if (B == 0.) return IPG_PI / 2.;
  double k = fabs(K[0] * Ucov[0] + K[1] * Ucov[1] + K[2] * Ucov[2] + K[3] * Ucov[3]);
  double mu = (K[0] * Bcov[0] + K[1] * Bcov[1] + K[2] * Bcov[2] + K[3] * Bcov[3]) / (k * B);
  if (fabs(mu) > 1.) mu /= fabs(mu);
  return acos(mu);
}

/* trilinear interpolation at X, with the weights of model_point
 * (src/grid.c:15-44, 216-283), of the trace-only fields and of fields the
 * image path does not report: out = rho, u, beta (from `extra`, zero when it
 * was not uploaded), sigma, U1..U3, B1..B3; all zero outside the grid, as
 * get_model_primitives / sigma / beta leave them */
__device__ void trace_gather_extra(const double *__restrict__ fields, const double *__restrict__ extra, double X1,
                                   double X2, double X3, double out[10])
{
  const DevGrid &G = c_grid;
  for (int q = 0; q < 10; q++) out[q] = 0.;
  if (X1 < G.startx[1] || X1 >= G.stopx[1] || X2 < G.startx[2] || X2 >= G.stopx[2]) return;
  double phi = fmod(X3, G.cstopx[3]);
  if (phi < 0.0) phi = G.cstopx[3] + phi;
  int i = (int)((X1 - G.startx[1]) / G.dx[1] - 0.5 + 1000) - 1000;
  int j = (int)((X2 - G.startx[2]) / G.dx[2] - 0.5 + 1000) - 1000;
  int k = (int)((phi - G.startx[3]) / G.dx[3] - 0.5 + 1000) - 1000;
  i = max(-1, min(i, G.n1 - 1));
  j = max(-1, min(j, G.n2 - 1));
  k = max(-1, min(k, G.n3 - 1));
  double d1 = fmin(fmax((X1 - ((i + 0.5) * G.dx[1] + G.startx[1])) / G.dx[1], 0.), 1.);
  double d2 = fmin(fmax((X2 - ((j + 0.5) * G.dx[2] + G.startx[2])) / G.dx[2], 0.), 1.);
  double d3 = fmin(fmax((phi - ((k + 0.5) * G.dx[3] + G.startx[3])) / G.dx[3], 0.), 1.);
  i += 1;
  j += 1;
  k += 1;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) {
        double w = (a ? d1 : 1. - d1) * (b ? d2 : 1. - d2) * (c ? d3 : 1. - d3);
        long long cell = (long long)(i + a) * G.si + (long long)(j + b) * G.sj + (k + c);
        if (extra) {
          out[0] += w * extra[cell * 3 + 0];
          out[1] += w * extra[cell * 3 + 1];
          out[2] += w * extra[cell * 3 + 2];
        }
        out[3] += w * fields[cell * IPG_NFIELD + IPG_F_SIGMA];
        for (int q = 0; q < 6; q++) out[4 + q] += w * fields[cell * IPG_NFIELD + IPG_F_U1 + q];
      }
}

/* the complete tetrad of make_plasma_tetrad (src/model_tetrads.c:35-127):
 * Econ rows as plasma_tetrad leaves them, Ecov = g Econ with row 0 negated */
template <int MET>
__device__ int full_tetrad(const ModelPt &mp, const double K[4], const double Bcon[4], double Econ[4][4],
                           double Ecov[4][4])
{
  double e1[4], e2[4];
  int f = plasma_tetrad<MET>(mp.Ucon, K, Bcon, mp.geo.g, mp.geo, Econ, e1, e2);
  for (int a = 0; a < 4; a++) lower(mp.geo.g, Econ[a], Ecov[a]);
  for (int l = 0; l < 4; l++) Ecov[0][l] *= -1.;
  return f;
}

template <int P>
__global__ void k_trace_local(const double *__restrict__ G, int nstep, const double *__restrict__ fields,
                              const double *__restrict__ extra, double *__restrict__ out, CoefBlock *__restrict__ cbs,
                              double *__restrict__ AA, Met *__restrict__ mets)
{
  constexpr int MET = PlugT<P>::MET;
  const DevGrid &Gd = c_grid;
  const DevCam &C = c_cam;
  int s = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (s > nstep) return;
  const double *g = G + (size_t)s * TR_GEO;
  double X[4] = {g[REC_X0], g[REC_X1], g[REC_X2], g[REC_X3]};
  double K[4] = {g[REC_K], g[REC_K + 1], g[REC_K + 2], g[REC_K + 3]};
  double Kh[4] = {g[REC_KH], g[REC_KH + 1], g[REC_KH + 2], g[REC_KH + 3]};
  const double dl = g[REC_DL];
  PointGeo pg;
  point_geo<MET>(X[1], X[2], &pg);
  ModelPt mp;
  model_point_t<P>(fields, X[1], X[2], X[3], pg, &mp);
  double ju, ku;
  Jar jar;
  coeffs_t<P>(mp, K, 1, C.emission_type, &ju, &ku, &jar);
  /* step nstep also writes its row (the walk needs its coefficient block
   * and transport matrices); k_trace_walk clears what the reference leaves
   * zero */
  double *o = out + (size_t)s * IPG_TRACE_DOUBLES;
  /* point queries */
  double ex[10] = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0.}; /* rho, u, beta, sigma, U1..B3 */
  if constexpr (P == IPG_PLUG_IHARM) {
    trace_gather_extra(fields, extra, X[1], X[2], X[3], ex);
    o[IPG_TRACE_PRIMS + 0] = ex[0];
    o[IPG_TRACE_PRIMS + 1] = ex[1];
    for (int q = 0; q < 6; q++) o[IPG_TRACE_PRIMS + 2 + q] = ex[4 + q];
  } else if constexpr (P == IPG_PLUG_SPHERE) {
    if (radiating_t<P>(pg)) {
      ex[2] = c_plug.beta0;
      ex[3] = c_plug.sigma0;
    }
  }
  o[IPG_TRACE_B] = mp.bmag;
  o[IPG_TRACE_NE] = mp.ne;
  o[IPG_TRACE_THETAE] = mp.thetae;
  double kdu = K[0] * mp.Ucov[0] + K[1] * mp.Ucov[1] + K[2] * mp.Ucov[2] + K[3] * mp.Ucov[3];
  o[IPG_TRACE_NU] = -kdu * IPG_ME * IPG_CL * IPG_CL / IPG_HPL;
  o[IPG_TRACE_BK_ANGLE] = bk_angle(K, mp.Ucov, mp.Bcon, mp.Bcov);
  o[IPG_TRACE_SIGMA] = ex[3];
  o[IPG_TRACE_BETA] = ex[2];
  o[IPG_TRACE_DL] = dl;
  o[IPG_TRACE_R] = pg.r;
  o[IPG_TRACE_TH] = pg.th;
  o[IPG_TRACE_PHI] = X[3];
  o[IPG_TRACE_J_UNPOL] = ju;
  o[IPG_TRACE_K_UNPOL] = ku;
  for (int m = 0; m < 4; m++) {
    o[IPG_TRACE_X + m] = X[m];
    o[IPG_TRACE_KCON + m] = K[m];
  }
  double jv[4] = {jar.jI, jar.jQ, jar.jU, jar.jV}, av[4] = {jar.aI, jar.aQ, jar.aU, jar.aV},
         rv[4] = {0., jar.rQ, jar.rU, jar.rV};
  for (int m = 0; m < 4; m++) {
    o[IPG_TRACE_J_INV + m] = jv[m];
    o[IPG_TRACE_ALPHA_INV + m] = av[m];
    o[IPG_TRACE_RHO_INV + m] = rv[m];
  }
  /* the tetrad dump_var_along builds (no B fallback) */
  double Econ[4][4], Ecov[4][4];
  full_tetrad<MET>(mp, K, mp.Bcon, Econ, Ecov);
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      o[IPG_TRACE_ECON + 4 * a + b] = Econ[a][b];
      o[IPG_TRACE_ECOV + 4 * a + b] = Ecov[a][b];
    }
  for (int m = 0; m < 4; m++) {
    o[IPG_TRACE_E2C + m] = Econ[2][m];
    o[IPG_TRACE_E2C_COV + m] = Ecov[2][m];
  }
  /* parallel_transport_vector twice (src/ipolarray.c:297-320): Gamma K at X
   * and at Xhalf, the transport matrices push_polar uses too */
  double A1[4][4], A2[4][4];
  {
    Conn cn;
    fd_connection<MET>(X[1], X[2], &cn);
    transport_matrix(cn, K, A1);
    fd_connection<MET>(g[REC_XH1], g[REC_XH2], &cn);
    transport_matrix(cn, Kh, A2);
  }
  const double f = dl * Gd.inv_dlfac;
  double mid[4], fin[4];
  for (int i = 0; i < 4; i++)
    mid[i] = Econ[2][i] - (A1[i][0] * Econ[2][0] + A1[i][1] * Econ[2][1] + A1[i][2] * Econ[2][2] +
                           A1[i][3] * Econ[2][3]) * f;
  for (int i = 0; i < 4; i++)
    fin[i] = Econ[2][i] - (A2[i][0] * mid[0] + A2[i][1] * mid[1] + A2[i][2] * mid[2] + A2[i][3] * mid[3]) * f;
  double *om = out + (size_t)(s - 1) * IPG_TRACE_DOUBLES;
  for (int m = 0; m < 4; m++) om[IPG_TRACE_E2T + m] = fin[m];
  double *aa = AA + (size_t)s * 32;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      aa[4 * a + b] = A1[a][b];
      aa[16 + 4 * a + b] = A2[a][b];
    }
  mets[s] = pg.g;
  /* the coefficient block of integrate_emission at this point (k_coeffs) */
  CoefBlock cb;
  memset(&cb, 0, sizeof(cb));
  int flags = radiating_t<P>(pg) ? 1 : 0;
  if (C.counterjet == 1) {
    if (X[2] < (Gd.cstopx[2] - Gd.cstartx[2]) / 2) flags |= 2;
  } else if (C.counterjet == 2) {
    if (X[2] > (Gd.cstopx[2] - Gd.cstartx[2]) / 2) flags |= 2;
  }
  if ((flags & 1) && !C.unpol) {
    double Bc[4] = {mp.Bcon[0], mp.Bcon[1], mp.Bcon[2], mp.Bcon[3]};
    double bsq = Bc[0] * mp.Bcov[0] + Bc[1] * mp.Bcov[1] + Bc[2] * mp.Bcov[2] + Bc[3] * mp.Bcov[3];
    if (bsq <= 0.) {
      Bc[0] = 0.;
      Bc[1] = Bc[2] = Bc[3] = 1.;
    }
    double E2[4][4];
    int tf = plasma_tetrad<MET>(mp.Ucon, K, Bc, mp.geo.g, mp.geo, E2, cb.e1, cb.e2);
    if (isnan(mp.Ucov[0])) tf |= 8;
    flags |= tf << 2;
    for (int m = 0; m < 4; m++) {
      cb.a[m] = E2[1][m];
      cb.b[m] = E2[2][m];
    }
  }
  cb.flags = flags;
  cb.ju = ju;
  cb.ku = ku;
  cb.dl = dl;
  cb.jI = jar.jI;
  cb.jQ = jar.jQ;
  cb.jV = jar.jV;
  cb.aI = jar.aI;
  cb.aQ = jar.aQ;
  cb.aV = jar.aV;
  cb.rQ = jar.rQ;
  cb.rV = jar.rV;
  cb.nturns = g[REC_NTURNS];
  cbs[s] = cb;
}

/* the sequential part of dump_var_along's loop (src/io.c:369-434) */
__global__ void k_trace_walk(int nstep, double *__restrict__ out, const CoefBlock *__restrict__ cbs,
                             const double *__restrict__ AA, const Met *__restrict__ mets)
{
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const DevGrid &G = c_grid;
  const DevCam &C = c_cam;
  /* the reference's loop runs i = nstep-1 .. 1: row nstep stays zero, and so
   * does e2Transported of row nstep-1 (written at step nstep only) */
  for (int k = 0; k < IPG_TRACE_DOUBLES; k++) out[(size_t)nstep * IPG_TRACE_DOUBLES + k] = 0.;
  if (nstep >= 1)
    for (int m = 0; m < 4; m++) out[(size_t)(nstep - 1) * IPG_TRACE_DOUBLES + IPG_TRACE_E2T + m] = 0.;
  HermN N;
  hn_zero(&N);
  for (int i = nstep - 1; i > 0; --i) {
    double *o = out + (size_t)i * IPG_TRACE_DOUBLES;
    double R[4][4], S[4][4], Ecov[4][4];
    hn_unpack(N, R, S);
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) Ecov[a][b] = o[IPG_TRACE_ECOV + 4 * a + b];
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) {
        double t = 0.;
        for (int mu = 0; mu < 4; mu++)
          for (int nu = 0; nu < 4; nu++) t += Ecov[a][mu] * Ecov[b][nu] * R[mu][nu];
        o[IPG_TRACE_NTETRAD + 4 * a + b] = t;
        o[IPG_TRACE_NCOORD + 4 * a + b] = R[a][b];
      }
    double T11, T22, T12r, T21i;
    hn_stokes(N, Ecov[1], Ecov[2], &T11, &T22, &T12r, &T21i);
    o[IPG_TRACE_STOKES + 0] = (T11 + T22) / 2;
    o[IPG_TRACE_STOKES + 1] = (T11 - T22) / 2;
    o[IPG_TRACE_STOKES + 2] = T12r;
    o[IPG_TRACE_STOKES + 3] = T21i;
    double e2[4] = {o[IPG_TRACE_E2T], o[IPG_TRACE_E2T + 1], o[IPG_TRACE_E2T + 2], o[IPG_TRACE_E2T + 3]}, e2c[4];
    lower(mets[i], e2, e2c);
    for (int m = 0; m < 4; m++) o[IPG_TRACE_E2T_COV + m] = e2c[m];
    /* integrate_emission(&traj[i], 1, ...): one step from i+1 to i, from I = 0 */
    const CoefBlock &ti = cbs[i + 1], &tf = cbs[i];
    const double dl = ti.dl;
    double I = 0., tau = 0., tauF = 0.;
    int flag = 0;
    if (!C.unpol) {
      double A[4][4];
      HermN Nh, Nn;
      const double *aa = AA + (size_t)(i + 1) * 32;
      for (int a = 0; a < 16; a++) A[a / 4][a % 4] = aa[a];
      hn_push(N, N, A, (0.5 * dl) * G.inv_dlfac, &Nh);
      for (int a = 0; a < 16; a++) A[a / 4][a % 4] = aa[16 + a];
      hn_push(N, Nh, A, dl * G.inv_dlfac, &Nn);
      N = Nn;
    }
    int flags = (int)tf.flags;
    if (flags & 1) {
      int zero_emission = (flags & 2) ? 1 : 0;
      if (C.target_nturns >= 0 && (int)ti.nturns != C.target_nturns) zero_emission = 1;
      if (zero_emission) I = approximate_solve(0., 0, ti.ku, 0, tf.ku, dl, &tau);
      else I = approximate_solve(0., ti.ju, ti.ku, tf.ju, tf.ku, dl, &tau);
      if (!C.unpol) {
        flag |= flags >> 2;
        flag |= evolve_N_coef(tf, dl, zero_emission, &N, &tauF, c_cam.stokes_floors);
      }
    }
    o[IPG_TRACE_I_UNPOL] = I;
    o[IPG_TRACE_FLAG] = flag;
  }
}

template <int P>
static int trace_ray_t(ipg_ctx *ctx, int nstep, long long used, double *d_out, double *G, CoefBlock *cbs, double *AA,
                       Met *mets)
{
  k_trace_gather<<<(int)((used * IPG_CHUNK_STEPS + 255) / 256), 256, 0, ctx->stream>>>(
      ctx->d_pool, ctx->d_chunk_meta, ctx->d_cnt, ctx->n_chunks, nstep, G);
  CK(cudaGetLastError());
  if (nstep >= 1) {
    k_trace_local<P><<<(nstep + 63) / 64, 64, 0, ctx->stream>>>(G, nstep, ctx->d_fields, ctx->d_trace_extra, d_out,
                                                               cbs, AA, mets);
    CK(cudaGetLastError());
    k_trace_walk<<<1, 1, 0, ctx->stream>>>(nstep, d_out, cbs, AA, mets);
    CK(cudaGetLastError());
  }
  return IPG_OK;
}

extern "C" int ipg_upload_trace_fields(ipg_ctx *ctx, const double *const extra[3])
{
  if (!ctx || !extra || !extra[0] || !extra[1] || !extra[2]) return IPG_E_ARG;
  if (!ctx->have_model || ctx->plug != IPG_PLUG_IHARM || !ctx->ncell) return IPG_E_STATE;
  CK(cudaSetDevice(ctx->device));
  std::vector<double> aos(ctx->ncell * 3);
  for (size_t c = 0; c < ctx->ncell; c++)
    for (int f = 0; f < 3; f++) aos[c * 3 + f] = extra[f][c];
  if (!ctx->d_trace_extra) CK(cudaMalloc(&ctx->d_trace_extra, ctx->ncell * 3 * sizeof(double)));
  CK(cudaMemcpy(ctx->d_trace_extra, aos.data(), ctx->ncell * 3 * sizeof(double), cudaMemcpyHostToDevice));
  return IPG_OK;
}

extern "C" int ipg_trace_ray(ipg_ctx *ctx, const ipg_camera *cam, int i, int j, size_t max_steps, double *steps,
                             int32_t *nstep_out)
{
  if (!ctx || !cam || !steps || !nstep_out || max_steps < 1) return IPG_E_ARG;
  CK(cudaSetDevice(ctx->device));
  if (!ctx->have_model) return IPG_E_STATE;
  int rc = ensure_pool(ctx);
  if (rc) return rc;
  rc = ensure_cap(ctx, 1);
  if (rc) return rc;
  DevCam dc;
  make_devcam(cam, &dc);
  CK(cudaMemcpyToSymbolAsync(c_grid, &ctx->dg, sizeof(DevGrid), 0, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyToSymbolAsync(c_plug, &ctx->dp, sizeof(DevPlug), 0, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyToSymbolAsync(c_cam, &dc, sizeof(DevCam), 0, cudaMemcpyHostToDevice, ctx->stream));
  int32_t hij[2] = {i, j};
  CK(cudaMemcpyAsync(ctx->d_ij, hij, sizeof(hij), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(ctx->d_cnt, 0, sizeof(unsigned long long) * CNT_N, ctx->stream));
  switch (ctx->plug) {
    case IPG_PLUG_ANALYTIC:
      k_geodesic<IPG_PLUG_ANALYTIC, 256, IPG_GEO_MINB><<<1, 32, 0, ctx->stream>>>(ctx->d_ij, NULL, 1, ctx->d_pool, ctx->d_chunk_prev,
                                                              ctx->d_chunk_meta, ctx->n_chunks, ctx->d_cnt,
                                                              ctx->d_rays, ctx->d_list[1], nullptr);
      break;
    case IPG_PLUG_SPHERE:
      k_geodesic<IPG_PLUG_SPHERE, 256, IPG_GEO_MINB><<<1, 32, 0, ctx->stream>>>(ctx->d_ij, NULL, 1, ctx->d_pool, ctx->d_chunk_prev,
                                                            ctx->d_chunk_meta, ctx->n_chunks, ctx->d_cnt,
                                                            ctx->d_rays, ctx->d_list[1], nullptr);
      break;
    default:
      k_geodesic<IPG_PLUG_IHARM, 256, IPG_GEO_MINB><<<1, 32, 0, ctx->stream>>>(ctx->d_ij, NULL, 1, ctx->d_pool, ctx->d_chunk_prev,
                                                           ctx->d_chunk_meta, ctx->n_chunks, ctx->d_cnt, ctx->d_rays,
                                                           ctx->d_list[1], nullptr);
  }
  CK(cudaGetLastError());
  RayRec rec;
  unsigned long long used = 0;
  CK(cudaMemcpyAsync(&rec, ctx->d_rays, sizeof(rec), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&used, ctx->d_cnt + CNT_POOL, sizeof(used), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if ((long long)used > ctx->n_chunks) used = (unsigned long long)ctx->n_chunks;
  if (rec.status == IPG_RAY_POOL_FULL) {
    snprintf(ctx->err, sizeof(ctx->err), "trajectory pool too small for the traced ray");
    return IPG_E_NOMEM;
  }
  *nstep_out = rec.nstep;
  if (rec.status == IPG_RAY_MAXNSTEP) {
    snprintf(ctx->err, sizeof(ctx->err), "MaxNStep exceeded in pixel %d %d", i, j);
    return IPG_E_MAXNSTEP;
  }
  const int nstep = rec.nstep;
  if ((size_t)nstep + 1 > max_steps) {
    snprintf(ctx->err, sizeof(ctx->err), "trace of pixel %d %d has %d steps, buffer holds %zu", i, j, nstep + 1,
             max_steps);
    return IPG_E_ARG;
  }
  const size_t rows = (size_t)nstep + 1;
  double *d_out = NULL, *G = NULL, *AA = NULL;
  CoefBlock *cbs = NULL;
  Met *mets = NULL;
  cudaError_t e = cudaMalloc(&d_out, rows * IPG_TRACE_DOUBLES * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&G, rows * TR_GEO * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&AA, rows * 32 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&cbs, rows * sizeof(CoefBlock));
  if (e == cudaSuccess) e = cudaMalloc(&mets, rows * sizeof(Met));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_out, 0, rows * IPG_TRACE_DOUBLES * sizeof(double), ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(cbs, 0, rows * sizeof(CoefBlock), ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(AA, 0, rows * 32 * sizeof(double), ctx->stream);
  if (e == cudaSuccess) {
    switch (ctx->plug) {
      case IPG_PLUG_ANALYTIC:
        rc = trace_ray_t<IPG_PLUG_ANALYTIC>(ctx, nstep, (long long)used, d_out, G, cbs, AA, mets);
        break;
      case IPG_PLUG_SPHERE:
        rc = trace_ray_t<IPG_PLUG_SPHERE>(ctx, nstep, (long long)used, d_out, G, cbs, AA, mets);
        break;
      default: rc = trace_ray_t<IPG_PLUG_IHARM>(ctx, nstep, (long long)used, d_out, G, cbs, AA, mets);
    }
  }
  if (e == cudaSuccess && rc == IPG_OK) {
    memset(steps, 0, max_steps * IPG_TRACE_DOUBLES * sizeof(double));
    e = cudaMemcpyAsync(steps, d_out, rows * IPG_TRACE_DOUBLES * sizeof(double), cudaMemcpyDeviceToHost,
                        ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  }
  cudaFree(d_out);
  cudaFree(G);
  cudaFree(AA);
  cudaFree(cbs);
  cudaFree(mets);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "ipg_trace_ray");
  return rc;
}

#endif
