/*
 * Reverse-mode adjoint of the polarized image (ipg_adjoint): the gradient of
 * a loss of the IQUV image with respect to the fluid fields ne, Theta_e and
 * |B| of every cell (the fields the fits read, model/iharm/model.c:
 * 510-593).  No counterpart in the reference, which only renders.
 *
 * The geodesics do not depend on the fluid, so only the radiative transfer
 * is differentiated (src/ipolarray.c:59-628).  Per ray, the transfer maps
 * the coherency tensor N from the source end (N = 0 at step nstep) to the
 * camera (N_0, projected to I, Q, U, V); step n -> n-1 is
 *
 *   N_h  = N_n - dl/2 (A1 N_n + N_n A1^T)       push_polar, half step
 *   N'   = N_n - dl   (A2 N_h + N_h A2^T)       push_polar, full step
 *   N_{n-1} = evolve_N(N', coefficients of step n-1)   at radiating points
 *
 * with A1, A2 from the step records.  The adjoint walks back from the
 * camera: G_0 = dL/dN_0 from dL/dIQUV, then for n = 1 .. nstep it maps
 * G_{n-1} = dL/dN_{n-1} to G_n through the transposes of these maps, and at
 * every radiating step it turns dL/d(coefficients) into dL/d(ne, Theta_e,
 * |B|) at the point and scatter-adds that to the eight cells of the
 * trilinear gather (src/grid.c:15-44), with their weights.
 *
 *   - The N it needs are recomputed, not stored: the forward pass keeps
 *     N every K steps (k_transfer with CKK = K), and the adjoint
 *     recomputes a segment from its top with the forward's own functions,
 *     so they are the forward's bits; it keeps, per step of the segment,
 *     N after the step's two pushes (the state evolve_N was applied to).
 *   - The walk (k_adjoint, one lane per ray) leaves dL/d(coefficients) at
 *     each radiating record; k_adj_scatter, one thread per record, turns
 *     them into dL/d(ne, Theta_e, |B|) and scatter-adds those to the cells,
 *     off the walk's critical path.
 *   - The coefficients' derivatives come from re-evaluating the fits
 *     (jar_fits) in forward-mode dual numbers along ne, Theta_e, |B|
 *     (ipg_dual.cuh), and the step's from re-evaluating the Faraday and
 *     absorption/emission step (faraday_rot, absorb_emit) in duals along
 *     the Stokes vector and the eight coefficients.
 *   - Gradients of N are kept as full-matrix gradients of its real
 *     (symmetric) and imaginary (antisymmetric) parts, upper triangles
 *     stored: every map here keeps those symmetries.
 *
 * Not differentiated: the sigma cut of ne and the Theta_e floor of the
 * host (their derivative is zero almost everywhere), the Stokes floors
 * (the call refuses stokes_floors), the unpolarized intensity.
 *
 * Included by ipg_kernels.cu.
 */

#include "ipg_step_vjp.cuh"

/* gradient of a Hermitian N: g.r[ij] = dL/dRe N[i][j] = dL/dRe N[j][i],
 * g.s[ij] = dL/dIm N[i][j] = -dL/dIm N[j][i] (the same layout as HermN) */
typedef HermN GradN;

__device__ __forceinline__ void gn_full(const GradN &g, double R[4][4], double S[4][4]) { hn_unpack(g, R, S); }

__device__ __forceinline__ void gn_pack(const double R[4][4], const double S[4][4], GradN *g)
{
  g->r00 = R[0][0]; g->r01 = R[0][1]; g->r02 = R[0][2]; g->r03 = R[0][3];
  g->r11 = R[1][1]; g->r12 = R[1][2]; g->r13 = R[1][3];
  g->r22 = R[2][2]; g->r23 = R[2][3]; g->r33 = R[3][3];
  g->s01 = S[0][1]; g->s02 = S[0][2]; g->s03 = S[0][3];
  g->s12 = S[1][2]; g->s13 = S[1][3]; g->s23 = S[2][3];
}

/* base + s (A^T G + G A), the transpose of X -> A X + X A^T, for both parts */
__device__ __forceinline__ void gn_push_adj(const GradN &base, const GradN &G, const double A[4][4], double s,
                                            GradN *out)
{
  double R[4][4], S[4][4], oR[4][4], oS[4][4];
  gn_full(G, R, S);
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      double ar = 0., as = 0., ra = 0., sa = 0.;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        ar += A[k][i] * R[k][j];
        as += A[k][i] * S[k][j];
        ra += R[i][k] * A[k][j];
        sa += S[i][k] * A[k][j];
      }
      oR[i][j] = ar + ra;
      oS[i][j] = as + sa;
    }
  double bR[4][4], bS[4][4];
  gn_full(base, bR, bS);
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      oR[i][j] = bR[i][j] + s * oR[i][j];
      oS[i][j] = bS[i][j] + s * oS[i][j];
    }
  gn_pack(oR, oS, out);
}

/* G += the transpose of hn_stokes at (gT11, gT22, gT12r, gT21i):
 * T11 = e1 R e1, T22 = e2 R e2, T12r = e1 R e2, T21i = e2 S e1 (symmetric
 * and antisymmetric parts of the outer products) */
__device__ __forceinline__ void gn_add_stokes_adj(const double e1[4], const double e2[4], double g11, double g22,
                                                  double g12r, double g21i, GradN *G)
{
  double R[4][4], S[4][4];
  gn_full(*G, R, S);
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      R[i][j] += g11 * e1[i] * e1[j] + g22 * e2[i] * e2[j] + 0.5 * g12r * (e1[i] * e2[j] + e2[i] * e1[j]);
      S[i][j] += 0.5 * g21i * (e2[i] * e1[j] - e1[i] * e2[j]);
    }
  gn_pack(R, S, G);
}

/* the polarized step S -> S' of evolve_N (Faraday half step, absorption and
 * emission, Faraday half step; src/ipolarray.c:390-520) in any number type */
template <class R>
__device__ __forceinline__ void stokes_step(const JarT<R> &c, double dlam, R S[4])
{
  const FaradayRotT<R> F = faraday_rot(c.rQ, c.rU, c.rV, dlam * 0.5);
  faraday_apply(F, c.rQ, c.rU, c.rV, &S[1], &S[2], &S[3]);
  absorb_emit(c, dlam, &S[0], &S[1], &S[2], &S[3]);
  faraday_apply(F, c.rQ, c.rU, c.rV, &S[1], &S[2], &S[3]);
}

/* the coefficient block cb as the step reads it, with zero_emission */
__device__ __forceinline__ void coef_values(const CoefBlock &cb, int zero_emission, double v[8])
{
  v[0] = zero_emission ? 0. : cb.jI;
  v[1] = zero_emission ? 0. : cb.jQ;
  v[2] = zero_emission ? 0. : cb.jV;
  v[3] = cb.aI;
  v[4] = cb.aQ;
  v[5] = cb.aV;
  v[6] = cb.rQ;
  v[7] = cb.rV;
}

/* One pass of the step in Dual<4>: directions d0..d3 among the 12 inputs
 * (S0..S3, then the eight coefficients); returns u . dS'/d(direction). */
__device__ __forceinline__ void step_vjp_pass(const double S0[4], const double cv[8], double dlam, const double u[4],
                                              int first, double out[4])
{
  Dual<4> S[4], cc[8];
#pragma unroll
  for (int k = 0; k < 4; k++) S[k] = (first == 0) ? dvar<4>(S0[k], k) : dconst<4>(S0[k]);
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int dir = 4 + k - first;
    cc[k] = (dir >= 0 && dir < 4 && first > 0) ? dvar<4>(cv[k], dir) : dconst<4>(cv[k]);
  }
  JarT<Dual<4>> c;
  c.jI = cc[0];
  c.jQ = cc[1];
  c.jU = dconst<4>(0.);
  c.jV = cc[2];
  c.aI = cc[3];
  c.aQ = cc[4];
  c.aU = dconst<4>(0.);
  c.aV = cc[5];
  c.rQ = cc[6];
  c.rU = dconst<4>(0.);
  c.rV = cc[7];
  stokes_step(c, dlam, S);
#pragma unroll
  for (int d = 0; d < 4; d++) out[d] = u[0] * S[0].d[d] + u[1] * S[1].d[d] + u[2] * S[2].d[d] + u[3] * S[3].d[d];
}

/* The transpose of evolve_N_coef at N (the state it was applied to):
 * G (dL/dN after the step) becomes dL/dN before it, and gc[8] receives
 * dL/d(jI, jQ, jV, aI, aQ, aV, rQ, rV) (zero for the emissivities when the
 * step had zero_emission). */
__device__ __forceinline__ void evolve_adj(const CoefBlock &cb, double dlam, int zero_emission, const HermN &N,
                                           GradN *G, double gc[8])
{
  double T11, T22, T12r, T21i;
  hn_stokes(N, cb.e1, cb.e2, &T11, &T22, &T12r, &T21i);
  const double S0[4] = {(T11 + T22) / 2, (T11 - T22) / 2, T12r, T21i};
  /* N' = N + D(d), d = (SI'+SQ' - T11, SI'-SQ' - T22, SU' - T12r, SV' - T21i) */
  double R[4][4], Sg[4][4];
  gn_full(*G, R, Sg);
  const double *a = cb.a, *b = cb.b;
  double aRa = 0., bRb = 0., aRb = 0., bSa = 0.;
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      aRa += a[i] * R[i][j] * a[j];
      bRb += b[i] * R[i][j] * b[j];
      aRb += a[i] * R[i][j] * b[j];
      bSa += b[i] * Sg[i][j] * a[j];
    }
  const double g11 = aRa, g22 = bRb, g12 = 2. * aRb, g21 = 2. * bSa;
  const double u[4] = {g11 + g22, g11 - g22, g12, g21};
  double cv[8];
  coef_values(cb, zero_emission, cv);
  double gS[4];
  stokes_step_vjp(cv, dlam, S0, u, gS, gc);
  if (zero_emission) gc[0] = gc[1] = gc[2] = 0.;
  /* d/dT: directly (-d) and through S = (T11+T22, T11-T22)/2, T12r, T21i */
  const double t11 = -g11 + 0.5 * (gS[0] + gS[1]);
  const double t22 = -g22 + 0.5 * (gS[0] - gS[1]);
  const double t12 = -g12 + gS[2];
  const double t21 = -g21 + gS[3];
  gn_add_stokes_adj(cb.e1, cb.e2, t11, t22, t12, t21, G);
}

/* step records by step index, walking the ray's chunk chain both ways */
struct ChunkWalk {
  int chunk, base; /* chunk holding steps base .. base + 31 */
};

__device__ __forceinline__ const double *walk_rec(ChunkWalk &w, int n, const double *pool, const int *prev,
                                                  const int *next)
{
  while (n < w.base) {
    w.chunk = prev[w.chunk];
    w.base -= IPG_CHUNK_STEPS;
  }
  while (n >= w.base + IPG_CHUNK_STEPS) {
    w.chunk = next[w.chunk];
    w.base += IPG_CHUNK_STEPS;
  }
  return step_ptr(const_cast<double *>(pool), w.chunk, n - w.base);
}

/* forward links of the chunk chains and each ray's first chunk */
__global__ void k_adj_link(const int *__restrict__ prev, const int2 *__restrict__ meta,
                           const unsigned long long *__restrict__ counters, long long n_chunks, int *__restrict__ next,
                           int *__restrict__ first)
{
  long long used = (long long)counters[CNT_POOL];
  if (used > n_chunks) used = n_chunks;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < used; c += (long long)gridDim.x * blockDim.x) {
    const int p = prev[c];
    if (p >= 0) next[p] = (int)c;
    else first[meta[c].x] = (int)c;
  }
}

/* one forward step n -> n-1 of N (the polarized part of xfer_step);
 * *Np receives N after the two pushes, before evolve_N */
__device__ __forceinline__ void fwd_N(const DevCam &C, const double *rec_n, const double *rec_m, HermN *N,
                                      HermN *Np)
{
  const DevGrid &G = c_grid;
  const double dl = rec_n[REC_DL];
  double A[4][4];
  HermN Nh, Nn;
  load_A(rec_n + REC_A1, A);
  hn_push(*N, *N, A, (0.5 * dl) * G.inv_dlfac, &Nh);
  load_A(rec_n + REC_A2, A);
  hn_push(*N, Nh, A, dl * G.inv_dlfac, &Nn);
  *Np = Nn;
  CoefBlock cb;
  load_coef(rec_m, cb);
  const int flags = (int)cb.flags;
  if (flags & 1) {
    int zero_emission = (flags & 2) ? 1 : 0;
    if (C.target_nturns >= 0 && (int)rec_n[REC_NTURNS] != C.target_nturns) zero_emission = 1;
    double tauF = 0.;
    evolve_N_coef(cb, dl, zero_emission, &Nn, &tauF, 0);
  }
  *N = Nn;
}

/* dL/d(ne, Theta_e, |B|) at the point of a radiating record from dL/d(its
 * coefficients), scattered to the eight cells of its gather */
__device__ __forceinline__ void fluid_scatter(const double *__restrict__ fields, const double *__restrict__ side,
                                              int emission_type, const double gc[8], double *__restrict__ g_ne,
                                              double *__restrict__ g_th, double *__restrict__ g_b)
{
  const int fl = (int)side[7];
  if (!(fl & 2)) return; /* outside the grid: no fluid */
  const double X1 = side[0], X2 = side[1], X3 = side[2];
  GridLoc gl;
  grid_locate(X1, X2, X3, &gl);
  double acc[10];
  gather_cells<10>(fields, gl, acc);
  const double ne = sigma_cut_ne(acc[6], acc[9]);
  if (!(ne > 0.)) return;
  const double dne = ne / acc[6]; /* 1, or the factor of the sigma cut's boundary */
  JarGeo jg;
  jg.nu = side[3];
  jg.inusq = 1. / (jg.nu * jg.nu);
  jg.sth = side[4];
  jg.cth = side[5];
  jg.theta = side[6];
  jg.along = fl & 1;
  Dual<3> Ne = dvar<3>(ne, 0), Th = dvar<3>(acc[7], 1), Bm = dvar<3>(acc[8], 2);
  Dual<3> ju, ku;
  JarT<Dual<3>> jr;
  const Dual<3> z = dconst<3>(0.);
  jr.jI = jr.jQ = jr.jU = jr.jV = jr.aI = jr.aQ = jr.aU = jr.aV = jr.rQ = jr.rU = jr.rV = z;
  jar_fits(Ne, Th, Bm, jg, 1, emission_type, &ju, &ku, &jr);
  const Dual<3> *cs[8] = {&jr.jI, &jr.jQ, &jr.jV, &jr.aI, &jr.aQ, &jr.aV, &jr.rQ, &jr.rV};
  double g[3] = {0., 0., 0.};
#pragma unroll
  for (int k = 0; k < 8; k++)
#pragma unroll
    for (int d = 0; d < 3; d++) g[d] += gc[k] * cs[k]->d[d];
  g[0] *= dne;
#pragma unroll
  for (int cc = 0; cc < 4; cc++)
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
      const long long cell = gl.cs[cc] + kk;
      const double w = gl.w[2 * cc + kk];
      if (w == 0.) continue;
      atomicAdd(g_ne + cell, w * g[0]);
      atomicAdd(g_th + cell, w * g[1]);
      atomicAdd(g_b + cell, w * g[2]);
    }
}

/* One lane per ray of the wave: the adjoint walk, camera to source. */
template <int K>
__global__ void __launch_bounds__(128, 1)
    k_adjoint(const int32_t *__restrict__ list, int n_list, double *__restrict__ pool,
              const double *__restrict__ adj_side, const double *__restrict__ ckpt, const int *__restrict__ prev,
              const int *__restrict__ next, const int *__restrict__ first, const RayRec *__restrict__ rays,
              const double *__restrict__ dL_dout, const double *__restrict__ fields, double *__restrict__ g_ne,
              double *__restrict__ g_th, double *__restrict__ g_b, unsigned long long *__restrict__ counter)
{
  const DevCam &C = c_cam;
  const DevGrid &Gd = c_grid;
  constexpr int KC = K < IPG_CHUNK_STEPS ? K : IPG_CHUNK_STEPS;
  HermN Nbuf[K];
  while (true) {
    const unsigned long long t = atomicAdd(counter, 1ULL);
    if (t >= (unsigned long long)n_list) return;
    const int ray = list ? list[t] : (int)t;
    const RayRec rec = rays[ray];
    if (rec.status != IPG_RAY_OK) continue;
    const int nstep = rec.nstep;
    /* G_0 from dL/d(I, Q, U, V) of project_N (src/ipolarray.c:578-598) */
    const double gI = dL_dout[4 * ray], gQ = dL_dout[4 * ray + 1], gU = dL_dout[4 * ray + 2],
                 gV = dL_dout[4 * ray + 3];
    const double gSQ = gQ * C.cproj + gU * C.sproj, gSU = -gQ * C.sproj + gU * C.cproj;
    GradN G;
    hn_zero(&G);
    gn_add_stokes_adj(C.Ecov[1], C.Ecov[2], 0.5 * (gI + gSQ), 0.5 * (gI - gSQ), gSU, gV, &G);
    ChunkWalk w = {first[ray], 0};
    for (int lo = 0; lo < nstep; lo += K) {
      const int hi = min(lo + K, nstep);
      /* N_hi: zero at the source end, else the forward's checkpoint */
      HermN N;
      if (hi == nstep) {
        hn_zero(&N);
      } else {
        walk_rec(w, hi, pool, prev, next);
        const double *q = ckpt + (((size_t)w.chunk * IPG_CHUNK_STEPS + (hi - w.base)) / KC) * 16;
        N.r00 = q[0]; N.r01 = q[1]; N.r02 = q[2]; N.r03 = q[3];
        N.r11 = q[4]; N.r12 = q[5]; N.r13 = q[6]; N.r22 = q[7];
        N.r23 = q[8]; N.r33 = q[9]; N.s01 = q[10]; N.s02 = q[11];
        N.s03 = q[12]; N.s12 = q[13]; N.s13 = q[14]; N.s23 = q[15];
      }
      /* for n = hi .. lo+1, N_n after the two pushes of step n (the
       * state evolve_N was applied to), the forward's values */
      for (int n = hi; n > lo; n--) {
        const double *rn = walk_rec(w, n, pool, prev, next);
        const double *rm = walk_rec(w, n - 1, pool, prev, next);
        HermN Np;
        fwd_N(C, rn, rm, &N, &Np);
        Nbuf[hi - n] = Np;
      }
      /* the adjoint of steps n = lo+1 .. hi */
      for (int n = lo + 1; n <= hi; n++) {
        const double *rn = walk_rec(w, n, pool, prev, next);
        double *rm = const_cast<double *>(walk_rec(w, n - 1, pool, prev, next));
        const double dl = rn[REC_DL];
        const double dlfull = dl * Gd.inv_dlfac, dlhalf = (0.5 * dl) * Gd.inv_dlfac;
        double A1[4][4], A2[4][4];
        load_A(rn + REC_A1, A1);
        load_A(rn + REC_A2, A2);
        CoefBlock cb;
        load_coef(rm, cb);
        const int flags = (int)cb.flags;
        if (flags & 1) {
          int zero_emission = (flags & 2) ? 1 : 0;
          if (C.target_nturns >= 0 && (int)rn[REC_NTURNS] != C.target_nturns) zero_emission = 1;
          double gc[8];
          evolve_adj(cb, dl, zero_emission, Nbuf[hi - n], &G, gc);
          /* dL/d(coefficients) of the record of step n-1, in place of its
           * A1, which this walk read for the last time at step n-1;
           * k_adj_scatter turns them into the cells' gradients */
          store4(rm + REC_A1, gc[0], gc[1], gc[2], gc[3]);
          store4(rm + REC_A1 + 4, gc[4], gc[5], gc[6], gc[7]);
        }
        /* push_polar twice, transposed: G_Nh = -dlfull (A2^T G + G A2),
         * G_N = G + G_Nh - dlhalf (A1^T G_Nh + G_Nh A1) */
        GradN Gh, zero;
        hn_zero(&zero);
        gn_push_adj(zero, G, A2, -dlfull, &Gh);
        GradN Gs;
        gn_push_adj(Gh, Gh, A1, -dlhalf, &Gs);
        G.r00 += Gs.r00; G.r01 += Gs.r01; G.r02 += Gs.r02; G.r03 += Gs.r03;
        G.r11 += Gs.r11; G.r12 += Gs.r12; G.r13 += Gs.r13; G.r22 += Gs.r22;
        G.r23 += Gs.r23; G.r33 += Gs.r33; G.s01 += Gs.s01; G.s02 += Gs.s02;
        G.s03 += Gs.s03; G.s12 += Gs.s12; G.s13 += Gs.s13; G.s23 += Gs.s23;
      }
    }
  }
}

/* One thread per step record of the wave: the coefficient gradients the
 * walk left at each radiating record (steps 0 .. nstep-1 of a traced ray)
 * become dL/d(ne, Theta_e, |B|) at its point and are scattered to the
 * cells of its gather (fluid_scatter).  Parallel over records, where the
 * walk is one lane per ray. */
__global__ void __launch_bounds__(128, 3)
    k_adj_scatter(const double *__restrict__ pool, const int2 *__restrict__ chunk_meta,
                  const unsigned long long *__restrict__ counters, long long n_chunks,
                  const RayRec *__restrict__ rays, const double *__restrict__ adj_side,
                  const double *__restrict__ fields, double *__restrict__ g_ne, double *__restrict__ g_th,
                  double *__restrict__ g_b)
{
  const DevCam &C = c_cam;
  long long used = (long long)counters[CNT_POOL];
  if (used > n_chunks) used = n_chunks;
  const long long total = used * IPG_CHUNK_STEPS;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / IPG_CHUNK_STEPS), slot = (int)(t % IPG_CHUNK_STEPS);
    const int2 meta = chunk_meta[c];
    const RayRec rec = rays[meta.x];
    const int s = meta.y + slot;
    if (rec.status != IPG_RAY_OK || s >= rec.nstep) continue;
    const double *p = step_ptr(const_cast<double *>(pool), c, slot);
    if (!((int)p[REC_FLAGS] & 1)) continue;
    double gc[8];
    load4(p + REC_A1, gc);
    load4(p + REC_A1 + 4, gc + 4);
    fluid_scatter(fields, adj_side + ((size_t)c * IPG_CHUNK_STEPS + slot) * IPG_ADJ_DOUBLES, C.emission_type, gc,
                  g_ne, g_th, g_b);
  }
}

/* Self-check of stokes_step_vjp against the forward-mode dual numbers
 * (step_vjp_pass, three passes of four directions) on seeded coefficients
 * and Stokes vectors in four regimes: 0 no polarized absorption
 * (approximate_solve), 1 no Faraday rotation, 2 both, 3 optically thin
 * steps (tau ~ 1e-7: absorb_emit's small-tau series).  err[i] = the largest
 * difference over the twelve gradients, each relative to its own size plus
 * 1e-9 of the largest gradient of its group (Stokes inputs, emissivities,
 * absorptivities, rotativities).  In regime 3 absorb_emit divides by
 * a_P^2 ~ 1e-17, and both forms carry the cancellation that follows. */
__device__ __forceinline__ double vjp_rand(unsigned long long seed, int i, int k)
{
  unsigned long long z = seed * 0x9e3779b97f4a7c15ULL + (unsigned long long)i * 0xbf58476d1ce4e5b9ULL + (unsigned)k;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return (double)(z >> 11) * (1. / 9007199254740992.); /* [0, 1) */
}

__global__ void k_check_step_vjp(int n, unsigned long long seed, double *__restrict__ err, double *__restrict__ info)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = pow(10., -3. + 4. * vjp_rand(seed, i, 0));
  const double aI = pow(10., -5. + 6. * vjp_rand(seed, i, 1));
  const int regime = (int)(vjp_rand(seed, i, 2) * 4.);
  double fq = 2. * vjp_rand(seed, i, 3) - 1., fv = 2. * vjp_rand(seed, i, 4) - 1.;
  const double nf = sqrt(fq * fq + fv * fv) + 1e-300;
  const double pf = 0.98 * vjp_rand(seed, i, 5); /* |a_P| < a_I */
  double aQ = regime == 0 ? 0. : aI * pf * fq / nf, aV = regime == 0 ? 0. : aI * pf * fv / nf;
  const double jI = pow(10., -3. + 4. * vjp_rand(seed, i, 6));
  const double jQ = jI * (2. * vjp_rand(seed, i, 7) - 1.) * 0.7, jV = jI * (2. * vjp_rand(seed, i, 8) - 1.) * 0.3;
  double rQ = pow(10., -4. + 6. * vjp_rand(seed, i, 9)) * (vjp_rand(seed, i, 10) < 0.5 ? -1. : 1.);
  double rV = pow(10., -4. + 6. * vjp_rand(seed, i, 11)) * (vjp_rand(seed, i, 12) < 0.5 ? -1. : 1.);
  if (regime == 1) rQ = rV = 0.;
  if (regime == 3) { /* small optical depths: the series */
    const double s = 1e-7 / (aI * x);
    aQ *= s;
    aV *= s;
  }
  const double aIx = regime == 3 ? 1e-7 / x : aI;
  const double cv[8] = {jI, jQ, jV, aIx, aQ, aV, rQ, rV};
  const double SI = pow(10., -2. + 3. * vjp_rand(seed, i, 13));
  const double S0[4] = {SI, SI * (2. * vjp_rand(seed, i, 14) - 1.) * 0.5, SI * (2. * vjp_rand(seed, i, 15) - 1.) * 0.5,
                        SI * (2. * vjp_rand(seed, i, 16) - 1.) * 0.3};
  const double u[4] = {2. * vjp_rand(seed, i, 17) - 1., 2. * vjp_rand(seed, i, 18) - 1.,
                       2. * vjp_rand(seed, i, 19) - 1., 2. * vjp_rand(seed, i, 20) - 1.};
  double gS[4], gc[8], dS[4], dA[4], dB[4];
  stokes_step_vjp(cv, x, S0, u, gS, gc);
  step_vjp_pass(S0, cv, x, u, 0, dS);
  step_vjp_pass(S0, cv, x, u, 4, dA);
  step_vjp_pass(S0, cv, x, u, 8, dB);
  const double a[12] = {gS[0], gS[1], gS[2], gS[3], gc[0], gc[1], gc[2], gc[3], gc[4], gc[5], gc[6], gc[7]};
  const double b[12] = {dS[0], dS[1], dS[2], dS[3], dA[0], dA[1], dA[2], dA[3], dB[0], dB[1], dB[2], dB[3]};
  /* each gradient against its own size and the scale of its group (the
   * Stokes inputs, the emissivities, the absorptivities, the rotativities) */
  const int grp[12] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3};
  double sc[4] = {0., 0., 0., 0.};
  for (int k = 0; k < 12; k++) sc[grp[k]] = fmax(sc[grp[k]], fabs(b[k]));
  double e = 0.;
  int kw = 0;
  for (int k = 0; k < 12; k++) {
    const double d = fabs(a[k] - b[k]), den = fabs(b[k]) + 1e-9 * sc[grp[k]] + 1e-300;
    const double r = (d != d) ? 1e300 : d / den;
    if (r > e) {
      e = r;
      kw = k;
    }
  }
  err[i] = e;
  /* the case itself: gradient index, both values, regime, x, the eight
   * coefficients and the Stokes vector */
  double *q = info + (size_t)i * 24;
  q[0] = kw;
  q[1] = a[kw];
  q[2] = b[kw];
  q[3] = regime;
  q[4] = x;
  for (int k = 0; k < 8; k++) q[5 + k] = cv[k];
  for (int k = 0; k < 4; k++) q[13 + k] = S0[k];
  q[17] = sc[grp[kw]];
  q[18] = u[0];
  q[19] = u[1];
  q[20] = u[2];
  q[21] = u[3];
}

extern "C" int ipg__check_step_vjp(int device, int n, unsigned long long seed, double max_err[4], double worst[96])
{
  ipg_ctx *ctx = NULL;
  if (n <= 0 || !max_err) return IPG_E_ARG;
  CK(cudaSetDevice(device));
  double *d = NULL;
  CK(cudaMalloc(&d, (size_t)n * 25 * sizeof(double)));
  k_check_step_vjp<<<(n + 127) / 128, 128>>>(n, seed, d, d + n);
  cudaError_t e = cudaGetLastError();
  std::vector<double> h((size_t)n * 25);
  if (e == cudaSuccess) e = cudaMemcpy(h.data(), d, (size_t)n * 25 * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return IPG_E_CUDA;
  int im[4] = {0, 0, 0, 0};
  for (int r = 0; r < 4; r++) max_err[r] = -1.;
  for (int i = 0; i < n; i++) {
    const int r = (int)h[n + (size_t)i * 24 + 3];
    if (r >= 0 && r < 4 && h[i] > max_err[r]) {
      max_err[r] = h[i];
      im[r] = i;
    }
  }
  if (worst)
    for (int r = 0; r < 4; r++)
      for (int k = 0; k < 24; k++) worst[24 * r + k] = h[n + (size_t)im[r] * 24 + k];
  return IPG_OK;
}

/* ===================================================================== */
/* host side                                                              */
/* ===================================================================== */
template <int K>
static int adjoint_wave(ipg_ctx *ctx, int em, const int32_t *d_ij, const int32_t *list, size_t run, double *pool,
                        double *side, double *ckpt, long long n_chunks, int *next, int *first, const double *dL,
                        ipg_pixel_out *d_out, double *g, size_t ncell, int32_t *deferred)
{
  const int threads = 128;
  cudaStream_t st = ctx->stream;
  unsigned long long *cnt = ctx->d_cnt;
  int gb = grid_blocks(ctx, (const void *)k_geodesic<IPG_PLUG_IHARM, 256, IPG_GEO_MINB>, threads, run);
  k_geodesic<IPG_PLUG_IHARM, 256, IPG_GEO_MINB><<<gb, threads, 0, st>>>(d_ij, list, (int)run, pool, ctx->d_chunk_prev,
                                                                        ctx->d_chunk_meta, n_chunks, cnt, ctx->d_rays,
                                                                        deferred, nullptr);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev[2], st)); /* stage boundaries, read by ipg_adjoint */
  if (em == 1) {
    int cb = grid_blocks(ctx, (const void *)k_coeffs<IPG_PLUG_IHARM, 1, true>, threads, (size_t)n_chunks * 32);
    k_coeffs<IPG_PLUG_IHARM, 1, true><<<cb, threads, 0, st>>>(pool, ctx->d_chunk_meta, cnt, n_chunks, ctx->d_rays,
                                                              ctx->d_fields, side);
  } else {
    int cb = grid_blocks(ctx, (const void *)k_coeffs<IPG_PLUG_IHARM, 4, true>, threads, (size_t)n_chunks * 32);
    k_coeffs<IPG_PLUG_IHARM, 4, true><<<cb, threads, 0, st>>>(pool, ctx->d_chunk_meta, cnt, n_chunks, ctx->d_rays,
                                                              ctx->d_fields, side);
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev[3], st));
  if (ctx->xstage < 0 || ctx->xstage == 2) {
    /* the walk of FP64 records with bulk copies into shared memory, as the
     * image's (bit-identical to the walk that loads from global memory) */
    const void *fn = (const void *)k_transfer_bulk<IPG_XFER_WIDE, IPG_XFER_MINB, false, 0, K>;
    const size_t sm = (size_t)threads * XStageOf<0>::T::LANE;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int tb = grid_blocks(ctx, fn, threads, run, sm);
    k_transfer_bulk<IPG_XFER_WIDE, IPG_XFER_MINB, false, 0, K><<<tb, threads, sm, st>>>(
        list, (int)run, pool, ctx->d_chunk_prev, ctx->d_rays, d_out, cnt, ckpt);
  } else {
    int tb = grid_blocks(ctx, (const void *)k_transfer<IPG_XFER_WIDE, IPG_XFER_MINB, false, 0, K>, threads, run);
    k_transfer<IPG_XFER_WIDE, IPG_XFER_MINB, false, 0, K><<<tb, threads, 0, st>>>(
        list, (int)run, pool, ctx->d_chunk_prev, ctx->d_rays, d_out, cnt, ckpt);
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev[4], st));
  k_adj_link<<<4 * ctx->n_sm, 256, 0, st>>>(ctx->d_chunk_prev, ctx->d_chunk_meta, cnt, n_chunks, next, first);
  CK(cudaGetLastError());
  int ab = grid_blocks(ctx, (const void *)k_adjoint<K>, threads, run);
  k_adjoint<K><<<ab, threads, 0, st>>>(list, (int)run, pool, side, ckpt, ctx->d_chunk_prev, next, first, ctx->d_rays,
                                       dL, ctx->d_fields, g, g + ncell, g + 2 * ncell, cnt + CNT_N);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev_pred[0], st));
  int sb = grid_blocks(ctx, (const void *)k_adj_scatter, threads, (size_t)n_chunks * IPG_CHUNK_STEPS);
  k_adj_scatter<<<sb, threads, 0, st>>>(pool, ctx->d_chunk_meta, cnt, n_chunks, ctx->d_rays, side, ctx->d_fields, g,
                                        g + ncell, g + 2 * ncell);
  CK(cudaGetLastError());
  return IPG_OK;
}

extern "C" int ipg_adjoint(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *ij, size_t n, const double *dL_dout,
                           int ckpt_interval, double *grad_ne, double *grad_thetae, double *grad_b,
                           ipg_pixel_out *out)
{
  if (!ctx || !cam || !ij || !dL_dout || n == 0 || n > 0x7fffffff) return IPG_E_ARG;
  if (!ctx->have_model) return IPG_E_STATE;
  const int K = ckpt_interval;
  if (K != 16 && K != 32 && K != 64) {
    snprintf(ctx->err, sizeof(ctx->err), "checkpoint interval %d: 16, 32 or 64", K);
    return IPG_E_ARG;
  }
  if (ctx->plug != IPG_PLUG_IHARM || cam->only_unpolarized || cam->stokes_floors ||
      (cam->emission_type != 4 && cam->emission_type != 1)) {
    snprintf(ctx->err, sizeof(ctx->err),
             "the adjoint needs an iharm dump, a polarized image, thermal emission and no Stokes floors");
    return IPG_E_ARG;
  }
  if (cam->maxnstep < 2 || cam->nx <= 0 || cam->ny <= 0) return IPG_E_ARG;
  CK(cudaSetDevice(ctx->device));
  int rc = ensure_pool(ctx);
  if (rc) return rc;
  rc = ensure_cap(ctx, n);
  if (rc) return rc;
  const size_t ncell = ctx->ncell;
  DevCam dc;
  make_devcam(cam, &dc);
  dc.mixed = 0;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyToSymbolAsync(c_grid, &ctx->dg, sizeof(DevGrid), 0, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyToSymbolAsync(c_plug, &ctx->dp, sizeof(DevPlug), 0, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyToSymbolAsync(c_cam, &dc, sizeof(DevCam), 0, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_ij, ij, 2 * n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  /* the pool per chunk: 32 records, their adjoint blocks, the checkpoints */
  const int KC = K < IPG_CHUNK_STEPS ? K : IPG_CHUNK_STEPS;
  const size_t rec_b = (size_t)IPG_CHUNK_STEPS * IPG_STEP_DOUBLES * sizeof(double);
  const size_t side_b = (size_t)IPG_CHUNK_STEPS * IPG_ADJ_DOUBLES * sizeof(double);
  const size_t ck_b = (size_t)(IPG_CHUNK_STEPS / KC) * 16 * sizeof(double);
  const long long n_chunks = (long long)(((size_t)ctx->n_chunks * rec_b) / (rec_b + side_b + ck_b));
  if (n_chunks < 16) return IPG_E_NOMEM;
  double *pool = ctx->d_pool;
  double *side = pool + (size_t)n_chunks * IPG_CHUNK_STEPS * IPG_STEP_DOUBLES;
  double *ckpt = side + (size_t)n_chunks * IPG_CHUNK_STEPS * IPG_ADJ_DOUBLES;
  /* scratch kept in the context between calls (grow-only) */
  auto grow = [](void **ptr, size_t *cap, size_t bytes) -> cudaError_t {
    if (*cap >= bytes) return cudaSuccess;
    cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e == cudaSuccess) *cap = bytes;
    return e;
  };
#define CKA(call)                       \
  do {                                  \
    cudaError_t e_ = (call);            \
    if (e_ != cudaSuccess) {            \
      return cuda_fail(ctx, e_, #call); \
    }                                   \
  } while (0)
  CKA(grow((void **)&ctx->d_adj_dl, &ctx->adj_dl_cap, 4 * n * sizeof(double)));
  CKA(grow((void **)&ctx->d_adj_g, &ctx->adj_g_cap, 3 * ncell * sizeof(double)));
  CKA(grow((void **)&ctx->d_adj_next, &ctx->adj_next_cap, (size_t)n_chunks * sizeof(int)));
  CKA(grow((void **)&ctx->d_adj_first, &ctx->adj_first_cap, n * sizeof(int)));
  double *dL = ctx->d_adj_dl, *g = ctx->d_adj_g;
  int *next = ctx->d_adj_next, *first = ctx->d_adj_first;
  CKA(cudaMemcpyAsync(dL, dL_dout, 4 * n * sizeof(double), cudaMemcpyHostToDevice, st));
  CKA(cudaMemsetAsync(g, 0, 3 * ncell * sizeof(double), st));
  memset(&ctx->stats, 0, sizeof(ctx->stats));
  /* waves as in the image trace (unsplit, longest predicted rays first):
   * rays that find the pool full go to the next wave, after this wave's
   * adjoint is done */
  rc = sort_by_length(ctx, ctx->d_ij, n, cam);
  if (rc) return rc;
  const int32_t *list = ctx->d_sorted;
  size_t pending = n, wave = n;
  int cur = 0;
  while (pending > 0) {
    size_t run = pending < wave ? pending : wave;
    size_t carry = pending - run;
    int32_t *nextl = ctx->d_list[cur ^ 1];
    unsigned long long h0[CNT_N + 1];
    memset(h0, 0, sizeof(h0));
    h0[CNT_DEFER] = carry;
    CKA(cudaMemcpyAsync(ctx->d_cnt, h0, sizeof(h0), cudaMemcpyHostToDevice, st));
    if (carry) {
      if (list) CKA(cudaMemcpyAsync(nextl, list + run, carry * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
      else k_iota<<<(int)((carry + 255) / 256), 256, 0, st>>>(nextl, (int)carry, (int)run);
    }
    CKA(cudaEventRecord(ctx->ev[0], st));
    const int em = cam->emission_type;
    if (K == 16) rc = adjoint_wave<16>(ctx, em, ctx->d_ij, list, run, pool, side, ckpt, n_chunks, next, first, dL,
                                       ctx->d_out, g, ncell, nextl);
    else if (K == 32) rc = adjoint_wave<32>(ctx, em, ctx->d_ij, list, run, pool, side, ckpt, n_chunks, next, first,
                                            dL, ctx->d_out, g, ncell, nextl);
    else rc = adjoint_wave<64>(ctx, em, ctx->d_ij, list, run, pool, side, ckpt, n_chunks, next, first, dL,
                               ctx->d_out, g, ncell, nextl);
    if (rc) return rc;
    CKA(cudaEventRecord(ctx->ev[1], st));
    unsigned long long h[CNT_N];
    CKA(cudaMemcpyAsync(h, ctx->d_cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
    CKA(cudaStreamSynchronize(st));
    if (h[CNT_STALL]) return stall_fail(ctx);
    float ms = 0.f, t[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&t[0], ctx->ev[0], ctx->ev[2]);
    cudaEventElapsedTime(&t[1], ctx->ev[2], ctx->ev[3]);
    cudaEventElapsedTime(&t[2], ctx->ev[3], ctx->ev[4]);
    cudaEventElapsedTime(&t[3], ctx->ev[4], ctx->ev_pred[0]);
    cudaEventElapsedTime(&t[4], ctx->ev_pred[0], ctx->ev[1]);
    ctx->stats.wall_ms += ms;
    ctx->stats.geodesic_ms += t[0];
    ctx->stats.coeffs_ms += t[1];
    ctx->stats.transfer_ms += t[2];
    ctx->stats.adjoint_ms += t[3];
    ctx->stats.adj_scatter_ms += t[4];
    ctx->stats.ray_steps += h[CNT_STEPS];
    ctx->stats.radiating_steps += h[CNT_RAD];
    ctx->stats.launches += 5;
    ctx->stats.waves += 1;
    size_t deferred = (size_t)h[CNT_DEFER];
    if (deferred == pending) {
      if (run == 1) {
        snprintf(ctx->err, sizeof(ctx->err), "trajectory pool too small for a single ray");
        return IPG_E_NOMEM;
      }
      wave = run / 2;
    }
    pending = deferred;
    cur ^= 1;
    list = ctx->d_list[cur];
  }
  if (grad_ne) CKA(cudaMemcpyAsync(grad_ne, g, ncell * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (grad_thetae) CKA(cudaMemcpyAsync(grad_thetae, g + ncell, ncell * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (grad_b) CKA(cudaMemcpyAsync(grad_b, g + 2 * ncell, ncell * sizeof(double), cudaMemcpyDeviceToHost, st));
  std::vector<ipg_pixel_out> hout(out ? 0 : n);
  ipg_pixel_out *o = out ? out : hout.data();
  CKA(cudaMemcpyAsync(o, ctx->d_out, n * sizeof(ipg_pixel_out), cudaMemcpyDeviceToHost, st));
  CKA(cudaStreamSynchronize(st));
#undef CKA
  for (size_t m = 0; m < n; m++)
    if (o[m].nstep >= cam->maxnstep - 1) {
      snprintf(ctx->err, sizeof(ctx->err), "MaxNStep exceeded in pixel %d %d", ij[2 * m], ij[2 * m + 1]);
      return IPG_E_MAXNSTEP;
    }
  return IPG_OK;
}
