/*
 * Kernels and C-ABI core of the ray pipeline.
 *
 * get_pixel (src/main.c:822-883) runs as three kernels per batch of pixels:
 *
 *   k_geodesic  one lane per ray, camera -> source: init_XK, trace_geodesic /
 *               push_photon with step control and the stop tests
 *               (src/model_geodesics.c:38-293, src/geodesics.c:9-70).  Each
 *               step goes to a record of the trajectory pool together with
 *               the two transport matrices Gamma^i_kl K^l that the polarized
 *               transfer needs there (they come out of the same connection
 *               evaluations).
 *   k_coeffs    one thread per stored step, fully parallel: radiating-region
 *               test, model point query (grid gather, four-vectors), the
 *               synchrotron coefficients of get_jkinv and jar_calc and the
 *               plasma tetrad (model/iharm/model.c:420-593,
 *               src/model_radiation.c:145-332, src/model_tetrads.c:35-127).
 *               None of these depend on the radiation field, so they leave
 *               the sequential loop; the coefficient block replaces the
 *               geodesic state of the record in place.
 *   k_transfer  one lane per ray, source -> camera over the records: parallel
 *               transport of N, the unpolarized and polarized transfer steps
 *               and the camera projection (src/ipolarray.c:59-628).
 *
 * The two sequential kernels take rays from a per-wave queue (one atomic per
 * ray), so lanes stay busy until the queue drains.  Records are chained in
 * chunks of 32 steps (chunk_prev, walked backwards by the transfer) and
 * tagged with their ray and first step (chunk_meta, read by k_coeffs).  Rays
 * that do not fit into the pool are deferred to the next wave.  Every loop is
 * bounded by maxnstep.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <vector>

#include "ipg_device.cuh"
#include "ipg_fits_f32.cuh"
#include "ipg_internal.h"
#include "ipg_plugins.cuh"
#include "ipole_b200.h"

struct RayRec {
  int last_chunk;
  int nstep;
  int status;
  int pad;
};

enum { CNT_POOL = 0, CNT_STEPS = 1, CNT_RAD = 2, CNT_DEFER = 3, CNT_NEXT_G = 4, CNT_NEXT_T = 5, CNT_STALL = 6, CNT_N = 7 };
/* the counters of a batch wave (ipg_batch.cuh) continue the list: transfer
 * items deferred, the wave's step budget (0: none), the budget-spent flag,
 * transfer steps done */
enum { CNT_XDEFER = CNT_N, CNT_BUDGET, CNT_TIMEOUT, CNT_XSTEPS, CNT_NB };

/* ===================================================================== */
/* helpers                                                                */
/* ===================================================================== */

/* src/model_geodesics.c:267-293.  The reference forms three step limits
 * dlx_i = eps c_i / (|K^i| + SS) and returns 1 / sum 1/(|dlx_i| + SS); with
 * a_i = |K^i| + SS and b_i = eps c_i that is
 * dl = eps b1 b2 / (eps (a1 b2 + a2 b1) + a3 b1 b2), one division instead of
 * nine (the + SS of the inner reciprocals matters only for steps near 1e-80,
 * i.e. a ray sitting exactly on the inner or polar boundary). */
__device__ __forceinline__ double stepsize(const double X[4], const double K[4], double eps)
{
  const DevGrid &G = c_grid;
  const double SS = IPG_SMALL * IPG_SMALL;
  const double cut = 0.02;
  double deh = fmin(fabs(X[1] - G.cstartx[1]), 0.1);
  double dpole = fmin(fabs(X[2] * G.inv_lx2), fabs((G.cstopx[2] - X[2]) * G.inv_lx2));
  double d2fac = (dpole < cut) ? dpole * (1. / 3.) : fmin(cut * (1. / 3.) + (dpole - cut) * 10., 1.);
  double a1 = fabs(K[1]) + SS, a2 = fabs(K[2]) + SS, a3 = fabs(K[3]) + SS;
  double b1 = eps * (10 * deh), b2 = eps * d2fac;
  double b12 = b1 * b2;
  return (eps * b12) / (eps * (a1 * b2 + a2 * b1) + a3 * b12);
}

__device__ __forceinline__ double *step_ptr(double *pool, int chunk, int slot)
{
  return pool + ((size_t)chunk * IPG_CHUNK_STEPS + slot) * IPG_STEP_DOUBLES;
}

__device__ __forceinline__ void store4(double *p, double a, double b, double c, double d)
{
  double2 *q = reinterpret_cast<double2 *>(p);
  q[0] = make_double2(a, b);
  q[1] = make_double2(c, d);
}

__device__ __forceinline__ void load4(const double *p, double v[4])
{
  const double2 *q = reinterpret_cast<const double2 *>(p);
  double2 a = q[0], b = q[1];
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}

__device__ __forceinline__ void store_A(double *p, const double A[4][4])
{
#pragma unroll
  for (int i = 0; i < 4; i++) store4(p + 4 * i, A[i][0], A[i][1], A[i][2], A[i][3]);
}

__device__ __forceinline__ void load_A(const double *p, double A[4][4])
{
#pragma unroll
  for (int i = 0; i < 4; i++) load4(p + 4 * i, A[i]);
}

/* Compact step records (IPG_RECORDS_MIXED), same 512-byte stride:
 *   floats  0..15  A1, floats 16..31  A2                      (bytes   0-127)
 *   doubles 16..28 flags ju ku dl jI jQ jV aI aQ aV nturns rQ rV, then
 *                  3 doubles of padding                       (bytes 128-255)
 *   floats 64..79  tetrad rows e1, e2 (covariant), a, b (contravariant)
 *                                                             (bytes 256-319)
 * Every write covers whole 32-byte sectors, so none needs the sector read
 * first.  The geodesic state (doubles 32..47, bytes 256-383) stays where the
 * FP64 layout has it; k_coeffs reads it before writing the coefficients,
 * whose tetrad floats overwrite its first 64 bytes. */
#define RECM_A1F 0
#define RECM_A2F 16
#define RECM_COEF 16
#define RECM_TETF 64
static_assert(RECM_COEF * 2 >= RECM_A2F + 16 && RECM_TETF >= (RECM_COEF + 16) * 2 && RECM_TETF + 16 <= 128,
              "compact record layout");

__device__ __forceinline__ void store_A_f(float *p, const double A[4][4])
{
  float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
  for (int i = 0; i < 4; i++)
    q[i] = make_float4((float)A[i][0], (float)A[i][1], (float)A[i][2], (float)A[i][3]);
}

__device__ __forceinline__ void load_A_f(const float *p, double A[4][4])
{
  const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    float4 v = q[i];
    A[i][0] = v.x;
    A[i][1] = v.y;
    A[i][2] = v.z;
    A[i][3] = v.w;
  }
}

/* A1 (which = 0) or A2 (which = 1) of a record, in the record's layout */
__device__ __forceinline__ void store_A_rec(double *rec, int which, const double A[4][4], int mixed)
{
  if (mixed) store_A_f(reinterpret_cast<float *>(rec) + (which ? RECM_A2F : RECM_A1F), A);
  else store_A(rec + (which ? REC_A2 : REC_A1), A);
}

template <int RM = -1>
__device__ __forceinline__ void load_A_rec(const double *rec, int which, double A[4][4])
{
  if (RM < 0 ? c_cam.mixed : RM) load_A_f(reinterpret_cast<const float *>(rec) + (which ? RECM_A2F : RECM_A1F), A);
  else load_A(rec + (which ? REC_A2 : REC_A1), A);
}

/* Gamma^k_ij K^i K^j = A^k_i K^i */
__device__ __forceinline__ void accel_from_A(const double A[4][4], const double K[4], double acc[4])
{
#pragma unroll
  for (int k = 0; k < 4; k++) acc[k] = A[k][0] * K[0] + A[k][1] * K[1] + A[k][2] * K[2] + A[k][3] * K[3];
}

/* Geodesic state of a record.  Xh3 never enters the fast-light computation
 * and is not kept; X0 rides in the slot after nturns (read only by the
 * trace output, before k_coeffs reuses the slot). */
__device__ __forceinline__ void store_geo(double *p, const double X[4], const double K[4], const double Xh[4],
                                          const double Kh[4], double dl, double nturns, int mixed)
{
  store4(p + REC_X1, X[1], X[2], X[3], dl);
  store4(p + REC_K, K[0], K[1], K[2], K[3]);
  store4(p + REC_XH1, Xh[1], Xh[2], nturns, X[0]); /* X0: for the trace output only */
  /* K at the half step: read only by the per-step trace, which always uses
   * the FP64 layout; the compact layout skips it */
  if (!mixed) store4(p + REC_KH, Kh[0], Kh[1], Kh[2], Kh[3]);
}

/* init_XK, src/model_geodesics.c:178-212, and Kcon *= freq (src/main.c:837).
 * Explicit round-to-nearest operations keep this block free of FMA
 * contraction so the initial wavevector matches the reference's bits. */
__device__ __forceinline__ void init_ray(const DevCam &C, int i, int j, double X[4], double K[4])
{
  double dxoff = __dadd_rn(__ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn((double)i, 0.5), C.xoff), -0.01), (double)C.nx), -0.5);
  double dyoff = __dadd_rn(__ddiv_rn(__dadd_rn(__dadd_rn((double)j, 0.5), C.yoff), (double)C.ny), -0.5);
  double kt1 = __dmul_rn(__dsub_rn(__dmul_rn(dxoff, C.crot), __dmul_rn(dyoff, C.srot)), C.fovx);
  double kt2 = __dmul_rn(__dadd_rn(__dmul_rn(dxoff, C.srot), __dmul_rn(dyoff, C.crot)), C.fovy);
  double kt3 = 1.;
  /* null_normalize, src/geometry.c:190-201 */
  double inorm = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(kt1, kt1), __dmul_rn(kt2, kt2)), __dmul_rn(kt3, kt3)));
  double f = __ddiv_rn(1., inorm);
  double kt[4] = {1., __dmul_rn(kt1, f), __dmul_rn(kt2, f), __dmul_rn(kt3, f)};
  /* tetrad_to_coordinate, src/tetrads.c:22-33 */
#pragma unroll
  for (int l = 0; l < 4; l++) {
    double s = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(C.Econ[0][l], kt[0]), __dmul_rn(C.Econ[1][l], kt[1])),
                                   __dmul_rn(C.Econ[2][l], kt[2])),
                         __dmul_rn(C.Econ[3][l], kt[3]));
    K[l] = __dmul_rn(s, C.freq);
    X[l] = C.Xcam[l];
  }
}

/* ===================================================================== */
/* k_geodesic                                                             */
/* ===================================================================== */
/* Camera of a ray: the context's one camera (CamOne), or a batch's camera
 * table indexed by the ray's camera group (CamTable).  Batched geodesic
 * kernels read the group of each ray from a list; CamOne compiles to the
 * constant-bank reads of the single-image path. */
struct CamOne {
  static constexpr bool batch = false;
  __device__ __forceinline__ static const DevCam &get(int) { return c_cam; }
};
struct CamTable {
  static constexpr bool batch = true;
  __device__ __forceinline__ static const DevCam &get(int g) { return c_cams[g]; }
};

struct GeoLane {
  double X[4], K[4], Xh[4], Kh[4];
  double X1m1, X2m1, X1m2, X2m2; /* sub-ring bookkeeping: X1, X2 of steps n-1, n-2 */
  double h;                      /* -dl of the step in progress */
  double *prev;                  /* record of the last stored step */
  int ray, nstep, chunk, passed, nturns;
  int phase;                     /* 0: next is Gamma at X, 1: Gamma at Xhalf */
  int grp;                       /* camera group of the ray (batches; 0 otherwise) */
};

/* Take the next ray from the wave's queue and store its camera point as
 * step 0; rays that find the pool full are deferred.  False when the queue
 * is empty. */
template <class CS>
__device__ __forceinline__ bool geo_fetch(GeoLane &L, const int32_t *__restrict__ ij, const int32_t *__restrict__ list,
                                          int n_list, double *__restrict__ pool, int *__restrict__ chunk_prev,
                                          int2 *__restrict__ chunk_meta, long long n_chunks,
                                          unsigned long long *__restrict__ counters, RayRec *__restrict__ rays,
                                          int32_t *__restrict__ deferred, const int32_t *__restrict__ ray_grp)
{
  while (true) {
    unsigned long long t = atomicAdd(&counters[CNT_NEXT_G], 1ULL);
    if (t >= (unsigned long long)n_list) return false;
    int ray = list ? list[t] : (int)t;
    if constexpr (CS::batch) {
      /* a batch's step budget: once it is spent no further ray starts */
      const unsigned long long budget = counters[CNT_BUDGET];
      if (budget && *(volatile unsigned long long *)&counters[CNT_STEPS] >= budget) {
        counters[CNT_TIMEOUT] = 1;
        return false;
      }
    }
    const int grp = CS::batch ? ray_grp[ray] : 0;
    const DevCam &C = CS::get(grp);
    long long c = (long long)atomicAdd(&counters[CNT_POOL], 1ULL);
    if (c >= n_chunks) {
      RayRec rec = {-1, 0, IPG_RAY_POOL_FULL, 0};
      rays[ray] = rec;
      deferred[atomicAdd(&counters[CNT_DEFER], 1ULL)] = ray;
      continue;
    }
    L.ray = ray;
    L.grp = grp;
    init_ray(C, ij[2 * ray], ij[2 * ray + 1], L.X, L.K);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      L.Xh[k] = L.X[k];
      L.Kh[k] = L.K[k];
    }
    L.chunk = (int)c;
    chunk_prev[L.chunk] = -1;
    chunk_meta[L.chunk] = make_int2(ray, 0);
    L.prev = step_ptr(pool, L.chunk, 0);
    store_geo(L.prev, L.X, L.K, L.Xh, L.Kh, 0., 0., C.mixed);
    L.nstep = 0;
    L.phase = 0;
    L.h = 0.;
    L.passed = (C.Xcam[2] < 0.5) ? 1 : ((C.Xcam[2] > 0.5) ? -1 : 0);
    L.nturns = 0;
    L.X1m1 = L.X1m2 = L.X[1];
    L.X2m1 = L.X2m2 = L.X[2];
    return true;
  }
}

/* Sub-ring counter, src/model_geodesics.c:129-165, after step nstep */
template <int MET>
__device__ __forceinline__ void count_turns(const DevCam &C, GeoLane &L)
{
  if (L.passed != 0) {
    if (L.passed > 0) {
      if (L.X[2] > 0.5) L.passed = 0;
    } else {
      if (L.X[2] < 0.5) L.passed = 0;
    }
  } else if (L.nstep > 3) {
    if (C.subring_dtheta == 1) {
      double dX2a = L.X2m1 - L.X2m2, dX2b = L.X[2] - L.X2m1;
      if (dX2a * dX2b < 0) L.nturns++;
    } else {
      double ra = geo_r<MET>(L.X1m2), rb = geo_r<MET>(L.X1m1), rc = geo_r<MET>(L.X[1]);
      double za = ra * cos(bl_theta<MET>(L.X1m2, L.X2m2)), zb = rb * cos(bl_theta<MET>(L.X1m1, L.X2m1));
      double zc = rc * cos(bl_theta<MET>(L.X[1], L.X[2]));
      if ((zb - za) * (zc - zb) < 0) L.nturns++;
    }
  }
  L.X1m2 = L.X1m1;
  L.X2m2 = L.X2m1;
  L.X1m1 = L.X[1];
  L.X2m1 = L.X[2];
}

/* One loop iteration is one half of push_photon (src/geodesics.c:9-70):
 * the connection at X (phase 0) or at Xhalf (phase 1).  Lanes of a warp in
 * different phases still run the connection code together, and the kernel
 * holds one copy of it, which keeps the loop body small: a lone ray's step
 * time is set by instruction-fetch and dependency latency, not by the FP64
 * throughput of the SM. */
#ifndef IPG_COEF_EM_SPECIALIZE
#define IPG_COEF_EM_SPECIALIZE 1
#endif
#ifndef IPG_GEO_FULLSTEP
#define IPG_GEO_FULLSTEP 0 /* whole midpoint steps (build option) */
#endif
template <int P, int TPB = 256, int MINB = IPG_GEO_MINB, bool FULL = (IPG_GEO_FULLSTEP != 0), class CS = CamOne>
__global__ void __launch_bounds__(TPB, MINB)
    k_geodesic(const int32_t *__restrict__ ij, const int32_t *__restrict__ list, int n_list,
               double *__restrict__ pool, int *__restrict__ chunk_prev, int2 *__restrict__ chunk_meta,
               long long n_chunks, unsigned long long *__restrict__ counters, RayRec *__restrict__ rays,
               int32_t *__restrict__ deferred, const int32_t *__restrict__ ray_grp, int *started = nullptr)
{
  const DevGrid &G = c_grid;
  /* a block marks its start in host memory when asked (the host waits for
   * the longest class's blocks to be resident before it launches the other
   * classes) */
  if (started && threadIdx.x == 0) {
    *(volatile int *)(started + blockIdx.x) = 1;
    __threadfence_system();
  }
  GeoLane L;
  bool has = geo_fetch<CS>(L, ij, list, n_list, pool, chunk_prev, chunk_meta, n_chunks, counters, rays, deferred, ray_grp);
  if constexpr (FULL) {
  /* One iteration is one whole midpoint step.  The second connection is
   * taken at Xhalf = X + h K / 2, which needs only the step size, not the
   * first connection: the two connections are independent chains, evaluated
   * side by side; only their contractions with K and Khalf are sequential.
   * It takes 250 registers instead of 226 and gives the same records. */
  while (__any_sync(0xffffffffu, has)) {
    if (!has) continue;
    const DevCam &C = CS::get(L.grp);
    const int pol = !C.unpol;
    const int track = C.target_nturns >= 0;
    /* stop_backward_integration, src/model_geodesics.c:218-254, and the step
     * limit of trace_geodesic's loop (:71) */
    double r = geo_r<PlugT<P>::MET>(L.X[1]);
    if ((r > G.rmax_geo && L.K[1] < 0.) || r < (G.Rh + 0.0001) || !(L.nstep < C.maxnstep - 1)) {
      int status = (L.nstep >= C.maxnstep - 1) ? IPG_RAY_MAXNSTEP : IPG_RAY_OK;
      if (status == IPG_RAY_OK && pol && L.nstep != 0) {
        /* the walk back starts at the last point: its Gamma(X) K too */
        Conn cn;
        double A[4][4];
        fd_connection<PlugT<P>::MET>(L.X[1], L.X[2], &cn);
        transport_matrix(cn, L.K, A);
        store_A_rec(L.prev, 0, A, C.mixed);
      }
      RayRec rec = {L.chunk, L.nstep, status, 0};
      rays[L.ray] = rec;
      atomicAdd(&counters[CNT_STEPS], (unsigned long long)L.nstep);
      has = geo_fetch<CS>(L, ij, list, n_list, pool, chunk_prev, chunk_meta, n_chunks, counters, rays, deferred, ray_grp);
      continue;
    }
    L.nstep++;
    L.h = -stepsize(L.X, L.K, C.eps);
#pragma unroll
    for (int k = 0; k < 4; k++) L.Xh[k] = L.X[k] + 0.5 * L.h * L.K[k];
    Conn c0, c1;
    fd_connection<PlugT<P>::MET>(L.X[1], L.X[2], &c0);
    fd_connection<PlugT<P>::MET>(L.Xh[1], L.Xh[2], &c1);
    double acc[4], A[4][4];
    if (pol) {
      transport_matrix(c0, L.K, A);
      accel_from_A(A, L.K, acc);
      store_A_rec(L.prev, 0, A, C.mixed);
    } else {
      geo_accel(c0, L.K, acc);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) L.Kh[k] = L.K[k] - 0.5 * L.h * acc[k];
    if (pol) {
      transport_matrix(c1, L.Kh, A);
      accel_from_A(A, L.Kh, acc);
    } else {
      geo_accel(c1, L.Kh, acc);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      L.K[k] = L.K[k] - L.h * acc[k];
      L.X[k] = L.X[k] + L.h * L.Kh[k];
    }
    double dl = -L.h;
    double dl_cgs = dl * G.L_unit * IPG_HPL / (IPG_ME * IPG_CL * IPG_CL);
    if (track) count_turns<PlugT<P>::MET>(C, L);
    int slot = L.nstep % IPG_CHUNK_STEPS;
    if (slot == 0) {
      long long nc = (long long)atomicAdd(&counters[CNT_POOL], 1ULL);
      if (nc >= n_chunks) {
        RayRec rec = {L.chunk, L.nstep, IPG_RAY_POOL_FULL, 0};
        rays[L.ray] = rec;
        deferred[atomicAdd(&counters[CNT_DEFER], 1ULL)] = L.ray;
        has = geo_fetch<CS>(L, ij, list, n_list, pool, chunk_prev, chunk_meta, n_chunks, counters, rays, deferred, ray_grp);
        continue;
      }
      chunk_prev[(int)nc] = L.chunk;
      chunk_meta[(int)nc] = make_int2(L.ray, L.nstep);
      L.chunk = (int)nc;
    }
    L.prev = step_ptr(pool, L.chunk, slot);
    store_geo(L.prev, L.X, L.K, L.Xh, L.Kh, dl_cgs, (double)L.nturns, C.mixed);
    if (pol) store_A_rec(L.prev, 1, A, C.mixed); /* Gamma(Xh_n) Kh_n */
  }
  } else {
  while (__any_sync(0xffffffffu, has)) {
    if (!has) continue;
    const DevCam &C = CS::get(L.grp);
    const int pol = !C.unpol;
    const int track = C.target_nturns >= 0;
    const int ph = L.phase;
    int stop = 0;
    if (ph == 0) {
      /* stop_backward_integration, src/model_geodesics.c:218-254, and the
       * step limit of trace_geodesic's loop (:71) */
      double r = geo_r<PlugT<P>::MET>(L.X[1]);
      if ((r > G.rmax_geo && L.K[1] < 0.) || r < (G.Rh + 0.0001) || !(L.nstep < C.maxnstep - 1)) {
        int status = (L.nstep >= C.maxnstep - 1) ? IPG_RAY_MAXNSTEP : IPG_RAY_OK;
        if (status != IPG_RAY_OK || !pol || L.nstep == 0) {
          RayRec rec = {L.chunk, L.nstep, status, 0};
          rays[L.ray] = rec;
          atomicAdd(&counters[CNT_STEPS], (unsigned long long)L.nstep);
          has = geo_fetch<CS>(L, ij, list, n_list, pool, chunk_prev, chunk_meta, n_chunks, counters, rays, deferred, ray_grp);
          continue;
        }
        stop = 1; /* the walk back starts at the last point: its Gamma(X) K too */
      }
    }
    double Ke[4];
#pragma unroll
    for (int k = 0; k < 4; k++) Ke[k] = ph ? L.Kh[k] : L.K[k];
    Conn cn;
    double acc[4], A[4][4];
    fd_connection<PlugT<P>::MET>(ph ? L.Xh[1] : L.X[1], ph ? L.Xh[2] : L.X[2], &cn);
    if (pol) {
      /* the transfer needs Gamma K at X_n and at Xhalf_n for each step */
      transport_matrix(cn, Ke, A);
      accel_from_A(A, Ke, acc);
    } else {
      geo_accel(cn, Ke, acc);
    }
    if (ph == 0) {
      if (pol) store_A_rec(L.prev, 0, A, C.mixed);
      if (stop) {
        RayRec rec = {L.chunk, L.nstep, IPG_RAY_OK, 0};
        rays[L.ray] = rec;
        atomicAdd(&counters[CNT_STEPS], (unsigned long long)L.nstep);
        has = geo_fetch<CS>(L, ij, list, n_list, pool, chunk_prev, chunk_meta, n_chunks, counters, rays, deferred, ray_grp);
        continue;
      }
      L.nstep++;
      L.h = -stepsize(L.X, L.K, C.eps);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        L.Kh[k] = L.K[k] - 0.5 * L.h * acc[k];
        L.Xh[k] = L.X[k] + 0.5 * L.h * L.K[k];
      }
      L.phase = 1;
      continue;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      L.K[k] = L.K[k] - L.h * acc[k];
      L.X[k] = L.X[k] + L.h * L.Kh[k];
    }
    L.phase = 0;
    double dl = -L.h;
    double dl_cgs = dl * G.L_unit * IPG_HPL / (IPG_ME * IPG_CL * IPG_CL);
    if (track) count_turns<PlugT<P>::MET>(C, L);
    int slot = L.nstep % IPG_CHUNK_STEPS;
    if (slot == 0) {
      long long nc = (long long)atomicAdd(&counters[CNT_POOL], 1ULL);
      if (nc >= n_chunks) {
        RayRec rec = {L.chunk, L.nstep, IPG_RAY_POOL_FULL, 0};
        rays[L.ray] = rec;
        deferred[atomicAdd(&counters[CNT_DEFER], 1ULL)] = L.ray;
        has = geo_fetch<CS>(L, ij, list, n_list, pool, chunk_prev, chunk_meta, n_chunks, counters, rays, deferred, ray_grp);
        continue;
      }
      chunk_prev[(int)nc] = L.chunk;
      chunk_meta[(int)nc] = make_int2(L.ray, L.nstep);
      L.chunk = (int)nc;
    }
    L.prev = step_ptr(pool, L.chunk, slot);
    store_geo(L.prev, L.X, L.K, L.Xh, L.Kh, dl_cgs, (double)L.nturns, C.mixed);
    if (pol) store_A_rec(L.prev, 1, A, C.mixed); /* Gamma(Xh_n) Kh_n */
  }
  }
}


/* Step count of each ray at a coarser accuracy (eps_scale x eps), without
 * storing anything: a cheap prediction of the ray lengths, so that the full
 * trace can start the longest rays first.  pred[t] is the count of list
 * entry t; a ray whose position turns non-finite, or that passes step_cap,
 * stops there.  CS, ray_grp: the camera of each ray, as in k_geodesic. */
template <int P, class CS = CamOne>
__global__ void __launch_bounds__(128, IPG_GEO_MINB)
    k_geodesic_count(const int32_t *__restrict__ ij, const int32_t *__restrict__ list, int n_list, double eps_scale,
                     int step_cap, int32_t *__restrict__ pred, unsigned long long *__restrict__ counter,
                     const int32_t *__restrict__ ray_grp)
{
  const DevGrid &G = c_grid;
  double eps = 0.;
  double X[4], K[4], Xh[4], Kh[4], h = 0.;
  int t = -1, nstep = 0, phase = 0;
  bool has = false, drained = false;
  while (true) {
    if (!has && !drained) {
      unsigned long long q = atomicAdd(counter, 1ULL);
      has = q < (unsigned long long)n_list;
      drained = !has;
      if (has) {
        t = (int)q;
        int ray = list ? list[t] : t;
        const DevCam &C = CS::get(ray_grp ? ray_grp[ray] : 0);
        init_ray(C, ij[2 * ray], ij[2 * ray + 1], X, K);
        eps = C.eps * eps_scale;
        nstep = 0;
        phase = 0;
      }
    }
    if (!__any_sync(0xffffffffu, has)) break;
    if (!has) continue;
    if (phase == 0) {
      double r = geo_r<PlugT<P>::MET>(X[1]);
      if ((r > G.rmax_geo && K[1] < 0.) || r < (G.Rh + 0.0001) || !(nstep < step_cap) || !isfinite(X[1])) {
        pred[t] = nstep;
        has = false;
        continue;
      }
    }
    double Ke[4];
#pragma unroll
    for (int k = 0; k < 4; k++) Ke[k] = phase ? Kh[k] : K[k];
    Conn cn;
    double acc[4];
    fd_connection<PlugT<P>::MET>(phase ? Xh[1] : X[1], phase ? Xh[2] : X[2], &cn);
    geo_accel(cn, Ke, acc);
    if (phase == 0) {
      nstep++;
      h = -stepsize(X, K, eps);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        Kh[k] = K[k] - 0.5 * h * acc[k];
        Xh[k] = X[k] + 0.5 * h * K[k];
      }
      phase = 1;
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        K[k] = K[k] - h * acc[k];
        X[k] = X[k] + h * Kh[k];
      }
      phase = 0;
    }
  }
}

/* ===================================================================== */
/* k_coeffs                                                               */
/* ===================================================================== */
/* One thread per stored step s of a finished ray: everything the transfer
 * step ending at s needs that does not depend on the radiation field.  The
 * record's geodesic block is overwritten by the coefficient block; dl and
 * nturns keep their slots. */
/* ADJ (the adjoint's forward pass, iharm only): each radiating or last
 * record also leaves an adjoint block of IPG_ADJ_DOUBLES in adj_side:
 * X1 X2 X3, the fluid frequency, sin and cos of the k-B angle, the angle,
 * and (along | in_domain << 1), from which the adjoint re-evaluates the fits
 * with their derivatives.  F32: the thermal fits with FP32 shapes
 * (jar_both_f32). */
#define IPG_ADJ_DOUBLES 8
template <int P, int EM = 0, bool ADJ = false, bool F32 = false>
__global__ void __launch_bounds__(128, IPG_COEF_MINB)
    k_coeffs(double *__restrict__ pool, const int2 *__restrict__ chunk_meta,
             const unsigned long long *__restrict__ counters, long long n_chunks,
             const RayRec *__restrict__ rays, const double *__restrict__ fields, double *__restrict__ adj_side)
{
  const DevGrid &G = c_grid;
  const DevCam &C = c_cam;
  const int pol = !C.unpol;
  long long used = (long long)counters[CNT_POOL];
  if (used > n_chunks) used = n_chunks;
  const long long total = used * IPG_CHUNK_STEPS;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int c = (int)(t / IPG_CHUNK_STEPS), slot = (int)(t % IPG_CHUNK_STEPS);
    int2 meta = chunk_meta[c];
    RayRec rec = rays[meta.x];
    int s = meta.y + slot;
    if (rec.status != IPG_RAY_OK || s > rec.nstep) continue;
    double *p = step_ptr(pool, c, slot);
    double X1 = p[REC_X1], X2 = p[REC_X2], X3 = p[REC_X3];
    double K[4];
    load4(p + REC_K, K);
    PointGeo pg;
    point_geo<PlugT<P>::MET>(X1, X2, &pg);
    int flags = radiating_t<P>(pg) ? 1 : 0;
    /* isolate_counterjet, src/ipolarray.c:128-136 */
    if (C.counterjet == 1) {
      if (X2 < (G.cstopx[2] - G.cstartx[2]) / 2) flags |= 2;
    } else if (C.counterjet == 2) {
      if (X2 > (G.cstopx[2] - G.cstartx[2]) / 2) flags |= 2;
    }
    double ju = 0., ku = 0.;
    Jar jar = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0.};
    double e1[4] = {0., 0., 0., 0.}, e2[4] = {0., 0., 0., 0.}, Econ[4][4];
#pragma unroll
    for (int q = 0; q < 4; q++) Econ[1][q] = Econ[2][q] = 0.;
    /* get_jkinv at every radiating point and at the far end of the ray
     * (src/ipolarray.c:74,143); jar_calc and the tetrad of evolve_N
     * (src/ipolarray.c:357-384) at radiating points */
    if ((flags & 1) || s == rec.nstep) {
      ModelPt mp;
      model_point_t<P>(fields, X1, X2, X3, pg, &mp);
      int want_pol = pol && (flags & 1);
      coeffs_t<P, F32>(mp, K, want_pol, EM ? EM : C.emission_type, &ju, &ku, &jar);
      if constexpr (ADJ) {
        JarGeo jg;
        jar_geo(mp, K, EM ? EM : C.emission_type, &jg);
        double *q = adj_side + ((size_t)c * IPG_CHUNK_STEPS + slot) * IPG_ADJ_DOUBLES;
        store4(q, X1, X2, X3, jg.nu);
        store4(q + 4, jg.sth, jg.cth, jg.theta, (double)(jg.along | (mp.in_domain << 1)));
      }
      if (want_pol) {
        double Bcon[4] = {mp.Bcon[0], mp.Bcon[1], mp.Bcon[2], mp.Bcon[3]};
        double bsq = Bcon[0] * mp.Bcov[0] + Bcon[1] * mp.Bcov[1] + Bcon[2] * mp.Bcov[2] + Bcon[3] * mp.Bcov[3];
        if (bsq <= 0.) {
          Bcon[0] = 0.;
          Bcon[1] = 1.;
          Bcon[2] = 1.;
          Bcon[3] = 1.;
        }
        int tf = plasma_tetrad<PlugT<P>::MET>(mp.Ucon, K, Bcon, mp.geo.g, mp.geo, Econ, e1, e2);
        if (isnan(mp.Ucov[0])) tf |= 8;
        flags |= tf << 2;
      }
    }
    if (C.mixed) {
      /* the compact layout: coefficients in FP64, tetrad rows in FP32; dl and
       * nturns move from the geodesic state, which this pass has not yet
       * overwritten */
      const double dl_rec = p[REC_DL], nturns_rec = p[REC_NTURNS];
      double *q = p + RECM_COEF;
      store4(q, (double)flags, ju, ku, dl_rec);
      store4(q + 4, jar.jI, jar.jQ, jar.jV, jar.aI);
      store4(q + 8, jar.aQ, jar.aV, nturns_rec, jar.rQ);
      store4(q + 12, jar.rV, 0., 0., 0.); /* padding: whole sectors */
      float4 *t = reinterpret_cast<float4 *>(reinterpret_cast<float *>(p) + RECM_TETF);
      t[0] = make_float4((float)e1[0], (float)e1[1], (float)e1[2], (float)e1[3]);
      t[1] = make_float4((float)e2[0], (float)e2[1], (float)e2[2], (float)e2[3]);
      t[2] = make_float4((float)Econ[1][0], (float)Econ[1][1], (float)Econ[1][2], (float)Econ[1][3]);
      t[3] = make_float4((float)Econ[2][0], (float)Econ[2][1], (float)Econ[2][2], (float)Econ[2][3]);
      continue;
    }
    p[REC_FLAGS] = (double)flags;
    p[REC_JU] = ju;
    p[REC_KU] = ku;
    store4(p + REC_JI, jar.jI, jar.jQ, jar.jV, jar.aI);
    p[REC_JI + 4] = jar.aQ;
    p[REC_JI + 5] = jar.aV;
    p[REC_RQ] = jar.rQ;
    p[REC_RV] = jar.rV;
    store4(p + REC_E1COV, e1[0], e1[1], e1[2], e1[3]);
    store4(p + REC_E2COV, e2[0], e2[1], e2[2], e2[3]);
    store4(p + REC_E1CON, Econ[1][0], Econ[1][1], Econ[1][2], Econ[1][3]);
    store4(p + REC_E2CON, Econ[2][0], Econ[2][1], Econ[2][2], Econ[2][3]);
  }
}

/* ===================================================================== */
/* k_transfer                                                             */
/* ===================================================================== */
/* The coefficient block of one step record (k_coeffs' output), loaded with
 * 16 two-double loads issued together: the transfer step then waits for one
 * round trip to memory instead of two (flags first, the rest behind the
 * radiating branch). */
struct CoefBlock {
  double flags, ju, ku, dl, jI, jQ, jV, aI, aQ, aV, nturns, rQ, rV;
  double e1[4], e2[4], a[4], b[4]; /* tetrad rows 1, 2: covariant, contravariant */
};

__device__ __forceinline__ void load_coef(const double *__restrict__ p, CoefBlock &c)
{
  const double2 *q = reinterpret_cast<const double2 *>(p + REC_FLAGS);
  double2 v[16];
#pragma unroll
  for (int k = 0; k < 16; k++) v[k] = q[k];
  c.flags = v[0].x;
  c.ju = v[0].y;
  c.ku = v[1].x;
  c.dl = v[1].y;
  c.jI = v[2].x;
  c.jQ = v[2].y;
  c.jV = v[3].x;
  c.aI = v[3].y;
  c.aQ = v[4].x;
  c.aV = v[4].y;
  c.nturns = v[5].x;
  c.rQ = v[5].y;
  c.rV = v[6].x;
  c.e1[0] = v[8].x; c.e1[1] = v[8].y; c.e1[2] = v[9].x; c.e1[3] = v[9].y;
  c.e2[0] = v[10].x; c.e2[1] = v[10].y; c.e2[2] = v[11].x; c.e2[3] = v[11].y;
  c.a[0] = v[12].x; c.a[1] = v[12].y; c.a[2] = v[13].x; c.a[3] = v[13].y;
  c.b[0] = v[14].x; c.b[1] = v[14].y; c.b[2] = v[15].x; c.b[3] = v[15].y;
}
static_assert(REC_FLAGS == 32 && REC_JU == 33 && REC_KU == 34 && REC_DL == 35 && REC_JI == 36 &&
                  REC_NTURNS == 42 && REC_RQ == 43 && REC_RV == 44 && REC_E1COV == 48 && REC_E2COV == 52 &&
                  REC_E1CON == 56 && REC_E2CON == 60,
              "load_coef follows the record layout");

/* the same from a compact record (IPG_RECORDS_MIXED) */
__device__ __forceinline__ void load_coef_m(const double *__restrict__ p, CoefBlock &c)
{
  const double2 *q = reinterpret_cast<const double2 *>(p + RECM_COEF);
  double2 v[7];
#pragma unroll
  for (int k = 0; k < 7; k++) v[k] = q[k];
  const float4 *t = reinterpret_cast<const float4 *>(reinterpret_cast<const float *>(p) + RECM_TETF);
  float4 w[4];
#pragma unroll
  for (int k = 0; k < 4; k++) w[k] = t[k];
  c.flags = v[0].x;
  c.ju = v[0].y;
  c.ku = v[1].x;
  c.dl = v[1].y;
  c.jI = v[2].x;
  c.jQ = v[2].y;
  c.jV = v[3].x;
  c.aI = v[3].y;
  c.aQ = v[4].x;
  c.aV = v[4].y;
  c.nturns = v[5].x;
  c.rQ = v[5].y;
  c.rV = v[6].x;
  c.e1[0] = w[0].x; c.e1[1] = w[0].y; c.e1[2] = w[0].z; c.e1[3] = w[0].w;
  c.e2[0] = w[1].x; c.e2[1] = w[1].y; c.e2[2] = w[1].z; c.e2[3] = w[1].w;
  c.a[0] = w[2].x; c.a[1] = w[2].y; c.a[2] = w[2].z; c.a[3] = w[2].w;
  c.b[0] = w[3].x; c.b[1] = w[3].y; c.b[2] = w[3].z; c.b[3] = w[3].w;
}

/* evolve_N (src/ipolarray.c:332-575) from a coefficient block: N to Stokes
 * in the plasma tetrad, Faraday half step, absorption/emission, Faraday half
 * step, back to N.  Returns the tauF / NaN oddflag bits. */
__device__ __forceinline__ int evolve_N_coef(const CoefBlock &cb, double dlam, int zero_emission, HermN *N,
                                             double *tauF, int stokes_floors)
{
  Jar c;
  c.jI = cb.jI;
  c.jQ = cb.jQ;
  c.jV = cb.jV;
  c.aI = cb.aI;
  c.aQ = cb.aQ;
  c.aV = cb.aV;
  c.rQ = cb.rQ;
  c.rV = cb.rV;
  c.jU = c.aU = c.rU = 0.;
  if (zero_emission) c.jI = c.jQ = c.jU = c.jV = 0.;
  double T11, T22, T12r, T21i;
  hn_stokes(*N, cb.e1, cb.e2, &T11, &T22, &T12r, &T21i);
  double SI = (T11 + T22) / 2, SQ = (T11 - T22) / 2, SU = T12r, SV = T21i;
  const FaradayRot R = faraday_rot(c.rQ, c.rU, c.rV, dlam * 0.5);
  faraday_apply(R, c.rQ, c.rU, c.rV, &SQ, &SU, &SV);
  absorb_emit(c, dlam, &SI, &SQ, &SU, &SV);
  faraday_apply(R, c.rQ, c.rU, c.rV, &SQ, &SU, &SV);
  *tauF += dlam * fabs(c.rV);
  if (stokes_floors) {
    if (SI < 0) {
      SI = SQ = SU = SV = 0;
    } else {
      double pf = sqrt(SQ * SQ + SU * SU + SV * SV) / SI;
      if (pf > 1.) {
        SQ /= pf;
        SU /= pf;
        SV /= pf;
      }
    }
  }
  /* N += Econ^T (new block - old block) Econ (stokes_to_tensor +
   * complex_tetrad_to_coord_rank2, src/ipolarray.c:673-682, 730-748) */
  const double *a = cb.a, *b = cb.b;
  double d11 = (SI + SQ) - T11, d22 = (SI - SQ) - T22, dr12 = SU - T12r, di21 = SV - T21i;
#define DR(i, j) (a[i] * a[j] * d11 + b[i] * b[j] * d22 + (a[i] * b[j] + b[i] * a[j]) * dr12)
#define DS(i, j) ((b[i] * a[j] - a[i] * b[j]) * di21)
  N->r00 += DR(0, 0); N->r01 += DR(0, 1); N->r02 += DR(0, 2); N->r03 += DR(0, 3);
  N->r11 += DR(1, 1); N->r12 += DR(1, 2); N->r13 += DR(1, 3);
  N->r22 += DR(2, 2); N->r23 += DR(2, 3); N->r33 += DR(3, 3);
  N->s01 += DS(0, 1); N->s02 += DS(0, 2); N->s03 += DS(0, 3);
  N->s12 += DS(1, 2); N->s13 += DS(1, 3); N->s23 += DS(2, 3);
#undef DR
#undef DS
  int flag = 0;
  if (*tauF > 1.e100 || *tauF < -1.e100 || isnan(*tauF)) flag |= 2;
  if (isnan(N->r00) || isnan(SI)) flag |= 4;
  return flag;
}



/* push_polar (src/ipolarray.c:253-289) with its increment in FP32, for the
 * FP32-step kernel: Mh is scaled by a power of two taken from its largest
 * diagonal entry (for N = sum f f^dagger every |N^ij| is at most the largest
 * N^ii), the products A Mh run in FP32, and the unscaled increment is
 * subtracted from base in FP64. */
__device__ __forceinline__ void hn_push_f32(const HermN &base, const HermN &Mh, const double A[4][4], double dl,
                                            HermN *out)
{
  const double big = fmax(fmax(fabs(Mh.r00), fabs(Mh.r11)), fmax(fmax(fabs(Mh.r22), fabs(Mh.r33)), 1e-300));
  const int ex = ilogb(big);
  const double sc = ldexp(1.0, -ex), us = ldexp(dl, ex);
  const float r00 = (float)(Mh.r00 * sc), r01 = (float)(Mh.r01 * sc), r02 = (float)(Mh.r02 * sc),
              r03 = (float)(Mh.r03 * sc), r11 = (float)(Mh.r11 * sc), r12 = (float)(Mh.r12 * sc),
              r13 = (float)(Mh.r13 * sc), r22 = (float)(Mh.r22 * sc), r23 = (float)(Mh.r23 * sc),
              r33 = (float)(Mh.r33 * sc);
  const float s01 = (float)(Mh.s01 * sc), s02 = (float)(Mh.s02 * sc), s03 = (float)(Mh.s03 * sc),
              s12 = (float)(Mh.s12 * sc), s13 = (float)(Mh.s13 * sc), s23 = (float)(Mh.s23 * sc);
  const float R[4][4] = {{r00, r01, r02, r03}, {r01, r11, r12, r13}, {r02, r12, r22, r23}, {r03, r13, r23, r33}};
  const float S[4][4] = {{0.f, s01, s02, s03}, {-s01, 0.f, s12, s13}, {-s02, -s12, 0.f, s23}, {-s03, -s13, -s23, 0.f}};
  float Af[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) Af[i][j] = (float)A[i][j];
  float AR[4][4], AS[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      AR[i][j] = Af[i][0] * R[0][j] + Af[i][1] * R[1][j] + Af[i][2] * R[2][j] + Af[i][3] * R[3][j];
      AS[i][j] = Af[i][0] * S[0][j] + Af[i][1] * S[1][j] + Af[i][2] * S[2][j] + Af[i][3] * S[3][j];
    }
  out->r00 = base.r00 - us * (double)(AR[0][0] + AR[0][0]);
  out->r01 = base.r01 - us * (double)(AR[0][1] + AR[1][0]);
  out->r02 = base.r02 - us * (double)(AR[0][2] + AR[2][0]);
  out->r03 = base.r03 - us * (double)(AR[0][3] + AR[3][0]);
  out->r11 = base.r11 - us * (double)(AR[1][1] + AR[1][1]);
  out->r12 = base.r12 - us * (double)(AR[1][2] + AR[2][1]);
  out->r13 = base.r13 - us * (double)(AR[1][3] + AR[3][1]);
  out->r22 = base.r22 - us * (double)(AR[2][2] + AR[2][2]);
  out->r23 = base.r23 - us * (double)(AR[2][3] + AR[3][2]);
  out->r33 = base.r33 - us * (double)(AR[3][3] + AR[3][3]);
  out->s01 = base.s01 - us * (double)(AS[0][1] - AS[1][0]);
  out->s02 = base.s02 - us * (double)(AS[0][2] - AS[2][0]);
  out->s03 = base.s03 - us * (double)(AS[0][3] - AS[3][0]);
  out->s12 = base.s12 - us * (double)(AS[1][2] - AS[2][1]);
  out->s13 = base.s13 - us * (double)(AS[1][3] - AS[3][1]);
  out->s23 = base.s23 - us * (double)(AS[2][3] - AS[3][2]);
}

/* (1 - e^-t) / t, bounded for every t (its limit 1 at t = 0) */
__device__ __forceinline__ float one_minus_exp_over(float t)
{
  return (fabsf(t) < 1e-6f) ? 1.f - 0.5f * t : -expm1f(-t) / t;
}

/* The same Faraday and absorption/emission step as evolve_N_coef, in FP32
 * (ipg_set_step_precision, IPG_STEP_FP32).  It is written in optical depths
 * tau = alpha dl and emission j dl: the divisions by alpha of absorb_emit
 * (src/ipolarray.c:410-500) become (1 - e^-tau) / tau factors, bounded for
 * optically thin points where 1/alpha would overflow FP32.  S and j dl are
 * scaled by one power of two taken from the step's magnitudes, so that the
 * FP32 values stay in range (the step is linear in S and j, so the scaling is
 * exact).  The Faraday angle is reduced modulo 2 pi in FP64 before its FP32
 * sine and cosine.  The N to Stokes projection and the update of N stay
 * FP64, so the accumulation along the ray is FP64. */
__device__ __forceinline__ int evolve_N_coef_f32(const CoefBlock &cb, double dlam, int zero_emission, HermN *N,
                                              double *tauF, int stokes_floors)
{
  double T11, T22, T12r, T21i;
  hn_stokes(*N, cb.e1, cb.e2, &T11, &T22, &T12r, &T21i);
  const double SId = (T11 + T22) / 2, SQd = (T11 - T22) / 2, SUd = T12r, SVd = T21i;
  const double jxId = zero_emission ? 0. : cb.jI * dlam, jxQd = zero_emission ? 0. : cb.jQ * dlam,
               jxVd = zero_emission ? 0. : cb.jV * dlam;
  const int ex = ilogb(fmax(fmax(fabs(SId), fabs(jxId)), 1e-300));
  const double sc = ldexp(1.0, -ex);
  float SI = (float)(SId * sc), SQ = (float)(SQd * sc), SU = (float)(SUd * sc), SV = (float)(SVd * sc);
  const float jI = (float)(jxId * sc), jQ = (float)(jxQd * sc), jV = (float)(jxVd * sc);
  /* Faraday half step (rU = 0): S turns about r by rho dl / 2 */
  const double rho2 = cb.rQ * cb.rQ + cb.rV * cb.rV;
  float fc, fs, fg, nQ, nV;
  if (rho2 > IPG_CUT_PREVENT_NAN) {
    const double rho = sqrt(rho2), phi = rho * dlam * 0.5;
    const float ph = (float)remainder(phi, 2. * IPG_PI);
    float sh = sinf(0.5f * ph);
    sincosf(ph, &fs, &fc);
    fg = 2.f * sh * sh;
    nQ = (float)(cb.rQ / rho);
    nV = (float)(cb.rV / rho);
  } else {
    /* the linear form: c = 1, no axial term, sin(rho x) / rho = x */
    fc = 1.f;
    fg = 0.f;
    fs = 1.f;
    nQ = (float)(cb.rQ * dlam * 0.5);
    nV = (float)(cb.rV * dlam * 0.5);
  }
  auto faraday = [&](float &Q, float &U, float &V) {
    const float Q0 = Q, U0 = U, V0 = V;
    const float f = (nQ * Q0 + nV * V0) * fg;
    Q = Q0 * fc + nQ * f - nV * U0 * fs;
    U = U0 * fc + (nV * Q0 - nQ * V0) * fs;
    V = V0 * fc + nV * f + nQ * U0 * fs;
  };
  faraday(SQ, SU, SV);
  /* absorption and emission over dl (aU = jU = 0).  The polarized form
   * divides by tau_P^2; below tau_P^2 = 1e-30 (where its FP32 square would
   * leave the normal range) the polarization coupling is negligible against
   * FP32's precision and the step takes the unpolarized-absorption form, as
   * the FP64 step does below alpha_P^2 = 1e-80 */
  const double tP2d = (cb.aQ * cb.aQ + cb.aV * cb.aV) * dlam * dlam;
  const float tI = (float)(cb.aI * dlam), tQ = (float)(cb.aQ * dlam), tV = (float)(cb.aV * dlam);
  if (tP2d > 1e-30) {
    const float tP2 = tQ * tQ + tV * tV, tP = sqrtf(tP2), itP2 = 1.f / tP2, ih = 0.5f / tP;
    const float ads0 = tQ * SQ + tV * SV, adj = tQ * jQ + tV * jV;
    const float em = expf(-(tI - tP)), ep = expf(-(tI + tP)), e0 = expf(-tI);
    float SI2 = em * (0.5f * SI - ads0 * ih) + ep * (0.5f * SI + ads0 * ih);
    const float cm = (-SI * tP + ads0) * (0.5f * itP2), cp = (SI * tP + ads0) * (0.5f * itP2);
    float SQ2 = em * tQ * cm + ep * tQ * cp + e0 * (SQ - ads0 * tQ * itP2);
    float SU2 = e0 * SU;
    float SV2 = em * tV * cm + ep * tV * cp + e0 * (SV - ads0 * tV * itP2);
    const float q0 = one_minus_exp_over(tI), qm = one_minus_exp_over(tI - tP), qp = one_minus_exp_over(tI + tP);
    const float adjP = adj * itP2;
    SQ2 += q0 * (jQ - tQ * adjP);
    SV2 += q0 * (jV - tV * adjP);
    SI2 += qm * (0.5f * jI - adj * ih) + qp * (0.5f * jI + adj * ih);
    const float m2 = qm * (-tP * jI + adj) * (0.5f * itP2), p2 = qp * (tP * jI + adj) * (0.5f * itP2);
    SQ2 += tQ * (m2 + p2);
    SV2 += tV * (m2 + p2);
    SI = SI2;
    SQ = SQ2;
    SU = SU2;
    SV = SV2;
  } else {
    /* approximate_solve per component with constant j and alpha_I */
    if (tI < 1e-3f) {
      const float w = 1.f - (0.5f * tI) * (1.f - tI * (1.f / 3.f));
      SI += (jI - SI * tI) * w;
      SQ += (jQ - SQ * tI) * w;
      SU += (0.f - SU * tI) * w;
      SV += (jV - SV * tI) * w;
    } else {
      const float e0 = expf(-tI), q0 = one_minus_exp_over(tI);
      SI = SI * e0 + jI * q0;
      SQ = SQ * e0 + jQ * q0;
      SU = SU * e0;
      SV = SV * e0 + jV * q0;
    }
  }
  faraday(SQ, SU, SV);
  *tauF += dlam * fabs(cb.rV);
  const double is = ldexp(1.0, ex);
  double SIo = SI * is, SQo = SQ * is, SUo = SU * is, SVo = SV * is;
  if (stokes_floors) {
    if (SIo < 0) {
      SIo = SQo = SUo = SVo = 0;
    } else {
      double pf = sqrt(SQo * SQo + SUo * SUo + SVo * SVo) / SIo;
      if (pf > 1.) {
        SQo /= pf;
        SUo /= pf;
        SVo /= pf;
      }
    }
  }
  const double *a = cb.a, *b = cb.b;
  double d11 = (SIo + SQo) - T11, d22 = (SIo - SQo) - T22, dr12 = SUo - T12r, di21 = SVo - T21i;
#define DR(i, j) (a[i] * a[j] * d11 + b[i] * b[j] * d22 + (a[i] * b[j] + b[i] * a[j]) * dr12)
#define DS(i, j) ((b[i] * a[j] - a[i] * b[j]) * di21)
  N->r00 += DR(0, 0); N->r01 += DR(0, 1); N->r02 += DR(0, 2); N->r03 += DR(0, 3);
  N->r11 += DR(1, 1); N->r12 += DR(1, 2); N->r13 += DR(1, 3);
  N->r22 += DR(2, 2); N->r23 += DR(2, 3); N->r33 += DR(3, 3);
  N->s01 += DS(0, 1); N->s02 += DS(0, 2); N->s03 += DS(0, 3);
  N->s12 += DS(1, 2); N->s13 += DS(1, 3); N->s23 += DS(2, 3);
#undef DR
#undef DS
  int flag = 0;
  if (*tauF > 1.e100 || *tauF < -1.e100 || isnan(*tauF)) flag |= 2;
  if (isnan(N->r00) || isnan(SIo)) flag |= 4;
  return flag;
}

/* block width of the transfer for the longest length class (its blocks fill
 * an SM's registers); the compiled kernel's thread bound for every class */
#ifndef IPG_XFER_WIDE
#define IPG_XFER_WIDE 256
#endif
/* the FP32-step kernel also pushes N with FP32 increments */
#ifndef IPG_S32_PUSH
#define IPG_S32_PUSH 1
#endif

struct XferLane {
  HermN N;
  const double *rec_i;
  double dl_i, nturns_i; /* dl and nturns of rec_i */
  double I, tau, tauF, js, ks;
  int ray, n, chunk, flag, nrad;
  int cprev; /* chunk_prev[chunk], loaded on entry to the chunk */
};

/* Software prefetch of a step record (four 128-byte lines) so that the walk
 * does not wait on DRAM round trips step after step: a lone ray's step time
 * is otherwise set by two to three dependent loads (transport matrices of
 * one record, then flags and coefficients of the next). */
#ifndef IPG_XFER_PREFETCH
#define IPG_XFER_PREFETCH 1
#endif
template <int RM = -1>
__device__ __forceinline__ void prefetch_rec(const double *p)
{
  /* the compact layout's walk reads only the first three 128-byte lines */
  const int nl = (RM < 0 ? c_cam.mixed : RM) ? 3 : 4;
#if IPG_XFER_PREFETCH == 1
#pragma unroll
  for (int l = 0; l < 4; l++)
    if (l < nl) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + 16 * l));
#elif IPG_XFER_PREFETCH == 2
#pragma unroll
  for (int l = 0; l < 4; l++)
    if (l < nl) asm volatile("prefetch.global.L1 [%0];" ::"l"(p + 16 * l));
#endif
}

/* Take the next ray whose trajectory is complete; rays that hit maxnstep get
 * an all-zero result, deferred rays are left for their next wave. */
template <int RM = -1>
__device__ __forceinline__ bool xfer_fetch(XferLane &L, const int32_t *__restrict__ list, int n_list,
                                           const double *__restrict__ pool, const int *__restrict__ chunk_prev,
                                           const RayRec *__restrict__ rays,
                                           ipg_pixel_out *__restrict__ out, unsigned long long *__restrict__ counters)
{
  while (true) {
    unsigned long long t = atomicAdd(&counters[CNT_NEXT_T], 1ULL);
    if (t >= (unsigned long long)n_list) return false;
    int ray = list ? list[t] : (int)t;
    RayRec rec = rays[ray];
    if (rec.status == IPG_RAY_POOL_FULL) continue;
    if (rec.status == IPG_RAY_MAXNSTEP) {
      ipg_pixel_out o;
      o.I_unpol = o.tau = o.tauF = o.I = o.Q = o.U = o.V = 0.;
      o.nstep = rec.nstep;
      o.flag = 0;
      out[ray] = o;
      continue;
    }
    L.ray = ray;
    L.n = rec.nstep;
    L.chunk = rec.last_chunk;
    L.rec_i = step_ptr(const_cast<double *>(pool), L.chunk, L.n % IPG_CHUNK_STEPS);
    L.cprev = chunk_prev[L.chunk];
    prefetch_rec<RM>(L.rec_i);
    if (L.n % IPG_CHUNK_STEPS) prefetch_rec<RM>(L.rec_i - IPG_STEP_DOUBLES);
    /* get_jkinv at the far end of the ray, src/ipolarray.c:74 */
    if (RM < 0 ? c_cam.mixed : RM) {
      L.js = L.rec_i[RECM_COEF + 1];
      L.ks = L.rec_i[RECM_COEF + 2];
      L.dl_i = L.rec_i[RECM_COEF + 3];
      L.nturns_i = L.rec_i[RECM_COEF + 10];
    } else {
      L.js = L.rec_i[REC_JU];
      L.ks = L.rec_i[REC_KU];
      L.dl_i = L.rec_i[REC_DL];
      L.nturns_i = L.rec_i[REC_NTURNS];
    }
    L.I = L.tau = L.tauF = 0.;
    hn_zero(&L.N);
    L.flag = 0;
    L.nrad = 0;
    return true;
  }
}

/* One step n -> n-1 of integrate_emission's loop (src/ipolarray.c:78-244)
 * for a lane whose record of step n is L.rec_i and whose coefficients of
 * step n-1 are cb: push_polar twice, then the unpolarized and polarized
 * transfer steps at radiating points. */
/* push_polar twice (src/ipolarray.c:85-89) with the transport matrices of
 * record rec and that record's step length dl */
template <bool S32, int RM, class Lane>
__device__ __forceinline__ void xfer_push(Lane &L, const double *rec, double dl)
{
  const DevGrid &G = c_grid;
  double dlfull = dl * G.inv_dlfac;
  double dlhalf = (0.5 * dl) * G.inv_dlfac;
  double A[4][4];
  HermN Nh, Nn;
  load_A_rec<RM>(rec, 0, A);
  if constexpr (S32 && IPG_S32_PUSH) {
    hn_push_f32(L.N, L.N, A, dlhalf, &Nh);
    load_A_rec<RM>(rec, 1, A);
    hn_push_f32(L.N, Nh, A, dlfull, &Nn);
  } else {
    hn_push(L.N, L.N, A, dlhalf, &Nh);
    load_A_rec<RM>(rec, 1, A);
    hn_push(L.N, Nh, A, dlfull, &Nn);
  }
  L.N = Nn;
}

/* the unpolarized and polarized transfer steps at a radiating point, with
 * the coefficient block cb of the step's end and the step length dl of its
 * start (src/ipolarray.c:91-244) */
template <bool S32, class Lane>
__device__ __forceinline__ void xfer_evolve(const DevCam &C, Lane &L, const CoefBlock &cb, double dl, int unpol)
{
  int flags = (int)cb.flags;
  if (flags & 1) {
    L.nrad++;
    int zero_emission = (flags & 2) ? 1 : 0;
    if (C.target_nturns >= 0 && (int)L.nturns_i != C.target_nturns) zero_emission = 1;
    double ji = L.js, ki = L.ks;
    double jf = cb.ju, kf = cb.ku;
    L.js = jf;
    L.ks = kf;
    if (zero_emission) L.I = approximate_solve(L.I, 0, ki, 0, kf, dl, &L.tau);
    else L.I = approximate_solve(L.I, ji, ki, jf, kf, dl, &L.tau);
    if (!unpol) {
      L.flag |= flags >> 2;
      if constexpr (S32) L.flag |= evolve_N_coef_f32(cb, dl, zero_emission, &L.N, &L.tauF, C.stokes_floors);
      else L.flag |= evolve_N_coef(cb, dl, zero_emission, &L.N, &L.tauF, C.stokes_floors);
    }
  }
}

template <bool S32, int RM, class Lane>
__device__ __forceinline__ void xfer_step(const DevCam &C, Lane &L, const CoefBlock &cb, int unpol)
{
  double dl = L.dl_i;
  if (!unpol) xfer_push<S32, RM>(L, L.rec_i, dl);
  xfer_evolve<S32>(C, L, cb, dl, unpol);
}

/* get_pixel's outputs at the end of a lane's walk: project_N
 * (src/ipolarray.c:578-598) in the camera's tetrad */
template <class Lane>
__device__ __forceinline__ void xfer_result(const DevCam &C, const Lane &L, int unpol, int nstep, ipg_pixel_out *o)
{
  o->I_unpol = L.I;
  o->tau = L.tau;
  o->tauF = L.tauF;
  o->I = o->Q = o->U = o->V = 0.;
  if (!unpol) {
    /* project_N, src/ipolarray.c:578-598 */
    double T11, T22, T12r, T21i;
    hn_stokes(L.N, C.Ecov[1], C.Ecov[2], &T11, &T22, &T12r, &T21i);
    double Q = (T11 - T22) / 2, U = T12r;
    o->I = (T11 + T22) / 2;
    /* the rotation by -2 rotcam with its roundings spelled out, so that
     * every kernel that inlines this (the image, the batch, the adjoint's
     * forward pass) gives the same bits whatever it contracts */
    o->Q = fma(Q, C.cproj, -__dmul_rn(U, C.sproj));
    o->U = fma(Q, C.sproj, __dmul_rn(U, C.cproj));
    o->V = T21i;
  }
  o->nstep = nstep;
  o->flag = L.flag;
}

/* RM: the step-record layout, 0 FP64, 1 compact, -1 from the camera (the
 * no-alloc path) */
/* CKK > 0 (the adjoint's forward pass): N of every step n with n % CKK == 0
 * is kept in ckpt, at entry (chunk * 32 + n % 32) / min(CKK, 32), so that
 * the adjoint recomputes N within a segment of CKK steps from its top. */
template <int TPB = IPG_XFER_WIDE, int MINB = IPG_XFER_MINB, bool S32 = false, int RM = -1, int CKK = 0>
__global__ void __launch_bounds__(TPB, MINB)
    k_transfer(const int32_t *__restrict__ list, int n_list, const double *__restrict__ pool,
               const int *__restrict__ chunk_prev, const RayRec *__restrict__ rays, ipg_pixel_out *__restrict__ out,
               unsigned long long *__restrict__ counters, double *__restrict__ ckpt)
{
  const DevGrid &G = c_grid;
  const DevCam &C = c_cam;
  const int unpol = C.unpol;
  XferLane L;
  bool has = xfer_fetch<RM>(L, list, n_list, pool, chunk_prev, rays, out, counters);
  while (__any_sync(0xffffffffu, has)) {
    if (!has) continue;
    if (L.n == 0) {
      ipg_pixel_out o;
      xfer_result(C, L, unpol, rays[L.ray].nstep, &o);
      out[L.ray] = o;
      atomicAdd(&counters[CNT_RAD], (unsigned long long)L.nrad);
      has = xfer_fetch<RM>(L, list, n_list, pool, chunk_prev, rays, out, counters);
      continue;
    }
    if constexpr (CKK > 0) {
      if (L.n % CKK == 0) {
        constexpr int KC = CKK < IPG_CHUNK_STEPS ? CKK : IPG_CHUNK_STEPS;
        double *q = ckpt + (((size_t)L.chunk * IPG_CHUNK_STEPS + L.n % IPG_CHUNK_STEPS) / KC) * 16;
        store4(q, L.N.r00, L.N.r01, L.N.r02, L.N.r03);
        store4(q + 4, L.N.r11, L.N.r12, L.N.r13, L.N.r22);
        store4(q + 8, L.N.r23, L.N.r33, L.N.s01, L.N.s02);
        store4(q + 12, L.N.s03, L.N.s12, L.N.s13, L.N.s23);
      }
    }
    /* step n -> n-1 of integrate_emission's loop, src/ipolarray.c:78-244 */
    int s = L.n - 1;
    if (s % IPG_CHUNK_STEPS == IPG_CHUNK_STEPS - 1) {
      L.chunk = L.cprev;
      L.cprev = chunk_prev[L.chunk];
    }
    const double *rec_f = step_ptr(const_cast<double *>(pool), L.chunk, s % IPG_CHUNK_STEPS);
    /* the record the next iteration reads (step s-1), and the one after */
    if (s >= 1) {
      if ((s - 1) % IPG_CHUNK_STEPS != IPG_CHUNK_STEPS - 1) prefetch_rec<RM>(rec_f - IPG_STEP_DOUBLES);
      else if (L.cprev >= 0) prefetch_rec<RM>(step_ptr(const_cast<double *>(pool), L.cprev, IPG_CHUNK_STEPS - 1));
    }
    CoefBlock cb;
    if (RM < 0 ? C.mixed : RM) load_coef_m(rec_f, cb);
    else load_coef(rec_f, cb);
    xfer_step<S32, RM>(C, L, cb, unpol);
    L.dl_i = cb.dl;
    L.nturns_i = cb.nturns;
    L.rec_i = rec_f;
    L.n--;
  }
}

/* ===================================================================== */
/* k_transfer with its step records staged in shared memory               */
/* ===================================================================== */
/* k_transfer loads a step's record when the step starts, so each step
 * waits for a round trip to L2 or DRAM (long_scoreboard is its largest
 * stall).  Here every lane copies its next record into its own slots of
 * shared memory with cp.async while it computes the current one.
 *
 * One iteration consumes one record k: the transfer step k+1 -> k with k's
 * coefficient block (and record k+1's step length), then the push of N for
 * the step k -> k-1 with k's transport matrices (and k's step length).
 * That is k_transfer's sequence of operations, regrouped by record, so the
 * images are bit-identical.
 *
 * A record is copied in two parts, each issued as soon as the previous
 * record's part has been read from its slot: the coefficient block with the
 * tetrad rows (P1) and the transport matrices (P2).  A part's copy then
 * overlaps the other part's arithmetic.  With NBC = 2 the P1 part has two
 * slots and its copy is issued a whole iteration ahead.  Each lane's slots
 * are NBC P1 + P2 + 16 bytes apart: the 16-byte skew puts the lanes of a
 * quarter-warp in different banks. */
template <int RM, int NBC>
struct XStage {
  static constexpr int P1_OFF = RM ? 128 : 256; /* byte offset of the coefficient block in the record */
  static constexpr int P1 = RM ? 192 : 256;     /* coefficient block + tetrad rows */
  static constexpr int P2 = RM ? 128 : 256;     /* transport matrices A1, A2 (from byte 0) */
  static constexpr int LANE = NBC * P1 + P2 + 16; /* bytes of shared memory per lane */
  static_assert(NBC == 1 || NBC == 2, "one or two coefficient slots");
  static_assert(LANE % 16 == 0 && LANE % 128 == 16, "16-byte copies; quarter-warp lanes in distinct banks");
  static_assert(IPG_XFER_WIDE * LANE <= 227 * 1024, "a wide block's slots fit an SM's shared memory");
};
/* slots per layout: FP64 records take one coefficient slot (528 bytes per
 * lane: three 128-lane blocks per SM, as many as the registers allow), the
 * compact records two (528 bytes as well) */
template <int RM>
struct XStageOf {
  static constexpr int NBC = RM ? 2 : 1;
  using T = XStage<RM, NBC>;
};

/* .ca: through L1, so the second 16 bytes of a 32-byte sector come from L1
 * instead of a second L2 request (with .cg the walk ran 30% slower) */
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int BYTES>
__device__ __forceinline__ void cp_async_bytes(unsigned char *dst, const unsigned char *src)
{
#pragma unroll
  for (int o = 0; o < BYTES; o += 16) cp_async16(dst + o, src + o);
}

template <int TPB = IPG_XFER_WIDE, int MINB = IPG_XFER_MINB, bool S32 = false, int RM = 0>
__global__ void __launch_bounds__(TPB, MINB)
    k_transfer_staged(const int32_t *__restrict__ list, int n_list, const double *__restrict__ pool,
                      const int *__restrict__ chunk_prev, const RayRec *__restrict__ rays,
                      ipg_pixel_out *__restrict__ out, unsigned long long *__restrict__ counters)
{
  static_assert(RM == 0 || RM == 1, "the staged walk is compiled per record layout");
  using X = typename XStageOf<RM>::T;
  constexpr int NBC = XStageOf<RM>::NBC;
  extern __shared__ __align__(16) unsigned char xsm[];
  unsigned char *slot_c = xsm + (size_t)threadIdx.x * X::LANE; /* NBC P1 slots */
  unsigned char *slot_a = slot_c + NBC * X::P1;                /* one P2 slot */
  const double *view_a = reinterpret_cast<const double *>(slot_a);
  const DevCam &C = c_cam;
  const int unpol = C.unpol;
  XferLane L;
  int n0 = 0;
  /* a new ray: its top record's coefficients were read by xfer_fetch, so
   * the first group is empty; the second copies the top record's matrices.
   * In flight at the top of the iteration for record k, oldest first: k's
   * P1 group, k's P2 group (NBC = 1: nothing else). */
  auto start = [&]() {
    n0 = L.n;
    cp_async_commit();
    if (!unpol && L.n > 0) cp_async_bytes<X::P2>(slot_a, reinterpret_cast<const unsigned char *>(L.rec_i));
    cp_async_commit();
  };
  bool has = xfer_fetch<RM>(L, list, n_list, pool, chunk_prev, rays, out, counters);
  if (has) start();
  while (__any_sync(0xffffffffu, has)) {
    if (!has) continue;
    const int k = L.n;
    const double *rec_f = nullptr; /* record k-1 */
    if (k >= 1) {
      const int s = k - 1;
      if (s % IPG_CHUNK_STEPS == IPG_CHUNK_STEPS - 1) {
        L.chunk = L.cprev;
        L.cprev = chunk_prev[L.chunk];
      }
      rec_f = step_ptr(const_cast<double *>(pool), L.chunk, s % IPG_CHUNK_STEPS);
      /* the record after it, into L2 */
      if (s >= 1) {
        if ((s - 1) % IPG_CHUNK_STEPS != IPG_CHUNK_STEPS - 1) prefetch_rec<RM>(rec_f - IPG_STEP_DOUBLES);
        else if (L.cprev >= 0) prefetch_rec<RM>(step_ptr(const_cast<double *>(pool), L.cprev, IPG_CHUNK_STEPS - 1));
      }
    }
    const unsigned char *src_c = reinterpret_cast<const unsigned char *>(rec_f) + X::P1_OFF;
    if constexpr (NBC == 2) {
      if (k >= 1) cp_async_bytes<X::P1>(slot_c + ((k - 1) & 1) * X::P1, src_c);
      cp_async_commit();
    }
    /* the transfer step k+1 -> k (integrate_emission's loop,
     * src/ipolarray.c:91-244) with record k's coefficients */
    if (k < n0) {
      if constexpr (NBC == 2) cp_async_wait<2>();
      else cp_async_wait<1>();
      CoefBlock cb;
      const double *view_c = reinterpret_cast<const double *>(slot_c + (NBC == 2 ? (k & 1) : 0) * X::P1 - X::P1_OFF);
      if constexpr (RM) load_coef_m(view_c, cb);
      else load_coef(view_c, cb);
      xfer_evolve<S32>(C, L, cb, L.dl_i, unpol);
      L.dl_i = cb.dl;
      L.nturns_i = cb.nturns;
    }
    if (k == 0) {
      if constexpr (NBC == 1) cp_async_commit();
      cp_async_commit();
      ipg_pixel_out o;
      xfer_result(C, L, unpol, rays[L.ray].nstep, &o);
      out[L.ray] = o;
      atomicAdd(&counters[CNT_RAD], (unsigned long long)L.nrad);
      has = xfer_fetch<RM>(L, list, n_list, pool, chunk_prev, rays, out, counters);
      if (has) start();
      continue;
    }
    if constexpr (NBC == 1) {
      cp_async_bytes<X::P1>(slot_c, src_c); /* the slot was read by the load above */
      cp_async_commit();
    }
    /* push_polar for the step k -> k-1 with record k's matrices, then the
     * copy of record k-1's matrices into the slot the push has read */
    if (!unpol) {
      cp_async_wait<1>();
      xfer_push<S32, RM>(L, view_a, L.dl_i);
      if (k >= 2) cp_async_bytes<X::P2>(slot_a, reinterpret_cast<const unsigned char *>(rec_f));
    }
    cp_async_commit();
    L.rec_i = rec_f;
    L.n = k - 1;
  }
  cp_async_wait<0>();
}

/* The same walk with each record part fetched by one bulk copy of the
 * tensor-memory-access unit (cp.async.bulk, completion on an mbarrier of the
 * lane's slot) instead of 16-byte copies through the load/store pipe: the
 * staged walk's largest stall is the shared-memory instruction queue (mio
 * throttle), which its 32 copies per step fill.  A slot's barrier flips its
 * phase when its copy has landed; before a slot is refilled, a proxy fence
 * orders the lane's reads of it before the copy's writes.  Every wait is
 * bounded: a copy that has not landed after IPG_XFER_BULK_SPINS polls sets
 * CNT_STALL and ends the lane, and the host reports the call as failed. */
#ifndef IPG_XFER_BULK_SPINS
#define IPG_XFER_BULK_SPINS (1u << 20)
#endif
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bulk_fetch(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

/* waits for the barrier's phase `parity` to complete; false if it did not
 * within the bound */
__device__ __forceinline__ bool bulk_wait(unsigned long long *bar, unsigned parity)
{
  for (unsigned it = 0; it < IPG_XFER_BULK_SPINS; it++) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_slot_refill() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

/* CKK > 0 (the adjoint's forward pass): N at every record k with
 * k % CKK == 0, before the push k -> k-1, is kept in ckpt as by k_transfer */
template <int TPB = IPG_XFER_WIDE, int MINB = IPG_XFER_MINB, bool S32 = false, int RM = 0, int CKK = 0>
__global__ void __launch_bounds__(TPB, MINB)
    k_transfer_bulk(const int32_t *__restrict__ list, int n_list, const double *__restrict__ pool,
                    const int *__restrict__ chunk_prev, const RayRec *__restrict__ rays,
                    ipg_pixel_out *__restrict__ out, unsigned long long *__restrict__ counters,
                    double *__restrict__ ckpt = nullptr)
{
  static_assert(RM == 0 || RM == 1, "the staged walk is compiled per record layout");
  using X = typename XStageOf<RM>::T;
  constexpr int NBC = XStageOf<RM>::NBC;
  extern __shared__ __align__(16) unsigned char xsm[];
  __shared__ __align__(8) unsigned long long xbar[TPB][NBC + 1]; /* per lane: coefficient slot(s), matrices slot */
  unsigned char *slot_c = xsm + (size_t)threadIdx.x * X::LANE;
  unsigned char *slot_a = slot_c + NBC * X::P1;
  const double *view_a = reinterpret_cast<const double *>(slot_a);
  unsigned long long *bar = xbar[threadIdx.x];
#pragma unroll
  for (int j = 0; j <= NBC; j++)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar + j)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  unsigned ph = 0;   /* phase parity of each barrier */
  unsigned pend = 0; /* barriers with a copy issued and not yet waited for */
  const DevCam &C = c_cam;
  const int unpol = C.unpol;
  XferLane L;
  int n0 = 0;
  bool has = xfer_fetch<RM>(L, list, n_list, pool, chunk_prev, rays, out, counters);
  auto fetch = [&](void *dst, const void *src, unsigned bytes, int j) {
    bulk_fetch(dst, src, bytes, bar + j);
    pend |= 1u << j;
  };
  auto wait = [&](int j) {
    bool ok = bulk_wait(bar + j, (ph >> j) & 1);
    ph ^= 1u << j;
    pend &= ~(1u << j);
    return ok;
  };
  auto start = [&]() {
    n0 = L.n;
    if (!unpol && L.n > 0) fetch(slot_a, L.rec_i, X::P2, NBC);
  };
  /* a copy that did not land: flag it, give the lane's other copies in
   * flight their bounded wait, and end the lane */
  auto stall = [&]() {
    atomicAdd(&counters[CNT_STALL], 1ULL);
    for (int j = 0; j <= NBC; j++)
      if (pend & (1u << j)) wait(j);
    has = false;
  };
  if (has) start();
  while (__any_sync(0xffffffffu, has)) {
    if (!has) continue;
    const int k = L.n;
    const int chunk_k = L.chunk; /* record k's chunk */
    const double *rec_f = nullptr; /* record k-1 */
    if (k >= 1) {
      const int s = k - 1;
      if (s % IPG_CHUNK_STEPS == IPG_CHUNK_STEPS - 1) {
        L.chunk = L.cprev;
        L.cprev = chunk_prev[L.chunk];
      }
      rec_f = step_ptr(const_cast<double *>(pool), L.chunk, s % IPG_CHUNK_STEPS);
      if (s >= 1) {
        if ((s - 1) % IPG_CHUNK_STEPS != IPG_CHUNK_STEPS - 1) prefetch_rec<RM>(rec_f - IPG_STEP_DOUBLES);
        else if (L.cprev >= 0) prefetch_rec<RM>(step_ptr(const_cast<double *>(pool), L.cprev, IPG_CHUNK_STEPS - 1));
      }
    }
    const unsigned char *src_c = reinterpret_cast<const unsigned char *>(rec_f) + X::P1_OFF;
    if constexpr (NBC == 2) {
      if (k >= 1) {
        fence_slot_refill();
        fetch(slot_c + ((k - 1) & 1) * X::P1, src_c, X::P1, (k - 1) & 1);
      }
    }
    /* the transfer step k+1 -> k with record k's coefficients */
    if (k < n0) {
      const int j = NBC == 2 ? (k & 1) : 0;
      if (!wait(j)) {
        stall();
        continue;
      }
      CoefBlock cb;
      const double *view_c = reinterpret_cast<const double *>(slot_c + j * X::P1 - X::P1_OFF);
      if constexpr (RM) load_coef_m(view_c, cb);
      else load_coef(view_c, cb);
      xfer_evolve<S32>(C, L, cb, L.dl_i, unpol);
      L.dl_i = cb.dl;
      L.nturns_i = cb.nturns;
    }
    if (k == 0) {
      ipg_pixel_out o;
      xfer_result(C, L, unpol, rays[L.ray].nstep, &o);
      out[L.ray] = o;
      atomicAdd(&counters[CNT_RAD], (unsigned long long)L.nrad);
      has = xfer_fetch<RM>(L, list, n_list, pool, chunk_prev, rays, out, counters);
      if (has) start();
      continue;
    }
    if constexpr (NBC == 1) {
      fence_slot_refill(); /* the slot was read by the load above */
      fetch(slot_c, src_c, X::P1, 0);
    }
    if constexpr (CKK > 0) {
      if (k % CKK == 0) {
        constexpr int KC = CKK < IPG_CHUNK_STEPS ? CKK : IPG_CHUNK_STEPS;
        double *q = ckpt + (((size_t)chunk_k * IPG_CHUNK_STEPS + k % IPG_CHUNK_STEPS) / KC) * 16;
        store4(q, L.N.r00, L.N.r01, L.N.r02, L.N.r03);
        store4(q + 4, L.N.r11, L.N.r12, L.N.r13, L.N.r22);
        store4(q + 8, L.N.r23, L.N.r33, L.N.s01, L.N.s02);
        store4(q + 12, L.N.s03, L.N.s12, L.N.s13, L.N.s23);
      }
    }
    /* push_polar for the step k -> k-1 with record k's matrices, then the
     * fetch of record k-1's matrices into the slot the push has read */
    if (!unpol) {
      if (!wait(NBC)) {
        stall();
        continue;
      }
      xfer_push<S32, RM>(L, view_a, L.dl_i);
      if (k >= 2) {
        fence_slot_refill();
        fetch(slot_a, rec_f, X::P2, NBC);
      }
    }
    L.rec_i = rec_f;
    L.n = k - 1;
  }
}

/* ===================================================================== */
/* longest-first order                                                    */
/* ===================================================================== */
/* The ray queues hand out rays in list order, and a ray costs its step
 * count in the sequential kernels, whose time is set by the longest rays
 * (a lone ray's step takes about as long as one under full load).  Handing
 * out the longest rays first keeps the kernels from ending on a few long
 * rays started last (longest-processing-time-first scheduling).  A counting
 * sort of list positions by a key (predicted step count), descending. */
#define LEN_BUCKETS 4096
#define LEN_SCAN_THREADS 1024

__device__ __forceinline__ int len_bucket(int key, int shift)
{
  int b = key >> shift;
  return b < 0 ? 0 : (b < LEN_BUCKETS - 1 ? b : LEN_BUCKETS - 1);
}

__global__ void k_len_hist(const int32_t *__restrict__ key, int n, int shift, int *hist)
{
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    atomicAdd(&hist[len_bucket(key[t], shift)], 1);
}

/* exclusive scan of the counts in descending bucket order, in place: one
 * block, LEN_SCAN_THREADS threads, LEN_BUCKETS / LEN_SCAN_THREADS buckets each */
__global__ void __launch_bounds__(LEN_SCAN_THREADS) k_len_scan(int *hist)
{
  constexpr int PER = LEN_BUCKETS / LEN_SCAN_THREADS;
  __shared__ int part[LEN_SCAN_THREADS];
  int t = threadIdx.x;
  int c[PER], s = 0;
#pragma unroll
  for (int q = 0; q < PER; q++) {
    c[q] = hist[LEN_BUCKETS - 1 - (PER * t + q)];
    s += c[q];
  }
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < LEN_SCAN_THREADS; off <<= 1) {
    int v = (t >= off) ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int base = part[t] - s;
#pragma unroll
  for (int q = 0; q < PER; q++) {
    hist[LEN_BUCKETS - 1 - (PER * t + q)] = base;
    base += c[q];
  }
}

/* sorted[] = the list's rays in descending key order (ties in any order) */
__global__ void k_len_scatter(const int32_t *__restrict__ list, const int32_t *__restrict__ key, int n, int shift,
                              int *offs, int32_t *__restrict__ sorted)
{
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    int pos = atomicAdd(&offs[len_bucket(key[t], shift)], 1);
    sorted[pos] = list ? list[t] : t;
  }
}

/* ===================================================================== */
/* FP64 / FP32 peak probes                                                */
/* ===================================================================== */
/* 8 independent FMA chains per thread, 16 x 8 FMAs per iteration */
template <class T>
__global__ void k_fma_peak(T *out, int iters, T seed)
{
  T a0 = seed + (T)threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
    a7 = a0 + 7;
  const T m = (T)0.999999, c = (T)1e-7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
      a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
      a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
  }
  T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == (T)12345.678) out[0] = s;
}

/* ===================================================================== */
/* context + C-ABI                                                        */
/* ===================================================================== */
/* reciprocals of grid constants used as divisors in the kernels */
static void devgrid_derived(DevGrid *d)
{
  d->inv_xt = 1. / d->poly_xt;
  d->inv_ap1 = 1. / (d->poly_alpha + 1.);
  d->j22c = (2. * d->poly_alpha * d->poly_norm) / ((1. + d->poly_alpha) * d->poly_xt);
  d->inv_dlfac = 1. / d->dlfac;
  d->inv_lx2 = 1. / (d->cstopx[2] - d->cstartx[2]);
}

/* Length classes of a split wave: rays predicted at least PRED_CLASS_FACS[c]
 * times the mean length go to class c (the first class runs wide), the rest
 * to the last class. */
#ifndef PRED_CLASS_FACS
#define PRED_CLASS_FACS 4., 2.
#endif
static const double k_class_facs[] = {PRED_CLASS_FACS};
#define NB_MAX ((int)(sizeof(k_class_facs) / sizeof(k_class_facs[0])) + 1)
#ifndef IPG_COEF_WAIT_LONGEST
#define IPG_COEF_WAIT_LONGEST 1 /* the shorter classes' coefficient passes wait for the longest class's geodesics */
#endif
#define IPG_STARTED_MAX 1024   /* geodesic blocks of the longest class that can mark their start */
#define IPG_STARTED_WAIT_US 2000 /* the host's wait for them */

struct ipg_ctx {
  int device;
  cudaStream_t stream;
  cudaEvent_t ev[5];
  cudaStream_t bstream[NB_MAX]; /* the length classes of a split wave */
  cudaEvent_t bev[NB_MAX][5];   /* per class: geodesic, coeffs, transfer boundaries (and coeffs start) */
  cudaEvent_t ev_fork, ev_join[NB_MAX], ev_pred[2];
  int *h_started, *d_started; /* mapped host flags: the longest class's geodesic blocks mark their start */
  double *d_fields;
  size_t ncell;
  int have_model;
  int plug;     /* IPG_PLUG_*: the model the kernels are instantiated for */
  DevGrid dg;
  DevPlug dp;   /* constants of a known-answer model */
  double *d_pool;
  int *d_chunk_prev;
  int2 *d_chunk_meta;
  long long n_chunks;
  size_t pool_bytes_req;
  unsigned long long *d_cnt;
  RayRec *d_rays;
  int32_t *d_list[2];
  int32_t *d_sorted; /* the wave's rays, longest predicted first */
  int32_t *d_pred;   /* predicted step counts (list positions), also staging */
  int *d_len_hist;   /* LEN_BUCKETS counters of the sort */
  int split;         /* 1: split waves into long and short batches */
  int xstage;        /* records of the walk: 0 global loads, 1 16-byte copies, 2 bulk copies, -1 per layout */
  int emission_type; /* of the camera being traced */
  int rec_mixed;     /* IPG_RECORDS_MIXED: compact step records */
  int step32;        /* IPG_STEP_FP32: the polarized step in FP32 */
  int fits32;        /* IPG_FITS_FP32: the thermal fits with FP32 shapes */
  int32_t *d_ij;
  ipg_pixel_out *d_out;
  size_t cap;
  int n_sm;
  ipg_stats stats;
  void *refine; /* buffers of the on-device image driver (ipg_refine.cu) */
  double *d_trace_extra; /* rho, u, beta per cell for the trace output (ipg_upload_trace_fields) */
  /* the adjoint's scratch, kept between calls (grow-only): dL/dout per
   * pixel, the cells' gradients, the walk's links */
  double *d_adj_dl, *d_adj_g;
  int *d_adj_next, *d_adj_first;
  size_t adj_dl_cap, adj_g_cap, adj_next_cap, adj_first_cap;
  struct BatchState *batch; /* batch model and work arrays (ipg_batch.cuh) */
  void *batch_arena;        /* buffers of the batch image driver (ipg_refine.cu) */
  char err[512];
};
static void batch_release(ipg_ctx *ctx);

static int cuda_fail(ipg_ctx *ctx, cudaError_t e, const char *where)
{
  if (ctx) snprintf(ctx->err, sizeof(ctx->err), "%s: %s", where, cudaGetErrorString(e));
  return IPG_E_CUDA;
}
#define CK(call)                                             \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

extern "C" const char *ipg_strerror(int code)
{
  switch (code) {
    case IPG_OK: return "ok";
    case IPG_E_ARG: return "invalid argument";
    case IPG_E_CUDA: return "CUDA error";
    case IPG_E_MAXNSTEP: return "MaxNStep exceeded";
    case IPG_E_NAN: return "NaN in image";
    case IPG_E_TIMEOUT: return "device step budget exhausted";
    case IPG_E_NOMEM: return "out of device memory";
    case IPG_E_IO: return "I/O error";
    case IPG_E_STATE: return "invalid call order";
    case IPG_E_FORMAT: return "unsupported dump format";
  }
  return "unknown error";
}

extern "C" const char *ipg_last_error(const ipg_ctx *ctx) { return ctx ? ctx->err : "no context"; }

extern "C" int ipg_create(ipg_ctx **out, int device, size_t pool_bytes)
{
  if (!out) return IPG_E_ARG;
  *out = NULL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return IPG_E_CUDA;
  if (device < 0 || device >= ndev) return IPG_E_ARG;
  ipg_ctx *ctx = (ipg_ctx *)calloc(1, sizeof(ipg_ctx));
  ctx->device = device;
  ctx->pool_bytes_req = pool_bytes;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  for (int i = 0; e == cudaSuccess && i < 5; i++) e = cudaEventCreate(&ctx->ev[i]);
  /* the length classes' streams share the highest priority.  Ranking them
   * (longest class first) measured 199-205 ms per 400x400 image against
   * 190-198 ms for equal ranks: once the shorter classes' coefficient passes
   * wait for the longest class's geodesics, the end of the image is the
   * shortest class's chain, which a lower rank delays. */
  int prio_lo = 0, prio_hi = 0;
  if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  for (int b = 0; e == cudaSuccess && b < NB_MAX; b++) {
    e = cudaStreamCreateWithPriority(&ctx->bstream[b], cudaStreamNonBlocking, prio_hi);
    for (int i = 0; e == cudaSuccess && i < 5; i++) e = cudaEventCreate(&ctx->bev[b][i]);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_join[b]);
  }
  for (int i = 0; e == cudaSuccess && i < 2; i++) e = cudaEventCreate(&ctx->ev_pred[i]);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_fork);
  if (e == cudaSuccess) e = cudaHostAlloc((void **)&ctx->h_started, IPG_STARTED_MAX * sizeof(int), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void **)&ctx->d_started, ctx->h_started, 0);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_cnt, (NB_MAX + 1) * CNT_N * sizeof(unsigned long long));
  ctx->split = 1;
  if (getenv("IPG_NO_SPLIT")) ctx->split = 0;
  /* how the transfer walk reads its step records: by default staged in
   * shared memory; for FP64 records by 16-byte copies in the longest length
   * class (lower latency per step: its walk alone takes 50 ms against 65 ms
   * with bulk copies) and by one bulk copy per record part in the others
   * (higher throughput: the bulk class's walk alone 29 ms against 50 ms),
   * for compact records by 16-byte copies in every class (measured a little
   * faster on the 400x400 image); IPG_XFER_STAGE=0 loads them from global
   * memory, =1 and =2 select the 16-byte and the bulk copies for every
   * class */
  {
    const char *xs = getenv("IPG_XFER_STAGE");
    ctx->xstage = (xs && xs[0] >= '0' && xs[0] <= '2') ? xs[0] - '0' : -1;
  }
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void *)k_transfer_staged<IPG_XFER_WIDE, IPG_XFER_MINB, false, 0>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, IPG_XFER_WIDE * XStageOf<0>::T::LANE);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void *)k_transfer_staged<IPG_XFER_WIDE, IPG_XFER_MINB, true, 0>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, IPG_XFER_WIDE * XStageOf<0>::T::LANE);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void *)k_transfer_staged<IPG_XFER_WIDE, IPG_XFER_MINB, false, 1>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, IPG_XFER_WIDE * XStageOf<1>::T::LANE);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void *)k_transfer_staged<IPG_XFER_WIDE, IPG_XFER_MINB, true, 1>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, IPG_XFER_WIDE * XStageOf<1>::T::LANE);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void *)k_transfer_bulk<IPG_XFER_WIDE, IPG_XFER_MINB, false, 0>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, IPG_XFER_WIDE * XStageOf<0>::T::LANE);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void *)k_transfer_bulk<IPG_XFER_WIDE, IPG_XFER_MINB, true, 0>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, IPG_XFER_WIDE * XStageOf<0>::T::LANE);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void *)k_transfer_bulk<IPG_XFER_WIDE, IPG_XFER_MINB, false, 1>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, IPG_XFER_WIDE * XStageOf<1>::T::LANE);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void *)k_transfer_bulk<IPG_XFER_WIDE, IPG_XFER_MINB, true, 1>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, IPG_XFER_WIDE * XStageOf<1>::T::LANE);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_len_hist, LEN_BUCKETS * sizeof(int));
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->n_sm, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    free(ctx);
    return IPG_E_CUDA;
  }
  *out = ctx;
  return IPG_OK;
}

extern "C" void ipg_destroy(ipg_ctx *ctx)
{
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  ipg__refine_release(ctx->refine);
  ipg__batch_arena_release(ctx->batch_arena);
  batch_release(ctx);
  cudaFree(ctx->d_trace_extra);
  cudaFree(ctx->d_adj_dl);
  cudaFree(ctx->d_adj_g);
  cudaFree(ctx->d_adj_next);
  cudaFree(ctx->d_adj_first);
  cudaFree(ctx->d_fields);
  cudaFree(ctx->d_pool);
  cudaFree(ctx->d_chunk_prev);
  cudaFree(ctx->d_chunk_meta);
  cudaFree(ctx->d_cnt);
  cudaFree(ctx->d_rays);
  cudaFree(ctx->d_list[0]);
  cudaFree(ctx->d_list[1]);
  cudaFree(ctx->d_sorted);
  cudaFree(ctx->d_pred);
  cudaFree(ctx->d_len_hist);
  cudaFree(ctx->d_ij);
  cudaFree(ctx->d_out);
  for (int i = 0; i < 5; i++) cudaEventDestroy(ctx->ev[i]);
  for (int b = 0; b < NB_MAX; b++) {
    for (int i = 0; i < 5; i++) cudaEventDestroy(ctx->bev[b][i]);
    cudaEventDestroy(ctx->ev_join[b]);
    cudaStreamDestroy(ctx->bstream[b]);
  }
  for (int i = 0; i < 2; i++) cudaEventDestroy(ctx->ev_pred[i]);
  cudaEventDestroy(ctx->ev_fork);
  cudaFreeHost(ctx->h_started);
  cudaStreamDestroy(ctx->stream);
  free(ctx);
}

static void devgrid_from(const ipg_grid *g, DevGrid *d);

extern "C" int ipg_upload_iharm(ipg_ctx *ctx, const ipg_grid *g, const double *const fields[IPG_NFIELD])
{
  if (!ctx || !g || !fields || g->n1 <= 0 || g->n2 <= 0 || g->n3 <= 0) return IPG_E_ARG;
  for (int f = 0; f < IPG_NFIELD; f++)
    if (!fields[f]) return IPG_E_ARG;
  if (g->metric != IPG_METRIC_FMKS) {
    snprintf(ctx->err, sizeof(ctx->err), "an iharm dump needs the FMKS metric (%d), grid has %d", IPG_METRIC_FMKS,
             g->metric);
    return IPG_E_ARG;
  }
  CK(cudaSetDevice(ctx->device));
  size_t ncell = (size_t)(g->n1 + 2) * (g->n2 + 2) * (g->n3 + 2);
  /* cell-major (AoS) layout: the 10 fields of a zone are 80 contiguous bytes
   * and the k+1 neighbour follows, so one trilinear gather reads 4 runs of
   * 160 B instead of 80 scattered words. */
  std::vector<double> aos(ncell * IPG_NFIELD);
  for (size_t c = 0; c < ncell; c++)
    for (int f = 0; f < IPG_NFIELD; f++) aos[c * IPG_NFIELD + f] = fields[f][c];
  if (ctx->d_fields && ctx->ncell != ncell) {
    cudaFree(ctx->d_fields);
    ctx->d_fields = NULL;
  }
  cudaFree(ctx->d_trace_extra); /* belongs to the previous dump */
  ctx->d_trace_extra = NULL;
  if (!ctx->d_fields) CK(cudaMalloc(&ctx->d_fields, ncell * IPG_NFIELD * sizeof(double)));
  CK(cudaMemcpy(ctx->d_fields, aos.data(), ncell * IPG_NFIELD * sizeof(double), cudaMemcpyHostToDevice));
  ctx->ncell = ncell;
  devgrid_from(g, &ctx->dg);
  memset(&ctx->dp, 0, sizeof(ctx->dp));
  ctx->plug = IPG_PLUG_IHARM;
  ctx->have_model = 1;
  return IPG_OK;
}

/* The known-answer models (model/analytic, model/sphere): no field arrays,
 * the model's constants go to the kernels' constant bank. */
extern "C" int ipg_upload_plugin(ipg_ctx *ctx, const ipg_grid *g, const ipg_plugin *pl)
{
  if (!ctx || !g || !pl) return IPG_E_ARG;
  int plug, met;
  if (pl->kind == IPG_PLUGIN_ANALYTIC) {
    plug = IPG_PLUG_ANALYTIC;
    met = IPG_METRIC_MKS;
  } else if (pl->kind == IPG_PLUGIN_SPHERE) {
    plug = IPG_PLUG_SPHERE;
    met = IPG_METRIC_EMINKOWSKI;
  } else {
    snprintf(ctx->err, sizeof(ctx->err), "unknown model plugin %d", pl->kind);
    return IPG_E_ARG;
  }
  if (g->metric != met) {
    snprintf(ctx->err, sizeof(ctx->err), "model plugin %d needs metric %d, grid has %d", pl->kind, met, g->metric);
    return IPG_E_ARG;
  }
  CK(cudaSetDevice(ctx->device));
  ipg_grid gg = *g;
  if (met != IPG_METRIC_FMKS) {
    /* the FMKS jet-coordinate constants are unused; keep them finite */
    gg.poly_xt = 1.;
    gg.poly_alpha = 1.;
    gg.poly_norm = 0.;
    gg.mks_smooth = 0.;
  }
  devgrid_from(&gg, &ctx->dg);
  DevPlug &d = ctx->dp;
  memset(&d, 0, sizeof(d));
  d.A = pl->A;
  d.alpha = pl->alpha;
  d.height = pl->height;
  d.l0 = pl->l0;
  d.freqcgs = pl->freqcgs;
  d.rho_unit = pl->rho_unit;
  d.R0 = pl->R0;
  d.Ne0 = pl->Ne0;
  d.Thetae0 = pl->Thetae0;
  d.B0 = pl->B0;
  d.b_unit = pl->B_unit;
  d.sigma0 = pl->sigma0;
  d.beta0 = pl->beta0;
  ctx->plug = plug;
  ctx->have_model = 1;
  return IPG_OK;
}

static void devgrid_from(const ipg_grid *g, DevGrid *dp)
{
  DevGrid &d = *dp;
  memset(&d, 0, sizeof(d));
  d.n1 = g->n1;
  d.n2 = g->n2;
  d.n3 = g->n3;
  for (int i = 0; i < 4; i++) {
    d.startx[i] = g->startx[i];
    d.stopx[i] = g->stopx[i];
    d.dx[i] = g->dx[i];
    d.cstartx[i] = g->cstartx[i];
    d.cstopx[i] = g->cstopx[i];
  }
  d.a = g->a;
  d.hslope = g->hslope;
  d.poly_xt = g->poly_xt;
  d.poly_alpha = g->poly_alpha;
  d.mks_smooth = g->mks_smooth;
  d.poly_norm = g->poly_norm;
  d.Rh = g->Rh;
  d.rmin_geo = g->rmin_geo;
  d.rmax_geo = g->rmax_geo;
  d.th_beg = g->th_beg;
  d.sigma_cut = g->sigma_cut;
  d.sigma_eq_factor = (g->sigma_cut_high > 0 && g->sigma_cut_high > g->sigma_cut) ? 1. : 0.;
  d.L_unit = g->L_unit;
  d.dlfac = g->L_unit * IPG_HPL / (IPG_ME * IPG_CL * IPG_CL);
  d.sj = g->n3 + 2;
  d.si = (long long)(g->n2 + 2) * (g->n3 + 2);
  double am1 = g->poly_alpha - 1.;
  d.alpha_int = (am1 >= 0 && am1 <= 64 && am1 == (double)(int)am1) ? (int)am1 : -1;
  devgrid_derived(&d);
}

/* The trajectory pool: 70% of the free device memory unless the caller asked
 * for a size.  One 400x400 image of a 288x128x128 dump stores ~2.1e8 steps
 * (108 GB at 512 B a step) and so fits in one wave on a 180 GB device. */
static int ensure_pool(ipg_ctx *ctx)
{
  if (ctx->d_pool) return IPG_OK;
  size_t freeb = 0, totalb = 0;
  CK(cudaMemGetInfo(&freeb, &totalb));
  size_t want = ctx->pool_bytes_req ? ctx->pool_bytes_req : (size_t)(0.7 * (double)freeb);
  size_t chunk_bytes = (size_t)IPG_CHUNK_STEPS * IPG_STEP_DOUBLES * sizeof(double) + sizeof(int) + sizeof(int2);
  long long n = (long long)(want / chunk_bytes);
  if (n > 0x7fffffffLL) n = 0x7fffffffLL;
  if (n < 16) return IPG_E_NOMEM;
  CK(cudaMalloc(&ctx->d_pool, (size_t)n * IPG_CHUNK_STEPS * IPG_STEP_DOUBLES * sizeof(double)));
  CK(cudaMalloc(&ctx->d_chunk_prev, (size_t)n * sizeof(int)));
  CK(cudaMalloc(&ctx->d_chunk_meta, (size_t)n * sizeof(int2)));
  ctx->n_chunks = n;
  return IPG_OK;
}

static int ensure_cap(ipg_ctx *ctx, size_t n)
{
  if (n <= ctx->cap) return IPG_OK;
  cudaFree(ctx->d_rays);
  cudaFree(ctx->d_list[0]);
  cudaFree(ctx->d_list[1]);
  cudaFree(ctx->d_sorted);
  cudaFree(ctx->d_pred);
  cudaFree(ctx->d_ij);
  cudaFree(ctx->d_out);
  ctx->cap = 0;
  CK(cudaMalloc(&ctx->d_rays, n * sizeof(RayRec)));
  CK(cudaMalloc(&ctx->d_list[0], n * sizeof(int32_t)));
  CK(cudaMalloc(&ctx->d_list[1], n * sizeof(int32_t)));
  CK(cudaMalloc(&ctx->d_sorted, n * sizeof(int32_t)));
  CK(cudaMalloc(&ctx->d_pred, n * sizeof(int32_t)));
  CK(cudaMalloc(&ctx->d_ij, 2 * n * sizeof(int32_t)));
  CK(cudaMalloc(&ctx->d_out, n * sizeof(ipg_pixel_out)));
  ctx->cap = n;
  return IPG_OK;
}

static void make_devcam(const ipg_camera *c, DevCam *d)
{
  memset(d, 0, sizeof(*d));
  for (int i = 0; i < 4; i++) {
    d->Xcam[i] = c->Xcam[i];
    for (int j = 0; j < 4; j++) {
      d->Econ[i][j] = c->Econ[i][j];
      d->Ecov[i][j] = c->Ecov[i][j];
    }
  }
  d->fovx = c->fovx;
  d->fovy = c->fovy;
  d->crot = cos(c->rotcam);
  d->srot = sin(c->rotcam);
  double rc = c->rotcam * -2.;
  d->cproj = cos(rc);
  d->sproj = sin(rc);
  d->xoff = c->xoff;
  d->yoff = c->yoff;
  d->freq = c->freq;
  d->eps = c->eps;
  d->nx = c->nx;
  d->ny = c->ny;
  d->maxnstep = c->maxnstep;
  d->unpol = c->only_unpolarized;
  d->emission_type = c->emission_type;
  d->stokes_floors = c->stokes_floors;
  d->target_nturns = c->target_nturns;
  d->subring_dtheta = c->subring_dtheta;
  d->counterjet = c->counterjet;
}

/* persistent grid: the resident blocks of the kernel on every SM, no more
 * than the work needs */
static int grid_blocks(ipg_ctx *ctx, const void *kernel, int threads, size_t n, size_t smem = 0)
{
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (per_sm < 1) per_sm = 1;
  size_t full = (size_t)ctx->n_sm * per_sm;
  size_t need = (n + threads - 1) / threads;
  if (need < 1) need = 1;
  return (int)(need < full ? need : full);
}

/* a bulk copy of the transfer walk that did not land within its bounded
 * wait (no such copy has been seen: its source is the pool, in bounds) */
static int stall_fail(ipg_ctx *ctx)
{
  snprintf(ctx->err, sizeof(ctx->err), "a step record's copy into shared memory did not complete");
  return IPG_E_CUDA;
}

/* The host waits (at most IPG_STARTED_WAIT_US) until the first n blocks of
 * a launch have marked their start.  Launched first but placed behind the
 * shorter classes' blocks, the longest class's SM-filling blocks wait for
 * whole SMs to drain, and its geodesics (the image's critical path) then end
 * 30-40 ms later.  No kernel waits here: if the marks do not come in time
 * the launches go on. */
static void wait_started(ipg_ctx *ctx, int n)
{
  const volatile int *f = ctx->h_started;
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    int k = 0;
    while (k < n && f[k]) k++;
    if (k == n) return;
    auto us = std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
    if (us > IPG_STARTED_WAIT_US) {
      ctx->stats.start_waits_timed_out++;
      return;
    }
  }
}

/* One batch of a wave: a slice of a ray list, a slice of the trajectory pool
 * and its own counters, run as geodesic -> coefficients -> transfer on one
 * stream.  wide = 1 launches the two sequential kernels in 256-thread blocks,
 * whose registers fill an SM: no block of another kernel fits beside them.
 * coef_after, when set, holds the batch's coefficient pass until another
 * batch's geodesics are done. */
struct Batch {
  const int32_t *list;
  size_t run;
  double *pool;
  int *chunk_prev;
  int2 *chunk_meta;
  long long n_chunks;
  unsigned long long *cnt;
  int32_t *deferred;
  cudaStream_t stream;
  cudaEvent_t *ev;
  int wide;
  cudaEvent_t coef_after; /* k_coeffs waits for this event (or none) */
  int *started;           /* device view of host flags: the geodesic's blocks mark their start (or none) */
  mutable int geo_blocks; /* the geodesic's grid, as launched */
};

template <int P>
static int launch_batch_t(ipg_ctx *ctx, const Batch &b, const int32_t *d_ij, ipg_pixel_out *d_out)
{
  /* Every class launches the same compiled geodesic and transfer kernels
   * (SM-filling blocks for the longest class, 128-thread blocks, two per SM,
   * for the others): classes that run side by side then share their
   * instructions instead of competing for instruction-cache space. */
  const int threads = 128;
  const int gthreads = b.wide ? 256 : threads, xthreads = b.wide ? IPG_XFER_WIDE : threads;
  CK(cudaEventRecord(b.ev[0], b.stream));
  int gb = grid_blocks(ctx, (const void *)k_geodesic<P, 256, IPG_GEO_MINB>, gthreads, b.run);
  if (b.started && gb > IPG_STARTED_MAX) gb = IPG_STARTED_MAX;
  b.geo_blocks = gb;
  k_geodesic<P, 256, IPG_GEO_MINB><<<gb, gthreads, 0, b.stream>>>(d_ij, b.list, (int)b.run, b.pool, b.chunk_prev,
                                                                  b.chunk_meta, b.n_chunks, b.cnt, ctx->d_rays,
                                                                  b.deferred, nullptr, b.started);
  CK(cudaGetLastError());
  CK(cudaEventRecord(b.ev[1], b.stream));
  if (b.coef_after) CK(cudaStreamWaitEvent(b.stream, b.coef_after, 0));
  CK(cudaEventRecord(b.ev[4], b.stream)); /* coefficients start (after any wait) */
  /* the thermal models get a coefficient kernel compiled for the one fit
   * family the camera selects (Dexter, type 4, or Pandya, type 1): 88.6 KB
   * of code for iharm with Dexter's fits instead of 99.7 KB, and a 400x400
   * image 1% faster, since instruction fetch is this kernel's largest stall */
#define IPG_LAUNCH_COEF(EMT, F)                                                                                 \
  do {                                                                                                         \
    int cb = grid_blocks(ctx, (const void *)k_coeffs<P, EMT, false, F>, threads,                              \
                         (size_t)b.n_chunks * IPG_CHUNK_STEPS);                                                \
    k_coeffs<P, EMT, false, F><<<cb, threads, 0, b.stream>>>(b.pool, b.chunk_meta, b.cnt, b.n_chunks,         \
                                                             ctx->d_rays, ctx->d_fields, nullptr);             \
  } while (0)
  if constexpr (P != IPG_PLUG_ANALYTIC && IPG_COEF_EM_SPECIALIZE) {
    if (ctx->emission_type == 1) {
      if (ctx->fits32)
        IPG_LAUNCH_COEF(1, true);
      else
        IPG_LAUNCH_COEF(1, false);
    } else {
      if (ctx->fits32)
        IPG_LAUNCH_COEF(4, true);
      else
        IPG_LAUNCH_COEF(4, false);
    }
#undef IPG_LAUNCH_COEF
  } else {
    int cb = grid_blocks(ctx, (const void *)k_coeffs<P>, threads, (size_t)b.n_chunks * IPG_CHUNK_STEPS);
    k_coeffs<P><<<cb, threads, 0, b.stream>>>(b.pool, b.chunk_meta, b.cnt, b.n_chunks, ctx->d_rays, ctx->d_fields,
                                              nullptr);
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(b.ev[2], b.stream));
  /* one compiled transfer per step arithmetic and record layout, each
   * holding only its own paths */
#define IPG_LAUNCH_XFER(S32, RM)                                                                              \
  do {                                                                                                       \
    const int xmode = ctx->xstage >= 0 ? ctx->xstage : ((RM || b.wide) ? 1 : 2);                             \
    if (xmode == 2) {                                                                                        \
      size_t sm = (size_t)xthreads * XStageOf<RM>::T::LANE;                                                  \
      int tb = grid_blocks(ctx, (const void *)k_transfer_bulk<IPG_XFER_WIDE, IPG_XFER_MINB, S32, RM>,        \
                           xthreads, b.run, sm);                                                             \
      k_transfer_bulk<IPG_XFER_WIDE, IPG_XFER_MINB, S32, RM><<<tb, xthreads, sm, b.stream>>>(               \
          b.list, (int)b.run, b.pool, b.chunk_prev, ctx->d_rays, d_out, b.cnt);                              \
    } else if (xmode == 1) {                                                                                 \
      size_t sm = (size_t)xthreads * XStageOf<RM>::T::LANE;                                                       \
      int tb = grid_blocks(ctx, (const void *)k_transfer_staged<IPG_XFER_WIDE, IPG_XFER_MINB, S32, RM>,      \
                           xthreads, b.run, sm);                                                             \
      k_transfer_staged<IPG_XFER_WIDE, IPG_XFER_MINB, S32, RM><<<tb, xthreads, sm, b.stream>>>(             \
          b.list, (int)b.run, b.pool, b.chunk_prev, ctx->d_rays, d_out, b.cnt);                              \
    } else {                                                                                                 \
      int tb = grid_blocks(ctx, (const void *)k_transfer<IPG_XFER_WIDE, IPG_XFER_MINB, S32, RM>, xthreads,  \
                           b.run);                                                                           \
      k_transfer<IPG_XFER_WIDE, IPG_XFER_MINB, S32, RM><<<tb, xthreads, 0, b.stream>>>(                     \
          b.list, (int)b.run, b.pool, b.chunk_prev, ctx->d_rays, d_out, b.cnt, nullptr);                     \
    }                                                                                                        \
  } while (0)
  if (ctx->step32) {
    if (ctx->rec_mixed) IPG_LAUNCH_XFER(true, 1);
    else IPG_LAUNCH_XFER(true, 0);
  } else {
    if (ctx->rec_mixed) IPG_LAUNCH_XFER(false, 1);
    else IPG_LAUNCH_XFER(false, 0);
  }
#undef IPG_LAUNCH_XFER
  CK(cudaGetLastError());
  CK(cudaEventRecord(b.ev[3], b.stream));
  return IPG_OK;
}

/* the model is fixed per context (ipg_upload_iharm / ipg_upload_plugin) */
static int launch_batch(ipg_ctx *ctx, const Batch &b, const int32_t *d_ij, ipg_pixel_out *d_out)
{
  switch (ctx->plug) {
    case IPG_PLUG_ANALYTIC: return launch_batch_t<IPG_PLUG_ANALYTIC>(ctx, b, d_ij, d_out);
    case IPG_PLUG_SPHERE: return launch_batch_t<IPG_PLUG_SPHERE>(ctx, b, d_ij, d_out);
    default: return launch_batch_t<IPG_PLUG_IHARM>(ctx, b, d_ij, d_out);
  }
}

static void add_batch_stats(ipg_ctx *ctx, cudaEvent_t *ev, const unsigned long long *cnt)
{
  float a = 0, b = 0, c = 0;
  cudaEventElapsedTime(&a, ev[0], ev[1]);
  cudaEventElapsedTime(&b, ev[4], ev[2]); /* from the coefficients' start */
  cudaEventElapsedTime(&c, ev[2], ev[3]);
  ctx->stats.geodesic_ms += a;
  ctx->stats.coeffs_ms += b;
  ctx->stats.transfer_ms += c;
  ctx->stats.ray_steps += cnt[CNT_STEPS];
  ctx->stats.radiating_steps += cnt[CNT_RAD];
  ctx->stats.launches += 3;
}

/* Length prediction and split of a wave (rays run..: the list, or the
 * identity).  Traces every ray at PRED_EPS_SCALE times the step size without
 * storing anything and sorts the rays by that step count, longest first, into
 * ctx->d_sorted.  The sorted list is cut into up to NB_MAX length classes
 * at the thresholds k_class_facs (times the mean).  Returns the class sizes and
 * predicted step shares; *nb = 0 means: do not split (the wave is small,
 * nothing is long, or the pool looks too small to hold the wave at once). */
#ifndef PRED_EPS_SCALE
#define PRED_EPS_SCALE 12.
#endif

template <int P>
static void launch_count_t(ipg_ctx *ctx, int threads, const int32_t *d_ij, const int32_t *list, size_t run, int cap,
                           unsigned long long *counter)
{
  int gb = grid_blocks(ctx, (const void *)k_geodesic_count<P>, threads, run);
  k_geodesic_count<P><<<gb, threads, 0, ctx->stream>>>(d_ij, list, (int)run, PRED_EPS_SCALE, cap, ctx->d_pred,
                                                       counter, nullptr);
}
#define SPLIT_MIN_RAYS 4096

static int plan_split(ipg_ctx *ctx, const int32_t *d_ij, const int32_t *list, size_t run, const ipg_camera *cam,
                      int *nb, size_t sizes[NB_MAX], double shares[NB_MAX], int wide[NB_MAX])
{
  *nb = 0;
  const int threads = 128;
  unsigned long long *cnt = ctx->d_cnt;
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * CNT_N, ctx->stream));
  int cap = (int)(cam->maxnstep / PRED_EPS_SCALE) + 1;
  if (cap > LEN_BUCKETS - 1) cap = LEN_BUCKETS - 1;
  CK(cudaEventRecord(ctx->ev_pred[0], ctx->stream));
  switch (ctx->plug) {
    case IPG_PLUG_ANALYTIC: launch_count_t<IPG_PLUG_ANALYTIC>(ctx, threads, d_ij, list, run, cap, cnt + CNT_NEXT_G); break;
    case IPG_PLUG_SPHERE: launch_count_t<IPG_PLUG_SPHERE>(ctx, threads, d_ij, list, run, cap, cnt + CNT_NEXT_G); break;
    default: launch_count_t<IPG_PLUG_IHARM>(ctx, threads, d_ij, list, run, cap, cnt + CNT_NEXT_G);
  }
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(ctx->d_len_hist, 0, LEN_BUCKETS * sizeof(int), ctx->stream));
  int sb = (int)((run + 255) / 256);
  if (sb > 4 * ctx->n_sm) sb = 4 * ctx->n_sm;
  k_len_hist<<<sb, 256, 0, ctx->stream>>>(ctx->d_pred, (int)run, 0, ctx->d_len_hist);
  CK(cudaGetLastError());
  std::vector<int> hist(LEN_BUCKETS);
  CK(cudaMemcpyAsync(hist.data(), ctx->d_len_hist, LEN_BUCKETS * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  double total = 0.;
  for (int b = 0; b < LEN_BUCKETS; b++) total += (double)b * hist[b];
  if (total <= 0.) return IPG_OK;
  /* the whole wave should fit: predicted steps scaled back to the real step
   * size (steps scale as 1/eps), against the pool; rays that do not fit
   * after all are deferred to the next wave like any other */
  if (total * PRED_EPS_SCALE > (double)ctx->n_chunks * IPG_CHUNK_STEPS) return IPG_OK;
  double mean = total / (double)run;
  int hi = LEN_BUCKETS; /* classes are bucket ranges [thr, hi) */
  size_t used = 0;
  int n = 0;
  for (int c = 0; c <= NB_MAX - 1; c++) {
    int thr = (c < NB_MAX - 1) ? (int)(k_class_facs[c] * mean) + 1 : 0;
    if (thr > hi) thr = hi;
    size_t cnt_c = 0;
    double st = 0.;
    for (int b = thr; b < hi; b++) {
      cnt_c += (size_t)hist[b];
      st += (double)b * hist[b];
    }
    hi = thr;
    if (!cnt_c) continue;
    sizes[n] = cnt_c;
    shares[n] = st / total;
    wide[n] = (c == 0);
    used += cnt_c;
    n++;
  }
  /* nothing long: no split */
  if (n < 2 || sizes[n - 1] == run) return IPG_OK;
  k_len_scan<<<1, LEN_SCAN_THREADS, 0, ctx->stream>>>(ctx->d_len_hist);
  k_len_scatter<<<sb, 256, 0, ctx->stream>>>(list, ctx->d_pred, (int)run, 0, ctx->d_len_hist, ctx->d_sorted);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev_pred[1], ctx->stream));
  *nb = n;
  return IPG_OK;
}

/* The rays 0..n-1 in ctx->d_sorted, longest predicted first (the length
 * prediction of plan_split without the classes): a lane-persistent kernel
 * that takes them in this order starts its longest rays first, so that their
 * tails overlap the rest of the wave. */
static int sort_by_length(ipg_ctx *ctx, const int32_t *d_ij, size_t n, const ipg_camera *cam)
{
  const int threads = 128;
  unsigned long long *cnt = ctx->d_cnt;
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * CNT_N, ctx->stream));
  int cap = (int)(cam->maxnstep / PRED_EPS_SCALE) + 1;
  if (cap > LEN_BUCKETS - 1) cap = LEN_BUCKETS - 1;
  switch (ctx->plug) {
    case IPG_PLUG_ANALYTIC: launch_count_t<IPG_PLUG_ANALYTIC>(ctx, threads, d_ij, NULL, n, cap, cnt + CNT_NEXT_G); break;
    case IPG_PLUG_SPHERE: launch_count_t<IPG_PLUG_SPHERE>(ctx, threads, d_ij, NULL, n, cap, cnt + CNT_NEXT_G); break;
    default: launch_count_t<IPG_PLUG_IHARM>(ctx, threads, d_ij, NULL, n, cap, cnt + CNT_NEXT_G);
  }
  CK(cudaMemsetAsync(ctx->d_len_hist, 0, LEN_BUCKETS * sizeof(int), ctx->stream));
  int sb = (int)((n + 255) / 256);
  if (sb > 4 * ctx->n_sm) sb = 4 * ctx->n_sm;
  k_len_hist<<<sb, 256, 0, ctx->stream>>>(ctx->d_pred, (int)n, 0, ctx->d_len_hist);
  k_len_scan<<<1, LEN_SCAN_THREADS, 0, ctx->stream>>>(ctx->d_len_hist);
  k_len_scatter<<<sb, 256, 0, ctx->stream>>>(NULL, ctx->d_pred, (int)n, 0, ctx->d_len_hist, ctx->d_sorted);
  CK(cudaGetLastError());
  return IPG_OK;
}

/* The geodesic items of a batch level in *sorted, longest predicted first
 * (k_geodesic_count with the batch's camera table; pred: n scratch ints).
 * Enqueued on the context's stream after ipg__batch_begin. */
extern "C" int ipg__batch_sort_geo(ipg_ctx *ctx, const int32_t *geo_ij, const int32_t *geo_grp, size_t n,
                                   int maxnstep, int32_t *pred, int32_t *sorted, size_t *n_long, double *long_steps,
                                   double *pred_steps)
{
  *n_long = 0;
  *long_steps = 0.;
  *pred_steps = 0.;
  if (!n) return IPG_OK;
  const int threads = 128;
  unsigned long long *cnt = ctx->d_cnt;
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * CNT_N, ctx->stream));
  int cap = (int)(maxnstep / PRED_EPS_SCALE) + 1;
  if (cap > LEN_BUCKETS - 1) cap = LEN_BUCKETS - 1;
  int gb = grid_blocks(ctx, (const void *)k_geodesic_count<IPG_PLUG_IHARM, CamTable>, threads, n);
  k_geodesic_count<IPG_PLUG_IHARM, CamTable><<<gb, threads, 0, ctx->stream>>>(
      geo_ij, NULL, (int)n, PRED_EPS_SCALE, cap, pred, cnt + CNT_NEXT_G, geo_grp);
  CK(cudaMemsetAsync(ctx->d_len_hist, 0, LEN_BUCKETS * sizeof(int), ctx->stream));
  int sb = (int)((n + 255) / 256);
  if (sb > 4 * ctx->n_sm) sb = 4 * ctx->n_sm;
  k_len_hist<<<sb, 256, 0, ctx->stream>>>(pred, (int)n, 0, ctx->d_len_hist);
  CK(cudaGetLastError());
  /* the longest class, as plan_split draws it for a single image */
  std::vector<int> hist(LEN_BUCKETS);
  CK(cudaMemcpyAsync(hist.data(), ctx->d_len_hist, LEN_BUCKETS * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  double total = 0.;
  for (int b = 0; b < LEN_BUCKETS; b++) total += (double)b * hist[b];
  *pred_steps = total * PRED_EPS_SCALE;
  if (total > 0. && n >= SPLIT_MIN_RAYS) {
    const int thr = (int)(k_class_facs[0] * total / (double)n) + 1;
    size_t c = 0;
    double st = 0.;
    for (int b = thr; b < LEN_BUCKETS; b++) {
      c += (size_t)hist[b];
      st += (double)b * hist[b];
    }
    if (c < n) {
      *n_long = c;
      *long_steps = st * PRED_EPS_SCALE;
    }
  }
  k_len_scan<<<1, LEN_SCAN_THREADS, 0, ctx->stream>>>(ctx->d_len_hist);
  k_len_scatter<<<sb, 256, 0, ctx->stream>>>(NULL, pred, (int)n, 0, ctx->d_len_hist, sorted);
  CK(cudaGetLastError());
  return IPG_OK;
}

/* device-resident core: d_ij/d_out on the device, enqueued on ctx->stream */
static int trace_core(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *d_ij, size_t n, ipg_pixel_out *d_out)
{
  if (!ctx->have_model) return IPG_E_STATE;
  if (ctx->plug == IPG_PLUG_ANALYTIC ? cam->emission_type != 10
                                     : (cam->emission_type != 4 && cam->emission_type != 1)) {
    snprintf(ctx->err, sizeof(ctx->err), "emission_type %d not supported by this model (%s)", cam->emission_type,
             ctx->plug == IPG_PLUG_ANALYTIC ? "its own coefficients, type 10, only" : "thermal types 1 and 4 only");
    return IPG_E_ARG;
  }
  if (cam->maxnstep < 2 || cam->nx <= 0 || cam->ny <= 0) return IPG_E_ARG;
  int rc = ensure_pool(ctx);
  if (rc) return rc;
  rc = ensure_cap(ctx, n);
  if (rc) return rc;
  DevCam dc;
  make_devcam(cam, &dc);
  dc.mixed = ctx->rec_mixed;
  ctx->emission_type = cam->emission_type;
  CK(cudaMemcpyToSymbolAsync(c_grid, &ctx->dg, sizeof(DevGrid), 0, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyToSymbolAsync(c_plug, &ctx->dp, sizeof(DevPlug), 0, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyToSymbolAsync(c_cam, &dc, sizeof(DevCam), 0, cudaMemcpyHostToDevice, ctx->stream));
  memset(&ctx->stats, 0, sizeof(ctx->stats));
  /* Waves: every pending ray starts; rays that find the pool full are
   * deferred to the next wave, after the finished ones have been transferred
   * and the pool recycled.  A large wave that fits the pool is split into
   * length classes by predicted step count, run concurrently on their own
   * streams, each longest first: the long rays' walks, whose step latency
   * bounds the sequential kernels, start at once (the longest on SMs of their
   * own), and the short rays' coefficient and transfer work fills the other
   * SMs meanwhile.  A wave that finishes no ray (too many rays sharing a
   * small pool) is retried unsplit with half as many rays; the rest of the
   * pending list is carried over unchanged. */
  const int32_t *list = NULL; /* identity on the first wave */
  size_t pending = n, wave = n;
  int cur = 0, split_ok = ctx->split;
  while (pending > 0) {
    size_t run = pending < wave ? pending : wave;
    size_t carry = pending - run;
    int32_t *next = ctx->d_list[cur ^ 1];
    size_t deferred = 0;
    int nb = 0;
    size_t sizes[NB_MAX];
    double shares[NB_MAX];
    int wide[NB_MAX];
    if (split_ok && carry == 0 && run >= SPLIT_MIN_RAYS) {
      rc = plan_split(ctx, d_ij, list, run, cam, &nb, sizes, shares, wide);
      if (rc) return rc;
      if (!nb) split_ok = 0; /* later waves are this wave's leftovers */
    }
    if (nb) {
      ctx->stats.launches += 4;
      /* pool shares: the predicted share of steps with a margin for the
       * longer classes (their rays are the hardest to predict); the last
       * class gets the rest */
      Batch bt[NB_MAX];
      long long c0 = 0;
      size_t r0 = 0;
      for (int b = 0; b < nb; b++) {
        long long ncb;
        if (b < nb - 1) {
          double f = shares[b] * 1.15 + 0.01;
          ncb = (long long)(f * (double)ctx->n_chunks);
          if (ncb < 16) ncb = 16;
          if (ncb > ctx->n_chunks - c0 - 16 * (nb - 1 - b)) ncb = ctx->n_chunks - c0 - 16 * (nb - 1 - b);
        } else {
          ncb = ctx->n_chunks - c0;
        }
        bt[b].list = ctx->d_sorted + r0;
        bt[b].run = sizes[b];
        bt[b].pool = ctx->d_pool + (size_t)c0 * IPG_CHUNK_STEPS * IPG_STEP_DOUBLES;
        bt[b].chunk_prev = ctx->d_chunk_prev + c0;
        bt[b].chunk_meta = ctx->d_chunk_meta + c0;
        bt[b].n_chunks = ncb;
        bt[b].cnt = ctx->d_cnt + (b + 1) * CNT_N;
        bt[b].deferred = next + r0;
        bt[b].stream = ctx->bstream[b];
        bt[b].ev = ctx->bev[b];
        bt[b].wide = wide[b];
        bt[b].coef_after = nullptr;
        bt[b].started = (b == 0 && wide[0] && nb > 1) ? ctx->d_started : nullptr;
        bt[b].geo_blocks = 0;
        /* the shorter classes' coefficient passes wait for the longest
         * class's geodesics: run beside them, they slow the longest rays'
         * steps four- to eightfold (those rays' SMs hold no other block) */
        if (IPG_COEF_WAIT_LONGEST && b > 0 && wide[0]) bt[b].coef_after = ctx->bev[0][1];
        c0 += ncb;
        r0 += sizes[b];
      }
      /* the classes' counters are cleared before the fork, so that each
       * class stream starts with its geodesic launch and the longest class's
       * SM-filling blocks, launched first, are placed first: placed behind
       * the shorter classes' blocks, they wait for whole SMs to drain */
      CK(cudaMemsetAsync(ctx->d_cnt + CNT_N, 0, sizeof(unsigned long long) * CNT_N * nb, ctx->stream));
      CK(cudaEventRecord(ctx->ev_fork, ctx->stream));
      if (bt[0].started) memset(ctx->h_started, 0, IPG_STARTED_MAX * sizeof(int));
      for (int b = 0; b < nb; b++) {
        CK(cudaStreamWaitEvent(bt[b].stream, ctx->ev_fork, 0));
        rc = launch_batch(ctx, bt[b], d_ij, d_out);
        if (rc) return rc;
        if (bt[b].started) wait_started(ctx, bt[b].geo_blocks);
        CK(cudaEventRecord(ctx->ev_join[b], bt[b].stream));
        CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join[b], 0));
      }
      unsigned long long cnt[NB_MAX * CNT_N];
      CK(cudaMemcpyAsync(cnt, ctx->d_cnt + CNT_N, nb * CNT_N * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                         ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      for (int b = 0; b < nb; b++)
        if (cnt[b * CNT_N + CNT_STALL]) return stall_fail(ctx);
      float pms = 0.f, wms = 0.f;
      cudaEventElapsedTime(&pms, ctx->ev_pred[0], ctx->ev_pred[1]);
      ctx->stats.predict_ms += pms;
      /* each kernel's wall span over the concurrent classes: first start
       * to last end, from the fork */
      float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {0.f, 0.f, 0.f};
      for (int b = 0; b < nb; b++) {
        float w = 0.f;
        cudaEventElapsedTime(&w, ctx->ev_fork, ctx->ev_join[b]);
        if (w > wms) wms = w;
        add_batch_stats(ctx, bt[b].ev, cnt + b * CNT_N);
        const int st[3] = {0, 4, 2}, en[3] = {1, 2, 3};
        for (int k = 0; k < 3; k++) {
          float t0 = 0.f, t1 = 0.f;
          cudaEventElapsedTime(&t0, ctx->ev_fork, bt[b].ev[st[k]]);
          cudaEventElapsedTime(&t1, ctx->ev_fork, bt[b].ev[en[k]]);
          lo[k] = fminf(lo[k], t0);
          hi[k] = fmaxf(hi[k], t1);
        }
      }
      ctx->stats.geodesic_span_ms += hi[0] - lo[0];
      ctx->stats.coeffs_span_ms += hi[1] - lo[1];
      ctx->stats.transfer_span_ms += hi[2] - lo[2];
      ctx->stats.wall_ms += wms + pms;
      ctx->stats.waves += 1;
#ifdef IPG_DEBUG_TIMING
      for (int b = 0; b < nb; b++) {
        float t[4];
        for (int i = 0; i < 4; i++) cudaEventElapsedTime(&t[i], ctx->ev_fork, bt[b].ev[i]);
        fprintf(stderr, "batch %d rays %zu chunks %lld wide %d: geodesic %.1f-%.1f coeffs -%.1f transfer -%.1f ms\n", b,
                bt[b].run, bt[b].n_chunks, bt[b].wide, t[0], t[1], t[2], t[3]);
      }
#endif
      /* gather the classes' deferred rays at the front of the next list */
      size_t r = 0;
      for (int b = 0; b < nb; b++) {
        size_t db = (size_t)cnt[b * CNT_N + CNT_DEFER];
        if (db && r != deferred) {
          CK(cudaMemcpyAsync(ctx->d_pred, next + r, db * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
          CK(cudaMemcpyAsync(next + deferred, ctx->d_pred, db * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                             ctx->stream));
        }
        deferred += db;
        r += sizes[b];
      }
      if (deferred == pending) split_ok = 0;
    } else {
      unsigned long long *cnt_d = ctx->d_cnt;
      CK(cudaMemsetAsync(cnt_d, 0, sizeof(unsigned long long) * CNT_N, ctx->stream));
      if (carry) {
        /* pending rays beyond this wave go first into the next list */
        if (list) {
          CK(cudaMemcpyAsync(next, list + run, carry * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
        } else {
          std::vector<int32_t> ids(carry);
          for (size_t q = 0; q < carry; q++) ids[q] = (int32_t)(run + q);
          CK(cudaMemcpyAsync(next, ids.data(), carry * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
          CK(cudaStreamSynchronize(ctx->stream));
        }
        unsigned long long c0 = carry;
        CK(cudaMemcpyAsync(cnt_d + CNT_DEFER, &c0, sizeof(c0), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
      }
      Batch bt = {list, run, ctx->d_pool, ctx->d_chunk_prev, ctx->d_chunk_meta, ctx->n_chunks, cnt_d, next,
                  ctx->stream, ctx->ev, 0};
      rc = launch_batch(ctx, bt, d_ij, d_out);
      if (rc) return rc;
      unsigned long long cnt[CNT_N];
      CK(cudaMemcpyAsync(cnt, cnt_d, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      if (cnt[CNT_STALL]) return stall_fail(ctx);
      float wms = 0.f;
      cudaEventElapsedTime(&wms, ctx->ev[0], ctx->ev[3]);
      ctx->stats.wall_ms += wms;
      add_batch_stats(ctx, ctx->ev, cnt);
      {
        float a = 0, b2 = 0, c = 0;
        cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&b2, ctx->ev[4], ctx->ev[2]);
        cudaEventElapsedTime(&c, ctx->ev[2], ctx->ev[3]);
        ctx->stats.geodesic_span_ms += a;
        ctx->stats.coeffs_span_ms += b2;
        ctx->stats.transfer_span_ms += c;
      }
      ctx->stats.waves += 1;
      deferred = (size_t)cnt[CNT_DEFER];
      if (deferred == pending) {
        if (run == 1) {
          snprintf(ctx->err, sizeof(ctx->err), "trajectory pool (%lld chunks) too small for a single ray",
                   (long long)ctx->n_chunks);
          return IPG_E_NOMEM;
        }
        wave = run / 2;
      }
    }
    pending = deferred;
    cur ^= 1;
    list = ctx->d_list[cur];
  }
  return IPG_OK;
}

extern "C" int ipg__trace_core(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *d_ij, size_t n,
                               ipg_pixel_out *d_out)
{
  if (!ctx || !cam || n == 0 || n > 0x7fffffff) return IPG_E_ARG;
  return trace_core(ctx, cam, d_ij, n, d_out);
}
extern "C" void *ipg__stream(const ipg_ctx *ctx) { return (void *)ctx->stream; }
extern "C" void ipg__set_error(ipg_ctx *ctx, const char *msg) { snprintf(ctx->err, sizeof(ctx->err), "%s", msg); }
extern "C" void **ipg__refine_slot(ipg_ctx *ctx) { return &ctx->refine; }
extern "C" void **ipg__batch_arena_slot(ipg_ctx *ctx) { return &ctx->batch_arena; }
extern "C" int ipg__step32(const ipg_ctx *ctx) { return ctx->step32; }
extern "C" int ipg__fits32(const ipg_ctx *ctx) { return ctx->fits32; }

extern "C" int ipg_trace_pixels_device(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *d_ij, size_t n,
                                       ipg_pixel_out *d_out, void *stream)
{
  if (!ctx || !cam || (n && (!d_ij || !d_out))) return IPG_E_ARG;
  if (n == 0) return IPG_OK;
  if (n > 0x7fffffff) return IPG_E_ARG;
  CK(cudaSetDevice(ctx->device));
  if (stream) CK(cudaStreamSynchronize((cudaStream_t)stream));
  int rc = trace_core(ctx, cam, d_ij, n, d_out);
  if (rc) return rc;
  /* MAXNSTEP check on the device results */
  std::vector<RayRec> recs(n);
  CK(cudaMemcpy(recs.data(), ctx->d_rays, n * sizeof(RayRec), cudaMemcpyDeviceToHost));
  for (size_t m = 0; m < n; m++)
    if (recs[m].status == IPG_RAY_MAXNSTEP) {
      snprintf(ctx->err, sizeof(ctx->err), "MaxNStep exceeded in ray %zu", m);
      return IPG_E_MAXNSTEP;
    }
  return IPG_OK;
}

extern "C" int ipg_trace_pixels(ipg_ctx *ctx, const ipg_camera *cam, const int32_t *ij, size_t n, ipg_pixel_out *out)
{
  if (!ctx || !cam || (n && (!ij || !out))) return IPG_E_ARG;
  if (n == 0) return IPG_OK;
  if (n > 0x7fffffff) return IPG_E_ARG;
  CK(cudaSetDevice(ctx->device));
  int rc = ensure_cap(ctx, n);
  if (rc) return rc;
  CK(cudaMemcpyAsync(ctx->d_ij, ij, 2 * n * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
  rc = trace_core(ctx, cam, ctx->d_ij, n, ctx->d_out);
  if (rc) return rc;
  CK(cudaMemcpyAsync(out, ctx->d_out, n * sizeof(ipg_pixel_out), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (size_t m = 0; m < n; m++)
    if (out[m].nstep >= cam->maxnstep - 1) {
      snprintf(ctx->err, sizeof(ctx->err), "MaxNStep exceeded in pixel %d %d", ij[2 * m], ij[2 * m + 1]);
      return IPG_E_MAXNSTEP;
    }
  return IPG_OK;
}

extern "C" int ipg_get_stats(const ipg_ctx *ctx, ipg_stats *stats)
{
  if (!ctx || !stats) return IPG_E_ARG;
  *stats = ctx->stats;
  return IPG_OK;
}

extern "C" int ipg_set_record_precision(ipg_ctx *ctx, int precision)
{
  if (!ctx || (precision != IPG_RECORDS_FP64 && precision != IPG_RECORDS_MIXED)) return IPG_E_ARG;
  ctx->rec_mixed = precision == IPG_RECORDS_MIXED;
  return IPG_OK;
}

extern "C" int ipg_set_step_precision(ipg_ctx *ctx, int precision)
{
  if (!ctx || (precision != IPG_STEP_FP64 && precision != IPG_STEP_FP32)) return IPG_E_ARG;
  ctx->step32 = precision == IPG_STEP_FP32;
  return IPG_OK;
}

extern "C" int ipg_set_fit_precision(ipg_ctx *ctx, int precision)
{
  if (!ctx || (precision != IPG_FITS_FP64 && precision != IPG_FITS_FP32)) return IPG_E_ARG;
  ctx->fits32 = precision == IPG_FITS_FP32;
  return IPG_OK;
}

/* The fits at given plasma parameters, one thread per point: the geometry
 * of jar_geo from the angle itself (sin and cos of theta; along the field
 * for theta <= 0 or >= pi, as get_bk_angle's callers test it) */
template <bool F32>
__global__ void k_thermal_coefficients(const double *__restrict__ in, long long n, int emission_type,
                                       double *__restrict__ out)
{
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double *q = in + 5 * i;
    double *o = out + 12 * i;
    double ju = 0., ku = 0.;
    Jar jr = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0.};
    if (q[1] > 0.) {
      JarGeo jg;
      jg.nu = q[0];
      jg.inusq = 1. / (q[0] * q[0]);
      jg.theta = q[4];
      jg.along = (q[4] <= 0. || q[4] >= IPG_PI);
      sincos(q[4], &jg.sth, &jg.cth);
      if constexpr (F32)
        jar_fits_f32(q[1], q[2], q[3], jg, 1, emission_type, &ju, &ku, &jr);
      else
        jar_fits(q[1], q[2], q[3], jg, 1, emission_type, &ju, &ku, &jr);
    }
    const double v[12] = {ju, ku, jr.jI, jr.jQ, jr.jU, jr.jV, jr.aI, jr.aQ, jr.aU, jr.aV, jr.rQ, jr.rV};
#pragma unroll
    for (int k = 0; k < 12; k++) o[k] = v[k];
  }
}

extern "C" int ipg_thermal_coefficients(ipg_ctx *ctx, const double *in, size_t n, int emission_type, int precision,
                                        double *out)
{
  if (!ctx || (n && (!in || !out)) || (emission_type != 1 && emission_type != 4) ||
      (precision != IPG_FITS_FP64 && precision != IPG_FITS_FP32))
    return IPG_E_ARG;
  if (!n) return IPG_OK;
  CK(cudaSetDevice(ctx->device));
  double *d = nullptr;
  CK(cudaMalloc(&d, n * 17 * sizeof(double)));
  int rc = IPG_OK;
  cudaError_t e = cudaMemcpyAsync(d, in, n * 5 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    const int blocks = (int)std::min<size_t>((n + 127) / 128, (size_t)ctx->n_sm * 8);
    if (precision == IPG_FITS_FP32)
      k_thermal_coefficients<true><<<blocks, 128, 0, ctx->stream>>>(d, (long long)n, emission_type, d + n * 5);
    else
      k_thermal_coefficients<false><<<blocks, 128, 0, ctx->stream>>>(d, (long long)n, emission_type, d + n * 5);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, d + n * 5, n * 12 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    snprintf(ctx->err, sizeof(ctx->err), "%s", cudaGetErrorString(e));
    rc = IPG_E_CUDA;
  }
  cudaFree(d);
  return rc;
}

extern "C" int ipg_get_stream(const ipg_ctx *ctx, void **stream)
{
  if (!ctx || !stream) return IPG_E_ARG;
  *stream = (void *)ctx->stream;
  return IPG_OK;
}

template <class T>
static int measure_fma_peak(int device, double ms, double *tflops)
{
  ipg_ctx *ctx = NULL;
  if (!tflops) return IPG_E_ARG;
  CK(cudaSetDevice(device));
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  T *d = NULL;
  CK(cudaMalloc(&d, sizeof(T)));
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  const int threads = 256, blocks = nsm * 8;
  int iters = 256;
  float t = 0;
  for (int rep = 0; rep < 12; rep++) {
    CK(cudaEventRecord(a));
    k_fma_peak<T><<<blocks, threads>>>(d, iters, (T)1);
    CK(cudaEventRecord(b));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(&t, a, b));
    if (t > ms) break;
    if (t < ms / 4) iters *= 2;
  }
  double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
  *tflops = flops / (t * 1e-3) / 1e12;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  return IPG_OK;
}

extern "C" int ipg_measure_fp64_peak(int device, double ms, double *tflops)
{
  return measure_fma_peak<double>(device, ms, tflops);
}

extern "C" int ipg_measure_fp32_peak(int device, double ms, double *tflops)
{
  return measure_fma_peak<float>(device, ms, tflops);
}

/* ===================================================================== */
/* tracing without device allocation                                      */
/* ===================================================================== */
/* ipg_trace_pixels_noalloc serves callers that cannot call cudaMalloc (a host
 * application that owns the device-memory budget through its own allocator,
 * or a pipeline that cannot afford the device-wide synchronisation of
 * cudaMalloc/cudaFree).  It runs the same three kernels as a context, with
 * every scratch buffer carved out of one file-scope device array of fixed
 * size instead of memory allocated at run time. */
#include <mutex>

#define NA_CHUNKS (IPG_NOALLOC_MAX_STEPS / IPG_CHUNK_STEPS)
#define NA_OFF_CNT ((size_t)0)
#define NA_OFF_RAYS ((size_t)256)
#define NA_OFF_LIST0 (NA_OFF_RAYS + (size_t)IPG_NOALLOC_MAX_RAYS * sizeof(RayRec))
#define NA_OFF_LIST1 (NA_OFF_LIST0 + (size_t)IPG_NOALLOC_MAX_RAYS * sizeof(int32_t))
#define NA_OFF_PREV (NA_OFF_LIST1 + (size_t)IPG_NOALLOC_MAX_RAYS * sizeof(int32_t))
#define NA_OFF_META (NA_OFF_PREV + (size_t)NA_CHUNKS * sizeof(int))
#define NA_OFF_POOL (NA_OFF_META + (size_t)NA_CHUNKS * sizeof(int2))
#define NA_BYTES (NA_OFF_POOL + (size_t)NA_CHUNKS * IPG_CHUNK_STEPS * IPG_STEP_DOUBLES * sizeof(double))
#define NA_MAX_DEVICES 64
#define NA_CNT_MAXN CNT_N /* extra counter after the wave counters: rays that hit maxnstep */

static_assert(NA_BYTES == IPG_NOALLOC_SCRATCH_BYTES, "scratch layout and its published size disagree");
static_assert(NA_OFF_LIST0 % 256 == 0 && NA_OFF_LIST1 % 256 == 0 && NA_OFF_PREV % 256 == 0 &&
                  NA_OFF_META % 256 == 0 && NA_OFF_POOL % 256 == 0,
              "scratch sections must stay 256-byte aligned");
static_assert((CNT_N + 1) * sizeof(unsigned long long) <= NA_OFF_RAYS, "counters overflow their section");
static_assert(IPG_NOALLOC_MAX_STEPS % IPG_CHUNK_STEPS == 0, "the step limit must be whole chunks");

/* The scratch array.  In host code this name only stands in for the symbol;
 * its device address comes from cudaGetSymbolAddress, once per device. */
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

static std::mutex g_na_mutex;
static unsigned char *g_na_base[NA_MAX_DEVICES];
static int g_na_nsm[NA_MAX_DEVICES];

/* Set-up, once per device with that device current: the device address of
 * the scratch array and the SM count. */
static int na_setup(int dev, unsigned char **base, int *n_sm)
{
  if (dev < 0 || dev >= NA_MAX_DEVICES) return IPG_E_ARG;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_base[dev]) {
    unsigned char *ptr = NULL;
    if (cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return IPG_E_CUDA;
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1)
      return IPG_E_CUDA;
    g_na_nsm[dev] = nsm;
    g_na_base[dev] = ptr;
  }
  *base = g_na_base[dev];
  *n_sm = g_na_nsm[dev];
  return IPG_OK;
}

__global__ void k_na_iota(int32_t *list, int n, int first)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) list[t] = first + t;
}

__global__ void k_na_count_maxnstep(const RayRec *__restrict__ rays, int n, unsigned long long *count)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n && rays[t].status == IPG_RAY_MAXNSTEP) atomicAdd(count, 1ULL);
}

static int na_blocks(int n_sm, const void *kernel, int threads, size_t n)
{
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  if (per_sm < 1) per_sm = 1;
  size_t full = (size_t)n_sm * per_sm;
  size_t need = (n + threads - 1) / threads;
  if (need < 1) need = 1;
  return (int)(need < full ? need : full);
}

#define NA_CK(call)                                \
  do {                                             \
    if ((call) != cudaSuccess) return IPG_E_CUDA;  \
  } while (0)

extern "C" int ipg_trace_pixels_noalloc(const ipg_grid *g, const double *d_fields, const ipg_camera *cam,
                                        const int32_t *d_ij, size_t n, ipg_pixel_out *d_out, void *stream_)
{
  if (!g || !d_fields || !cam || (n && (!d_ij || !d_out))) return IPG_E_ARG;
  if (n > IPG_NOALLOC_MAX_RAYS || cam->maxnstep > IPG_NOALLOC_MAX_STEPS) return IPG_E_ARG;
  if (g->n1 <= 0 || g->n2 <= 0 || g->n3 <= 0 || g->metric != IPG_METRIC_FMKS) return IPG_E_ARG;
  if (cam->emission_type != 4 && cam->emission_type != 1) return IPG_E_ARG;
  if (cam->maxnstep < 2 || cam->nx <= 0 || cam->ny <= 0) return IPG_E_ARG;
  if (n == 0) return IPG_OK;
  cudaStream_t stream = (cudaStream_t)stream_;
  int dev = 0;
  NA_CK(cudaGetDevice(&dev));
  unsigned char *base = NULL;
  int n_sm = 0;
  int rc = na_setup(dev, &base, &n_sm);
  if (rc) return rc;
  unsigned long long *cnt_d = (unsigned long long *)(base + NA_OFF_CNT);
  RayRec *rays = (RayRec *)(base + NA_OFF_RAYS);
  int32_t *lists[2] = {(int32_t *)(base + NA_OFF_LIST0), (int32_t *)(base + NA_OFF_LIST1)};
  int *chunk_prev = (int *)(base + NA_OFF_PREV);
  int2 *chunk_meta = (int2 *)(base + NA_OFF_META);
  double *pool = (double *)(base + NA_OFF_POOL);
  const long long n_chunks = NA_CHUNKS;

  /* grid constants as ipg_upload_iharm derives them */
  DevGrid d;
  devgrid_from(g, &d);
  DevCam dc;
  make_devcam(cam, &dc);
  NA_CK(cudaMemcpyToSymbolAsync(c_grid, &d, sizeof(DevGrid), 0, cudaMemcpyHostToDevice, stream));
  NA_CK(cudaMemcpyToSymbolAsync(c_cam, &dc, sizeof(DevCam), 0, cudaMemcpyHostToDevice, stream));

  /* the wave loop of a context's trace, on the scratch buffers; the
   * counters are the only scratch that must start at zero, and they are
   * cleared before every wave */
  const int threads = 128;
  const int32_t *list = NULL;
  size_t pending = n, wave = n;
  int cur = 0;
  while (pending > 0) {
    size_t run = pending < wave ? pending : wave;
    size_t carry = pending - run;
    NA_CK(cudaMemsetAsync(cnt_d, 0, sizeof(unsigned long long) * (CNT_N + 1), stream));
    if (carry) {
      if (list) {
        NA_CK(cudaMemcpyAsync(lists[cur ^ 1], list + run, carry * sizeof(int32_t), cudaMemcpyDeviceToDevice, stream));
      } else {
        k_na_iota<<<(int)((carry + 255) / 256), 256, 0, stream>>>(lists[cur ^ 1], (int)carry, (int)run);
        NA_CK(cudaGetLastError());
      }
      unsigned long long c0 = carry;
      NA_CK(cudaMemcpyAsync(cnt_d + CNT_DEFER, &c0, sizeof(c0), cudaMemcpyHostToDevice, stream));
      NA_CK(cudaStreamSynchronize(stream));
    }
    int gb = na_blocks(n_sm, (const void *)k_geodesic<IPG_PLUG_IHARM, 256, IPG_GEO_MINB>, threads, run);
    k_geodesic<IPG_PLUG_IHARM, 256, IPG_GEO_MINB><<<gb, threads, 0, stream>>>(d_ij, list, (int)run, pool, chunk_prev, chunk_meta,
                                                           n_chunks, cnt_d, rays, lists[cur ^ 1], nullptr);
    NA_CK(cudaGetLastError());
    /* the compiled kernels of a context's FP64 path, so that both give the
     * same bits for every ray */
    if (cam->emission_type == 1) {
      int cb = na_blocks(n_sm, (const void *)k_coeffs<IPG_PLUG_IHARM, 1>, threads, (size_t)n_chunks * IPG_CHUNK_STEPS);
      k_coeffs<IPG_PLUG_IHARM, 1><<<cb, threads, 0, stream>>>(pool, chunk_meta, cnt_d, n_chunks, rays, d_fields,
                                                              nullptr);
    } else {
      int cb = na_blocks(n_sm, (const void *)k_coeffs<IPG_PLUG_IHARM, 4>, threads, (size_t)n_chunks * IPG_CHUNK_STEPS);
      k_coeffs<IPG_PLUG_IHARM, 4><<<cb, threads, 0, stream>>>(pool, chunk_meta, cnt_d, n_chunks, rays, d_fields,
                                                              nullptr);
    }
    NA_CK(cudaGetLastError());
    int tb = na_blocks(n_sm, (const void *)k_transfer<IPG_XFER_WIDE, IPG_XFER_MINB, false, 0>, threads, run);
    k_transfer<IPG_XFER_WIDE, IPG_XFER_MINB, false, 0><<<tb, threads, 0, stream>>>(list, (int)run, pool, chunk_prev,
                                                                                   rays, d_out, cnt_d, nullptr);
    NA_CK(cudaGetLastError());
    unsigned long long cnt[CNT_N];
    NA_CK(cudaMemcpyAsync(cnt, cnt_d, sizeof(cnt), cudaMemcpyDeviceToHost, stream));
    NA_CK(cudaStreamSynchronize(stream));
    size_t deferred = (size_t)cnt[CNT_DEFER];
    if (deferred == pending) {
      /* no ray finished: fewer rays share the scratch next time; a single
       * ray always fits because maxnstep <= IPG_NOALLOC_MAX_STEPS */
      if (run == 1) return IPG_E_NOMEM;
      wave = run / 2;
    }
    pending = deferred;
    cur ^= 1;
    list = lists[cur];
  }
  /* every ray's record now holds its final status */
  k_na_count_maxnstep<<<(int)((n + 255) / 256), 256, 0, stream>>>(rays, (int)n, cnt_d + NA_CNT_MAXN);
  NA_CK(cudaGetLastError());
  unsigned long long n_maxn = 0;
  NA_CK(cudaMemcpyAsync(&n_maxn, cnt_d + NA_CNT_MAXN, sizeof(n_maxn), cudaMemcpyDeviceToHost, stream));
  NA_CK(cudaStreamSynchronize(stream));
  return n_maxn ? IPG_E_MAXNSTEP : IPG_OK;
}

/* batches of image instances */
#include "ipg_batch.cuh"

/* the adjoint of the polarized image */
#include "ipg_adjoint.cuh"

/* per-step trace of single rays (dump_var_along) */
#include "ipg_trace.cuh"
