/*
 * Device-side physics of the ray pipeline (sm_100a, FP64).
 *
 * Each function restates the reference routine it cites.  The arithmetic is
 * regrouped for the GPU where the regrouping changes results only at the
 * rounding level (the finite-difference connection amplifies every rounding
 * of the metric by 1/(2 DEL) = 5e6, so the reference's own noise floor in the
 * connection is ~1e-9 relative; the regroupings here stay far below that):
 *
 *   - the metric and its derivatives use the sparsity of the FMKS Jacobian
 *     and of the Kerr-Schild metric (g02 = g23 = 0) instead of 4^4 loops;
 *   - the five metric evaluations of one finite-difference connection share
 *     their transcendentals (exp, sin/cos of 2 pi X2, sin/cos theta) through
 *     exact argument differences and short Taylor polynomials;
 *   - the connection is contracted with the wavevector before it is formed
 *     (Gamma^k_ij K^i K^j and Gamma^i_kl K^l), never stored as 64 numbers;
 *   - g^{mu nu} is the closed-form inverse of the FMKS Kerr-Schild metric,
 *     with one division for its four reciprocals;
 *   - divisions by grid constants are multiplications by reciprocals
 *     computed once on the host, and the offset metrics of the connection take
 *     1/rho^2 from the centre's by a two-term series (a lone ray's step is
 *     latency-bound, and each FP64 division is a long dependent sequence);
 *   - the coherency tensor N is kept Hermitian (16 reals instead of 32), and
 *     evolve_N updates it by the 2x2 tetrad block that the step changes.
 */
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "ipg_constants.h"
#include "ipg_dual.cuh"

#define IPG_DEL 1.e-7            /* finite-difference step, src/geometry.c:91 */
#define IPG_CUT_SMALL_TAU 1e-5   /* src/ipolarray.c:34 */
#define IPG_CUT_PREVENT_NAN 1e-80 /* src/ipolarray.c:37 */
/* Trajectory record of one step, 64 doubles (512 B):
 *   [ 0..15]  A1 = Gamma^i_kl K^l at (X_n, K_n)        written by k_geodesic
 *   [16..31]  A2 = Gamma^i_kl K^l at (Xh_n, Kh_n)      written by k_geodesic
 *   [32..47]  geodesic state (REC_X1 ...)               written by k_geodesic,
 *   [32..63]  replaced in place by the coefficient block of k_coeffs
 *             (REC_FLAGS ...); dl and nturns keep their slots. */
#define IPG_STEP_DOUBLES 64
#define IPG_CHUNK_STEPS 32
#define REC_A1 0
#define REC_A2 16
#define REC_X1 32
#define REC_X2 33
#define REC_X3 34
#define REC_DL 35
#define REC_K 36
#define REC_XH1 40
#define REC_XH2 41
#define REC_NTURNS 42
#define REC_X0 43    /* X^0 (trace output only; k_coeffs overwrites it) */
#define REC_KH 44
#define REC_FLAGS 32 /* bit 0 radiating, bit 1 counterjet cut, bits 2.. oddflag of the point */
#define REC_JU 33    /* unpolarized j_I / nu^2 and alpha_I (get_jkinv) */
#define REC_KU 34
#define REC_JI 36    /* jar_calc: jI jQ jV aI aQ aV (U components are zero) */
#define REC_RQ 43    /* rho_Q, rho_V */
#define REC_RV 44
#define REC_E1COV 48 /* plasma tetrad rows 1, 2: covariant, then contravariant */
#define REC_E2COV 52
#define REC_E1CON 56
#define REC_E2CON 60

/* Code-generation knobs (build-time): minimum resident blocks per SM of the
 * kernels (register budget) and whether the large device functions are
 * kept out of line (smaller code, fewer instruction-cache misses).
 * k_coeffs is fully parallel, so it trades a few spilled registers for
 * occupancy: 4 blocks of 128 threads (128 registers) measured 104 ms against
 * 144 ms at 2 blocks (254 registers) on a 400x400 image; the sequential
 * kernels measured best without a cap. */
#ifndef IPG_GEO_MINB
#define IPG_GEO_MINB 1
#endif
#ifndef IPG_XFER_MINB
#define IPG_XFER_MINB 1
#endif
#ifndef IPG_COEF_MINB
#define IPG_COEF_MINB 4
#endif
#ifdef IPG_NOINLINE_HEAVY
#define IPG_HEAVY __device__ __noinline__
#else
#define IPG_HEAVY __device__
#endif

/* ray status */
#define IPG_RAY_OK 0
#define IPG_RAY_MAXNSTEP 1
#define IPG_RAY_POOL_FULL 2

/* Metrics of the native coordinates (src/coordinates.h:8-19): the iharm
 * FMKS, MKS (the analytic models, hslope = 1), flat space in spherical
 * coordinates with r = X1 (Minkowski) or r = exp(X1) (eMinkowski). */
#define IPG_MET_FMKS 0
#define IPG_MET_MKS 1
#define IPG_MET_MINK 2
#define IPG_MET_EMINK 3

struct DevGrid {
  int n1, n2, n3;
  int alpha_int;            /* poly_alpha - 1 as an integer exponent, or -1 */
  double startx[4], stopx[4], dx[4], cstartx[4], cstopx[4];
  double a, hslope, poly_xt, poly_alpha, mks_smooth, poly_norm;
  double Rh, rmin_geo, rmax_geo, th_beg, sigma_cut;
  double sigma_eq_factor;   /* ne factor when sigma == sigma_cut exactly */
  double L_unit;
  double dlfac;             /* L_unit * HPL / (ME CL^2), src/model_geodesics.c:94 */
  /* reciprocals of the grid constants that divide in the hot loops
   * (devgrid_derived): 1/poly_xt, 1/(poly_alpha+1),
   * 2 poly_alpha poly_norm / ((1+poly_alpha) poly_xt), 1/dlfac,
   * 1/(cstopx2 - cstartx2) */
  double inv_xt, inv_ap1, j22c, inv_dlfac, inv_lx2;
  long long sj, si;         /* cell strides (k fastest) */
};

struct DevCam {
  double Xcam[4];
  double Econ[4][4], Ecov[4][4];
  double fovx, fovy;
  double crot, srot;        /* cos, sin of rotcam */
  double cproj, sproj;      /* cos, sin of -2 rotcam (project_N) */
  double xoff, yoff;
  double freq;
  double eps;
  int nx, ny, maxnstep;
  int unpol, emission_type, stokes_floors, target_nturns, subring_dtheta, counterjet;
  int mixed; /* IPG_RECORDS_MIXED: compact step records (ipg_set_record_precision) */
};

/* Defined here: the header is included by exactly one translation unit. */
__constant__ DevGrid c_grid;
__constant__ DevCam c_cam;
/* Cameras of a batch of image instances, one per camera group (instances
 * whose geodesics coincide share one entry). */
#define IPG_BATCH_MAX_GROUPS 64
__constant__ DevCam c_cams[IPG_BATCH_MAX_GROUPS];

/* --------------------------------------------------------------------- */
/* small helpers                                                           */
/* --------------------------------------------------------------------- */
/* q^n for 0 <= n < 128 by binary powering, without branches */
__device__ __forceinline__ double ipow_int(double q, int n)
{
  double r = 1.0, b = q;
#pragma unroll
  for (int k = 0; k < 7; k++) {
    r *= (n & 1) ? b : 1.0;
    b *= b;
    n >>= 1;
  }
  return r;
}

/* q^(alpha-1) of the FMKS polar map */
__device__ __forceinline__ double fmks_pow_am1(double q)
{
  const DevGrid &G = c_grid;
  return (G.alpha_int >= 0) ? ipow_int(q, G.alpha_int) : pow(q, G.poly_alpha - 1.);
}

/* exp(d) and sin/cos(d) for |d| < 1e-5 (Taylor; exact to rounding) */
__device__ __forceinline__ double expm_small(double d) { return d * (1. + d * (0.5 + d * (1. / 6.))); }
__device__ __forceinline__ void sincos_small(double d, double *s, double *c)
{
  double d2 = d * d;
  *s = d * (1. - d2 * (1. / 6.));
  *c = 1. - 0.5 * d2;
}

/* --------------------------------------------------------------------- */
/* FMKS metric (src/coordinates.c:46-97, 175-239, 263-305)                 */
/* --------------------------------------------------------------------- */
struct Met {  /* symmetric; g02 = g23 = 0 in FMKS */
  double g00, g01, g03, g11, g12, g13, g22, g33;
};

/* X2-dependent parts of theta(X1,X2) and its Jacobian */
struct X2P {
  double S2, C2, y, P, P1;  /* sin 2piX2, cos 2piX2, 2X2-1, q^alpha, q^(alpha-1), q = y/xt */
};

__device__ __forceinline__ void x2_parts_from(double X2, double S2, double C2, X2P *o)
{
  const DevGrid &G = c_grid;
  o->S2 = S2;
  o->C2 = C2;
  o->y = 2. * X2 - 1.;
  double q = o->y * G.inv_xt;
  o->P1 = fmks_pow_am1(q);
  o->P = o->P1 * q;
}

/* theta, dtheta/dX1 (J21) and dtheta/dX2 (J22) from the parts;
 * E = exp(mks_smooth (startx1 - X1)) */
__device__ __forceinline__ void theta_jac(double X2, double E, const X2P &p, double *th, double *J21, double *J22)
{
  const DevGrid &G = c_grid;
  const double omh = 1. - G.hslope;
  double poly = 1. + p.P * G.inv_ap1;
  double thG = IPG_PI * X2 + (omh * 0.5) * p.S2;
  double thJ = G.poly_norm * p.y * poly + 0.5 * IPG_PI;
  *th = thG + E * (thJ - thG);
  *J21 = -E * G.mks_smooth * (IPG_PI * 0.5 - IPG_PI * X2 + G.poly_norm * p.y * poly - 0.5 * omh * p.S2);
  *J22 = IPG_PI + omh * IPG_PI * p.C2 +
         E * (-IPG_PI + 2. * G.poly_norm * poly +
              G.j22c * p.y * p.P1 - omh * IPG_PI * p.C2);
}

/* g_{mu nu} of FMKS at (r, theta) with Jacobian J21, J22 (J11 = r) */
__device__ __forceinline__ Met met_from(double r, double sth, double cth, double J21, double J22)
{
  const double a = c_grid.a;
  double s2 = sth * sth;
  double rho2 = r * r + a * a * cth * cth;
  double t = 2. * r / rho2;
  double G00 = -1. + t, G01 = t, G03 = -a * s2 * t, G11 = 1. + t, G13 = -a * s2 * (1. + t);
  double G22 = rho2, G33 = s2 * (rho2 + a * a * s2 * (1. + t));
  Met m;
  m.g00 = G00;
  m.g01 = G01 * r;
  m.g03 = G03;
  m.g11 = G11 * r * r + G22 * J21 * J21;
  m.g12 = G22 * J21 * J22;
  m.g13 = G13 * r;
  m.g22 = G22 * J22 * J22;
  m.g33 = G33;
  return m;
}

/* met_from at a point a finite-difference offset away from a centre where
 * rho^2 = rho2c and 1/rho^2 = irho2c are known: 1/rho^2 from the centre's by
 * 1/(1+e) = 1 - e(1 - e), e ~ 1e-7 (the e^3 term is below rounding), which
 * saves the division of each offset metric. */
__device__ __forceinline__ Met met_from_near(double r, double sth, double cth, double J21, double J22, double rho2c,
                                             double irho2c)
{
  const double a = c_grid.a;
  double s2 = sth * sth;
  double rho2 = r * r + a * a * cth * cth;
  double e = (rho2 - rho2c) * irho2c;
  double t = 2. * r * (irho2c * (1. - e * (1. - e)));
  double G00 = -1. + t, G01 = t, G03 = -a * s2 * t, G11 = 1. + t, G13 = -a * s2 * (1. + t);
  double G22 = rho2, G33 = s2 * (rho2 + a * a * s2 * (1. + t));
  Met m;
  m.g00 = G00;
  m.g01 = G01 * r;
  m.g03 = G03;
  m.g11 = G11 * r * r + G22 * J21 * J21;
  m.g12 = G22 * J21 * J22;
  m.g13 = G13 * r;
  m.g22 = G22 * J22 * J22;
  m.g33 = G33;
  return m;
}

/* Closed-form g^{mu nu} of FMKS Kerr-Schild (the reference inverts gcov by LU,
 * src/geometry.c:54-64, 252-287; both agree to rounding). */
struct Gcon {
  double u00, u01, u02, u11, u12, u13, u22, u23, u33;  /* g^03 = 0 */
};

__device__ __forceinline__ Gcon gcon_from(double r, double sth, double cth, double J21, double J22,
                                          double *rho2_out = nullptr, double *irho2_out = nullptr)
{
  const double a = c_grid.a;
  double s2 = sth * sth;
  double rho2 = r * r + a * a * cth * cth;
  /* one division for the four reciprocals */
  double rJ = r * J22;
  double p2 = rho2 * rJ;
  double inv = 1. / (p2 * s2);
  double irho2 = inv * rJ * s2;
  double ir = inv * rho2 * J22 * s2;
  double iJ22 = inv * rho2 * r * s2;
  double is2 = inv * p2;
  if (rho2_out) {
    *rho2_out = rho2;
    *irho2_out = irho2;
  }
  double Delta = r * r - 2. * r + a * a;
  double Gtt = -(1. + 2. * r * irho2), Gtr = 2. * r * irho2, Grr = Delta * irho2, Grp = a * irho2;
  double Gthth = irho2, Gpp = irho2 * is2;
  double M21 = -J21 * ir * iJ22; /* dX2/dr */
  Gcon u;
  u.u00 = Gtt;
  u.u01 = Gtr * ir;
  u.u02 = M21 * Gtr;
  u.u11 = ir * ir * Grr;
  u.u12 = ir * M21 * Grr;
  u.u13 = ir * Grp;
  u.u22 = M21 * M21 * Grr + iJ22 * iJ22 * Gthth;
  u.u23 = M21 * Grp;
  u.u33 = Gpp;
  return u;
}

__device__ __forceinline__ void lower(const Met &g, const double v[4], double o[4])
{
  o[0] = g.g00 * v[0] + g.g01 * v[1] + g.g03 * v[3];
  o[1] = g.g01 * v[0] + g.g11 * v[1] + g.g12 * v[2] + g.g13 * v[3];
  o[2] = g.g12 * v[1] + g.g22 * v[2];
  o[3] = g.g03 * v[0] + g.g13 * v[1] + g.g33 * v[3];
}

__device__ __forceinline__ void raise(const Gcon &u, const double v[4], double o[4])
{
  o[0] = u.u00 * v[0] + u.u01 * v[1] + u.u02 * v[2];
  o[1] = u.u01 * v[0] + u.u11 * v[1] + u.u12 * v[2] + u.u13 * v[3];
  o[2] = u.u02 * v[0] + u.u12 * v[1] + u.u22 * v[2] + u.u23 * v[3];
  o[3] = u.u13 * v[1] + u.u23 * v[2] + u.u33 * v[3];
}

/* Everything of one point evaluation of the metric */
struct PointGeo {
  double r, th, sth, cth, J21, J22;
  Met g;
};

/* r of bl_coord (src/coordinates.c:46-58) */
template <int MET>
__device__ __forceinline__ double geo_r(double X1)
{
  return (MET == IPG_MET_MINK) ? X1 : exp(X1);
}

/* flat space in spherical coordinates (src/coordinates.c:180-193) */
template <int MET>
__device__ __forceinline__ Met met_flat(double r, double sth)
{
  Met m;
  m.g00 = -1.;
  m.g01 = m.g03 = m.g12 = m.g13 = 0.;
  m.g11 = (MET == IPG_MET_MINK) ? 1. : r * r;
  m.g22 = r * r;
  m.g33 = r * r * sth * sth;
  return m;
}

/* point evaluation for metric MET: FMKS as written above; MKS is FMKS with
 * the jet term switched off (theta = thetaG, src/coordinates.c:68-70,
 * 278-280), which keeps its arithmetic; the flat metrics have theta = X2 */
template <int MET = IPG_MET_FMKS>
__device__ __forceinline__ void point_geo(double X1, double X2, PointGeo *pg)
{
  const DevGrid &G = c_grid;
  if constexpr (MET == IPG_MET_MINK || MET == IPG_MET_EMINK) {
    pg->r = geo_r<MET>(X1);
    pg->th = X2;
    sincos(X2, &pg->sth, &pg->cth);
    pg->J21 = 0.;
    pg->J22 = 1.;
    pg->g = met_flat<MET>(pg->r, pg->sth);
    return;
  }
  double r = exp(X1);
  double E = (MET == IPG_MET_FMKS) ? exp(G.mks_smooth * (G.startx[1] - X1)) : 0.;
  double S2, C2;
  sincospi(2. * X2, &S2, &C2);
  X2P p;
  x2_parts_from(X2, S2, C2, &p);
  theta_jac(X2, E, p, &pg->th, &pg->J21, &pg->J22);
  sincos(pg->th, &pg->sth, &pg->cth);
  pg->r = r;
  pg->g = met_from(r, pg->sth, pg->cth, pg->J21, pg->J22);
}

/* --------------------------------------------------------------------- */
/* Finite-difference connection (src/geometry.c:93-144)                    */
/* --------------------------------------------------------------------- */
/* d_d g_{mu nu} for d = 1, 2 (the metric does not depend on X0, X3, so the
 * reference's differences in those directions are exactly zero). */
struct Conn {
  Met D1, D2;   /* partial_1 g, partial_2 g */
  Gcon gu;      /* g^{mu nu} at X */
  double r;     /* r at X */
};

__device__ __forceinline__ Met met_diff(const Met &h, const Met &l, double inv)
{
  Met d;
  d.g00 = (h.g00 - l.g00) * inv;
  d.g01 = (h.g01 - l.g01) * inv;
  d.g03 = (h.g03 - l.g03) * inv;
  d.g11 = (h.g11 - l.g11) * inv;
  d.g12 = (h.g12 - l.g12) * inv;
  d.g13 = (h.g13 - l.g13) * inv;
  d.g22 = (h.g22 - l.g22) * inv;
  d.g33 = (h.g33 - l.g33) * inv;
  return d;
}

/* g^{mu nu} of the flat metrics (the reference inverts by LU; diagonal) */
template <int MET>
__device__ __forceinline__ Gcon gcon_flat(double r, double sth)
{
  Gcon u;
  u.u00 = -1.;
  u.u01 = u.u02 = u.u12 = u.u13 = u.u23 = 0.;
  u.u11 = (MET == IPG_MET_MINK) ? 1. : 1. / (r * r);
  u.u22 = 1. / (r * r);
  u.u33 = 1. / (r * r * sth * sth);
  return u;
}

template <int MET>
__device__ void fd_connection_flat(double X1, double X2, Conn *cn)
{
  double r = geo_r<MET>(X1), s0, c0;
  sincos(X2, &s0, &c0);
  cn->gu = gcon_flat<MET>(r, s0);
  cn->r = r;
  {
    double Xh = X1 + IPG_DEL, Xl = X1 - IPG_DEL;
    cn->D1 = met_diff(met_flat<MET>(geo_r<MET>(Xh), s0), met_flat<MET>(geo_r<MET>(Xl), s0), 1. / (Xh - Xl));
  }
  {
    double Xh = X2 + IPG_DEL, Xl = X2 - IPG_DEL;
    cn->D2 = met_diff(met_flat<MET>(r, sin(Xh)), met_flat<MET>(r, sin(Xl)), 1. / (Xh - Xl));
  }
}

template <int MET = IPG_MET_FMKS>
IPG_HEAVY void fd_connection(double X1, double X2, Conn *cn)
{
  if constexpr (MET == IPG_MET_MINK || MET == IPG_MET_EMINK) {
    fd_connection_flat<MET>(X1, X2, cn);
    return;
  }
  const DevGrid &G = c_grid;
  const double sm = G.mks_smooth;
  /* center */
  double r = exp(X1);
  double E = (MET == IPG_MET_FMKS) ? exp(sm * (G.startx[1] - X1)) : 0.;
  double S2, C2;
  sincospi(2. * X2, &S2, &C2);
  X2P p0;
  x2_parts_from(X2, S2, C2, &p0);
  double th0, J21, J22;
  theta_jac(X2, E, p0, &th0, &J21, &J22);
  double s0, c0;
  sincos(th0, &s0, &c0);
  double rho2c, irho2c;
  cn->gu = gcon_from(r, s0, c0, J21, J22, &rho2c, &irho2c);
  cn->r = r;

  /* X1 +- DEL: r and E by exact offsets, theta by its exact difference */
  {
    double Xh = X1 + IPG_DEL, Xl = X1 - IPG_DEL;
    double dh = Xh - X1, dl = Xl - X1; /* exact */
    double rh = r + r * expm_small(dh), rl = r + r * expm_small(dl);
    double Eh = E + E * expm_small(-sm * dh), El = E + E * expm_small(-sm * dl);
    double thh, J21h, J22h, thl, J21l, J22l;
    theta_jac(X2, Eh, p0, &thh, &J21h, &J22h);
    theta_jac(X2, El, p0, &thl, &J21l, &J22l);
    double sd, cd, sh, ch, sl, cl;
    sincos_small(thh - th0, &sd, &cd);
    sh = s0 * cd + c0 * sd;
    ch = c0 * cd - s0 * sd;
    sincos_small(thl - th0, &sd, &cd);
    sl = s0 * cd + c0 * sd;
    cl = c0 * cd - s0 * sd;
    Met gh = met_from_near(rh, sh, ch, J21h, J22h, rho2c, irho2c);
    Met gl = met_from_near(rl, sl, cl, J21l, J22l, rho2c, irho2c);
    cn->D1 = met_diff(gh, gl, 1. / (Xh - Xl));
  }
  /* X2 +- DEL */
  {
    double Xh = X2 + IPG_DEL, Xl = X2 - IPG_DEL;
    double dh = Xh - X2, dl = Xl - X2; /* exact */
    double sd, cd;
    sincos_small(2. * IPG_PI * dh, &sd, &cd);
    X2P ph, pl;
    x2_parts_from(Xh, S2 * cd + C2 * sd, C2 * cd - S2 * sd, &ph);
    sincos_small(2. * IPG_PI * dl, &sd, &cd);
    x2_parts_from(Xl, S2 * cd + C2 * sd, C2 * cd - S2 * sd, &pl);
    double thh, J21h, J22h, thl, J21l, J22l;
    theta_jac(Xh, E, ph, &thh, &J21h, &J22h);
    theta_jac(Xl, E, pl, &thl, &J21l, &J22l);
    double sh, ch, sl, cl;
    sincos_small(thh - th0, &sd, &cd);
    sh = s0 * cd + c0 * sd;
    ch = c0 * cd - s0 * sd;
    sincos_small(thl - th0, &sd, &cd);
    sl = s0 * cd + c0 * sd;
    cl = c0 * cd - s0 * sd;
    Met gh = met_from_near(r, sh, ch, J21h, J22h, rho2c, irho2c);
    Met gl = met_from_near(r, sl, cl, J21l, J22l, rho2c, irho2c);
    cn->D2 = met_diff(gh, gl, 1. / (Xh - Xl));
  }
}

/* v = (partial_d g) K */
__device__ __forceinline__ void dg_dot(const Met &D, const double K[4], double v[4])
{
  v[0] = D.g00 * K[0] + D.g01 * K[1] + D.g03 * K[3];
  v[1] = D.g01 * K[0] + D.g11 * K[1] + D.g12 * K[2] + D.g13 * K[3];
  v[2] = D.g12 * K[1] + D.g22 * K[2];
  v[3] = D.g03 * K[0] + D.g13 * K[1] + D.g33 * K[3];
}

/* Gamma^k_ij K^i K^j (the contraction of push_photon, src/geodesics.c:19-49) */
__device__ __forceinline__ void geo_accel(const Conn &cn, const double K[4], double acc[4])
{
  double v1[4], v2[4], T[4];
  dg_dot(cn.D1, K, v1);
  dg_dot(cn.D2, K, v2);
  double kv1 = K[0] * v1[0] + K[1] * v1[1] + K[2] * v1[2] + K[3] * v1[3];
  double kv2 = K[0] * v2[0] + K[1] * v2[1] + K[2] * v2[2] + K[3] * v2[3];
#pragma unroll
  for (int m = 0; m < 4; m++) T[m] = K[1] * v1[m] + K[2] * v2[m];
  T[1] -= 0.5 * kv1;
  T[2] -= 0.5 * kv2;
  raise(cn.gu, T, acc);
}

/* A^i_k = Gamma^i_kl K^l (the contraction of push_polar, src/ipolarray.c:253-289) */
__device__ __forceinline__ void transport_matrix(const Conn &cn, const double K[4], double A[4][4])
{
  double v1[4], v2[4], B[4][4];
  dg_dot(cn.D1, K, v1);
  dg_dot(cn.D2, K, v2);
  const Met &D1 = cn.D1, &D2 = cn.D2;
  /* B[m][k] = 1/2 (K1 d1 g_km + K2 d2 g_km + delta_k1 v1_m + delta_k2 v2_m - delta_m1 v1_k - delta_m2 v2_k) */
  double d[4][4];
  d[0][0] = K[1] * D1.g00 + K[2] * D2.g00;
  d[0][1] = K[1] * D1.g01 + K[2] * D2.g01;
  d[0][2] = 0.;
  d[0][3] = K[1] * D1.g03 + K[2] * D2.g03;
  d[1][1] = K[1] * D1.g11 + K[2] * D2.g11;
  d[1][2] = K[1] * D1.g12 + K[2] * D2.g12;
  d[1][3] = K[1] * D1.g13 + K[2] * D2.g13;
  d[2][2] = K[1] * D1.g22 + K[2] * D2.g22;
  d[2][3] = 0.;
  d[3][3] = K[1] * D1.g33 + K[2] * D2.g33;
  d[1][0] = d[0][1];
  d[2][0] = d[0][2];
  d[3][0] = d[0][3];
  d[2][1] = d[1][2];
  d[3][1] = d[1][3];
  d[3][2] = d[2][3];
#pragma unroll
  for (int m = 0; m < 4; m++)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      double b = d[k][m];
      if (k == 1) b += v1[m];
      if (k == 2) b += v2[m];
      if (m == 1) b -= v1[k];
      if (m == 2) b -= v2[k];
      B[m][k] = 0.5 * b;
    }
  const Gcon &u = cn.gu;
  double gu[4][4] = {{u.u00, u.u01, u.u02, 0.},
                     {u.u01, u.u11, u.u12, u.u13},
                     {u.u02, u.u12, u.u22, u.u23},
                     {0., u.u13, u.u23, u.u33}};
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) A[i][k] = gu[i][0] * B[0][k] + gu[i][1] * B[1][k] + gu[i][2] * B[2][k] + gu[i][3] * B[3][k];
}

/* --------------------------------------------------------------------- */
/* Hermitian coherency tensor N = R + i S (R symmetric, S antisymmetric)   */
/* --------------------------------------------------------------------- */
struct HermN {
  double r00, r01, r02, r03, r11, r12, r13, r22, r23, r33;  /* symmetric real part */
  double s01, s02, s03, s12, s13, s23;                      /* antisymmetric imaginary part, s_ij = Im N^ij (i<j) */
};

__device__ __forceinline__ void hn_zero(HermN *n)
{
  n->r00 = n->r01 = n->r02 = n->r03 = n->r11 = n->r12 = n->r13 = n->r22 = n->r23 = n->r33 = 0.;
  n->s01 = n->s02 = n->s03 = n->s12 = n->s13 = n->s23 = 0.;
}

__device__ __forceinline__ void hn_unpack(const HermN &n, double R[4][4], double S[4][4])
{
  R[0][0] = n.r00; R[0][1] = n.r01; R[0][2] = n.r02; R[0][3] = n.r03;
  R[1][0] = n.r01; R[1][1] = n.r11; R[1][2] = n.r12; R[1][3] = n.r13;
  R[2][0] = n.r02; R[2][1] = n.r12; R[2][2] = n.r22; R[2][3] = n.r23;
  R[3][0] = n.r03; R[3][1] = n.r13; R[3][2] = n.r23; R[3][3] = n.r33;
  S[0][0] = 0.; S[0][1] = n.s01; S[0][2] = n.s02; S[0][3] = n.s03;
  S[1][0] = -n.s01; S[1][1] = 0.; S[1][2] = n.s12; S[1][3] = n.s13;
  S[2][0] = -n.s02; S[2][1] = -n.s12; S[2][2] = 0.; S[2][3] = n.s23;
  S[3][0] = -n.s03; S[3][1] = -n.s13; S[3][2] = -n.s23; S[3][3] = 0.;
}

/* out = base - dl (A M + M A^T), M Hermitian (push_polar, src/ipolarray.c:277-287) */
__device__ __forceinline__ void hn_push(const HermN &base, const HermN &Mh, const double A[4][4], double dl, HermN *out)
{
  double R[4][4], S[4][4], AR[4][4], AS[4][4];
  hn_unpack(Mh, R, S);
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      AR[i][j] = A[i][0] * R[0][j] + A[i][1] * R[1][j] + A[i][2] * R[2][j] + A[i][3] * R[3][j];
      AS[i][j] = A[i][0] * S[0][j] + A[i][1] * S[1][j] + A[i][2] * S[2][j] + A[i][3] * S[3][j];
    }
  out->r00 = base.r00 - dl * (AR[0][0] + AR[0][0]);
  out->r01 = base.r01 - dl * (AR[0][1] + AR[1][0]);
  out->r02 = base.r02 - dl * (AR[0][2] + AR[2][0]);
  out->r03 = base.r03 - dl * (AR[0][3] + AR[3][0]);
  out->r11 = base.r11 - dl * (AR[1][1] + AR[1][1]);
  out->r12 = base.r12 - dl * (AR[1][2] + AR[2][1]);
  out->r13 = base.r13 - dl * (AR[1][3] + AR[3][1]);
  out->r22 = base.r22 - dl * (AR[2][2] + AR[2][2]);
  out->r23 = base.r23 - dl * (AR[2][3] + AR[3][2]);
  out->r33 = base.r33 - dl * (AR[3][3] + AR[3][3]);
  out->s01 = base.s01 - dl * (AS[0][1] - AS[1][0]);
  out->s02 = base.s02 - dl * (AS[0][2] - AS[2][0]);
  out->s03 = base.s03 - dl * (AS[0][3] - AS[3][0]);
  out->s12 = base.s12 - dl * (AS[1][2] - AS[2][1]);
  out->s13 = base.s13 - dl * (AS[1][3] - AS[3][1]);
  out->s23 = base.s23 - dl * (AS[2][3] - AS[3][2]);
}

/* Stokes parameters of N in a tetrad with covariant rows e1 = Ecov[1],
 * e2 = Ecov[2] (complex_coord_to_tetrad_rank2 + tensor_to_stokes,
 * src/ipolarray.c:684-728); also returns the block entries. */
__device__ __forceinline__ void hn_stokes(const HermN &n, const double e1[4], const double e2[4], double *T11,
                                          double *T22, double *T12r, double *T21i)
{
  double R[4][4], S[4][4];
  hn_unpack(n, R, S);
  double Re1[4], Re2[4], Se1[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    Re1[k] = R[k][0] * e1[0] + R[k][1] * e1[1] + R[k][2] * e1[2] + R[k][3] * e1[3];
    Re2[k] = R[k][0] * e2[0] + R[k][1] * e2[1] + R[k][2] * e2[2] + R[k][3] * e2[3];
    Se1[k] = S[k][0] * e1[0] + S[k][1] * e1[1] + S[k][2] * e1[2] + S[k][3] * e1[3];
  }
  *T11 = e1[0] * Re1[0] + e1[1] * Re1[1] + e1[2] * Re1[2] + e1[3] * Re1[3];
  *T22 = e2[0] * Re2[0] + e2[1] * Re2[1] + e2[2] * Re2[2] + e2[3] * Re2[3];
  *T12r = e1[0] * Re2[0] + e1[1] * Re2[1] + e1[2] * Re2[2] + e1[3] * Re2[3];
  /* Im T21 = e2 . S . e1 */
  *T21i = e2[0] * Se1[0] + e2[1] * Se1[1] + e2[2] * Se1[2] + e2[3] * Se1[3];
}

/* --------------------------------------------------------------------- */
/* Modified Bessel functions K0, K1, K2 of the thermal fits (the reference
 * calls GSL's gsl_sf_bessel_Kn, src/symphony/maxwell_juettner_fits.c:
 * 227-228,263-264,376).  x <= 2: ascending series (Abramowitz & Stegun
 * 9.6.10-11) as Horner polynomials in y = x^2/4 with exact coefficients;
 * x > 2: Chebyshev expansions of K_n(x) sqrt(x) e^x (coefficients from
 * gen_bessel_coeffs.py); K2 = K0 + (2/x) K1.  Relative error <= 2e-15 where
 * the result is a normal number; values that underflow are returned as 0. */
/* --------------------------------------------------------------------- */
#include "ipg_bessel_coeffs.h"

/* Rolled loops keep the code of k_coeffs small (its straight-line code
 * otherwise outgrows the instruction cache). */
#ifndef IPG_ROLL_POLY
#define IPG_ROLL_POLY 1
#endif
#if IPG_ROLL_POLY
#define IPG_POLY_LOOP _Pragma("unroll 1")
#else
#define IPG_POLY_LOOP _Pragma("unroll")
#endif

template <int N>
__device__ __forceinline__ double horner(const double (&c)[N], double y)
{
  double r = c[N - 1];
  IPG_POLY_LOOP
  for (int k = N - 2; k >= 0; k--) r = fma(r, y, c[k]);
  return r;
}

template <int N>
__device__ __forceinline__ double clenshaw(const double (&c)[N], double s)
{
  double b1 = 0., b2 = 0., s2 = 2. * s;
  IPG_POLY_LOOP
  for (int k = N - 1; k >= 1; k--) {
    double t = fma(s2, b1, c[k] - b2);
    b2 = b1;
    b1 = t;
  }
  return fma(s, b1, c[0] - b2);
}

IPG_HEAVY void bessel_k012(double x, double *k0, double *k1, double *k2)
{
  if (x <= 2.0) {
    const double EG = 0.57721566490153286061;
    double y = 0.25 * x * x;
    double lg = log(0.5 * x);
    *k0 = -(lg + EG) * horner(kI0, y) + horner(kK0R, y);
    *k1 = 1.0 / x + lg * (0.5 * x * horner(kI1, y)) - 0.25 * x * horner(kK1R, y);
    *k2 = *k0 + 2.0 / x * *k1;
    return;
  }
  double f0, f1;
  if (x <= 8.0) {
    double s = (16. / x - 5.) * (1. / 3.);
    f0 = clenshaw(kK0M, s);
    f1 = clenshaw(kK1M, s);
  } else {
    double s = 16. / x - 1.;
    f0 = clenshaw(kK0F, s);
    f1 = clenshaw(kK1F, s);
  }
  double pre = exp(-x) * rsqrt(x);
  *k0 = f0 * pre;
  *k1 = f1 * pre;
  *k2 = (f0 + 2. / x * f1) * pre;
}

/* --------------------------------------------------------------------- */
/* Model point evaluation: grid gather + four-vectors                     */
/* (src/grid.c:15-44, 216-334; model/iharm/model.c:420-593)               */
/* --------------------------------------------------------------------- */
struct ModelPt {
  PointGeo geo;
  Gcon gu;
  double Ucon[4], Ucov[4], Bcon[4], Bcov[4];
  double ne, thetae, bmag;
  int in_domain;
};

/* Xtoijk_ghost (src/grid.c:216-283) and the trilinear weights of
 * interp_scalar (src/grid.c:15-44): the four (i, j) columns of the k, k+1
 * cell pairs the gather reads, as cell indices, and the eight weights in the
 * order [2 cc + kk] (column cc, cell k + kk). */
struct GridLoc {
  long long cs[4];
  double w[8];
};

__device__ __forceinline__ void grid_locate(double X1, double X2, double X3, GridLoc *gl)
{
  const DevGrid &G = c_grid;
  double phi = fmod(X3, G.cstopx[3]);
  if (phi < 0.0) phi = G.cstopx[3] + phi;
  int i = (int)((X1 - G.startx[1]) / G.dx[1] - 0.5 + 1000) - 1000;
  int j = (int)((X2 - G.startx[2]) / G.dx[2] - 0.5 + 1000) - 1000;
  int k = (int)((phi - G.startx[3]) / G.dx[3] - 0.5 + 1000) - 1000;
  i = max(-1, min(i, G.n1 - 1));
  j = max(-1, min(j, G.n2 - 1));
  k = max(-1, min(k, G.n3 - 1));
  double d1 = (X1 - ((i + 0.5) * G.dx[1] + G.startx[1])) / G.dx[1];
  double d2 = (X2 - ((j + 0.5) * G.dx[2] + G.startx[2])) / G.dx[2];
  double d3 = (phi - ((k + 0.5) * G.dx[3] + G.startx[3])) / G.dx[3];
  d1 = fmin(fmax(d1, 0.), 1.);
  d2 = fmin(fmax(d2, 0.), 1.);
  d3 = fmin(fmax(d3, 0.), 1.);
  i += 1;
  j += 1;
  k += 1;
  double b1 = 1. - d1, b2 = 1. - d2, b3 = 1. - d3;
  gl->w[0] = b1 * b2 * b3;
  gl->w[1] = b1 * b2 * d3;
  gl->w[2] = b1 * d2 * b3;
  gl->w[3] = b1 * d2 * d3;
  gl->w[4] = d1 * b2 * b3;
  gl->w[5] = d1 * b2 * d3;
  gl->w[6] = d1 * d2 * b3;
  gl->w[7] = d1 * d2 * d3;
  long long c0 = ((long long)i * G.si + (long long)j * G.sj + k);
  gl->cs[0] = c0;
  gl->cs[1] = c0 + G.sj;
  gl->cs[2] = c0 + G.si;
  gl->cs[3] = c0 + G.si + G.sj;
}

/* interp_scalar for NF fields at once from a cell-major array (the NF
 * fields of a cell contiguous): each column's k and k+1 cells are 2 NF
 * contiguous doubles.  Every field sums its eight corners in the same order
 * whatever NF is, so the same values give the same bits from any layout. */
template <int NF>
__device__ __forceinline__ void gather_cells(const double *__restrict__ fields, const GridLoc &gl, double acc[NF])
{
  static_assert(NF % 2 == 0, "pairs of fields are loaded together");
#pragma unroll
  for (int f = 0; f < NF; f++) acc[f] = 0.;
#pragma unroll
  for (int cc = 0; cc < 4; cc++) {
    const double2 *p = reinterpret_cast<const double2 *>(fields + gl.cs[cc] * NF);
#pragma unroll
    for (int h = 0; h < NF; h++) {
      double2 v = __ldg(p + h);
      int f0 = (2 * h) % NF, kk = (2 * h) / NF;
      double wt = gl.w[2 * cc + kk];
      acc[f0] += wt * v.x;
      acc[f0 + 1] += wt * v.y;
    }
  }
}

/* get_model_fourv, model/iharm/model.c:455-492, from the interpolated
 * velocity and field primitives (code units) */
__device__ __forceinline__ void fourv_from(double V1, double V2, double V3, double Bp1, double Bp2, double Bp3,
                                           ModelPt *mp)
{
  const Met &g = mp->geo.g;
  double VdotV = g.g11 * V1 * V1 + g.g12 * V1 * V2 + g.g13 * V1 * V3 + g.g12 * V2 * V1 + g.g22 * V2 * V2 +
                 g.g13 * V3 * V1 + g.g33 * V3 * V3;
  double Vfac = sqrt(-1. / mp->gu.u00 * (1. + fabs(VdotV)));
  mp->Ucon[0] = -Vfac * mp->gu.u00;
  mp->Ucon[1] = V1 - Vfac * mp->gu.u01;
  mp->Ucon[2] = V2 - Vfac * mp->gu.u02;
  mp->Ucon[3] = V3; /* g^03 = 0 */
  lower(g, mp->Ucon, mp->Ucov);
  mp->Bcon[0] = Bp1 * mp->Ucov[1] + Bp2 * mp->Ucov[2] + Bp3 * mp->Ucov[3];
  double iu0 = 1. / mp->Ucon[0];
  mp->Bcon[1] = (Bp1 + mp->Ucon[1] * mp->Bcon[0]) * iu0;
  mp->Bcon[2] = (Bp2 + mp->Ucon[2] * mp->Bcon[0]) * iu0;
  mp->Bcon[3] = (Bp3 + mp->Ucon[3] * mp->Bcon[0]) * iu0;
  lower(g, mp->Bcon, mp->Bcov);
}

/* the point outside the grid: normal observer, no field
 * (model/iharm/model.c:427-446) */
__device__ __forceinline__ void outside_point(ModelPt *mp)
{
  double u0 = -1. / sqrt(-mp->gu.u00);
  mp->Ucov[0] = u0;
  mp->Ucov[1] = mp->Ucov[2] = mp->Ucov[3] = 0.;
  mp->Ucon[0] = u0 * mp->gu.u00;
  mp->Ucon[1] = u0 * mp->gu.u01;
  mp->Ucon[2] = u0 * mp->gu.u02;
  mp->Ucon[3] = 0.;
  for (int m = 0; m < 4; m++) mp->Bcon[m] = mp->Bcov[m] = 0.;
  mp->ne = mp->thetae = mp->bmag = 0.;
}

/* get_model_ne's sigma cut, model/iharm/model.c:567-593 */
__device__ __forceinline__ double sigma_cut_ne(double ne, double sig)
{
  const DevGrid &G = c_grid;
  if (sig > G.sigma_cut) return 0.;
  if (!(sig < G.sigma_cut)) return ne * G.sigma_eq_factor;
  return ne;
}

__device__ __forceinline__ bool in_grid(double X1, double X2)
{
  const DevGrid &G = c_grid;
  return !(X1 < G.startx[1] || X1 >= G.stopx[1] || X2 < G.startx[2] || X2 >= G.stopx[2]);
}

__device__ __forceinline__ void model_point(const double *__restrict__ fields, double X1, double X2, double X3,
                                            const PointGeo &pg, ModelPt *mp)
{
  mp->geo = pg;
  mp->gu = gcon_from(mp->geo.r, mp->geo.sth, mp->geo.cth, mp->geo.J21, mp->geo.J22);
  mp->in_domain = in_grid(X1, X2);
  if (!mp->in_domain) {
    outside_point(mp);
    return;
  }
  GridLoc gl;
  grid_locate(X1, X2, X3, &gl);
  double acc[10];
  gather_cells<10>(fields, gl, acc);
  fourv_from(acc[0], acc[1], acc[2], acc[3], acc[4], acc[5], mp);
  mp->ne = sigma_cut_ne(acc[6], acc[9]);
  mp->thetae = acc[7];
  mp->bmag = acc[8];
}

/* --------------------------------------------------------------------- */
/* Radiation coefficients (src/model_radiation.c:145-332, src/radiation.c) */
/* --------------------------------------------------------------------- */
/* The fits below are written once for any number type R: double for the
 * image, and the dual numbers of ipg_dual.cuh for the adjoint, which carry
 * the derivatives with respect to ne, Theta_e and |B| through the same
 * operations.  NumT<R>::c(v) is a constant of type R. */
template <class R>
struct NumT {
  __device__ __forceinline__ static R c(double v) { return v; }
};
template <int D>
struct NumT<Dual<D>> {
  __device__ __forceinline__ static Dual<D> c(double v) { return dconst<D>(v); }
};

/* K0, K1, K2 of a dual argument: the values of bessel_k012 and the
 * derivatives K0' = -K1, K1' = -K0 - K1/x, K2' = -K1 - 2 K2/x */
__device__ __forceinline__ void bessel_k012_t(double x, double *k0, double *k1, double *k2)
{
  bessel_k012(x, k0, k1, k2);
}
template <int D>
__device__ __forceinline__ void bessel_k012_t(const Dual<D> &x, Dual<D> *k0, Dual<D> *k1, Dual<D> *k2)
{
  double a, b, c;
  bessel_k012(x.v, &a, &b, &c);
  *k0 = dchain(x, a, -b);
  *k1 = dchain(x, b, -a - b / x.v);
  *k2 = dchain(x, c, -b - 2. * c / x.v);
}

/* src/radiation.c:14-23 */
template <class R>
__device__ __forceinline__ R Bnu_inv(double nu, R Thetae)
{
  R x = IPG_HPL * nu / (IPG_ME * IPG_CL * IPG_CL * Thetae);
  if (x < 2.e-3)
    return ((2. * IPG_HPL / (IPG_CL * IPG_CL)) / (x / 24. * (24. + x * (12. + x * (4. + x)))));
  return ((2. * IPG_HPL / (IPG_CL * IPG_CL)) / (exp(x) - 1.));
}

template <class R>
struct JarT {
  R jI, jQ, jU, jV, aI, aQ, aU, aV, rQ, rU, rV;
};
typedef JarT<double> Jar;

/* Faraday rotativities rho_Q (Dexter 2016), rho_V (Shcherbakov 2008, or
 * Dexter's g(X) when dexter_v and K2 > 0), both times nu
 * (src/symphony/maxwell_juettner_fits.c:207-284).  sth, cth: sin, cos of the
 * angle between k and B.  Regrouped for the GPU: the three powers of x share
 * one log(x), and divisions by constants are multiplications by their
 * reciprocals (last-bit changes only). */
template <class R>
__device__ __forceinline__ void rho_QV(R Ne, double nu, R Thetae, R B, double sth, double cth, R k0, R k1, R k2,
                                       int want_q, int dexter_v, R *rQ, R *rV)
{
  const double pi = 3.1415926535897932384;
  R omega0 = (IPG_EE / (IPG_ME * IPG_CL)) * B;
  R wp2 = (4. * pi * IPG_EE * IPG_EE / IPG_ME) * Ne;
  double tpn = 2. * pi * nu;
  double itpn = 1. / tpn;
  R x = Thetae * sqrt(1.4142135623730951 * sth * (1.e3 * omega0 * itpn));
  if (want_q) {
    R lx = log(x);
    R l16 = (val(x) + 1.e-16 == val(x)) ? lx : log(x + 1.e-16);
    R e472 = exp(x * (-1. / 47.2));
    R extraterm = (.011 * e472 - 0.011767707320949831 * pi * 1.e4 * exp((-8. / 3.) * l16)) *
                  (0.5 + 0.5 * tanh((lx - 4.78749174278204599425) * 10.));
    R jffunc = 2.011 * exp(exp(1.035 * lx) * (-1. / 4.7)) - cos(0.5 * x) * exp(exp(1.2 * lx) * (-1. / 2.73)) -
               .011 * e472 + extraterm;
    /* K1/K2 by division, as the reference: for Theta_e < 1/708 both are
     * subnormal and a reciprocal of K2 overflows */
    R k_ratio = (k2 > 0.) ? k1 / k2 : NumT<R>::c(1.);
    double itpn2 = itpn * itpn;
    R eps11m22 = jffunc * wp2 * (omega0 * omega0) * (itpn2 * itpn2) * (k_ratio + 6. * Thetae) * (sth * sth);
    *rQ = tpn * (0.5 / IPG_CL) * eps11m22 * nu;
  }
  R fit_factor;
  if (dexter_v && k2 > 0.) {
    R shgmfunc = 0.43793091 * log(1. + 0.00185777 * pow(x, 1.50316886));
    fit_factor = (k0 - shgmfunc) / k2;
  } else {
    R k_ratio = (k2 > 0.) ? k0 / k2 : NumT<R>::c(1.);
    R shgmfunc = 1 - 0.11 * log(1 + 0.035 * x);
    fit_factor = k_ratio * shgmfunc;
  }
  R eps12 = wp2 * omega0 * (itpn * itpn * itpn) * fit_factor * cth;
  *rV = tpn * (1. / IPG_CL) * eps12 * nu;
}

/* The geometry of the coefficients at a point: the fluid-frame frequency
 * (get_fluid_nu, src/radiation.c:26-44) and the k-B angle (get_bk_angle,
 * src/radiation.c:47-72).  sin and cos of the angle come from its cosine
 * directly (sin = sqrt((1-mu)(1+mu)), cos = mu) instead of through acos; the
 * angle itself is formed only where a fit needs it (theta, Pandya's fits). */
struct JarGeo {
  double nu, inusq, sth, cth, theta;
  int along; /* theta = 0 or pi: no emission or absorption, only rho_V */
};

__device__ __forceinline__ void jar_geo(const ModelPt &mp, const double K[4], int emission_type, JarGeo *jg)
{
  const double pi = IPG_PI;
  double kdu = K[0] * mp.Ucov[0] + K[1] * mp.Ucov[1] + K[2] * mp.Ucov[2] + K[3] * mp.Ucov[3];
  jg->nu = -kdu * IPG_ME * IPG_CL * IPG_CL / IPG_HPL;
  jg->inusq = 1. / (jg->nu * jg->nu);
  jg->theta = pi / 2.;
  jg->along = 0;
  double Bm = sqrt(fabs(mp.Bcon[0] * mp.Bcov[0] + mp.Bcon[1] * mp.Bcov[1] + mp.Bcon[2] * mp.Bcov[2] +
                        mp.Bcon[3] * mp.Bcov[3]));
  if (Bm == 0.) {
    jg->sth = 1.;                    /* sin(pi/2) */
    jg->cth = 6.123233995736766e-17; /* cos(pi/2) in double */
  } else {
    double kk = fabs(kdu);
    double mu = (K[0] * mp.Bcov[0] + K[1] * mp.Bcov[1] + K[2] * mp.Bcov[2] + K[3] * mp.Bcov[3]) / (kk * Bm);
    if (fabs(mu) > 1.) mu /= fabs(mu);
    if (mu >= 1. || mu <= -1.) {
      jg->along = 1;
      jg->theta = (mu >= 1.) ? 0. : pi;
      sincos(jg->theta, &jg->sth, &jg->cth);
    } else {
      jg->cth = mu;
      jg->sth = sqrt((1. - mu) * (1. + mu));
      if (emission_type == 1) jg->theta = acos(mu);
    }
  }
}

/* The fits of both calls the reference makes at a point: pol = 0
 * (get_jkinv: Leung j_I / nu^2, Kirchhoff a_I) into (*ju, *ku) and pol = 1
 * (jar_calc) into *jr, src/model_radiation.c:145-332 with emission_type 4
 * (Dexter) or 1 (Pandya); U components are zero.  Ne > 0. */
template <class R>
__device__ __forceinline__ void jar_fits(R Ne, R Thetae, R B, const JarGeo &jg, int want_pol, int emission_type,
                                         R *ju, R *ku, JarT<R> *jr)
{
  const double pi = IPG_PI;
  const double nu = jg.nu, inusq = jg.inusq, sth = jg.sth, cth = jg.cth, theta = jg.theta;
  R k0, k1, k2;
  bessel_k012_t(1. / Thetae, &k0, &k1, &k2);
  if (jg.along) {
    /* only rho_V; the reference still has dexter_fit = 1 set for the Dexter
     * emission type here (src/model_radiation.c:202-207, 212-221) */
    if (want_pol) {
      R rq;
      rho_QV(Ne, nu, Thetae, B, sth, cth, k0, k1, k2, 0, emission_type == 4, &rq, &jr->rV);
    }
    return;
  }
  R Bnuinv = Bnu_inv(nu, Thetae);
  R bnu = (Bnuinv > 0.) ? 1. / Bnuinv : NumT<R>::c(0.); /* Kirchhoff: a = j / B_nu-inverse */
  const R Th2 = Thetae * Thetae;
  /* pol = 0: Leung fit, src/symphony/maxwell_juettner_fits.c:368-395 */
  {
    R K2 = fmax(k2, IPG_SMALL);
    R nus = ((2. / 9.) * IPG_EE / (2. * pi * IPG_ME * IPG_CL)) * B * Th2 * sth;
    R j = NumT<R>::c(0.);
    if (!(nu > val(1.e12 * nus))) {
      R x = nu / nus;
      R cx = cbrt(x);
      R f = sqrt(x) + 1.8877486253633868 * sqrt(cx); /* 2^(11/12) x^(1/6) */
      f = f * f;
      j = ((1.4142135623730951 * pi * IPG_EE * IPG_EE / (3. * IPG_CL)) * Ne * nus / K2) * f * exp(-cx);
    }
    *ju = j * inusq;
    *ku = *ju * bnu;
  }
  if (!want_pol) return;
  /* pol = 1 */
  R jI, jQ, jV;
  if (emission_type == 1) {
    /* Pandya+ 2016, src/symphony/maxwell_juettner_fits.c:27-129 */
    R nu_c = IPG_EE * B / (2. * pi * IPG_ME * IPG_CL);
    R nu_s = (2. / 9.) * nu_c * sth * Th2;
    R X = nu / nu_s;
    R prefactor = (Ne * (IPG_EE * IPG_EE) * nu_c) / IPG_CL;
    R cX = cbrt(X);
    R eX = exp(-cX);
    R sX = sqrt(X), X16 = sqrt(cX);
    double t1 = 1.4142135623730951 * pi / 27. * sth;
    R tI = sX + 1.8877486253633868 * X16;
    jI = prefactor * t1 * (tI * tI) * eX;
    R te = pow(Thetae, 24. / 25.);
    R tq = (7. * te + 35.) / (10. * te + 75.);
    R tQ = sX + tq * 1.8877486253633868 * X16;
    jQ = prefactor * t1 * (tQ * tQ) * eX;
    R v1 = (37. - 87. * sin(theta - 28. / 25.)) / (100. * (Thetae + 1.));
    R v2 = pow(1. + (pow(Thetae, 3. / 5.) / 25. + 7. / 10.) * pow(X, 9. / 25.), 5. / 3.);
    jV = prefactor * v1 * v2 * eX;
  } else {
    /* Dexter 2016, src/symphony/maxwell_juettner_fits.c:287-356 */
    R nus = (3.0 * IPG_EE / (4.0 * pi * IPG_ME * IPG_CL)) * B * sth * Th2 + 1.0;
    R x = nu / nus;
    R cx = cbrt(x), icx = 1. / cx;
    R icx2 = icx * icx;
    R ex = exp(-1.8899 * cx);
    R iTh2 = 1. / Th2;
    R pre = (IPG_EE * IPG_EE / (2. * 1.7320508075688772 * IPG_CL)) * Ne * nu * iTh2;
    R II = 2.5651 * (1 + 1.92 * icx + 0.9977 * icx2) * ex;
    R IQ = 2.5651 * (1 + 0.93193 * icx + 0.499873 * icx2) * ex;
    R IV = (1.81384 * (icx2 * icx) + 3.42319 * icx2 + 0.0292545 * rsqrt(x) + 2.03773 * icx) * ex;
    jI = pre * II;
    jQ = pre * IQ;
    jV = (2. * IPG_EE * IPG_EE / (3. * 1.7320508075688772 * IPG_CL)) * Ne * nu * (cth / sth) * (iTh2 / Thetae) * IV;
  }
  jI *= inusq;
  jQ *= inusq;
  jV *= inusq;
  R jU = NumT<R>::c(-0. * inusq);
  R jP = sqrt(jQ * jQ + jU * jU + jV * jV);
  if (jI < jP / 0.99) {
    R pf = jI / jP * 0.99;
    jQ *= pf;
    jU *= pf;
    jV *= pf;
  }
  jr->jI = jI;
  jr->jQ = jQ;
  jr->jU = jU;
  jr->jV = jV;
  jr->aI = jI * bnu;
  jr->aQ = jQ * bnu;
  jr->aU = jU * bnu;
  jr->aV = jV * bnu;
  rho_QV(Ne, nu, Thetae, B, sth, cth, k0, k1, k2, 1, 0, &jr->rQ, &jr->rV);
  jr->rU = NumT<R>::c(0.);
}

/* Coefficients at one point for both calls the reference makes there:
 * pol = 0 (get_jkinv) into (*ju, *ku) and pol = 1 (jar_calc) into *jr. */
IPG_HEAVY void jar_both(const ModelPt &mp, const double K[4], int want_pol, int emission_type, double *ju,
                         double *ku, Jar *jr)
{
  Jar z = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0.};
  *jr = z;
  *ju = 0.;
  *ku = 0.;
  double Ne = mp.ne;
  if (Ne <= 0.) return;
  JarGeo jg;
  jar_geo(mp, K, emission_type, &jg);
  jar_fits(Ne, mp.thetae, mp.bmag, jg, want_pol, emission_type, ju, ku, jr);
}

/* --------------------------------------------------------------------- */
/* Transfer steps (src/ipolarray.c:332-628)                               */
/* --------------------------------------------------------------------- */
/* The transfer step below is written once for any number type R, like the
 * fits: double for the image, dual numbers for the adjoint (derivatives
 * with respect to the Stokes vector and the coefficients).  Same<R>::T keeps
 * R deduced from the first argument only. */
template <class R>
struct Same {
  typedef R T;
};

/* src/ipolarray.c:607-628 */
template <class R>
__device__ __forceinline__ R approximate_solve(R Ii, typename Same<R>::T ji, typename Same<R>::T ki,
                                               typename Same<R>::T jf, typename Same<R>::T kf, double dl,
                                               typename Same<R>::T *tau)
{
  R javg = (ji + jf) / 2.;
  R kavg = (ki + kf) / 2.;
  R dtau = dl * kavg;
  *tau += dtau;
  if (dtau < 1.e-3) return Ii + (javg - Ii * kavg) * dl * (1. - (dtau / 2.) * (1. - dtau / 3.));
  R efac = exp(-dtau);
  return Ii * efac + (javg / kavg) * (1. - efac);
}

/* Faraday rotation over x (src/ipolarray.c:390-408 and :502-520).  evolve_N
 * turns S by the same angle in both of its half steps, so the sines and
 * cosines are computed once (faraday_rot) and applied twice (faraday_apply);
 * the small-rho branch is the linear form: c = 1, f = 0, s/rho = x. */
template <class R>
struct FaradayRotT {
  R c, ir, g; /* cos(rho x), sin(rho x) / rho, 2 sin^2(rho x / 2) / rho^2 */
};
typedef FaradayRotT<double> FaradayRot;

template <class R>
__device__ __forceinline__ FaradayRotT<R> faraday_rot(R rQ, R rU, R rV, double x)
{
  FaradayRotT<R> F;
  R rho2 = rQ * rQ + rU * rU + rV * rV;
  if (rho2 > IPG_CUT_PREVENT_NAN) {
    R rho = sqrt(rho2);
    R irho = 1. / rho;
    R s, c;
    sincos(rho * x, &s, &c);
    R sh = sin(0.5 * rho * x);
    F.c = c;
    F.ir = s * irho;
    F.g = 2. * sh * sh * (irho * irho);
  } else {
    F.c = NumT<R>::c(1.);
    F.ir = NumT<R>::c(x);
    F.g = NumT<R>::c(0.);
  }
  return F;
}

template <class R>
__device__ __forceinline__ void faraday_apply(const FaradayRotT<R> &F, typename Same<R>::T rQ,
                                              typename Same<R>::T rU, typename Same<R>::T rV, R *SQ, R *SU, R *SV)
{
  R SQ0 = *SQ, SU0 = *SU, SV0 = *SV;
  R f = (rQ * SQ0 + rU * SU0 + rV * SV0) * F.g;
  *SQ = SQ0 * F.c + rQ * f + (rU * SV0 - rV * SU0) * F.ir;
  *SU = SU0 * F.c + rU * f + (rV * SQ0 - rQ * SV0) * F.ir;
  *SV = SV0 * F.c + rV * f + (rQ * SU0 - rU * SQ0) * F.ir;
}

/* Absorption/emission full step (src/ipolarray.c:410-500) */
template <class R>
__device__ __forceinline__ void absorb_emit(const JarT<R> &c, double x, R *SI, R *SQ, R *SU, R *SV)
{
  R SI1 = *SI, SQ1 = *SQ, SU1 = *SU, SV1 = *SV;
  R aI = c.aI, aQ = c.aQ, aU = c.aU, aV = c.aV, jI = c.jI, jQ = c.jQ, jU = c.jU, jV = c.jV;
  R aP2 = aQ * aQ + aU * aU + aV * aV;
  if (aP2 > IPG_CUT_PREVENT_NAN) {
    R aP = sqrt(aP2);
    R tauP = aP * x;
    R tauI = aI * x;
    R ads0 = aQ * SQ1 + aU * SU1 + aV * SV1;
    R adj = aQ * jQ + aU * jU + aV * jV;
    R efacm = exp(-tauI + tauP);
    R efacp = exp(-tauI - tauP);
    R efac = exp(-tauI);
    /* four divisions in all: 1/aP2, 1/aI, 1/(aI - aP), 1/(aI + aP) */
    R iaP2 = 1. / aP2, i2aP2 = 0.5 * iaP2, i2aP = aP * i2aP2;
    R SI2 = efacm * (0.5 * SI1 - ads0 * i2aP) + efacp * (0.5 * SI1 + ads0 * i2aP);
    R cm = (-SI1 * aP + ads0) * i2aP2, cp = (SI1 * aP + ads0) * i2aP2;
    R SQ2 = efacm * aQ * cm + efacp * aQ * cp + efac * (SQ1 - ads0 * aQ * iaP2);
    R SU2 = efacm * aU * cm + efacp * aU * cp + efac * (SU1 - ads0 * aU * iaP2);
    R SV2 = efacm * aV * cm + efacp * aV * cp + efac * (SV1 - ads0 * aV * iaP2);
    R afacm = 1. - efacm, afac = 1. - efac, afacp = 1. - efacp;
    if (tauI - tauP <= IPG_CUT_SMALL_TAU) {
      R e = tauI - tauP;
      afacm = e * (1. - (0.5 * e) * (1. - e * (1. / 3.)));
      if (tauI <= IPG_CUT_SMALL_TAU) {
        e = tauI;
        afac = e * (1. - (0.5 * e) * (1. - e * (1. / 3.)));
        if (tauI + tauP <= IPG_CUT_SMALL_TAU) {
          e = tauI + tauP;
          afacp = e * (1. - (0.5 * e) * (1. - e * (1. / 3.)));
        }
      }
    }
    R iaI = 1. / aI;
    R adjP = adj * iaI * iaP2;
    SQ2 += afac * (jQ * iaI - aQ * adjP);
    SU2 += afac * (jU * iaI - aU * adjP);
    SV2 += afac * (jV * iaI - aV * adjP);
    R iam = 1. / (aI - aP), iap = 1. / (aI + aP);
    R m1 = (aP * jI - adj) * i2aP * iam;
    R m2 = (-aP * jI + adj) * i2aP2 * iam;
    SI2 += afacm * m1;
    SQ2 += afacm * aQ * m2;
    SU2 += afacm * aU * m2;
    SV2 += afacm * aV * m2;
    R p1 = (aP * jI + adj) * i2aP * iap;
    R p2 = (aP * jI + adj) * i2aP2 * iap;
    SI2 += afacp * p1;
    SQ2 += afacp * aQ * p2;
    SU2 += afacp * aU * p2;
    SV2 += afacp * aV * p2;
    *SI = SI2;
    *SQ = SQ2;
    *SU = SU2;
    *SV = SV2;
  } else {
    R tf = NumT<R>::c(0.);
    *SI = approximate_solve(SI1, jI, aI, jI, aI, x, &tf);
    *SQ = approximate_solve(SQ1, jQ, aI, jQ, aI, x, &tf);
    *SU = approximate_solve(SU1, jU, aI, jU, aI, x, &tf);
    *SV = approximate_solve(SV1, jV, aI, jV, aI, x, &tf);
  }
}

/* --------------------------------------------------------------------- */
/* Plasma tetrad (src/model_tetrads.c:35-127, src/tetrads.c:40-115)        */
/* --------------------------------------------------------------------- */
/* Gram-Schmidt with the lowered basis vectors kept: once e_b is normalised,
 * g e_b and e_b.g.e_b are fixed, so each projection of a vector out of e_b is
 * a 4-term dot product instead of two metric contractions (same arithmetic
 * as set_Econ_from_trial / project_out / normalize up to rounding order). */
__device__ __forceinline__ double dot4(const double a[4], const double b[4])
{
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

/* normalize (src/tetrads.c:82-98): v /= sqrt|v.g.v|; also returns g v and v.g.v */
__device__ __forceinline__ void t_normalize(const Met &g, double v[4], double gv[4], double *sq)
{
  lower(g, v, gv);
  double n2 = dot4(v, gv);
  double in = 1. / sqrt(fabs(n2));
#pragma unroll
  for (int k = 0; k < 4; k++) {
    v[k] *= in;
    gv[k] *= in;
  }
  *sq = n2 * in * in;
}

/* project_out (src/tetrads.c:100-115): a -= b (a.g.b)/(b.g.b), from g b and b.g.b */
__device__ __forceinline__ void t_project_out(double a[4], const double b[4], const double gb[4], double bsq)
{
  double f = dot4(a, gb) / bsq;
#pragma unroll
  for (int k = 0; k < 4; k++) a[k] -= b[k] * f;
}

__device__ __forceinline__ void t_trial(double E[4], int defdir, const double t[4])
{
  double norm = fabs(t[1]) + fabs(t[2]) + fabs(t[3]);
  for (int k = 0; k < 4; k++) E[k] = (norm <= IPG_SMALL) ? (double)(k == defdir) : t[k];
}

__device__ __forceinline__ double det4(const double E[4][4])
{
  double s0 = E[0][0] * E[1][1] - E[1][0] * E[0][1];
  double s1 = E[0][0] * E[1][2] - E[1][0] * E[0][2];
  double s2 = E[0][0] * E[1][3] - E[1][0] * E[0][3];
  double s3 = E[0][1] * E[1][2] - E[1][1] * E[0][2];
  double s4 = E[0][1] * E[1][3] - E[1][1] * E[0][3];
  double s5 = E[0][2] * E[1][3] - E[1][2] * E[0][3];
  double c5 = E[2][2] * E[3][3] - E[3][2] * E[2][3];
  double c4 = E[2][1] * E[3][3] - E[3][1] * E[2][3];
  double c3 = E[2][1] * E[3][2] - E[3][1] * E[2][2];
  double c2 = E[2][0] * E[3][3] - E[3][0] * E[2][3];
  double c1 = E[2][0] * E[3][2] - E[3][0] * E[2][2];
  double c0 = E[2][0] * E[3][1] - E[3][0] * E[2][1];
  return s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
}

/* Econ[a][mu] rows; returns oddflag bits 1 / 16.  Only Ecov rows 1 and 2
 * and Econ rows 1 and 2 are consumed downstream. */
/* sqrt|det g| at a point (check_handedness): Kerr-Schild based metrics
 * rho^2 sin(th) r J22; flat r^2 sin(th) (Minkowski), r^3 sin(th) (eMinkowski) */
template <int MET = IPG_MET_FMKS>
__device__ __forceinline__ double pg_gdet(const PointGeo &pg)
{
  if constexpr (MET == IPG_MET_MINK) return fabs(pg.r * pg.r * pg.sth);
  if constexpr (MET == IPG_MET_EMINK) return fabs(pg.r * pg.r * pg.r * pg.sth);
  const double a = c_grid.a;
  double rho2 = pg.r * pg.r + a * a * pg.cth * pg.cth;
  return fabs(rho2 * pg.sth * pg.r * pg.J22);
}

template <int MET = IPG_MET_FMKS>
IPG_HEAVY int plasma_tetrad(const double Ucon[4], const double Kcon[4], const double Bcon[4], const Met &g,
                             const PointGeo &pg, double Econ[4][4], double Ecov1[4], double Ecov2[4])
{
  const double ones[4] = {1., 1., 1., 1.};
  double g0[4], g1[4], g2[4], g3[4], s0, s1, s2, s3;
  t_trial(Econ[0], 0, Ucon);
  t_trial(Econ[1], 3, ones);
  t_trial(Econ[2], 2, Bcon);
  t_trial(Econ[3], 3, Kcon);
  t_normalize(g, Econ[0], g0, &s0);
  t_project_out(Econ[3], Econ[0], g0, s0);
  t_project_out(Econ[3], Econ[0], g0, s0);
  t_normalize(g, Econ[3], g3, &s3);
  t_project_out(Econ[2], Econ[0], g0, s0);
  t_project_out(Econ[2], Econ[3], g3, s3);
  t_project_out(Econ[2], Econ[0], g0, s0);
  t_project_out(Econ[2], Econ[3], g3, s3);
  t_normalize(g, Econ[2], g2, &s2);
  t_project_out(Econ[1], Econ[0], g0, s0);
  t_project_out(Econ[1], Econ[2], g2, s2);
  t_project_out(Econ[1], Econ[3], g3, s3);
  t_project_out(Econ[1], Econ[0], g0, s0);
  t_project_out(Econ[1], Econ[2], g2, s2);
  t_project_out(Econ[1], Econ[3], g3, s3);
  t_normalize(g, Econ[1], g1, &s1);
  /* check_handedness: sqrt|det g| * det(Econ) */
  double dot = pg_gdet<MET>(pg) * det4(Econ);
  int flag = 0;
  if (fabs(fabs(dot) - 1.) > 1.e-10) flag |= 1;
  double sgn = (dot < 0.) ? -1. : 1.;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    Econ[1][k] *= sgn;
    Ecov1[k] = g1[k] * sgn;
    Ecov2[k] = g2[k];
  }
  return flag;
}
