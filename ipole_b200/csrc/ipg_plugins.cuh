/* Model plugins of the ray kernels: the iharm grid model and the reference's
 * known-answer models, as compile-time policies.
 *
 * ipole selects its model at build time (makefile:2, MODEL=...), and so do
 * the kernels: k_geodesic, k_geodesic_count and k_coeffs are templates on
 * the plugin, whose traits fix the metric of the native coordinates; the
 * plugin's point queries (radiating_region, get_model_fourv, get_model_ne/
 * thetae/b, get_model_jar) are the functions below.  The iharm instantiation
 * is the code of ipg_device.cuh unchanged.
 *
 *   IPG_PLUG_IHARM     model/iharm/model.c: FMKS grid, thermal synchrotron
 *   IPG_PLUG_ANALYTIC  model/analytic/model.c: the GRRT test problems of
 *                      Gold et al. 2020 (models 1-5) in MKS with hslope = 1,
 *                      custom emissivities (emission_type 10)
 *   IPG_PLUG_SPHERE    model/sphere/model.c: isothermal sphere with a
 *                      poloidal field in eMinkowski, thermal synchrotron
 *
 * Header included by ipg_kernels.cu after ipg_device.cuh. */
#ifndef IPG_PLUGINS_CUH
#define IPG_PLUGINS_CUH

#define IPG_PLUG_IHARM 0
#define IPG_PLUG_ANALYTIC 1
#define IPG_PLUG_SPHERE 2

/* constants of the known-answer models (set by ipg_upload_plugin) */
struct DevPlug {
  /* analytic (model/analytic/model.c:26-27, 81-122, 146-152) */
  double A, alpha, height, l0, freqcgs, rho_unit;
  /* sphere (model/sphere/model.c:19-35, 53-85) */
  double R0, Ne0, Thetae0, B0;
  /* trace output only: analytic B_unit; sphere sigma and beta (model/sphere/model.c:161-185) */
  double b_unit, sigma0, beta0;
};
__constant__ DevPlug c_plug;

template <int P>
struct PlugT;
template <>
struct PlugT<IPG_PLUG_IHARM> {
  static constexpr int MET = IPG_MET_FMKS;
};
template <>
struct PlugT<IPG_PLUG_ANALYTIC> {
  static constexpr int MET = IPG_MET_MKS;
};
template <>
struct PlugT<IPG_PLUG_SPHERE> {
  static constexpr int MET = IPG_MET_EMINK;
};

/* theta of bl_coord (src/coordinates.c:46-97), for the sub-ring counter */
template <int MET>
__device__ __forceinline__ double bl_theta(double X1, double X2)
{
  if constexpr (MET == IPG_MET_MINK || MET == IPG_MET_EMINK) return X2;
  const DevGrid &G = c_grid;
  double E = (MET == IPG_MET_FMKS) ? exp(G.mks_smooth * (G.startx[1] - X1)) : 0.;
  double S2, C2;
  sincospi(2. * X2, &S2, &C2);
  X2P p;
  x2_parts_from(X2, S2, C2, &p);
  double th, j1, j2;
  theta_jac(X2, E, p, &th, &j1, &j2);
  return th;
}

/* radiating_region of each model */
template <int P>
__device__ __forceinline__ int radiating_t(const PointGeo &pg)
{
  const DevGrid &G = c_grid;
  if constexpr (P == IPG_PLUG_ANALYTIC) /* model/analytic/model.c:302-309 */
    return pg.r > G.Rh + 0.0001 && pg.r > G.rmin_geo && pg.r < 1000.0;
  if constexpr (P == IPG_PLUG_SPHERE) /* model/sphere/model.c:206-211 */
    return pg.r < c_plug.R0;
  /* model/iharm/model.c:2093-2098 */
  return (pg.r > G.rmin_geo && pg.r < G.rmax_geo && pg.th > G.th_beg && pg.th < (IPG_PI - G.th_beg));
}

/* get_model_ne of the analytic models (model/analytic/model.c:194-202):
 * a Gaussian torus of scale height `height` */
__device__ __forceinline__ double analytic_ne(const PointGeo &pg)
{
  double x = pg.r / 10, z = c_plug.height * pg.cth;
  double n_exp = 1. / 2 * (x * x + z * z);
  return (n_exp < 200) ? c_plug.rho_unit * exp(-n_exp) : 0;
}

/* get_model_fourv of the analytic models (model/analytic/model.c:242-298):
 * the normal observer of Boyer-Lindquist coordinates with angular momentum
 * l = l0 R^1.5 / (1 + R), R = r sin(th), carried to KS and to MKS; the field
 * is the unit X2 vector.  bl_Ucon has no r component, so bl_to_ks and
 * vec_from_ks leave it unchanged (dX/dx is diagonal in MKS). */
__device__ __forceinline__ void analytic_fourv(const PointGeo &pg, double Ucon[4], double Ucov[4], double Bcon[4],
                                               double Bcov[4])
{
  const double a = c_grid.a;
  const double r = pg.r;
  double R = r * pg.sth;
  double l = (c_plug.l0 / (1 + R)) * pow(R, 1 + 0.5);
  /* gcov_bl (src/coordinates.c:242-260) and the inverse of its t-phi block */
  double sth = fabs(pg.sth), cth = pg.cth;
  double s2 = sth * sth, a2 = a * a, r2 = r * r;
  double mu = 1. + a2 * cth * cth / r2;
  double g00 = -(1. - 2. / (r * mu));
  double g03 = -2. * a * s2 / (r * mu);
  double g33 = r2 * sth * sth * (1. + a2 / r2 + 2. * a2 * s2 / (r2 * r * mu));
  double det = g00 * g33 - g03 * g03;
  double u00 = g33 / det, u03 = -g03 / det, u33 = g00 / det;
  double ubar = sqrt(-1. / (u00 - 2. * u03 * l + u33 * l * l));
  double c0 = -ubar, c3 = l * ubar; /* bl_Ucov */
  Ucon[0] = u00 * c0 + u03 * c3;
  Ucon[1] = 0.;
  Ucon[2] = 0.;
  Ucon[3] = u03 * c0 + u33 * c3;
  lower(pg.g, Ucon, Ucov);
  Bcon[0] = 0.;
  Bcon[1] = 0.;
  Bcon[2] = 1.;
  Bcon[3] = 0.;
  lower(pg.g, Bcon, Bcov);
}

/* point queries of a non-grid model into the ModelPt of the iharm path */
template <int P>
__device__ __forceinline__ void model_point_t(const double *__restrict__ fields, double X1, double X2, double X3,
                                              const PointGeo &pg, ModelPt *mp)
{
  if constexpr (P == IPG_PLUG_IHARM) {
    model_point(fields, X1, X2, X3, pg, mp);
  } else if constexpr (P == IPG_PLUG_ANALYTIC) {
    mp->geo = pg;
    mp->in_domain = 1;
    analytic_fourv(pg, mp->Ucon, mp->Ucov, mp->Bcon, mp->Bcov);
    mp->ne = analytic_ne(pg);
    mp->thetae = 0.;
    /* get_model_b, model/analytic/model.c:300-308 (not used by its coefficients) */
    mp->bmag = sqrt(mp->Bcon[0] * mp->Bcov[0] + mp->Bcon[1] * mp->Bcov[1] + mp->Bcon[2] * mp->Bcov[2] +
                    mp->Bcon[3] * mp->Bcov[3]) *
               c_plug.b_unit;
  } else {
    /* model/sphere/model.c:124-197: fluid at rest, poloidal field */
    mp->geo = pg;
    mp->in_domain = 1;
    const int rad = radiating_t<P>(pg);
    const double B0 = c_plug.B0;
    mp->Ucon[0] = 1.;
    mp->Ucon[1] = mp->Ucon[2] = mp->Ucon[3] = 0.;
    mp->Bcon[0] = 0.;
    mp->Bcon[1] = B0 * pg.cth / pg.r;
    mp->Bcon[2] = -B0 * pg.sth / (pg.r + 1.e-8);
    mp->Bcon[3] = 0.;
    lower(pg.g, mp->Ucon, mp->Ucov);
    lower(pg.g, mp->Bcon, mp->Bcov);
    mp->ne = rad ? c_plug.Ne0 : 0.;
    mp->thetae = rad ? c_plug.Thetae0 : 0.;
    mp->bmag = rad ? B0 : 0.;
  }
}

/* get_jkinv and jar_calc at a point (src/model_radiation.c:104-169): the
 * thermal fits (with FP32 shapes when F32), or the model's own coefficients
 * for emission_type 10 (E_CUSTOM), here those of model/analytic/model.c:204-240 */
template <int P, bool F32 = false>
__device__ __forceinline__ void coeffs_t(const ModelPt &mp, const double K[4], int want_pol, int emission_type,
                                         double *ju, double *ku, Jar *jr)
{
  if constexpr (P == IPG_PLUG_ANALYTIC) {
    Jar z = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0.};
    *jr = z;
    *ju = *ku = 0.;
    const double n = mp.ne;
    if (n <= 0.) return;
    double kdu = K[0] * mp.Ucov[0] + K[1] * mp.Ucov[1] + K[2] * mp.Ucov[2] + K[3] * mp.Ucov[3];
    double nu = -kdu * IPG_ME * IPG_CL * IPG_CL / IPG_HPL;
    double f = nu / c_plug.freqcgs;
    double j = fmax(n * pow(f, -c_plug.alpha) / (nu * nu), 0.);
    double k = fmax((c_plug.A * n * pow(f, -(2.5 + c_plug.alpha)) + 1.e-54) * nu, 0.);
    *ju = j;
    *ku = k;
    if (want_pol) {
      jr->jI = j;
      jr->aI = k;
    }
  } else if constexpr (F32) {
    jar_both_f32(mp, K, want_pol, emission_type, ju, ku, jr);
  } else {
    jar_both(mp, K, want_pol, emission_type, ju, ku, jr);
  }
}

#endif
