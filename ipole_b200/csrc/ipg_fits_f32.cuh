/*
 * The thermal synchrotron fits with FP32 shapes (ipg_set_fit_precision
 * IPG_FITS_FP32): the formulas of jar_fits (src/symphony/
 * maxwell_juettner_fits.c:27-395, src/radiation.c:14-23), with the work split
 * by what FP32 can hold:
 *
 *   - the shape of each fit, where the transcendental functions are (cube
 *     roots, powers, logarithms, tanh, cos, the Bessel expansions), in FP32:
 *     arguments and values of order one, or cut off long before FP32's range
 *     ends;
 *   - the prefactors (products of the constants with ne, B, nu and Theta_e,
 *     whose magnitudes run from 1e-40 to 1e+40) in FP64, a few
 *     multiplications each;
 *   - every exponential whose argument can leave FP32's range (the fits'
 *     e^-X^(1/3), the Kirchhoff e^(h nu / k T), 1 / K_2 for cold electrons)
 *     as an FP64 exponent, reduced to 2^n e^r with |r| <= ln(2)/2 in FP64
 *     and e^r taken in FP32 (exp_split);
 *   - K_n(a), a = 1/Theta_e, as a mantissa and an exponent: K_n itself for
 *     a <= 2, K_n e^a above, so that the ratios K_0/K_2, K_1/K_2 and ln K_2
 *     stay exact in FP32 where K_n underflows.  The reference's cut-offs on
 *     K_2 (its SMALL floor in the Leung fit, K_2 > 0 in the rotativities) are
 *     taken on ln K_2.
 *
 * Each coefficient keeps the relative error of its FP32 shape (about 1e-6);
 * the errors of the images against the FP64 fits are measured by the tests
 * of this mode.  Included by ipg_kernels.cu after ipg_device.cuh.
 */

template <int N>
__device__ __forceinline__ float hornerf(const double (&c)[N], float y)
{
  float r = (float)c[N - 1];
  IPG_POLY_LOOP
  for (int k = N - 2; k >= 0; k--) r = fmaf(r, y, (float)c[k]);
  return r;
}

template <int N>
__device__ __forceinline__ float clenshawf(const double (&c)[N], float s)
{
  float b1 = 0.f, b2 = 0.f, s2 = 2.f * s;
  IPG_POLY_LOOP
  for (int k = N - 1; k >= 1; k--) {
    float t = fmaf(s2, b1, (float)c[k] - b2);
    b2 = b1;
    b1 = t;
  }
  return fmaf(s, b1, (float)c[0] - b2);
}

/* 2^n as a double, n in [-1075, 1023] (built from the exponent bits; below
 * the normal range through a second factor 2^-54) */
__device__ __forceinline__ double pow2_int(int n)
{
  if (n >= -1022) return __longlong_as_double((long long)(n + 1023) << 52);
  return __longlong_as_double((long long)(n + 54 + 1023) << 52) * 5.5511151231257827e-17;
}

/* e^E for an FP64 exponent E: n = round(E / ln 2), r = E - n ln 2 in FP64,
 * e^r in FP32, times 2^n.  0 below FP64's range, inf above it. */
__device__ __forceinline__ double exp_split(double E)
{
  if (!(E > -745.1)) return (E != E) ? E : 0.;
  if (E > 709.78) return __longlong_as_double(0x7ff0000000000000LL);
  const double n = rint(E * 1.4426950408889634);
  const float r = (float)fma(n, -0.69314718055994531, E);
  return (double)expf(r) * pow2_int((int)n);
}

/* K_0, K_1, K_2 at a = 1/Theta_e (the expansions of bessel_k012) as
 * K_n = m[n] e^-shift: shift = 0 for a <= 2, shift = a above */
struct BesselF {
  float m0, m1, m2;
  double shift;
};

__device__ __forceinline__ BesselF bessel_k012_f(double a_d)
{
  BesselF b;
  const float a = (float)a_d;
  if (a <= 2.f) {
    const float EG = 0.57721566490153286061f;
    const float y = 0.25f * a * a, lg = logf(0.5f * a);
    b.m0 = -(lg + EG) * hornerf(kI0, y) + hornerf(kK0R, y);
    b.m1 = 1.f / a + lg * (0.5f * a * hornerf(kI1, y)) - 0.25f * a * hornerf(kK1R, y);
    b.m2 = b.m0 + 2.f / a * b.m1;
    b.shift = 0.;
    return b;
  }
  float f0, f1;
  if (a <= 8.f) {
    const float s = (16.f / a - 5.f) * (1.f / 3.f);
    f0 = clenshawf(kK0M, s);
    f1 = clenshawf(kK1M, s);
  } else {
    const float s = 16.f / a - 1.f;
    f0 = clenshawf(kK0F, s);
    f1 = clenshawf(kK1F, s);
  }
  const float r = rsqrtf(a);
  b.m0 = f0 * r;
  b.m1 = f1 * r;
  b.m2 = (f0 + 2.f / a * f1) * r;
  b.shift = a_d;
  return b;
}

/* 1 / Bnu_inv (src/radiation.c:14-23): (e^x - 1) c^2 / (2 h),
 * x = h nu / (me c^2 Theta_e); 0 where e^x overflows FP64, as there */
__device__ __forceinline__ double bnu_f32(double nu, double Thetae)
{
  const double x = IPG_HPL * nu / (IPG_ME * IPG_CL * IPG_CL * Thetae);
  const double c2h = (IPG_CL * IPG_CL) / (2. * IPG_HPL);
  if (x < 2.e-3) return c2h * (x / 24. * (24. + x * (12. + x * (4. + x))));
  if (x < 80.) return c2h * (double)expm1f((float)x);
  if (x > 709.78) return 0.;
  return c2h * exp_split(x);
}

/* rho_Q, rho_V (rho_QV) with FP32 shapes.  lnk2 = ln K_2 decides the
 * reference's K_2 > 0 branches (K_2 underflows in FP64 below e^-744.4);
 * kr0 = K_0/K_2 and kr1 = K_1/K_2. */
__device__ __forceinline__ void rho_QV_f32(double Ne, double nu, double Thetae, double B, double sth, double cth,
                                           float kr0, float kr1, double lnk2, int want_q, int dexter_v, double *rQ,
                                           double *rV)
{
  const double pi = 3.1415926535897932384;
  const double omega0 = (IPG_EE / (IPG_ME * IPG_CL)) * B;
  const double wp2 = (4. * pi * IPG_EE * IPG_EE / IPG_ME) * Ne;
  const double tpn = 2. * pi * nu, itpn = 1. / tpn;
  const float x = (float)(Thetae * sqrt(1.4142135623730951 * sth * (1.e3 * omega0 * itpn)));
  const bool k2pos = lnk2 > -744.44;
  if (want_q) {
    const float lx = logf(x);
    const float l16 = (x + 1.e-16f == x) ? lx : logf(x + 1.e-16f);
    const float e472 = expf(x * (-1.f / 47.2f));
    const float extraterm = (.011f * e472 - 0.011767707320949831f * 3.14159265358979f * 1.e4f * expf((-8.f / 3.f) * l16)) *
                            (0.5f + 0.5f * tanhf((lx - 4.78749174278204599425f) * 10.f));
    const float jffunc = 2.011f * expf(expf(1.035f * lx) * (-1.f / 4.7f)) -
                         cosf(0.5f * x) * expf(expf(1.2f * lx) * (-1.f / 2.73f)) - .011f * e472 + extraterm;
    const float k_ratio = k2pos ? kr1 : 1.f;
    const double itpn2 = itpn * itpn;
    const double eps11m22 = (double)jffunc * wp2 * (omega0 * omega0) * (itpn2 * itpn2) *
                            ((double)k_ratio + 6. * Thetae) * (sth * sth);
    *rQ = tpn * (0.5 / IPG_CL) * eps11m22 * nu;
  }
  double fit_factor;
  if (dexter_v && k2pos) {
    /* (K_0 - shgm) / K_2; log1p keeps the small shgm that 1/K_2 (up to
     * e^744) magnifies, which log(1 + y) loses in FP32 below y ~ 1e-7 */
    const float shgm = 0.43793091f * log1pf(0.00185777f * powf(x, 1.50316886f));
    fit_factor = (double)kr0 - (double)shgm * exp_split(-lnk2);
  } else {
    const float k_ratio = k2pos ? kr0 : 1.f;
    fit_factor = (double)(k_ratio * (1.f - 0.11f * log1pf(0.035f * x)));
  }
  const double eps12 = wp2 * omega0 * (itpn * itpn * itpn) * fit_factor * cth;
  *rV = tpn * (1. / IPG_CL) * eps12 * nu;
}

/* jar_fits with FP32 shapes and FP64 prefactors and exponents: pol = 0
 * (get_jkinv) into (*ju, *ku), pol = 1 (jar_calc) into *jr.  Ne > 0. */
__device__ __forceinline__ void jar_fits_f32(double Ne, double Thetae, double B, const JarGeo &jg, int want_pol,
                                             int emission_type, double *ju, double *ku, Jar *jr)
{
  const double pi = IPG_PI;
  const double nu = jg.nu, inusq = jg.inusq, sth = jg.sth, cth = jg.cth;
  const BesselF bk = bessel_k012_f(1. / Thetae);
  const double lnk2 = (double)logf(bk.m2) - bk.shift; /* ln K_2 */
  const float ik2 = 1.f / bk.m2;
  const float kr0 = bk.m0 * ik2, kr1 = bk.m1 * ik2;
  if (jg.along) {
    /* only rho_V, with Dexter's g(X) for emission type 4 (as jar_fits) */
    if (want_pol) {
      double rq;
      rho_QV_f32(Ne, nu, Thetae, B, sth, cth, kr0, kr1, lnk2, 0, emission_type == 4, &rq, &jr->rV);
    }
    return;
  }
  const double bnu = bnu_f32(nu, Thetae);
  const double Th2 = Thetae * Thetae;
  /* pol = 0: Leung fit, K_2 floored at SMALL */
  {
    const double nus = ((2. / 9.) * IPG_EE / (2. * pi * IPG_ME * IPG_CL)) * B * Th2 * sth;
    double j = 0.;
    if (!(nu > 1.e12 * nus)) {
      const float X = (float)(nu / nus);
      const float cx = cbrtf(X);
      float f = sqrtf(X) + 1.8877486253633868f * sqrtf(cx); /* 2^(11/12) X^(1/6) */
      f = f * f;
      const double lnK2 = fmax(lnk2, -92.103403719761836); /* ln SMALL */
      /* e^-X^(1/3) underflows to 0 in the FP64 fit beyond 745.13 */
      if (cx <= 745.13f)
        j = ((1.4142135623730951 * pi * IPG_EE * IPG_EE / (3. * IPG_CL)) * Ne * nus) * (double)f *
            exp_split(-(double)cx - lnK2);
    }
    *ju = j * inusq;
    *ku = *ju * bnu;
  }
  if (!want_pol) return;
  double jI, jQ, jV;
  if (emission_type == 1) {
    /* Pandya+ 2016 */
    const double nu_c = IPG_EE * B / (2. * pi * IPG_ME * IPG_CL);
    const double nu_s = (2. / 9.) * nu_c * sth * Th2;
    const float X = (float)(nu / nu_s);
    const double prefactor = (Ne * (IPG_EE * IPG_EE) * nu_c) / IPG_CL;
    const float cX = cbrtf(X), sX = sqrtf(X), X16 = sqrtf(cX);
    const double eX = exp_split(-(double)cX);
    const double t1 = 1.4142135623730951 * pi / 27. * sth;
    const float tI = sX + 1.8877486253633868f * X16;
    jI = prefactor * t1 * (double)(tI * tI) * eX;
    const float te = powf((float)Thetae, 24.f / 25.f);
    const float tq = (7.f * te + 35.f) / (10.f * te + 75.f);
    const float tQ = sX + tq * 1.8877486253633868f * X16;
    jQ = prefactor * t1 * (double)(tQ * tQ) * eX;
    const float v1 = (37.f - 87.f * sinf((float)(jg.theta - 28. / 25.))) / (100.f * ((float)Thetae + 1.f));
    const float v2 = powf(1.f + (powf((float)Thetae, 3.f / 5.f) / 25.f + 7.f / 10.f) * powf(X, 9.f / 25.f), 5.f / 3.f);
    jV = prefactor * (double)(v1 * v2) * eX;
  } else {
    /* Dexter 2016 */
    const double nus = (3.0 * IPG_EE / (4.0 * pi * IPG_ME * IPG_CL)) * B * sth * Th2 + 1.0;
    const float x = (float)(nu / nus);
    const float cx = cbrtf(x), icx = 1.f / cx, icx2 = icx * icx;
    const double ex = exp_split(-1.8899 * (double)cx);
    const double iTh2 = 1. / Th2;
    const double pre = (IPG_EE * IPG_EE / (2. * 1.7320508075688772 * IPG_CL)) * Ne * nu * iTh2 * ex;
    const float II = 2.5651f * (1.f + 1.92f * icx + 0.9977f * icx2);
    const float IQ = 2.5651f * (1.f + 0.93193f * icx + 0.499873f * icx2);
    const float IV = 1.81384f * (icx2 * icx) + 3.42319f * icx2 + 0.0292545f * rsqrtf(x) + 2.03773f * icx;
    jI = pre * (double)II;
    jQ = pre * (double)IQ;
    jV = (2. * IPG_EE * IPG_EE / (3. * 1.7320508075688772 * IPG_CL)) * Ne * nu * (cth / sth) * (iTh2 / Thetae) *
         (double)IV * ex;
  }
  jI *= inusq;
  jQ *= inusq;
  jV *= inusq;
  const double jP = sqrt(jQ * jQ + jV * jV);
  if (jI < jP / 0.99) {
    const double pf = jI / jP * 0.99;
    jQ *= pf;
    jV *= pf;
  }
  jr->jI = jI;
  jr->jQ = jQ;
  jr->jU = 0.;
  jr->jV = jV;
  jr->aI = jI * bnu;
  jr->aQ = jQ * bnu;
  jr->aU = 0.;
  jr->aV = jV * bnu;
  rho_QV_f32(Ne, nu, Thetae, B, sth, cth, kr0, kr1, lnk2, 1, 0, &jr->rQ, &jr->rV);
  jr->rU = 0.;
}

/* jar_both with the FP32-shape fits */
__device__ __forceinline__ void jar_both_f32(const ModelPt &mp, const double K[4], int want_pol, int emission_type,
                                             double *ju, double *ku, Jar *jr)
{
  Jar z = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0., 0.};
  *jr = z;
  *ju = 0.;
  *ku = 0.;
  if (mp.ne <= 0.) return;
  JarGeo jg;
  jar_geo(mp, K, emission_type, &jg);
  jar_fits_f32(mp.ne, mp.thetae, mp.bmag, jg, want_pol, emission_type, ju, ku, jr);
}
