/*
 * Reverse mode of the polarized transfer step (stokes_step: Faraday half
 * step, absorption and emission, Faraday half step; src/ipolarray.c:
 * 390-520), for the adjoint's walk.  Given u = dL/dS' it returns
 * dL/dS and dL/d(jI, jQ, jV, aI, aQ, aV, rQ, rV) in one backward sweep over
 * the forward's intermediates: about three times one forward step, where
 * forward-mode dual numbers need twelve directions.  The U components of the
 * coefficients are zero on this path (the thermal fits), which the sweep
 * uses.  Each statement of the forward step (faraday_rot, faraday_apply,
 * absorb_emit, approximate_solve in ipg_device.cuh) has its transpose below,
 * in reverse order, including the small-tau series and the branches, which
 * follow the forward's values.  Included by ipg_adjoint.cuh.
 */

/* d/de of e (1 - (e/2)(1 - e/3)) = e - e^2/2 + e^3/6: the small-tau series
 * of 1 - exp(-e) in absorb_emit */
__device__ __forceinline__ double afac_series_d(double e) { return 1. - e + 0.5 * e * e; }

/* Faraday rotation with rU = 0: its three functions of rho = |(rQ, rV)| and
 * their derivatives in rho */
struct FaradayVjp {
  double c, ir, g;       /* cos(rho x), sin(rho x)/rho, 2 sin^2(rho x/2)/rho^2 */
  double dc, dir, dg;    /* their derivatives in rho (0 in the small-rho form) */
  double irho;           /* 1/rho (0 in the small-rho form) */
};

__device__ __forceinline__ FaradayVjp faraday_vjp_fwd(double rQ, double rV, double x)
{
  FaradayVjp F;
  const double rho2 = rQ * rQ + rV * rV;
  if (rho2 > IPG_CUT_PREVENT_NAN) {
    const double rho = sqrt(rho2), irho = 1. / rho;
    double s, c;
    sincos(rho * x, &s, &c);
    double sh, ch;
    sincos(0.5 * rho * x, &sh, &ch);
    F.c = c;
    F.ir = s * irho;
    F.g = 2. * sh * sh * (irho * irho);
    F.dc = -s * x;
    F.dir = (c * x - F.ir) * irho;
    F.dg = 2. * sh * ch * x * (irho * irho) - 2. * F.g * irho;
    F.irho = irho;
  } else {
    F.c = 1.;
    F.ir = x;
    F.g = 0.;
    F.dc = F.dir = F.dg = 0.;
    F.irho = 0.;
  }
  return F;
}

/* the values of faraday_apply (rU = 0) */
__device__ __forceinline__ void faraday_vjp_apply(const FaradayVjp &F, double rQ, double rV, const double S[4],
                                                  double O[4])
{
  const double f = (rQ * S[1] + rV * S[3]) * F.g;
  O[0] = S[0];
  O[1] = S[1] * F.c + rQ * f - rV * S[2] * F.ir;
  O[2] = S[2] * F.c + (rV * S[1] - rQ * S[3]) * F.ir;
  O[3] = S[3] * F.c + rV * f + rQ * S[2] * F.ir;
}

/* transpose of faraday_vjp_apply at input S: v (dL/dO) -> w (dL/dS), and
 * the gradients of its parameters added to bF[3] (c, ir, g), brQ, brV */
__device__ __forceinline__ void faraday_vjp_back(const FaradayVjp &F, double rQ, double rV, const double S[4],
                                                 const double v[4], double w[4], double bF[3], double *brQ,
                                                 double *brV)
{
  const double f = (rQ * S[1] + rV * S[3]) * F.g;
  const double bf = v[1] * rQ + v[3] * rV;
  w[0] = v[0];
  w[1] = v[1] * F.c + v[2] * rV * F.ir + bf * rQ * F.g;
  w[2] = v[2] * F.c - v[1] * rV * F.ir + v[3] * rQ * F.ir;
  w[3] = v[3] * F.c - v[2] * rQ * F.ir + bf * rV * F.g;
  bF[0] += v[1] * S[1] + v[2] * S[2] + v[3] * S[3];
  bF[1] += -v[1] * rV * S[2] + v[2] * (rV * S[1] - rQ * S[3]) + v[3] * rQ * S[2];
  bF[2] += bf * (rQ * S[1] + rV * S[3]);
  *brQ += v[1] * f - v[2] * S[3] * F.ir + v[3] * S[2] * F.ir + bf * S[1] * F.g;
  *brV += -v[1] * S[2] * F.ir + v[2] * S[1] * F.ir + v[3] * f + bf * S[3] * F.g;
}

/* approximate_solve (src/ipolarray.c:607-628) with ji = jf = j, ki = kf = k:
 * its value's gradient in (I, j, k) */
__device__ __forceinline__ void approx_solve_vjp(double I, double j, double k, double dl, double w, double *bI,
                                                 double *bj, double *bk)
{
  const double dtau = dl * k;
  if (dtau < 1.e-3) {
    const double h = 1. - (dtau / 2.) * (1. - dtau / 3.); /* 1 - d/2 + d^2/6 */
    const double dh = -0.5 + dtau / 3.;
    *bI += w * (1. - k * dl * h);
    *bj += w * dl * h;
    *bk += w * (-I * dl * h + (j - I * k) * dl * dh * dl);
  } else {
    const double e = exp(-dtau), ik = 1. / k;
    *bI += w * e;
    *bj += w * (1. - e) * ik;
    *bk += w * (-I * dl * e - j * ik * ik * (1. - e) + j * ik * dl * e);
  }
}

/* absorb_emit (src/ipolarray.c:410-500) with aU = jU = 0, reversed: w =
 * dL/d(S after) -> bS = dL/d(S before), and the coefficient gradients added
 * to bj[3] (jI, jQ, jV) and ba[3] (aI, aQ, aV) */
__device__ __forceinline__ void absorb_emit_vjp(const double S1[4], double jI, double jQ, double jV, double aI,
                                                double aQ, double aV, double x, const double w[4], double bS[4],
                                                double bj[3], double ba[3])
{
  const double SI1 = S1[0], SQ1 = S1[1], SU1 = S1[2], SV1 = S1[3];
  const double wI = w[0], wQ = w[1], wU = w[2], wV = w[3];
  const double aP2 = aQ * aQ + aV * aV;
  bS[0] = bS[1] = bS[2] = bS[3] = 0.;
  if (!(aP2 > IPG_CUT_PREVENT_NAN)) {
    approx_solve_vjp(SI1, jI, aI, x, wI, &bS[0], &bj[0], &ba[0]);
    approx_solve_vjp(SQ1, jQ, aI, x, wQ, &bS[1], &bj[1], &ba[0]);
    double bjU = 0.;
    approx_solve_vjp(SU1, 0., aI, x, wU, &bS[2], &bjU, &ba[0]);
    approx_solve_vjp(SV1, jV, aI, x, wV, &bS[3], &bj[2], &ba[0]);
    return;
  }
  /* forward intermediates */
  const double aP = sqrt(aP2), tauP = aP * x, tauI = aI * x;
  const double ads0 = aQ * SQ1 + aV * SV1, adj = aQ * jQ + aV * jV;
  const double efacm = exp(-tauI + tauP), efacp = exp(-tauI - tauP), efac = exp(-tauI);
  const double iaP2 = 1. / aP2, i2aP2 = 0.5 * iaP2, i2aP = aP * i2aP2;
  const double cm = (-SI1 * aP + ads0) * i2aP2, cp = (SI1 * aP + ads0) * i2aP2;
  double afacm = 1. - efacm, afac = 1. - efac, afacp = 1. - efacp;
  int sm = 0, s0 = 0, sp = 0; /* the small-tau series taken */
  if (tauI - tauP <= IPG_CUT_SMALL_TAU) {
    double e = tauI - tauP;
    afacm = e * (1. - (0.5 * e) * (1. - e * (1. / 3.)));
    sm = 1;
    if (tauI <= IPG_CUT_SMALL_TAU) {
      e = tauI;
      afac = e * (1. - (0.5 * e) * (1. - e * (1. / 3.)));
      s0 = 1;
      if (tauI + tauP <= IPG_CUT_SMALL_TAU) {
        e = tauI + tauP;
        afacp = e * (1. - (0.5 * e) * (1. - e * (1. / 3.)));
        sp = 1;
      }
    }
  }
  const double iaI = 1. / aI, adjP = adj * iaI * iaP2;
  const double iam = 1. / (aI - aP), iap = 1. / (aI + aP);
  const double M = aP * jI - adj, m1 = M * i2aP * iam, m2 = -M * i2aP2 * iam;
  const double P = aP * jI + adj, p1 = P * i2aP * iap, p2 = P * i2aP2 * iap;
  /* reverse sweep */
  double b_aI = 0., b_aQ = 0., b_aV = 0., b_aP = 0., b_aP2 = 0., b_jI = 0., b_jQ = 0., b_jV = 0.;
  double b_tauI = 0., b_tauP = 0., b_ads0 = 0., b_adj = 0., b_efacm = 0., b_efacp = 0., b_efac = 0.;
  double b_iaP2 = 0., b_i2aP2 = 0., b_i2aP = 0., b_cm = 0., b_cp = 0., b_iaI = 0.;
  /* SI2 += afacp p1; SQ2 += afacp aQ p2; SV2 += afacp aV p2 */
  const double b_afacp = wI * p1 + (wQ * aQ + wV * aV) * p2;
  {
    const double b_p1 = wI * afacp, b_p2 = (wQ * aQ + wV * aV) * afacp;
    b_aQ += wQ * afacp * p2;
    b_aV += wV * afacp * p2;
    const double b_P = b_p1 * i2aP * iap + b_p2 * i2aP2 * iap;
    b_i2aP += b_p1 * P * iap;
    b_i2aP2 += b_p2 * P * iap;
    const double b_iap = b_p1 * P * i2aP + b_p2 * P * i2aP2;
    b_aP += b_P * jI;
    b_jI += b_P * aP;
    b_adj += b_P;
    b_aI += -b_iap * iap * iap;
    b_aP += -b_iap * iap * iap;
  }
  /* SI2 += afacm m1; SQ2 += afacm aQ m2; SV2 += afacm aV m2 */
  const double b_afacm = wI * m1 + (wQ * aQ + wV * aV) * m2;
  {
    const double b_m1 = wI * afacm, b_m2 = (wQ * aQ + wV * aV) * afacm;
    b_aQ += wQ * afacm * m2;
    b_aV += wV * afacm * m2;
    const double b_M = b_m1 * i2aP * iam - b_m2 * i2aP2 * iam;
    b_i2aP += b_m1 * M * iam;
    b_i2aP2 += -b_m2 * M * iam;
    const double b_iam = b_m1 * M * i2aP - b_m2 * M * i2aP2;
    b_aP += b_M * jI;
    b_jI += b_M * aP;
    b_adj -= b_M;
    b_aI += -b_iam * iam * iam;
    b_aP += b_iam * iam * iam;
  }
  /* SQ2 += afac (jQ iaI - aQ adjP); SV2 += afac (jV iaI - aV adjP) */
  const double b_afac = wQ * (jQ * iaI - aQ * adjP) + wV * (jV * iaI - aV * adjP);
  {
    b_jQ += wQ * afac * iaI;
    b_jV += wV * afac * iaI;
    b_iaI += afac * (wQ * jQ + wV * jV);
    b_aQ += -wQ * afac * adjP;
    b_aV += -wV * afac * adjP;
    const double b_adjP = -afac * (wQ * aQ + wV * aV);
    b_adj += b_adjP * iaI * iaP2;
    b_iaI += b_adjP * adj * iaP2;
    b_iaP2 += b_adjP * adj * iaI;
    b_aI += -b_iaI * iaI * iaI;
  }
  /* the three attenuation factors */
  if (sm) {
    const double g = b_afacm * afac_series_d(tauI - tauP);
    b_tauI += g;
    b_tauP -= g;
  } else {
    b_efacm -= b_afacm;
  }
  if (s0) b_tauI += b_afac * afac_series_d(tauI);
  else b_efac -= b_afac;
  if (sp) {
    const double g = b_afacp * afac_series_d(tauI + tauP);
    b_tauI += g;
    b_tauP += g;
  } else {
    b_efacp -= b_afacp;
  }
  /* SV2 = efacm aV cm + efacp aV cp + efac (SV1 - ads0 aV iaP2), and SQ2 alike */
  b_efacm += (wQ * aQ + wV * aV) * cm;
  b_efacp += (wQ * aQ + wV * aV) * cp;
  b_efac += wQ * (SQ1 - ads0 * aQ * iaP2) + wV * (SV1 - ads0 * aV * iaP2) + wU * SU1;
  b_aQ += wQ * (efacm * cm + efacp * cp - efac * ads0 * iaP2);
  b_aV += wV * (efacm * cm + efacp * cp - efac * ads0 * iaP2);
  b_cm += (wQ * aQ + wV * aV) * efacm;
  b_cp += (wQ * aQ + wV * aV) * efacp;
  bS[1] += wQ * efac;
  bS[2] += wU * efac; /* SU2 = efac SU1 */
  bS[3] += wV * efac;
  b_ads0 += -efac * iaP2 * (wQ * aQ + wV * aV);
  b_iaP2 += -efac * ads0 * (wQ * aQ + wV * aV);
  /* cp = (SI1 aP + ads0) i2aP2, cm = (-SI1 aP + ads0) i2aP2 */
  bS[0] += (b_cp - b_cm) * aP * i2aP2;
  b_aP += (b_cp - b_cm) * SI1 * i2aP2;
  b_ads0 += (b_cp + b_cm) * i2aP2;
  b_i2aP2 += b_cp * (SI1 * aP + ads0) + b_cm * (-SI1 * aP + ads0);
  /* SI2 = efacm (SI1/2 - ads0 i2aP) + efacp (SI1/2 + ads0 i2aP) */
  b_efacm += wI * (0.5 * SI1 - ads0 * i2aP);
  b_efacp += wI * (0.5 * SI1 + ads0 * i2aP);
  bS[0] += wI * 0.5 * (efacm + efacp);
  b_ads0 += wI * i2aP * (efacp - efacm);
  b_i2aP += wI * ads0 * (efacp - efacm);
  /* i2aP = aP i2aP2, i2aP2 = iaP2 / 2, iaP2 = 1 / aP2 */
  b_aP += b_i2aP * i2aP2;
  b_i2aP2 += b_i2aP * aP;
  b_iaP2 += 0.5 * b_i2aP2;
  b_aP2 += -b_iaP2 * iaP2 * iaP2;
  /* the exponentials */
  b_tauI += -b_efacm * efacm - b_efacp * efacp - b_efac * efac;
  b_tauP += b_efacm * efacm - b_efacp * efacp;
  /* adj, ads0 */
  b_aQ += b_adj * jQ + b_ads0 * SQ1;
  b_aV += b_adj * jV + b_ads0 * SV1;
  b_jQ += b_adj * aQ;
  b_jV += b_adj * aV;
  bS[1] += b_ads0 * aQ;
  bS[3] += b_ads0 * aV;
  /* tauI = aI x, tauP = aP x, aP = sqrt(aP2), aP2 = aQ^2 + aV^2 */
  b_aI += b_tauI * x;
  b_aP += b_tauP * x;
  b_aP2 += b_aP * 0.5 / aP;
  b_aQ += b_aP2 * 2. * aQ;
  b_aV += b_aP2 * 2. * aV;
  bj[0] += b_jI;
  bj[1] += b_jQ;
  bj[2] += b_jV;
  ba[0] += b_aI;
  ba[1] += b_aQ;
  ba[2] += b_aV;
}

/* The VJP of stokes_step (Faraday half step x/2, absorb_emit over x,
 * Faraday half step) at S0 with coefficients cv = (jI, jQ, jV, aI, aQ, aV,
 * rQ, rV): gS = u . dS'/dS0, gc = u . dS'/dcv. */
__device__ __forceinline__ void stokes_step_vjp(const double cv[8], double x, const double S0[4], const double u[4],
                                                double gS[4], double gc[8])
{
  const double rQ = cv[6], rV = cv[7];
  const FaradayVjp F = faraday_vjp_fwd(rQ, rV, 0.5 * x);
  double S1[4], S2[4];
  faraday_vjp_apply(F, rQ, rV, S0, S1);
  double bF[3] = {0., 0., 0.}, brQ = 0., brV = 0.;
  /* S2 = absorb_emit(S1), the second rotation's input */
  {
    JarT<double> c;
    c.jI = cv[0];
    c.jQ = cv[1];
    c.jU = 0.;
    c.jV = cv[2];
    c.aI = cv[3];
    c.aQ = cv[4];
    c.aU = 0.;
    c.aV = cv[5];
    c.rQ = rQ;
    c.rU = 0.;
    c.rV = rV;
    S2[0] = S1[0];
    S2[1] = S1[1];
    S2[2] = S1[2];
    S2[3] = S1[3];
    absorb_emit(c, x, &S2[0], &S2[1], &S2[2], &S2[3]);
  }
  double v2[4], v1[4];
  faraday_vjp_back(F, rQ, rV, S2, u, v2, bF, &brQ, &brV);
  double bj[3] = {0., 0., 0.}, ba[3] = {0., 0., 0.};
  absorb_emit_vjp(S1, cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], x, v2, v1, bj, ba);
  faraday_vjp_back(F, rQ, rV, S0, v1, gS, bF, &brQ, &brV);
  /* through the rotation's functions of rho */
  const double brho = bF[0] * F.dc + bF[1] * F.dir + bF[2] * F.dg;
  brQ += brho * rQ * F.irho;
  brV += brho * rV * F.irho;
  gc[0] = bj[0];
  gc[1] = bj[1];
  gc[2] = bj[2];
  gc[3] = ba[0];
  gc[4] = ba[1];
  gc[5] = ba[2];
  gc[6] = brQ;
  gc[7] = brV;
}
