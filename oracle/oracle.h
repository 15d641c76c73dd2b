/*
 * CPU oracle for the ipole ray pipeline -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's per-pixel computation (get_pixel,
 * src/main.c:822-883, and everything it calls on the iharm FMKS thermal path),
 * keeping the reference's operation order so that, built with
 * -ffp-contract=off, it reproduces the reference binary built the same way
 * bit for bit.  Used only by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py, as the checker of the CUDA path; nothing in
 * the product links or calls it.
 *
 * Parity pins: tests/test_oracle_pins.py checks this restatement against the
 * reference itself (oracle/_ref/ipole_nofma, built from the reference's own
 * sources) on the synthetic iharm dumps, and gsl_sf_bessel_Kn (shim) against
 * scipy/mpmath.
 */
#ifndef IPG_ORACLE_H
#define IPG_ORACLE_H

typedef struct {
  int n1, n2, n3;
  double startx[4], stopx[4], dx[4], cstartx[4], cstopx[4];
  double a, hslope, poly_xt, poly_alpha, mks_smooth, poly_norm;
  double Rh, rmin_geo, rmax_geo, th_beg, sigma_cut, sigma_cut_high;
  double L_unit;
  /* ghost-padded [(n1+2)(n2+2)(n3+2)], k fastest: U1 U2 U3 B1 B2 B3 ne thetae b sigma */
  const double *f[10];
} orc_model;

typedef struct {
  double Xcam[4];
  double Econ[4][4], Ecov[4][4];
  double fovx, fovy, rotcam, xoff, yoff, freq;
  double eps;
  int nx, ny, maxnstep;
  int only_unpolarized, emission_type, stokes_floors, target_nturns, subring_dtheta, counterjet;
} orc_camera;

/* out[9] = I_unpol, tau, tauF, I, Q, U, V, nstep, oddflag  (get_pixel outputs) */
int orc_trace_pixel(const orc_model *m, const orc_camera *c, int i, int j, double out[9]);
/* n pixels, ij[2n]; OpenMP over pixels with `threads` threads (<= 0: default) */
void orc_trace_pixels(const orc_model *m, const orc_camera *c, const int *ij, int n, double *out, int threads);
/* camera of main.c:125-168 + make_camera_tetrad; returns scale */
double orc_camera_setup(const orc_model *m, double rcam, double thetacam, double phicam, double rotcam_deg,
                        double fov_muas, double dsource_pc, int nx, int ny, double freqcgs, orc_camera *c);
/* sum of nstep over pixels from the last orc_trace_pixels call */
long long orc_last_steps(void);
/* the thermal fits of jar_calc_dist at given plasma parameters: in[5n] =
 * (nu, Ne, Thetae, B, theta), out[12n] = (jI/nu^2 and aI of pol = 0, then
 * jI jQ jU jV aI aQ aU aV rQ rV of pol = 1), zeros where Ne <= 0 */
void orc_thermal_coefficients(const double *in, int n, int dist, double *out);

#endif
