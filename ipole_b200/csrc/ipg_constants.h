/* CGS constants used on the ray path.  The values are those of the
 * reference's src/constants.h:3-62 (they must be identical for parity). */
#ifndef IPG_CONSTANTS_H
#define IPG_CONSTANTS_H
#define IPG_EE (4.80320680e-10)        /* electron charge */
#define IPG_CL (2.99792458e10)         /* speed of light */
#define IPG_ME (9.1093826e-28)         /* electron mass */
#define IPG_MP (1.67262171e-24)        /* proton mass */
#define IPG_HPL (6.6260693e-27)        /* Planck constant */
#define IPG_KBOL (1.3806505e-16)       /* Boltzmann constant */
#define IPG_GNEWT (6.6742e-8)          /* gravitational constant */
#define IPG_SIGMA_THOMSON (0.665245873e-24)
#define IPG_JY (1.e-23)
#define IPG_MUAS_PER_RAD (2.06265e11)
#define IPG_PC (3.085678e18)
#define IPG_MSUN (1.989e33)
#define IPG_YEAR (31536000.)
#define IPG_SMALL (1.e-40)
#define IPG_PI 3.14159265358979323846
#endif
