/*
 * corruscant-b200: C ABI of libcoords.so, the RA/DEC conversions
 * (replaces the reference's src/coordmath.c, same symbols and signatures,
 * bound by corruscant/twopoint/angular.py:29-35, threedim.py:30-37 and
 * fields.py:49-55).
 *
 * The results are defined by the reference as the platform libm's cos()
 * and sin() of the FP64 angles (coordmath.c:38-80).  glibc's sin/cos are not
 * correctly rounded, so no independent implementation reproduces them bit
 * for bit; these functions therefore run on the host, calling the same libm
 * in the same operation order, split over host threads for large inputs.
 */
#ifndef CORRUSCANT_B200_COORDMATH_H
#define CORRUSCANT_B200_COORDMATH_H

#ifdef __cplusplus
extern "C" {
#endif

/* coordmath.c:38-51: unit vectors, xyz interleaved (n,3) */
void radec2cart64(double *ra, double *dec, double *xyz, int n);

/* coordmath.c:58-71: scaled by distance */
void radecdist2cart64(double *ra, double *dec, double *dist, double *xyz, int n);

/* coordmath.c:73-80: theta = (90 - dec) deg, phi = ra deg, in radians */
void radec2sph64(double *ra, double *dec, double *theta, double *phi, int n);

#ifdef __cplusplus
}
#endif
#endif
