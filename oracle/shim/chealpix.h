/*
 * Stand-in for the one function of the HEALPix C library (chealpix, HEALPix
 * 3.x) that ARGOT's diffuse-radiation code calls, pix2ang_ring
 * (src/diffuse_photon/set_angle.c:45).  Test infrastructure only: chealpix
 * is not part of the reference tree and is not installed here, so its
 * published algorithm (Gorski et al. 2005, ApJ 622, 759, section 4: the
 * RING scheme) is restated: 12 nside^2 pixels of equal area in 4 nside - 1
 * iso-latitude rings; the north polar cap holds the first 2 nside (nside - 1)
 * pixels, ring i (1-based from the pole) with 4 i pixels at
 * z = 1 - i^2 / (3 nside^2), phi = (j - 1/2) pi / (2 i); the equatorial belt
 * rings hold 4 nside pixels each at z = 4/3 - 2 i / (3 nside), phi shifted by
 * half a pixel on every other ring; the south cap mirrors the north one.
 * theta = acos(z).  The library's own build (libargot_b200) computes the same
 * table with its own code; the two are compared bit for bit in the tests.
 */
#ifndef ARGOT_ORACLE_CHEALPIX_SHIM_H
#define ARGOT_ORACLE_CHEALPIX_SHIM_H

#include <math.h>

static long argot_shim_isqrt(long v)
{
  long r = (long)sqrt((double)v + 0.5);
  while (r * r > v) r--;
  while ((r + 1) * (r + 1) <= v) r++;
  return r;
}

static void pix2ang_ring(long nside, long ipix, double *theta, double *phi)
{
  const long npix = 12 * nside * nside;
  const long ncap = 2 * nside * (nside - 1);
  const double pi = 3.141592653589793238462643383279502884197;
  double z;
  if (ipix < ncap) {
    const long iring = (1 + argot_shim_isqrt(1 + 2 * ipix)) >> 1;
    const long iphi = ipix + 1 - 2 * iring * (iring - 1);
    z = 1.0 - (double)(iring * iring) / (3.0 * (double)(nside * nside));
    *phi = ((double)iphi - 0.5) * pi / (2.0 * (double)iring);
  } else if (ipix < npix - ncap) {
    const long ip = ipix - ncap;
    const long iring = ip / (4 * nside) + nside;
    const long iphi = ip % (4 * nside) + 1;
    const double fodd = ((iring + nside) & 1) ? 1.0 : 0.5;
    z = (double)(2 * nside - iring) * 2.0 / (3.0 * (double)nside);
    *phi = ((double)iphi - fodd) * pi / (2.0 * (double)nside);
  } else {
    const long ip = npix - ipix;
    const long iring = (1 + argot_shim_isqrt(2 * ip - 1)) >> 1;
    const long iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
    z = -1.0 + (double)(iring * iring) / (3.0 * (double)(nside * nside));
    *phi = ((double)iphi - 0.5) * pi / (2.0 * (double)iring);
  }
  *theta = acos(z);
}

#endif /* ARGOT_ORACLE_CHEALPIX_SHIM_H */
