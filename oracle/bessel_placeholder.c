/* Placeholder for the reference's nbody/src/nbody_bessel.c, which is a missing blob
 * in the reference tree.  Test infrastructure for the oracle build (oracle/ref.mk) only.
 * The Bessel functions feed only the double-exponential and sech^2 disks
 * (nbody/src/nbody_potential.c), which no oracle case uses; every entry point here
 * aborts so that an accidental use cannot go unnoticed. */
#include <stdio.h>
#include <stdlib.h>

static double bessel_missing(const char* name)
{
    fprintf(stderr, "oracle: %s called, but the reference's Bessel source is missing\n", name);
    abort();
    return 0.0;
}

double besselJ0(const double x) { (void) x; return bessel_missing("besselJ0"); }
double besselJ1(const double x) { (void) x; return bessel_missing("besselJ1"); }
double besselJ2(const double x) { (void) x; return bessel_missing("besselJ2"); }
double besselI0(const double x) { (void) x; return bessel_missing("besselI0"); }
double besselI1(const double x) { (void) x; return bessel_missing("besselI1"); }
double besselK0(const double x) { (void) x; return bessel_missing("besselK0"); }
double besselK1(const double x) { (void) x; return bessel_missing("besselK1"); }
double besselK2(const double x) { (void) x; return bessel_missing("besselK2"); }
double besselJ0_zero(const int n) { (void) n; return bessel_missing("besselJ0_zero"); }
double besselJ1_zero(const int n) { (void) n; return bessel_missing("besselJ1_zero"); }
double aExp(const double k, const double R, const double Rd) { (void) k; (void) R; (void) Rd; return bessel_missing("aExp"); }
double bExp(const double k, const double R, const double Rd) { (void) k; (void) R; (void) Rd; return bessel_missing("bExp"); }
