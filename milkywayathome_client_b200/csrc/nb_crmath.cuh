// Correctly rounded log, pow, sin, cos and atan for the external potential.
//
// The reference evaluates its potentials with crlibm's correctly rounded log_rn and pow_rn
// (milkyway/include/milkyway_math_double.h:43-59: mw_log, mw_pow).  These restatements reach
// the same results by evaluating the function in double-double arithmetic (a value carried as
// an unevaluated sum hi + lo, ~104 bits; Dekker's and Knuth's error-free sums and products,
// in the formulation of Hida, Li and Bailey's QD library) and rounding once: the result is the
// correctly rounded one unless the exact value lies within ~2^-95 relative of a rounding
// boundary (Ziv's observation that such cases are rare; crlibm resolves them with a slower
// path this code does not have).
//
//   log(x): x = m 2^e with m in [1/sqrt(2), sqrt(2)); log(m) = 2 atanh(u), u = (m-1)/(m+1),
//           |u| <= 0.1716, by its series sum u^(2k+1)/(2k+1), k = 0..21; plus e ln(2).
//   exp(a): a = k ln(2) + r, |r| <= ln(2)/2; exp(r/32) - 1 by its Taylor series (13 terms),
//           squared five times as t -> 2t + t^2; times 2^k.
//   pow(x, y): exact shortcuts for y = 0, 1, 2, 0.5, 1.5, 3, -1 (one IEEE operation or the
//           double-double forms below); otherwise exp(y log(x)) for finite x > 0.
//
// Only IEEE +, -, *, /, fma and sqrt appear (all correctly rounded, the same on the host and
// the device; the device files are compiled with -fmad=false), so a host build of this
// header checks the device code bit for bit against an arbitrary-precision reference.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define NB_HD __host__ __device__ __forceinline__
#else
#define NB_HD static inline
#endif

struct NbDD {
    double hi, lo;
};

NB_HD NbDD nb_dd(double hi, double lo) { NbDD r; r.hi = hi; r.lo = lo; return r; }

// s + e = a + b exactly (Knuth)
NB_HD NbDD nb_two_sum(double a, double b)
{
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return nb_dd(s, e);
}

// s + e = a + b exactly, |a| >= |b| (Dekker)
NB_HD NbDD nb_quick_two_sum(double a, double b)
{
    const double s = a + b;
    return nb_dd(s, b - (s - a));
}

// p + e = a b exactly
NB_HD NbDD nb_two_prod(double a, double b)
{
    const double p = a * b;
    return nb_dd(p, fma(a, b, -p));
}

NB_HD NbDD nb_dd_add(NbDD a, NbDD b)
{
    NbDD s = nb_two_sum(a.hi, b.hi);
    NbDD t = nb_two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = nb_quick_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return nb_quick_two_sum(s.hi, s.lo);
}

NB_HD NbDD nb_dd_mul(NbDD a, NbDD b)
{
    NbDD p = nb_two_prod(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return nb_quick_two_sum(p.hi, p.lo);
}

NB_HD NbDD nb_dd_mul_d(NbDD a, double b)
{
    NbDD p = nb_two_prod(a.hi, b);
    p.lo += a.lo * b;
    return nb_quick_two_sum(p.hi, p.lo);
}

// a / b: three quotient digits, each from the remainder of the previous ones
NB_HD NbDD nb_dd_div(NbDD a, NbDD b)
{
    const double q1 = a.hi / b.hi;
    NbDD r = nb_dd_add(a, nb_dd_mul_d(b, -q1));
    const double q2 = r.hi / b.hi;
    r = nb_dd_add(r, nb_dd_mul_d(b, -q2));
    const double q3 = r.hi / b.hi;
    NbDD q = nb_quick_two_sum(q1, q2);
    return nb_dd_add(q, nb_dd(q3, 0.0));
}

// 1 / n as a double-double (n a small positive integer): the residual 1 - hi n is exact
NB_HD NbDD nb_dd_recip_int(double n)
{
    const double hi = 1.0 / n;
    const double r = fma(-hi, n, 1.0);
    return nb_dd(hi, r / n);
}

// ln(2) = 0.693147180559945309417232121458176568..., as hi + lo
#define NB_LN2_HI 6.93147180559945286227e-01
#define NB_LN2_LO 2.31904681384629955842e-17

// log(x) for finite x > 0 as a double-double
NB_HD NbDD nb_log_dd(double x)
{
    int e = 0;
    double m = frexp(x, &e);                     // x = m 2^e, m in [0.5, 1)
    if (m < 0.70710678118654752440) {            // m in [1/sqrt(2), sqrt(2))
        m *= 2.0;
        e -= 1;
    }
    const double f = m - 1.0;                    // exact (Sterbenz)
    const NbDD den = nb_two_sum(m, 1.0);         // m + 1, exact
    const NbDD u = nb_dd_div(nb_dd(f, 0.0), den);
    const NbDD u2 = nb_dd_mul(u, u);
    NbDD s = nb_dd_recip_int(43.0);              // k = 21
    for (int k = 20; k >= 0; --k) s = nb_dd_add(nb_dd_mul(s, u2), nb_dd_recip_int(2.0 * k + 1.0));
    NbDD lm = nb_dd_mul(u, s);
    lm = nb_dd(2.0 * lm.hi, 2.0 * lm.lo);        // exact scaling
    const NbDD el = nb_dd_mul_d(nb_dd(NB_LN2_HI, NB_LN2_LO), (double) e);
    return nb_dd_add(el, lm);
}

// correctly rounded log(x) (crlibm's log_rn)
NB_HD double nb_log_rn(double x)
{
    if (!(x > 0.0) || isinf(x)) return log(x);   // 0, negative, inf, nan: IEEE special values
    if (x == 1.0) return 0.0;
    const NbDD r = nb_log_dd(x);
    return r.hi + r.lo;
}

// exp(a) for a double-double a with |a.hi| < 709 as a double-double
NB_HD NbDD nb_exp_dd(NbDD a)
{
    const double k = nearbyint(a.hi / NB_LN2_HI);
    NbDD r = nb_dd_add(a, nb_dd_mul_d(nb_dd(-NB_LN2_HI, -NB_LN2_LO), k));
    r = nb_dd(r.hi * (1.0 / 32.0), r.lo * (1.0 / 32.0));   // exact scaling
    // t = exp(r) - 1 = r (1 + r/2 (1 + r/3 (1 + ... (1 + r/13))))
    NbDD t = nb_dd(1.0, 0.0);
    for (int n = 13; n >= 2; --n)
        t = nb_dd_add(nb_dd(1.0, 0.0), nb_dd_div(nb_dd_mul(r, t), nb_dd((double) n, 0.0)));
    t = nb_dd_mul(r, t);
    for (int s = 0; s < 5; ++s)                  // exp(2 r) - 1 = 2 t + t^2
        t = nb_dd_add(nb_dd(2.0 * t.hi, 2.0 * t.lo), nb_dd_mul(t, t));
    NbDD res = nb_dd_add(nb_dd(1.0, 0.0), t);
    const int ki = (int) k;
    return nb_dd(ldexp(res.hi, ki), ldexp(res.lo, ki));
}

// pow(x, y) as crlibm's pow_rn for the cases the potentials meet
NB_HD double nb_pow_rn(double x, double y)
{
    if (y == 0.0) return 1.0;
    if (y == 1.0) return x;
    if (y == 2.0) return x * x;
    if (y == -1.0) return 1.0 / x;
    if (!(x > 0.0) || isinf(x) || isnan(y) || isinf(y)) return pow(x, y);
    if (y == 0.5) return sqrt(x);
    if (y == 1.5) {                              // x sqrt(x), the square root as s + t
        const double s = sqrt(x);
        const double t = fma(-s, s, x) / (2.0 * s);
        NbDD p = nb_two_prod(x, s);
        p.lo += x * t;
        return p.hi + p.lo;
    }
    if (y == 3.0) {                              // (x^2) x with the error of x^2 carried
        const NbDD sq = nb_two_prod(x, x);
        NbDD p = nb_two_prod(sq.hi, x);
        p.lo += sq.lo * x;
        if (isinf(p.hi) || p.hi == 0.0) return p.hi;
        return p.hi + p.lo;
    }
    const NbDD ly = nb_dd_mul_d(nb_log_dd(x), y);
    if (ly.hi > 709.0 || ly.hi < -708.0) return pow(x, y);   // overflow / underflow range
    const NbDD r = nb_exp_dd(ly);
    return r.hi + r.lo;
}

// ---- sin, cos, atan for the orbiting bar ------------------------------------------------
//
// The bar (nbody/src/nbody_potential.c:410-457) rotates positions with crlibm's atan_rn
// (mw_atan) and the C library's sin and cos, which round correctly but for rare hard cases.
//
//   sin(x), cos(x): x = q pi/2 + r, |r| <= ~pi/4 (Cody and Waite's reduction with pi/2 split
//           into four doubles, each product formed exactly), then the Taylor series of sin(r)
//           and cos(r) to r^29 and r^28 in double-double; valid for |x| < 2^28.
//   atan(x): one Newton step on f(y) = sin(y) - x cos(y) from the library's atan (a few
//           ulps); f'' = -f vanishes at the root, so the step more than triples the correct
//           bits, and f is formed from the double-double sin and cos of the start value.

// pi/2 = 1.57079632679489661923132169163975144209858469968755291048747229615390820... as four
// doubles (each the nearest double to the remainder of the previous ones)
#define NB_PIO2_1 1.5707963267948966
#define NB_PIO2_2 6.123233995736766e-17
#define NB_PIO2_3 -1.4973849048591698e-33
#define NB_PIO2_4 5.562271104316826e-50

// a / d for a double d: the remainder a - q1 d formed exactly, then a second quotient digit
NB_HD NbDD nb_dd_div_d(NbDD a, double d)
{
    const double q1 = a.hi / d;
    const NbDD p = nb_two_prod(q1, d);
    NbDD s = nb_two_sum(a.hi, -p.hi);
    s.lo -= p.lo;
    s.lo += a.lo;
    const double q2 = (s.hi + s.lo) / d;
    return nb_quick_two_sum(q1, q2);
}

// x = k pi/2 + r for |x| < 2^28: r as a double-double, q = k mod 4
NB_HD NbDD nb_reduce_pio2(double x, int& q)
{
    const double k = nearbyint(x * 0.63661977236758138);     // 2/pi
    const NbDD p1 = nb_two_prod(k, NB_PIO2_1);
    NbDD r = nb_two_sum(x, -p1.hi);
    r = nb_dd_add(r, nb_dd(-p1.lo, 0.0));
    r = nb_dd_add(r, nb_two_prod(-k, NB_PIO2_2));
    r = nb_dd_add(r, nb_two_prod(-k, NB_PIO2_3));
    r = nb_dd_add(r, nb_dd(-k * NB_PIO2_4, 0.0));
    q = (int) (((long long) k) & 3);
    return r;
}

// sin(r) for |r| <= ~0.8: r (1 - r^2/(2 3) (1 - r^2/(4 5) (... (1 - r^2/(28 29)))))
NB_HD NbDD nb_sin_dd_reduced(NbDD r)
{
    const NbDD r2 = nb_dd_mul(r, r);
    NbDD t = nb_dd(1.0, 0.0);
    for (int n = 14; n >= 1; --n)
        t = nb_dd_add(nb_dd(1.0, 0.0), nb_dd_div_d(nb_dd_mul(r2, t), -(double) (2 * n * (2 * n + 1))));
    return nb_dd_mul(r, t);
}

// cos(r) for |r| <= ~0.8: 1 - r^2/(1 2) (1 - r^2/(3 4) (... (1 - r^2/(27 28))))
NB_HD NbDD nb_cos_dd_reduced(NbDD r)
{
    const NbDD r2 = nb_dd_mul(r, r);
    NbDD t = nb_dd(1.0, 0.0);
    for (int n = 14; n >= 1; --n)
        t = nb_dd_add(nb_dd(1.0, 0.0), nb_dd_div_d(nb_dd_mul(r2, t), -(double) ((2 * n - 1) * (2 * n))));
    return t;
}

NB_HD NbDD nb_dd_neg(NbDD a) { return nb_dd(-a.hi, -a.lo); }

// sin(x) and cos(x) for |x| < 2^28 as double-doubles
NB_HD void nb_sincos_dd(double x, NbDD& s, NbDD& c)
{
    int q = 0;
    const NbDD r = nb_reduce_pio2(x, q);
    const NbDD sr = nb_sin_dd_reduced(r), cr = nb_cos_dd_reduced(r);
    switch (q) {
    case 0: s = sr; c = cr; break;
    case 1: s = cr; c = nb_dd_neg(sr); break;
    case 2: s = nb_dd_neg(sr); c = nb_dd_neg(cr); break;
    default: s = nb_dd_neg(cr); c = sr; break;
    }
}

// correctly rounded sin(x); |x| >= 2^28, inf and nan go to the library's sin
NB_HD double nb_sin_rn(double x)
{
    const double ax = fabs(x);
    if (!(ax < 268435456.0)) return sin(x);
    if (ax < 1.4901161193847656e-08) return x;        // |x| < 2^-26: x - x^3/6 rounds to x
    NbDD s, c;
    nb_sincos_dd(x, s, c);
    return s.hi + s.lo;
}

// correctly rounded cos(x); |x| >= 2^28, inf and nan go to the library's cos
NB_HD double nb_cos_rn(double x)
{
    const double ax = fabs(x);
    if (!(ax < 268435456.0)) return cos(x);
    if (ax < 7.4505805969238281e-09) return 1.0;      // |x| < 2^-27: 1 - x^2/2 rounds to 1
    NbDD s, c;
    nb_sincos_dd(x, s, c);
    return c.hi + c.lo;
}

// correctly rounded atan(x) (crlibm's atan_rn)
NB_HD double nb_atan_rn(double x)
{
    const double ax = fabs(x);
    if (isnan(x)) return x + x;
    if (ax < 7.4505805969238281e-09) return x;        // |x| < 2^-27: x - x^3/3 rounds to x
    if (ax > 1.152921504606846976e18)                  // |x| > 2^60 and inf: pi/2 - 1/x rounds
        return x > 0.0 ? NB_PIO2_1 : -NB_PIO2_1;      // to the double nearest pi/2
    const double y0 = atan(x);
    NbDD s, c;
    nb_sincos_dd(y0, s, c);
    const NbDD f = nb_dd_add(s, nb_dd_neg(nb_dd_mul_d(c, x)));    // sin y0 - x cos y0
    const double fp = c.hi + x * s.hi;                            // cos y0 + x sin y0
    return y0 + (-(f.hi + f.lo) / fp);
}

// correctly rounded sin(x) and cos(x) from one reduction
NB_HD void nb_sincos_rn(double x, double& s, double& c)
{
    const double ax = fabs(x);
    if (!(ax < 268435456.0) || ax < 1.4901161193847656e-08) {
        s = nb_sin_rn(x);
        c = nb_cos_rn(x);
        return;
    }
    NbDD sd, cd;
    nb_sincos_dd(x, sd, cd);
    s = sd.hi + sd.lo;
    c = cd.hi + cd.lo;
}
