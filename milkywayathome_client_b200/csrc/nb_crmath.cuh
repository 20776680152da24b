// Correctly rounded log and pow for the external potential.
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
