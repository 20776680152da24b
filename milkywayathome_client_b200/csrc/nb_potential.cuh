// External Milky Way potential and the per-body force epilogue, shared by the walk kernels.
// Included only by translation units compiled with -fmad=false, so the expressions keep the
// reference's rounding.
#pragma once
#include "nb_common.cuh"
#include "nb_crmath.cuh"

// ---- the caustic halo (causticHaloAccel, nbody/src/nbody_caustic.c) ----
// Twenty cold dark-matter flows, each a ring caustic of radius a_n, speed V_n, infall rate
// rate_n and width p_n (the reference's tables, :32-35; the halo's Lua parameters are not
// used).  Far from a caustic a flow's field has a closed form (gfield_far, :46-62); near one
// (inside the tricusp, :286-292) it is a sum over the real roots of a quartic, found in
// complex arithmetic as the reference does it (T1..T4, f1..f5, gfield_close, :65-250):
// principal square roots, and powers as exp(c log z) with the principal logarithm (C99's
// cpow).  The reference's T2 applies the real sqrt to a complex value in its near-zero branch,
// which takes the real part (C99 6.3.1.7); that is kept.  Complex arithmetic and the library's
// log/exp/sin/cos/atan2 round differently from the C library's, so the field agrees with the
// reference's to rounding (a root-count or tricusp test that sits on its threshold can differ).
struct NbCx {
    double re, im;
};
__device__ __forceinline__ NbCx nb_cx(double re, double im = 0.0) { NbCx c; c.re = re; c.im = im; return c; }
__device__ __forceinline__ NbCx operator+(NbCx a, NbCx b) { return nb_cx(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ NbCx operator-(NbCx a, NbCx b) { return nb_cx(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ NbCx operator*(NbCx a, NbCx b)
{
    return nb_cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__device__ __forceinline__ NbCx operator*(double s, NbCx a) { return nb_cx(s * a.re, s * a.im); }
__device__ __forceinline__ NbCx nb_cx_divr(NbCx a, double s) { return nb_cx(a.re / s, a.im / s); }
// a / b by Smith's method
__device__ __forceinline__ NbCx operator/(NbCx a, NbCx b)
{
    if (fabs(b.re) >= fabs(b.im)) {
        const double r = b.im / b.re, d = b.re + b.im * r;
        return nb_cx((a.re + a.im * r) / d, (a.im - a.re * r) / d);
    }
    const double r = b.re / b.im, d = b.re * r + b.im;
    return nb_cx((a.re * r + a.im) / d, (a.im * r - a.re) / d);
}
__device__ __forceinline__ double nb_cx_abs(NbCx a) { return hypot(a.re, a.im); }
// principal square root
__device__ __forceinline__ NbCx nb_cx_sqrt(NbCx a)
{
    if (a.im == 0.0) {
        if (a.re < 0.0) return nb_cx(0.0, copysign(sqrt(-a.re), a.im));
        return nb_cx(fabs(sqrt(a.re)), copysign(0.0, a.im));
    }
    const double d = hypot(a.re, a.im);
    if (a.re > 0.0) {
        const double r = sqrt(0.5 * (d + a.re));
        return nb_cx(r, 0.5 * (a.im / r));
    }
    const double t = sqrt(0.5 * (d - a.re));
    return nb_cx(fabs(0.5 * (a.im / t)), copysign(t, a.im));
}
// a^c for a real exponent c: exp(c log a), principal branch
__device__ __forceinline__ NbCx nb_cx_pow(NbCx a, double c)
{
    if (a.re == 0.0 && a.im == 0.0) return nb_cx(0.0, 0.0);
    const double lr = log(hypot(a.re, a.im)), li = atan2(a.im, a.re);
    const double m = exp(c * lr);
    double sn, cs;
    sincos(c * li, &sn, &cs);
    return nb_cx(m * cs, m * sn);
}

__device__ const double kCauA[21] = {1.0, 40.1, 20.1, 13.6, 10.4, 8.4, 7.0, 6.1, 5.3, 4.8, 4.3,
                                     4.0, 3.7, 3.4, 3.2, 3.0, 2.8, 2.7, 2.5, 2.4, 2.3};
__device__ const double kCauV[21] = {1.0, 517, 523, 523, 523, 522, 521, 521, 520, 517, 515,
                                     512, 510, 507, 505, 503, 501, 499, 497, 496, 494};
__device__ const double kCauRate[21] = {1.0, 53, 23, 14, 10, 7.8, 6.3, 5.3, 4.5, 3.9, 3.4,
                                        3.1, 2.8, 2.5, 2.3, 2.1, 2.0, 1.8, 1.7, 1.6, 1.5};
__device__ const double kCauP[21] = {1.0, 0.3, 0.3, 1.0, 0.3, 0.15, 0.12, 0.6, 0.23, 0.41, 0.25,
                                     0.19, 0.17, 0.11, 0.09, 0.09, 0.09, 0.09, 0.09, 0.09, 0.09};

__device__ __forceinline__ NbCx nb_cau_f1(NbCx x) { return nb_cx_divr(nb_cx(2.0) + 4.0 * x, 3.0); }
__device__ __forceinline__ NbCx nb_cau_f2(NbCx x, NbCx z)
{
    const NbCx om = nb_cx(1.0) - x;
    return 4.0 * (om * om - 3.0 * z * z);
}
__device__ __forceinline__ NbCx nb_cau_f3(NbCx x, NbCx z)
{
    const NbCx xm = x - nb_cx(1.0);
    return -128.0 * nb_cx_pow(xm, 3.0) - 1728.0 * z * z - 1152.0 * xm * z * z;
}
__device__ __forceinline__ NbCx nb_cau_f4(NbCx x, NbCx z)
{
    const NbCx f2 = nb_cau_f2(x, z), f3 = nb_cau_f3(x, z);
    const NbCx disc = nb_cx_sqrt(-256.0 * f2 * f2 * f2 + f3 * f3);
    return nb_cx_pow(nb_cx_divr(f3 + disc, 2.0), 1.0 / 3.0);
}
// T1..T4 (k = 0..3): the roots of the quartic, the signs of the reference's four forms
__device__ __forceinline__ NbCx nb_cau_T(int k, NbCx x, NbCx z)
{
    const double sA = (k < 2) ? -1.0 : 1.0;              // before the first square root
    const double sB = (k == 0 || k == 2) ? -1.0 : 1.0;   // before the second
    const double sX = (k < 2) ? -1.0 : 1.0;              // before 2 x / (first root)
    const NbCx f1 = nb_cau_f1(x), f4 = nb_cau_f4(x, z);
    if (x.re >= -0.125 && nb_cx_abs(f4) < 0.001) {
        const NbCx poly = nb_cx(-1.0) - 6.0 * x + 15.0 * x * x - 8.0 * x * x * x;
        const NbCx temp = nb_cx_divr(nb_cx_pow(poly, 1.0 / 3.0), 3.0);
        const NbCx half = nb_cx_divr(f1, 2.0) + temp;
        NbCx inner;
        if (k == 1)                                      // T2: the real sqrt of the real part
            inner = f1 - temp - nb_cx_divr(2.0 * x, sqrt(half.re));
        else
            inner = f1 - temp + sX * (2.0 * x / nb_cx_sqrt(half));
        return 0.5 * (nb_cx(1.0) + sA * nb_cx_sqrt(half) + sB * nb_cx_sqrt(inner));
    }
    const NbCx f2 = nb_cau_f2(x, z);
    const NbCx temp = nb_cx_sqrt(nb_cx_divr(f1, 2.0) + f2 / (3.0 * f4) + nb_cx_divr(f4, 12.0));
    const NbCx inner = f1 - f2 / (3.0 * f4) - nb_cx_divr(f4, 12.0) + sX * (2.0 * x / temp);
    return 0.5 * (nb_cx(1.0) + sA * temp + sB * nb_cx_sqrt(inner));
}
__device__ __forceinline__ NbCx nb_cau_f5(NbCx x, NbCx z, double T)
{
    return nb_cx_divr(nb_cx_sqrt(nb_cx(2.0 * T - 1.0) + x - nb_cx(0.0, 1.0) * z), 2.0);
}

__device__ __forceinline__ void nb_cau_far(double rho, double z, int n, double& rf, double& zf)
{
    const double rsq = rho * rho + z * z;
    const double shift = kCauA[n] + kCauP[n] / 4.0;
    const double An = (8.0 * M_PI * 1.0 * kCauRate[n] * 4498.6589) / (kCauV[n] * 1.0226831);
    const double sv = hypot(rsq - shift * shift, 2.0 * shift * z);
    const double factor = (-An) / (sv * (2.0 * shift * shift + sv));
    rf += factor * (rsq * rho - shift * shift * rho);
    zf += factor * (rsq * z + shift * shift * z);
}

static __device__ __noinline__ void nb_cau_close(double rho, double zIn, int n, double& rf,
                                                 double& zf)
{
    const NbCx z = nb_cx(zIn / kCauP[n]);
    const NbCx x = nb_cx((rho - kCauA[n]) / kCauP[n]);
    double im[4], re[4];
    for (int k = 0; k < 4; ++k) {
        const NbCx t = nb_cau_T(k, x, z);
        im[k] = fabs(t.im);
        re[k] = t.re;
    }
    int count = 0;
    for (int i = 0; i < 4; ++i) if (im[i] < 0.00001) count++;
    if (count == 4)                                      // ascending
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j)
                if (re[i] > re[j]) { const double t = re[i]; re[i] = re[j]; re[j] = t; }
    double re2[2] = {0.0, 0.0};
    if (count == 2) {
        int c = 0;
        for (int i = 0; i < 4; ++i)
            if (im[i] < 0.00001 && c < 2) re2[c++] = re[i];
        if (re2[0] > re2[1]) { const double t = re2[0]; re2[0] = re2[1]; re2[1] = t; }
    }
    const double factor = -8.0 * M_PI * 1.0 * kCauRate[n] * 4498.6589 / (rho * kCauV[n] * 1.0226831);
    if (count == 2) {                                    // outside the caustic
        const NbCx a = nb_cau_f5(x, z, re2[1]), b = nb_cau_f5(x, z, re2[0]);
        rf += factor * (a.re - b.re - 0.5);
        zf += factor * (a.im - b.im);
    } else {                                             // inside: four roots
        const NbCx a = nb_cau_f5(x, z, re[3]), b = nb_cau_f5(x, z, re[2]);
        const NbCx c = nb_cau_f5(x, z, re[1]), d = nb_cau_f5(x, z, re[0]);
        rf += factor * (a.re - b.re + c.re - d.re - 0.5);
        zf += factor * (a.im - b.im + c.im - d.im);
    }
}

static __device__ __noinline__ double3 nb_caustic_accel(double x, double y, double z)
{
    double rf = 0.0, zf = 0.0;
    const double rho = sqrt(x * x + y * y);
    for (int n = 1; n <= 20; ++n) {
        const double an = kCauA[n], pn = kCauP[n];
        const double root = sqrt(1.0 + (8.0 / pn) * (rho - an));
        const double R = (3.0 - root) / 4.0, l = (3.0 + root) / 4.0;
        const double tr = 2.0 * pn * sqrt((R * R * R) * (1.0 - R));
        const double tl = 2.0 * pn * sqrt((l * l * l) * (1.0 - l));
        if ((z <= tr && z >= 0.0 && rho >= an && rho <= an + pn) ||
            (z >= tl && z <= tr && rho >= (an - pn / 8.0) && rho <= an) ||
            (z >= -tr && z <= 0.0 && rho >= an && rho <= an + pn) ||
            (z <= -tl && z >= -tr && rho >= (an - pn / 8.0) && rho <= an))
            nb_cau_close(rho, z, n, rf, zf);
        else
            nb_cau_far(rho, z, n, rf, zf);
    }
    if (rho < 0.000001) return make_double3(0.0, 0.0, zf);
    return make_double3((rf * x) / rho, (rf * y) / rho, zf);
}

// The halos of nbody/src/nbody_potential.c:518-625 beyond the logarithmic and NFW ones:
// the caustic halo (above), triaxial logarithmic (:518-541, constants c1..c3 as
// nbody/src/nbody_check_params.c:182-194 sets them), Allen-Santillan (:543-561),
// Wilkinson-Evans (:563-573), NFW by mass (:575-585), Plummer (:587-592), Hernquist
// (:594-599) and the Ninkovic special case (:601-625), in the reference's operation order.
// Their powers and logarithms are correctly rounded (nb_crmath.cuh), as crlibm's pow_rn and
// log_rn in the reference, so these halos reproduce the reference bit for bit.
// CAUSTIC = false leaves the caustic halo's code out (callers that never meet it: its register
// demand would otherwise set the allocation of the whole kernel).
template <bool CAUSTIC = true>
__device__ __forceinline__ void nb_halo_accel_more(const NbPot& p, double x, double y, double z,
                                                   double r, double& tx, double& ty, double& tz)
{
    const double a = p.haloA, M = p.haloMass;
    double c = 0.0;                    // acceleration = pos * c for the spherical halos
    switch (p.haloType) {
    case NBCUDA_CAUSTIC_HALO: {
        if (CAUSTIC) {
            const double3 t = nb_caustic_accel(x, y, z);
            tx = t.x; ty = t.y; tz = t.z;
        } else {
            tx = ty = tz = 0.0;
        }
        return;
    }
    case NBCUDA_TRIAXIAL_HALO: {
        const double qzs = p.haloQz * p.haloQz;
        const double rhalosqr = a * a;
        const double mvsqr = -(p.haloV * p.haloV);
        const double xsqr = x * x, ysqr = y * y, zsqr = z * z;
        const double arst = rhalosqr + (p.haloC1 * xsqr) + (p.haloC3 * x * y) + (p.haloC2 * ysqr);
        const double arst2 = (zsqr / qzs) + arst;
        tx = mvsqr * (((2.0 * p.haloC1) * x) + (p.haloC3 * y)) / arst2;
        ty = mvsqr * (((2.0 * p.haloC2) * y) + (p.haloC3 * x)) / arst2;
        tz = (2.0 * mvsqr * z) / ((qzs * arst) + zsqr);
        return;
    }
    case NBCUDA_ALLEN_SANTILLAN_HALO: {
        const double gam = p.haloGamma, lam = p.haloLambda;
        const double scaleR = r / a, scaleL = lam / a;
        double cc;
        if (r < lam) {
            const double pw = nb_pow_rn(scaleR, gam - 1.0);
            cc = -(M / (a * r)) * pw / (1.0 + pw);
        } else {
            cc = -(M / (r * r)) * nb_pow_rn(scaleL, gam) / (1.0 + nb_pow_rn(scaleL, gam - 1.0));
        }
        c = cc / r;
        break;
    }
    case NBCUDA_WILKINSON_EVANS_HALO: {
        const double sum2 = a * a + r * r;
        const double cc = (-M / r) * (a + sqrt(sum2)) / (sum2 + a * sqrt(sum2));
        c = cc / r;
        break;
    }
    case NBCUDA_NFW_MASS_HALO: {
        const double ar = a + r;
        c = (-M / (r * r)) * (nb_log_rn(ar / a) / r - 1 / ar);
        break;
    }
    case NBCUDA_PLUMMER_HALO: {
        const double tmp = sqrt(a * a + r * r);
        c = -M / (tmp * tmp * tmp);
        break;
    }
    case NBCUDA_HERNQUIST_HALO: {
        const double tmp = a + r;
        c = -M / (r * (tmp * tmp));
        break;
    }
    case NBCUDA_NINKOVIC_HALO: {
        const double pi = 3.1415926535;                 // the reference's constant (:35)
        const double lambda = p.haloLambda;
        const double zr = r / a, zl = lambda / a;
        const double f = 4.0 * pi / 3.0 * p.haloRho0 * (a * a * a);
        const double zl3 = zl * zl * zl;
        double menc;
        if (r > lambda) menc = f * (nb_log_rn(1.0 + zl3) - zl3 / (1 + zl3));
        else {
            const double z3 = zr * zr * zr;
            menc = f * (nb_log_rn(1.0 + z3) - z3 / (1 + zl3));
        }
        c = -menc / (r * r * r);
        break;
    }
    default:
        break;
    }
    tx = x * c; ty = y * c; tz = z * c;
}

// orbitingBarAccel (nbody/src/nbody_potential.c:410-457): the softened needle bar rotating at
// patternSpeed, at the time p.time; atan, sin and cos correctly rounded (nb_crmath.cuh: the
// reference's atan is crlibm's atan_rn, its sin and cos the C library's, which agree with the
// correctly rounded values but for ~0.1 % of arguments).
// (out of line: its double-double trigonometry would otherwise raise the register count of every
// kernel that evaluates the potential)
static __device__ __noinline__ void nb_bar_accel(const NbPot& p, double x, double y, double z,
                                             double& ox, double& oy, double& oz)
{
    const double amp = p.disk2Mass, a = p.disk2A;
    const double b = 1.4, c = 1;
    const double curAngle = (p.disk2Pattern * p.time * -1) + p.disk2StartAngle;
    double Radi = sqrt(x * x + y * y);
    double Phi = nb_atan_rn(y / x);
    Phi -= curAngle;
    if (x < 0) Radi = Radi * -1;
    double sPhi, cPhi;
    nb_sincos_rn(Phi, sPhi, cPhi);
    const double xr = Radi * cPhi;
    const double yr = Radi * sPhi;
    const double zr = z;
    const double sq = sqrt(c * c + zr * zr);
    const double secondpart = yr * yr + (b + sq) * (b + sq);
    const double Tp = sqrt((a + xr) * (a + xr) + secondpart);
    const double Tm = sqrt((a - xr) * (a - xr) + secondpart);
    const double fx = -2. * xr / Tp / Tm / (Tp + Tm);
    const double sq2 = sqrt(zr * zr + c * c);
    const double fy = -yr / 2. / Tp / Tm * (Tp + Tm - 4. * (xr * xr) / (Tp + Tm)) /
                      (yr * yr + (b + sq2) * (b + sq2));
    const double fz = fy * zr / yr * (b + sq2) / sq2;
    double sp, cp;
    nb_sincos_rn(curAngle, sp, cp);
    ox = (cp * fx - sp * fy) * amp;
    oy = (sp * fx + cp * fy) * amp;
    oz = fz * amp;
}

// nbExtAcceleration (nbody/src/nbody_potential.c:627-762) for the supported components:
// Miyamoto-Nagai disks (:173-194), logarithmic (:488-504) and NFW (:506-515) halos,
// Hernquist (:157-162) and Plummer (:164-169) bulges.
template <bool CAUSTIC = true>
__device__ __forceinline__ void nb_ext_accel(const NbPot& p, double x, double y, double z,
                                             double& ox, double& oy, double& oz)
{
    const double absv = sqrt(z * z + (y * y + x * x));
    const double limit = 0.00390625;          // mw_pow(2.0, -8.0)
    const double r = (double) (absv <= limit) * limit + (double) (absv > limit) * absv;
    double axx = 0.0, ayy = 0.0, azz = 0.0;
    if (p.diskType == NBCUDA_MIYAMOTO_NAGAI_DISK) {
        const double zp = sqrt(z * z + p.diskB * p.diskB);
        const double azp = p.diskA + zp;
        const double rp = x * x + y * y + azp * azp;
        const double rth = nb_pow_1p5(rp);
        axx = -p.diskMass * x / rth;
        ayy = -p.diskMass * y / rth;
        azz = -p.diskMass * z * azp / (zp * rth);
    }
    {
        double tx = 0.0, ty = 0.0, tz = 0.0;
        if (p.disk2Type == NBCUDA_MIYAMOTO_NAGAI_DISK) {
            const double zp = sqrt(z * z + p.disk2B * p.disk2B);
            const double azp = p.disk2A + zp;
            const double rp = x * x + y * y + azp * azp;
            const double rth = nb_pow_1p5(rp);
            tx = -p.disk2Mass * x / rth;
            ty = -p.disk2Mass * y / rth;
            tz = -p.disk2Mass * z * azp / (zp * rth);
        } else if (p.disk2Type == NBCUDA_ORBITING_BAR) {
            nb_bar_accel(p, x, y, z, tx, ty, tz);
        }
        axx = axx + tx; ayy = ayy + ty; azz = azz + tz;
    }
    {
        double tx = 0.0, ty = 0.0, tz = 0.0;
        if (p.haloType == NBCUDA_LOGARITHMIC_HALO) {
            const double q = p.haloQz, d = p.haloA, v0 = p.haloV;
            const double zq = z / q;
            const double denom = d * d + x * x + y * y + zq * zq;
            const double k = -2.0 * v0 * v0 / denom;
            tx = k * x; ty = k * y; tz = k * z / (q * q);
        } else if (p.haloType == NBCUDA_NFW_HALO) {
            const double a = p.haloA;
            const double M = p.haloV * p.haloV * a / 0.2162165954;
            const double ar = a + r;
            const double c = (-M / (r * r)) * (nb_log_rn(ar / a) / r - 1 / ar);
            tx = c * x; ty = c * y; tz = c * z;
        } else if (p.haloType != NBCUDA_NO_HALO) {
            nb_halo_accel_more<CAUSTIC>(p, x, y, z, r, tx, ty, tz);
        }
        axx = axx + tx; ayy = ayy + ty; azz = azz + tz;
    }
    {
        double tx = 0.0, ty = 0.0, tz = 0.0;
        if (p.sphType == NBCUDA_HERNQUIST_SPHERICAL) {
            const double tmp = p.sphScale + r;
            const double c = -p.sphMass / (r * (tmp * tmp));
            tx = c * x; ty = c * y; tz = c * z;
        } else if (p.sphType == NBCUDA_PLUMMER_SPHERICAL) {
            const double tmp = sqrt(p.sphScale * p.sphScale + r * r);
            const double c = -p.sphMass / nb_pow_3(tmp);
            tx = c * x; ty = c * y; tz = c * z;
        }
        axx = axx + tx; ayy = ayy + ty; azz = azz + tz;
    }
    ox = axx; oy = ayy; oz = azz;
}

// The potential Phi whose gradient nb_ext_accel returns (a = -grad Phi), for energy checks
// (not on the bit-exact path): Miyamoto-Nagai -M / sqrt(R^2 + (a + sqrt(z^2 + b^2))^2),
// logarithmic v0^2 ln(d^2 + x^2 + y^2 + z^2/q^2), NFW -M ln(1 + r/a) / r, Hernquist
// -M / (r + a), Plummer -M / sqrt(r^2 + a^2), with the same r floor of 2^-8 as the forces.
__device__ __forceinline__ double nb_ext_potential(const NbPot& p, double x, double y, double z)
{
    const double absv = sqrt(z * z + (y * y + x * x));
    const double r = absv > 0.00390625 ? absv : 0.00390625;
    double phi = 0.0;
    for (int d = 0; d < 2; ++d) {
        const int type = d == 0 ? p.diskType : p.disk2Type;
        if (type != NBCUDA_MIYAMOTO_NAGAI_DISK) continue;
        const double M = d == 0 ? p.diskMass : p.disk2Mass;
        const double a = d == 0 ? p.diskA : p.disk2A, b = d == 0 ? p.diskB : p.disk2B;
        const double azp = a + sqrt(z * z + b * b);
        phi -= M / sqrt(x * x + y * y + azp * azp);
    }
    if (p.haloType == NBCUDA_LOGARITHMIC_HALO) {
        const double zq = z / p.haloQz;
        phi += p.haloV * p.haloV * nb_log_rn(p.haloA * p.haloA + x * x + y * y + zq * zq);
    } else if (p.haloType == NBCUDA_NFW_HALO) {
        const double a = p.haloA;
        const double M = p.haloV * p.haloV * a / 0.2162165954;
        phi -= M * nb_log_rn((a + r) / a) / r;
    }
    if (p.sphType == NBCUDA_HERNQUIST_SPHERICAL)
        phi -= p.sphMass / (r + p.sphScale);
    else if (p.sphType == NBCUDA_PLUMMER_SPHERICAL)
        phi -= p.sphMass / sqrt(r * r + p.sphScale * p.sphScale);
    return phi;
}

// nbMapForceBody's epilogue (nbody/src/nbody_grav.c:167-176): a += nbExtAcceleration(pos)
// + plummerAccel(pos, LMC at the origin, mass 0, scale 1), whose value is (0 - pos) * 0.
template <bool CAUSTIC = true>
__device__ __forceinline__ void nb_finish_body(const NbPot& pot, const NbWalkParams& wp, unsigned j,
                                               double x0, double y0, double z0, double accx,
                                               double accy, double accz, double* __restrict__ ax,
                                               double* __restrict__ ay, double* __restrict__ az,
                                               double* __restrict__ vx, double* __restrict__ vy,
                                               double* __restrict__ vz)
{
    if (pot.enabled) {
        double ex, ey, ez;
        nb_ext_accel<CAUSTIC>(pot, x0, y0, z0, ex, ey, ez);
        if (pot.lmc) {
            // plummerAccel(pos, LMCpos, LMCmass, LMCscale) (nbody/src/nbody_potential.c:145-152)
            const double lx = pot.lmc[0], ly = pot.lmc[1], lz = pot.lmc[2];
            const double dist = sqrt((x0 - lx) * (x0 - lx) + (y0 - ly) * (y0 - ly) +
                                     (z0 - lz) * (z0 - lz));
            const double tmp = sqrt(pot.lmcScale * pot.lmcScale + dist * dist);
            const double c = pot.lmcMass / nb_pow_3(tmp);
            ex = ex + (lx - x0) * c;
            ey = ey + (ly - y0) * c;
            ez = ez + (lz - z0) * c;
        } else {
            // without an LMC the reference adds a massless one at the origin
            ex = ex + (0.0 - x0) * 0.0;
            ey = ey + (0.0 - y0) * 0.0;
            ez = ez + (0.0 - z0) * 0.0;
        }
        accx = accx + ex; accy = accy + ey; accz = accz + ez;
    }
    ax[j] = accx; ay[j] = accy; az[j] = accz;
    if (wp.kick) {
        // advanceVelocities (nbody/src/nbody_plain.c:301-315): v += (a + acc_i1) * dtHalf
        vx[j] = vx[j] + wp.dtHalf * (accx + wp.shift[0]);
        vy[j] = vy[j] + wp.dtHalf * (accy + wp.shift[1]);
        vz[j] = vz[j] + wp.dtHalf * (accz + wp.shift[2]);
    }
}

