// External Milky Way potential and the per-body force epilogue, shared by the walk kernels.
// Included only by translation units compiled with -fmad=false, so the expressions keep the
// reference's rounding.
#pragma once
#include "nb_common.cuh"
#include "nb_crmath.cuh"

// The halos of nbody/src/nbody_potential.c:518-625 beyond the logarithmic and NFW ones
// (the caustic halo is not supported): triaxial logarithmic (:518-541, constants c1..c3 as
// nbody/src/nbody_check_params.c:182-194 sets them), Allen-Santillan (:543-561),
// Wilkinson-Evans (:563-573), NFW by mass (:575-585), Plummer (:587-592), Hernquist
// (:594-599) and the Ninkovic special case (:601-625), in the reference's operation order.
// Their powers and logarithms are correctly rounded (nb_crmath.cuh), as crlibm's pow_rn and
// log_rn in the reference, so these halos reproduce the reference bit for bit.
__device__ __forceinline__ void nb_halo_accel_more(const NbPot& p, double x, double y, double z,
                                                   double r, double& tx, double& ty, double& tz)
{
    const double a = p.haloA, M = p.haloMass;
    double c = 0.0;                    // acceleration = pos * c for the spherical halos
    switch (p.haloType) {
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
            nb_halo_accel_more(p, x, y, z, r, tx, ty, tz);
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
__device__ __forceinline__ void nb_finish_body(const NbPot& pot, const NbWalkParams& wp, unsigned j,
                                               double x0, double y0, double z0, double accx,
                                               double accy, double accz, double* __restrict__ ax,
                                               double* __restrict__ ay, double* __restrict__ az,
                                               double* __restrict__ vx, double* __restrict__ vy,
                                               double* __restrict__ vz)
{
    if (pot.enabled) {
        double ex, ey, ez;
        nb_ext_accel(pot, x0, y0, z0, ex, ey, ez);
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

