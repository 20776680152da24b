// The LMC of the reference's LMC runs: a moving Plummer sphere whose orbit is integrated with
// the dwarf's steps (nbStepSystemPlain, nbody/src/nbody_plain.c:268-360), kicked by the
// external potential and by Chandrasekhar dynamical friction (dynamicalFriction_LMC,
// nbody/src/nbody_friction.c:85-132).  The friction needs the potential's density
// (nbExtDensity, nbody/src/nbody_density.c:250-369) and an isotropic velocity dispersion from a
// 10 x 5-point Gauss quadrature (velDispersion / dispIntegrand, nbody_friction.c:19-68).  One
// thread updates the LMC's position and velocity in device memory, so a step needs no host
// round trip.  Expressions follow the reference's operation order; powers are correctly
// rounded (nb_crmath.cuh, as crlibm's pow_rn), so are the bar's atan, sin and cos; erf and exp
// are CUDA's (the reference's are the C library's): with friction on, an LMC orbit agrees with
// the reference's to rounding.
#include "nb_common.cuh"
#include "nb_potential.cuh"
#include "nb_crmath.cuh"

namespace {

constexpr double kPiRef = 3.1415926535;   // the reference's pi (nbody_density.c:20, nbody_friction.c:17)

__device__ __forceinline__ double nb_p(double x, double y) { return nb_pow_rn(x, y); }

// ---- component densities (nbody/src/nbody_density.c:23-239) ----
__device__ double nb_hernquist_density(double M, double a, double r)
{
    if (r * nb_p(r + a, 3) == 0) return 0;
    return ((M) / (2 * kPiRef * nb_p(a, 3))) * nb_p(a, 4) / (r * nb_p(r + a, 3));
}

__device__ double nb_plummer_density(double M, double a, double r)
{
    if (a == 0) return 0;
    const double r_a = r / a;
    const double rho_peak = 3 * M / (4.0 * kPiRef * nb_p(a, 3.0));
    return rho_peak * nb_p((1.0 + nb_p(r_a, 2.0)), -2.5);
}

__device__ double nb_mn_density(double M, double a, double b, double x, double y, double z)
{
    const double R = nb_p(nb_p(x, 2.0) + nb_p(y, 2.0), 0.5);
    const double zp = nb_p(nb_p(z, 2.0) + nb_p(b, 2.0), 0.5);
    const double azp = a + zp;
    const double numer = M * b * b * (a * R * R + (a + 3.0 * zp) * nb_p(azp, 2));
    const double denom = 4.0 * kPiRef * nb_p(R * R + azp * azp, 2.5) * nb_p(zp, 3.0);
    if (denom == 0) return 0;
    return numer / denom;
}

__device__ double nb_bar_density(const NbPot& p, double px, double py, double pz)
{
    const double a = p.disk2A, b = 1.4, c = 1;
    const double curAngle = (p.disk2Pattern * p.time * -1) + p.disk2StartAngle;
    double Radi = sqrt(px * px + py * py);
    double Phi = nb_atan_rn(py / px);
    Phi -= curAngle;
    if (px < 0) Radi = Radi * -1;
    double sPhi, cPhi;
    nb_sincos_rn(Phi, sPhi, cPhi);
    const double x = Radi * cPhi;
    const double y = Radi * sPhi;
    const double z = pz;
    const double zc = sqrt(nb_p(z, 2) + nb_p(c, 2));
    const double bzc2 = nb_p(b + zc, 2);
    const double bigA = b * nb_p(y, 2) + (b + 3 * zc) * bzc2;
    const double bigC = nb_p(y, 2) + bzc2;
    const double unscaled =
        nb_p(c, 2) / 24 / kPiRef / a / nb_p(bigC, 2) / nb_p(zc, 3) *
        ((x + a) * (3 * bigA * bigC + (2 * bigA + b * bigC) * nb_p(x + a, 2)) /
             nb_p(bigC + nb_p(x + a, 2), 1.5) -
         (x - a) * (3 * bigA * bigC + (2 * bigA + b * bigC) * nb_p(x - a, 2)) /
             nb_p(bigC + nb_p(x - a, 2), 1.5));
    return unscaled * p.disk2Mass;
}

// a disk's density (the orbiting bar as the second disk, as the potential supports it)
__device__ double nb_disk_density(int type, double M, double a, double b, const NbPot& p,
                                  bool second, double x, double y, double z)
{
    if (type == NBCUDA_MIYAMOTO_NAGAI_DISK) return nb_mn_density(M, a, b, x, y, z);
    if (second && type == NBCUDA_ORBITING_BAR) return nb_bar_density(p, x, y, z);
    return 0.0;                                  // none (and the Freeman disk: infinitely thin)
}

__device__ double nb_halo_density(const NbPot& p, double x, double y, double z, double r)
{
    const double a = p.haloA;
    switch (p.haloType) {
    case NBCUDA_LOGARITHMIC_HALO: {
        const double v = p.haloV, q = p.haloQz;
        const double R2 = nb_p(x, 2.0) + nb_p(y, 2.0);
        const double numer = (2.0 * q * q + 1.0) * a * a + R2 + nb_p(z, 2.0) * (2.0 - 1.0 / q / q);
        const double denom = q * q * nb_p(R2 + a * a + nb_p(z / q, 2.0), 2.0);
        return v * v * numer / 2.0 / kPiRef / denom;
    }
    case NBCUDA_NFW_HALO: {
        const double v = p.haloV;
        const double rho = v * v / 4.0 / kPiRef / a / a / 0.2162165954;
        if (r == 0) return 0;
        return rho / (r / a) / nb_p(1.0 + (r / a), 2.0);
    }
    case NBCUDA_TRIAXIAL_HALO: {
        const double v = p.haloV, q = p.haloQz;
        const double c1 = p.haloC1, c2 = p.haloC2, c3 = p.haloC3;
        const double D = a * a + c1 * nb_p(x, 2.0) + c2 * nb_p(y, 2.0) + c3 * x * y +
                         nb_p(z, 2.0) / q / q;
        const double num = 2.0 * c1 * D + 2.0 * c2 * D + 2.0 * D / q / q -
                           nb_p(2.0 * c1 * x + c3 * y, 2.0) - nb_p(2.0 * c2 * y + c3 * x, 2.0) -
                           nb_p(2.0 * z / q / q, 2.0);
        return v * v * num / 4.0 / kPiRef / D / D;
    }
    case NBCUDA_ALLEN_SANTILLAN_HALO: {
        const double M = p.haloMass, lam = p.haloLambda, gam = p.haloGamma;
        const double b = gam - 1.0;
        const double numer = nb_p(r / a, b) * (nb_p(r / a, b) + b + 1.0);
        const double denom = r * r * nb_p(1.0 + nb_p(r / a, b), 2.0);
        if (r == 0.0) return 0.0;
        if (r > lam) return 0.0;
        return M * numer / a / denom / 4.0 / kPiRef;
    }
    case NBCUDA_WILKINSON_EVANS_HALO: {
        const double M = p.haloMass;
        if (r == 0.0) return 0.0;
        return (1 / (4 * kPiRef)) * M * a * a / (r * r * nb_p(r * r + a * a, 1.5));
    }
    case NBCUDA_NFW_MASS_HALO: {
        const double M = p.haloMass;
        if (r == 0) return 0;
        return M / (r * (a + r) * (a + r) * 4.0 * kPiRef);
    }
    case NBCUDA_PLUMMER_HALO:
        return nb_plummer_density(p.haloMass, a, r);
    case NBCUDA_HERNQUIST_HALO: {
        const double M = p.haloMass;
        if (r * nb_p(r + a, 3) == 0 || 2 * kPiRef * nb_p(a, 3) == 0) return 0;
        return ((M) / (2 * kPiRef * nb_p(a, 3))) * nb_p(a, 4) / (r * nb_p(r + a, 3));
    }
    case NBCUDA_NINKOVIC_HALO: {
        const double rho = p.haloRho0, lam = p.haloLambda;
        const double density = rho * (1.0 / (1.0 + nb_p(r / a, 3.0)) - 1.0 / (1.0 + nb_p(lam / a, 3.0)));
        if (density < 0) return 0.0;
        return density;
    }
    default:
        return 0.0;
    }
}

// nbExtDensity: bulge, disk, second disk and halo, summed in that order
__device__ double nb_ext_density(const NbPot& p, double x, double y, double z)
{
    double density = 0.0;
    const double limit = 0.00390625;             // mw_pow(2.0, -8.0)
    const double absv = sqrt(z * z + (y * y + x * x));
    const double r = (double) (absv <= limit) * limit + (double) (absv > limit) * absv;
    if (p.sphType == NBCUDA_HERNQUIST_SPHERICAL) density += nb_hernquist_density(p.sphMass, p.sphScale, r);
    else if (p.sphType == NBCUDA_PLUMMER_SPHERICAL) density += nb_plummer_density(p.sphMass, p.sphScale, r);
    density += nb_disk_density(p.diskType, p.diskMass, p.diskA, p.diskB, p, false, x, y, z);
    density += nb_disk_density(p.disk2Type, p.disk2Mass, p.disk2A, p.disk2B, p, true, x, y, z);
    density += nb_halo_density(p, x, y, z, r);
    return density;
}

// dispIntegrand (nbody_friction.c:19-31): density times the radial external acceleration
__device__ double nb_disp_integrand(const NbPot& p, double x, double y, double z)
{
    double ax, ay, az;
    nb_ext_accel(p, x, y, z, ax, ay, az);
    const double mag = nb_p(z * z + (y * y + x * x), 0.5);
    const double ux = x * (1.0 / mag), uy = y * (1.0 / mag), uz = z * (1.0 / mag);
    const double a_r = fabs(az * uz + (ay * uy + ax * ux));
    const double rho = nb_ext_density(p, x, y, z);
    return rho * a_r;
}

// velDispersion (nbody_friction.c:33-68): the radial velocity dispersion at pos, integrated
// from |pos| to upperlimit in 10 intervals of 5-point Gauss quadrature; -1 when undefined
__device__ double nb_vel_dispersion(const NbPot& p, double x, double y, double z,
                                    double upperlimit)
{
    const double weights[5] = {0.2369268850561891, 0.4786286704993665, 0.5688888888888889,
                               0.4786286704993665, 0.2369268850561891};
    const double points[5] = {-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831,
                              0.9061798459386640};
    const double dist = nb_p(z * z + (y * y + x * x), 0.5);
    const int nDivs = 10;
    const double width = (upperlimit - dist) / (nDivs * 1.0);
    const double rho0 = nb_ext_density(p, x, y, z);
    if ((width <= 0) || (rho0 == 0.0)) return -1;
    double integral = 0.0;
    for (int i = 0; i < nDivs; i++) {
        const double a = dist + i * width;
        const double b = dist + (i + 1) * width;
        for (int j = 0; j < 5; j++) {
            const double r = width * points[j] / 2.0 + (a + b) / 2.0;
            const double s = r / dist;
            integral += weights[j] * nb_disp_integrand(p, x * s, y * s, z * s) * width / 2.0;
        }
    }
    return integral / rho0;
}

// dynamicalFriction_LMC (nbody_friction.c:85-132)
__device__ void nb_dyn_friction(const NbPot& p, double x, double y, double z, double vx, double vy,
                                double vz, double massLMC, int dynaFric, double coulombLog,
                                double& fx, double& fy, double& fz)
{
    fx = fy = fz = 0.0;
    if (!dynaFric) return;
    const double G_CONST = 1;
    const double thresh = 0.00390625;            // mw_pow(2, -8)
    double objectVel = sqrt(vz * vz + (vy * vy + vx * vx));
    objectVel = (double) (objectVel >= thresh) * objectVel + (double) (objectVel < thresh) * thresh;
    const double scaleLength_halo = p.haloA == 0.0 ? 1.0 : p.haloA;
    const double ln_lambda = coulombLog;
    const double density = nb_ext_density(p, x, y, z);
    const double sigma2 = nb_vel_dispersion(p, x, y, z, 50.0 * scaleLength_halo);
    const double X = sigma2 <= 0.0 ? 0.0 : objectVel / (nb_p(2 * sigma2, 0.5));
    const double acc = (-4 * kPiRef * nb_p(G_CONST, 2) * massLMC * ln_lambda * density /
                        nb_p(objectVel, 2)) *
                       (erf(X) - 2 * X / nb_p(kPiRef, 0.5) * exp(-1.0 * nb_p(X, 2)));
    fx = (acc * vx / objectVel);
    fy = (acc * vy / objectVel);
    fz = (acc * vz / objectVel);
}

// One half of the LMC's step (nbStepSystemPlain, nbody_plain.c:329-360), one thread.
// lmc = {pos.xyz, vel.xyz}.  The acceleration is the external potential's plus the friction at
// the LMC's current state; phase 0 (advancePosVel_LMC, :286-299) drifts the LMC with its
// velocity and then kicks it by (acc + shift) dt/2, phase 1 (advanceVelocities_LMC, :317-327)
// only kicks.
// advancePosVel_LMC (phase 0: drift with the old velocity, then half kick) or
// advanceVelocities_LMC (phase 1: half kick) with the external potential, the friction and the
// step's reflex acceleration (sx, sy, sz) (nbody/src/nbody_plain.c:286-325, :338-352).
__device__ void nb_lmc_update(const NbPot& p, double* lmc, int phase, double dt, double sx,
                              double sy, double sz, double massLMC, int dynaFric, double coulombLog)
{
    const double x = lmc[0], y = lmc[1], z = lmc[2];
    const double vx = lmc[3], vy = lmc[4], vz = lmc[5];
    double ex, ey, ez, fx, fy, fz;
    nb_ext_accel(p, x, y, z, ex, ey, ez);
    nb_dyn_friction(p, x, y, z, vx, vy, vz, massLMC, dynaFric, coulombLog, fx, fy, fz);
    const double ax = ex + fx, ay = ey + fy, az = ez + fz;
    const double dtHalf = 0.5 * dt;
    if (phase == 0) {
        lmc[0] = x + vx * dt;
        lmc[1] = y + vy * dt;
        lmc[2] = z + vz * dt;
    }
    lmc[3] = vx + (ax + sx) * dtHalf;
    lmc[4] = vy + (ay + sy) * dtHalf;
    lmc[5] = vz + (az + sz) * dtHalf;
}

__global__ void k_lmc_half(NbPot p, double* __restrict__ lmc, int phase, double dt, double sx,
                           double sy, double sz, double massLMC, int dynaFric, double coulombLog)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    nb_lmc_update(p, lmc, phase, dt, sx, sy, sz, massLMC, dynaFric, coulombLog);
}

// Every dwarf's LMC of a batch, one thread per dwarf: the dwarf's time step and bar time, its
// reflex acceleration of the step (sc->step in phase 0, sc->step + 1 in phase 1).  Phase 1
// follows the bodies' kick and is skipped when the evaluation failed (it is redone).
__global__ void k_b_lmc_half(NbBatchLMC L, NbForest f, const NbScalars* __restrict__ sc,
                             int phase)
{
    if (phase == 1 && nb_failed(sc)) return;
    const int k = sc->step + phase;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < f.nDwarfs; d += gridDim.x * blockDim.x) {
        NbDwarfDev& dw = f.dwarfs[d];
        NbPot p = L.pot;
        p.time = dw.time;
        const double* sh = f.lmcShift + 3 * ((size_t) d * f.nShift + k);
        nb_lmc_update(p, dw.lmc, phase, dw.dt, sh[0], sh[1], sh[2], L.mass, L.dynaFric,
                      L.coulombLog);
    }
}

}  // namespace

void nb_launch_b_lmc_half(const NbBatchLMC& lmc, const NbForest& f, const NbScalars* sc, int phase,
                          cudaStream_t s)
{
    k_b_lmc_half<<<(f.nDwarfs + 127) / 128, 128, 0, s>>>(lmc, f, sc, phase);
    nb_count_launch();
}

void nb_launch_lmc_half(const NbPot& p, double* lmc, int phase, double dt, const double* shift,
                        double massLMC, int dynaFric, double coulombLog, cudaStream_t s)
{
    k_lmc_half<<<1, 32, 0, s>>>(p, lmc, phase, dt, shift[0], shift[1], shift[2], massLMC, dynaFric,
                                coulombLog);
    nb_count_launch();
}
