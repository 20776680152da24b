// Two-component dwarf initial conditions on the GPU, one thread per body.
//
// Restates the sampler of nbGenerateMixedDwarfCore (nbody/src/nbody_mixeddwarf.c:765-1026)
// for the reference's dwarf profiles (Dwarf.plummer, nfw, general_hernquist and cored,
// nbody/src/nbody_dwarf_potential.c:36-175; Einasto has no case in the reference's
// get_density/get_potential): radii by rejection from r^2 rho(r) of the body's own component
// (r_mag, :538-574), speeds by rejection from the Eddington distribution function of that
// component in the combined potential (vel_mag, :576-618, dist_fun :471-535), the DF evaluated
// as the reference does -- five-point stencil derivatives (:63-95), the d^2rho/dpsi^2 integrand
// (fun, :368-445), a bisection root finder for the integration limit (:247-366) and its
// composite three-point Gauss quadrature (:97-209), the DF maximum by golden-section search
// (:211-245) -- then isotropic directions by rejection in the unit cube (get_components,
// :620-647), and each component recentred on its own centre of mass and velocity and shifted
// onto the orbit (cm_correction_by_comp, :649-694).  The per-component constants -- r200, the
// NFW/cored normalisations (set_vars, :696-726), the NFW/cored mass reset to the mass inside
// the sampling bound (get_extra_nfw_mass, :728-762), the bounds and the r^2 rho maxima
// (:797-903) -- are computed once on the host in the reference's order.
//
// The random numbers are not the reference's dSFMT stream: every body draws from its own
// counter-based stream (splitmix64 of the seed and the body index), so the samples agree with
// the reference's in distribution, not body for body.  The per-body work (tens of DF
// evaluations of ~330 integrand points each) is what makes the reference's sampler take ~12 min
// per 10^6 bodies on one core; here the bodies are independent threads.
#include "nb_common.cuh"
#include "nb_crmath.cuh"
#include <vector>

namespace {

// pcrit and vol_pcrit = 200 pcrit 4 pi / 3 (milkyway/include/milkyway_math_supplemental.h:224-225)
constexpr double kPcrit = 0.000679087369829744220469326744094105320596648627735869652;
constexpr double kVolPcrit = 0.568910904587397184785763397846734505212216314432372653620;

// One component of the dwarf with the constants its density and potential need.
struct NbIcComp {
    int type;                    // NBCUDA_DWARF_*
    double M, a;                 // mass (after the NFW/cored reset) and scale length
    double p0, ps, r1, rc;       // NFW/cored normalisations, cored radii
    double C2, C3;               // cored potential constants (cored_pot)
    double bound, rhoMax;        // r_mag's sampling bound and maximum of r^2 rho

    // get_density (nbody_dwarf_potential.c:207-236); the Plummer case inline, the others out of
    // line, so that the DF integrand's many evaluations keep the Plummer sampler's registers
    NB_HD double den(double r) const
    {
        if (type == NBCUDA_DWARF_PLUMMER) {
            const double x = 1.0 + (r / a) * (r / a);
            return (3.0 / (4.0 * M_PI)) * (M / (a * a * a)) * (1.0 / sqrt(x * x * x * x * x));
        }
        return den_profile(r);
    }
    // get_potential (nbody_dwarf_potential.c:176-205), the positive psi
    NB_HD double pot(double r) const
    {
        if (type == NBCUDA_DWARF_PLUMMER) return M / sqrt(r * r + a * a);
        return pot_profile(r);
    }
    __host__ __device__ __noinline__ double den_profile(double r) const
    {
        switch (type) {
        case NBCUDA_DWARF_NFW: {
            const double R = r / a;
            return p0 * (1.0 / R) * (1.0 / ((1.0 + R) * (1.0 + R)));
        }
        case NBCUDA_DWARF_GEN_HERNQUIST:
            return (1.0 / (2.0 * M_PI)) * M * a / (r * ((r + a) * (r + a) * (r + a)));
        default:                                     // cored
            if (r <= r1) return p0 / (1.0 + (r / rc) * (r / rc));
            return ps / ((r / a) * ((1.0 + r / a) * (1.0 + r / a)));
        }
    }
    // log and atan are the CUDA library's here (the samples match the reference's in
    // distribution only, and psi is evaluated ~10^5 times per body); the set-up's below are
    // correctly rounded as the reference's
    __host__ __device__ __noinline__ double pot_profile(double r) const
    {
        switch (type) {
        case NBCUDA_DWARF_NFW: {
            const double R = r / a;
            return 4.0 * M_PI * (a * a) * p0 * (1.0 / R) * log(1.0 + R);
        }
        case NBCUDA_DWARF_GEN_HERNQUIST:
            return M / (r + a);
        default:                                     // cored
            if (r <= r1)
                return -1.0 * (4.0 * M_PI * p0 * ((rc * rc) / 2.0 * log(r * r + rc * rc) +
                                                  (rc * rc * rc) / r * atan(r / rc)) + C2);
            return -1.0 * (-4.0 * M_PI * ps * (a * a * a) / r * log(1.0 + r / a) + C3 / r);
        }
    }
};

struct NbIcDwarf {
    int first, count, nBaryon;
    NbIcComp L, D;
    double pos[3], vel[3];
    unsigned long long seed;
};

// ---- random numbers: splitmix64 (Steele, Lea & Flood 2014) per body ----
struct NbRng {
    unsigned long long s;
    __device__ double uniform()                      // [0, 1)
    {
        s += 0x9E3779B97F4A7C15ull;
        unsigned long long z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double) (z >> 11) * 0x1.0p-53;
    }
};

// The two components of the body's dwarf as the DF evaluation sees them: potL/potD/psi/den
// and the masses and scale lengths.  Two forms: both components Plummer, held in four
// registers (the common case; the potential is evaluated ~10^5 times per body), and any
// profiles, read from the device table.
struct NbIcPlummerModel {
    double ML, aL, MD, aD;
    __device__ double potL(double r) const { return ML / sqrt(r * r + aL * aL); }
    __device__ double potD(double r) const { return MD / sqrt(r * r + aD * aD); }
    __device__ double psi(double r) const { return potL(r) + potD(r); }
    __device__ double den(bool dark, double r) const
    {
        const double M = dark ? MD : ML, a = dark ? aD : aL;
        const double x = 1.0 + (r / a) * (r / a);
        return (3.0 / (4.0 * M_PI)) * (M / (a * a * a)) * (1.0 / sqrt(x * x * x * x * x));
    }
    __device__ double massL() const { return ML; }
    __device__ double massD() const { return MD; }
    __device__ double scaleL() const { return aL; }
    __device__ double scaleD() const { return aD; }
};
struct NbIcModel {
    const NbIcComp* __restrict__ L;
    const NbIcComp* __restrict__ D;
    __device__ double potL(double r) const { return L->pot(r); }
    __device__ double potD(double r) const { return D->pot(r); }
    __device__ double psi(double r) const { return L->pot(r) + D->pot(r); }
    __device__ double den(bool dark, double r) const { return dark ? D->den(r) : L->den(r); }
    __device__ double massL() const { return L->M; }
    __device__ double massD() const { return D->M; }
    __device__ double scaleL() const { return L->a; }
    __device__ double scaleD() const { return D->a; }
};

// five-point stencils with h = 0.001 (first_derivative / second_derivative)
template <typename F>
__device__ __forceinline__ double d1(F f, double x)
{
    const double h = 0.001;
    const double p1 = 1.0 * f(x - 2.0 * h), p2 = -8.0 * f(x - h);
    const double p3 = -1.0 * f(x + 2.0 * h), p4 = 8.0 * f(x + h);
    return (p1 + p2 + p3 + p4) * (1.0 / (12.0 * h));
}
template <typename F>
__device__ __forceinline__ double d2(F f, double x)
{
    const double h = 0.001;
    const double p1 = -1.0 * f(x + 2.0 * h), p2 = 16.0 * f(x + h), p3 = -30.0 * f(x);
    const double p4 = 16.0 * f(x - h), p5 = -1.0 * f(x - 2.0 * h);
    return (p1 + p2 + p3 + p4 + p5) * (1.0 / (12.0 * h * h));
}

// the DF integrand d^2 rho / d psi^2 / sqrt(|E - psi|) at radius ri (fun)
template <typename Model>
__device__ double ic_integrand(const Model& m, double ri, double energy, bool dark)
{
    auto potL = [&](double r) { return m.potL(r); };
    auto potD = [&](double r) { return m.potD(r); };
    auto denC = [&](double r) { return m.den(dark, r); };
    double dpsi = d1(potL, ri) + d1(potD, ri);
    const double d2psi = d2(potL, ri) + d2(potD, ri);
    const double dden = d1(denC, ri), d2den = d2(denC, ri);
    if (dpsi == 0.0) dpsi = 1.0e-6;
    const double dsq = d2den * (1.0 / dpsi) - dden * d2psi * (1.0 / (dpsi * dpsi));
    const double diff = fabs(energy - m.psi(ri));
    const double denom = diff != 0.0 ? 1.0 / sqrt(diff)
                                     : 1.0 / sqrt(fabs(energy - m.psi(ri + 0.0001)));
    return dsq * denom;
}

// composite three-point Gauss quadrature: 100 panels over [a, 1.5 a], then 10 up to b
template <typename Model>
__device__ double ic_gauss_quad(const Model& m, double lower, double upper, double energy,
                                bool dark)
{
    const double a = lower > upper ? upper : lower, b = lower > upper ? lower : upper;
    const double benchmark = 1.5 * a;
    double hg = (benchmark - a) / 100.0;
    double lowerg = a, upperg = lowerg + hg;
    double coef2 = (lowerg + upperg) / 2.0, coef1 = (upperg - lowerg) / 2.0;
    const double c1 = 0.55555555555, c2 = 0.88888888888, c3 = 0.55555555555;
    const double x1 = -0.77459666924, x3 = 0.77459666924;
    double intv = 0.0;
    for (int counter = 0; counter <= 100000; ++counter) {
        const double x1n = coef1 * x1 + coef2, x2n = coef2, x3n = coef1 * x3 + coef2;
        intv = intv + c1 * ic_integrand(m, x1n, energy, dark) * coef1 +
               c2 * ic_integrand(m, x2n, energy, dark) * coef1 +
               c3 * ic_integrand(m, x3n, energy, dark) * coef1;
        lowerg = upperg;
        upperg = upperg + hg;
        coef2 = (lowerg + upperg) / 2.0;
        coef1 = (upperg - lowerg) / 2.0;
        if (lowerg > benchmark) hg = (b - benchmark) / 10.0;
        if (upper > lower) { if (lowerg >= upper) break; }
        else if (lower > upper) { if (lowerg >= lower) break; }
    }
    return lower > upper ? -intv : intv;
}

// bisection for psi(r) = value on [lo, hi] split in 4 intervals (root_finder); 0 if none
template <typename Model>
__device__ double ic_root(const Model& m, double value, double lo, double hi)
{
    double vals[5], bounds[5];
    for (int i = 0; i < 5; ++i) {
        double x = ((hi - lo) * (double) i) / 4.0 + lo;
        double v = m.psi(x) - value;
        if (isnan(v)) { x += 0.0001; v = m.psi(x) - value; }
        vals[i] = v;
        bounds[i] = x;
    }
    for (int q = 0; q < 4; ++q) {
        double nlo, nhi;
        if (vals[q] < 0 && vals[q + 1] > 0) { nlo = bounds[q]; nhi = bounds[q + 1]; }
        else if (vals[q] > 0 && vals[q + 1] < 0) { nlo = bounds[q + 1]; nhi = bounds[q]; }
        else continue;
        double mid = 0.0, f = 1.0;
        for (int counter = 0; fabs(f) > .0001 && counter <= 10000; ++counter) {
            mid = (nlo + nhi) / 2.0;
            f = m.psi(mid) - value;
            if (f < 0.0) nlo = mid; else nhi = mid;
        }
        return mid;
    }
    return 0.0;
}

// the Eddington DF at speed v and radius r (dist_fun)
template <typename Model>
__device__ double ic_df(const Model& m, double v, double r, bool dark)
{
    const double cons = 0.03582244801567226;
    const double energy = m.psi(r) - 0.5 * v * v;
    const double ML = m.massL(), MD = m.massD(), aL = m.scaleL(), aD = m.scaleD();
    double range = MD == 0 ? 20.0 * sqrt(fabs((ML / energy) * (ML / energy) - aL * aL))
                           : 20.0 * sqrt(fabs((MD / energy) * (MD / energy) - aD * aD));
    for (int counter = 0; m.psi(range) > energy; ++counter) {
        range = 100.0 * range;
        if (counter > 100) { range = 100.0 * (aL + aD); break; }
    }
    double up = ic_root(m, energy, 0.0, range);
    if (isinf(up) || up == 0.0 || isnan(up)) up = r;        // find_upperlimit_r's fallback
    up = fabs(up);
    const double lo = 10.0 * up;
    return v * v * cons * ic_gauss_quad(m, lo, up, energy, dark);
}

// golden-section search for the DF maximum over speeds (max_finder)
template <typename Model>
__device__ double ic_df_max(const Model& m, double r, bool dark, double a, double b,
                            double c, int limit, double tol)
{
    const double R = 0.61803399, C = 1.0 - R;
    double x0 = a, x3 = c, x1, x2;
    if (fabs(b - c) > fabs(b - a)) { x1 = b; x2 = b + (C * (c - b)); }
    else { x2 = b; x1 = b - (C * (b - a)); }
    double f1 = -ic_df(m, x1, r, dark), f2 = -ic_df(m, x2, r, dark);
    int counter = 0;
    while (fabs(x3 - x0) > (tol * (fabs(x1) + fabs(x2)))) {
        ++counter;
        if (f2 < f1) {
            x0 = x1; x1 = x2; x2 = R * x2 + C * x3;
            f1 = f2; f2 = -ic_df(m, x2, r, dark);
        } else {
            x3 = x2; x2 = x1; x1 = R * x1 + C * x0;
            f2 = f1; f1 = -ic_df(m, x1, r, dark);
        }
        if (counter > limit) break;
    }
    return f1 < f2 ? -f1 : -f2;
}

__device__ void ic_direction(NbRng& rng, double rad, double out[3])
{
    double x, y, z, rsq;
    int guard = 0;
    do {
        x = 2.0 * rng.uniform() - 1.0;
        y = 2.0 * rng.uniform() - 1.0;
        z = 2.0 * rng.uniform() - 1.0;
        rsq = x * x + y * y + z * z;
    } while ((rsq > 1.0 || rsq == 0.0) && ++guard < 1000);
    const double s = rad / sqrt(rsq);
    out[0] = x * s; out[1] = y * s; out[2] = z * s;
}

__device__ __forceinline__ unsigned long long ic_mix(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ int ic_dwarf_of(const NbIcDwarf* dw, int nD, int i)
{
    int lo = 0, hi = nD - 1;
    while (lo < hi) {                                 // last dwarf with first <= i
        const int mid = (lo + hi + 1) >> 1;
        if (dw[mid].first <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The radius and speed of one body by rejection (r_mag, vel_mag); r = v = 0 when either fails.
template <typename Model>
__device__ void ic_sample_rv(const Model& m, const NbIcComp& comp, bool dark, NbRng& rng,
                             double& rOut, double& vOut)
{
    double r = 0.0;
    for (int tries = 0; tries <= 1000 && !(isfinite(r) && r != 0.0); ++tries) {
        r = 0.0;
        for (int counter = 0; counter <= 1000; ++counter) {      // r_mag
            const double rr = rng.uniform() * comp.bound;
            const double u = rng.uniform();
            if (rr * rr * m.den(dark, rr) / comp.rhoMax > u) { r = rr; break; }
        }
    }
    double v = 0.0;
    if (isfinite(r) && r != 0.0) {
        const double vesc = 0.99 * sqrt(fabs(2.0 * m.psi(r)));
        const double dfMax = ic_df_max(m, r, dark, 0.0, 0.5 * vesc, vesc, 10, 1.0e-2);
        for (int tries = 0; tries <= 1000 && !(isfinite(v) && v != 0.0); ++tries) {
            v = 0.0;
            for (int counter = 0; counter <= 1000; ++counter) {  // vel_mag
                const double vv = rng.uniform() * vesc;
                const double u = rng.uniform();
                if (fabs(ic_df(m, vv, r, dark) / dfMax) > u) { v = vv; break; }
            }
        }
    }
    rOut = r;
    vOut = v;
}

// One body per thread: radius and speed by rejection, isotropic directions.  ALL_PLUMMER: every
// dwarf of the table has two Plummer components (their model in registers).
template <bool ALL_PLUMMER>
__global__ void k_ic_sample(const NbIcDwarf* __restrict__ dwarfs, int nD, int n,
                            double* __restrict__ px, double* __restrict__ py,
                            double* __restrict__ pz, double* __restrict__ vx,
                            double* __restrict__ vy, double* __restrict__ vz,
                            double* __restrict__ mass, int* __restrict__ types,
                            NbScalars* __restrict__ sc)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const NbIcDwarf& d = dwarfs[ic_dwarf_of(dwarfs, nD, i)];
        const int k = i - d.first;
        const bool dark = k >= d.nBaryon;
        NbRng rng{ic_mix(d.seed ^ ic_mix((unsigned long long) k + 0x51ED27ull))};
        const NbIcComp& comp = dark ? d.D : d.L;
        double r, v;
        if (ALL_PLUMMER) {
            const NbIcPlummerModel m{d.L.M, d.L.a, d.D.M, d.D.a};
            ic_sample_rv(m, comp, dark, rng, r, v);
        } else {
            const NbIcModel m{&d.L, &d.D};
            ic_sample_rv(m, comp, dark, rng, r, v);
        }
        if (!(isfinite(r) && r != 0.0 && isfinite(v) && v != 0.0)) {
            nb_raise(sc, NBODY_ERROR);                // the reference exits here
            r = v = 0.0;
        }
        double dv[3], dr[3];
        ic_direction(rng, v, dv);
        ic_direction(rng, r, dr);
        px[i] = dr[0]; py[i] = dr[1]; pz[i] = dr[2];
        vx[i] = dv[0]; vy[i] = dv[1]; vz[i] = dv[2];
        const int nDark = d.count - d.nBaryon;
        mass[i] = dark ? (nDark ? d.D.M / (double) nDark : 0.0)
                       : (d.nBaryon ? d.L.M / (double) d.nBaryon : 0.0);
        types[i] = dark ? -1 : 1;
    }
}

// Per (dwarf, component): sums of m x and m v, one block per component.  Each thread adds its
// strided share of the component's bodies in index order and the block combines the threads'
// sums by a fixed tree, so the sums -- and the recentred bodies -- are the same on every run
// (floating-point atomics would add in arrival order).
constexpr int kIcMomentThreads = 512;

__global__ void __launch_bounds__(kIcMomentThreads)
k_ic_moments(const NbIcDwarf* __restrict__ dwarfs, int nD,
             const double* __restrict__ px, const double* __restrict__ py,
             const double* __restrict__ pz, const double* __restrict__ vx,
             const double* __restrict__ vy, const double* __restrict__ vz,
             const double* __restrict__ mass, double* __restrict__ sums)
{
    __shared__ double part[6][kIcMomentThreads];
    const int seg = blockIdx.x;                       // 2 * dwarf + (dark component)
    const NbIcDwarf& d = dwarfs[seg >> 1];
    const bool dark = seg & 1;
    const int lo = d.first + (dark ? d.nBaryon : 0);
    const int hi = dark ? d.first + d.count : d.first + d.nBaryon;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int i = lo + (int) threadIdx.x; i < hi; i += kIcMomentThreads) {
        const double mi = mass[i];
        s[0] += mi * px[i]; s[1] += mi * py[i]; s[2] += mi * pz[i];
        s[3] += mi * vx[i]; s[4] += mi * vy[i]; s[5] += mi * vz[i];
    }
    for (int c = 0; c < 6; ++c) part[c][threadIdx.x] = s[c];
    __syncthreads();
    for (int w = kIcMomentThreads / 2; w > 0; w >>= 1) {
        if ((int) threadIdx.x < w)
            for (int c = 0; c < 6; ++c) part[c][threadIdx.x] += part[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 6) sums[6 * (size_t) seg + threadIdx.x] = part[threadIdx.x][0];
}

// x - cm + shift, v - cv + shift per component (cm = sum m x / component mass)
__global__ void k_ic_shift(const NbIcDwarf* __restrict__ dwarfs, int nD, int n,
                           double* __restrict__ px, double* __restrict__ py,
                           double* __restrict__ pz, double* __restrict__ vx,
                           double* __restrict__ vy, double* __restrict__ vz,
                           const double* __restrict__ sums)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int dwi = ic_dwarf_of(dwarfs, nD, i);
        const NbIcDwarf& d = dwarfs[dwi];
        const bool dark = i - d.first >= d.nBaryon;
        const double cm = dark ? d.D.M : d.L.M;
        const double* s = sums + 6 * (size_t) (2 * dwi + dark);
        px[i] = px[i] - s[0] / cm + d.pos[0];
        py[i] = py[i] - s[1] / cm + d.pos[1];
        pz[i] = pz[i] - s[2] / cm + d.pos[2];
        vx[i] = vx[i] - s[3] / cm + d.vel[0];
        vy[i] = vy[i] - s[4] / cm + d.vel[1];
        vz[i] = vz[i] - s[5] / cm + d.vel[2];
    }
}

}  // namespace

namespace {

// The component's constants as nbGenerateMixedDwarfCore sets them up: set_vars
// (nbody_mixeddwarf.c:696-726), the sampling bound with get_extra_nfw_mass for NFW and cored
// components (:728-762, :797-831), the cored potential's constants (cored_pot,
// nbody_dwarf_potential.c:139-175) and the maximum of r^2 rho at its analytic radius (:873-903).
// rscaleL and rscaleD: both components' scale lengths (the Plummer/Hernquist bound).
NbIcComp nb_ic_setup(const NBodyCudaDwarfComponent& in, double rscaleL, double rscaleD)
{
    NbIcComp c{};
    c.type = in.type;
    c.M = in.mass;
    c.a = in.scaleLength;
    c.r1 = in.r1;
    c.rc = in.rc;
    const double rs = c.a, r1 = c.r1, rc = c.rc;
    const bool cored = c.type == NBCUDA_DWARF_CORED;
    const double r200 = cbrt(c.M / kVolPcrit);
    if (cored) {
        const double D1 = r1 * ((1.0 + r1 / rs) * (1.0 + r1 / rs)) / (rs + rs * ((r1 / rc) * (r1 / rc)));
        const double D2 = (rs * rs * rs) * (nb_log_rn(1.0 + r200 / rs) - nb_log_rn(1.0 + r1 / rs) -
                                            r200 / (rs + r200) + r1 / (rs + r1));
        const double D3 = (rc * rc) * (r1 - rc * nb_atan_rn(r1 / rc));
        c.p0 = c.M / (4.0 * M_PI * (D1 * D2 + D3));
        c.ps = c.p0 * D1;
    } else {
        const double conc = r200 / rs;
        const double term = nb_log_rn(1.0 + conc) - conc / (1.0 + conc);
        c.p0 = 200.0 * (conc * conc * conc) * kPcrit / (3.0 * term);
    }
    if (c.type == NBCUDA_DWARF_NFW || cored) {
        c.bound = 5.0 * r200;
        const double r = c.bound;                    // the mass inside the bound
        if (cored) {
            const double C1 = 0;
            const double C3 = C1 + 4 * M_PI * (c.ps * (rs * rs * rs) * (nb_log_rn((1 + r1 / rs)) - r1 / (rs + r1)) -
                                               c.p0 * (rc * rc) * (r1 - rc * nb_atan_rn(r1 / rc)));
            if (r <= r1)
                c.M = 4.0 * M_PI * c.p0 * (rc * rc) * (r - rc * nb_atan_rn(r / rc)) - C1;
            else
                c.M = 4.0 * M_PI * c.ps * (rs * rs * rs) * (nb_log_rn((rs + r) / rs) - r / (rs + r)) - C3;
        } else {
            c.M = 4.0 * M_PI * c.p0 * (rs * rs * rs) * (nb_log_rn((rs + r) / rs) - r / (rs + r));
        }
    } else {
        c.bound = 50.0 * (rscaleL + rscaleD);
    }
    if (cored) {
        c.C3 = 4.0 * M_PI * (c.ps * (rs * rs * rs) * (nb_log_rn((1.0 + r1 / rs)) - r1 / (rs + r1)) -
                             c.p0 * (rc * rc) * (r1 - rc * nb_atan_rn(r1 / rc)));
        c.C2 = c.C3 / r1 - (4.0 * M_PI) / r1 *
                               (c.ps * (rs * rs * rs) * nb_log_rn(1 + r1 / rs) +
                                c.p0 * (((rc * rc) * r1) / 2.0 * nb_log_rn((r1 * r1) + (rc * rc)) +
                                        (rc * rc * rc) * nb_atan_rn(r1 / rc)));
    }
    double rmax;
    switch (c.type) {
    case NBCUDA_DWARF_NFW: rmax = rs; break;
    case NBCUDA_DWARF_GEN_HERNQUIST: rmax = rs / 2.0; break;
    case NBCUDA_DWARF_CORED: rmax = rs > r1 ? rs : r1; break;
    default: rmax = sqrt(2.0 / 3.0) * rs; break;
    }
    c.rhoMax = (rmax * rmax) * c.den(rmax);
    return c;
}

}  // namespace

// The two components' particle masses as the sampler assigns them (after the NFW/cored reset).
void nb_ic_particle_masses(const NBodyCudaMixedDwarf& h, double out[2])
{
    const NbIcComp L = nb_ic_setup(h.light, h.light.scaleLength, h.dark.scaleLength);
    const NbIcComp D = nb_ic_setup(h.dark, h.light.scaleLength, h.dark.scaleLength);
    const int nDark = h.nbody - h.nbodyBaryon;
    out[0] = h.nbodyBaryon ? L.M / (double) h.nbodyBaryon : 0.0;
    out[1] = nDark ? D.M / (double) nDark : 0.0;
}

// Samples every dwarf of the table into the SoA body arrays (bodies [first, first + count) of
// each dwarf) and their types; scratch needs 12 doubles per dwarf.  One launch per phase for all
// dwarfs.  Returns the number of launches.
int nb_launch_ic(const NBodyCudaMixedDwarf* host, int nD, const int* firsts, void* dTable,
                 double* scratch, NbTreeBuffers& b, int* types, int n, int numSMs, NbScalars* sc,
                 cudaStream_t s)
{
    std::vector<NbIcDwarf> t(nD);
    for (int k = 0; k < nD; ++k) {
        const NBodyCudaMixedDwarf& h = host[k];
        NbIcDwarf& d = t[k];
        d.first = firsts[k];
        d.count = h.nbody;
        d.nBaryon = h.nbodyBaryon;
        d.L = nb_ic_setup(h.light, h.light.scaleLength, h.dark.scaleLength);
        d.D = nb_ic_setup(h.dark, h.light.scaleLength, h.dark.scaleLength);
        for (int c = 0; c < 3; ++c) { d.pos[c] = h.position[c]; d.vel[c] = h.velocity[c]; }
        d.seed = h.seed;
    }
    cudaMemcpyAsync(dTable, t.data(), sizeof(NbIcDwarf) * nD, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(scratch, 0, sizeof(double) * 12 * (size_t) nD, s);
    const NbIcDwarf* dt = (const NbIcDwarf*) dTable;
    // few bodies per thread, many threads: the per-body work is long and uneven
    const int g = min((n + 127) / 128, numSMs * 64);
    bool allPlummer = true;
    for (const NbIcDwarf& d : t)
        allPlummer = allPlummer && d.L.type == NBCUDA_DWARF_PLUMMER && d.D.type == NBCUDA_DWARF_PLUMMER;
    if (allPlummer)
        k_ic_sample<true><<<g, 128, 0, s>>>(dt, nD, n, b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.mass, types, sc);
    else
        k_ic_sample<false><<<g, 128, 0, s>>>(dt, nD, n, b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.mass, types, sc);
    const int g2 = min((n + 255) / 256, numSMs * 8);
    k_ic_moments<<<2 * nD, kIcMomentThreads, 0, s>>>(dt, nD, b.px, b.py, b.pz, b.vx, b.vy, b.vz,
                                                     b.mass, scratch);
    k_ic_shift<<<g2, 256, 0, s>>>(dt, nD, n, b.px, b.py, b.pz, b.vx, b.vy, b.vz, scratch);
    nb_count_launch(3);
    return 3;
}

size_t nb_ic_table_bytes(int nD) { return sizeof(NbIcDwarf) * (size_t) nD; }
