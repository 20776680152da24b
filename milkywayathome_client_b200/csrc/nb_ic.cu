// Two-component Plummer dwarf initial conditions on the GPU, one thread per body.
//
// Restates the sampler of nbGenerateMixedDwarfCore (nbody/src/nbody_mixeddwarf.c:765-1026)
// for Plummer components (Dwarf.plummer, nbody/src/nbody_dwarf_potential.c): radii by rejection
// from r^2 rho(r) of the body's own component (r_mag, :538-574), speeds by rejection from the
// Eddington distribution function of that component in the combined potential (vel_mag,
// :576-618, dist_fun :471-535), the DF evaluated as the reference does -- five-point stencil
// derivatives (:63-95), the d^2rho/dpsi^2 integrand (fun, :368-445), a bisection root finder for
// the integration limit (:247-366) and its composite three-point Gauss quadrature (:97-209),
// the DF maximum by golden-section search (:211-245) -- then isotropic directions by rejection in
// the unit cube (get_components, :620-647), and each component recentred on its own centre of
// mass and velocity and shifted onto the orbit (cm_correction_by_comp, :649-694).
//
// The random numbers are not the reference's dSFMT stream: every body draws from its own
// counter-based stream (splitmix64 of the seed and the body index), so the samples agree with
// the reference's in distribution, not body for body.  The per-body work (tens of DF
// evaluations of ~330 integrand points each) is what makes the reference's sampler take ~12 min
// per 10^6 bodies on one core; here the bodies are independent threads.
#include "nb_common.cuh"
#include <vector>

namespace {

struct NbIcDwarf {
    int first, count, nBaryon;
    double massL, rsL, massD, rsD;
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

// ---- the Plummer model of nbody_dwarf_potential.c (psi: the positive potential) ----
__device__ __forceinline__ double pl_den(double M, double a, double r)
{
    const double x = 1.0 + (r / a) * (r / a);
    const double x5 = x * x * x * x * x;
    return (3.0 / (4.0 * M_PI)) * (M / (a * a * a)) * (1.0 / sqrt(x5));
}
__device__ __forceinline__ double pl_pot(double M, double a, double r)
{
    return M / sqrt(r * r + a * a);
}

struct NbIcModel {
    double ML, aL, MD, aD;
    __device__ double psi(double r) const { return pl_pot(ML, aL, r) + pl_pot(MD, aD, r); }
    __device__ double den(bool dark, double r) const
    {
        return dark ? pl_den(MD, aD, r) : pl_den(ML, aL, r);
    }
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
__device__ double ic_integrand(const NbIcModel& m, double ri, double energy, bool dark)
{
    auto potL = [&](double r) { return pl_pot(m.ML, m.aL, r); };
    auto potD = [&](double r) { return pl_pot(m.MD, m.aD, r); };
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
__device__ double ic_gauss_quad(const NbIcModel& m, double lower, double upper, double energy,
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
__device__ double ic_root(const NbIcModel& m, double value, double lo, double hi)
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
__device__ double ic_df(const NbIcModel& m, double v, double r, bool dark)
{
    const double cons = 0.03582244801567226;
    const double energy = m.psi(r) - 0.5 * v * v;
    double range = m.MD == 0 ? 20.0 * sqrt(fabs((m.ML / energy) * (m.ML / energy) - m.aL * m.aL))
                             : 20.0 * sqrt(fabs((m.MD / energy) * (m.MD / energy) - m.aD * m.aD));
    for (int counter = 0; m.psi(range) > energy; ++counter) {
        range = 100.0 * range;
        if (counter > 100) { range = 100.0 * (m.aL + m.aD); break; }
    }
    double up = ic_root(m, energy, 0.0, range);
    if (isinf(up) || up == 0.0 || isnan(up)) up = r;        // find_upperlimit_r's fallback
    up = fabs(up);
    const double lo = 10.0 * up;
    return v * v * cons * ic_gauss_quad(m, lo, up, energy, dark);
}

// golden-section search for the DF maximum over speeds (max_finder)
__device__ double ic_df_max(const NbIcModel& m, double r, bool dark, double a, double b,
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

// One body per thread: radius and speed by rejection, isotropic directions.
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
        const NbIcModel m{d.massL, d.rsL, d.massD, d.rsD};
        NbRng rng{ic_mix(d.seed ^ ic_mix((unsigned long long) k + 0x51ED27ull))};
        const double M = dark ? d.massD : d.massL, a = dark ? d.rsD : d.rsL;
        const double bound = 50.0 * (d.rsL + d.rsD);
        const double rmax = sqrt(2.0 / 3.0) * a;
        const double rhoMax = rmax * rmax * pl_den(M, a, rmax);
        double r = 0.0;
        for (int tries = 0; tries <= 1000 && !(isfinite(r) && r != 0.0); ++tries) {
            r = 0.0;
            for (int counter = 0; counter <= 1000; ++counter) {      // r_mag
                const double rr = rng.uniform() * bound;
                const double u = rng.uniform();
                if (rr * rr * pl_den(M, a, rr) / rhoMax > u) { r = rr; break; }
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
        mass[i] = dark ? (nDark ? d.massD / (double) nDark : 0.0)
                       : (d.nBaryon ? d.massL / (double) d.nBaryon : 0.0);
        types[i] = dark ? -1 : 1;
    }
}

// Per (dwarf, component): sums of m x and m v (warp-segmented, one atomic per segment).
__global__ void k_ic_moments(const NbIcDwarf* __restrict__ dwarfs, int nD, int n,
                             const double* __restrict__ px, const double* __restrict__ py,
                             const double* __restrict__ pz, const double* __restrict__ vx,
                             const double* __restrict__ vy, const double* __restrict__ vz,
                             const double* __restrict__ mass, double* __restrict__ sums)
{
    const int lane = threadIdx.x & 31;
    const int warpsTotal = (gridDim.x * blockDim.x) >> 5;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n;
         base += warpsTotal * 32) {
        const int i = base + lane;
        const bool valid = i < n;
        int key = -1;
        double s[6] = {0, 0, 0, 0, 0, 0};
        if (valid) {
            const int dwi = ic_dwarf_of(dwarfs, nD, i);
            key = 2 * dwi + (i - dwarfs[dwi].first >= dwarfs[dwi].nBaryon);
            const double mi = mass[i];
            s[0] = mi * px[i]; s[1] = mi * py[i]; s[2] = mi * pz[i];
            s[3] = mi * vx[i]; s[4] = mi * vy[i]; s[5] = mi * vz[i];
        }
        unsigned pending = __ballot_sync(NB_FULL_MASK, valid);
        while (pending) {
            const int leader = __ffs(pending) - 1;
            const int kl = __shfl_sync(NB_FULL_MASK, key, leader);
            for (int c = 0; c < 6; ++c) {
                double v = key == kl ? s[c] : 0.0;
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(NB_FULL_MASK, v, o);
                if (lane == leader) atomicAdd(&sums[6 * (size_t) kl + c], v);
            }
            pending &= ~__ballot_sync(NB_FULL_MASK, key == kl);
        }
    }
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
        const double cm = dark ? d.massD : d.massL;
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

// Samples every dwarf of the table into the SoA body arrays (bodies [first, first + count) of
// each dwarf) and their types; scratch needs 12 doubles per dwarf.  One launch per phase for all
// dwarfs.  Returns the number of launches.
int nb_launch_ic(const NBodyCudaPlummerDwarf* host, int nD, const int* firsts, void* dTable,
                 double* scratch, NbTreeBuffers& b, int* types, int n, int numSMs, NbScalars* sc,
                 cudaStream_t s)
{
    std::vector<NbIcDwarf> t(nD);
    for (int k = 0; k < nD; ++k) {
        const NBodyCudaPlummerDwarf& h = host[k];
        NbIcDwarf& d = t[k];
        d.first = firsts[k];
        d.count = h.nbody;
        d.nBaryon = h.nbodyBaryon;
        d.massL = h.massLight; d.rsL = h.scaleLight;
        d.massD = h.massDark; d.rsD = h.scaleDark;
        for (int c = 0; c < 3; ++c) { d.pos[c] = h.position[c]; d.vel[c] = h.velocity[c]; }
        d.seed = h.seed;
    }
    cudaMemcpyAsync(dTable, t.data(), sizeof(NbIcDwarf) * nD, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(scratch, 0, sizeof(double) * 12 * (size_t) nD, s);
    const NbIcDwarf* dt = (const NbIcDwarf*) dTable;
    // few bodies per thread, many threads: the per-body work is long and uneven
    const int g = min((n + 127) / 128, numSMs * 64);
    k_ic_sample<<<g, 128, 0, s>>>(dt, nD, n, b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.mass, types, sc);
    const int g2 = min((n + 255) / 256, numSMs * 8);
    k_ic_moments<<<g2, 256, 0, s>>>(dt, nD, n, b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.mass, scratch);
    k_ic_shift<<<g2, 256, 0, s>>>(dt, nD, n, b.px, b.py, b.pz, b.vx, b.vy, b.vz, scratch);
    nb_count_launch(3);
    return 3;
}

size_t nb_ic_table_bytes(int nD) { return sizeof(NbIcDwarf) * (size_t) nD; }
