// Lambda-Beta histograms and the likelihood of every dwarf, from the device-resident bodies.
//
// nbCreateHistogram (nbody/src/nbody_histogram.c:671-1139) builds up to eight histograms over
// the same bins: the normalised counts (histogram 0), the beta and line-of-sight velocity
// dispersions (1, 2; always built) and, when the run compares them, the averages of the
// line-of-sight velocity, beta, heliocentric distance and the two proper motions (3..7).
// Each dispersion comes from the per-bin sums of the body values with IterMax passes of
// sigma clipping (nbCalcDisp, nbRemoveOutliers: nbody/src/nbody_mass.c:190-316);
// nbSystemLikelihood (nbody/src/nbody_likelihood.c:155-324) adds the EMD and cost components
// and one nbLikelihood comparison (nbody_mass.c:395-469) per enabled histogram.
//
// Layout: one thread per body computes its bin and quantities (k_hist_bodies).  A stable
// counting sort then lists the bodies of every bin in body order: one warp per chunk of bodies
// (chunks never straddle a dwarf) counts its bins (k_bin_rows), one block turns the counts into
// list offsets (k_bin_offsets), and the chunk warps place their bodies (k_bin_scatter, lanes
// of one bin ranked in lane order).  Finally one thread per (quantity, dwarf, bin) walks its
// bin's list once per pass -- the initial sums and IterMax outlier passes, each followed by
// nbCalcDisp -- adding in body order, as the reference does (k_disp_bins): the dispersions
// and averages equal the reference's bit for bit.  Counts are integers and exact.
#include "nb_common.cuh"
#include "nb_crmath.cuh"
#include "nb_emd.cuh"

#include <math.h>

namespace {

constexpr int HW = 4;   // warps per block of the chunk kernels

// nbXYZToLambdaBeta (nbody/src/nbody_coordinates.c:129-164): lambda, beta in degrees
__device__ __forceinline__ void nb_lambda_beta(const NbHistDev& h, double x, double y, double z,
                                               double& lambda, double& beta)
{
    const double tx = h.rot[0] * x + h.rot[1] * y + h.rot[2] * z;
    const double ty = h.rot[3] * x + h.rot[4] * y + h.rot[5] * z;
    double tz = h.rot[6] * x + h.rot[7] * y + h.rot[8] * z;
    const double r = sqrt(tx * tx + ty * ty + tz * tz);
    tz = -tz;
    lambda = atan2(ty, tx) * 180.0 / M_PI;               // r2d
    beta = asin(tz / r) * 180.0 / M_PI;
}

// cartesianalign (nbody/src/nbody_coordinates.c:192-224)
__device__ __forceinline__ void nb_align(const double* m, double& x, double& y, double& z)
{
    const double tx = x, ty = y, tz = z;
    x = m[0] * tx + m[1] * ty + m[2] * tz;
    y = m[3] * tx + m[4] * ty + m[5] * tz;
    z = m[6] * tx + m[7] * ty + m[8] * tz;
}

// nbVXVYVZtomuDec / nbVXVYVZtomuRA (nbody/src/nbody_coordinates.c:226-288): proper motions in
// milliarcseconds per year; cartesianToLbr_rad (:24-39), findLatUnitVec / findLongUnitVec
// (:166-190), mw_dotv and mw_length of milkyway/include/milkyway_vectors.h:106-124.
__device__ __forceinline__ void nb_proper_motion(const NbHistDev& h, double x, double y, double z,
                                                 double vx, double vy, double vz, double& mudec,
                                                 double& mura)
{
    x += h.sunGCDist;
    vx -= h.sunVel[0];
    vy -= h.sunVel[1];
    vz -= h.sunVel[2];
    nb_align(h.align, x, y, z);
    nb_align(h.align, vx, vy, vz);
    const double xp = x + 0.0;
    double l = atan2(y, xp);
    const double b = atan2(z, sqrt(xp * xp + y * y));
    if (l < 0.0) l += 2.0 * M_PI;
    const double dist = sqrt(x * x + y * y + z * z);
    // e_ra = (-sin l, cos l, 0)
    const double era_x = -sin(l), era_y = cos(l), era_z = 0;
    const double comp_ra = vz * era_z + (vy * era_y + vx * era_x);
    // e_dec from b' = d2r(90 - r2d(b))
    const double bd = b * 180.0 / M_PI;
    const double bb = (90 - bd) * M_PI / 180.0;
    const double edec_x = -cos(l) * cos(bb), edec_y = -cos(bb) * sin(l), edec_z = sin(bb);
    const double comp_dec = vz * edec_z + (vy * edec_y + vx * edec_x);
    double ra = comp_ra / dist;
    ra = ra * 180.0 / M_PI;
    ra = ra * 3600;
    mura = ra / 1000000.0;
    double dec = comp_dec / dist;
    dec = dec * 180.0 / M_PI;
    dec = dec * 3600;
    mudec = dec / 1000000.0;
}

// The body pass of nbCreateHistogram: a body of type +1 counts towards totalSimulated and
// sets massPerParticle (the last such body in body order); a body of type >= 0 is binned
// (nbXYZToLambdaBeta after x += sunGCDist, index = floor((lambda - lambdaStart) / lambdaSize),
// likewise for beta) and, in range, records its quantities: beta, calc_vLOS, calc_distance
// (nbody/src/nbody_mass.c:171-188) and the proper motions.
__global__ void k_hist_bodies(const double* __restrict__ px, const double* __restrict__ py,
                              const double* __restrict__ pz, const double* __restrict__ vx,
                              const double* __restrict__ vy, const double* __restrict__ vz,
                              const int* __restrict__ types, const int* __restrict__ bodyDwarf,
                              int n, NbHistDev h, unsigned int* __restrict__ counts,
                              unsigned int* __restrict__ inRange, unsigned int* __restrict__ nLight,
                              int* __restrict__ lastLight, int* __restrict__ binOf,
                              double* __restrict__ val)
{
    const int nBins = h.lambdaBins * h.betaBins;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int t = types[i];
        int bin = -1;
        if (t >= 0) {                                     // ignoreBody: dark matter
            const int d = bodyDwarf ? bodyDwarf[i] : 0;
            if (t == 1) {
                atomicAdd(&nLight[d], 1u);
                atomicMax(&lastLight[d], i);
            }
            const double x = px[i], y = py[i], z = pz[i];
            double lambda, beta;
            nb_lambda_beta(h, x + h.sunGCDist, y, z, lambda, beta);
            // (unsigned int) of the floor as the reference's x86-64 build converts it: through
            // a 64-bit signed integer, so a negative index wraps out of range
            const unsigned li = (unsigned) (long long) floor((lambda - h.lambdaStart) / h.lambdaSize);
            const unsigned bi = (unsigned) (long long) floor((beta - h.betaStart) / h.betaSize);
            if (li < (unsigned) h.lambdaBins && bi < (unsigned) h.betaBins) {
                bin = (int) (li * h.betaBins + bi);
                atomicAdd(&counts[(size_t) d * nBins + bin], 1u);
                atomicAdd(&inRange[d], 1u);
                if (h.nq > 0) {
                    const double xsol = x + h.sunGCDist;
                    const double mag = sqrt(xsol * xsol + y * y + z * z);
                    double mudec = 0.0, mura = 0.0;
                    bool pm = false;
                    for (int k = 0; k < h.nq; ++k) pm |= h.q[k] >= NB_Q_MUDEC;
                    if (pm) nb_proper_motion(h, x, y, z, vx[i], vy[i], vz[i], mudec, mura);
                    for (int k = 0; k < h.nq; ++k) {
                        double v;
                        switch (h.q[k]) {
                        case NB_Q_BETA: v = beta; break;
                        case NB_Q_VLOS: {
                            const double vl = xsol * vx[i] + y * vy[i] + z * vz[i];
                            v = vl / mag;
                            break;
                        }
                        case NB_Q_DIST: v = mag; break;
                        case NB_Q_MUDEC: v = mudec; break;
                        default: v = mura; break;
                        }
                        val[(size_t) k * n + i] = v;
                    }
                }
            }
        }
        binOf[i] = bin;
    }
}

// Bodies of each bin in every chunk: rows[c * B + b].  Lanes holding the same bin form a group
// (__match_any_sync); its lowest lane adds the group's size.
__global__ void __launch_bounds__(HW * 32) k_bin_rows(NbHistPlan p)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int c = blockIdx.x * HW + w;
    if (c >= p.nChunks) return;                           // the whole warp leaves together
    const int4 ch = p.chunks[c];
    int* row = p.rows + (size_t) c * p.B;
    for (int j = lane; j < p.B; j += 32) row[j] = 0;
    __syncwarp();
    for (int base = ch.x; base < ch.y; base += 32) {
        const int i = base + lane;
        const int b = i < ch.y ? p.binOf[i] : -1;
        const unsigned grp = __match_any_sync(0xffffffffu, b);
        if (b >= 0 && __ffs(grp) - 1 == lane) row[b] += __popc(grp);
        __syncwarp();
    }
}

// One block: segStart = exclusive prefix of the counts over (dwarf, bin); then, per (dwarf,
// bin), the chunk rows become the first list entry of each chunk's bodies of that bin.
__global__ void k_bin_offsets(NbHistPlan p)
{
    __shared__ int carry;
    const int DB = p.D * p.B;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < DB; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const int v = t < DB ? (int) p.counts[t] : 0;
        // block-wide inclusive scan of v (Hillis-Steele in shared memory)
        __shared__ int sc[1024];
        sc[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < blockDim.x; o <<= 1) {
            const int u = threadIdx.x >= o ? sc[threadIdx.x - o] : 0;
            __syncthreads();
            sc[threadIdx.x] += u;
            __syncthreads();
        }
        if (t < DB) p.segStart[t] = carry + sc[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += sc[threadIdx.x];
        __syncthreads();
    }
    for (int t = threadIdx.x; t < DB; t += blockDim.x) {
        const int d = t / p.B, b = t - d * p.B;
        int acc = p.segStart[t];
        for (int c = p.chunkFirst[d]; c < p.chunkFirst[d + 1]; ++c) {
            int* r = p.rows + (size_t) c * p.B + b;
            const int k = *r;
            *r = acc;
            acc += k;
        }
    }
}

// Every chunk places its binned bodies: a body goes to its bin's next list entry, lanes of one
// bin in lane order, batches in order -- so each bin's list is in body order.
__global__ void __launch_bounds__(HW * 32) k_bin_scatter(NbHistPlan p)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int c = blockIdx.x * HW + w;
    if (c >= p.nChunks) return;
    const int4 ch = p.chunks[c];
    int* row = p.rows + (size_t) c * p.B;
    const unsigned lt = (1u << lane) - 1u;
    for (int base = ch.x; base < ch.y; base += 32) {
        const int i = base + lane;
        const int b = i < ch.y ? p.binOf[i] : -1;
        const unsigned grp = __match_any_sync(0xffffffffu, b);
        int at = 0;
        if (b >= 0) at = row[b];
        __syncwarp();
        if (b >= 0) {
            p.list[at + __popc(grp & lt)] = i;
            if (__ffs(grp) - 1 == lane) row[b] = at + __popc(grp);
        }
        __syncwarp();
    }
}

// The dispersions of one (quantity, dwarf, bin) per thread: the initial sums over the bin's
// bodies, then IterMax passes of nbRemoveOutliers (nbody/src/nbody_mass.c:246-316: a body is
// kept if |bin mean - value| < cut-off x bin dispersion, mean and dispersion of the previous
// pass), each followed by nbCalcDisp (:190-244: a bin with more than 10 kept bodies gets its
// dispersion, corrected after an outlier pass, and its error; other bins keep their previous
// values).  Values are added in body order, as the reference adds them.
__global__ void k_disp_bins(NbHistPlan p)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int B = p.B, nq = p.h.nq;
    if (t >= nq * p.D * B) return;
    const int k = t / (p.D * B), r = t - k * p.D * B;
    const int first = p.segStart[r];
    const unsigned raw = p.counts[r];
    const double* val = p.val + (size_t) k * p.n;
    const double cut = p.cut[k], corr = p.corr[k];
    double sum = 0.0, sq = 0.0, rem = 0.0, var = 0.0, err = 0.0;
    for (int pass = 0; pass <= p.iterMax; ++pass) {
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (pass == 0) {
            for (unsigned j = 0; j < raw; ++j) {
                const double v = val[p.list[first + j]];
                s1 += v;
                s2 += v * v;
            }
        } else {
            const double newCount = (double) raw - rem;
            const double ave = sum / newCount;
            for (unsigned j = 0; j < raw; ++j) {
                const double v = val[p.list[first + j]];
                if (fabs(ave - v) < cut * var) {
                    s1 += v;
                    s2 += v * v;
                } else {
                    s3 += 1.0;
                }
            }
        }
        sum = s1;
        sq = s2;
        rem = s3;
        double count = (double) raw;
        count -= rem;
        if (count > 10.0) {
            const double n_new = count - 1.0;
            const double n_ratio = count / n_new;
            const double mean = sum / count;
            double dispsq = (sq / n_new) - n_ratio * (mean * mean);
            if (pass > 0) dispsq *= corr;
            var = sqrt(dispsq);
            err = sqrt((count + 1) / (count * n_new)) * var;
        }
    }
    p.sum[t] = sum;
    p.sq[t] = sq;
    p.rem[t] = rem;
    p.var[t] = var;
    p.err[t] = err;
}

// Bin b of the simulated histogram comp + 1 (1..7) of dwarf d: the dispersions (1, 2) as
// they stand after the outlier passes; the averages (3..7) as nbCreateHistogram turns them
// (nbody/src/nbody_histogram.c:995-1115): with more than 10 kept bodies the error is the
// dispersion / sqrt(kept) and the value the kept sum / kept, else error -1 and value 0.
__device__ void nb_sim_bin(const NbHistPlan& p, int comp, int d, int b, double& v, double& e)
{
    const int k = p.histSlot[comp];
    if (k < 0) {
        v = 0.0;
        e = 0.0;
        return;
    }
    const size_t g = ((size_t) k * p.D + d) * p.B + b;
    if (comp < 2) {
        v = p.var[g];
        e = p.err[g];
        return;
    }
    const int denom = (int) ((double) p.counts[(size_t) d * p.B + b] - p.rem[g]);
    if (denom > 10) {
        e = p.var[g] / sqrt((double) denom);
        v = p.sum[g] / denom;
    } else {
        e = -1;
        v = 0;
    }
}

// nbLikelihood (nbody/src/nbody_mass.c:395-469): over the data's used bins with a positive
// error, (data - sim)^2 / (data err^2 + sim err^2), or 25 (five sigma) when the simulated bin
// has no error; avgBins > 1 compares with the average of that many neighbouring simulated
// bins (an even count is reduced by one).  Returns half the sum.
__device__ double nb_compare(const NbHistPlan& p, const NbDataHistDev& dh, int comp, int d,
                             int avgBins)
{
    const unsigned nbins = (unsigned) dh.nBins;
    const double* dv = dh.compVar[comp];
    const double* de = dh.compErr[comp];
    double nsig = 0.0;
    for (unsigned i = 0; i < nbins; ++i) {
        if (!dh.useBin[i]) continue;
        double data, hist, errData, errHist;
        if (avgBins > 1) {
            if (avgBins % 2 == 0) avgBins -= 1;
            unsigned cnt = (unsigned) avgBins;
            double varSum = 0.0, valSum = 0.0;
            for (unsigned k = 0; k < (unsigned) avgBins; ++k) {
                const int index = (int) (i - (unsigned) ((avgBins - 1) / 2) + k);
                if (index < 0 || (unsigned) index >= nbins) {
                    cnt -= 1;
                    continue;
                }
                double hv, he;
                nb_sim_bin(p, comp, d, index, hv, he);
                if (he <= 0) {
                    cnt -= 1;
                } else {
                    varSum += he * he;
                    valSum += hv;
                }
            }
            errHist = sqrt(varSum) / cnt;
            errData = de[i];
            hist = valSum / cnt;
            data = dv[i];
        } else {
            double hv, he;
            nb_sim_bin(p, comp, d, (int) i, hv, he);
            errData = de[i];
            errHist = he;
            data = dv[i];
            hist = hv;
        }
        if (errData > 0) {
            if (errHist > 0)
                nsig += (data - hist) * (data - hist) / (errData * errData + errHist * errHist);
            else
                nsig += 25;
        }
    }
    return nsig / 2.0;
}

// ---- the two-dimensional EMD (betaBins > 1): nb_emd.cuh run by one block per problem ----
constexpr int EMD_THREADS = 256;

// The block as an EMD team: first minimum in (value, index) order and maximum over its
// threads, by warp shuffles and one shared slot per warp.
struct NbEmdBlock {
    NbEmdMin* partM;            // shared, one per warp
    double* partD;
    NbEmdMin* resM;             // shared result
    double* resD;
    __device__ int rank() const { return (int) threadIdx.x; }
    __device__ int size() const { return (int) blockDim.x; }
    __device__ void sync() const { __syncthreads(); }
    __device__ NbEmdMin argmin(NbEmdMin a) const
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int o = 16; o > 0; o >>= 1) {
            NbEmdMin b;
            b.val = __shfl_xor_sync(NB_FULL_MASK, a.val, o);
            b.idx = __shfl_xor_sync(NB_FULL_MASK, a.idx, o);
            if (nb_emd_before(b, a)) a = b;
        }
        if (lane == 0) partM[warp] = a;
        __syncthreads();
        if (warp == 0) {
            a = lane < (int) (blockDim.x >> 5) ? partM[lane] : NbEmdMin{NB_EMD_INF, -1};
            for (int o = 16; o > 0; o >>= 1) {
                NbEmdMin b;
                b.val = __shfl_xor_sync(NB_FULL_MASK, a.val, o);
                b.idx = __shfl_xor_sync(NB_FULL_MASK, a.idx, o);
                if (nb_emd_before(b, a)) a = b;
            }
            if (lane == 0) *resM = a;
        }
        __syncthreads();
        return *resM;
    }
    __device__ double maxv(double a) const
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(NB_FULL_MASK, a, o));
        if (lane == 0) partD[warp] = a;
        __syncthreads();
        if (warp == 0) {
            a = lane < (int) (blockDim.x >> 5) ? partD[lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_xor_sync(NB_FULL_MASK, a, o));
            if (lane == 0) *resD = a;
        }
        __syncthreads();
        return *resD;
    }
};

#define NB_EMD_BLOCK_SHARED                                                                  \
    __shared__ NbEmdScalars sc;                                                              \
    __shared__ NbEmdMin partM[EMD_THREADS / 32], resM;                                       \
    __shared__ double partD[EMD_THREADS / 32], resD;                                         \
    const NbEmdBlock team{partM, partD, &resM, &resD}

__global__ void __launch_bounds__(EMD_THREADS)
k_emd_direct(const double* __restrict__ sig1, int n1, const double* __restrict__ sig2, int n2,
             char* __restrict__ work, double* __restrict__ out)
{
    NB_EMD_BLOCK_SHARED;
    const NbEmdWork w = nb_emd_carve(work, n1, n2);
    const double e = nb_emd_calc(team, sig1, n1, sig2, n2, w, sc);
    if (threadIdx.x == 0) *out = e;
}

// nbMatchEMD's emdCalc calls (nbody/src/nbody_emd.c:1332-1402) for two-dimensional histograms,
// one block per (dwarf, lambda range): the data side -- the used bins whose data-file lambda
// lies in the range, weight variable n / (the range's rounded counts), at the file's centres
// -- and the simulated side -- the used bins whose own centre lies in the range, weight
// (count / n_sim) n_sim / (its rounded counts), at the centres (i + 1/2) size + start --
// as the reference builds them; the reference passes the data side's bin count for both
// sides, and so does this (simulated bins beyond their own count weigh nothing).
__global__ void __launch_bounds__(EMD_THREADS)
k_emd_ranges(NbHistPlan p, NbDataHistDev dh)
{
    NB_EMD_BLOCK_SHARED;
    __shared__ int nData;
    const int nProb = dh.nRange > 0 ? dh.nRange / 2 : 1;
    const int d = blockIdx.x / nProb, r = blockIdx.x % nProb;
    const int nb = dh.nBins;
    char* base = dh.emdWork + (size_t) blockIdx.x * dh.emdWorkBytes;
    double* sigData = (double*) base;
    double* sigSim = (double*) (base + nb_emd_align(8 * 3 * (size_t) nb));
    char* work = base + 2 * nb_emd_align(8 * 3 * (size_t) nb);
    const unsigned* c = p.counts + (size_t) d * nb;
    const unsigned nSimU = p.inRange[d];
    const unsigned nDataU = dh.totalNum;
    if (threadIdx.x == 0) {
        const bool every = dh.nRange == 0;
        const double lo = every ? 0.0 : dh.emdRange[2 * r];
        const double hi = every ? 0.0 : dh.emdRange[2 * r + 1];
        unsigned simRange = 0, dataRange = 0;
        for (int j = 0; j < nb; ++j) {
            if (!dh.useBin[j]) continue;
            const double simL = ((double) (j / p.h.betaBins) + 0.5) * p.h.lambdaSize + p.h.lambdaStart;
            if (every || (simL >= lo && simL <= hi))
                simRange += (unsigned) round(((double) c[j] / (double) nSimU) * (double) nSimU);
            if (every || (dh.lambda[j] >= lo && dh.lambda[j] <= hi))
                dataRange += (unsigned) round(dh.variable[j] * (double) nDataU);
        }
        int ns = 0, ndat = 0;
        for (int j = 0; j < nb; ++j) {
            if (!dh.useBin[j]) continue;
            const double simL = ((double) (j / p.h.betaBins) + 0.5) * p.h.lambdaSize + p.h.lambdaStart;
            if (every || (simL >= lo && simL <= hi)) {
                const double var = (double) c[j] / (double) nSimU;
                sigSim[3 * ns] = var * (double) nSimU / (1.0 * simRange);
                sigSim[3 * ns + 1] = simL;
                sigSim[3 * ns + 2] = ((double) (j % p.h.betaBins) + 0.5) * p.h.betaSize + p.h.betaStart;
                ++ns;
            }
            if (every || (dh.lambda[j] >= lo && dh.lambda[j] <= hi)) {
                sigData[3 * ndat] = dh.variable[j] * (double) nDataU / (1.0 * dataRange);
                sigData[3 * ndat + 1] = dh.lambda[j];
                sigData[3 * ndat + 2] = dh.beta[j];
                ++ndat;
            }
        }
        for (int k = ns; k < ndat; ++k) sigSim[3 * k] = sigSim[3 * k + 1] = sigSim[3 * k + 2] = 0.0;
        nData = ndat;
    }
    __syncthreads();
    const int n = nData;
    const NbEmdWork w = nb_emd_carve(work, n, n);
    const double e = nb_emd_calc(team, sigData, n, sigSim, n, w, sc);
    if (threadIdx.x == 0) dh.emd2d[blockIdx.x] = e;
}

// nbSystemLikelihood (nbody/src/nbody_likelihood.c:155-324), one thread per dwarf.  The EMD
// per lambda range (nbMatchEMD, nbody/src/nbody_emd.c:1278-1427): with one beta bin the two
// weight sets lie on the lambda axis and the reference's emdCalc with the L2 ground distance
// is the 1-D transport cost sum_k |F_sim(k) - F_data(k)| (lambda_{k+1} - lambda_k) over the
// used bins; with more beta bins each range's emdCalc comes from k_emd_ranges (the
// transportation simplex of nb_emd.cuh); nbCostComponent (nbody_mass.c:318-391);
// then the enabled comparisons in the reference's order.
// out[NB_LIKELIHOOD_TERMS d ..]: likelihood, EMD component, cost component, beta dispersion,
// velocity dispersion, beta average, line-of-sight velocity, distance, dec and RA proper
// motion (NaN where not compared), and the EMD itself.
__global__ void k_likelihood(NbHistPlan p, const double* __restrict__ mass,
                             const int* __restrict__ nbodyOf, NbDataHistDev dh, NbLikeFlags f,
                             double* __restrict__ out)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= p.D) return;
    const int nb = dh.nBins;
    const unsigned* c = p.counts + (size_t) d * nb;
    const unsigned nSimU = p.inRange[d];                // histogram->totalNum
    const double histMass = p.lastLight[d] >= 0 ? mass[p.lastLight[d]] : 0.0;
    const double n = (double) p.nLight[d];              // totalSimulated
    double* o = out + (size_t) NB_LIKELIHOOD_TERMS * d;
    for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t) o[t] = NAN;
    const double worst = 9999999.9;                     // DEFAULT_WORST_CASE
    // too few bodies in range (nbody_likelihood.c:198-227)
    if ((double) nSimU < 0.0001 * (double) nbodyOf[d]) {
        o[0] = worst;
        o[1] = worst;
        for (int t = 2; t < 10; ++t) o[t] = 0.0;
        o[10] = worst;
        return;
    }
    const unsigned nData = dh.totalNum;
    double emdComp;
    double emd = 0.0;
    if (nSimU == 0 || nData == 0) {
        emdComp = INFINITY;
    } else if (histMass <= 0.0 || dh.massPerParticle <= 0.0) {
        emdComp = NAN;
    } else if (dh.nRange % 2 != 0) {
        emdComp = NAN;                                  // an odd number of range bounds
    } else {
        // per lambda range (one over every bin by default): the used bins whose centres lie in
        // it -- the simulated histogram's centres (i + 0.5) lambdaSize + lambdaStart, the data
        // file's own -- each side renormalised to the range, the range's EMD weighted by its
        // share of the data counts
        // (without ranges every used bin counts: the file's default range reaches half a bin
        // beyond the outer centres)
        const bool every = dh.nRange == 0;
        const int nR = every ? 2 : dh.nRange;
        double emdSum = 0.0;
        unsigned totalRange = 0;
        bool bad = false;
        for (int r = 0; r < nR && !bad; r += 2) {
            const double lo = every ? 0.0 : dh.emdRange[r];
            const double hi = every ? 0.0 : dh.emdRange[r + 1];
            if (lo > hi) { bad = true; break; }
            unsigned simRange = 0, dataRange = 0;
            for (int j = 0; j < nb; ++j) {
                if (!dh.useBin[j]) continue;
                const double simL = ((double) (j / p.h.betaBins) + 0.5) * p.h.lambdaSize + p.h.lambdaStart;
                if (every || (simL >= lo && simL <= hi))
                    simRange += (unsigned) round(((double) c[j] / (double) nSimU) * (double) nSimU);
                if (every || (dh.lambda[j] >= lo && dh.lambda[j] <= hi))
                    dataRange += (unsigned) round(dh.variable[j] * (double) nData);
            }
            double Fs = 0.0, Fd = 0.0, cost = 0.0, prevL = 0.0;
            bool first = true;
            if (p.h.betaBins > 1) {
                // the range's emdCalc, solved by k_emd_ranges
                cost = dh.emd2d[(size_t) d * (nR / 2) + r / 2];
            } else {
                for (int j = 0; j < nb; ++j) {
                    if (!dh.useBin[j] || !(every || (dh.lambda[j] >= lo && dh.lambda[j] <= hi))) continue;
                    if (!first) cost += fabs(Fs - Fd) * (dh.lambda[j] - prevL);
                    const double var = (double) c[j] / (double) nSimU;
                    Fs += var * (double) nSimU / (1.0 * simRange);
                    Fd += dh.variable[j] * (double) nData / (1.0 * dataRange);
                    prevL = dh.lambda[j];
                    first = false;
                }
            }
            totalRange += dataRange;
            emdSum += cost * ((double) dataRange / (1.0 * nData));
        }
        if (bad || totalRange == 0) {
            emdComp = NAN;
        } else {
            emd = emdSum * (double) (nData / totalRange);   // integer division, as the reference
            emd = round(emd * 1.0e9) * 1.0e-9;
            emdComp = emd > 50.0 ? NAN : -(300.0 * nb_log_rn(1.0 - emd / 50.0));   // mw_log
        }
    }
    double costComp;
    if (nSimU == 0 || nData == 0) {
        costComp = INFINITY;
    } else if (histMass <= 0.0 || dh.massPerParticle <= 0.0) {
        costComp = NAN;
    } else {
        double nSim = (double) nSimU, nDataVar = 0.0;
        const double nDataD = (double) nData;
        for (int j = 0; j < nb; ++j) {
            if (!dh.useBin[j]) nSim -= round(((double) c[j] / (double) nSimU) * (double) nSimU);
            else nDataVar += (dh.err[j] * nDataD) * (dh.err[j] * nDataD);
        }
        const double pr = nSim / n;
        const double dm = dh.massPerParticle * nDataD - histMass * nSim;
        const double num = -(dm * dm);
        const double denom = 2.0 * ((dh.massPerParticle * dh.massPerParticle) * nDataVar +
                                    (histMass * histMass) * nSim * pr * (1.0 - pr));
        costComp = -(num / denom);
    }
    double like = emdComp + costComp;
    double terms[7];
    for (int t = 0; t < 7; ++t) terms[t] = NAN;
    if (f.betaDisp) {
        terms[0] = nb_compare(p, dh, 0, d, dh.betaDispBins);
        like += terms[0];
    }
    if (f.velDisp) {
        terms[1] = nb_compare(p, dh, 1, d, 1);
        like += terms[1];
    }
    bool missing = false;
    if (f.vlos) {
        if (!dh.compVar[2] || p.histSlot[2] < 0) missing = true;
        else like += (terms[3] = nb_compare(p, dh, 2, d, 1));
    }
    if (!missing && f.betaComp) {
        if (!dh.compVar[3] || p.histSlot[3] < 0) missing = true;
        else like += (terms[2] = nb_compare(p, dh, 3, d, 1));
    }
    if (!missing && f.dist) {
        if (!dh.compVar[4] || p.histSlot[4] < 0) missing = true;
        else like += (terms[4] = nb_compare(p, dh, 4, d, 1));
    }
    if (!missing && f.propMot) {
        if (!dh.compVar[5] || p.histSlot[5] < 0) {
            missing = true;
        } else {
            like += (terms[5] = nb_compare(p, dh, 5, d, 1));
            if (!dh.compVar[6] || p.histSlot[6] < 0) missing = true;
            else like += (terms[6] = nb_compare(p, dh, 6, d, 1));
        }
    }
    o[10] = emd;
    if (missing) return;                                // the reference's NaN array
    o[0] = like;
    o[1] = emdComp;
    o[2] = costComp;
    for (int t = 0; t < 7; ++t) o[3 + t] = terms[t];
}

// Histograms 1..7 of every dwarf: comps[((d * 7 + h) * 2 + {0: value, 1: error}) * B + b].
__global__ void k_hist_export(NbHistPlan p, double* __restrict__ comps)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int B = p.B;
    if (t >= p.D * NB_HIST_COMPONENTS * B) return;
    const int b = t % B, h = (t / B) % NB_HIST_COMPONENTS, d = t / (B * NB_HIST_COMPONENTS);
    double v, e;
    nb_sim_bin(p, h, d, b, v, e);
    double* o = comps + ((size_t) (d * NB_HIST_COMPONENTS + h) * 2) * B;
    o[b] = v;
    o[B + b] = e;
}

// get_likelihood (nbody/src/nbody_plain.c:100-237), one thread per dwarf: the likelihood is
// clamped (NaN or beyond the worst case: the worst case; 0: the best case) and kept when its
// magnitude is below the best's; terms of comparisons not made are kept as 0.
__global__ void k_best_update(const double* __restrict__ out, NbBestDev* __restrict__ best, int D,
                              int step, int nStep, NbLikeFlags f)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= D) return;
    const double* o = out + (size_t) NB_LIKELIHOOD_TERMS * d;
    NbBestDev& b = best[d];
    const double worst = 9999999.9, bestCase = 1e-9;  // DEFAULT_WORST_CASE, DEFAULT_BEST_CASE
    double like = o[0];
    if (like > worst || like < -1 * worst || isnan(like)) like = worst;
    else if (like == 0.0) like = bestCase;
    b.improved = 0;
    if (fabs(like) < fabs(b.best[0])) {
        b.best[0] = like;
        b.best[1] = o[1];
        b.best[2] = o[2];
        b.best[3] = f.betaDisp ? o[3] : 0.0;
        b.best[4] = f.velDisp ? o[4] : 0.0;
        b.best[5] = f.betaComp ? o[5] : 0.0;
        b.best[6] = f.vlos ? o[6] : 0.0;
        b.best[7] = f.dist ? o[7] : 0.0;
        b.best[8] = f.propMot ? o[8] : 0.0;
        b.best[9] = f.propMot ? o[9] : 0.0;
        b.best[10] = o[10];
        b.bestTime = ((double) step / (double) nStep) * b.timeEvolve;
        b.bestStep = step;
        b.count += 1;
        b.improved = 1;
    }
}

// The bodies of every dwarf whose likelihood just improved (bestLikelihoodBodyTab).
__global__ void k_keep_best(const NbBestDev* __restrict__ best, const int* __restrict__ bodyDwarf,
                            const double* __restrict__ px, const double* __restrict__ py,
                            const double* __restrict__ pz, const double* __restrict__ vx,
                            const double* __restrict__ vy, const double* __restrict__ vz, int n,
                            double* __restrict__ keepPos, double* __restrict__ keepVel)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int d = bodyDwarf ? bodyDwarf[i] : 0;
        if (!best[d].improved) continue;
        keepPos[3 * (size_t) i + 0] = px[i];
        keepPos[3 * (size_t) i + 1] = py[i];
        keepPos[3 * (size_t) i + 2] = pz[i];
        keepVel[3 * (size_t) i + 0] = vx[i];
        keepVel[3 * (size_t) i + 1] = vy[i];
        keepVel[3 * (size_t) i + 2] = vz[i];
    }
}

}  // namespace

void nb_launch_best_update(const double* out, NbBestDev* best, int D, int step, int nStep,
                           NbLikeFlags f, cudaStream_t s)
{
    k_best_update<<<(D + 127) / 128, 128, 0, s>>>(out, best, D, step, nStep, f);
    nb_count_launch();
}

void nb_launch_keep_best(const NbBestDev* best, const int* bodyDwarf, const double* px,
                         const double* py, const double* pz, const double* vx, const double* vy,
                         const double* vz, int n, double* keepPos, double* keepVel, int numSMs,
                         cudaStream_t s)
{
    int g = (n + 255) / 256;
    if (g > numSMs * 8) g = numSMs * 8;
    if (g < 1) g = 1;
    k_keep_best<<<g, 256, 0, s>>>(best, bodyDwarf, px, py, pz, vx, vy, vz, n, keepPos, keepVel);
    nb_count_launch();
}

static inline int nb_l_grid(int n, int threads, int cap)
{
    int g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    return g < cap ? g : cap;
}

// Bodies per chunk: 1024, more when the chunk rows (B ints each) would exceed 64 MB.
size_t nb_hist_chunk_bodies(int n, int nq, int B)
{
    (void) nq;
    const double rowBytes = 4.0 * (double) B;
    size_t ch = 1024;
    const double limit = 64.0 * 1024.0 * 1024.0;
    while ((double) n / (double) ch * rowBytes > limit) ch *= 2;
    return ch;
}

// Counts, totals and per-body quantities, then (with quantities to bin) the per-bin lists and
// the dispersions with their iterMax outlier passes.  Returns the number of kernel launches.
int nb_launch_hist_plan(const NbHistPlan& p, const double* px, const double* py, const double* pz,
                        const double* vx, const double* vy, const double* vz, const int* types,
                        const int* bodyDwarf, int numSMs, cudaStream_t s)
{
    const size_t DB = (size_t) p.D * p.B;
    cudaMemsetAsync(p.counts, 0, sizeof(unsigned) * DB, s);
    cudaMemsetAsync(p.inRange, 0, sizeof(unsigned) * p.D, s);
    cudaMemsetAsync(p.nLight, 0, sizeof(unsigned) * p.D, s);
    cudaMemsetAsync(p.lastLight, 0xff, sizeof(int) * p.D, s);    // -1
    int launches = 0;
    if (p.n > 0) {
        k_hist_bodies<<<nb_l_grid(p.n, 256, numSMs * 8), 256, 0, s>>>(
            px, py, pz, vx, vy, vz, types, bodyDwarf, p.n, p.h, p.counts, p.inRange, p.nLight,
            p.lastLight, p.binOf, p.val);
        ++launches;
    }
    if (p.h.nq > 0 && p.n > 0) {
        const int chunkBlocks = (p.nChunks + HW - 1) / HW;
        const size_t Q = (size_t) p.h.nq * DB;
        k_bin_rows<<<chunkBlocks, HW * 32, 0, s>>>(p);
        k_bin_offsets<<<1, 1024, 0, s>>>(p);
        k_bin_scatter<<<chunkBlocks, HW * 32, 0, s>>>(p);
        k_disp_bins<<<(int) ((Q + 127) / 128), 128, 0, s>>>(p);
        launches += 4;
    }
    nb_count_launch(launches);
    return launches;
}

int nb_emd_ranges(const NbDataHistDev& dh) { return dh.nRange > 0 ? dh.nRange / 2 : 1; }

size_t nb_emd_problem_bytes(int nBins)
{
    return 2 * nb_emd_align(8 * 3 * (size_t) nBins) + nb_emd_work_bytes(nBins, nBins);
}

void nb_launch_emd_ranges(const NbHistPlan& p, const NbDataHistDev& dh, cudaStream_t s)
{
    k_emd_ranges<<<p.D * nb_emd_ranges(dh), EMD_THREADS, 0, s>>>(p, dh);
    nb_count_launch();
}

void nb_launch_emd_direct(const double* sig1, int n1, const double* sig2, int n2, char* work,
                          double* out, cudaStream_t s)
{
    k_emd_direct<<<1, EMD_THREADS, 0, s>>>(sig1, n1, sig2, n2, work, out);
    nb_count_launch();
}

void nb_launch_likelihood(const NbHistPlan& p, const double* mass, const int* nbodyOf,
                          const NbDataHistDev& dh, NbLikeFlags f, double* out, cudaStream_t s)
{
    if (p.h.betaBins > 1) nb_launch_emd_ranges(p, dh, s);
    k_likelihood<<<(p.D + 127) / 128, 128, 0, s>>>(p, mass, nbodyOf, dh, f, out);
    nb_count_launch();
}

void nb_launch_hist_export(const NbHistPlan& p, double* comps, cudaStream_t s)
{
    const int total = p.D * NB_HIST_COMPONENTS * p.B;
    k_hist_export<<<(total + 127) / 128, 128, 0, s>>>(p, comps);
    nb_count_launch();
}
