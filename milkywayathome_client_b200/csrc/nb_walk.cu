// Force evaluation: FP64 Barnes-Hut walk, FP64 direct summation and the external Milky Way
// potential.  Compiled with -fmad=false so every expression keeps the reference's rounding
// (the reference CPU build uses SSE2 without FMA, milkyway/include/milkyway_math_double.h:128).
//
// Walk (nbGravity, nbody/src/nbody_grav.c:42-124).  One warp walks for 32 bodies that are
// consecutive in octree-path order.  Every lane keeps its own position in the reference's
// stackless walk: at node q it accepts (interacts, then jumps to Next(q)) if q is a body or
// |dr|^2 >= rcrit2(q), otherwise it opens q (goes to More(q) = q + 1 in walk order).  Two
// forms: the warp-union walk (k_walk_fp64) visits the smallest pending node of its lanes, each
// node record read once per warp visit (uniform address); the per-lane walk
// (k_walk_fp64_lanes) lets each lane take its own next node every iteration.  Either way each
// lane sees exactly the nodes of its own CPU walk, in the CPU's order, and accumulates the same
// terms in the same order.  A monopole interaction is 18 flops + sqrt + 2 divisions, a
// quadrupole cell adds 38 flops + 2 divisions: the FP64 pipe (and, per lane, the L1 data pipe
// that gathers the records) bounds the walk.
#include "nb_common.cuh"
#include "nb_potential.cuh"

constexpr int WALK_THREADS = 128;

// FOREST: the nodes hold one tree per dwarf (batched dwarfs); each lane walks its own
// dwarf's tree, [rootNode, rootEnd), with that dwarf's softening and time step.  A warp whose
// 32 bodies straddle two dwarfs visits the union of both walks, each lane its own.
// The walk reads one packed record per node (k_pack_walk): 96 bytes, three double4 --
// {CoM, mass}, {rcrit2, Next and body index as one 64-bit word, Qxx, Qxy},
// {Qxz, Qyy, Qyz, Qzz} -- so a visit touches one record instead of four arrays.
__global__ void k_pack_walk(const double4* __restrict__ nodePM, const double* __restrict__ nodeCrit,
                            const int2* __restrict__ nodeLink, const double* __restrict__ nodeQuad,
                            double4* __restrict__ rec, const NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int nNodes = sc->nNodes;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nNodes; k += gridDim.x * blockDim.x) {
        const int2 l = nodeLink[k];
        const long long word = (long long) (unsigned) l.x | ((long long) l.y << 32);
        const double* Q = nodeQuad + 6 * (size_t) k;
        const bool body = l.y >= 0;
        rec[3 * (size_t) k] = nodePM[k];
        rec[3 * (size_t) k + 1] = make_double4(nodeCrit[k], __longlong_as_double(word),
                                               body ? 0.0 : Q[0], body ? 0.0 : Q[1]);
        rec[3 * (size_t) k + 2] = body ? make_double4(0.0, 0.0, 0.0, 0.0)
                                       : make_double4(Q[2], Q[3], Q[4], Q[5]);
    }
}

template <bool COUNT, bool FOREST>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_fp64(const double4* __restrict__ rec,
            const unsigned int* __restrict__ order, const double* __restrict__ px,
            const double* __restrict__ py, const double* __restrict__ pz,
            double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
            double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
            NbWalkParams wp, NbPot pot, NbScalars* __restrict__ sc, NbForest forest)
{
    if (nb_failed(sc)) return;
    const int end = sc->nNodes;
    const int lane = threadIdx.x & 31;
    const int i = (int) ((blockIdx.x * (unsigned) blockDim.x + threadIdx.x) >> 5) * 32 + lane;
    const bool valid = i < wp.n;
    const unsigned j = valid ? order[i] : 0u;
    const double x0 = valid ? px[j] : 0.0, y0 = valid ? py[j] : 0.0, z0 = valid ? pz[j] : 0.0;
    double eps2 = wp.eps2;
    const bool useQuad = wp.useQuad != 0;
    int start = 0, myEnd = end;
    NbDwarfDev* dw = nullptr;
    if (FOREST && valid) {
        dw = &forest.dwarfs[forest.bodyDwarf[i]];
        eps2 = dw->eps2;
        wp.dtHalf = 0.5 * dw->dt;
        start = dw->rootNode;
        myEnd = dw->rootEnd;
    }
    int ptr = valid ? start : end;
    double accx = 0.0, accy = 0.0, accz = 0.0;
    bool metSelf = false;
    unsigned long long cVisit = 0, cBB = 0, cBC = 0, cSteps = 0;
    for (;;) {
        if (FOREST && ptr >= myEnd) ptr = end;          // this lane's tree is done
        const int q = __reduce_min_sync(NB_FULL_MASK, ptr);
        if (q >= end) break;
        if (COUNT) ++cSteps;
        if (ptr != q) continue;
        const double4 nd = nb_ld32(rec + 3 * (size_t) q);
        const double4 r1 = nb_ld32(rec + 3 * (size_t) q + 1);
        const long long word = __double_as_longlong(r1.y);
        const int2 link = make_int2((int) (unsigned) (word & 0xffffffffll), (int) (word >> 32));
        const double dx = nd.x - x0, dy = nd.y - y0, dz = nd.z - z0;
        double drSq = dz * dz + (dy * dy + dx * dx);
        const bool isBody = link.y >= 0;
        if (COUNT) ++cVisit;
        if (isBody || drSq >= r1.x) {
            ptr = link.x;
            if (isBody && (unsigned) link.y == j) { metSelf = true; continue; }
            if (COUNT) { if (isBody) ++cBB; else ++cBC; }
            drSq = drSq + eps2;
            const double drab = sqrt(drSq);
            const double phii = nd.w / drab;
            const double mor3 = phii / drSq;
            accx = accx + mor3 * dx;
            accy = accy + mor3 * dy;
            accz = accz + mor3 * dz;
            if (useQuad && !isBody) {
                const double4 r2 = nb_ld32(rec + 3 * (size_t) q + 2);
                const double qxx = r1.z, qxy = r1.w, qxz = r2.x, qyy = r2.y, qyz = r2.z, qzz = r2.w;
                const double qdx = qxx * dx + qxy * dy + qxz * dz;
                const double qdy = qxy * dx + qyy * dy + qyz * dz;
                const double qdz = qxz * dx + qyz * dy + qzz * dz;
                const double drQdr = qdx * dx + qdy * dy + qdz * dz;
                const double dr5inv = 1.0 / ((drSq * drSq) * drab);
                const double phiQ = 2.5 * (dr5inv * drQdr) / drSq;
                accx = accx + phiQ * dx;
                accy = accy + phiQ * dy;
                accz = accz + phiQ * dz;
                accx = accx - dr5inv * qdx;
                accy = accy - dr5inv * qdy;
                accz = accz - dr5inv * qdz;
            }
        } else {
            ptr = q + 1;
        }
    }
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) {
            cVisit += __shfl_xor_sync(NB_FULL_MASK, cVisit, o);
            cBB += __shfl_xor_sync(NB_FULL_MASK, cBB, o);
            cBC += __shfl_xor_sync(NB_FULL_MASK, cBC, o);
        }
        if (lane == 0) {
            atomicAdd(&sc->nWarpSteps, cSteps);
            atomicAdd(&sc->nVisit, cVisit);
            atomicAdd(&sc->nBodyBody, cBB);
            atomicAdd(&sc->nBodyCell, cBC);
        }
    }
    if (!valid) return;
    // a body that never meets itself is tree incest (nbody/src/nbody_grav.c:111-118)
    if (!metSelf) {
        atomicOr(&sc->incest, 1);
        if (FOREST) atomicOr(&dw->status, NBODY_TREE_INCEST_NONFATAL);
    }
    // self-gravity only; k_body_epilogue adds the external potential and kicks (kept out of
    // this kernel so that its registers serve the walk)
    ax[j] = accx; ay[j] = accy; az[j] = accz;
}

// The same walk with every lane on its own path (no warp union): each iteration every lane
// that has not finished takes the next node of its own walk (a per-lane gather of the node
// record, one 32-byte load per sector, instead of one broadcast), so a lane is idle only when
// its walk is over.  Each lane still meets exactly its CPU walk's nodes in the CPU's order and
// sums the same terms in the same order.  Bodies consecutive in path order have walks of
// similar length, so the warp runs about as many iterations as its longest walk, while the
// union walk runs one iteration per node any of its lanes visits: on the 131k-body dwarf at
// theta 0.5, 0.96 of the lane slots do work against 0.70 in the union walk (a CPU count over
// the oracle's tree).  Walks in groups of 2 to 16 lanes (the union of each group's paths) were
// measured between the two and slower than both.
template <bool COUNT, bool FOREST, bool PREFETCH>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_fp64_lanes(const double4* __restrict__ rec,
                  const unsigned int* __restrict__ order, const double* __restrict__ px,
                  const double* __restrict__ py, const double* __restrict__ pz,
                  double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
                  NbWalkParams wp, NbScalars* __restrict__ sc, NbForest forest)
{
    if (nb_failed(sc)) return;
    const int end = sc->nNodes;
    const int lane = threadIdx.x & 31;
    const int i = (int) ((blockIdx.x * (unsigned) blockDim.x + threadIdx.x) >> 5) * 32 + lane;
    const bool valid = i < wp.n;
    const unsigned j = valid ? order[i] : 0u;
    const double x0 = valid ? px[j] : 0.0, y0 = valid ? py[j] : 0.0, z0 = valid ? pz[j] : 0.0;
    double eps2 = wp.eps2;
    const bool useQuad = wp.useQuad != 0;
    int myEnd = end;
    int ptr = 0;
    NbDwarfDev* dw = nullptr;
    if (FOREST && valid) {
        dw = &forest.dwarfs[forest.bodyDwarf[i]];
        eps2 = dw->eps2;
        ptr = dw->rootNode;
        myEnd = dw->rootEnd;
    }
    if (!valid) ptr = myEnd;
    double accx = 0.0, accy = 0.0, accz = 0.0;
    bool metSelf = false;
    unsigned long long cVisit = 0, cBB = 0, cBC = 0, cSteps = 0;
    // PREFETCH: the next node's record is loaded as soon as the opening test has chosen it,
    // before this node's terms are computed, so its latency overlaps the FP64 arithmetic (72
    // registers against 56: it pays where few warps are resident, tens of thousands of bodies,
    // and costs at a million, where other warps already hide the latency)
    double4 nd = make_double4(0.0, 0.0, 0.0, 0.0), r1 = nd;
    if (PREFETCH && ptr < myEnd) {
        nd = nb_ld32(rec + 3 * (size_t) ptr);
        r1 = nb_ld32(rec + 3 * (size_t) ptr + 1);
    }
    for (;;) {
        // every lane takes part in the vote of every iteration (a finished lane idles in the
        // loop), and the warp leaves the loop together when all its walks are over
        const bool active = ptr < myEnd;
        if (!__any_sync(NB_FULL_MASK, active)) break;
        if (COUNT) ++cSteps;
        if (!active) continue;
        const int q = ptr;
        if (!PREFETCH) {
            nd = nb_ld32(rec + 3 * (size_t) q);
            r1 = nb_ld32(rec + 3 * (size_t) q + 1);
        }
        const long long word = __double_as_longlong(r1.y);
        const int2 link = make_int2((int) (unsigned) (word & 0xffffffffll), (int) (word >> 32));
        const double dx = nd.x - x0, dy = nd.y - y0, dz = nd.z - z0;
        double drSq = dz * dz + (dy * dy + dx * dx);
        const bool isBody = link.y >= 0;
        if (COUNT) ++cVisit;
        const bool accept = isBody || drSq >= r1.x;
        ptr = accept ? link.x : q + 1;
        double4 ndNext = nd, r1Next = r1;
        if (PREFETCH && ptr < myEnd) {
            ndNext = nb_ld32(rec + 3 * (size_t) ptr);
            r1Next = nb_ld32(rec + 3 * (size_t) ptr + 1);
        }
        if (accept && isBody && (unsigned) link.y == j) metSelf = true;
        else if (accept) {
            if (COUNT) { if (isBody) ++cBB; else ++cBC; }
            drSq = drSq + eps2;
            const double drab = sqrt(drSq);
            const double phii = nd.w / drab;
            const double mor3 = phii / drSq;
            accx = accx + mor3 * dx;
            accy = accy + mor3 * dy;
            accz = accz + mor3 * dz;
            if (useQuad && !isBody) {
                const double4 r2 = nb_ld32(rec + 3 * (size_t) q + 2);
                const double qxx = r1.z, qxy = r1.w, qxz = r2.x, qyy = r2.y, qyz = r2.z, qzz = r2.w;
                const double qdx = qxx * dx + qxy * dy + qxz * dz;
                const double qdy = qxy * dx + qyy * dy + qyz * dz;
                const double qdz = qxz * dx + qyz * dy + qzz * dz;
                const double drQdr = qdx * dx + qdy * dy + qdz * dz;
                const double dr5inv = 1.0 / ((drSq * drSq) * drab);
                const double phiQ = 2.5 * (dr5inv * drQdr) / drSq;
                accx = accx + phiQ * dx;
                accy = accy + phiQ * dy;
                accz = accz + phiQ * dz;
                accx = accx - dr5inv * qdx;
                accy = accy - dr5inv * qdy;
                accz = accz - dr5inv * qdz;
            }
        }
        if (PREFETCH) { nd = ndNext; r1 = r1Next; }
    }
    if (COUNT) {
        // every lane counted the warp's iterations alike
        for (int o = 16; o > 0; o >>= 1) {
            cVisit += __shfl_xor_sync(NB_FULL_MASK, cVisit, o);
            cBB += __shfl_xor_sync(NB_FULL_MASK, cBB, o);
            cBC += __shfl_xor_sync(NB_FULL_MASK, cBC, o);
        }
        if (lane == 0) {
            atomicAdd(&sc->nWarpSteps, cSteps);
            atomicAdd(&sc->nVisit, cVisit);
            atomicAdd(&sc->nBodyBody, cBB);
            atomicAdd(&sc->nBodyCell, cBC);
        }
    }
    if (!valid) return;
    // a body that never meets itself is tree incest (nbody/src/nbody_grav.c:111-118)
    if (!metSelf) {
        atomicOr(&sc->incest, 1);
        if (FOREST) atomicOr(&dw->status, NBODY_TREE_INCEST_NONFATAL);
    }
    ax[j] = accx; ay[j] = accy; az[j] = accz;
}

// nbMapForceBody's epilogue for every body after a tree walk: a = self-gravity (as the walk
// stored it) + nbExtAcceleration + the zero LMC term, then the optional kick (nb_finish_body).
// FOREST: each body with its dwarf's time step and the bar's time of its dwarf.
// CAUSTIC: the potential's halo is the caustic one (its code compiled in only then).
template <bool FOREST, bool CAUSTIC>
__global__ void k_body_epilogue(const double* __restrict__ px, const double* __restrict__ py,
                                const double* __restrict__ pz, double* __restrict__ ax,
                                double* __restrict__ ay, double* __restrict__ az,
                                double* __restrict__ vx, double* __restrict__ vy,
                                double* __restrict__ vz, NbWalkParams wp, NbPot pot,
                                const NbScalars* __restrict__ sc, NbForest forest)
{
    if (nb_failed(sc)) return;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < wp.n; j += gridDim.x * blockDim.x) {
        NbWalkParams w = wp;
        NbPot p = pot;
        if (FOREST) {
            const int dj = forest.bodyDwarf[j];
            NbDwarfDev& d = forest.dwarfs[dj];
            w.dtHalf = 0.5 * d.dt;
            p.time = d.time;
            // LMC runs: this dwarf's LMC and its reflex acceleration acc_i1 (selects, not
            // branches: a conditional update of the copies costs the kernel ~70 registers)
            const bool lmc = forest.lmcShift != nullptr;
            p.lmc = lmc ? d.lmc : p.lmc;
            const double* sh = lmc && w.kick
                ? forest.lmcShift + 3 * ((size_t) dj * forest.nShift + sc->step + 1) : w.shift;
            const double s0 = sh[0], s1 = sh[1], s2 = sh[2];
            w.shift[0] = s0; w.shift[1] = s1; w.shift[2] = s2;
        }
        nb_finish_body<CAUSTIC>(p, w, (unsigned) j, px[j], py[j], pz[j], ax[j], ay[j], az[j], ax, ay, az,
                       vx, vy, vz);
    }
}

void nb_launch_body_epilogue(const double* px, const double* py, const double* pz, double* ax,
                             double* ay, double* az, double* vx, double* vy, double* vz,
                             const NbWalkParams& wp, const NbPot& pot, const NbScalars* sc,
                             int numSMs, cudaStream_t s, const NbForest* forest)
{
    if (wp.n <= 0) return;
    const int g = numSMs > 0 ? min((wp.n + 255) / 256, numSMs * 8) : (wp.n + 255) / 256;
    const NbForest f = forest ? *forest : NbForest{nullptr, nullptr, 0, nullptr, 0};
    const bool caustic = pot.enabled && pot.haloType == NBCUDA_CAUSTIC_HALO;
#define NB_EPI_ARGS px, py, pz, ax, ay, az, vx, vy, vz, wp, pot, sc, f
    if (forest) {
        if (caustic) k_body_epilogue<true, true><<<g, 256, 0, s>>>(NB_EPI_ARGS);
        else k_body_epilogue<true, false><<<g, 256, 0, s>>>(NB_EPI_ARGS);
    } else {
        if (caustic) k_body_epilogue<false, true><<<g, 256, 0, s>>>(NB_EPI_ARGS);
        else k_body_epilogue<false, false><<<g, 256, 0, s>>>(NB_EPI_ARGS);
    }
#undef NB_EPI_ARGS
    nb_count_launch();
}

// nbGravity_Exact (nbody/src/nbody_grav.c:205-227): direct sum over all bodies in input
// order (the self term contributes 0 * dr).  One thread per body; sources staged in tiles.
constexpr int EXACT_TILE = 256;
__global__ void __launch_bounds__(EXACT_TILE)
k_direct_fp64(const double* __restrict__ px, const double* __restrict__ py,
              const double* __restrict__ pz, const double* __restrict__ mass,
              double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
              double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
              NbWalkParams wp, NbPot pot, NbScalars* __restrict__ sc)
{
    __shared__ double4 tile[EXACT_TILE];
    const int n = wp.n;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const double x0 = valid ? px[i] : 0.0, y0 = valid ? py[i] : 0.0, z0 = valid ? pz[i] : 0.0;
    const double eps2 = wp.eps2;
    double accx = 0.0, accy = 0.0, accz = 0.0;
    for (int base = 0; base < n; base += EXACT_TILE) {
        const int k = base + threadIdx.x;
        __syncthreads();
        tile[threadIdx.x] = k < n ? make_double4(px[k], py[k], pz[k], mass[k]) : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int lim = min(EXACT_TILE, n - base);
        for (int t = 0; t < lim; ++t) {
            const double4 b = tile[t];
            const double dx = b.x - x0, dy = b.y - y0, dz = b.z - z0;
            const double drSq = (dz * dz + (dy * dy + dx * dx)) + eps2;
            const double drab = sqrt(drSq);
            const double phii = b.w / drab;
            const double mor3 = phii / drSq;
            accx = accx + mor3 * dx;
            accy = accy + mor3 * dy;
            accz = accz + mor3 * dz;
        }
    }
    if (valid) nb_finish_body(pot, wp, (unsigned) i, x0, y0, z0, accx, accy, accz, ax, ay, az, vx, vy, vz);
}

// Direct FP64 sums (nbGravity_Exact arithmetic) for a sample of target bodies: the accuracy
// oracle of the walk forms.  Self-gravity only.
__global__ void __launch_bounds__(EXACT_TILE)
k_direct_sample(const double* __restrict__ px, const double* __restrict__ py,
                const double* __restrict__ pz, const double* __restrict__ mass, int n,
                const int* __restrict__ targets, int count, double eps2, double* __restrict__ out)
{
    __shared__ double4 tile[EXACT_TILE];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = t < count;
    const int i = valid ? targets[t] : 0;
    const double x0 = px[i], y0 = py[i], z0 = pz[i];
    double accx = 0.0, accy = 0.0, accz = 0.0;
    for (int base = 0; base < n; base += EXACT_TILE) {
        const int k = base + threadIdx.x;
        __syncthreads();
        tile[threadIdx.x] = k < n ? make_double4(px[k], py[k], pz[k], mass[k]) : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int lim = min(EXACT_TILE, n - base);
        for (int s = 0; s < lim; ++s) {
            const double4 b = tile[s];
            const double dx = b.x - x0, dy = b.y - y0, dz = b.z - z0;
            const double drSq = (dz * dz + (dy * dy + dx * dx)) + eps2;
            const double drab = sqrt(drSq);
            const double phii = b.w / drab;
            const double mor3 = phii / drSq;
            accx = accx + mor3 * dx;
            accy = accy + mor3 * dy;
            accz = accz + mor3 * dz;
        }
    }
    if (valid) { out[3 * t] = accx; out[3 * t + 1] = accy; out[3 * t + 2] = accz; }
}

// Total energy of the current state, FP64 direct summation (the energy-drift oracle of the
// walk forms; O(N^2)): out[0] += sum m v^2 / 2, out[1] += -sum_{i<j} m_i m_j / sqrt(r^2 + eps^2)
// (the softened pair potential whose gradient the walk's forces are), out[2] += sum m Phi_ext.
__global__ void __launch_bounds__(EXACT_TILE)
k_energy(const double* __restrict__ px, const double* __restrict__ py,
         const double* __restrict__ pz, const double* __restrict__ vx,
         const double* __restrict__ vy, const double* __restrict__ vz,
         const double* __restrict__ mass, int n, double eps2, NbPot pot, double* __restrict__ out)
{
    __shared__ double4 tile[EXACT_TILE];
    __shared__ double red[3][EXACT_TILE / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const double x0 = valid ? px[i] : 0.0, y0 = valid ? py[i] : 0.0, z0 = valid ? pz[i] : 0.0;
    double phi = 0.0;
    for (int base = 0; base < n; base += EXACT_TILE) {
        const int k = base + threadIdx.x;
        __syncthreads();
        tile[threadIdx.x] = k < n ? make_double4(px[k], py[k], pz[k], mass[k]) : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int lim = min(EXACT_TILE, n - base);
        for (int s = 0; s < lim; ++s) {
            const double4 b = tile[s];
            const double dx = b.x - x0, dy = b.y - y0, dz = b.z - z0;
            const double drSq = (dz * dz + (dy * dy + dx * dx)) + eps2;
            phi += base + s == i ? 0.0 : b.w / sqrt(drSq);
        }
    }
    double e[3] = {0.0, 0.0, 0.0};
    if (valid) {
        const double m = mass[i];
        e[0] = 0.5 * m * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
        e[1] = -0.5 * m * phi;
        e[2] = pot.enabled ? m * nb_ext_potential(pot, x0, y0, z0) : 0.0;
    }
    for (int c = 0; c < 3; ++c) {
        double v = e[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(NB_FULL_MASK, v, o);
        if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int w = 0; w < EXACT_TILE / 32; ++w) v += red[threadIdx.x][w];
        atomicAdd(out + threadIdx.x, v);
    }
}

void nb_launch_energy(const double* px, const double* py, const double* pz, const double* vx,
                      const double* vy, const double* vz, const double* mass, int n, double eps2,
                      const NbPot& pot, double* out, cudaStream_t s)
{
    cudaMemsetAsync(out, 0, 3 * sizeof(double), s);
    if (n <= 0) return;
    k_energy<<<(n + EXACT_TILE - 1) / EXACT_TILE, EXACT_TILE, 0, s>>>(px, py, pz, vx, vy, vz, mass,
                                                                     n, eps2, pot, out);
    nb_count_launch();
}

// FMA throughput probe: independent FMA chains per thread (the denominator of the walk's
// pipe roofline).  fp64 selects DFMA or FFMA.
template <typename T>
__global__ void k_fma_probe(T* out, int iters, T seed)
{
    T a0 = seed + (T) threadIdx.x, a1 = a0 + (T) 1, a2 = a0 + (T) 2, a3 = a0 + (T) 3;
    T a4 = a0 + (T) 4, a5 = a0 + (T) 5, a6 = a0 + (T) 6, a7 = a0 + (T) 7;
    const T m = (T) 0.999999, c = (T) 1e-7;
    for (int k = 0; k < iters; ++k) {
        a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
        a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
    const T s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == (T) -1) out[0] = s;   // keeps the chains live
}

__global__ void k_ext_only(const double* __restrict__ pos, double* __restrict__ acc, int n, NbPot pot)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ex, ey, ez;
        nb_ext_accel(pot, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], ex, ey, ez);
        acc[3 * i] = ex; acc[3 * i + 1] = ey; acc[3 * i + 2] = ez;
    }
}

// ---- host launchers ----

void nb_launch_body_epilogue(const double* px, const double* py, const double* pz, double* ax,
                             double* ay, double* az, double* vx, double* vy, double* vz,
                             const NbWalkParams& wp, const NbPot& pot, const NbScalars* sc,
                             int numSMs, cudaStream_t s, const NbForest* forest);

void nb_launch_pack_walk(const double4* nodePM, const double* nodeCrit, const int2* nodeLink,
                         const double* nodeQuad, double4* rec, int capNodes, const NbScalars* sc,
                         cudaStream_t s)
{
    k_pack_walk<<<min((capNodes + 255) / 256, 4096), 256, 0, s>>>(nodePM, nodeCrit, nodeLink,
                                                                  nodeQuad, rec, sc);
    nb_count_launch();
}

void nb_launch_walk_fp64(const double4* nodePM, const double* nodeCrit, const int2* nodeLink,
                         const double* nodeQuad, const unsigned* order, const double* px,
                         const double* py, const double* pz, double* ax, double* ay, double* az,
                         double* vx, double* vy, double* vz, const NbWalkParams& wp,
                         const NbPot& pot, NbScalars* sc, bool count, cudaStream_t s,
                         double4* walkRec, int capNodes, const NbForest* forest, int form)
{
    const int warps = (wp.n + 31) / 32;
    const int blocks = (warps * 32 + WALK_THREADS - 1) / WALK_THREADS;
    if (blocks <= 0) return;
    nb_launch_pack_walk(nodePM, nodeCrit, nodeLink, nodeQuad, walkRec, capNodes, sc, s);
    const NbForest f = forest ? *forest : NbForest{nullptr, nullptr, 0};
#define NB_WALK_ARGS walkRec, order, px, py, pz, ax, ay, az, vx, vy, vz, wp, pot, sc, f
#define NB_LANES_ARGS walkRec, order, px, py, pz, ax, ay, az, wp, sc, f
    if (forest) {
        if (form == 2) {
            if (count) k_walk_fp64_lanes<true, true, true><<<blocks, WALK_THREADS, 0, s>>>(NB_LANES_ARGS);
            else k_walk_fp64_lanes<false, true, true><<<blocks, WALK_THREADS, 0, s>>>(NB_LANES_ARGS);
        } else if (form == 1) {
            if (count) k_walk_fp64_lanes<true, true, false><<<blocks, WALK_THREADS, 0, s>>>(NB_LANES_ARGS);
            else k_walk_fp64_lanes<false, true, false><<<blocks, WALK_THREADS, 0, s>>>(NB_LANES_ARGS);
        } else {
            if (count) k_walk_fp64<true, true><<<blocks, WALK_THREADS, 0, s>>>(NB_WALK_ARGS);
            else k_walk_fp64<false, true><<<blocks, WALK_THREADS, 0, s>>>(NB_WALK_ARGS);
        }
    } else {
        if (form == 2) {
            if (count) k_walk_fp64_lanes<true, false, true><<<blocks, WALK_THREADS, 0, s>>>(NB_LANES_ARGS);
            else k_walk_fp64_lanes<false, false, true><<<blocks, WALK_THREADS, 0, s>>>(NB_LANES_ARGS);
        } else if (form == 1) {
            if (count) k_walk_fp64_lanes<true, false, false><<<blocks, WALK_THREADS, 0, s>>>(NB_LANES_ARGS);
            else k_walk_fp64_lanes<false, false, false><<<blocks, WALK_THREADS, 0, s>>>(NB_LANES_ARGS);
        } else {
            if (count) k_walk_fp64<true, false><<<blocks, WALK_THREADS, 0, s>>>(NB_WALK_ARGS);
            else k_walk_fp64<false, false><<<blocks, WALK_THREADS, 0, s>>>(NB_WALK_ARGS);
        }
    }
#undef NB_WALK_ARGS
#undef NB_LANES_ARGS
    nb_count_launch();
    nb_launch_body_epilogue(px, py, pz, ax, ay, az, vx, vy, vz, wp, pot, sc, 0, s, forest);
}

void nb_launch_direct_fp64(const double* px, const double* py, const double* pz,
                           const double* mass, double* ax, double* ay, double* az, double* vx,
                           double* vy, double* vz, const NbWalkParams& wp, const NbPot& pot,
                           NbScalars* sc, cudaStream_t s)
{
    const int blocks = (wp.n + EXACT_TILE - 1) / EXACT_TILE;
    if (blocks <= 0) return;
    k_direct_fp64<<<blocks, EXACT_TILE, 0, s>>>(px, py, pz, mass, ax, ay, az, vx, vy, vz, wp, pot, sc);
    nb_count_launch();
}

void nb_launch_ext_only(const double* dpos, double* dacc, int n, const NbPot& pot, cudaStream_t s)
{
    if (n <= 0) return;
    k_ext_only<<<(n + 255) / 256, 256, 0, s>>>(dpos, dacc, n, pot);
    nb_count_launch();
}

void nb_launch_direct_sample(const double* px, const double* py, const double* pz,
                             const double* mass, int n, const int* targets, int count,
                             double eps2, double* out, cudaStream_t s)
{
    if (count <= 0) return;
    k_direct_sample<<<(count + EXACT_TILE - 1) / EXACT_TILE, EXACT_TILE, 0, s>>>(
        px, py, pz, mass, n, targets, count, eps2, out);
    nb_count_launch();
}

// Returns the achieved FMA rate in TFLOP/s (2 flops per FMA) over blocks x 256 threads.
double nb_fma_probe(int fp64, int numSMs, cudaStream_t s)
{
    const int threads = 256, blocks = numSMs * 8, iters = 1 << 14;
    void* out = nullptr;
    cudaMalloc(&out, 16);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0.0;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0, s);
        if (fp64) k_fma_probe<double><<<blocks, threads, 0, s>>>((double*) out, iters, 1.0);
        else k_fma_probe<float><<<blocks, threads, 0, s>>>((float*) out, iters, 1.0f);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8.0 * (double) iters * threads * (double) blocks;
        if (ms > 0.f) best = fmax(best, flops / (ms * 1e-3) / 1e12);
    }
    nb_count_launch(3);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return best;
}
