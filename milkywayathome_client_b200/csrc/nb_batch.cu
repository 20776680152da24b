// Batched dwarfs: many independent simulations stepped together, one launch per phase.
//
// No reference counterpart as such: the reference runs one dwarf per process.  Each dwarf here
// is exactly the reference's simulation -- its own root (centred at the origin, its own root
// size doubled by expandBox, nbody/src/nbody_tree.c:156-176), its own octree, its own
// softening and time step -- and its accelerations are bit for bit those of a single-dwarf run
// (nb_tree.cu, nb_walk.cu).  The trees of all dwarfs live in one set of node arrays, a forest:
//   * bodies are concatenated dwarf after dwarf and sorted by (dwarf, octree path): the
//     Morton-key passes of the radix sort, then two passes over the dwarf index;
//   * the parting depth of two sorted neighbours of different dwarfs is -1 (they part above
//     any root), so the owned-cell prefix sum lays out every dwarf's tree in walk order, one
//     after the other: dwarf d's nodes are [rootNode_d, rootEnd_d) and Next(root_d) is the
//     next dwarf's root;
//   * cell geometry, rcrit2 and the structure checks use the dwarf's own root size;
//   * the walks start every body at its dwarf's root and stop at Next(root).
// Every phase is one launch over all dwarfs (bodies or nodes of all trees), so a batch of
// small dwarfs fills the GPU where one of them alone would not.  Compiled with -fmad=false
// like the single-tree build.  Bare line citations (:N) refer to nbody/src/nbody_tree.c.
#include "nb_common.cuh"
#include "nb_tree_util.cuh"
#include <cfloat>

namespace {

__device__ __forceinline__ int nb_b_cells_before_body(const int* cum, int i, int n)
{
    return i < 0 ? 0 : cum[min(i, n - 2)];
}

// Per-evaluation reset of the scalars (root sizes, capacity and sticky dwarf status kept).
__global__ void k_b_reset(NbScalars* __restrict__ sc, NbDwarfDev* __restrict__ dw, int nDwarfs,
                          int n)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        sc->xyzmaxBits = 0;
        sc->nTree = n;
        sc->status = 0;
        sc->incest = 0;
        sc->nBodyBody = sc->nBodyCell = sc->nVisit = sc->nWarpSteps = 0;
        sc->groupNext = 0;
        sc->nGroups = 0;
        sc->maxDepth = 0;
    }
    for (int d = t; d < nDwarfs; d += gridDim.x * blockDim.x) {
        dw[d].xyzmaxBits = 0;
        // barTime of this evaluation: the shared origin, or the dwarf's own (the other is 0)
        dw[d].time = sc->step * dw[d].dt - sc->timeOrigin - dw[d].timeOrigin;
    }
}

// advancePosVel (nbody/src/nbody_plain.c:268-284) with each dwarf's time step, fused with
// expandBox's max |x| per dwarf.  A warp handles 32 consecutive bodies per iteration and
// reduces their maxima per dwarf (at most a few dwarfs per warp).
__global__ void k_b_drift_bbox(double* __restrict__ px, double* __restrict__ py,
                               double* __restrict__ pz, double* __restrict__ vx,
                               double* __restrict__ vy, double* __restrict__ vz,
                               const double* __restrict__ ax, const double* __restrict__ ay,
                               const double* __restrict__ az, const int* __restrict__ bodyDwarf,
                               NbDwarfDev* __restrict__ dw, int n, int drift,
                               const double* __restrict__ lmcShift, int nShift,
                               const NbScalars* __restrict__ sc)
{
    const int lane = threadIdx.x & 31;
    const int warpsTotal = (gridDim.x * blockDim.x) >> 5;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n;
         base += warpsTotal * 32) {
        const int i = base + lane;
        const bool valid = i < n;
        int d = valid ? bodyDwarf[i] : -1;
        double m = 0.0;
        if (valid) {
            double x = px[i], y = py[i], z = pz[i];
            if (drift) {
                const double dt = dw[d].dt;
                const double dtHalf = 0.5 * dt;
                // the Milky Way's reflex acceleration of LMC runs (acc_i), else 0
                double sx = 0.0, sy = 0.0, sz = 0.0;
                if (lmcShift) {
                    const double* sh = lmcShift + 3 * ((size_t) d * nShift + sc->step);
                    sx = sh[0]; sy = sh[1]; sz = sh[2];
                }
                double vvx = vx[i], vvy = vy[i], vvz = vz[i];
                vvx = vvx + dtHalf * (ax[i] + sx);
                vvy = vvy + dtHalf * (ay[i] + sy);
                vvz = vvz + dtHalf * (az[i] + sz);
                x = x + dt * vvx;
                y = y + dt * vvy;
                z = z + dt * vvz;
                vx[i] = vvx; vy[i] = vvy; vz[i] = vvz;
                px[i] = x; py[i] = y; pz[i] = z;
            }
            m = fmax(m, fabs(x - 0.0));
            m = fmax(m, fabs(y - 0.0));
            m = fmax(m, fabs(z - 0.0));
        }
        // segmented maximum: one round per distinct dwarf in this warp (<= 32 rounds)
        unsigned pending = __ballot_sync(NB_FULL_MASK, valid);
        while (pending) {
            const int leader = __ffs(pending) - 1;
            const int dl = __shfl_sync(NB_FULL_MASK, d, leader);
            double v = d == dl ? m : 0.0;
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(NB_FULL_MASK, v, o));
            if (lane == leader)
                atomicMax(&dw[dl].xyzmaxBits, (unsigned long long) __double_as_longlong(v));
            pending &= ~__ballot_sync(NB_FULL_MASK, d == dl);
        }
    }
}

// expandBox's doubling (:172-175) and the grid constants, per dwarf.
__global__ void k_b_root_size(NbDwarfDev* __restrict__ dw, int nDwarfs, NbScalars* __restrict__ sc)
{
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nDwarfs; d += gridDim.x * blockDim.x) {
        const double xyzmax = __longlong_as_double((long long) dw[d].xyzmaxBits);
        double rsize = dw[d].rsize;
        while (rsize < 2.0 * xyzmax) rsize *= 2.0;
        dw[d].rsize = rsize;
        if (!isfinite(rsize)) {
            atomicOr(&dw[d].status, NBODY_TREE_STRUCTURE_ERROR);
            nb_raise(sc, NBODY_TREE_STRUCTURE_ERROR);
            continue;
        }
        dw[d].gridScale = ldexp(1.0, NB_GRID_LEVELS - ilogb(rsize));
        int e = 0;
        double q = rsize;
        while (!(q <= DBL_EPSILON)) { q *= 0.5; ++e; }   // nbLoadBody: qsize <= REAL_EPSILON
        dw[d].depthEps = e;
    }
}

__global__ void k_b_keys(const double* __restrict__ px, const double* __restrict__ py,
                         const double* __restrict__ pz, const double* __restrict__ mass,
                         const int* __restrict__ bodyDwarf, const NbDwarfDev* __restrict__ dw,
                         int n, unsigned long long* __restrict__ key, unsigned int* __restrict__ idx,
                         NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    int massless = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double scale = dw[bodyDwarf[i]].gridScale;
        key[i] = nb_morton63(nb_grid(px[i], scale), nb_grid(py[i], scale), nb_grid(pz[i], scale));
        idx[i] = (unsigned) i;
        massless |= mass[i] == 0.0;
    }
    // a batch holds massive bodies only (test particles would sort outside their dwarf)
    if (massless) nb_raise(sc, NBODY_UNSUPPORTED);
}

__global__ void k_b_gather_grid(const double* __restrict__ px, const double* __restrict__ py,
                                const double* __restrict__ pz, const unsigned int* __restrict__ idx,
                                const int* __restrict__ bodyDwarf, const NbDwarfDev* __restrict__ dw,
                                long long* __restrict__ gx, long long* __restrict__ gy,
                                long long* __restrict__ gz, int n, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned j = idx[i];
        const double scale = dw[bodyDwarf[i]].gridScale;   // sorted position i is in j's dwarf
        gx[i] = nb_grid(px[j], scale);
        gy[i] = nb_grid(py[j], scale);
        gz[i] = nb_grid(pz[j], scale);
    }
}

// Runs of equal 21-level keys inside one dwarf, put in full-path order (as k_fix_runs).
__global__ void k_b_fix_runs(const unsigned long long* __restrict__ key,
                             const int* __restrict__ bodyDwarf, unsigned int* __restrict__ idx,
                             long long* __restrict__ gx, long long* __restrict__ gy,
                             long long* __restrict__ gz, int n, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n; i += gridDim.x * blockDim.x) {
        const int d = bodyDwarf[i];
        if (key[i + 1] != key[i] || bodyDwarf[i + 1] != d) continue;
        if (i > 0 && key[i - 1] == key[i] && bodyDwarf[i - 1] == d) continue;
        int end = i + 2;
        while (end < n && key[end] == key[i] && bodyDwarf[end] == d) ++end;
        for (int a = i + 1; a < end; ++a) {
            long long x = gx[a], y = gy[a], z = gz[a];
            unsigned int id = idx[a];
            int b = a - 1;
            while (b >= i && nb_path_less(x, y, z, gx[b], gy[b], gz[b])) {
                gx[b + 1] = gx[b]; gy[b + 1] = gy[b]; gz[b + 1] = gz[b]; idx[b + 1] = idx[b];
                --b;
            }
            gx[b + 1] = x; gy[b + 1] = y; gz[b + 1] = z; idx[b + 1] = id;
        }
    }
}

// Parting depth of sorted neighbours (-1 across a dwarf boundary) and owned-cell counts.
__device__ __forceinline__ int nb_b_part(const long long* gx, const long long* gy,
                                         const long long* gz, const int* bodyDwarf, int i)
{
    if (bodyDwarf[i] != bodyDwarf[i + 1]) return -1;
    return nb_part_depth(gx[i], gy[i], gz[i], gx[i + 1], gy[i + 1], gz[i + 1]);
}

__global__ void k_b_delta(const long long* __restrict__ gx, const long long* __restrict__ gy,
                          const long long* __restrict__ gz, const int* __restrict__ bodyDwarf,
                          NbDwarfDev* __restrict__ dw, int* __restrict__ delta,
                          int* __restrict__ cnt, int n, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n; i += gridDim.x * blockDim.x) {
        int d = nb_b_part(gx, gy, gz, bodyDwarf, i);
        if (d >= 0) {
            // nbLoadBody's structure error (:256-264): a pair parting beyond depthEps
            const int dd = bodyDwarf[i];
            if (d >= dw[dd].depthEps + 1 || d >= NB_GRID_LEVELS) {
                bad = 1;
                atomicOr(&dw[dd].status, NBODY_TREE_STRUCTURE_ERROR);
                d = min(d, NB_GRID_LEVELS - 1);
            }
        }
        delta[i] = d;
        int prev = -1;
        if (i > 0) prev = min(nb_b_part(gx, gy, gz, bodyDwarf, i - 1), NB_GRID_LEVELS - 1);
        cnt[i] = d > prev ? d - prev : 0;
    }
    if (bad) nb_raise(sc, NBODY_TREE_STRUCTURE_ERROR);
}

__global__ void k_b_count_nodes(const int* __restrict__ cum, int n, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int cells = cum[n - 2];
    sc->nCells = cells;
    sc->nNodes = n + cells;
    sc->neededNodes = n + cells;
    sc->maxDepth = 0;
    if (n + cells > sc->capNodes) nb_raise(sc, NBODY_CELL_OVERFLOW_ERROR);
}

// Node records of the bodies in walk order (as k_emit_bodies, parting depths -1 at dwarf
// boundaries).
__global__ void k_b_emit_bodies(const double* __restrict__ px, const double* __restrict__ py,
                                const double* __restrict__ pz, const double* __restrict__ mass,
                                const unsigned int* __restrict__ idx, const int* __restrict__ delta,
                                const int* __restrict__ cum, double4* __restrict__ nodePM,
                                double* __restrict__ nodeCrit, int2* __restrict__ nodeLink,
                                int* __restrict__ nodeDepth, int* __restrict__ bodyNode,
                                int2* __restrict__ nodeRange, int n, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    int maxLev = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned j = idx[i];
        const int p = i + nb_b_cells_before_body(cum, i, n);
        nodePM[p] = make_double4(px[j], py[j], pz[j], mass[j]);
        nodeCrit[p] = 0.0;
        nodeLink[p] = make_int2(p + 1, (int) j);
        nodeRange[p] = make_int2(i, i);
        const int dl = i > 0 ? delta[i - 1] : -1, dr = i < n - 1 ? delta[i] : -1;
        const int lev = max(0, max(dl, dr));
        nodeDepth[p] = lev + 1;
        bodyNode[i] = p;
        maxLev = max(maxLev, lev);
    }
    for (int o = 16; o > 0; o >>= 1) maxLev = max(maxLev, __shfl_xor_sync(NB_FULL_MASK, maxLev, o));
    if ((threadIdx.x & 31) == 0 && maxLev) atomicMax(&sc->maxDepth, maxLev);
}

// Cells owned by boundary a (as k_emit_cells), geometry from the dwarf's root size; the
// depth-0 cell of a dwarf is its root and records the dwarf's node range.
__global__ void k_b_emit_cells(const long long* __restrict__ gx, const long long* __restrict__ gy,
                               const long long* __restrict__ gz, const int* __restrict__ delta,
                               const int* __restrict__ cum, const int* __restrict__ bodyDwarf,
                               NbDwarfDev* __restrict__ dw, double4* __restrict__ nodePM,
                               double* __restrict__ nodeCrit, int2* __restrict__ nodeLink,
                               int* __restrict__ nodeDepth, int2* __restrict__ nodeRange, int n,
                               NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n - 1; a += gridDim.x * blockDim.x) {
        const int dPrev = a > 0 ? delta[a - 1] : -1, dHere = delta[a];
        if (dHere <= dPrev) continue;
        const int dwi = bodyDwarf[a];
        const double rsize = dw[dwi].rsize;
        const int dEnd = dw[dwi].first + dw[dwi].count;      // first body past this dwarf
        const int cellsBefore = a > 0 ? cum[a - 1] : 0;
        double cx = 0.0, cy = 0.0, cz = 0.0, size = rsize;
        const long long bx = gx[a], by = gy[a], bz = gz[a];
        for (int d = 0; d <= dPrev; ++d) {
            const int sh = NB_GRID_LEVELS - 1 - d;
            cx = cx + 0.25 * (((bx >> sh) & 1) ? size : -size);
            cy = cy + 0.25 * (((by >> sh) & 1) ? size : -size);
            cz = cz + 0.25 * (((bz >> sh) & 1) ? size : -size);
            size *= 0.5;
        }
        for (int D = dPrev + 1; D <= dHere; ++D) {
            const int p = a + cellsBefore + (D - dPrev - 1);
            const int last = nb_range_end(gx, gy, gz, a, D, dEnd);
            const int next = last + nb_b_cells_before_body(cum, last, n) + 1;
            nodeRange[p] = make_int2(a, last);
            nodePM[p] = make_double4(cx, cy, cz, 0.0);
            nodeCrit[p] = 0.0;
            nodeLink[p] = make_int2(next, -1);
            nodeDepth[p] = D;
            if (D == 0) { dw[dwi].rootNode = p; dw[dwi].rootEnd = next; }
            const int sh = NB_GRID_LEVELS - 1 - D;
            if (sh >= 0) {
                cx = cx + 0.25 * (((bx >> sh) & 1) ? size : -size);
                cy = cy + 0.25 * (((by >> sh) & 1) ? size : -size);
                cz = cz + 0.25 * (((bz >> sh) & 1) ? size : -size);
            }
            size *= 0.5;
        }
    }
}

// Parents (-1 for every dwarf's root) and child counts from Next().
__global__ void k_b_link_children(const int2* __restrict__ nodeLink, const int* __restrict__ nodeDepth,
                                  int* __restrict__ parent, int* __restrict__ nchild,
                                  int* __restrict__ arrive, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int nNodes = sc->nNodes;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nNodes; c += gridDim.x * blockDim.x) {
        const int2 l = nodeLink[c];
        if (l.y >= 0) continue;            // body
        if (nodeDepth[c] == 0) parent[c] = -1;
        int k = c + 1, count = 0;
        while (k < l.x) {
            parent[k] = c;
            ++count;
            k = nodeLink[k].x;
        }
        nchild[c] = count;
        arrive[c] = 0;
    }
}

// Bottom-up moments (as k_moments) with the dwarf's root size.
__global__ void k_b_moments(double4* __restrict__ nodePM, double* __restrict__ nodeCrit,
                            const int2* __restrict__ nodeLink, const int* __restrict__ nodeDepth,
                            double* __restrict__ nodeQuad, const int* __restrict__ parent,
                            const int* __restrict__ nchild, int* __restrict__ arrive,
                            const int* __restrict__ bodyNode, const int* __restrict__ bodyDwarf,
                            NbDwarfDev* __restrict__ dw, int criterion, double theta, int useQuad,
                            int n, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    int structErr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int dwi = bodyDwarf[i];
        const double rsize = dw[dwi].rsize;
        int c = parent[bodyNode[i]];
        while (c >= 0) {
            __threadfence();
            if (atomicAdd(&arrive[c], 1) != nchild[c] - 1) break;   // not the last child
            __threadfence();
            const int end = __ldcg(&nodeLink[c].x);
            const double4 geo = nb_ld_pm(&nodePM[c]);
            double M = 0.0, cmx = 0.0, cmy = 0.0, cmz = 0.0;
            for (int k = c + 1; k < end; k = __ldcg(&nodeLink[k].x)) {
                const double4 q = nb_ld_pm(&nodePM[k]);
                M = M + q.w;
                cmx = cmx + q.w * q.x;
                cmy = cmy + q.w * q.y;
                cmz = cmz + q.w * q.z;
            }
            if (M > 0.0) { cmx = cmx / M; cmy = cmy / M; cmz = cmz / M; }
            else { cmx = geo.x; cmy = geo.y; cmz = geo.z; }
            const int D = __ldcg(&nodeDepth[c]);
            double psize = rsize;
            for (int d = 0; d < D; ++d) psize *= 0.5;
            const double h = 0.5 * psize;
            if (cmx < geo.x - h || cmx > geo.x + h || cmy < geo.y - h || cmy > geo.y + h ||
                cmz < geo.z - h || cmz > geo.z + h) {
                structErr = 1;
                atomicOr(&dw[dwi].status, NBODY_TREE_STRUCTURE_ERROR);
            }
            nodeCrit[c] = nb_find_rcrit2(criterion, theta, rsize, geo.x, geo.y, geo.z,
                                         cmx, cmy, cmz, psize);
            if (useQuad) {
                double qxx = 0.0, qxy = 0.0, qxz = 0.0, qyy = 0.0, qyz = 0.0, qzz = 0.0;
                for (int k = c + 1; k < end; k = __ldcg(&nodeLink[k].x)) {
                    const double4 q = nb_ld_pm(&nodePM[k]);
                    const double dx = q.x - cmx, dy = q.y - cmy, dz = q.z - cmz;
                    const double drsq = dz * dz + (dy * dy + dx * dx);
                    const double mq = q.w;
                    double txx = mq * (3.0 * (dx * dx) - drsq);
                    double txy = mq * (3.0 * (dx * dy));
                    double txz = mq * (3.0 * (dx * dz));
                    double tyy = mq * (3.0 * (dy * dy) - drsq);
                    double tyz = mq * (3.0 * (dy * dz));
                    double tzz = mq * (3.0 * (dz * dz) - drsq);
                    if (__ldcg(&nodeLink[k].y) < 0) {
                        const double* Q = nodeQuad + 6 * (size_t) k;
                        txx = txx + __ldcg(Q + 0); txy = txy + __ldcg(Q + 1); txz = txz + __ldcg(Q + 2);
                        tyy = tyy + __ldcg(Q + 3); tyz = tyz + __ldcg(Q + 4); tzz = tzz + __ldcg(Q + 5);
                    }
                    qxx = qxx + txx; qxy = qxy + txy; qxz = qxz + txz;
                    qyy = qyy + tyy; qyz = qyz + tyz; qzz = qzz + tzz;
                }
                double* Q = nodeQuad + 6 * (size_t) c;
                Q[0] = qxx; Q[1] = qxy; Q[2] = qxz; Q[3] = qyy; Q[4] = qyz; Q[5] = qzz;
            } else {
                // no quadrupoles: the record reads as zero (as the restated CPU tree does)
                double* Q = nodeQuad + 6 * (size_t) c;
                for (int k = 0; k < 6; ++k) Q[k] = 0.0;
            }
            nodePM[c] = make_double4(cmx, cmy, cmz, M);
            c = parent[c];
        }
    }
    if (structErr) nb_raise(sc, NBODY_TREE_STRUCTURE_ERROR);
}

}  // namespace

static inline int nb_b_grid(int n, int threads, int cap)
{
    int g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    return g < cap ? g : cap;
}

// One forest evaluation's tree phases: reset, drift + bounding boxes, root sizes, keys,
// grouped sort, parting depths, node emission, links and moments.  Every launch covers all
// dwarfs; nothing here synchronises with the host (the sequence is captured in a graph).
// Requires every dwarf to hold >= 2 bodies.  Returns the number of launches issued.
int nb_build_forest(NbTreeBuffers& b, const NbForest& f, int n, int capNodes, int criterion,
                    double theta, int useQuad, int drift, int numSMs, cudaStream_t s,
                    const NbBatchLMC* lmc)
{
    const int T = 256;
    const int gB = nb_b_grid(n, T, numSMs * 8);
    const int g = nb_b_grid(n, T, 1 << 20);
    int launches = 0;
    k_b_reset<<<nb_b_grid(f.nDwarfs, T, 64), T, 0, s>>>(b.sc, f.dwarfs, f.nDwarfs, n);
    // LMC runs: each LMC drifts and takes its first half kick before the bodies drift
    // (nbStepSystemPlain's advancePosVel_LMC follows advancePosVel but reads no body)
    if (lmc && drift) nb_launch_b_lmc_half(*lmc, f, b.sc, 0, s);
    k_b_drift_bbox<<<gB, T, 0, s>>>(b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.ax, b.ay, b.az,
                                    f.bodyDwarf, f.dwarfs, n, drift,
                                    lmc && drift ? f.lmcShift : nullptr, f.nShift, b.sc);
    k_b_root_size<<<nb_b_grid(f.nDwarfs, 128, 64), 128, 0, s>>>(f.dwarfs, f.nDwarfs, b.sc);
    k_b_keys<<<gB, T, 0, s>>>(b.px, b.py, b.pz, b.mass, f.bodyDwarf, f.dwarfs, n, b.sort.keyA,
                              b.sort.idxA, b.sc);
    launches += 4;
    nb_radix_sort_grouped(b.sort, n, f.bodyDwarf, s);
    launches += 50;
    k_b_gather_grid<<<g, T, 0, s>>>(b.px, b.py, b.pz, b.sort.idxA, f.bodyDwarf, f.dwarfs, b.gx,
                                    b.gy, b.gz, n, b.sc);
    k_b_fix_runs<<<g, T, 0, s>>>(b.sort.keyA, f.bodyDwarf, b.sort.idxA, b.gx, b.gy, b.gz, n, b.sc);
    k_b_delta<<<g, T, 0, s>>>(b.gx, b.gy, b.gz, f.bodyDwarf, f.dwarfs, b.delta, b.cum, n, b.sc);
    launches += 3;
    nb_inclusive_scan(b.cum, n - 1, b.scanTmp, s);
    launches += 3;
    k_b_count_nodes<<<1, 1, 0, s>>>(b.cum, n, b.sc);
    k_b_emit_bodies<<<g, T, 0, s>>>(b.px, b.py, b.pz, b.mass, b.sort.idxA, b.delta, b.cum,
                                    b.nodePM, b.nodeCrit, b.nodeLink, b.nodeDepth, b.bodyNode,
                                    b.nodeRange, n, b.sc);
    k_b_emit_cells<<<g, T, 0, s>>>(b.gx, b.gy, b.gz, b.delta, b.cum, f.bodyDwarf, f.dwarfs,
                                   b.nodePM, b.nodeCrit, b.nodeLink, b.nodeDepth, b.nodeRange, n,
                                   b.sc);
    k_b_link_children<<<nb_b_grid(capNodes, T, 1 << 20), T, 0, s>>>(b.nodeLink, b.nodeDepth,
                                                                    b.parent, b.nchild, b.arrive,
                                                                    b.sc);
    k_b_moments<<<g, T, 0, s>>>(b.nodePM, b.nodeCrit, b.nodeLink, b.nodeDepth, b.nodeQuad,
                                b.parent, b.nchild, b.arrive, b.bodyNode, f.bodyDwarf, f.dwarfs,
                                criterion, theta, useQuad, n, b.sc);
    launches += 5;
    nb_count_launch(launches - 53);       // the sort and the scan count their own
    return launches;
}

