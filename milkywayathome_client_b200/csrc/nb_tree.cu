// Octree build on the GPU, bit-exact with the reference CPU tree (nbMakeTree,
// nbody/src/nbody_tree.c:429-460).  Compiled with -fmad=false: every floating-point
// expression below is evaluated with the reference's operation order and no FMA
// contraction, so cell centres, centres of mass, rcrit2 and quadrupole moments carry the
// same bits as the CPU's.
//
// The CPU builds its tree by top-down insertion (nbLoadBody, :242-282) from a root centred
// at the origin whose size is doubled until it covers the bodies (expandBox, :156-176).
// The resulting octree is unique: a cell exists at depth D for every octree path prefix
// that at least two massive bodies share (chains of single-child cells included), plus
// the root.  Here the same octree is derived from bodies sorted by octree path:
//   1. bounding box (max |x|,|y|,|z|) and the root size doubling of expandBox;
//   2. integer grid coordinates floor(x*2^62/rsize) + 2^61: bit (61-d) is the child
//      octant bit at depth d, i.e. exactly the CPU's `mid <= pos` test (:42-49);
//   3. sort by the top 21 levels (63-bit Morton key, radix sort) and order the rare runs
//      of equal keys by the full 62-level path;
//   4. delta_i = depth at which sorted bodies i and i+1 part; boundary i "owns" the cells
//      at depths (delta_{i-1}, delta_i], so a prefix sum of owned counts gives every
//      node its position in the walk (preorder) order of threadTree (:127-150) directly;
//   5. each cell finds the last body of its range (galloping search on the sorted grid
//      coordinates), which gives Next(); parents and child counts follow from Next();
//   6. centres of mass, rcrit2 (findRCrit, :308-343) and quadrupoles (hackQuad, :70-121)
//      bottom-up: the last child to finish (atomic arrival counter) computes its parent,
//      reading the children in octant order as hackCofM does (:386-424).  No thread ever
//      waits on another.
#include "nb_common.cuh"
#include "nb_tree_util.cuh"
#include <cfloat>

// ---------------------------------------------------------------------------------
// 1. bounding box (optionally fused with the first half of the leapfrog step)
// ---------------------------------------------------------------------------------
// advancePosVel (nbody/src/nbody_plain.c:268-284): v += (a + acc_i) * dtHalf; x += v * dt
// with acc_i = 0 when the LMC is off; then expandBox's max |x - root| with root = 0.
__global__ void k_drift_bbox(double* __restrict__ px, double* __restrict__ py, double* __restrict__ pz,
                             double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
                             const double* __restrict__ ax, const double* __restrict__ ay,
                             const double* __restrict__ az, int n, int drift, double dt,
                             double sx, double sy, double sz, NbScalars* __restrict__ sc)
{
    double m = 0.0;
    const double dtHalf = 0.5 * dt;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x = px[i], y = py[i], z = pz[i];
        if (drift) {
            double vvx = vx[i], vvy = vy[i], vvz = vz[i];
            // advancePosVel (nbody/src/nbody_plain.c:268-284): v += (a + acc_i) dt/2, acc_i
            // the Milky Way's reflex acceleration of LMC runs (0 otherwise)
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
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(NB_FULL_MASK, m, o));
    __shared__ double wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(NB_FULL_MASK, m, o));
        // non-negative doubles order like their bit patterns
        if (threadIdx.x == 0) atomicMax(&sc->xyzmaxBits, (unsigned long long) __double_as_longlong(m));
    }
}

// expandBox's doubling loop (:172-175) and the grid constants derived from rsize.
__global__ void k_root_size(NbScalars* sc)
{
    if (nb_failed(sc)) return;
    const double xyzmax = __longlong_as_double((long long) sc->xyzmaxBits);
    double rsize = sc->rsize;
    while (rsize < 2.0 * xyzmax) rsize *= 2.0;
    sc->rsize = rsize;
    if (!isfinite(rsize)) { nb_raise(sc, NBODY_TREE_STRUCTURE_ERROR); return; }
    sc->gridScale = ldexp(1.0, NB_GRID_LEVELS - ilogb(rsize));
    int d = 0;
    double q = rsize;
    while (!(q <= DBL_EPSILON)) { q *= 0.5; ++d; }   // nbLoadBody: qsize <= REAL_EPSILON
    sc->depthEps = d;
}

// ---------------------------------------------------------------------------------
// 2. keys
// ---------------------------------------------------------------------------------
__global__ void k_keys(const double* __restrict__ px, const double* __restrict__ py,
                       const double* __restrict__ pz, const double* __restrict__ mass, int n,
                       unsigned long long* __restrict__ key, unsigned int* __restrict__ idx,
                       NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const double scale = sc->gridScale;
    int cnt = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned long long k = NB_MASSLESS_KEY;      // test particles are not in the tree (:440)
        if (mass[i] != 0.0) {
            k = nb_morton63(nb_grid(px[i], scale), nb_grid(py[i], scale), nb_grid(pz[i], scale));
            ++cnt;
        }
        key[i] = k;
        idx[i] = (unsigned) i;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(NB_FULL_MASK, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&sc->nTree, cnt);
}

// Grid coordinates of the sorted bodies.
__global__ void k_gather_grid(const double* __restrict__ px, const double* __restrict__ py,
                              const double* __restrict__ pz, const unsigned int* __restrict__ idx,
                              long long* __restrict__ gx, long long* __restrict__ gy,
                              long long* __restrict__ gz, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int m = sc->nTree;
    const double scale = sc->gridScale;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const unsigned j = idx[i];
        gx[i] = nb_grid(px[j], scale);
        gy[i] = nb_grid(py[j], scale);
        gz[i] = nb_grid(pz[j], scale);
    }
}

// Runs of bodies whose 21-level keys are equal are put in full-path order (insertion sort
// by the run's first thread; such runs hold only close pairs in practice).
__global__ void k_fix_runs(const unsigned long long* __restrict__ key, unsigned int* __restrict__ idx,
                           long long* __restrict__ gx, long long* __restrict__ gy,
                           long long* __restrict__ gz, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int m = sc->nTree;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i + 1 < m; i += gridDim.x * blockDim.x) {
        if (key[i + 1] != key[i] || (i > 0 && key[i - 1] == key[i])) continue;
        int end = i + 2;
        while (end < m && key[end] == key[i]) ++end;
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

// ---------------------------------------------------------------------------------
// 4. parting depths and owned-cell counts
// ---------------------------------------------------------------------------------
// delta[i] for boundary i in [0, m-2]; cnt[i] = cells owned by boundary i.
__global__ void k_delta(const long long* __restrict__ gx, const long long* __restrict__ gy,
                        const long long* __restrict__ gz, int* __restrict__ delta,
                        int* __restrict__ cnt, int n, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int m = sc->nTree;
    const int depthEps = sc->depthEps;
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i + 1 < n; i += gridDim.x * blockDim.x) {
        if (i + 1 >= m) { cnt[i] = 0; continue; }   // keep the scanned tail finite
        int d = nb_part_depth(gx[i], gy[i], gz[i], gx[i + 1], gy[i + 1], gz[i + 1]);
        // nbLoadBody raises a structure error when it must descend through a cell whose
        // size is <= REAL_EPSILON (:256-264): that happens iff some pair parts at a depth
        // beyond depthEps.
        if (d >= depthEps + 1 || d >= NB_GRID_LEVELS) { bad = 1; d = min(d, NB_GRID_LEVELS - 1); }
        delta[i] = d;
        int prev = -1;
        if (i > 0) {
            prev = nb_part_depth(gx[i - 1], gy[i - 1], gz[i - 1], gx[i], gy[i], gz[i]);
            prev = min(prev, NB_GRID_LEVELS - 1);
        }
        cnt[i] = d > prev ? d - prev : 0;
    }
    if (bad) nb_raise(sc, NBODY_TREE_STRUCTURE_ERROR);
}

__device__ __forceinline__ int nb_delta_or(const int* delta, int i, int m)
{
    return (i < 0 || i > m - 2) ? -1 : delta[i];
}

// Number of cells owned by boundaries 0..i (inclusive prefix, clamped to the last boundary).
__device__ __forceinline__ int nb_cells_before_body(const int* cum, int i, int m)
{
    if (m <= 1) return 1;                              // root only
    if (i < 0) return 0;
    return cum[min(i, m - 2)];
}

// Total node count; checks the capacity.
__global__ void k_count_nodes(const int* __restrict__ cum, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int m = sc->nTree;
    const int cells = m <= 1 ? 1 : cum[m - 2];
    sc->nCells = cells;
    sc->nNodes = m + cells;
    sc->neededNodes = m + cells;
    sc->maxDepth = 0;
    if (m + cells > sc->capNodes) nb_raise(sc, NBODY_CELL_OVERFLOW_ERROR);
}

// ---------------------------------------------------------------------------------
// 5. node emission in walk order
// ---------------------------------------------------------------------------------
__global__ void k_emit_bodies(const double* __restrict__ px, const double* __restrict__ py,
                              const double* __restrict__ pz, const double* __restrict__ mass,
                              const unsigned int* __restrict__ idx, const int* __restrict__ delta,
                              const int* __restrict__ cum, double4* __restrict__ nodePM,
                              double* __restrict__ nodeCrit, int2* __restrict__ nodeLink,
                              int* __restrict__ nodeDepth, int* __restrict__ bodyNode,
                              int2* __restrict__ nodeRange, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int m = sc->nTree;
    int maxLev = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const unsigned j = idx[i];
        const int p = i + nb_cells_before_body(cum, i, m);
        nodePM[p] = make_double4(px[j], py[j], pz[j], mass[j]);
        nodeCrit[p] = 0.0;
        nodeLink[p] = make_int2(p + 1, (int) j);
        nodeRange[p] = make_int2(i, i);
        const int lev = max(0, max(nb_delta_or(delta, i - 1, m), nb_delta_or(delta, i, m)));
        nodeDepth[p] = lev + 1;
        bodyNode[i] = p;
        maxLev = max(maxLev, lev);
    }
    for (int o = 16; o > 0; o >>= 1) maxLev = max(maxLev, __shfl_xor_sync(NB_FULL_MASK, maxLev, o));
    if ((threadIdx.x & 31) == 0 && maxLev) atomicMax(&sc->maxDepth, maxLev);
}

// Cells owned by boundary a: depths (delta_{a-1}, delta_a].  Writes the geometric centre
// (nbInitMidpoint/calcOffset, :226-239: c += 0.25 * (+-size) level by level from the
// origin) into nodePM.xyz until the moment pass replaces it by the centre of mass.
__global__ void k_emit_cells(const long long* __restrict__ gx, const long long* __restrict__ gy,
                             const long long* __restrict__ gz, const int* __restrict__ delta,
                             const int* __restrict__ cum, double4* __restrict__ nodePM,
                             double* __restrict__ nodeCrit, int2* __restrict__ nodeLink,
                             int* __restrict__ nodeDepth, double* __restrict__ nodeQuad,
                             int2* __restrict__ nodeRange, int criterion, double theta,
                             NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int m = sc->nTree;
    const double rsize = sc->rsize;
    const int nb = m <= 1 ? 1 : m - 1;        // boundaries (the root-only tree uses one slot)
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nb; a += gridDim.x * blockDim.x) {
        int dPrev, dHere;
        if (m <= 1) { dPrev = -1; dHere = 0; }
        else { dPrev = nb_delta_or(delta, a - 1, m); dHere = delta[a]; }
        if (dHere <= dPrev) continue;
        const int cellsBefore = a > 0 ? cum[a - 1] : 0;
        // centre of the depth-(dPrev+1) cell on body a's path
        double cx = 0.0, cy = 0.0, cz = 0.0, size = rsize;
        const long long bx = m >= 1 ? gx[a] : 0, by = m >= 1 ? gy[a] : 0, bz = m >= 1 ? gz[a] : 0;
        int d = 0;
        for (; d <= dPrev; ++d) {
            const int sh = NB_GRID_LEVELS - 1 - d;
            cx = cx + 0.25 * (((bx >> sh) & 1) ? size : -size);
            cy = cy + 0.25 * (((by >> sh) & 1) ? size : -size);
            cz = cz + 0.25 * (((bz >> sh) & 1) ? size : -size);
            size *= 0.5;
        }
        for (int D = dPrev + 1; D <= dHere; ++D) {
            const int p = a + cellsBefore + (D - dPrev - 1);
            int next, last;
            if (m <= 1) { next = m + 1; last = m - 1; }
            else {
                last = nb_range_end(gx, gy, gz, a, D, m);
                next = last + nb_cells_before_body(cum, last, m) + 1;
            }
            nodeRange[p] = make_int2(a, last);
            nodePM[p] = make_double4(cx, cy, cz, 0.0);
            nodeCrit[p] = 0.0;
            nodeLink[p] = make_int2(next, -1);
            nodeDepth[p] = D;
            if (m == 0) {
                // empty tree: hackCofM of a massless root keeps the geometric centre
                nodeCrit[p] = nb_find_rcrit2(criterion, theta, rsize, cx, cy, cz, cx, cy, cz, rsize);
                for (int k = 0; k < 6; ++k) nodeQuad[6 * (size_t) p + k] = 0.0;
            }
            // step to the child on body a's path
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

// Parent pointers and child counts from Next() (children of cell c: c+1, then Next()).
__global__ void k_link_children(const int2* __restrict__ nodeLink, int* __restrict__ parent,
                                int* __restrict__ nchild, int* __restrict__ arrive,
                                NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int nNodes = sc->nNodes;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nNodes; c += gridDim.x * blockDim.x) {
        if (c == 0) parent[0] = -1;
        const int2 l = nodeLink[c];
        if (l.y >= 0) continue;            // body
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

// ---------------------------------------------------------------------------------
// 6. moments, bottom-up
// ---------------------------------------------------------------------------------
__global__ void k_moments(double4* __restrict__ nodePM, double* __restrict__ nodeCrit,
                          const int2* __restrict__ nodeLink, const int* __restrict__ nodeDepth,
                          double* __restrict__ nodeQuad, const int* __restrict__ parent,
                          const int* __restrict__ nchild, int* __restrict__ arrive,
                          const int* __restrict__ bodyNode, int criterion, double theta,
                          int useQuad, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int m = sc->nTree;
    const double rsize = sc->rsize;
    int structErr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int c = parent[bodyNode[i]];
        while (c >= 0) {
            __threadfence();
            if (atomicAdd(&arrive[c], 1) != nchild[c] - 1) break;   // not the last child
            __threadfence();
            const int end = __ldcg(&nodeLink[c].x);
            const double4 geo = nb_ld_pm(&nodePM[c]);
            // hackCofM (:394-424)
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
            // nbCheckTreeStructure (:345-380)
            const double h = 0.5 * psize;
            if (cmx < geo.x - h || cmx > geo.x + h || cmy < geo.y - h || cmy > geo.y + h ||
                cmz < geo.z - h || cmz > geo.z + h)
                structErr = 1;
            nodeCrit[c] = nb_find_rcrit2(criterion, theta, rsize, geo.x, geo.y, geo.z,
                                         cmx, cmy, cmz, psize);
            if (useQuad) {
                // hackQuad (:70-121), children in octant order
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

// ---------------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------------


static inline int nb_grid_for(int n, int threads, int cap)
{
    int g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    return g < cap ? g : cap;
}

// Kernel sequence of nbMakeTree.  drift != 0 fuses advancePosVel into the bounding box.
void nb_build_tree(NbTreeBuffers& b, int n, int criterion, double theta, int useQuad,
                   int drift, double dt, int numSMs, cudaStream_t s, const double* shift)
{
    const double sx = shift ? shift[0] : 0.0, sy = shift ? shift[1] : 0.0;
    const double sz = shift ? shift[2] : 0.0;
    const int T = 256;
    const int gCap = numSMs * 8;
    cudaMemsetAsync(&b.sc->xyzmaxBits, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(&b.sc->nTree, 0, sizeof(int), s);
    k_drift_bbox<<<nb_grid_for(n, T, gCap), T, 0, s>>>(b.px, b.py, b.pz, b.vx, b.vy, b.vz,
                                                       b.ax, b.ay, b.az, n, drift, dt, sx, sy,
                                                       sz, b.sc);
    k_root_size<<<1, 1, 0, s>>>(b.sc);
    k_keys<<<nb_grid_for(n, T, gCap), T, 0, s>>>(b.px, b.py, b.pz, b.mass, n, b.sort.keyA,
                                                 b.sort.idxA, b.sc);
    nb_count_launch(3);
    nb_radix_sort(b.sort, n, s);
    const int g = nb_grid_for(n, T, 1 << 20);
    k_gather_grid<<<g, T, 0, s>>>(b.px, b.py, b.pz, b.sort.idxA, b.gx, b.gy, b.gz, b.sc);
    k_fix_runs<<<g, T, 0, s>>>(b.sort.keyA, b.sort.idxA, b.gx, b.gy, b.gz, b.sc);
    k_delta<<<g, T, 0, s>>>(b.gx, b.gy, b.gz, b.delta, b.cum, n, b.sc);
    nb_count_launch(3);
    // cum = inclusive prefix sum of owned-cell counts over boundaries [0, n-2] (the kernels
    // only read the first m-1 entries; entries past m-2 hold stale counts and are unused)
    if (n > 1) nb_inclusive_scan(b.cum, n - 1, b.scanTmp, s);
    k_count_nodes<<<1, 1, 0, s>>>(b.cum, b.sc);
    k_emit_bodies<<<g, T, 0, s>>>(b.px, b.py, b.pz, b.mass, b.sort.idxA, b.delta, b.cum, b.nodePM,
                                  b.nodeCrit, b.nodeLink, b.nodeDepth, b.bodyNode, b.nodeRange, b.sc);
    k_emit_cells<<<g, T, 0, s>>>(b.gx, b.gy, b.gz, b.delta, b.cum, b.nodePM, b.nodeCrit,
                                 b.nodeLink, b.nodeDepth, b.nodeQuad, b.nodeRange, criterion, theta,
                                 b.sc);
    nb_count_launch(3);
}

void nb_link_and_moments(NbTreeBuffers& b, int n, int capNodes, int criterion, double theta,
                         int useQuad, cudaStream_t s)
{
    const int T = 256;
    const int gNodes = nb_grid_for(capNodes, T, 1 << 20);
    const int g = nb_grid_for(n, T, 1 << 20);
    k_link_children<<<gNodes, T, 0, s>>>(b.nodeLink, b.parent, b.nchild, b.arrive, b.sc);
    k_moments<<<g, T, 0, s>>>(b.nodePM, b.nodeCrit, b.nodeLink, b.nodeDepth, b.nodeQuad, b.parent,
                              b.nchild, b.arrive, b.bodyNode, criterion, theta, useQuad, b.sc);
    nb_count_launch(2);
}

void nb_launch_drift_only(NbTreeBuffers& b, int n, double dt, int numSMs, cudaStream_t s,
                          const double* shift)
{
    const int T = 256;
    const double sx = shift ? shift[0] : 0.0, sy = shift ? shift[1] : 0.0;
    const double sz = shift ? shift[2] : 0.0;
    k_drift_bbox<<<nb_grid_for(n, T, numSMs * 8), T, 0, s>>>(b.px, b.py, b.pz, b.vx, b.vy, b.vz,
                                                             b.ax, b.ay, b.az, n, 1, dt, sx, sy,
                                                             sz, b.sc);
    nb_count_launch();
}
