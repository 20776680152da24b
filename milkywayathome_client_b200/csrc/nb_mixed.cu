// Mixed-precision force walk (no counterpart in the reference).
//
// Same tree and moments as the FP64 walk (nbGravity, nbody/src/nbody_grav.c:42-124); the
// walk and the interaction arithmetic are FP32, the accumulation FP64.  After the FP64 moment
// pass, k_pack_f32 stores every node as FP32 data relative to the root's centre of mass c:
// position as an unevaluated sum hi + lo (hi = f32(x - c), lo = f32((x - c) - hi)), mass,
// rcrit2, the quadrupole and the list of its children.  k_groups cuts the sorted bodies into
// walk groups of <= 32 consecutive bodies, none straddling two children of a cell with more
// than 32 bodies (so every group is spatially compact).  k_walk_mixed gives each group to one
// warp (persistent warps take groups from an atomic counter): the warp walks the tree
// depth-first, 32 nodes per step, with the group test |CoM - box|^2 >= rcrit2 (box = the
// group's bounding box), which implies the per-body test for every body of the group, so a
// group opens a superset of the cells its bodies would open.  Accepted cells and visited bodies
// go to per-warp interaction lists in shared memory, positions taken relative to the group's
// centre ((hi - centre) + lo, formed once by the appending lane): the walk runs in coordinates
// relative to the walking leaf group, so FP32 keeps its relative precision however far the
// dwarf sits from the origin.  All 32 lanes then evaluate the list, each for its own body
// (rsqrtf, explicit fmaf), and add the partial sums into FP64 after every cell list.  Centres
// of mass, moments, the external potential and the leapfrog stay FP64 (shared with the FP64
// code, compiled with -fmad=false so the shared epilogue keeps the reference's rounding).
#include "nb_common.cuh"
#include "nb_potential.cuh"


__device__ __forceinline__ void nb_split(double v, float& hi, float& lo)
{
    hi = __double2float_rn(v);
    lo = __double2float_rn(v - (double) hi);
}

// FP32 node records for the mixed walk (one pass over the nodes after the moments).
// FOREST: positions relative to the centre of mass of the node's own dwarf's root.
template <bool FOREST>
__global__ void k_pack_f32(const double4* __restrict__ nodePM, const double* __restrict__ nodeCrit,
                           const int2* __restrict__ nodeLink, const double* __restrict__ nodeQuad,
                           float4* __restrict__ nodeHi, float4* __restrict__ nodeLo,
                           float4* __restrict__ nodeQ32, int4* __restrict__ child8,
                           const int2* __restrict__ nodeRange, const NbScalars* __restrict__ sc,
                           NbForest forest)
{
    if (nb_failed(sc)) return;
    const int nNodes = sc->nNodes;
    double4 root = nodePM[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nNodes; k += gridDim.x * blockDim.x) {
        if (FOREST) root = nodePM[forest.dwarfs[forest.bodyDwarf[nodeRange[k].x]].rootNode];
        const double4 p = nodePM[k];
        float hx, hy, hz, lx, ly, lz;
        nb_split(p.x - root.x, hx, lx);
        nb_split(p.y - root.y, hy, ly);
        nb_split(p.z - root.z, hz, lz);
        const bool isBody = nodeLink[k].y >= 0;
        // bodies carry an rcrit2 of -inf, so the acceptance test needs no body branch
        const float crit = isBody ? __int_as_float(0xff800000) : __double2float_rn(nodeCrit[k]);
        nodeHi[k] = make_float4(hx, hy, hz, crit);
        if (isBody) {
            nodeLo[k] = make_float4(lx, ly, lz, __double2float_rn(p.w));
        } else {
            // a cell's slot c = k minus the tree bodies before it (they are the sorted bodies
            // below its first one): the cells' quadrupoles, masses and child lists are stored
            // densely by slot, and lo.w carries the slot (the mass is in the slot's record)
            const int c = k - nodeRange[k].x;
            nodeLo[k] = make_float4(lx, ly, lz, __int_as_float(c));
            // the children of a cell: k+1, then Next() up to Next(k) (threadTree order)
            int ch[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
            const int stop = nodeLink[k].x;
            int kc = k + 1;
            for (int m = 0; m < 8 && kc < stop; ++m) { ch[m] = kc; kc = nodeLink[kc].x; }
            child8[2 * (size_t) c] = make_int4(ch[0], ch[1], ch[2], ch[3]);
            child8[2 * (size_t) c + 1] = make_int4(ch[4], ch[5], ch[6], ch[7]);
            const double* Q = nodeQuad + 6 * (size_t) k;
            nodeQ32[2 * (size_t) c] = make_float4(__double2float_rn(Q[0]), __double2float_rn(Q[1]),
                                                  __double2float_rn(Q[2]), __double2float_rn(Q[3]));
            nodeQ32[2 * (size_t) c + 1] = make_float4(__double2float_rn(Q[4]), __double2float_rn(Q[5]),
                                                      __double2float_rn(p.w), 0.f);
        }
    }
}

// ---- group walk -------------------------------------------------------------------------
// A warp walks for a group of <= 32 bodies of one compact cell (k_groups).  Cells are tested
// against the group's bounding box: a cell is accepted when |CoM - box|^2 >= rcrit2, which
// implies the reference's per-body test |CoM - x|^2 >= rcrit2 (nbody/src/nbody_grav.c:58) for
// every body x of the group, so the group opens every cell any of its bodies would open.
//
// Walk: warp-parallel depth-first traversal.  Each step pops up to 32 nodes from the warp's
// stack (one per lane), tests them at once, appends visited bodies and accepted cells to two
// per-warp interaction lists in shared memory and pushes the children of opened cells
// (explicit child lists built by k_pack_f32).  Popping from the top keeps the stack sorted by
// depth, so at most 8 x 32 nodes of any one depth are ever on it: 256 x 63 levels bounds it
// (NB_GROUP_STACK).  A full list is evaluated by all 32 lanes at once (each lane for its own
// body, entries read as shared-memory broadcasts), FP32 with FMA and rsqrtf; partial sums go
// into FP64 accumulators after every list.  Persistent warps take groups from a counter.
constexpr int GROUP_WARPS = 4;
constexpr int GROUP_THREADS = 32 * GROUP_WARPS;
constexpr int NB_GROUP_STACK = 16384;     // >= 256 x 63 + 32

// Interaction lists in shared memory, one float4 array per field so that the 32 lanes'
// appends hit consecutive 16-byte slots (no bank conflicts) while the evaluation reads each
// entry as broadcasts.  Positions are stored relative to the walking group's centre (FP32):
// the lane that appends an entry forms (hi - centre) + lo once, so an interaction costs each
// body one subtraction per coordinate.  Cell entry: {rel, mass} {qxx, qxy, qxz, qyy}
// {qyz, qzz, use[0], use[1]}; body entry: {rel, mass} and use[q][e].
// use[q]: the lanes whose body q takes the entry (all lanes, except in the exact-set walk); a
// cell entry carries its masks as the bits of its third record's last two floats.
template <int LIST_CAP> struct CellList {
    float4 a[LIST_CAP], b[LIST_CAP], c[LIST_CAP];
};
template <int LIST_CAP> struct BodyList { float4 a[LIST_CAP]; unsigned use[2][LIST_CAP]; };

// Evaluation of a full list by the 32 lanes, each for its BPL bodies (entries read once as
// shared-memory broadcasts and used for every body of the lane).
// Accumulations of a masked entry: the lane adds only when its bit of the entry's use mask is
// set (tk != 0), as predicated FMAs under one predicate.
__device__ __forceinline__ void nb_acc_if(unsigned tk, float s, float dx, float dy, float dz,
                                          float& fx, float& fy, float& fz)
{
    asm("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %3, 0;\n\t"
        "@p fma.rn.f32 %0, %4, %5, %0;\n\t@p fma.rn.f32 %1, %4, %6, %1;\n\t"
        "@p fma.rn.f32 %2, %4, %7, %2;\n\t}"
        : "+f"(fx), "+f"(fy), "+f"(fz)
        : "r"(tk), "f"(s), "f"(dx), "f"(dy), "f"(dz));
}
// f += s d - dr5inv qd under the predicate (a masked cell's monopole and quadrupole terms)
__device__ __forceinline__ void nb_acc_quad_if(unsigned tk, float sr, float dx, float dy,
                                               float dz, float ndr5, float qx, float qy, float qz,
                                               float& fx, float& fy, float& fz)
{
    asm("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %3, 0;\n\t"
        "@p fma.rn.f32 %0, %8, %9, %0;\n\t@p fma.rn.f32 %0, %4, %5, %0;\n\t"
        "@p fma.rn.f32 %1, %8, %10, %1;\n\t@p fma.rn.f32 %1, %4, %6, %1;\n\t"
        "@p fma.rn.f32 %2, %8, %11, %2;\n\t@p fma.rn.f32 %2, %4, %7, %2;\n\t}"
        : "+f"(fx), "+f"(fy), "+f"(fz)
        : "r"(tk), "f"(sr), "f"(dx), "f"(dy), "f"(dz), "f"(ndr5), "f"(qx), "f"(qy), "f"(qz));
}

// MASKED (the exact-set walk): lanes outside an entry's use mask skip its accumulation.
template <int LIST_CAP, int BPL, bool MASKED>
__device__ __forceinline__ void nb_eval_bodies(const BodyList<LIST_CAP>& list, int n, int lane,
                                               const float (&rb)[BPL][3], float eps2,
                                               float (&f)[BPL][3])
{
    for (int e = 0; e < n; ++e) {
        const float4 a = list.a[e];
#pragma unroll
        for (int q = 0; q < BPL; ++q) {
            const float dx = a.x - rb[q][0], dy = a.y - rb[q][1], dz = a.z - rb[q][2];
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
            const float rinv = r2 > 0.f ? rsqrtf(r2) : 0.f;
            const float mor3 = a.w * rinv * rinv * rinv;
            if (MASKED) {
                nb_acc_if(list.use[q][e] & (1u << lane), mor3, dx, dy, dz, f[q][0], f[q][1],
                          f[q][2]);
            } else {
                f[q][0] = fmaf(mor3, dx, f[q][0]);
                f[q][1] = fmaf(mor3, dy, f[q][1]);
                f[q][2] = fmaf(mor3, dz, f[q][2]);
            }
        }
    }
}

template <int LIST_CAP, int BPL, bool MASKED>
__device__ __forceinline__ void nb_eval_cells(const CellList<LIST_CAP>& list, int n, int lane,
                                              const float (&rb)[BPL][3], float eps2, bool useQuad,
                                              float (&f)[BPL][3])
{
    for (int e = 0; e < n; ++e) {
        const float4 a = list.a[e];
        float4 b = make_float4(0.f, 0.f, 0.f, 0.f), c = b;
        if (useQuad) b = list.b[e];
        if (useQuad || MASKED) c = list.c[e];
#pragma unroll
        for (int q = 0; q < BPL; ++q) {
            const unsigned tk = MASKED ? __float_as_uint(q == 0 ? c.z : c.w) & (1u << lane) : 1u;
            const float dx = a.x - rb[q][0], dy = a.y - rb[q][1], dz = a.z - rb[q][2];
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, eps2)));
            const float rinv = rsqrtf(r2);
            const float rinv2 = rinv * rinv;
            const float rinv3 = rinv * rinv2;
            const float mor3 = a.w * rinv3;
            if (useQuad) {
                const float qxx = b.x, qxy = b.y, qxz = b.z, qyy = b.w, qyz = c.x, qzz = c.y;
                const float qdx = fmaf(qxz, dz, fmaf(qxy, dy, qxx * dx));
                const float qdy = fmaf(qyz, dz, fmaf(qyy, dy, qxy * dx));
                const float qdz = fmaf(qzz, dz, fmaf(qyz, dy, qxz * dx));
                const float drQdr = fmaf(qdz, dz, fmaf(qdy, dy, qdx * dx));
                const float dr5inv = rinv3 * rinv2;
                // the monopole's and the quadrupole's radial terms in one factor:
                // f += (m r^-3 + 2.5 (r.Q.r) r^-7) r - r^-5 Q.r
                const float sr = fmaf(2.5f * drQdr * rinv2, dr5inv, mor3);
                if (MASKED) {
                    nb_acc_quad_if(tk, sr, dx, dy, dz, -dr5inv, qdx, qdy, qdz, f[q][0], f[q][1],
                                   f[q][2]);
                } else {
                    f[q][0] = fmaf(sr, dx, fmaf(-dr5inv, qdx, f[q][0]));
                    f[q][1] = fmaf(sr, dy, fmaf(-dr5inv, qdy, f[q][1]));
                    f[q][2] = fmaf(sr, dz, fmaf(-dr5inv, qdz, f[q][2]));
                }
            } else if (MASKED) {
                nb_acc_if(tk, mor3, dx, dy, dz, f[q][0], f[q][1], f[q][2]);
            } else {
                f[q][0] = fmaf(mor3, dx, f[q][0]);
                f[q][1] = fmaf(mor3, dy, f[q][1]);
                f[q][2] = fmaf(mor3, dz, f[q][2]);
            }
        }
    }
}

// Walk groups: contiguous runs of <= G sorted bodies (G <= 64, the tuned group size).  Every
// cell with more than T = 32 G bodies lays out its direct children in octant order: a child
// with more than T bodies is descended by its own thread; a child with G < count <= T bodies
// is cut into runs of G consecutive sorted bodies (Morton order, so each run is compact and
// all runs but the last are full); consecutive children with <= G bodies (cells or single
// bodies) are packed into groups of <= G.  A root with <= T bodies is cut into runs of G; test
// particles (not in the tree, sorted last) form runs of G.  The groups partition the sorted
// bodies, and no group straddles two children of a cell with more than G bodies, so a group's
// box never spans octants of a large cell (such boxes open most of the tree).  Compared with
// packing only children of <= G bodies (T = G), the runs fill the warps better (95 % against
// 72 % of the lanes on a 1M-body Plummer dwarf at theta = 0.5) and cut the interaction work
// by 17 %, the most expensive group staying within 1.5 x the mean.
// With a forest every dwarf's root counts as a root.
__device__ __forceinline__ void nb_put_runs(int2* __restrict__ groups, NbScalars* __restrict__ sc,
                                            int first, int count, int G)
{
    for (int o = 0; o < count; o += G)
        groups[atomicAdd(&sc->nGroups, 1)] = make_int2(first + o, min(G, count - o));
}

__global__ void k_groups(const int2* __restrict__ nodeLink, const int2* __restrict__ nodeRange,
                         int2* __restrict__ groups, int n, NbScalars* __restrict__ sc, int G,
                         NbForest forest)
{
    if (nb_failed(sc)) return;
    const int nNodes = sc->nNodes, m = sc->nTree;
    const int T = 32 * G;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int c = tid; c < nNodes; c += stride) {
        const int2 l = nodeLink[c];
        if (l.y >= 0) continue;                              // bodies are handled by parents
        const int2 r = nodeRange[c];
        const int cnt = r.y - r.x + 1;
        if (cnt <= T) {
            const bool root = forest.dwarfs ? c == forest.dwarfs[forest.bodyDwarf[r.x]].rootNode
                                            : c == 0;
            if (root && cnt > 0) nb_put_runs(groups, sc, r.x, cnt, G);
            continue;
        }
        int gFirst = -1, gCount = 0;
        for (int k = c + 1; k < l.x; k = nodeLink[k].x) {
            const int2 rk = nodeRange[k];
            const int ck = rk.y - rk.x + 1;
            if (ck > G) {
                if (gCount) groups[atomicAdd(&sc->nGroups, 1)] = make_int2(gFirst, gCount);
                gCount = 0;
                if (ck <= T) nb_put_runs(groups, sc, rk.x, ck, G);   // else its own thread
                continue;
            }
            if (gCount && gCount + ck > G) {
                groups[atomicAdd(&sc->nGroups, 1)] = make_int2(gFirst, gCount);
                gCount = 0;
            }
            if (!gCount) gFirst = rk.x;
            gCount += ck;
        }
        if (gCount) groups[atomicAdd(&sc->nGroups, 1)] = make_int2(gFirst, gCount);
    }
    for (int t = tid; m + G * t < n; t += stride)
        groups[atomicAdd(&sc->nGroups, 1)] = make_int2(m + G * t, min(G, n - m - G * t));
}

// FOREST: a group belongs to one dwarf; its warp walks that dwarf's tree from its root,
// with the dwarf's softening and time step.  BPL: bodies per lane (groups of up to 32 BPL
// bodies; each lane walks for bodies lane and lane + 32).
template <bool COUNT, bool FOREST, int LIST_CAP, int BPL, bool EXACT>
__global__ void __launch_bounds__(GROUP_THREADS)
k_walk_mixed(const float4* __restrict__ nodeHi, const float4* __restrict__ nodeLo,
             const float4* __restrict__ nodeQ32, const int4* __restrict__ child8,
             const double4* __restrict__ nodePM, const unsigned int* __restrict__ order,
             const double* __restrict__ px, const double* __restrict__ py,
             const double* __restrict__ pz, const double* __restrict__ mass,
             double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
             int* __restrict__ stacks, const int2* __restrict__ groups, NbWalkParams wp,
             NbScalars* __restrict__ sc, NbForest forest)
{
    __shared__ CellList<LIST_CAP> sCells[GROUP_WARPS];
    __shared__ BodyList<LIST_CAP> sBodies[GROUP_WARPS];
    if (nb_failed(sc)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    CellList<LIST_CAP>& cells = sCells[warp];
    BodyList<LIST_CAP>& bodies = sBodies[warp];
    int* stack = stacks + (size_t) (blockIdx.x * GROUP_WARPS + warp) * (3 * NB_GROUP_STACK);
    // covered-lanes masks of every stack entry, one array per body slot
    unsigned* stackCover = reinterpret_cast<unsigned*>(stack + NB_GROUP_STACK);
    const unsigned ltMask = (1u << lane) - 1u;
    const int nGroups = sc->nGroups;
    double4 root = nodePM[0];
    float eps2 = (float) wp.eps2;
    int rootNode = 0;
    const bool useQuad = wp.useQuad != 0;
    const float inf = __int_as_float(0x7f800000);
    unsigned long long cVisit = 0, cBB = 0, cBC = 0, cSteps = 0;

    for (;;) {
        int g = 0;
        if (lane == 0) g = atomicAdd(&sc->groupNext, 1);
        g = __shfl_sync(NB_FULL_MASK, g, 0);
        if (g >= nGroups) break;
        const int2 grp = groups[g];
        if (FOREST) {
            const NbDwarfDev& dw = forest.dwarfs[forest.bodyDwarf[grp.x]];
            rootNode = dw.rootNode;
            root = nodePM[rootNode];
            eps2 = (float) dw.eps2;
        }
        bool valid[BPL];
        unsigned jb[BPL];
        float bh[BPL][3], bl[BPL][3];
        float mnx = inf, mny = inf, mnz = inf, mxx = -inf, mxy = -inf, mxz = -inf;
#pragma unroll
        for (int q = 0; q < BPL; ++q) {
            const int slot = lane + 32 * q;
            valid[q] = slot < grp.y;
            jb[q] = valid[q] ? order[grp.x + slot] : 0u;
            const double x0 = valid[q] ? px[jb[q]] : 0.0, y0 = valid[q] ? py[jb[q]] : 0.0;
            const double z0 = valid[q] ? pz[jb[q]] : 0.0;
            nb_split(x0 - root.x, bh[q][0], bl[q][0]);
            nb_split(y0 - root.y, bh[q][1], bl[q][1]);
            nb_split(z0 - root.z, bh[q][2], bl[q][2]);
            if (valid[q]) {
                const float X = bh[q][0] + bl[q][0], Y = bh[q][1] + bl[q][1], Z = bh[q][2] + bl[q][2];
                mnx = fminf(mnx, X); mny = fminf(mny, Y); mnz = fminf(mnz, Z);
                mxx = fmaxf(mxx, X); mxy = fmaxf(mxy, Y); mxz = fmaxf(mxz, Z);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fminf(mnx, __shfl_xor_sync(NB_FULL_MASK, mnx, o));
            mny = fminf(mny, __shfl_xor_sync(NB_FULL_MASK, mny, o));
            mnz = fminf(mnz, __shfl_xor_sync(NB_FULL_MASK, mnz, o));
            mxx = fmaxf(mxx, __shfl_xor_sync(NB_FULL_MASK, mxx, o));
            mxy = fmaxf(mxy, __shfl_xor_sync(NB_FULL_MASK, mxy, o));
            mxz = fmaxf(mxz, __shfl_xor_sync(NB_FULL_MASK, mxz, o));
        }
        const float cx = 0.5f * (mnx + mxx), cy = 0.5f * (mny + mxy), cz = 0.5f * (mnz + mxz);
        const float hx = 0.5f * (mxx - mnx), hy = 0.5f * (mxy - mny), hz = 0.5f * (mxz - mnz);
        // the bodies relative to the group centre
        float rb[BPL][3], f[BPL][3];
        double acc[BPL][3];
#pragma unroll
        for (int q = 0; q < BPL; ++q) {
            rb[q][0] = (bh[q][0] - cx) + bl[q][0];
            rb[q][1] = (bh[q][1] - cy) + bl[q][1];
            rb[q][2] = (bh[q][2] - cz) + bl[q][2];
            f[q][0] = f[q][1] = f[q][2] = 0.f;
            acc[q][0] = acc[q][1] = acc[q][2] = 0.0;
        }
        int nC = 0, nB = 0;
        // exact-set walk: lanes without a body count as covered from the start
        unsigned cover0[BPL];
#pragma unroll
        for (int q = 0; q < BPL; ++q) cover0[q] = ~__ballot_sync(NB_FULL_MASK, valid[q]);
        if (lane == 0) {
            stack[0] = rootNode;                 // the (dwarf's) root
            if (EXACT)
                for (int q = 0; q < BPL; ++q) stackCover[q * NB_GROUP_STACK] = cover0[q];
        }
        int top = 1;
        __syncwarp();
        while (top > 0) {
            const int take = min(32, top);
            const int base = top - take;
            const int k = lane < take ? stack[base + lane] : -1;
            // lanes that already took an ancestor of this node (exact-set walk)
            unsigned cover[BPL];
#pragma unroll
            for (int q = 0; q < BPL; ++q)
                cover[q] = EXACT && k >= 0 ? stackCover[q * NB_GROUP_STACK + base + lane] : 0u;
            top = base;
            float4 hi = make_float4(0.f, 0.f, 0.f, 0.f), lo = hi;
            bool isBody = false, accCell = false, openCell = false, boundary = false;
            if (k >= 0) {
                hi = nodeHi[k];
                lo = nodeLo[k];
                isBody = hi.w == -inf;          // bodies carry rcrit2 = -inf
                if (!isBody) {
                    const float ox = fabsf((hi.x + lo.x) - cx), oy = fabsf((hi.y + lo.y) - cy);
                    const float oz = fabsf((hi.z + lo.z) - cz);
                    const float ddx = fmaxf(ox - hx, 0.f);
                    const float ddy = fmaxf(oy - hy, 0.f);
                    const float ddz = fmaxf(oz - hz, 0.f);
                    const float d2 = fmaf(ddz, ddz, fmaf(ddy, ddy, ddx * ddx));
                    accCell = d2 >= hi.w;
                    openCell = !accCell;
                    if (EXACT && openCell) {
                        // some body of the group may still accept it: its farthest corner does
                        const float fx = ox + hx, fy = oy + hy, fz = oz + hz;
                        boundary = fmaf(fz, fz, fmaf(fy, fy, fx * fx)) >= hi.w;
                    }
                }
            }
            const float4 rel = make_float4((hi.x - cx) + lo.x, (hi.y - cy) + lo.y,
                                           (hi.z - cz) + lo.z, lo.w);
            // exact-set walk: use = the lanes that take this node.  An accepted cell or a body
            // is taken by every lane not yet covered; a cell the group opens is taken by the
            // lanes whose own body test (|CoM - x|^2 >= rcrit2, nbody/src/nbody_grav.c:58)
            // passes, and its subtree is then skipped for them -- each lane gets exactly its
            // body's interaction set.
            unsigned use[BPL];
            bool anyUse = false, allCovered = true;
#pragma unroll
            for (int q = 0; q < BPL; ++q) use[q] = EXACT && openCell ? 0u : ~cover[q];
            if (EXACT) {
                unsigned bm = __ballot_sync(NB_FULL_MASK, boundary);
                while (bm) {
                    const int j = __ffs(bm) - 1;
                    bm &= bm - 1;
                    const float qx = __shfl_sync(NB_FULL_MASK, rel.x, j);
                    const float qy = __shfl_sync(NB_FULL_MASK, rel.y, j);
                    const float qz = __shfl_sync(NB_FULL_MASK, rel.z, j);
                    const float rc2 = __shfl_sync(NB_FULL_MASK, hi.w, j);
#pragma unroll
                    for (int q = 0; q < BPL; ++q) {
                        const float ex = qx - rb[q][0], ey = qy - rb[q][1], ez = qz - rb[q][2];
                        const unsigned pass = __ballot_sync(
                            NB_FULL_MASK, fmaf(ez, ez, fmaf(ey, ey, ex * ex)) >= rc2);
                        if (lane == j) use[q] = pass & ~cover[q];
                    }
                }
#pragma unroll
                for (int q = 0; q < BPL; ++q) {
                    anyUse |= use[q] != 0u;
                    allCovered &= (cover[q] | use[q]) == 0xffffffffu;
                }
                if (openCell && allCovered) openCell = false;      // every body is covered
            }
            const bool addCell = accCell || (EXACT && boundary && anyUse);
            int4 c0 = make_int4(-1, -1, -1, -1), c1 = c0;
            const size_t cs = (size_t) __float_as_int(lo.w);     // a cell's slot
            if (openCell) { c0 = child8[2 * cs]; c1 = child8[2 * cs + 1]; }
            const unsigned bodyMask = __ballot_sync(NB_FULL_MASK, isBody);
            const unsigned cellMask = __ballot_sync(NB_FULL_MASK, addCell);
            if (COUNT) {
                ++cSteps;
                cVisit += 32ull * (unsigned) __popc(__ballot_sync(NB_FULL_MASK, k >= 0));
                cBB += 32ull * __popc(bodyMask);
                cBC += 32ull * __popc(cellMask);
            }
            if (nB + __popc(bodyMask) > LIST_CAP) {
                nb_eval_bodies<LIST_CAP, BPL, EXACT>(bodies, nB, lane, rb, eps2, f);
                nB = 0;
                __syncwarp();
                // near-field terms are large and cancel: add every list's partial sum into FP64
#pragma unroll
                for (int q = 0; q < BPL; ++q) {
                    acc[q][0] += (double) f[q][0]; acc[q][1] += (double) f[q][1];
                    acc[q][2] += (double) f[q][2];
                    f[q][0] = f[q][1] = f[q][2] = 0.f;
                }
            }
            if (nC + __popc(cellMask) > LIST_CAP) {
                nb_eval_cells<LIST_CAP, BPL, EXACT>(cells, nC, lane, rb, eps2, useQuad, f);
                nC = 0;
                __syncwarp();
#pragma unroll
                for (int q = 0; q < BPL; ++q) {
                    acc[q][0] += (double) f[q][0]; acc[q][1] += (double) f[q][1];
                    acc[q][2] += (double) f[q][2];
                    f[q][0] = f[q][1] = f[q][2] = 0.f;
                }
            }
            if (isBody) {
                const int e = nB + __popc(bodyMask & ltMask);
                bodies.a[e] = rel;
                if (EXACT)
                    for (int q = 0; q < BPL; ++q) bodies.use[q][e] = use[q];
            }
            if (addCell) {
                const int e = nC + __popc(cellMask & ltMask);
                const float4 qa = nodeQ32[2 * cs], qb = nodeQ32[2 * cs + 1];
                cells.a[e] = make_float4(rel.x, rel.y, rel.z, qb.z);   // the cell's mass
                cells.b[e] = qa;
                cells.c[e] = make_float4(qb.x, qb.y, EXACT ? __uint_as_float(use[0]) : 0.f,
                                         EXACT && BPL > 1 ? __uint_as_float(use[BPL - 1]) : 0.f);
            }
            nB += __popc(bodyMask);
            nC += __popc(cellMask);
            // push the children of opened cells (warp prefix sum of their counts)
            const int nch = (c0.x >= 0) + (c0.y >= 0) + (c0.z >= 0) + (c0.w >= 0) +
                            (c1.x >= 0) + (c1.y >= 0) + (c1.z >= 0) + (c1.w >= 0);
            int incl = nch;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(NB_FULL_MASK, incl, o);
                if (lane >= o) incl += u;
            }
            const int total = __shfl_sync(NB_FULL_MASK, incl, 31);
            if (top + total > NB_GROUP_STACK) {      // cannot happen (depth-sorted stack bound)
                if (lane == 0) nb_raise(sc, NBODY_CAPABILITY_ERROR);
                top = 0;
                break;
            }
            int w = top + incl - nch;
            const int cl[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
            for (int m = 0; m < 8; ++m)
                if (cl[m] >= 0) {
                    if (EXACT)
                        for (int q = 0; q < BPL; ++q)
                            stackCover[q * NB_GROUP_STACK + w] = cover[q] | use[q];
                    stack[w++] = cl[m];
                }
            top += total;
            __syncwarp();
        }
        __syncwarp();
        nb_eval_bodies<LIST_CAP, BPL, EXACT>(bodies, nB, lane, rb, eps2, f);
#pragma unroll
        for (int q = 0; q < BPL; ++q) {
            acc[q][0] += (double) f[q][0]; acc[q][1] += (double) f[q][1];
            acc[q][2] += (double) f[q][2];
            f[q][0] = f[q][1] = f[q][2] = 0.f;
        }
        nb_eval_cells<LIST_CAP, BPL, EXACT>(cells, nC, lane, rb, eps2, useQuad, f);
        __syncwarp();
#pragma unroll
        for (int q = 0; q < BPL; ++q) {
            if (!valid[q]) continue;
            const unsigned j = jb[q];
            // test particles are not in the tree and never meet themselves (nbody_grav.c:111-118)
            if (mass[j] == 0.0) atomicOr(&sc->incest, 1);
            // self-gravity only; k_body_epilogue adds the rest
            ax[j] = acc[q][0] + (double) f[q][0];
            ay[j] = acc[q][1] + (double) f[q][1];
            az[j] = acc[q][2] + (double) f[q][2];
        }
    }
    if (COUNT && lane == 0) {
        atomicAdd(&sc->nWarpSteps, cSteps);
        atomicAdd(&sc->nVisit, cVisit);
        atomicAdd(&sc->nBodyBody, cBB);
        atomicAdd(&sc->nBodyCell, cBC);
    }
}

template <bool COUNT, bool FOREST, int LC, int BPL>
static void nb_walk_mixed_launch(const NbTreeBuffers& b, const NbMixedBuffers& m,
                                 const NbWalkParams& wp, int blocks, const NbForest& f,
                                 cudaStream_t s)
{
    if (m.exact)
        k_walk_mixed<COUNT, FOREST, LC, BPL, true><<<blocks, GROUP_THREADS, 0, s>>>(
            m.hi, m.lo, m.q32, m.child8, b.nodePM, b.sort.idxA, b.px, b.py, b.pz, b.mass, b.ax,
            b.ay, b.az, m.stacks, m.groups, wp, b.sc, f);
    else
        k_walk_mixed<COUNT, FOREST, LC, BPL, false><<<blocks, GROUP_THREADS, 0, s>>>(
            m.hi, m.lo, m.q32, m.child8, b.nodePM, b.sort.idxA, b.px, b.py, b.pz, b.mass, b.ax,
            b.ay, b.az, m.stacks, m.groups, wp, b.sc, f);
}

template <bool COUNT, bool FOREST>
static void nb_walk_mixed_cap(const NbTreeBuffers& b, const NbMixedBuffers& m,
                              const NbWalkParams& wp, int blocks, const NbForest& f,
                              cudaStream_t s)
{
    if (m.groupMax > 32) {                    // two bodies per lane
        switch (m.listCap) {
        case 32: nb_walk_mixed_launch<COUNT, FOREST, 32, 2>(b, m, wp, blocks, f, s); break;
        case 128: nb_walk_mixed_launch<COUNT, FOREST, 128, 2>(b, m, wp, blocks, f, s); break;
        default: nb_walk_mixed_launch<COUNT, FOREST, 64, 2>(b, m, wp, blocks, f, s); break;
        }
        return;
    }
    switch (m.listCap) {
    case 32: nb_walk_mixed_launch<COUNT, FOREST, 32, 1>(b, m, wp, blocks, f, s); break;
    case 128: nb_walk_mixed_launch<COUNT, FOREST, 128, 1>(b, m, wp, blocks, f, s); break;
    default: nb_walk_mixed_launch<COUNT, FOREST, 64, 1>(b, m, wp, blocks, f, s); break;
    }
}

void nb_launch_body_epilogue(const double* px, const double* py, const double* pz, double* ax,
                             double* ay, double* az, double* vx, double* vy, double* vz,
                             const NbWalkParams& wp, const NbPot& pot, const NbScalars* sc,
                             int numSMs, cudaStream_t s, const NbForest* forest);

void nb_launch_walk_mixed(const NbTreeBuffers& b, const NbMixedBuffers& m, int capNodes,
                          const NbWalkParams& wp, const NbPot& pot, bool count, int numSMs,
                          cudaStream_t s, const NbForest* forest)
{
    const NbForest f = forest ? *forest : NbForest{nullptr, nullptr, 0};
    const int g = min((capNodes + 255) / 256, numSMs * 16);
    if (forest)
        k_pack_f32<true><<<g, 256, 0, s>>>(b.nodePM, b.nodeCrit, b.nodeLink, b.nodeQuad, m.hi, m.lo,
                                           m.q32, m.child8, b.nodeRange, b.sc, f);
    else
        k_pack_f32<false><<<g, 256, 0, s>>>(b.nodePM, b.nodeCrit, b.nodeLink, b.nodeQuad, m.hi, m.lo,
                                            m.q32, m.child8, b.nodeRange, b.sc, f);
    const int G = m.groupMax >= 1 && m.groupMax <= 64 ? m.groupMax : 32;
    k_groups<<<g, 256, 0, s>>>(b.nodeLink, b.nodeRange, m.groups, wp.n, b.sc, G, f);
    nb_count_launch(2);
    if (wp.n <= 0) return;
    const int blocks = m.walkBlocks;
    if (forest) {
        if (count) nb_walk_mixed_cap<true, true>(b, m, wp, blocks, f, s);
        else nb_walk_mixed_cap<false, true>(b, m, wp, blocks, f, s);
    } else {
        if (count) nb_walk_mixed_cap<true, false>(b, m, wp, blocks, f, s);
        else nb_walk_mixed_cap<false, false>(b, m, wp, blocks, f, s);
    }
    nb_count_launch();
    nb_launch_body_epilogue(b.px, b.py, b.pz, b.ax, b.ay, b.az, b.vx, b.vy, b.vz, wp, pot, b.sc,
                            numSMs, s, forest);
}

// Persistent grid of the group walk: as many blocks as fit on the device at once (for the
// given interaction-list capacity, 0 = the default of 64, and group size).
template <int LC, int BPL>
static int nb_walk_per_sm()
{
    // the fewer of the two variants' resident blocks, so one grid (and stack allocation)
    // serves both
    int perSM = 0, perSM2 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_walk_mixed<false, false, LC, BPL, false>,
                                                      GROUP_THREADS, 0) != cudaSuccess ||
        perSM < 1) {
        cudaGetLastError();
        perSM = 1;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &perSM2, k_walk_mixed<false, false, LC, BPL, true>, GROUP_THREADS, 0) != cudaSuccess ||
        perSM2 < 1) {
        cudaGetLastError();
        perSM2 = 1;
    }
    perSM = perSM2 < perSM ? perSM2 : perSM;
    return perSM;
}

int nb_mixed_walk_blocks(int numSMs, int listCap, int groupMax)
{
    int perSM;
    if (groupMax > 32)
        perSM = listCap == 32 ? nb_walk_per_sm<32, 2>() : listCap == 128 ? nb_walk_per_sm<128, 2>()
                                                                          : nb_walk_per_sm<64, 2>();
    else
        perSM = listCap == 32 ? nb_walk_per_sm<32, 1>() : listCap == 128 ? nb_walk_per_sm<128, 1>()
                                                                          : nb_walk_per_sm<64, 1>();
    return perSM * numSMs;
}

// per warp: the node stack and, beside it, the covered-lanes mask of every entry
size_t nb_mixed_stack_ints(int blocks) { return (size_t) blocks * GROUP_WARPS * 3 * NB_GROUP_STACK; }
