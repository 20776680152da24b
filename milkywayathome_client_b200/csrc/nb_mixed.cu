// Mixed-precision force walk (no counterpart in the reference).
//
// Same tree, same walk order and the same per-body opening test as the FP64 walk
// (nbGravity, nbody/src/nbody_grav.c:42-124), but the interaction arithmetic is FP32.
// After the FP64 moment pass, k_pack_f32 stores every node as FP32 data relative to the
// root's centre of mass c: position as an unevaluated sum hi + lo (hi = f32(x - c),
// lo = f32((x - c) - hi)), mass, rcrit2 and the quadrupole.  A lane forms
// dr = (hi_node - hi_body) + (lo_node - lo_body) in FP32: the hi difference is exact for
// nearby nodes (Sterbenz), so dr keeps FP32 relative precision however far the dwarf sits
// from the origin -- the walk runs in coordinates relative to the walking body's own
// neighbourhood.  Then |dr|^2, the softened inverse distance (rsqrtf), the monopole and
// quadrupole terms are FP32; partial sums are flushed into FP64 accumulators every
// NB_MIXED_FLUSH interactions.  Centres of mass, moments, the external potential and the
// leapfrog stay FP64 (shared with the FP64 code).  Compiled with -fmad=false like the FP64 code (so the shared FP64 epilogue keeps the
// reference's rounding); the FP32 interaction uses explicit fmaf.
#include "nb_common.cuh"
#include "nb_potential.cuh"

constexpr int MIXED_THREADS = 256;
constexpr int NB_MIXED_FLUSH = 16;

__device__ __forceinline__ void nb_split(double v, float& hi, float& lo)
{
    hi = __double2float_rn(v);
    lo = __double2float_rn(v - (double) hi);
}

// FP32 node records for the mixed walk (one pass over the nodes after the moments).
__global__ void k_pack_f32(const double4* __restrict__ nodePM, const double* __restrict__ nodeCrit,
                           const int2* __restrict__ nodeLink, const double* __restrict__ nodeQuad,
                           float4* __restrict__ nodeHi, float4* __restrict__ nodeLo,
                           float4* __restrict__ nodeQ32, const NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int nNodes = sc->nNodes;
    const double4 root = nodePM[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nNodes; k += gridDim.x * blockDim.x) {
        const double4 p = nodePM[k];
        float hx, hy, hz, lx, ly, lz;
        nb_split(p.x - root.x, hx, lx);
        nb_split(p.y - root.y, hy, ly);
        nb_split(p.z - root.z, hz, lz);
        const bool isBody = nodeLink[k].y >= 0;
        // bodies carry an rcrit2 of -inf, so the acceptance test needs no body branch
        const float crit = isBody ? __int_as_float(0xff800000) : __double2float_rn(nodeCrit[k]);
        nodeHi[k] = make_float4(hx, hy, hz, crit);
        nodeLo[k] = make_float4(lx, ly, lz, __double2float_rn(p.w));
        const double* Q = nodeQuad + 6 * (size_t) k;
        if (isBody) {
            nodeQ32[2 * (size_t) k] = make_float4(0.f, 0.f, 0.f, 0.f);
            nodeQ32[2 * (size_t) k + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            nodeQ32[2 * (size_t) k] = make_float4(__double2float_rn(Q[0]), __double2float_rn(Q[1]),
                                                  __double2float_rn(Q[2]), __double2float_rn(Q[3]));
            nodeQ32[2 * (size_t) k + 1] = make_float4(__double2float_rn(Q[4]), __double2float_rn(Q[5]), 0.f, 0.f);
        }
    }
}

template <bool COUNT>
__global__ void __launch_bounds__(MIXED_THREADS)
k_walk_mixed(const float4* __restrict__ nodeHi, const float4* __restrict__ nodeLo,
             const float4* __restrict__ nodeQ32, const int2* __restrict__ nodeLink,
             const double4* __restrict__ nodePM,
             const unsigned int* __restrict__ order, const double* __restrict__ px,
             const double* __restrict__ py, const double* __restrict__ pz,
             double* __restrict__ ax, double* __restrict__ ay, double* __restrict__ az,
             double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz,
             NbWalkParams wp, NbPot pot, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int end = sc->nNodes;
    const int lane = threadIdx.x & 31;
    const int i = (int) ((blockIdx.x * (unsigned) blockDim.x + threadIdx.x) >> 5) * 32 + lane;
    const bool valid = i < wp.n;
    const unsigned j = valid ? order[i] : 0u;
    const double x0 = valid ? px[j] : 0.0, y0 = valid ? py[j] : 0.0, z0 = valid ? pz[j] : 0.0;
    const double4 root = nodePM[0];
    float bhx, bhy, bhz, blx, bly, blz;
    nb_split(x0 - root.x, bhx, blx);
    nb_split(y0 - root.y, bhy, bly);
    nb_split(z0 - root.z, bhz, blz);
    const float eps2 = (float) wp.eps2;
    const bool useQuad = wp.useQuad != 0;
    int ptr = valid ? 0 : end;
    double accx = 0.0, accy = 0.0, accz = 0.0;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    int pending = 0;
    bool metSelf = false;
    unsigned long long cVisit = 0, cBB = 0, cBC = 0, cSteps = 0;
    for (;;) {
        const int q = __reduce_min_sync(NB_FULL_MASK, ptr);
        if (q >= end) break;
        if (COUNT) ++cSteps;
        if (ptr != q) continue;
        const float4 hi = nodeHi[q];
        const float4 lo = nodeLo[q];
        const int2 link = nodeLink[q];
        const float dx = (hi.x - bhx) + (lo.x - blx);
        const float dy = (hi.y - bhy) + (lo.y - bly);
        const float dz = (hi.z - bhz) + (lo.z - blz);
        float drSq = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        if (COUNT) ++cVisit;
        if (drSq >= hi.w) {        // bodies carry -inf: always accepted
            ptr = link.x;
            const bool isBody = link.y >= 0;
            if (isBody && (unsigned) link.y == j) { metSelf = true; continue; }
            if (COUNT) { if (isBody) ++cBB; else ++cBC; }
            drSq += eps2;
            const float rinv = rsqrtf(drSq);
            const float rinv2 = rinv * rinv;
            const float mor3 = lo.w * rinv * rinv2;
            fx = fmaf(mor3, dx, fx);
            fy = fmaf(mor3, dy, fy);
            fz = fmaf(mor3, dz, fz);
            if (useQuad && !isBody) {
                const float4 qa = nodeQ32[2 * (size_t) q];
                const float4 qb = nodeQ32[2 * (size_t) q + 1];
                const float qxx = qa.x, qxy = qa.y, qxz = qa.z, qyy = qa.w, qyz = qb.x, qzz = qb.y;
                const float qdx = fmaf(qxz, dz, fmaf(qxy, dy, qxx * dx));
                const float qdy = fmaf(qyz, dz, fmaf(qyy, dy, qxy * dx));
                const float qdz = fmaf(qzz, dz, fmaf(qyz, dy, qxz * dx));
                const float drQdr = fmaf(qdz, dz, fmaf(qdy, dy, qdx * dx));
                const float dr5inv = rinv2 * rinv2 * rinv;
                const float phiQ = 2.5f * dr5inv * drQdr * rinv2;
                fx = fmaf(phiQ, dx, fmaf(-dr5inv, qdx, fx));
                fy = fmaf(phiQ, dy, fmaf(-dr5inv, qdy, fy));
                fz = fmaf(phiQ, dz, fmaf(-dr5inv, qdz, fz));
            }
            if (++pending == NB_MIXED_FLUSH) {
                accx += (double) fx; accy += (double) fy; accz += (double) fz;
                fx = fy = fz = 0.f;
                pending = 0;
            }
        } else {
            ptr = q + 1;
        }
    }
    accx += (double) fx; accy += (double) fy; accz += (double) fz;
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
    if (!metSelf) atomicOr(&sc->incest, 1);
    nb_finish_body(pot, wp, j, x0, y0, z0, accx, accy, accz, ax, ay, az, vx, vy, vz);
}

void nb_launch_walk_mixed(const NbTreeBuffers& b, const NbMixedBuffers& m, int capNodes,
                          const NbWalkParams& wp, const NbPot& pot, bool count, int numSMs,
                          cudaStream_t s)
{
    k_pack_f32<<<min((capNodes + 255) / 256, numSMs * 16), 256, 0, s>>>(
        b.nodePM, b.nodeCrit, b.nodeLink, b.nodeQuad, m.hi, m.lo, m.q32, b.sc);
    nb_count_launch();
    const int warps = (wp.n + 31) / 32;
    const int blocks = (warps * 32 + MIXED_THREADS - 1) / MIXED_THREADS;
    if (blocks <= 0) return;
    if (count)
        k_walk_mixed<true><<<blocks, MIXED_THREADS, 0, s>>>(m.hi, m.lo, m.q32, b.nodeLink, b.nodePM,
                                                            b.sort.idxA, b.px, b.py, b.pz, b.ax, b.ay,
                                                            b.az, b.vx, b.vy, b.vz, wp, pot, b.sc);
    else
        k_walk_mixed<false><<<blocks, MIXED_THREADS, 0, s>>>(m.hi, m.lo, m.q32, b.nodeLink, b.nodePM,
                                                             b.sort.idxA, b.px, b.py, b.pz, b.ax, b.ay,
                                                             b.az, b.vx, b.vy, b.vz, wp, pot, b.sc);
    nb_count_launch();
}
