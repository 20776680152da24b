// Mixed-precision force walk (no counterpart in the reference).
//
// Same tree, same walk order and the same per-body opening test as the FP64 walk
// (nbGravity, nbody/src/nbody_grav.c:42-124), but the interaction arithmetic is FP32:
// each lane forms dr = node - body in FP64 (the separation is small next to the absolute
// coordinates, so it is exact to FP32 precision after conversion: the walk runs in
// coordinates relative to the walking body's own leaf), then evaluates |dr|^2, the
// softened inverse distance (rsqrtf), the monopole and quadrupole terms in FP32.  Partial
// sums are flushed into FP64 accumulators every NB_MIXED_FLUSH interactions.  Centres of
// mass, moments, the external potential and the leapfrog stay FP64 (they share the FP64
// code).  Compiled with -fmad=false like the FP64 code (so the shared FP64 epilogue keeps the
// reference's rounding); the FP32 interaction uses explicit fmaf.
#include "nb_common.cuh"
#include "nb_potential.cuh"

constexpr int MIXED_THREADS = 256;
constexpr int NB_MIXED_FLUSH = 16;

template <bool COUNT>
__global__ void __launch_bounds__(MIXED_THREADS)
k_walk_mixed(const double4* __restrict__ nodePM, const double* __restrict__ nodeCrit,
             const int2* __restrict__ nodeLink, const double* __restrict__ nodeQuad,
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
    const float eps2 = (float) wp.eps2;
    const bool useQuad = wp.useQuad != 0;
    int ptr = valid ? 0 : end;
    double accx = 0.0, accy = 0.0, accz = 0.0;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    int pending = 0;
    bool metSelf = false;
    unsigned long long cVisit = 0, cBB = 0, cBC = 0;
    for (;;) {
        const int q = __reduce_min_sync(NB_FULL_MASK, ptr);
        if (q >= end) break;
        if (ptr != q) continue;
        const double4 nd = nodePM[q];
        const int2 link = nodeLink[q];
        const float dx = (float) (nd.x - x0), dy = (float) (nd.y - y0), dz = (float) (nd.z - z0);
        float drSq = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        const bool isBody = link.y >= 0;
        if (COUNT) ++cVisit;
        if (isBody || drSq >= (float) nodeCrit[q]) {
            ptr = link.x;
            if (isBody && (unsigned) link.y == j) { metSelf = true; continue; }
            if (COUNT) { if (isBody) ++cBB; else ++cBC; }
            drSq += eps2;
            const float rinv = rsqrtf(drSq);
            const float rinv2 = rinv * rinv;
            const float mor3 = (float) nd.w * rinv * rinv2;
            fx = fmaf(mor3, dx, fx);
            fy = fmaf(mor3, dy, fy);
            fz = fmaf(mor3, dz, fz);
            if (useQuad && !isBody) {
                const double2* Q2 = reinterpret_cast<const double2*>(nodeQuad + 6 * (size_t) q);
                const double2 q01 = Q2[0], q23 = Q2[1], q45 = Q2[2];
                const float qxx = (float) q01.x, qxy = (float) q01.y, qxz = (float) q23.x;
                const float qyy = (float) q23.y, qyz = (float) q45.x, qzz = (float) q45.y;
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
            atomicAdd(&sc->nVisit, cVisit);
            atomicAdd(&sc->nBodyBody, cBB);
            atomicAdd(&sc->nBodyCell, cBC);
        }
    }
    if (!valid) return;
    if (!metSelf) atomicOr(&sc->incest, 1);
    nb_finish_body(pot, wp, j, x0, y0, z0, accx, accy, accz, ax, ay, az, vx, vy, vz);
}

void nb_launch_walk_mixed(const double4* nodePM, const double* nodeCrit, const int2* nodeLink,
                          const double* nodeQuad, const unsigned* order, const double* px,
                          const double* py, const double* pz, double* ax, double* ay, double* az,
                          double* vx, double* vy, double* vz, const NbWalkParams& wp,
                          const NbPot& pot, NbScalars* sc, bool count, cudaStream_t s)
{
    const int warps = (wp.n + 31) / 32;
    const int blocks = (warps * 32 + MIXED_THREADS - 1) / MIXED_THREADS;
    if (blocks <= 0) return;
    if (count)
        k_walk_mixed<true><<<blocks, MIXED_THREADS, 0, s>>>(nodePM, nodeCrit, nodeLink, nodeQuad, order,
                                                            px, py, pz, ax, ay, az, vx, vy, vz, wp, pot, sc);
    else
        k_walk_mixed<false><<<blocks, MIXED_THREADS, 0, s>>>(nodePM, nodeCrit, nodeLink, nodeQuad, order,
                                                             px, py, pz, ax, ay, az, vx, vy, vz, wp, pot, sc);
    nb_count_launch();
}
