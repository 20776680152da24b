// Adjoint (vector-Jacobian product) of the force evaluation with the tree frozen.
//
// No reference counterpart: the reference has no adjoint.  Given the adjoint abar_i of every
// body's acceleration, computes xbar_j = sum_i abar_i . d a_i / d x_j and
// mbar_j = sum_i abar_i . d a_i / d m_j for the accelerations of the last force evaluation,
// keeping every opening decision of that evaluation (the tree is frozen).  Through the tree
// the accelerations depend on the bodies via the cell moments, so the adjoint has two parts:
//   1. k_walk_vjp: the same warp-union walk as k_walk_fp64 (nbody_grav.c:42-124); for every
//      interaction (body i, node q) it forms the tidal-tensor product
//          dbar_r = m (abar s^-3/2 - 3 r (r.abar) s^-5/2)   (+ quadrupole terms)
//      with r = x_q - x_i, s = |r|^2 + eps^2, subtracts it from body i and adds it, with the
//      node's mass and quadrupole adjoints, to node q (warp-reduced, one atomic per warp visit);
//      plus the Jacobian of the external potential at x_i (forward-mode dual numbers).
//   2. k_moments_vjp: top-down over depth levels, each cell hands its CoM / mass / quadrupole
//      adjoints to its children by differentiating hackCofM and hackQuad
//      (nbody/src/nbody_tree.c:70-121, 386-424).
// k_direct_vjp does the same for the Exact criterion (direct sum, nbody_grav.c:205-227).
#include "nb_common.cuh"

// ---- forward-mode dual numbers for the external potential's Jacobian ----
struct D3 {
    double v, dx, dy, dz;
};
__device__ __forceinline__ D3 dc(double c) { return {c, 0.0, 0.0, 0.0}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.v + b.v, a.dx + b.dx, a.dy + b.dy, a.dz + b.dz}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.v - b.v, a.dx - b.dx, a.dy - b.dy, a.dz - b.dz}; }
__device__ __forceinline__ D3 operator*(D3 a, D3 b)
{
    return {a.v * b.v, a.dx * b.v + a.v * b.dx, a.dy * b.v + a.v * b.dy, a.dz * b.v + a.v * b.dz};
}
__device__ __forceinline__ D3 operator*(double c, D3 a) { return {c * a.v, c * a.dx, c * a.dy, c * a.dz}; }
__device__ __forceinline__ D3 operator/(D3 a, D3 b)
{
    const double q = a.v / b.v, ib = 1.0 / b.v;
    return {q, (a.dx - q * b.dx) * ib, (a.dy - q * b.dy) * ib, (a.dz - q * b.dz) * ib};
}
__device__ __forceinline__ D3 dchain(D3 a, double f, double fp)
{
    return {f, fp * a.dx, fp * a.dy, fp * a.dz};
}
__device__ __forceinline__ D3 dsqrt(D3 a) { const double s = sqrt(a.v); return dchain(a, s, 0.5 / s); }
__device__ __forceinline__ D3 dpow15(D3 a) { const double s = sqrt(a.v); return dchain(a, a.v * s, 1.5 * s); }
__device__ __forceinline__ D3 dpow3(D3 a) { return dchain(a, a.v * a.v * a.v, 3.0 * a.v * a.v); }
__device__ __forceinline__ D3 dlog(D3 a) { return dchain(a, log(a.v), 1.0 / a.v); }

// nbExtAcceleration (nbody/src/nbody_potential.c:627-762) on dual numbers: value and gradient
// of each acceleration component.
__device__ void nb_ext_accel_dual(const NbPot& p, double x, double y, double z, D3& ox, D3& oy, D3& oz)
{
    const D3 X = {x, 1.0, 0.0, 0.0}, Y = {y, 0.0, 1.0, 0.0}, Z = {z, 0.0, 0.0, 1.0};
    const double limit = 0.00390625;
    const D3 absv = dsqrt(Z * Z + (Y * Y + X * X));
    const D3 r = absv.v > limit ? absv : dc(limit);
    D3 ax = dc(0.0), ay = dc(0.0), az = dc(0.0);
    for (int d = 0; d < 2; ++d) {
        const int type = d == 0 ? p.diskType : p.disk2Type;
        if (type != NBCUDA_MIYAMOTO_NAGAI_DISK) continue;
        const double M = d == 0 ? p.diskMass : p.disk2Mass;
        const double a = d == 0 ? p.diskA : p.disk2A, b = d == 0 ? p.diskB : p.disk2B;
        const D3 zp = dsqrt(Z * Z + dc(b * b));
        const D3 azp = dc(a) + zp;
        const D3 rth = dpow15(X * X + Y * Y + azp * azp);
        ax = ax + (-M) * X / rth;
        ay = ay + (-M) * Y / rth;
        az = az + (-M) * Z * azp / (zp * rth);
    }
    if (p.haloType == NBCUDA_LOGARITHMIC_HALO) {
        const double q = p.haloQz, dd = p.haloA, v0 = p.haloV;
        const D3 zq = Z / dc(q);
        const D3 denom = dc(dd * dd) + X * X + Y * Y + zq * zq;
        const D3 k = dc(-2.0 * v0 * v0) / denom;
        ax = ax + k * X;
        ay = ay + k * Y;
        az = az + k * Z / dc(q * q);
    } else if (p.haloType == NBCUDA_NFW_HALO) {
        const double a = p.haloA;
        const double M = p.haloV * p.haloV * a / 0.2162165954;
        const D3 ar = dc(a) + r;
        const D3 c = (dc(-M) / (r * r)) * (dlog(ar / dc(a)) / r - dc(1.0) / ar);
        ax = ax + c * X; ay = ay + c * Y; az = az + c * Z;
    }
    if (p.sphType == NBCUDA_HERNQUIST_SPHERICAL) {
        const D3 tmp = dc(p.sphScale) + r;
        const D3 c = dc(-p.sphMass) / (r * (tmp * tmp));
        ax = ax + c * X; ay = ay + c * Y; az = az + c * Z;
    } else if (p.sphType == NBCUDA_PLUMMER_SPHERICAL) {
        const D3 tmp = dsqrt(dc(p.sphScale * p.sphScale) + r * r);
        const D3 c = dc(-p.sphMass) / dpow3(tmp);
        ax = ax + c * X; ay = ay + c * Y; az = az + c * Z;
    }
    ox = ax; oy = ay; oz = az;
}

// xbar += J_ext(x)^T abar
__device__ __forceinline__ void nb_ext_vjp(const NbPot& pot, double x, double y, double z,
                                           double abx, double aby, double abz, double& gx,
                                           double& gy, double& gz)
{
    if (!pot.enabled) return;
    D3 ax, ay, az;
    nb_ext_accel_dual(pot, x, y, z, ax, ay, az);
    gx += abx * ax.dx + aby * ay.dx + abz * az.dx;
    gy += abx * ax.dy + aby * ay.dy + abz * az.dy;
    gz += abx * ax.dz + aby * ay.dz + abz * az.dz;
}

// d(a . abar)/d r, d/dm and d/dQ of one interaction a = m r s^-3/2 + quad(r, Q) with
// r = x_node - x_body, s = |r|^2 + eps^2 (the terms of nbGravity, nbody_grav.c:66-100).
struct Vjp1 {
    double rx, ry, rz, m, q[6];
};
__device__ __forceinline__ Vjp1 nb_interaction_vjp(double dx, double dy, double dz, double m,
                                                   double Q0, double Q1, double Q2, double Q3,
                                                   double Q4, double Q5, bool quad, double eps2,
                                                   double abx, double aby, double abz)
{
    Vjp1 o;
    const double s = dx * dx + dy * dy + dz * dz + eps2;
    const double rs = rsqrt(s);               // s^-1/2 (within 1 ulp)
    const double is = rs * rs;
    const double r3 = is * rs;                // s^-3/2
    const double r5 = r3 * is;                // s^-5/2
    const double al = dx * abx + dy * aby + dz * abz;
    o.rx = m * (abx * r3 - 3.0 * dx * al * r5);
    o.ry = m * (aby * r3 - 3.0 * dy * al * r5);
    o.rz = m * (abz * r3 - 3.0 * dz * al * r5);
    o.m = al * r3;
    for (int c = 0; c < 6; ++c) o.q[c] = 0.0;
    if (quad) {
        const double qxx = Q0, qxy = Q1, qxz = Q2, qyy = Q3, qyz = Q4, qzz = Q5;
        const double qdx = qxx * dx + qxy * dy + qxz * dz;
        const double qdy = qxy * dx + qyy * dy + qyz * dz;
        const double qdz = qxz * dx + qyz * dy + qzz * dz;
        const double qax = qxx * abx + qxy * aby + qxz * abz;
        const double qay = qxy * abx + qyy * aby + qyz * abz;
        const double qaz = qxz * abx + qyz * aby + qzz * abz;
        const double be = qdx * dx + qdy * dy + qdz * dz;            // r.Q.r
        const double ga = dx * qax + dy * qay + dz * qaz;            // r.Q.abar
        const double r7 = r5 * is;                                   // s^-7/2
        // a_q = 2.5 s^-7/2 (r.Q.r) r - s^-5/2 Q r
        const double c1 = 2.5 * r7;
        o.rx += c1 * (-7.0 * be * al * dx * is + 2.0 * al * qdx + be * abx) + 5.0 * r7 * ga * dx - r5 * qax;
        o.ry += c1 * (-7.0 * be * al * dy * is + 2.0 * al * qdy + be * aby) + 5.0 * r7 * ga * dy - r5 * qay;
        o.rz += c1 * (-7.0 * be * al * dz * is + 2.0 * al * qdz + be * abz) + 5.0 * r7 * ga * dz - r5 * qaz;
        o.q[0] = c1 * al * dx * dx - r5 * abx * dx;
        o.q[1] = c1 * al * 2.0 * dx * dy - r5 * (abx * dy + aby * dx);
        o.q[2] = c1 * al * 2.0 * dx * dz - r5 * (abx * dz + abz * dx);
        o.q[3] = c1 * al * dy * dy - r5 * aby * dy;
        o.q[4] = c1 * al * 2.0 * dy * dz - r5 * (aby * dz + abz * dy);
        o.q[5] = c1 * al * dz * dz - r5 * abz * dz;
    }
    return o;
}

// Sums V values (V a power of two, at most 32) over the warp by recursive halving: at each
// step a lane keeps half of its values and receives its partner's sums for that half, so the
// whole reduction takes V - 1 + log2(32 / V) shuffles instead of 5 V.  Afterwards the lanes
// L with L % (32 / V) == 0 hold the warp total of value L / (32 / V) in r[0].
template <int V>
__device__ __forceinline__ double nb_warp_sum_transposed(double (&r)[V], int lane)
{
#pragma unroll
    for (int w = V / 2, o = 16; w >= 1; w >>= 1, o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int t = 0; t < w; ++t) {
            const double send = up ? r[t] : r[t + w];
            const double keep = up ? r[t + w] : r[t];
            r[t] = keep + __shfl_xor_sync(NB_FULL_MASK, send, o);
        }
    }
#pragma unroll
    for (int o = 16 / V; o > 0; o >>= 1) r[0] += __shfl_xor_sync(NB_FULL_MASK, r[0], o);
    return r[0];
}

// Node adjoints: nodeBar[k*10 + 0..2] = CoM, [3] = mass, [4..9] = quadrupole.
// Seven resident blocks of 128 (72 registers, a few spilled): 28 warps per SM, so the
// 131,072-body dwarf's 4,096 warps run in one wave on 148 SMs (5 blocks, 96 registers: 1.4
// waves and a 6 % slower walk).
__global__ void __launch_bounds__(128, 7)
k_walk_vjp(const double4* __restrict__ rec,
           const unsigned int* __restrict__ order, const double* __restrict__ px,
           const double* __restrict__ py, const double* __restrict__ pz,
           const double* __restrict__ abar, double* __restrict__ xbar,
           double* __restrict__ nodeBar, NbWalkParams wp, NbPot pot, NbScalars* __restrict__ sc)
{
    if (nb_failed(sc)) return;
    const int end = sc->nNodes;
    const int lane = threadIdx.x & 31;
    const int i = (int) ((blockIdx.x * (unsigned) blockDim.x + threadIdx.x) >> 5) * 32 + lane;
    const bool valid = i < wp.n;
    const unsigned j = valid ? order[i] : 0u;
    const double x0 = valid ? px[j] : 0.0, y0 = valid ? py[j] : 0.0, z0 = valid ? pz[j] : 0.0;
    const double abx = valid ? abar[3 * j] : 0.0, aby = valid ? abar[3 * j + 1] : 0.0;
    const double abz = valid ? abar[3 * j + 2] : 0.0;
    const bool useQuad = wp.useQuad != 0;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    int ptr = valid ? 0 : end;
    for (;;) {
        const int q = __reduce_min_sync(NB_FULL_MASK, ptr);
        if (q >= end) break;
        const bool active = ptr == q;
        // the FP64 walk's packed record: {CoM, mass}, {rcrit2, links, Qxx, Qxy}, {Qxz .. Qzz}
        const double4 nd = nb_ld32(rec + 3 * (size_t) q);
        const double4 r1 = nb_ld32(rec + 3 * (size_t) q + 1);
        const long long word = __double_as_longlong(r1.y);
        const int2 link = make_int2((int) (unsigned) (word & 0xffffffffll), (int) (word >> 32));
        const bool isBody = link.y >= 0;
        bool inter = false;
        Vjp1 v;
        if (active) {
            const double dx = nd.x - x0, dy = nd.y - y0, dz = nd.z - z0;
            const double drSq = dz * dz + (dy * dy + dx * dx);
            if (isBody || drSq >= r1.x) {
                ptr = link.x;
                inter = !(isBody && (unsigned) link.y == j);
                if (inter) {
                    double4 r2 = make_double4(0.0, 0.0, 0.0, 0.0);
                    if (useQuad && !isBody) r2 = nb_ld32(rec + 3 * (size_t) q + 2);
                    v = nb_interaction_vjp(dx, dy, dz, nd.w, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w,
                                           useQuad && !isBody, wp.eps2, abx, aby, abz);
                    gx -= v.rx; gy -= v.ry; gz -= v.rz;
                }
            } else {
                ptr = q + 1;
            }
        }
        if (!inter) {
            v.rx = v.ry = v.rz = v.m = 0.0;
            for (int c = 0; c < 6; ++c) v.q[c] = 0.0;
        }
        const unsigned interMask = __ballot_sync(NB_FULL_MASK, inter);
        const bool cellQ = useQuad && !isBody;        // warp-uniform: q is the same node
        double* nb = nodeBar + 10 * (size_t) q;
        if (__popc(interMask) == 1) {
            // a single lane interacted: it adds its own terms, no reduction needed
            if (inter) {
                atomicAdd(nb + 0, v.rx); atomicAdd(nb + 1, v.ry); atomicAdd(nb + 2, v.rz);
                atomicAdd(nb + 3, v.m);
                if (cellQ)
                    for (int c = 0; c < 6; ++c) atomicAdd(nb + 4 + c, v.q[c]);
            }
        } else if (interMask && cellQ) {
            // ten values as eight plus two (14 shuffles, against 16 for ten padded to sixteen)
            double r8[8] = {v.rx, v.ry, v.rz, v.m, v.q[0], v.q[1], v.q[2], v.q[3]};
            double r2[2] = {v.q[4], v.q[5]};
            const double s8 = nb_warp_sum_transposed<8>(r8, lane);
            const double s2 = nb_warp_sum_transposed<2>(r2, lane);
            if ((lane & 3) == 0) atomicAdd(nb + (lane >> 2), s8);
            if ((lane & 15) == 0) atomicAdd(nb + 8 + (lane >> 4), s2);
        } else if (interMask) {
            double r[4] = {v.rx, v.ry, v.rz, v.m};
            const double sum = nb_warp_sum_transposed<4>(r, lane);
            if ((lane & 7) == 0) atomicAdd(nb + (lane >> 3), sum);
        }
    }
    if (!valid) return;
    nb_ext_vjp(pot, x0, y0, z0, abx, aby, abz, gx, gy, gz);
    xbar[3 * j] = gx; xbar[3 * j + 1] = gy; xbar[3 * j + 2] = gz;
}

// One depth level of the moment adjoint: every cell at depth D hands its adjoints to its
// children (hackQuad and hackCofM differentiated; children in octant order).
__global__ void k_moments_vjp(const double4* __restrict__ nodePM, const int2* __restrict__ nodeLink,
                              const int* __restrict__ nodeDepth, double* __restrict__ nodeBar,
                              int depth, int useQuad, const NbScalars* __restrict__ sc)
{
    const int nNodes = sc->nNodes;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nNodes; c += gridDim.x * blockDim.x) {
        const int2 l = nodeLink[c];
        if (l.y >= 0 || nodeDepth[c] != depth) continue;
        const double4 pc = nodePM[c];
        double* bc = nodeBar + 10 * (size_t) c;
        double ptx = bc[0], pty = bc[1], ptz = bc[2];
        const double mbar = bc[3];
        const double Qb[6] = {bc[4], bc[5], bc[6], bc[7], bc[8], bc[9]};
        // quadrupole: Q = sum_k m_k (3 d d^T - |d|^2 I) + Q_k, d = p_k - p
        for (int k = c + 1; k < l.x; k = nodeLink[k].x) {
            const double4 pk = nodePM[k];
            double* bk = nodeBar + 10 * (size_t) k;
            if (useQuad) {
                const double dx = pk.x - pc.x, dy = pk.y - pc.y, dz = pk.z - pc.z;
                const double gx = dx * (4.0 * Qb[0] - 2.0 * Qb[3] - 2.0 * Qb[5]) + 3.0 * (dy * Qb[1] + dz * Qb[2]);
                const double gy = dy * (4.0 * Qb[3] - 2.0 * Qb[0] - 2.0 * Qb[5]) + 3.0 * (dx * Qb[1] + dz * Qb[4]);
                const double gz = dz * (4.0 * Qb[5] - 2.0 * Qb[0] - 2.0 * Qb[3]) + 3.0 * (dx * Qb[2] + dy * Qb[4]);
                bk[0] += pk.w * gx; bk[1] += pk.w * gy; bk[2] += pk.w * gz;
                ptx -= pk.w * gx; pty -= pk.w * gy; ptz -= pk.w * gz;
                const double r2 = dx * dx + dy * dy + dz * dz;
                bk[3] += Qb[0] * (3.0 * dx * dx - r2) + Qb[1] * 3.0 * dx * dy + Qb[2] * 3.0 * dx * dz +
                         Qb[3] * (3.0 * dy * dy - r2) + Qb[4] * 3.0 * dy * dz + Qb[5] * (3.0 * dz * dz - r2);
                if (nodeLink[k].y < 0)
                    for (int q = 0; q < 6; ++q) bk[4 + q] += Qb[q];
            }
        }
        // centre of mass p = sum m_k p_k / M and mass M = sum m_k
        const double M = pc.w;
        for (int k = c + 1; k < l.x; k = nodeLink[k].x) {
            const double4 pk = nodePM[k];
            double* bk = nodeBar + 10 * (size_t) k;
            if (M != 0.0) {
                const double w = pk.w / M;
                bk[0] += w * ptx; bk[1] += w * pty; bk[2] += w * ptz;
                bk[3] += ((pk.x - pc.x) * ptx + (pk.y - pc.y) * pty + (pk.z - pc.z) * ptz) / M;
            }
            bk[3] += mbar;
        }
    }
}

// Body adjoints = walker part + the body's node adjoint (position, mass).
__global__ void k_vjp_finish(const int* __restrict__ bodyNode, const unsigned* __restrict__ order,
                             const double* __restrict__ nodeBar, double* __restrict__ xbar,
                             double* __restrict__ mbar, const NbScalars* __restrict__ sc, int n)
{
    const int m = sc->nTree;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned j = order[i];
        if (i < m) {
            const double* b = nodeBar + 10 * (size_t) bodyNode[i];
            xbar[3 * j] += b[0]; xbar[3 * j + 1] += b[1]; xbar[3 * j + 2] += b[2];
            if (mbar) mbar[j] = b[3];
        } else if (mbar) {
            mbar[j] = 0.0;
        }
    }
}

// Exact criterion: direct-sum adjoint.  Target j collects -dbar(j <- i) as the walker and
// +dbar(i <- j) as the source of every other body i, and the mass adjoint of its own mass.
constexpr int VJP_TILE = 128;
__global__ void __launch_bounds__(VJP_TILE)
k_direct_vjp(const double* __restrict__ px, const double* __restrict__ py,
             const double* __restrict__ pz, const double* __restrict__ mass,
             const double* __restrict__ abar, double* __restrict__ xbar, double* __restrict__ mbar,
             NbWalkParams wp, NbPot pot)
{
    __shared__ double4 tp[VJP_TILE];
    __shared__ double4 ta[VJP_TILE];
    const int n = wp.n;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = j < n;
    const double xj = valid ? px[j] : 0.0, yj = valid ? py[j] : 0.0, zj = valid ? pz[j] : 0.0;
    const double mj = valid ? mass[j] : 0.0;
    const double abx = valid ? abar[3 * j] : 0.0, aby = valid ? abar[3 * j + 1] : 0.0;
    const double abz = valid ? abar[3 * j + 2] : 0.0;
    double gx = 0.0, gy = 0.0, gz = 0.0, gm = 0.0;
    for (int base = 0; base < n; base += VJP_TILE) {
        const int k = base + threadIdx.x;
        __syncthreads();
        tp[threadIdx.x] = k < n ? make_double4(px[k], py[k], pz[k], mass[k]) : make_double4(0, 0, 0, 0);
        ta[threadIdx.x] = k < n ? make_double4(abar[3 * k], abar[3 * k + 1], abar[3 * k + 2], 0.0)
                                : make_double4(0, 0, 0, 0);
        __syncthreads();
        const int lim = min(VJP_TILE, n - base);
        for (int t = 0; t < lim; ++t) {
            const double4 b = tp[t];
            const double4 ab = ta[t];
            // j as the walker, source b: r = x_b - x_j
            const Vjp1 w = nb_interaction_vjp(b.x - xj, b.y - yj, b.z - zj, b.w, 0, 0, 0, 0, 0, 0,
                                              false, wp.eps2, abx, aby, abz);
            // j as the source of walker b: r = x_j - x_b
            const Vjp1 s = nb_interaction_vjp(xj - b.x, yj - b.y, zj - b.z, mj, 0, 0, 0, 0, 0, 0,
                                              false, wp.eps2, ab.x, ab.y, ab.z);
            gx += s.rx - w.rx; gy += s.ry - w.ry; gz += s.rz - w.rz;
            gm += s.m;
        }
    }
    if (!valid) return;
    nb_ext_vjp(pot, xj, yj, zj, abx, aby, abz, gx, gy, gz);
    xbar[3 * j] = gx; xbar[3 * j + 1] = gy; xbar[3 * j + 2] = gz;
    if (mbar) mbar[j] = gm;
}

// ---- host driver ----
void nb_launch_vjp(NbTreeBuffers& b, double* nodeBar, int capNodes, int maxDepth, int criterion,
                   const NbWalkParams& wp, const NbPot& pot, const double* abar, double* xbar,
                   double* mbar, int numSMs, cudaEvent_t walkStart, cudaEvent_t walkEnd,
                   cudaStream_t s)
{
    const int n = wp.n;
    if (n <= 0) return;
    if (criterion == NBCUDA_EXACT) {
        cudaEventRecord(walkStart, s);
        k_direct_vjp<<<(n + VJP_TILE - 1) / VJP_TILE, VJP_TILE, 0, s>>>(b.px, b.py, b.pz, b.mass, abar,
                                                                         xbar, mbar, wp, pot);
        cudaEventRecord(walkEnd, s);
        nb_count_launch();
        return;
    }
    cudaMemsetAsync(nodeBar, 0, 10 * sizeof(double) * (size_t) capNodes, s);
    const int warps = (n + 31) / 32;
    cudaEventRecord(walkStart, s);
    // packed records from the (possibly restored) tree arrays
    nb_launch_pack_walk(b.nodePM, b.nodeCrit, b.nodeLink, b.nodeQuad, b.walkRec, capNodes, b.sc, s);
    k_walk_vjp<<<(warps * 32 + 127) / 128, 128, 0, s>>>(b.walkRec, b.sort.idxA, b.px, b.py, b.pz,
                                                        abar, xbar, nodeBar, wp, pot, b.sc);
    cudaEventRecord(walkEnd, s);
    const int g = min((capNodes + 255) / 256, numSMs * 16);
    for (int d = 0; d <= maxDepth; ++d)
        k_moments_vjp<<<g, 256, 0, s>>>(b.nodePM, b.nodeLink, b.nodeDepth, nodeBar, d, wp.useQuad, b.sc);
    k_vjp_finish<<<min((n + 255) / 256, numSMs * 8), 256, 0, s>>>(b.bodyNode, b.sort.idxA, nodeBar,
                                                                    xbar, mbar, b.sc, n);
    nb_count_launch(3 + maxDepth);
}

// ---- reverse leapfrog step ----
// The forward step k (nbody/src/nbody_plain.c:329-364 with the kicks of
// nbody/src/nbody_grav.c:296-303): vh = v_k + h a_k, x_{k+1} = x_k + dt vh,
// a_{k+1} = A(x_{k+1}), v_{k+1} = vh + h a_{k+1}, h = dt / 2.  Given the adjoints (xbar, vbar)
// of (x_{k+1}, v_{k+1}) and abarNext, the adjoint a_{k+1} receives from step k+1's first kick,
// the reverse step is
//   abar = h vbar + abarNext;  (gx, gm) = VJP of A at x_{k+1} applied to abar
//   xbar += gx;  mbar += gm
//   dtbar += vbar . a_{k+1} / 2 + xbar . vh + (vbar + dt xbar) . a_k / 2
//   vbar += dt xbar;  abarNext = h vbar
__global__ void k_adj_pre(const double* __restrict__ vbar, const double* __restrict__ abarNext,
                          double* __restrict__ abar, double h, int n3)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
        abar[i] = h * vbar[i] + abarNext[i];
}

__global__ void __launch_bounds__(256)
k_adj_post(const double* __restrict__ ax, const double* __restrict__ ay,
           const double* __restrict__ az, const double* __restrict__ vx,
           const double* __restrict__ vy, const double* __restrict__ vz,
           const double* __restrict__ ak, const double* __restrict__ gx,
           const double* __restrict__ gm, double* __restrict__ xbar, double* __restrict__ vbar,
           double* __restrict__ mbar, double* __restrict__ abarNext, double* __restrict__ dtbar,
           double dt, int n)
{
    const double h = 0.5 * dt;
    double part = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double a1[3] = {ax[i], ay[i], az[i]};
        const double v1[3] = {vx[i], vy[i], vz[i]};
        for (int c = 0; c < 3; ++c) {
            const int k = 3 * i + c;
            const double vh = v1[c] - h * a1[c];
            const double xb = xbar[k] + gx[k];
            double vb = vbar[k];
            part += 0.5 * vb * a1[c] + xb * vh;
            vb += dt * xb;
            part += 0.5 * vb * ak[k];
            xbar[k] = xb;
            vbar[k] = vb;
            abarNext[k] = h * vb;
        }
        if (mbar) mbar[i] += gm[i];
    }
    // block sum of the time-step adjoint, one atomic per block
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(NB_FULL_MASK, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x < 32) {
        part = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(NB_FULL_MASK, part, o);
        if (threadIdx.x == 0 && dtbar) atomicAdd(dtbar, part);
    }
}

void nb_launch_step_adjoint(NbTreeBuffers& b, double* nodeBar, int capNodes, int maxDepth,
                            int criterion, const NbWalkParams& wp, const NbPot& pot, double dt,
                            const double* ak, double* xbar, double* vbar, double* mbar,
                            double* abarNext, double* dtbar, double* scratch, int numSMs,
                            cudaEvent_t walkStart, cudaEvent_t walkEnd, cudaStream_t s)
{
    const int n = wp.n;
    if (n <= 0) return;
    double* abar = scratch;                    // 3 n
    double* gx = scratch + 3 * (size_t) n;     // 3 n
    double* gm = scratch + 6 * (size_t) n;     // n
    const int blocks = min((3 * n + 255) / 256, numSMs * 8);
    k_adj_pre<<<blocks, 256, 0, s>>>(vbar, abarNext, abar, 0.5 * dt, 3 * n);
    nb_launch_vjp(b, nodeBar, capNodes, maxDepth, criterion, wp, pot, abar, gx, gm, numSMs,
                  walkStart, walkEnd, s);
    k_adj_post<<<min((n + 255) / 256, numSMs * 8), 256, 0, s>>>(
        b.ax, b.ay, b.az, b.vx, b.vy, b.vz, ak, gx, gm, xbar, vbar, mbar, abarNext, dtbar, dt, n);
    nb_count_launch(2);
}
