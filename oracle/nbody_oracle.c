/*
 * nbody_oracle.c -- CPU restatement of the reference N-body client's Barnes-Hut step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the GPU library is checked against
 * (tests/, __graft_entry__.smoke() and bench.py's CPU baseline); the product never links,
 * loads or calls it.  It restates, in plain C and in the reference's own operation order
 * (no FMA contraction: build with -ffp-contract=off), the functions of the reference's CPU
 * path, each citing the file:line it follows:
 *
 *   or_make_tree     nbMakeTree           nbody/src/nbody_tree.c:429-460
 *                    (expandBox :156-176, nbLoadBody :242-282, nbSubIndex :36-52,
 *                     calcOffset/nbInitMidpoint :226-239, hackCofM :386-424,
 *                     findRCrit :308-343, nbCheckTreeStructure :345-380,
 *                     threadTree :127-150, hackQuad :70-121)
 *   or_gravity       nbGravity            nbody/src/nbody_grav.c:42-124
 *   or_gravity_exact nbGravity_Exact      nbody/src/nbody_grav.c:205-227
 *   or_ext_accel     nbExtAcceleration    nbody/src/nbody_potential.c:627-762
 *   or_grav_map      nbGravMap            nbody/src/nbody_grav.c:305-328
 *   or_step          nbStepSystemPlain    nbody/src/nbody_plain.c:251-364
 *
 * Parity pins: tests/test_oracle_ref.py checks every function here against the reference
 * itself, compiled from its sources by oracle/ref.mk (bit-for-bit on trees, accelerations
 * and trajectories), and that build against the reference's golden likelihoods
 * (nbody/tests/RunTestUnits.lua).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/nbody_b200.h"

/* ---- correctly rounded powers (crlibm pow_rn, milkyway_math_double.h:43-59) ----
 * x^1.5 and x^3 as double-double values rounded once (error-free products with fma). */
double or_pow_1p5(double x)
{
    double s, r, t, hi, lo;
    if (!(x > 0.0) || isinf(x)) {
        if (x == 0.0) return 0.0;
        return (isinf(x) && x > 0.0) ? x : NAN;
    }
    s = sqrt(x);
    r = fma(-s, s, x);
    t = r / (2.0 * s);
    hi = x * s;
    lo = fma(x, s, -hi);
    lo = lo + x * t;
    return hi + lo;
}

double or_pow_3(double x)
{
    double sq = x * x;
    double e1 = fma(x, x, -sq);
    double hi = sq * x;
    double lo = fma(sq, x, -hi);
    lo = lo + e1 * x;
    if (isinf(hi) || hi == 0.0) return hi;
    return hi + lo;
}

/* ---- correctly rounded log (crlibm log_rn, the reference's mw_log) ----
 * x = m 2^e with m in [1/sqrt(2), sqrt(2)); log(m) = 2 atanh(u), u = (m-1)/(m+1), by the
 * series sum u^(2k+1)/(2k+1) (|u| <= 0.1716, k = 0..21) in double-double arithmetic (values
 * hi + lo; error-free sums and fma products), plus e ln(2); rounded once. */
typedef struct { double hi, lo; } OrDD;

static OrDD or_dd(double hi, double lo) { OrDD r; r.hi = hi; r.lo = lo; return r; }

static OrDD or_sum(double a, double b)              /* exact: s + e = a + b */
{
    double s = a + b, bb = s - a;
    return or_dd(s, (a - (s - bb)) + (b - bb));
}

static OrDD or_fast_sum(double a, double b)         /* exact for |a| >= |b| */
{
    double s = a + b;
    return or_dd(s, b - (s - a));
}

static OrDD or_add(OrDD a, OrDD b)
{
    OrDD s = or_sum(a.hi, b.hi), t = or_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = or_fast_sum(s.hi, s.lo);
    s.lo += t.lo;
    return or_fast_sum(s.hi, s.lo);
}

static OrDD or_mul(OrDD a, OrDD b)
{
    double p = a.hi * b.hi;
    double e = fma(a.hi, b.hi, -p);
    e += a.hi * b.lo + a.lo * b.hi;
    return or_fast_sum(p, e);
}

static OrDD or_div(OrDD a, OrDD b)
{
    double q1 = a.hi / b.hi, q2, q3;
    OrDD r = or_add(a, or_mul(b, or_dd(-q1, 0.0)));
    q2 = r.hi / b.hi;
    r = or_add(r, or_mul(b, or_dd(-q2, 0.0)));
    q3 = r.hi / b.hi;
    return or_add(or_fast_sum(q1, q2), or_dd(q3, 0.0));
}

double or_log_rn(double x)
{
    int e = 0, k;
    double m, f;
    OrDD u, u2, s, lm, el;
    if (!(x > 0.0) || isinf(x)) return log(x);
    if (x == 1.0) return 0.0;
    m = frexp(x, &e);
    if (m < 0.70710678118654752440) { m *= 2.0; e -= 1; }
    f = m - 1.0;
    u = or_div(or_dd(f, 0.0), or_sum(m, 1.0));
    u2 = or_mul(u, u);
    s = or_dd(0.0, 0.0);
    for (k = 21; k >= 0; --k) {
        const double n = 2.0 * k + 1.0, c = 1.0 / n;   /* 1/n = c + (1 - c n)/n */
        s = or_add(or_mul(s, u2), or_dd(c, fma(-c, n, 1.0) / n));
    }
    lm = or_mul(u, s);
    lm.hi *= 2.0; lm.lo *= 2.0;
    /* ln 2 = 0.6931471805599453094172321214581765680755... */
    el = or_mul(or_dd(6.93147180559945286227e-01, 2.31904681384629955842e-17), or_dd((double) e, 0.0));
    lm = or_add(el, lm);
    return lm.hi + lm.lo;
}

/* ---- external potential: nbExtAcceleration (nbody_potential.c:627-762) ---- */
static void or_mn_disk(double M, double a, double b, double x, double y, double z, double* o)
{   /* miyamotoNagaiDiskAccel, nbody_potential.c:173-194 */
    const double zp = sqrt(z * z + b * b);
    const double azp = a + zp;
    const double rp = x * x + y * y + azp * azp;
    const double rth = or_pow_1p5(rp);
    o[0] = -M * x / rth;
    o[1] = -M * y / rth;
    o[2] = -M * z * azp / (zp * rth);
}

void or_ext_accel_one(const NBodyCudaPotential* p, const double* pos, double* out)
{
    const double x = pos[0], y = pos[1], z = pos[2];
    const double absv = sqrt(z * z + (y * y + x * x));
    const double limit = 0.00390625;
    const double r = (double) (absv <= limit) * limit + (double) (absv > limit) * absv;
    double acc[3] = { 0.0, 0.0, 0.0 }, t[3];
    if (p->disk.type == NBCUDA_MIYAMOTO_NAGAI_DISK)
        or_mn_disk(p->disk.mass, p->disk.scaleLength, p->disk.scaleHeight, x, y, z, acc);
    t[0] = t[1] = t[2] = 0.0;
    if (p->disk2.type == NBCUDA_MIYAMOTO_NAGAI_DISK)
        or_mn_disk(p->disk2.mass, p->disk2.scaleLength, p->disk2.scaleHeight, x, y, z, t);
    acc[0] = acc[0] + t[0]; acc[1] = acc[1] + t[1]; acc[2] = acc[2] + t[2];
    t[0] = t[1] = t[2] = 0.0;
    if (p->halo.type == NBCUDA_LOGARITHMIC_HALO) {   /* logHaloAccel, :488-504 */
        const double v0 = p->halo.vhalo, q = p->halo.flattenZ, d = p->halo.scaleLength;
        const double zq = z / q;
        const double denom = d * d + x * x + y * y + zq * zq;
        const double k = -2.0 * v0 * v0 / denom;
        t[0] = k * x; t[1] = k * y; t[2] = k * z / (q * q);
    } else if (p->halo.type == NBCUDA_NFW_HALO) {    /* nfwHaloAccel, :506-515 */
        const double a = p->halo.scaleLength;
        const double M = p->halo.vhalo * p->halo.vhalo * a / 0.2162165954;
        const double ar = a + r;
        const double c = (-M / (r * r)) * (or_log_rn(ar / a) / r - 1 / ar);
        t[0] = c * x; t[1] = c * y; t[2] = c * z;
    }
    acc[0] = acc[0] + t[0]; acc[1] = acc[1] + t[1]; acc[2] = acc[2] + t[2];
    t[0] = t[1] = t[2] = 0.0;
    if (p->sphere.type == NBCUDA_HERNQUIST_SPHERICAL) {   /* hernquistSphericalAccel, :157-162 */
        const double tmp = p->sphere.scale + r;
        const double c = -p->sphere.mass / (r * (tmp * tmp));
        t[0] = c * x; t[1] = c * y; t[2] = c * z;
    } else if (p->sphere.type == NBCUDA_PLUMMER_SPHERICAL) {   /* plummerSphericalAccel, :164-169 */
        const double tmp = sqrt(p->sphere.scale * p->sphere.scale + r * r);
        const double c = -p->sphere.mass / or_pow_3(tmp);
        t[0] = c * x; t[1] = c * y; t[2] = c * z;
    }
    acc[0] = acc[0] + t[0]; acc[1] = acc[1] + t[1]; acc[2] = acc[2] + t[2];
    out[0] = acc[0]; out[1] = acc[1]; out[2] = acc[2];
}

void or_ext_accel(const NBodyCudaPotential* p, const double* pos, double* acc, int n)
{
    int i;
    for (i = 0; i < n; ++i) or_ext_accel_one(p, pos + 3 * i, acc + 3 * i);
}

/* ---- tree ---- */
typedef struct {
    double pos[3];      /* geometric centre, then centre of mass */
    double mass;
    double rcrit2;
    double quad[6];
    int sub[8];         /* children: >= 0 cell index, <= -2 body (-2 - index), -1 empty */
    int next, more;     /* threaded links as node codes (see or_code) */
    int depth;
} OrCell;

typedef struct {
    OrCell* cells;
    int nCells, cap;
    double rsize;
    int maxDepth;
    int structureError;
} OrTree;

#define OR_EMPTY (-1)
#define OR_BODY(i) (-2 - (i))
#define OR_IS_BODY(c) ((c) <= -2)
#define OR_BODY_INDEX(c) (-2 - (c))
#define OR_NULL (-1)

static int or_new_cell(OrTree* t)
{
    OrCell* c;
    if (t->nCells == t->cap) {
        t->cap = t->cap ? 2 * t->cap : 1024;
        t->cells = (OrCell*) realloc(t->cells, sizeof(OrCell) * (size_t) t->cap);
    }
    c = &t->cells[t->nCells];
    memset(c, 0, sizeof *c);
    memset(c->sub, 0xff, sizeof c->sub);
    c->next = c->more = OR_NULL;
    return t->nCells++;
}

static int or_sub_index(const double* p, const double* q)
{   /* nbSubIndex, nbody_tree.c:36-52 */
    int ind = 0;
    if (q[0] <= p[0]) ind += 4;
    if (q[1] <= p[1]) ind += 2;
    if (q[2] <= p[2]) ind += 1;
    return ind;
}

static void or_load_body(OrTree* t, const double* pos, int i)
{   /* nbLoadBody, nbody_tree.c:242-282 */
    int q = 0, qind, lev = 0;
    double qsize = t->rsize;
    qind = or_sub_index(pos + 3 * i, t->cells[q].pos);
    while (t->cells[q].sub[qind] != OR_EMPTY) {
        if (qsize <= DBL_EPSILON) {
            t->structureError = 1;
            return;
        }
        if (OR_IS_BODY(t->cells[q].sub[qind])) {
            const int other = OR_BODY_INDEX(t->cells[q].sub[qind]);
            const int c = or_new_cell(t);
            int k;
            for (k = 0; k < 3; ++k) {   /* calcOffset, nbody_tree.c:227-231 */
                const double pp = pos[3 * i + k], qp = t->cells[q].pos[k];
                t->cells[c].pos[k] = qp + 0.25 * (pp < qp ? -qsize : qsize);
            }
            t->cells[c].depth = lev + 1;
            t->cells[c].sub[or_sub_index(pos + 3 * other, t->cells[c].pos)] = OR_BODY(other);
            t->cells[q].sub[qind] = c;
        }
        q = t->cells[q].sub[qind];
        qind = or_sub_index(pos + 3 * i, t->cells[q].pos);
        qsize *= 0.5;
        ++lev;
    }
    t->cells[q].sub[qind] = OR_BODY(i);
    if (lev > t->maxDepth) t->maxDepth = lev;
}

static double or_find_rcrit2(const NBodyCudaCtx* ctx, const double* geo, const double* cm,
                             double psize, double rsize)
{   /* findRCrit, nbody_tree.c:308-343 */
    double rc, bmax2, dmin, b;
    int k;
    if (ctx->theta == 0.0) {
        rc = 2.0 * rsize;
        return rc * rc;
    }
    switch (ctx->criterion) {
    case NBCUDA_TREECODE: {
        const double dx = cm[0] - geo[0], dy = cm[1] - geo[1], dz = cm[2] - geo[2];
        rc = psize / ctx->theta + sqrt(dx * dx + dy * dy + dz * dz);
        return rc * rc;
    }
    case NBCUDA_SW93:
        bmax2 = 0.0;
        for (k = 0; k < 3; ++k) {
            dmin = cm[k] - (geo[k] - 0.5 * psize);
            b = fmax(dmin, psize - dmin);
            bmax2 = k == 0 ? b * b : bmax2 + b * b;
        }
        return bmax2 / (ctx->theta * ctx->theta);
    case NBCUDA_BH86:
        rc = psize / ctx->theta;
        return rc * rc;
    default:
        return 0.0;
    }
}

static void or_cofm(const NBodyCudaCtx* ctx, OrTree* t, const double* pos, const double* mass,
                    int p, double psize)
{   /* hackCofM, nbody_tree.c:386-424 */
    double cm[3] = { 0.0, 0.0, 0.0 }, M = 0.0, h;
    int i, k;
    for (i = 0; i < 8; ++i) {
        const int q = t->cells[p].sub[i];
        const double* qp;
        double qm;
        if (q == OR_EMPTY) continue;
        if (OR_IS_BODY(q)) {
            qp = pos + 3 * OR_BODY_INDEX(q);
            qm = mass[OR_BODY_INDEX(q)];
        } else {
            or_cofm(ctx, t, pos, mass, q, 0.5 * psize);
            qp = t->cells[q].pos;
            qm = t->cells[q].mass;
        }
        M = M + qm;
        for (k = 0; k < 3; ++k) cm[k] = cm[k] + qm * qp[k];
    }
    if (M > 0.0) { for (k = 0; k < 3; ++k) cm[k] = cm[k] / M; }
    else { for (k = 0; k < 3; ++k) cm[k] = t->cells[p].pos[k]; }
    h = 0.5 * psize;   /* nbCheckTreeStructure, nbody_tree.c:345-380 */
    for (k = 0; k < 3; ++k)
        if (cm[k] < t->cells[p].pos[k] - h || cm[k] > t->cells[p].pos[k] + h) t->structureError = 1;
    t->cells[p].mass = M;
    t->cells[p].rcrit2 = or_find_rcrit2(ctx, t->cells[p].pos, cm, psize, t->rsize);
    for (k = 0; k < 3; ++k) t->cells[p].pos[k] = cm[k];
}

/* Node codes for threaded links: cells are >= 0, bodies OR_BODY(i), end OR_NULL. */
static void or_thread(OrTree* t, int p, int n, int* bodyNext)
{   /* threadTree, nbody_tree.c:127-150 */
    int desc[9], nd = 0, i;
    if (OR_IS_BODY(p)) { bodyNext[OR_BODY_INDEX(p)] = n; return; }
    t->cells[p].next = n;
    for (i = 0; i < 8; ++i)
        if (t->cells[p].sub[i] != OR_EMPTY) desc[nd++] = t->cells[p].sub[i];
    t->cells[p].more = nd ? desc[0] : OR_NULL;
    desc[nd] = n;
    for (i = 0; i < nd; ++i) or_thread(t, desc[i], desc[i + 1], bodyNext);
}

static void or_quad(OrTree* t, const double* pos, const double* mass, int p)
{   /* hackQuad, nbody_tree.c:70-121; the moment starts from zero */
    int i, k;
    double* Q = t->cells[p].quad;
    for (k = 0; k < 6; ++k) Q[k] = 0.0;
    for (i = 0; i < 8; ++i) {
        const int q = t->cells[p].sub[i];
        const double* qp;
        double m, dr[3], drsq, tq[6];
        if (q == OR_EMPTY) continue;
        if (!OR_IS_BODY(q)) or_quad(t, pos, mass, q);
        qp = OR_IS_BODY(q) ? pos + 3 * OR_BODY_INDEX(q) : t->cells[q].pos;
        m = OR_IS_BODY(q) ? mass[OR_BODY_INDEX(q)] : t->cells[q].mass;
        for (k = 0; k < 3; ++k) dr[k] = qp[k] - t->cells[p].pos[k];
        drsq = dr[2] * dr[2] + (dr[1] * dr[1] + dr[0] * dr[0]);
        tq[0] = m * (3.0 * (dr[0] * dr[0]) - drsq);
        tq[1] = m * (3.0 * (dr[0] * dr[1]));
        tq[2] = m * (3.0 * (dr[0] * dr[2]));
        tq[3] = m * (3.0 * (dr[1] * dr[1]) - drsq);
        tq[4] = m * (3.0 * (dr[1] * dr[2]));
        tq[5] = m * (3.0 * (dr[2] * dr[2]) - drsq);
        if (!OR_IS_BODY(q)) for (k = 0; k < 6; ++k) tq[k] = tq[k] + t->cells[q].quad[k];
        for (k = 0; k < 6; ++k) Q[k] = Q[k] + tq[k];
    }
}

/* nbMakeTree (nbody_tree.c:429-460).  Returns a status; bodyNext gets Next() of bodies. */
static int or_make_tree(const NBodyCudaCtx* ctx, OrTree* t, const double* pos,
                        const double* mass, int n, int* bodyNext)
{
    double xyzmax = 0.0;
    int i;
    t->nCells = 0;
    t->maxDepth = 0;
    t->structureError = 0;
    or_new_cell(t);                              /* root at the origin (nbNewTree) */
    for (i = 0; i < n; ++i) {                    /* expandBox */
        xyzmax = fmax(xyzmax, fabs(pos[3 * i] - 0.0));
        xyzmax = fmax(xyzmax, fabs(pos[3 * i + 1] - 0.0));
        xyzmax = fmax(xyzmax, fabs(pos[3 * i + 2] - 0.0));
    }
    while (t->rsize < 2.0 * xyzmax) t->rsize *= 2.0;
    for (i = 0; i < n; ++i)
        if (mass[i] != 0.0) or_load_body(t, pos, i);
    if (t->structureError) return NBODY_TREE_STRUCTURE_ERROR;
    or_cofm(ctx, t, pos, mass, 0, t->rsize);
    if (t->structureError) return NBODY_TREE_STRUCTURE_ERROR;
    for (i = 0; i < n; ++i) bodyNext[i] = OR_NULL;
    or_thread(t, 0, OR_NULL, bodyNext);
    if (ctx->useQuad) or_quad(t, pos, mass, 0);
    return NBODY_SUCCESS;
}

/* nbGravity (nbody_grav.c:42-124): the stackless walk of one body. */
static void or_gravity(const NBodyCudaCtx* ctx, const OrTree* t, const double* pos,
                       const double* mass, const int* bodyNext, int self, double* acc,
                       int* metSelf, unsigned long long* counts)
{
    const double x0 = pos[3 * self], y0 = pos[3 * self + 1], z0 = pos[3 * self + 2];
    double ax = 0.0, ay = 0.0, az = 0.0;
    int q = 0;   /* root */
    *metSelf = 0;
    while (q != OR_NULL) {
        const int isBody = OR_IS_BODY(q);
        const double* qp = isBody ? pos + 3 * OR_BODY_INDEX(q) : t->cells[q].pos;
        const double dx = qp[0] - x0, dy = qp[1] - y0, dz = qp[2] - z0;
        double drSq = dz * dz + (dy * dy + dx * dx);
        if (counts) counts[2]++;
        if (isBody || drSq >= t->cells[q].rcrit2) {
            if (!(isBody && OR_BODY_INDEX(q) == self)) {
                const double m = isBody ? mass[OR_BODY_INDEX(q)] : t->cells[q].mass;
                double drab, phii, mor3;
                if (counts) counts[isBody ? 0 : 1]++;
                drSq = drSq + ctx->eps2;
                drab = sqrt(drSq);
                phii = m / drab;
                mor3 = phii / drSq;
                ax = ax + mor3 * dx;
                ay = ay + mor3 * dy;
                az = az + mor3 * dz;
                if (ctx->useQuad && !isBody) {
                    const double* Q = t->cells[q].quad;
                    const double qdx = Q[0] * dx + Q[1] * dy + Q[2] * dz;
                    const double qdy = Q[1] * dx + Q[3] * dy + Q[4] * dz;
                    const double qdz = Q[2] * dx + Q[4] * dy + Q[5] * dz;
                    const double drQdr = qdx * dx + qdy * dy + qdz * dz;
                    const double dr5inv = 1.0 / ((drSq * drSq) * drab);
                    const double phiQ = 2.5 * (dr5inv * drQdr) / drSq;
                    ax = ax + phiQ * dx;
                    ay = ay + phiQ * dy;
                    az = az + phiQ * dz;
                    ax = ax - dr5inv * qdx;
                    ay = ay - dr5inv * qdy;
                    az = az - dr5inv * qdz;
                }
            } else {
                *metSelf = 1;
            }
            q = isBody ? bodyNext[OR_BODY_INDEX(q)] : t->cells[q].next;
        } else {
            q = t->cells[q].more;
        }
    }
    acc[0] = ax; acc[1] = ay; acc[2] = az;
}

/* nbGravity_Exact (nbody_grav.c:205-227) */
static void or_gravity_exact(const NBodyCudaCtx* ctx, const double* pos, const double* mass,
                             int n, int self, double* acc)
{
    const double x0 = pos[3 * self], y0 = pos[3 * self + 1], z0 = pos[3 * self + 2];
    double ax = 0.0, ay = 0.0, az = 0.0;
    int i;
    for (i = 0; i < n; ++i) {
        const double dx = pos[3 * i] - x0, dy = pos[3 * i + 1] - y0, dz = pos[3 * i + 2] - z0;
        const double drSq = (dz * dz + (dy * dy + dx * dx)) + ctx->eps2;
        const double drab = sqrt(drSq);
        const double phii = mass[i] / drab;
        const double mor3 = phii / drSq;
        ax = ax + mor3 * dx;
        ay = ay + mor3 * dy;
        az = az + mor3 * dz;
    }
    acc[0] = ax; acc[1] = ay; acc[2] = az;
}

/* nbMapForceBody's per-body epilogue (nbody_grav.c:160-176) */
static void or_add_external(const NBodyCudaCtx* ctx, const double* p, double* a)
{
    double e[3];
    if (ctx->potentialType != NBCUDA_POTENTIAL_DEFAULT) return;
    or_ext_accel_one(&ctx->pot, p, e);
    /* plummerAccel of the absent LMC (mass 0 at the origin): (0 - pos) * 0 */
    e[0] = e[0] + (0.0 - p[0]) * 0.0;
    e[1] = e[1] + (0.0 - p[1]) * 0.0;
    e[2] = e[2] + (0.0 - p[2]) * 0.0;
    a[0] = a[0] + e[0]; a[1] = a[1] + e[1]; a[2] = a[2] + e[2];
}

/* nbGravMap (nbody_grav.c:305-328).  rsize carries t->rsize between calls; *incest is the
 * sticky st->treeIncest.  counts (optional): body-body, body-cell interactions, visits. */
int or_grav_map(const NBodyCudaCtx* ctx, const double* pos, const double* mass, int n,
                double* rsize, double* acc, int* incest, unsigned long long* counts)
{
    int i, rc = NBODY_SUCCESS;
    if (ctx->criterion == NBCUDA_EXACT) {
#pragma omp parallel for schedule(dynamic, 64)
        for (i = 0; i < n; ++i) {
            or_gravity_exact(ctx, pos, mass, n, i, acc + 3 * i);
            or_add_external(ctx, pos + 3 * i, acc + 3 * i);
        }
    } else {
        OrTree t;
        int* bodyNext = (int*) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
        int anyIncest = 0;
        memset(&t, 0, sizeof t);
        t.rsize = *rsize;
        rc = or_make_tree(ctx, &t, pos, mass, n, bodyNext);
        *rsize = t.rsize;
        if (rc == NBODY_SUCCESS) {
            unsigned long long c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel for schedule(dynamic, 128) reduction(| : anyIncest) reduction(+ : c0, c1, c2)
            for (i = 0; i < n; ++i) {
                int met;
                unsigned long long cnt[3] = { 0, 0, 0 };
                or_gravity(ctx, &t, pos, mass, bodyNext, i, acc + 3 * i, &met, counts ? cnt : NULL);
                if (!met) anyIncest = 1;
                c0 += cnt[0]; c1 += cnt[1]; c2 += cnt[2];
                or_add_external(ctx, pos + 3 * i, acc + 3 * i);
            }
            if (counts) { counts[0] = c0; counts[1] = c1; counts[2] = c2; }
            if (anyIncest) *incest = 1;
        }
        free(bodyNext);
        free(t.cells);
    }
    if (rc != NBODY_SUCCESS) return rc;
    if (*incest) rc |= ctx->allowIncest ? NBODY_TREE_INCEST_NONFATAL : NBODY_TREE_INCEST_FATAL;
    return rc;
}

/* nsteps of nbStepSystemPlain (nbody_plain.c:268-364) with acc_i = acc_i1 = 0.  acc holds
 * the accelerations of the current positions on entry (from or_grav_map) and on exit. */
int or_step(const NBodyCudaCtx* ctx, double* pos, double* vel, const double* mass, int n,
            double* rsize, double* acc, int nsteps, int* incest)
{
    const double dt = ctx->timestep, dtHalf = 0.5 * dt;
    int s, i, k, all = NBODY_SUCCESS;
    for (s = 0; s < nsteps; ++s) {
        int rc;
        for (i = 0; i < n; ++i) {      /* advancePosVel */
            for (k = 0; k < 3; ++k) vel[3 * i + k] = vel[3 * i + k] + dtHalf * (acc[3 * i + k] + 0.0);
            for (k = 0; k < 3; ++k) pos[3 * i + k] = pos[3 * i + k] + dt * vel[3 * i + k];
        }
        rc = or_grav_map(ctx, pos, mass, n, rsize, acc, incest, NULL);
        for (i = 0; i < n; ++i)        /* advanceVelocities */
            for (k = 0; k < 3; ++k) vel[3 * i + k] = vel[3 * i + k] + dtHalf * (acc[3 * i + k] + 0.0);
        all |= rc;
        if (rc & ~(int) NBODY_STATUS_WARNINGS_MASK) break;
    }
    return all;
}

/* Tree in walk order, in the layout of nbGetTreeCUDA (include/nbody_b200.h); returns the node
 * count (negative: -count when cap is too small), or 0 with *status set on a build error. */
int or_tree(const NBodyCudaCtx* ctx, const double* pos, const double* mass, int n,
            double* rsize, int cap, double* npos, double* nmass, double* rcrit2, double* quad,
            int* next, int* body, int* depth, int* maxDepth, int* status)
{
    OrTree t;
    int* bodyNext = (int*) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
    int* cellIdx;
    int* bodyIdx;
    int count = 0, q, k;
    memset(&t, 0, sizeof t);
    t.rsize = *rsize;
    *status = or_make_tree(ctx, &t, pos, mass, n, bodyNext);
    *rsize = t.rsize;
    *maxDepth = t.maxDepth;
    if (*status != NBODY_SUCCESS) { free(bodyNext); free(t.cells); return 0; }
    cellIdx = (int*) malloc(sizeof(int) * (size_t) t.nCells);
    bodyIdx = (int*) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
    /* number the nodes in walk order */
    for (q = 0; q != OR_NULL;) {
        if (OR_IS_BODY(q)) { bodyIdx[OR_BODY_INDEX(q)] = count++; q = bodyNext[OR_BODY_INDEX(q)]; }
        else { cellIdx[q] = count++; q = t.cells[q].more != OR_NULL ? t.cells[q].more : t.cells[q].next; }
    }
    if (count > cap) { free(bodyNext); free(t.cells); free(cellIdx); free(bodyIdx); return -count; }
    for (q = 0; q != OR_NULL;) {
        const int isBody = OR_IS_BODY(q);
        const int bi = isBody ? OR_BODY_INDEX(q) : -1;
        const int idx = isBody ? bodyIdx[bi] : cellIdx[q];
        const int nx = isBody ? bodyNext[bi] : t.cells[q].next;
        const int nxIdx = nx == OR_NULL ? count : (OR_IS_BODY(nx) ? bodyIdx[OR_BODY_INDEX(nx)] : cellIdx[nx]);
        if (next) next[idx] = nxIdx;
        if (body) body[idx] = bi;
        if (isBody) {
            if (npos) for (k = 0; k < 3; ++k) npos[3 * idx + k] = pos[3 * bi + k];
            if (nmass) nmass[idx] = mass[bi];
            if (rcrit2) rcrit2[idx] = 0.0;
            if (quad) for (k = 0; k < 6; ++k) quad[6 * idx + k] = 0.0;
            q = nx;
        } else {
            const OrCell* c = &t.cells[q];
            if (npos) for (k = 0; k < 3; ++k) npos[3 * idx + k] = c->pos[k];
            if (nmass) nmass[idx] = c->mass;
            if (rcrit2) rcrit2[idx] = c->rcrit2;
            if (quad) for (k = 0; k < 6; ++k) quad[6 * idx + k] = ctx->useQuad ? c->quad[k] : 0.0;
            if (depth) {
                depth[idx] = c->depth;
                for (k = 0; k < 8; ++k)
                    if (OR_IS_BODY(c->sub[k])) depth[bodyIdx[OR_BODY_INDEX(c->sub[k])]] = c->depth + 1;
            }
            q = c->more != OR_NULL ? c->more : c->next;
        }
    }
    free(bodyNext); free(t.cells); free(cellIdx); free(bodyIdx);
    return count;
}

/* A bounded sample of one step for the CPU baseline (the restatement's counterpart of
 * nbref_sample_step): the whole tree, then the walk + external potential for `count` bodies.
 * Times in seconds (omp_get_wtime). */
#include <omp.h>
int or_sample_step(const NBodyCudaCtx* ctx, const double* pos, const double* mass, int n,
                   double* rsize, const int* idx, int count, double* acc, double* tTree,
                   double* tWalk)
{
    OrTree t;
    int* bodyNext = (int*) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
    double t0, t1, t2;
    int k, rc;
    memset(&t, 0, sizeof t);
    t.rsize = *rsize;
    t0 = omp_get_wtime();
    rc = or_make_tree(ctx, &t, pos, mass, n, bodyNext);
    t1 = omp_get_wtime();
    *rsize = t.rsize;
    if (rc == NBODY_SUCCESS) {
#pragma omp parallel for schedule(dynamic, 64)
        for (k = 0; k < count; ++k) {
            int met;
            or_gravity(ctx, &t, pos, mass, bodyNext, idx[k], acc + 3 * k, &met, NULL);
            or_add_external(ctx, pos + 3 * idx[k], acc + 3 * k);
        }
    }
    t2 = omp_get_wtime();
    *tTree = t1 - t0;
    *tWalk = t2 - t1;
    free(bodyNext);
    free(t.cells);
    return rc;
}

int or_threads(void) { return omp_get_max_threads(); }
