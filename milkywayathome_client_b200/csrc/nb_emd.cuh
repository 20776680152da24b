// Earth mover's distance between two weighted point sets in (lambda, beta): the transportation
// simplex the reference's emdCalc runs (nbody/src/nbody_emd.c:1207-1268), which is Rubner's
// published EMD (Y. Rubner, emd.c, 1998, after the transportation simplex of Hillier and
// Lieberman, "Introduction to Mathematical Programming", 1990), restated for host and device.
//
// The reference returns the cost of the basis its simplex stops at: Russell's approximation
// gives the first basis, then entering variables are taken while some reduced cost is below
// -1e-5 x the largest ground distance, so the final basis -- and the EMD, before nbMatchEMD
// rounds it to 1e-9 -- depends on every decision of that sequence, not only on the optimum.
// This code therefore takes the same decisions in the same order with the same arithmetic:
//   * supplies (first set) and demands (second set) of positive weight, in input order; a
//     zero-cost dummy node on the short side when the totals differ by >= 1e-5 x the supply;
//   * Russell: u_i, v_j = row and column maxima of the cost, delta = c - u - v; repeatedly the
//     first smallest delta over the active rows x columns in row-major order enters the basis
//     with the smaller of its supply and demand (the supply when s < d + 1e-5 W); the exhausted
//     row is dropped if two or more rows remain, else the column; then the row (column) maxima
//     are refreshed for the lines whose maximum sat in the dropped column (row) -- the
//     reference's test for which line was dropped selects these the other way round, and that
//     choice is kept -- and delta moves with a refreshed maximum only when it moved by less
//     than 1e-5 x the largest distance;
//   * each simplex iteration: potentials along the basis tree from v_0 = 0; the entering cell is
//     the first smallest reduced cost (c - u) - v over the non-basic cells in row-major order;
//     stop when it is >= -1e-5 x the largest distance; the cycle through the entering cell
//     starts along its row; the leaving cell is the first smallest flow at the odd positions
//     of that cycle; at most 2,499 iterations;
//   * the cost is summed over the basis slots in slot order (a leaving cell's slot takes the
//     next entering cell), divided by the larger total weight.
// Data layout and traversal are this file's own: dense arrays, per-line slot lists, a
// breadth-first search for potentials and cycles, and block-wide first-minimum scans (the
// first minimum in row-major order is the lexicographic minimum of (value, index)).
#pragma once
#include <math.h>
#include <stddef.h>

#ifdef __CUDACC__
#define NB_EMD_HD __host__ __device__
#else
#define NB_EMD_HD
#endif

constexpr int NB_EMD_MAX_ITERATIONS = 2500;
constexpr double NB_EMD_INF = 1.0e20;
constexpr double NB_EMD_EPS = 1.0e-5;

struct NbEmdMin {
    double val;
    int idx;
};

// scalars every thread of a team reads after a sync
struct NbEmdScalars {
    int ss, ds;                 // supplies, demands (dummy included)
    int nSlots, enter;          // slots used; the free slot the next entering cell takes
    int actRows, actCols;       // Russell: active lines
    int rowDropped;             // Russell: the last step dropped its row
    int status;                 // 0 running, 1 done, -1 failed
    double weight, maxCost, eps;
    NbEmdMin m;                 // the last scan's first minimum
};

// Workspace of one problem with at most n1 supplies and n2 demands (a dummy node is added on
// one side: S = n1 + 1 rows, D = n2 + 1 columns, K = S + D slots and tree nodes).
struct NbEmdWork {
    double *s, *d, *u, *v, *cost, *delta, *slotVal;
    int *idx1, *idx2, *slotI, *slotJ, *slotNR, *slotNC, *rowFirst, *colFirst;
    int *queue, *via, *loop;
    unsigned char *isx, *rowAct, *colAct, *seen;
    int S, D;
};

NB_EMD_HD inline size_t nb_emd_align(size_t b) { return (b + 15) & ~(size_t) 15; }

NB_EMD_HD inline size_t nb_emd_work_bytes(int n1, int n2)
{
    const size_t S = (size_t) n1 + 1, D = (size_t) n2 + 1, K = S + D;
    return 2 * nb_emd_align(8 * S) + 2 * nb_emd_align(8 * D) + 2 * nb_emd_align(8 * S * D) +
           nb_emd_align(8 * K) + nb_emd_align(4 * S) + nb_emd_align(4 * D) + 4 * nb_emd_align(4 * K) +
           nb_emd_align(4 * S) + nb_emd_align(4 * D) + 2 * nb_emd_align(4 * K) +
           nb_emd_align(4 * (K + 1)) + nb_emd_align(S * D) + nb_emd_align(S) + nb_emd_align(D) +
           nb_emd_align(K);
}

NB_EMD_HD inline NbEmdWork nb_emd_carve(void* base, int n1, int n2)
{
    NbEmdWork w;
    const size_t S = (size_t) n1 + 1, D = (size_t) n2 + 1, K = S + D;
    char* p = (char*) base;
    auto take = [&p](size_t b) { char* q = p; p += nb_emd_align(b); return q; };
    w.s = (double*) take(8 * S);
    w.u = (double*) take(8 * S);
    w.d = (double*) take(8 * D);
    w.v = (double*) take(8 * D);
    w.cost = (double*) take(8 * S * D);
    w.delta = (double*) take(8 * S * D);
    w.slotVal = (double*) take(8 * K);
    w.idx1 = (int*) take(4 * S);
    w.idx2 = (int*) take(4 * D);
    w.slotI = (int*) take(4 * K);
    w.slotJ = (int*) take(4 * K);
    w.slotNR = (int*) take(4 * K);
    w.slotNC = (int*) take(4 * K);
    w.rowFirst = (int*) take(4 * S);
    w.colFirst = (int*) take(4 * D);
    w.queue = (int*) take(4 * K);
    w.via = (int*) take(4 * K);
    w.loop = (int*) take(4 * (K + 1));
    w.isx = (unsigned char*) take(S * D);
    w.rowAct = (unsigned char*) take(S);
    w.colAct = (unsigned char*) take(D);
    w.seen = (unsigned char*) take(K);
    w.S = (int) S;
    w.D = (int) D;
    return w;
}

// The team that runs one problem: a single thread on the host.  A device block provides the
// same interface (rank, size, sync, first-minimum and maximum over its threads).
struct NbEmdSerial {
    NB_EMD_HD int rank() const { return 0; }
    NB_EMD_HD int size() const { return 1; }
    NB_EMD_HD void sync() const {}
    NB_EMD_HD NbEmdMin argmin(NbEmdMin a) const { return a; }
    NB_EMD_HD double maxv(double a) const { return a; }
};

// (value, index) a before b in the first-minimum order; candidates are values < NB_EMD_INF
NB_EMD_HD inline bool nb_emd_before(const NbEmdMin& a, const NbEmdMin& b)
{
    return a.val < b.val || (a.val == b.val && a.idx < b.idx);
}

// L2 distance of two (lambda, beta) points, the reference's dimension loop unrolled
NB_EMD_HD inline double nb_emd_dist(const double* x, const double* y)
{
    const double t0 = x[0] - y[0];
    double acc = 0.0;
    acc += t0 * t0;
    const double t1 = x[1] - y[1];
    acc += t1 * t1;
    return sqrt(acc);
}

// Breadth-first search over the basis tree (rows 0..S-1, columns S..S+D-1 as nodes) from
// node `from`, skipping slot `skip`.  Returns the number of nodes reached; via[node] = the slot
// the node was reached through (-1 for the start).  With `potentials`, assigns u and v along
// the tree edges as the reference's potentials (u_i = c_ij - v_j, v_j = c_ij - u_i).
NB_EMD_HD inline int nb_emd_bfs(const NbEmdWork& w, int ss, int ds, int from, int skip,
                                bool potentials)
{
    const int S = w.S;
    for (int k = 0; k < ss; ++k) w.seen[k] = 0;
    for (int k = 0; k < ds; ++k) w.seen[S + k] = 0;
    int head = 0, tail = 0;
    w.queue[tail++] = from;
    w.seen[from] = 1;
    w.via[from] = -1;
    while (head < tail) {
        const int node = w.queue[head++];
        if (node < S) {
            const int i = node;
            for (int k = w.rowFirst[i]; k >= 0; k = w.slotNR[k]) {
                if (k == skip) continue;
                const int c = S + w.slotJ[k];
                if (w.seen[c]) continue;
                w.seen[c] = 1;
                w.via[c] = k;
                if (potentials) w.v[w.slotJ[k]] = w.cost[(size_t) i * w.D + w.slotJ[k]] - w.u[i];
                w.queue[tail++] = c;
            }
        } else {
            const int j = node - S;
            for (int k = w.colFirst[j]; k >= 0; k = w.slotNC[k]) {
                if (k == skip) continue;
                const int r = w.slotI[k];
                if (w.seen[r]) continue;
                w.seen[r] = 1;
                w.via[r] = k;
                if (potentials) w.u[r] = w.cost[(size_t) r * w.D + j] - w.v[j];
                w.queue[tail++] = r;
            }
        }
    }
    return tail;
}

NB_EMD_HD inline void nb_emd_unlink(const NbEmdWork& w, int k)
{
    const int i = w.slotI[k], j = w.slotJ[k];
    if (w.rowFirst[i] == k) {
        w.rowFirst[i] = w.slotNR[k];
    } else {
        int p = w.rowFirst[i];
        while (w.slotNR[p] != k) p = w.slotNR[p];
        w.slotNR[p] = w.slotNR[k];
    }
    if (w.colFirst[j] == k) {
        w.colFirst[j] = w.slotNC[k];
    } else {
        int p = w.colFirst[j];
        while (w.slotNC[p] != k) p = w.slotNC[p];
        w.slotNC[p] = w.slotNC[k];
    }
}

NB_EMD_HD inline void nb_emd_link(const NbEmdWork& w, int k, int i, int j)
{
    w.slotI[k] = i;
    w.slotJ[k] = j;
    w.slotNR[k] = w.rowFirst[i];
    w.rowFirst[i] = k;
    w.slotNC[k] = w.colFirst[j];
    w.colFirst[j] = k;
}

// emdCalc(sig1, sig2, n1, n2) with signatures of (weight, lambda, beta) triples; every thread
// of the team calls it with the same arguments and workspace, sc shared by the team.  Returns
// the EMD, or NaN where the reference returns EMD_INVALID (no positive weight on a side, a
// negative weight, an iteration that finds no entering cell or no cycle).
template <class Team>
NB_EMD_HD double nb_emd_calc(const Team& t, const double* sig1, int n1, const double* sig2, int n2,
                             const NbEmdWork& w, NbEmdScalars& sc)
{
    const int me = t.rank(), T = t.size();
    const int D = w.D;
    // ---- supplies, demands, dummy node, weight ----
    if (me == 0) {
        double sSum = 0.0, dSum = 0.0;
        int ss = 0, ds = 0;
        sc.status = 0;
        for (int i = 0; i < n1; ++i) {
            const double wt = sig1[3 * i];
            if (wt > 0.0) { sSum += wt; w.s[ss] = wt; w.idx1[ss++] = i; }
            else if (wt < 0.0) sc.status = -1;
        }
        for (int i = 0; i < n2; ++i) {
            const double wt = sig2[3 * i];
            if (wt > 0.0) { dSum += wt; w.d[ds] = wt; w.idx2[ds++] = i; }
            else if (wt < 0.0) sc.status = -1;
        }
        if (ss == 0 || ds == 0) sc.status = -1;
        const double diff = sSum - dSum;
        if (sc.status == 0 && fabs(diff) >= NB_EMD_EPS * sSum) {
            if (diff < 0) { w.s[ss] = -diff; w.idx1[ss++] = -1; }
            else { w.d[ds] = diff; w.idx2[ds++] = -1; }
        }
        sc.ss = ss;
        sc.ds = ds;
        sc.weight = sSum > dSum ? sSum : dSum;
    }
    t.sync();
    if (sc.status < 0) return NAN;
    const int ss = sc.ss, ds = sc.ds;
    const int cells = ss * ds;
    // ---- ground distances (a dummy's are zero) and their maximum ----
    double myMax = 0.0;
    for (int c = me; c < cells; c += T) {
        const int i = c / ds, j = c % ds;
        const int ci = w.idx1[i], cj = w.idx2[j];
        double val = 0.0;
        if (ci >= 0 && cj >= 0) val = nb_emd_dist(sig1 + 3 * ci + 1, sig2 + 3 * cj + 1);
        w.cost[(size_t) i * D + j] = val;
        w.isx[(size_t) i * D + j] = 0;
        if (myMax < val) myMax = val;
    }
    const double maxCost = t.maxv(myMax);
    if (me == 0) {
        sc.maxCost = maxCost;
        sc.eps = NB_EMD_EPS * maxCost;
        sc.nSlots = 0;
        sc.actRows = ss;
        sc.actCols = ds;
    }
    for (int i = me; i < ss; i += T) { w.rowAct[i] = 1; w.rowFirst[i] = -1; }
    for (int j = me; j < ds; j += T) { w.colAct[j] = 1; w.colFirst[j] = -1; }
    t.sync();
    const double eps = sc.eps;
    // ---- Russell's approximation ----
    for (int i = me; i < ss; i += T) {
        double m = -NB_EMD_INF;
        for (int j = 0; j < ds; ++j) {
            const double c = w.cost[(size_t) i * D + j];
            if (m < c) m = c;
        }
        w.u[i] = m;
    }
    for (int j = me; j < ds; j += T) {
        double m = -NB_EMD_INF;
        for (int i = 0; i < ss; ++i) {
            const double c = w.cost[(size_t) i * D + j];
            if (m < c) m = c;
        }
        w.v[j] = m;
    }
    t.sync();
    for (int c = me; c < cells; c += T) {
        const int i = c / ds, j = c % ds;
        w.delta[(size_t) i * D + j] = w.cost[(size_t) i * D + j] - w.u[i] - w.v[j];
    }
    t.sync();
    for (;;) {
        NbEmdMin best{NB_EMD_INF, -1};
        for (int c = me; c < cells; c += T) {
            const int i = c / ds, j = c % ds;
            if (!w.rowAct[i] || !w.colAct[j]) continue;
            const double dl = w.delta[(size_t) i * D + j];
            if (dl < best.val) { best.val = dl; best.idx = c; }
        }
        best = t.argmin(best);
        if (best.idx < 0) break;
        const int mi = best.idx / ds, mj = best.idx % ds;
        if (me == 0) {
            double moved;
            if (w.s[mi] < w.d[mj] + sc.weight * NB_EMD_EPS) {      // supply exhausted
                moved = w.s[mi];
                w.s[mi] = 0;
                w.d[mj] -= moved;
            } else {                                               // demand exhausted
                moved = w.d[mj];
                w.d[mj] = 0;
                w.s[mi] -= moved;
            }
            w.isx[(size_t) mi * D + mj] = 1;
            const int k = sc.nSlots++;
            w.slotVal[k] = moved;
            nb_emd_link(w, k, mi, mj);
            if (w.s[mi] == 0.0 && sc.actRows >= 2) {
                w.rowAct[mi] = 0;
                --sc.actRows;
                sc.rowDropped = 1;
            } else {
                w.colAct[mj] = 0;
                --sc.actCols;
                sc.rowDropped = 0;
            }
        }
        t.sync();
        if (!sc.rowDropped) {
            // the column was dropped: refresh the column maxima that sat in row mi
            for (int j = me; j < ds; j += T) {
                if (!w.colAct[j] || w.v[j] != w.cost[(size_t) mi * D + j]) continue;
                double m = -NB_EMD_INF;
                for (int i = 0; i < ss; ++i)
                    if (w.rowAct[i] && m < w.cost[(size_t) i * D + j]) m = w.cost[(size_t) i * D + j];
                const double diff = m - w.v[j];
                w.v[j] = m;
                if (fabs(diff) < eps)
                    for (int i = 0; i < ss; ++i)
                        if (w.rowAct[i]) w.delta[(size_t) i * D + j] += diff;
            }
        } else {
            // the row was dropped: refresh the row maxima that sat in column mj
            for (int i = me; i < ss; i += T) {
                if (!w.rowAct[i] || w.u[i] != w.cost[(size_t) i * D + mj]) continue;
                double m = -NB_EMD_INF;
                for (int j = 0; j < ds; ++j)
                    if (w.colAct[j] && m < w.cost[(size_t) i * D + j]) m = w.cost[(size_t) i * D + j];
                const double diff = m - w.u[i];
                w.u[i] = m;
                if (fabs(diff) < eps)
                    for (int j = 0; j < ds; ++j)
                        if (w.colAct[j]) w.delta[(size_t) i * D + j] += diff;
            }
        }
        t.sync();
        if (sc.actRows == 0 && sc.actCols == 0) break;
    }
    if (me == 0) {
        sc.enter = sc.nSlots++;            // the free slot
        w.slotVal[sc.enter] = 0.0;
        w.slotI[sc.enter] = 0;
        w.slotJ[sc.enter] = 0;
    }
    t.sync();
    // ---- simplex iterations ----
    if (ss > 1 && ds > 1) {
        for (int itr = 1; itr < NB_EMD_MAX_ITERATIONS; ++itr) {
            if (me == 0) {
                // potentials along the basis tree from v_0 = 0
                w.v[0] = 0.0;
                const int reached = nb_emd_bfs(w, ss, ds, w.S + 0, -1, true);
                sc.status = reached < ss + ds ? 1 : 0;     // a broken tree ends the iterations
            }
            t.sync();
            if (sc.status) break;
            NbEmdMin best{NB_EMD_INF, -1};
            for (int c = me; c < cells; c += T) {
                const int i = c / ds, j = c % ds;
                if (w.isx[(size_t) i * D + j]) continue;
                const double dl = w.cost[(size_t) i * D + j] - w.u[i] - w.v[j];
                if (dl < best.val) { best.val = dl; best.idx = c; }
            }
            best = t.argmin(best);
            if (best.idx < 0) {                             // no non-basic cell
                if (me == 0) sc.status = -1;
                t.sync();
                break;
            }
            if (best.val >= -eps) break;                   // optimal within the tolerance
            if (me == 0) {
                const int ie = best.idx / ds, je = best.idx % ds;
                const int E = sc.enter;
                // the cycle: the entering cell, then the tree path from row ie to column je
                const int reached = nb_emd_bfs(w, ss, ds, ie, -1, false);
                (void) reached;
                if (!w.seen[w.S + je]) {
                    sc.status = -1;
                } else {
                    int n = 0;
                    for (int node = w.S + je; w.via[node] >= 0;) {
                        const int k = w.via[node];
                        w.loop[1 + n++] = k;
                        node = node >= w.S ? w.slotI[k] : w.S + w.slotJ[k];
                    }
                    // the path was collected from column je back to row ie: reverse it
                    for (int a = 1, b = n; a < b; ++a, --b) {
                        const int x = w.loop[a];
                        w.loop[a] = w.loop[b];
                        w.loop[b] = x;
                    }
                    const int steps = n + 1;
                    w.isx[(size_t) ie * D + je] = 1;
                    w.slotVal[E] = 0.0;
                    nb_emd_link(w, E, ie, je);
                    w.loop[0] = E;
                    double minVal = NB_EMD_INF;
                    int leave = -1;
                    for (int a = 1; a < steps; a += 2) {
                        const double x = w.slotVal[w.loop[a]];
                        if (minVal > x) { leave = w.loop[a]; minVal = x; }
                    }
                    if (leave < 0) {
                        sc.status = -1;
                    } else {
                        for (int a = 0; a < steps; a += 2) {
                            const double t0 = w.slotVal[w.loop[a]] + minVal;
                            const double t1 = w.slotVal[w.loop[a + 1]] - minVal;
                            w.slotVal[w.loop[a]] = t0;
                            w.slotVal[w.loop[a + 1]] = t1;
                        }
                        w.isx[(size_t) w.slotI[leave] * D + w.slotJ[leave]] = 0;
                        nb_emd_unlink(w, leave);
                        sc.enter = leave;
                    }
                }
            }
            t.sync();
            if (sc.status < 0) break;
        }
    }
    if (sc.status < 0) return NAN;
    // ---- the total cost over the basis slots, in slot order ----
    double total = 0.0;
    if (me == 0) {
        for (int k = 0; k < sc.nSlots; ++k) {
            if (k == sc.enter) continue;
            const int i = w.slotI[k], j = w.slotJ[k];
            if (w.idx1[i] >= 0 && w.idx2[j] >= 0) total += w.slotVal[k] * w.cost[(size_t) i * D + j];
        }
        sc.m.val = total / sc.weight;
    }
    t.sync();
    return sc.m.val;
}
