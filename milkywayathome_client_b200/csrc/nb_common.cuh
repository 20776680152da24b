// Shared declarations of the B200 Barnes-Hut step (sm_100a).
//
// Device data layout (all in HBM, one NBodyCudaState per simulation):
//   bodies      SoA FP64 in the caller's order: px py pz vx vy vz ax ay az mass
//   sort        63-bit Morton keys of the top 21 levels + body index (LSD radix sort),
//               then 62-bit integer grid coordinates per axis of the sorted bodies
//   tree        nodes in the reference's walk order (threadTree preorder,
//               nbody/src/nbody_tree.c:127-150): for node k
//                 nodePM[k]   = {x, y, z, mass}   (CoM for cells, position for bodies)
//                 nodeCrit[k] = rcrit2            (cells only)
//                 nodeLink[k] = {next, body}      (Next() index, body index or -1)
//                 nodeQuad[k] = 6 quadrupole components (cells only)
//   scalars     NbScalars below (root size, counts, status bits)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/nbody_b200.h"

#define NB_FULL_MASK 0xffffffffu

// Levels of the integer grid used for the octant decisions: coordinates are
// floor(pos * 2^62 / rsize) + 2^61, so every cell midpoint of depth < 62 is an
// integer on this grid and `mid <= pos` (nbody/src/nbody_tree.c:42-49) is an exact
// integer comparison.
#define NB_GRID_LEVELS 62
#define NB_KEY_LEVELS 21          // levels in the 63-bit sort key
#define NB_MASSLESS_KEY 0xffffffffffffffffull

struct NbScalars {
    unsigned long long xyzmaxBits;  // max |coordinate| over bodies (bit pattern, >= 0)
    double rsize;                   // root side length (t->rsize), kept between steps
    double gridScale;               // 2^62 / rsize
    int depthEps;                   // first depth whose cell size is <= DBL_EPSILON
    int nTree;                      // bodies with nonzero mass
    int nCells;
    int nNodes;
    int maxDepth;                   // deepest parent level of a body (t->maxDepth)
    int status;                     // NBodyStatus bits raised on the device
    int incest;                     // a body did not meet itself in the walk
    int capNodes;                   // node capacity of the allocation
    int neededNodes;                // nodes the last build asked for (overflow recovery)
    unsigned long long nBodyBody;   // interaction counters (counting build of the walk)
    unsigned long long nBodyCell;
    unsigned long long nVisit;
    unsigned long long nWarpSteps;  // walk iterations summed over warps (SIMT utilisation)
    int groupNext;                  // next group for the persistent group walk
    int nGroups;                    // walk groups formed for the mixed walk
    int step;                       // batched dwarfs: steps taken (the bar's time)
    double timeOrigin;              // batched dwarfs: the bar's time origin
};

// Potential parameters in constant-friendly POD form.
struct NbPot {
    int sphType; double sphMass, sphScale;
    int diskType; double diskMass, diskA, diskB;
    int disk2Type; double disk2Mass, disk2A, disk2B;
    double disk2Pattern, disk2StartAngle;            // orbiting bar (disk2)
    int haloType; double haloV, haloA, haloQz;
    double haloMass, haloGamma, haloLambda, haloRho0;  // mass-parameterised halos
    double haloC1, haloC2, haloC3;                     // triaxial halo constants
    double time;   // the bar's time: step * timestep (nbody/src/nbody_grav.c:141)
    int enabled;   // potentialType == DEFAULT
    const double* lmc;          // the LMC's {pos, vel} in device memory (nullptr: no LMC)
    double lmcMass, lmcScale;   // its Plummer sphere
};

struct NbWalkParams {
    double eps2;
    double dtHalf;
    double shift[3];   // the Milky Way's reflex acceleration of the second half kick (LMC runs)
    int useQuad;
    int kick;      // 1: v += (a + 0) * dtHalf after the force (advanceVelocities)
    int n;
};

// ---- correctly rounded powers ------------------------------------------------------
// The reference evaluates the disk/bulge terms with crlibm's correctly rounded pow_rn
// (milkyway/include/milkyway_math_double.h:43-59).  x^2 and x^0.5 are correctly rounded
// by one IEEE multiply / sqrt.  x^1.5 and x^3 are formed here as a double-double value
// (error-free products via fma) and rounded once: the double-double carries ~104 bits,
// so its rounding equals the correctly rounded result except for arguments whose exact
// power lies within 2^-100 relative of a rounding boundary.
__device__ __forceinline__ double nb_pow_1p5(double x)
{
    if (!(x > 0.0) || isinf(x)) {
        if (x == 0.0) return 0.0;
        return isinf(x) && x > 0.0 ? x : __longlong_as_double(0x7ff8000000000000ll);
    }
    double s = __dsqrt_rn(x);
    double r = __fma_rn(-s, s, x);                 // x - s^2, exact
    double t = __ddiv_rn(r, __dmul_rn(2.0, s));    // sqrt(x) = s + t (+ O(t^2/s))
    double hi = __dmul_rn(x, s);
    double lo = __fma_rn(x, s, -hi);               // x*s - hi, exact
    lo = __dadd_rn(lo, __dmul_rn(x, t));
    return __dadd_rn(hi, lo);
}

__device__ __forceinline__ double nb_pow_3(double x)
{
    double sq = __dmul_rn(x, x);
    double e1 = __fma_rn(x, x, -sq);               // x^2 - sq, exact
    double hi = __dmul_rn(sq, x);
    double lo = __fma_rn(sq, x, -hi);              // sq*x - hi, exact
    lo = __dadd_rn(lo, __dmul_rn(e1, x));
    if (isinf(hi) || hi == 0.0) return hi;
    return __dadd_rn(hi, lo);
}

// Device error checks produce NBodyStatus bits; kernels stop doing work once a fatal
// bit is set so the state is left as it was at the failure point.
__device__ __forceinline__ void nb_raise(NbScalars* sc, int bits) { atomicOr(&sc->status, bits); }
__device__ __forceinline__ bool nb_failed(const NbScalars* sc)
{
    return (*(volatile const int*) &sc->status & ~(int) NBODY_STATUS_WARNINGS_MASK) != 0;
}

// One 32-byte read-only load of a 32-byte-aligned double4 (ld.global.nc.v4.f64, sm_100).
// double4 itself is only 16-byte aligned, so a plain load of one is two 16-byte requests that
// each count the same sector; this is one request, one sector per lane.  For buffers a kernel
// only reads.
__device__ __forceinline__ double4 nb_ld32(const double4* p)
{
    double4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
    return r;
}

// ---- batched dwarfs: a forest of independent trees in one set of arrays ----
// Dwarf d owns bodies [first, first + count) (input order and sorted order alike: the sort
// orders by dwarf first) and the nodes [rootNode, rootEnd) in walk order.
struct NbDwarfDev {
    unsigned long long xyzmaxBits;  // max |coordinate| over the dwarf's bodies (bit pattern)
    double rsize;                   // the dwarf's root size, kept between steps
    double gridScale;               // 2^62 / rsize
    double eps2;                    // softening^2 of this dwarf
    double dt;                      // time step of this dwarf
    int first, count;               // body range
    int rootNode, rootEnd;          // root node and Next(root)
    int depthEps;                   // first depth whose cell size is <= DBL_EPSILON
    int status;                     // status bits raised while building this dwarf's tree
    double time;                    // the bar's time of this evaluation: step * dt - origin
    double timeOrigin;              // this dwarf's own bar time origin (calibration runs; else 0)
    double lmc[6];                  // LMC runs: this dwarf's LMC position and velocity
};
struct NbForest {
    const int* bodyDwarf;           // dwarf of every body (input = sorted position)
    NbDwarfDev* dwarfs;
    int nDwarfs;
    // LMC runs: each dwarf's reflex accelerations, nShift vectors of 3 doubles from
    // lmcShift + 3 nShift d (shiftByLMC; step k takes k in the drift and k + 1 in the kick)
    const double* lmcShift;
    int nShift;
};
// The LMC of a batch's LMC runs: the context's LMC parameters and the potential it moves in.
struct NbBatchLMC {
    NbPot pot;
    double mass;
    int dynaFric;
    double coulombLog;
};

// ---- Lambda-Beta histograms and the likelihood (nb_likelihood.cu) ----
// Per-body quantities that the comparison histograms bin (a slot of the plan holds one):
enum { NB_Q_BETA = 0, NB_Q_VLOS = 1, NB_Q_DIST = 2, NB_Q_MUDEC = 3, NB_Q_MURA = 4, NB_NQ = 5 };
constexpr int NB_HIST_COMPONENTS = 7;     // histograms 1..7 of the reference's MainStruct
constexpr int NB_LIKELIHOOD_TERMS = 11;   // nbSystemLikelihood's 10 terms + the EMD itself

// Histogram geometry and the per-body quantities to evaluate (device copy).
struct NbHistDev {
    double rot[9];                  // rot11 .. rot33 of nbXYZToLambdaBeta
    double sunGCDist, lambdaStart, lambdaSize, betaStart, betaSize;
    int lambdaBins, betaBins;
    double align[9];                // cartesianalign's rotation (proper motions)
    double sunVel[3];
    int nq;                         // active quantity slots
    int q[NB_NQ];                   // quantity of each slot
};
// One histogram evaluation of nDwarfs dwarfs: device arrays (carved from one scratch block)
// and the outlier-rejection constants.  A stable counting sort (chunks of bodies that never
// straddle a dwarf, one warp per chunk) lists every bin's bodies in body order, so each bin's
// sums are formed in the reference's order.
struct NbHistPlan {
    NbHistDev h;
    int n, D, B, nChunks, iterMax;
    double cut[NB_NQ], corr[NB_NQ]; // sigma cut-off and dispersion correction of each slot
    int histSlot[NB_HIST_COMPONENTS];  // slot of histograms 1..7 (-1: not built)
    unsigned int* counts;           // D*B raw counts
    unsigned int* inRange;          // D
    unsigned int* nLight;           // D
    int* lastLight;                 // D (-1: none)
    int* binOf;                     // n: bin of the body within its dwarf, -1 if not binned
    double* val;                    // nq*n: the body's quantities
    int4* chunks;                   // {first, end, dwarf, 0}
    int* chunkFirst;                // D+1: first chunk of each dwarf
    int* rows;                      // nChunks*B: bodies of each bin in a chunk, then offsets
    int* segStart;                  // D*B: first list entry of each (dwarf, bin)
    int* list;                      // n: the binned bodies, bin after bin, in body order
    double* sum;                    // nq*D*B: the reference's HistData sum, sq_sum,
    double* sq;                     //   outliersRemoved, variable and err of each
    double* rem;                    //   dispersion quantity
    double* var;
    double* err;
};
// A data histogram to compare against (device pointers to nBins entries).
struct NbDataHistDev {
    const int* useBin;
    const double* lambda;           // bin centres
    const double* variable;         // normalised counts
    const double* err;
    const double* compVar[NB_HIST_COMPONENTS];  // histograms 1..7 (nullptr: absent)
    const double* compErr[NB_HIST_COMPONENTS];
    double massPerParticle;
    unsigned int totalNum;
    int nBins;
    int betaDispBins;
    int nRange;                     // EMD lambda ranges (0: one over every bin)
    const double* emdRange;
    const double* beta;             // bin centres in beta (two-dimensional histograms)
    double* emd2d;                  // betaBins > 1: emdCalc of every (dwarf, range) problem
    char* emdWork;                  //   and the workspace of each problem,
    size_t emdWorkBytes;            //   emdWorkBytes apart
};
// emdCalc problems of the two-dimensional likelihood: one per dwarf and lambda range.
int nb_emd_ranges(const NbDataHistDev& dh);
size_t nb_emd_problem_bytes(int nBins);
void nb_launch_emd_ranges(const NbHistPlan& p, const NbDataHistDev& dh, cudaStream_t s);
// emdCalc of two host-given signatures on the device (work: nb_emd_problem_bytes(max(n1, n2))).
void nb_launch_emd_direct(const double* sig1, int n1, const double* sig2, int n2, char* work,
                          double* out, cudaStream_t s);
// Which comparison terms nbSystemLikelihood adds (the reference's st->use* flags).
struct NbLikeFlags {
    int betaDisp, velDisp, betaComp, vlos, dist, propMot;
};
// Counts, per-body quantities and the dispersions with their outlier passes.
int nb_launch_hist_plan(const NbHistPlan& p, const double* px, const double* py, const double* pz,
                        const double* vx, const double* vy, const double* vz, const int* types,
                        const int* bodyDwarf, int numSMs, cudaStream_t s);
// out: NB_LIKELIHOOD_TERMS doubles per dwarf.
void nb_launch_likelihood(const NbHistPlan& p, const double* mass, const int* nbodyOf,
                          const NbDataHistDev& dh, NbLikeFlags f, double* out, cudaStream_t s);
// comps: per dwarf, histograms 1..7 x {variable[B], err[B]} (zeros where not built).
void nb_launch_hist_export(const NbHistPlan& p, double* comps, cudaStream_t s);
size_t nb_hist_chunk_bodies(int n, int nq, int B);
// The best likelihood of a run so far (st->bestLikelihood* of the reference), per dwarf.
struct NbBestDev {
    double best[NB_LIKELIHOOD_TERMS];
    double timeEvolve;              // in: the dwarf's timeEvolve
    double bestTime;
    int bestStep, count, improved, pad;
};
// get_likelihood's update (nbody/src/nbody_plain.c:155-232) after step `step` of nStep, from
// the likelihoods in out; with keep, the improved dwarfs' bodies are copied to keepPos/keepVel
// (3n each, xyz interleaved).
void nb_launch_best_update(const double* out, NbBestDev* best, int D, int step, int nStep,
                           NbLikeFlags f, cudaStream_t s);
void nb_launch_keep_best(const NbBestDev* best, const int* bodyDwarf, const double* px,
                         const double* py, const double* pz, const double* vx, const double* vy,
                         const double* vz, int n, double* keepPos, double* keepVel, int numSMs,
                         cudaStream_t s);

// Launch accounting (all launches of this library go through nb_count_launch).
void nb_count_launch(int n = 1);

// ---- kernels-facing host entry points (implemented in the .cu files) ----
struct NbSortBuffers {
    unsigned long long* keyA; unsigned long long* keyB;
    unsigned int* idxA; unsigned int* idxB;
    unsigned int* hist;    // 256 * nTiles
    int* histTmp;          // tile sums of the scan over hist
    int capTiles;
};
// Sorts (keyA, idxA) by key in place (result in keyA/idxA); n items.
void nb_radix_sort(NbSortBuffers& b, int n, cudaStream_t s);
// Sorts (keyA, idxA) by (group[idx], key): the key passes, then two stable passes over the
// 16-bit group of each item's index (result in keyA/idxA).
void nb_radix_sort_grouped(NbSortBuffers& b, int n, const int* group, cudaStream_t s);
// Device buffers of one simulation.
struct NbTreeBuffers {
    double *px, *py, *pz, *vx, *vy, *vz, *ax, *ay, *az, *mass;
    NbSortBuffers sort;
    long long *gx, *gy, *gz;
    int *delta, *cum, *scanTmp, *bodyNode;
    double4* nodePM; double* nodeCrit; int2* nodeLink; double* nodeQuad;
    int *nodeDepth, *parent, *nchild, *arrive;
    int2* nodeRange;   // first and last sorted body of every node's subtree
    double4* walkRec;  // 3 per node: the FP64 walk's packed node records
    NbScalars* sc;
};

// FP32 node records of the mixed-precision walk.
struct NbMixedBuffers {
    float4* hi;    // {hi.x, hi.y, hi.z, rcrit2 (-inf for bodies)}
    float4* lo;    // {lo.x, lo.y, lo.z, mass}
    float4* q32;   // 2 per node: {xx, xy, xz, yy}, {yz, zz, 0, 0}
    int4* child8;  // 2 per node: up to 8 child indices of a cell (-1 = none)
    int* stacks;   // per resident warp: the group walk's depth-first stack
    int2* groups;  // walk groups: first sorted body, body count (<= 32)
    int walkBlocks;
    int groupMax;  // bodies per walk group, 1..64 (0: 32; above 32, two bodies per lane)
    int listCap;   // interaction-list entries per warp: 32, 64 or 128 (0: 64)
    int exact;     // 1: every lane takes exactly its own body's interaction set (groups <= 32)
};
int nb_mixed_walk_blocks(int numSMs, int listCap = 0, int groupMax = 32);
size_t nb_mixed_stack_ints(int blocks);

// The FP64 walks' packed node records (3 double4 per node) from the tree arrays.
void nb_launch_pack_walk(const double4* nodePM, const double* nodeCrit, const int2* nodeLink,
                         const double* nodeQuad, double4* rec, int capNodes, const NbScalars* sc,
                         cudaStream_t s);

// The walks (forest != nullptr: one tree per dwarf, see NbForest).  form: the FP64 walk's
// form, 0 the warp-union walk, 1 the walk per lane.
void nb_launch_walk_fp64(const double4* nodePM, const double* nodeCrit, const int2* nodeLink,
                         const double* nodeQuad, const unsigned* order, const double* px,
                         const double* py, const double* pz, double* ax, double* ay, double* az,
                         double* vx, double* vy, double* vz, const NbWalkParams& wp,
                         const NbPot& pot, NbScalars* sc, bool count, cudaStream_t s,
                         double4* walkRec, int capNodes, const NbForest* forest = nullptr,
                         int form = 0);
void nb_launch_walk_mixed(const NbTreeBuffers& b, const NbMixedBuffers& m, int capNodes,
                          const NbWalkParams& wp, const NbPot& pot, bool count, int numSMs,
                          cudaStream_t s, const NbForest* forest = nullptr);

void nb_build_tree(NbTreeBuffers& b, int n, int criterion, double theta, int useQuad, int drift,
                   double dt, int numSMs, cudaStream_t s, const double* shift = nullptr);
void nb_link_and_moments(NbTreeBuffers& b, int n, int capNodes, int criterion, double theta,
                         int useQuad, cudaStream_t s);
void nb_launch_drift_only(NbTreeBuffers& b, int n, double dt, int numSMs, cudaStream_t s,
                          const double* shift = nullptr);
// One half of the LMC's step (nb_lmc.cu): phase 0 drifts and kicks, phase 1 kicks; shift is
// the Milky Way's reflex acceleration of that half (3 host doubles).
void nb_launch_b_lmc_half(const NbBatchLMC& lmc, const NbForest& f, const NbScalars* sc, int phase,
                          cudaStream_t s);
void nb_launch_lmc_half(const NbPot& p, double* lmc, int phase, double dt, const double* shift,
                        double massLMC, int dynaFric, double coulombLog, cudaStream_t s);

// Inclusive prefix sum of n ints in place; tmp needs nb_scan_tmp_ints(n) ints.
int nb_scan_tmp_ints(int n);
void nb_inclusive_scan(int* data, int n, int* tmp, cudaStream_t s);
