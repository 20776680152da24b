// C ABI of the B200 step (include/nbody_b200.h): device state, marshalling and the
// host-side sequencing of the kernels of nbGravMap / nbStepSystem.
#include "nb_common.cuh"
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <algorithm>
#include <vector>

// ---- kernels defined in the other translation units ----
void nb_launch_direct_sample(const double* px, const double* py, const double* pz,
                             const double* mass, int n, const int* targets, int count,
                             double eps2, double* out, cudaStream_t s);
double nb_fma_probe(int fp64, int numSMs, cudaStream_t s);
void nb_launch_energy(const double* px, const double* py, const double* pz, const double* vx,
                      const double* vy, const double* vz, const double* mass, int n, double eps2,
                      const NbPot& pot, double* out, cudaStream_t s);
void nb_launch_vjp(NbTreeBuffers& b, double* nodeBar, int capNodes, int maxDepth, int criterion,
                   const NbWalkParams& wp, const NbPot& pot, const double* abar, double* xbar,
                   double* mbar, int numSMs, cudaEvent_t walkStart, cudaEvent_t walkEnd,
                   cudaStream_t s);
void nb_launch_step_adjoint(NbTreeBuffers& b, double* nodeBar, int capNodes, int maxDepth,
                            int criterion, const NbWalkParams& wp, const NbPot& pot, double dt,
                            const double* ak, double* xbar, double* vbar, double* mbar,
                            double* abarNext, double* dtbar, double* scratch, int numSMs,
                            cudaEvent_t walkStart, cudaEvent_t walkEnd, cudaStream_t s);
void nb_launch_direct_fp64(const double* px, const double* py, const double* pz,
                           const double* mass, double* ax, double* ay, double* az, double* vx,
                           double* vy, double* vz, const NbWalkParams& wp, const NbPot& pot,
                           NbScalars* sc, cudaStream_t s);
void nb_launch_ext_only(const double* dpos, double* dacc, int n, const NbPot& pot, cudaStream_t s);
int nb_launch_ic(const NBodyCudaMixedDwarf* host, int nD, const int* firsts, void* dTable,
                 double* scratch, NbTreeBuffers& b, int* types, int n, int numSMs, NbScalars* sc,
                 cudaStream_t s);
size_t nb_ic_table_bytes(int nD);
void nb_ic_particle_masses(const NBodyCudaMixedDwarf& h, double out[2]);

static std::atomic<unsigned long long> g_launches{0};
void nb_count_launch(int n) { g_launches.fetch_add((unsigned long long) n); }

thread_local std::string g_lastError;
static NBodyCudaStatus nb_cuda_fail(cudaError_t e, const char* what)
{
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    g_lastError = buf;
    return NBODY_CUDA_ERROR;
}
#define NB_CHECK(call)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return nb_cuda_fail(e_, #call);                \
    } while (0)

// 256-byte rounding of the pieces carved from one device allocation
static size_t nb_al(size_t x) { return (x + 255) & ~(size_t) 255; }

// ---- small kernels: SoA <-> interleaved / AoS Body ----
__global__ void k_split_xyz(const double* __restrict__ in, double* __restrict__ x,
                            double* __restrict__ y, double* __restrict__ z, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = in[3 * i]; y[i] = in[3 * i + 1]; z[i] = in[3 * i + 2];
    }
}
__global__ void k_join_xyz(const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, double* __restrict__ out, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[3 * i] = x[i]; out[3 * i + 1] = y[i]; out[3 * i + 2] = z[i];
    }
}
__global__ void k_from_bodies(const unsigned char* __restrict__ aos, double* px, double* py,
                              double* pz, double* vx, double* vy, double* vz, double* mass, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double* b = reinterpret_cast<const double*>(aos + (size_t) i * NBCUDA_BODY_STRIDE);
        px[i] = b[0]; py[i] = b[1]; pz[i] = b[2];
        mass[i] = b[NBCUDA_BODY_MASS_OFFSET / 8];
        vx[i] = b[NBCUDA_BODY_VEL_OFFSET / 8];
        vy[i] = b[NBCUDA_BODY_VEL_OFFSET / 8 + 1];
        vz[i] = b[NBCUDA_BODY_VEL_OFFSET / 8 + 2];
    }
}
// positions and velocities, six doubles per body (x y z vx vy vz), for the copy-out of
// nbMarshalBodiesCUDA, which writes them into the caller's Body records on the host
__global__ void k_to_posvel(double* __restrict__ out, const double* px, const double* py,
                            const double* pz, const double* vx, const double* vy,
                            const double* vz, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double* b = out + 6 * (size_t) i;
        b[0] = px[i]; b[1] = py[i]; b[2] = pz[i];
        b[3] = vx[i]; b[4] = vy[i]; b[5] = vz[i];
    }
}
// advanceVelocities alone, for a step whose force evaluation failed (the reference still
// kicks with the previous accelerations, nbody/src/nbody_plain.c:352-353).
__global__ void k_kick(double* vx, double* vy, double* vz, const double* ax, const double* ay,
                       const double* az, int n, double dtHalf, double sx, double sy, double sz)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        vx[i] = vx[i] + dtHalf * (ax[i] + sx);
        vy[i] = vy[i] + dtHalf * (ay[i] + sy);
        vz[i] = vz[i] + dtHalf * (az[i] + sz);
    }
}

// A saved force evaluation: the bodies (positions, velocities, accelerations, masses) and the
// tree the accelerations were computed with, for the reverse pass of the adjoint.
struct NbSlot {
    char* mem = nullptr;
    size_t bytes = 0;
    double* body = nullptr;             // 10 arrays of n: px py pz vx vy vz ax ay az mass
    unsigned* order = nullptr;          // sorted body order
    int* bodyNode = nullptr;
    double4* nodePM = nullptr;
    double* nodeCrit = nullptr;
    int2* nodeLink = nullptr;
    double* nodeQuad = nullptr;
    int* nodeDepth = nullptr;
    NbScalars sc{};
    double rsize = 0.0;
    int haveTree = 0, criterion = -1, step = 0, treeIncest = 0, valid = 0;
    double lmc[6] = {0, 0, 0, 0, 0, 0};   // the LMC's position and velocity (LMC runs)
};

// The FP64 walk forms the automatic choice times (nbSetWalkFormCUDA): 0 the warp union,
// 1 the walk per lane, 2 the walk per lane that loads the next node's record early.
static const int kWalkTuneForms[] = {0, 1, 2};
static const int kWalkTuneN = (int) (sizeof kWalkTuneForms / sizeof kWalkTuneForms[0]);

struct NBodyCudaState {
    int device = 0;
    int nbody = 0;
    int capBodies = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    NbTreeBuffers b{};
    NbMixedBuffers mx{};
    int capNodes = 0;
    NbScalars* scHost = nullptr;        // pinned mirror of the device scalars
    double* stage = nullptr;            // device staging: 3 doubles per body
    unsigned char* aos = nullptr;       // device staging for Body[] records
    size_t aosBytes = 0;
    double rsize = 4.0;                 // t->rsize carried between steps
    int step = 0;
    int treeIncest = 0;                 // st->treeIncest (sticky)
    int counting = 0;
    int haveTree = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;    // around the walk kernel
    cudaEvent_t evS = nullptr, evE = nullptr;    // around a whole force evaluation / step
    float walkMs = 0.0f;
    float stepMs = 0.0f;
    int walkLaunches = 0;
    unsigned long long cBB = 0, cBC = 0, cVisit = 0, cWarpSteps = 0;
    double* nodeBar = nullptr;          // adjoint: 10 doubles per node
    int nodeBarCap = 0;
    int lastCriterion = -1;             // criterion of the last force evaluation
    std::vector<NbSlot> slots;          // saved evaluations (nbSaveStateCUDA)
    double* adjScratch = nullptr;       // reverse step: 7 doubles per body
    int* types = nullptr;               // body types (+1 light, -1 dark), for histograms
    double timeOrigin = 0.0;            // st->previousForwardTime: barTime = step * dt - this
    int mixGroupMax = 32, mixListCap = 64, mixBlocksPerSM = 0;   // mixed-walk tuning
    int mixExact = 1;                   // 1: each body's own interaction set (nbSetMixedModeCUDA)
    char* histScratch = nullptr;        // histogram / likelihood buffers
    size_t histScratchBytes = 0;
    double* lmcDev = nullptr;           // the LMC's {pos, vel} (nbSetLMCCUDA)
    std::vector<double> lmcShift;       // shiftByLMC: 3 doubles per step
    NbSlot runStart;                    // nbRunSystemCUDA: the initial state of the runs
    NbBestDev* best = nullptr;          // nbRunSystemCUDA: device best-likelihood record
    // the step replayed as one captured CUDA graph (nb_force, tree criteria without an orbiting
    // bar or an LMC): the graph, what it was captured for, and the pinned per-evaluation
    // scalars its first copy uploads
    cudaGraphExec_t stepGraph = nullptr;
    NBodyCudaCtx stepGraphCtx{};
    int stepGraphDrift = -1, stepGraphKick = -1, stepGraphCap = -1;
    int stepGraphMx[4] = {0, 0, 0, 0};
    unsigned long long stepGraphLaunches = 0;
    int useStepGraph = 1;
    int stepGraphForm = -1;
    NbScalars* scInit = nullptr;
    // the FP64 walk's form (nbSetWalkFormCUDA): -1 chooses by timing -- the first 2C uncounted
    // FP64 tree evaluations cycle twice through the C candidate forms, the second round (past
    // each kernel's first launch, which also loads it) is timed, the fastest form is kept
    int walkForm = -1;
    int walkFormChosen = -1;
    int walkTuneStep = 0;
    float walkFormMs[8] = {-1.0f, -1.0f, -1.0f, -1.0f, -1.0f, -1.0f, -1.0f, -1.0f};
    double* keepPos = nullptr;          // bodies at the best likelihood (3n each)
    double* keepVel = nullptr;
    int haveKeep = 0;
};

template <typename T>
static cudaError_t nb_alloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void**) p, count * sizeof(T));
}

static void nb_drop_step_graph(NBodyCudaState* st)
{
    if (st->stepGraph) cudaGraphExecDestroy(st->stepGraph);
    st->stepGraph = nullptr;
    st->stepGraphCap = -1;
}

static void nb_free_nodes(NBodyCudaState* st)
{
    nb_drop_step_graph(st);             // its kernels hold the node arrays' addresses
    NbTreeBuffers& b = st->b;
    cudaFree(b.nodePM); cudaFree(b.nodeCrit); cudaFree(b.nodeLink); cudaFree(b.nodeQuad);
    cudaFree(b.nodeDepth); cudaFree(b.parent); cudaFree(b.nchild); cudaFree(b.arrive);
    cudaFree(b.nodeRange); b.nodeRange = nullptr;
    cudaFree(b.walkRec); b.walkRec = nullptr;
    cudaFree(st->mx.groups);
    cudaFree(st->mx.hi); cudaFree(st->mx.lo); cudaFree(st->mx.q32); cudaFree(st->mx.child8);
    b.nodePM = nullptr; b.nodeCrit = nullptr; b.nodeLink = nullptr; b.nodeQuad = nullptr;
    b.nodeDepth = b.parent = b.nchild = b.arrive = nullptr;
    int* stacks = st->mx.stacks;
    const int wb = st->mx.walkBlocks;
    st->mx = NbMixedBuffers{};
    st->mx.stacks = stacks;          // the walk stacks do not depend on the node count
    st->mx.walkBlocks = wb;
    st->capNodes = 0;
}

static NBodyCudaStatus nb_alloc_nodes(NBodyCudaState* st, int cap)
{
    nb_free_nodes(st);
    NbTreeBuffers& b = st->b;
    NB_CHECK(nb_alloc(&b.nodePM, cap));
    NB_CHECK(nb_alloc(&b.nodeCrit, cap));
    NB_CHECK(nb_alloc(&b.nodeLink, cap));
    NB_CHECK(nb_alloc(&b.nodeQuad, 6 * (size_t) cap));
    NB_CHECK(nb_alloc(&b.nodeDepth, cap));
    NB_CHECK(nb_alloc(&b.parent, cap));
    NB_CHECK(nb_alloc(&b.nchild, cap));
    NB_CHECK(nb_alloc(&b.arrive, cap));
    NB_CHECK(nb_alloc(&b.nodeRange, cap));
    NB_CHECK(nb_alloc(&b.walkRec, 3 * (size_t) cap));
    NB_CHECK(nb_alloc(&st->mx.groups, cap));
    NB_CHECK(nb_alloc(&st->mx.hi, cap));
    NB_CHECK(nb_alloc(&st->mx.lo, cap));
    NB_CHECK(nb_alloc(&st->mx.q32, 2 * (size_t) cap));
    NB_CHECK(nb_alloc(&st->mx.child8, 2 * (size_t) cap));
    st->capNodes = cap;
    return NBODY_SUCCESS;
}

static NBodyCudaStatus nb_alloc_bodies(NBodyCudaState* st, int n)
{
    NbTreeBuffers& b = st->b;
    const size_t N = (size_t) (n > 0 ? n : 1);
    NB_CHECK(nb_alloc(&b.px, N)); NB_CHECK(nb_alloc(&b.py, N)); NB_CHECK(nb_alloc(&b.pz, N));
    NB_CHECK(nb_alloc(&b.vx, N)); NB_CHECK(nb_alloc(&b.vy, N)); NB_CHECK(nb_alloc(&b.vz, N));
    NB_CHECK(nb_alloc(&b.ax, N)); NB_CHECK(nb_alloc(&b.ay, N)); NB_CHECK(nb_alloc(&b.az, N));
    NB_CHECK(nb_alloc(&b.mass, N));
    NB_CHECK(cudaMemsetAsync(b.ax, 0, N * sizeof(double), st->stream));
    NB_CHECK(cudaMemsetAsync(b.ay, 0, N * sizeof(double), st->stream));
    NB_CHECK(cudaMemsetAsync(b.az, 0, N * sizeof(double), st->stream));
    NB_CHECK(nb_alloc(&b.sort.keyA, N)); NB_CHECK(nb_alloc(&b.sort.keyB, N));
    NB_CHECK(nb_alloc(&b.sort.idxA, N)); NB_CHECK(nb_alloc(&b.sort.idxB, N));
    const int tiles = (int) ((N + 2047) / 2048);
    NB_CHECK(nb_alloc(&b.sort.hist, 256 * (size_t) tiles));
    NB_CHECK(nb_alloc(&b.sort.histTmp, (size_t) nb_scan_tmp_ints(256 * tiles)));
    b.sort.capTiles = tiles;
    NB_CHECK(nb_alloc(&b.gx, N)); NB_CHECK(nb_alloc(&b.gy, N)); NB_CHECK(nb_alloc(&b.gz, N));
    NB_CHECK(nb_alloc(&b.delta, N)); NB_CHECK(nb_alloc(&b.cum, N));
    NB_CHECK(nb_alloc(&b.scanTmp, (size_t) nb_scan_tmp_ints((int) N)));
    NB_CHECK(nb_alloc(&b.bodyNode, N));
    NB_CHECK(nb_alloc(&st->stage, 3 * N + 3));
    st->capBodies = (int) N;
    return nb_alloc_nodes(st, 2 * (int) N + 64);
}

static void nb_free_all(NBodyCudaState* st)
{
    NbTreeBuffers& b = st->b;
    double* d[] = {b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.ax, b.ay, b.az, b.mass, st->stage};
    for (double* p : d) cudaFree(p);
    cudaFree(b.sort.keyA); cudaFree(b.sort.keyB); cudaFree(b.sort.idxA); cudaFree(b.sort.idxB);
    cudaFree(b.sort.hist); cudaFree(b.sort.histTmp);
    cudaFree(b.gx); cudaFree(b.gy); cudaFree(b.gz);
    cudaFree(b.delta); cudaFree(b.cum); cudaFree(b.scanTmp); cudaFree(b.bodyNode);
    cudaFree(b.sc);
    cudaFree(st->aos);
    nb_free_nodes(st);
    cudaFree(st->mx.stacks);
    st->mx.stacks = nullptr;
    cudaFree(st->nodeBar);
    st->nodeBar = nullptr;
    for (NbSlot& sl : st->slots) cudaFree(sl.mem);
    st->slots.clear();
    cudaFree(st->adjScratch);
    st->adjScratch = nullptr;
    cudaFree(st->types);
    st->types = nullptr;
    cudaFree(st->histScratch);
    st->histScratch = nullptr;
    cudaFree(st->runStart.mem);
    st->runStart = NbSlot{};
    cudaFree(st->lmcDev);
    st->lmcDev = nullptr;
    cudaFree(st->best);
    st->best = nullptr;
    cudaFree(st->keepPos);
    cudaFree(st->keepVel);
    st->keepPos = st->keepVel = nullptr;
    if (st->scHost) cudaFreeHost(st->scHost);
    if (st->scInit) cudaFreeHost(st->scInit);
    if (st->ev0) cudaEventDestroy(st->ev0);
    if (st->ev1) cudaEventDestroy(st->ev1);
    if (st->evS) cudaEventDestroy(st->evS);
    if (st->evE) cudaEventDestroy(st->evE);
    if (st->stream) cudaStreamDestroy(st->stream);
}

NbPot nb_pot_from(const NBodyCudaCtx* c)
{
    NbPot p{};
    p.enabled = c->potentialType == NBCUDA_POTENTIAL_DEFAULT;
    p.sphType = c->pot.sphere.type; p.sphMass = c->pot.sphere.mass; p.sphScale = c->pot.sphere.scale;
    p.diskType = c->pot.disk.type; p.diskMass = c->pot.disk.mass;
    p.diskA = c->pot.disk.scaleLength; p.diskB = c->pot.disk.scaleHeight;
    p.disk2Type = c->pot.disk2.type; p.disk2Mass = c->pot.disk2.mass;
    p.disk2A = c->pot.disk2.scaleLength; p.disk2B = c->pot.disk2.scaleHeight;
    p.haloType = c->pot.halo.type; p.haloV = c->pot.halo.vhalo;
    p.haloA = c->pot.halo.scaleLength; p.haloQz = c->pot.halo.flattenZ;
    p.haloMass = c->pot.halo.mass; p.haloGamma = c->pot.halo.gamma;
    p.haloLambda = c->pot.halo.lambda; p.haloRho0 = c->pot.halo.rho0;
    p.haloC1 = c->pot.halo.c1; p.haloC2 = c->pot.halo.c2; p.haloC3 = c->pot.halo.c3;
    p.disk2Pattern = c->pot.disk2.patternSpeed; p.disk2StartAngle = c->pot.disk2.startAngle;
    p.time = 0.0;
    return p;
}

static bool nb_pow2(double x)
{
    int e;
    return x > 0.0 && std::isfinite(x) && std::frexp(x, &e) == 0.5;
}

// Options this implementation evaluates on the GPU; anything else is NBODY_UNSUPPORTED,
// as the reference's OpenCL path does for a custom Lua potential (nbody_types.c:297-301).
NBodyCudaStatus nb_check_ctx(const NBodyCudaCtx* c, std::string& why)
{
    if (!c) { why = "null context"; return NBODY_USER_ERROR; }
    if (c->criterion < NBCUDA_TREECODE || c->criterion > NBCUDA_EXACT) { why = "invalid criterion"; return NBODY_USER_ERROR; }
    if (c->precision != NBCUDA_PRECISION_FP64 && c->precision != NBCUDA_PRECISION_MIXED) { why = "invalid precision"; return NBODY_USER_ERROR; }
    if (c->potentialType == NBCUDA_POTENTIAL_CUSTOM_LUA) { why = "custom Lua potential"; return NBODY_UNSUPPORTED; }
    if (c->potentialType == NBCUDA_POTENTIAL_DEFAULT) {
        const NBodyCudaPotential& p = c->pot;
        if (p.sphere.type != NBCUDA_NO_SPHERICAL && p.sphere.type != NBCUDA_HERNQUIST_SPHERICAL &&
            p.sphere.type != NBCUDA_PLUMMER_SPHERICAL) { why = "bulge type"; return NBODY_UNSUPPORTED; }
        if (p.disk.type != NBCUDA_NO_DISK && p.disk.type != NBCUDA_MIYAMOTO_NAGAI_DISK) { why = "disk type"; return NBODY_UNSUPPORTED; }
        if (p.disk2.type != NBCUDA_NO_DISK && p.disk2.type != NBCUDA_MIYAMOTO_NAGAI_DISK &&
            p.disk2.type != NBCUDA_ORBITING_BAR) { why = "disk2 type"; return NBODY_UNSUPPORTED; }
        // every halo of the reference
        if (p.halo.type < NBCUDA_NO_HALO || p.halo.type > NBCUDA_NINKOVIC_HALO) {
            why = "halo type";
            return NBODY_UNSUPPORTED;
        }
    }
    if (c->lmc && c->potentialType != NBCUDA_POTENTIAL_DEFAULT) {
        why = "the LMC moves in the default (Milky Way) potential";
        return NBODY_USER_ERROR;
    }
    return NBODY_SUCCESS;
}

// Potentials whose Jacobian (the adjoint's dual numbers) and potential energy are implemented:
// Miyamoto-Nagai disks, logarithmic and NFW halos, Hernquist and Plummer bulges.
static bool nb_pot_basic(const NBodyCudaCtx* c, std::string& why)
{
    if (c->lmc) {
        why = "not implemented with an LMC";
        return false;
    }
    if (c->potentialType != NBCUDA_POTENTIAL_DEFAULT) return true;
    const int d2 = c->pot.disk2.type, h = c->pot.halo.type;
    if ((d2 == NBCUDA_NO_DISK || d2 == NBCUDA_MIYAMOTO_NAGAI_DISK) &&
        (h == NBCUDA_NO_HALO || h == NBCUDA_LOGARITHMIC_HALO || h == NBCUDA_NFW_HALO))
        return true;
    why = "implemented for Miyamoto-Nagai disks, logarithmic/NFW halos and Hernquist/Plummer bulges";
    return false;
}

static int nb_blocks(NBodyCudaState* st, int n)
{
    int g = (n + 255) / 256;
    int cap = st->numSMs * 8;
    if (g < 1) g = 1;
    return g < cap ? g : cap;
}

// One force evaluation; drift/kick select the fused halves of the leapfrog.  allowGraph: the
// evaluation may be replayed from a captured CUDA graph (the same kernels in the same order,
// launched as one graph instead of ~60 launches; used for whole steps).
static NBodyCudaStatus nb_force(const NBodyCudaCtx* ctx, NBodyCudaState* st, int drift, int kick,
                                bool allowGraph = false)
{
    std::string why;
    NBodyCudaStatus rc = nb_check_ctx(ctx, why);
    if (rc) { g_lastError = why; return rc; }
    if (ctx->criterion != NBCUDA_EXACT && !nb_pow2(st->rsize)) {
        g_lastError = "root size must be a power of two";
        return NBODY_UNSUPPORTED;
    }
    NB_CHECK(cudaSetDevice(st->device));
    const int n = st->nbody;
    const cudaStream_t s = st->stream;
    NbTreeBuffers& b = st->b;
    NbPot pot = nb_pot_from(ctx);
    pot.time = st->step * ctx->timestep - st->timeOrigin;   // barTime (nbody/src/nbody_grav.c:141)
    NbWalkParams wp{};
    wp.eps2 = ctx->eps2;
    wp.dtHalf = 0.5 * ctx->timestep;
    wp.useQuad = ctx->useQuad;
    wp.kick = kick;
    wp.n = n;
    const bool mixed = ctx->precision == NBCUDA_PRECISION_MIXED;
    // the LMC (nbody/src/nbody_plain.c:329-360): its state, the step's reflex accelerations
    const bool lmc = ctx->lmc != 0;
    double shift0[3] = {0.0, 0.0, 0.0}, shift1[3] = {0.0, 0.0, 0.0};
    if (lmc) {
        if (!st->lmcDev) {
            g_lastError = "an LMC context needs the LMC's state (nbSetLMCCUDA)";
            return NBODY_USER_ERROR;
        }
        pot.lmc = st->lmcDev;
        pot.lmcMass = ctx->lmcMass;
        pot.lmcScale = ctx->lmcScale;
        if (drift || kick) {
            const size_t k = (size_t) st->step;
            if (3 * (k + 2) > st->lmcShift.size()) {
                g_lastError = "the LMC's reflex accelerations do not reach this step";
                return NBODY_USER_ERROR;
            }
            for (int c = 0; c < 3; ++c) {
                shift0[c] = st->lmcShift[3 * k + c];
                shift1[c] = st->lmcShift[3 * (k + 1) + c];
            }
        }
        for (int c = 0; c < 3; ++c) wp.shift[c] = shift1[c];
        if (drift)                      // advancePosVel_LMC with the acceleration at its state
            nb_launch_lmc_half(pot, st->lmcDev, 0, ctx->timestep, shift0, ctx->lmcMass,
                               ctx->lmcDynaFric, ctx->coulombLog, s);
    }

    if (mixed) {
        if (!st->mx.stacks) {
            // stacks for the largest persistent grid any list capacity allows
            int mxb = 0;
            for (int cap : {32, 64, 128})
                for (int gm : {32, 64})
                    mxb = std::max(mxb, nb_mixed_walk_blocks(st->numSMs, cap, gm));
            NB_CHECK(nb_alloc(&st->mx.stacks, nb_mixed_stack_ints(mxb)));
        }
        const int fit = nb_mixed_walk_blocks(st->numSMs, st->mixListCap, st->mixGroupMax) / st->numSMs;
        const int per = st->mixBlocksPerSM > 0 ? std::min(st->mixBlocksPerSM, fit) : fit;
        st->mx.walkBlocks = std::max(1, per) * st->numSMs;
        st->mx.groupMax = st->mixGroupMax;
        st->mx.listCap = st->mixListCap;
        st->mx.exact = st->mixExact;
    }
    // the FP64 walk's form for this evaluation (its timing decides the automatic choice)
    const bool fp64Tree = !mixed && ctx->criterion != NBCUDA_EXACT;
    int form = 0;
    bool tuning = false;
    if (fp64Tree) {
        if (st->walkForm >= 0) form = st->walkForm;
        else if (st->walkFormChosen >= 0) form = st->walkFormChosen;
        else { form = kWalkTuneForms[st->walkTuneStep % kWalkTuneN]; tuning = !st->counting; }
    }
    // The device work of the evaluation, enqueued without host synchronisation: the scalars
    // from the pinned st->scInit, the tree or the direct sum, the walk, the scalars back into
    // st->scHost.  capturing: inside a stream capture (events become graph nodes).
    auto enqueue = [&](bool capturing) {
        auto rec = [&](cudaEvent_t ev) {
            if (capturing) cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal);
            else cudaEventRecord(ev, s);
        };
        cudaMemcpyAsync(b.sc, st->scInit, sizeof(NbScalars), cudaMemcpyHostToDevice, s);
        rec(st->evS);
        if (ctx->criterion == NBCUDA_EXACT) {
            if (drift) {
                // advancePosVel without the tree: reuse the bounding-box pass for the drift
                nb_launch_drift_only(b, n, ctx->timestep, st->numSMs, s, shift0);
            }
            rec(st->ev0);
            nb_launch_direct_fp64(b.px, b.py, b.pz, b.mass, b.ax, b.ay, b.az, b.vx, b.vy, b.vz, wp,
                                  pot, b.sc, s);
            rec(st->ev1);
        } else {
            nb_build_tree(b, n, ctx->criterion, ctx->theta, ctx->useQuad, drift, ctx->timestep,
                          st->numSMs, s, shift0);
            nb_link_and_moments(b, n, st->capNodes, ctx->criterion, ctx->theta, ctx->useQuad, s);
            rec(st->ev0);
            if (mixed)
                nb_launch_walk_mixed(b, st->mx, st->capNodes, wp, pot, st->counting != 0,
                                     st->numSMs, s);
            else
                nb_launch_walk_fp64(b.nodePM, b.nodeCrit, b.nodeLink, b.nodeQuad, b.sort.idxA, b.px,
                                    b.py, b.pz, b.ax, b.ay, b.az, b.vx, b.vy, b.vz, wp, pot, b.sc,
                                    st->counting != 0, s, b.walkRec, st->capNodes, nullptr,
                                    form);
            rec(st->ev1);
        }
        rec(st->evE);
        cudaMemcpyAsync(st->scHost, b.sc, sizeof(NbScalars), cudaMemcpyDeviceToHost, s);
    };
    // the orbiting bar's time and an LMC's reflex accelerations change every step and are
    // kernel arguments: those evaluations are launched directly
    const bool graphable = allowGraph && st->useStepGraph && ctx->criterion != NBCUDA_EXACT &&
                           !lmc && !st->counting && ctx->pot.disk.type != NBCUDA_ORBITING_BAR &&
                           ctx->pot.disk2.type != NBCUDA_ORBITING_BAR;

    for (int attempt = 0; attempt < 4; ++attempt) {
        // reset per-evaluation device scalars (keep rsize)
        *st->scInit = NbScalars{};
        st->scInit->rsize = st->rsize;
        st->scInit->capNodes = st->capNodes;
        st->walkLaunches = 1;
        if (graphable) {
            const int mxKey[4] = {mixed ? st->mx.walkBlocks : 0, mixed ? st->mx.groupMax : 0,
                                  mixed ? st->mx.listCap : 0, mixed ? st->mx.exact : 0};
            const bool same = st->stepGraph && st->stepGraphDrift == drift &&
                              st->stepGraphKick == kick && st->stepGraphCap == st->capNodes &&
                              st->stepGraphForm == form &&
                              std::memcmp(st->stepGraphMx, mxKey, sizeof mxKey) == 0 &&
                              std::memcmp(&st->stepGraphCtx, ctx, sizeof *ctx) == 0;
            if (!same) {
                nb_drop_step_graph(st);
                const unsigned long long l0 = g_launches.load();
                cudaGraph_t g = nullptr;
                NB_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                enqueue(true);
                cudaError_t e = cudaStreamEndCapture(s, &g);
                if (e == cudaSuccess) e = cudaGraphInstantiate(&st->stepGraph, g, 0);
                if (g) cudaGraphDestroy(g);
                if (e != cudaSuccess) {
                    st->stepGraph = nullptr;
                    return nb_cuda_fail(e, "step graph capture");
                }
                st->stepGraphLaunches = g_launches.load() - l0;
                st->stepGraphCtx = *ctx;
                st->stepGraphDrift = drift;
                st->stepGraphKick = kick;
                st->stepGraphCap = st->capNodes;
                st->stepGraphForm = form;
                std::memcpy(st->stepGraphMx, mxKey, sizeof mxKey);
            } else {
                nb_count_launch((int) st->stepGraphLaunches);
            }
            NB_CHECK(cudaGraphLaunch(st->stepGraph, s));
        } else {
            enqueue(false);
        }
        st->haveTree = ctx->criterion != NBCUDA_EXACT;
        NB_CHECK(cudaGetLastError());
        NB_CHECK(cudaStreamSynchronize(s));
        NbScalars& h = *st->scHost;
        st->rsize = h.rsize;
        if (h.status & NBODY_CELL_OVERFLOW_ERROR) {
            // grow the node arrays and redo this evaluation (positions already drifted)
            int need = h.neededNodes + h.neededNodes / 4 + 64;
            rc = nb_alloc_nodes(st, need);
            if (rc) return rc;
            drift = 0;
            continue;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, st->ev0, st->ev1);
        st->walkMs = ms;
        if (tuning && !(h.status & ~(int) NBODY_STATUS_WARNINGS_MASK)) {
            const int c = st->walkTuneStep % kWalkTuneN;
            if (st->walkTuneStep >= kWalkTuneN) st->walkFormMs[c] = ms;
            if (++st->walkTuneStep == 2 * kWalkTuneN) {
                int best = 0;
                for (int k = 1; k < kWalkTuneN; ++k)
                    if (st->walkFormMs[k] < st->walkFormMs[best]) best = k;
                st->walkFormChosen = kWalkTuneForms[best];
            }
        }
        ms = 0.0f;
        cudaEventElapsedTime(&ms, st->evS, st->evE);
        st->stepMs = ms;
        st->cBB = h.nBodyBody; st->cBC = h.nBodyCell; st->cVisit = h.nVisit;
        st->cWarpSteps = h.nWarpSteps;
        NBodyCudaStatus out = h.status;
        if ((out & ~(int) NBODY_STATUS_WARNINGS_MASK) == 0) {
            if (h.incest) st->treeIncest = 1;
        } else if (kick) {
            // the failed evaluation left the accelerations untouched; the reference still
            // applies advanceVelocities with them
            k_kick<<<nb_blocks(st, n), 256, 0, s>>>(b.vx, b.vy, b.vz, b.ax, b.ay, b.az, n, wp.dtHalf,
                                                    shift1[0], shift1[1], shift1[2]);
            nb_count_launch();
            NB_CHECK(cudaStreamSynchronize(s));
        }
        if (lmc && kick) {               // advanceVelocities_LMC after the bodies' kick
            nb_launch_lmc_half(pot, st->lmcDev, 1, ctx->timestep, shift1, ctx->lmcMass,
                               ctx->lmcDynaFric, ctx->coulombLog, s);
            NB_CHECK(cudaGetLastError());
        }
        if (st->treeIncest)
            out |= ctx->allowIncest ? NBODY_TREE_INCEST_NONFATAL : NBODY_TREE_INCEST_FATAL;
        st->lastCriterion = ctx->criterion;
        return out;
    }
    g_lastError = "node capacity could not be grown";
    return NBODY_CELL_OVERFLOW_ERROR;
}

extern "C" {

NBodyCudaStatus nbInitCUDA(NBodyCudaState** out, int device, int nbody)
{
    if (!out || nbody < 0) return NBODY_USER_ERROR;
    *out = nullptr;
    int count = 0;
    NB_CHECK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) { g_lastError = "no such CUDA device"; return NBODY_CUDA_ERROR; }
    NB_CHECK(cudaSetDevice(device));
    NBodyCudaState* st = new NBodyCudaState();
    st->device = device;
    st->nbody = nbody;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) st->numSMs = prop.multiProcessorCount;
    NBodyCudaStatus rc = NBODY_SUCCESS;
    cudaError_t e = cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&st->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&st->ev1);
    if (e == cudaSuccess) e = cudaEventCreate(&st->evS);
    if (e == cudaSuccess) e = cudaEventCreate(&st->evE);
    if (e == cudaSuccess) e = cudaMallocHost((void**) &st->scHost, sizeof(NbScalars));
    if (e == cudaSuccess) e = cudaMallocHost((void**) &st->scInit, sizeof(NbScalars));
    if (e == cudaSuccess) e = cudaMalloc((void**) &st->b.sc, sizeof(NbScalars));
    if (e != cudaSuccess) rc = nb_cuda_fail(e, "nbInitCUDA");
    if (!rc) rc = nb_alloc_bodies(st, nbody);
    if (rc) { nb_free_all(st); delete st; return rc; }
    *out = st;
    return NBODY_SUCCESS;
}

void nbDestroyCUDA(NBodyCudaState* st)
{
    if (!st) return;
    cudaSetDevice(st->device);
    if (st->stream) cudaStreamSynchronize(st->stream);
    nb_free_all(st);
    delete st;
}

static NBodyCudaStatus nb_reset_run(NBodyCudaState* st, double treeRSize)
{
    if (!(treeRSize > 0.0) || !nb_pow2(treeRSize)) {
        g_lastError = "treeRSize must be a positive power of two";
        return NBODY_UNSUPPORTED;
    }
    st->rsize = treeRSize;
    st->step = 0;
    st->treeIncest = 0;
    st->haveTree = 0;
    return NBODY_SUCCESS;
}

static bool nb_is_pinned(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeHost;
}

NBodyCudaStatus nbMarshalBodiesCUDA(NBodyCudaState* st, void* bodytab, int nbody, int toDevice,
                                    double treeRSize)
{
    if (!st || !bodytab || nbody != st->nbody) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    const size_t bytes = (size_t) nbody * NBCUDA_BODY_STRIDE;
    if (st->aosBytes < bytes) {
        cudaFree(st->aos);
        st->aos = nullptr;
        NB_CHECK(cudaMalloc((void**) &st->aos, bytes ? bytes : 1));
        st->aosBytes = bytes;
    }
    NbTreeBuffers& b = st->b;
    const cudaStream_t s = st->stream;
    if (toDevice) {
        NBodyCudaStatus rc = nb_reset_run(st, treeRSize);
        if (rc) return rc;
        if (nbody) {
            NB_CHECK(cudaMemcpyAsync(st->aos, bodytab, bytes, cudaMemcpyHostToDevice, s));
            k_from_bodies<<<nb_blocks(st, nbody), 256, 0, s>>>(st->aos, b.px, b.py, b.pz, b.vx, b.vy,
                                                                b.vz, b.mass, nbody);
            nb_count_launch();
        }
    } else if (nbody) {
        // only pos and vel of the caller's records change (mass, type, id and the rest of each
        // record are the caller's): stage them compactly, then scatter on the host
        k_to_posvel<<<nb_blocks(st, nbody), 256, 0, s>>>((double*) st->aos, b.px, b.py, b.pz,
                                                          b.vx, b.vy, b.vz, nbody);
        nb_count_launch();
        std::vector<double> pv(6 * (size_t) nbody);
        NB_CHECK(cudaMemcpyAsync(pv.data(), st->aos, pv.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
        NB_CHECK(cudaGetLastError());
        NB_CHECK(cudaStreamSynchronize(s));
        unsigned char* rec = (unsigned char*) bodytab;
        for (size_t i = 0; i < (size_t) nbody; ++i) {
            memcpy(rec + i * NBCUDA_BODY_STRIDE + NBCUDA_BODY_POS_OFFSET, &pv[6 * i], 3 * sizeof(double));
            memcpy(rec + i * NBCUDA_BODY_STRIDE + NBCUDA_BODY_VEL_OFFSET, &pv[6 * i + 3], 3 * sizeof(double));
        }
        return NBODY_SUCCESS;
    }
    NB_CHECK(cudaGetLastError());
    NB_CHECK(cudaStreamSynchronize(s));
    return NBODY_SUCCESS;
}

static NBodyCudaStatus nb_upload3(NBodyCudaState* st, const double* host, double* x, double* y,
                                  double* z, int n)
{
    if (!n) return NBODY_SUCCESS;
    const size_t bytes = 3 * (size_t) n * sizeof(double);
    NB_CHECK(cudaMemcpyAsync(st->stage, host, bytes, cudaMemcpyHostToDevice, st->stream));
    k_split_xyz<<<nb_blocks(st, n), 256, 0, st->stream>>>(st->stage, x, y, z, n);
    nb_count_launch();
    if (!nb_is_pinned(host)) NB_CHECK(cudaStreamSynchronize(st->stream));
    return NBODY_SUCCESS;
}

static NBodyCudaStatus nb_download3(NBodyCudaState* st, double* host, const double* x,
                                    const double* y, const double* z, int n)
{
    if (!n) return NBODY_SUCCESS;
    k_join_xyz<<<nb_blocks(st, n), 256, 0, st->stream>>>(x, y, z, st->stage, n);
    nb_count_launch();
    NB_CHECK(cudaMemcpyAsync(host, st->stage, 3 * (size_t) n * sizeof(double),
                             cudaMemcpyDeviceToHost, st->stream));
    return NBODY_SUCCESS;          // the caller synchronises (stream order protects the stage)
}

NBodyCudaStatus nbSetBodiesCUDA(NBodyCudaState* st, const double* pos, const double* vel,
                                const double* mass, int nbody, double treeRSize)
{
    if (!st || nbody != st->nbody || (nbody && (!pos || !vel || !mass))) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    NBodyCudaStatus rc = nb_reset_run(st, treeRSize);
    if (rc) return rc;
    NbTreeBuffers& b = st->b;
    rc = nb_upload3(st, pos, b.px, b.py, b.pz, nbody);
    if (rc) return rc;
    rc = nb_upload3(st, vel, b.vx, b.vy, b.vz, nbody);
    if (rc) return rc;
    if (nbody) NB_CHECK(cudaMemcpyAsync(b.mass, mass, (size_t) nbody * sizeof(double),
                                        cudaMemcpyHostToDevice, st->stream));
    NB_CHECK(cudaStreamSynchronize(st->stream));
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbGetBodiesCUDA(NBodyCudaState* st, double* pos, double* vel)
{
    if (!st) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    NbTreeBuffers& b = st->b;
    NBodyCudaStatus rc = NBODY_SUCCESS;
    if (pos) rc = nb_download3(st, pos, b.px, b.py, b.pz, st->nbody);
    if (!rc && vel) rc = nb_download3(st, vel, b.vx, b.vy, b.vz, st->nbody);
    if (!rc) NB_CHECK(cudaStreamSynchronize(st->stream));
    return rc;
}

NBodyCudaStatus nbGetAccelsCUDA(NBodyCudaState* st, double* acc)
{
    if (!st || !acc) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    NBodyCudaStatus rc = nb_download3(st, acc, st->b.ax, st->b.ay, st->b.az, st->nbody);
    if (!rc) NB_CHECK(cudaStreamSynchronize(st->stream));
    return rc;
}

NBodyCudaStatus nbSetBodiesDeviceCUDA(NBodyCudaState* st, const double* dpos, const double* dvel,
                                      const double* dmass, int nbody, double treeRSize)
{
    if (!st || nbody != st->nbody) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    NBodyCudaStatus rc = nb_reset_run(st, treeRSize);
    if (rc) return rc;
    if (!nbody) return NBODY_SUCCESS;
    NbTreeBuffers& b = st->b;
    const cudaStream_t s = st->stream;
    k_split_xyz<<<nb_blocks(st, nbody), 256, 0, s>>>(dpos, b.px, b.py, b.pz, nbody);
    k_split_xyz<<<nb_blocks(st, nbody), 256, 0, s>>>(dvel, b.vx, b.vy, b.vz, nbody);
    nb_count_launch(2);
    NB_CHECK(cudaMemcpyAsync(b.mass, dmass, (size_t) nbody * sizeof(double),
                             cudaMemcpyDeviceToDevice, s));
    NB_CHECK(cudaGetLastError());
    NB_CHECK(cudaStreamSynchronize(s));
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbGetBodiesDeviceCUDA(NBodyCudaState* st, double* dpos, double* dvel, double* dacc)
{
    if (!st) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    NbTreeBuffers& b = st->b;
    const cudaStream_t s = st->stream;
    const int n = st->nbody;
    if (!n) return NBODY_SUCCESS;
    if (dpos) k_join_xyz<<<nb_blocks(st, n), 256, 0, s>>>(b.px, b.py, b.pz, dpos, n);
    if (dvel) k_join_xyz<<<nb_blocks(st, n), 256, 0, s>>>(b.vx, b.vy, b.vz, dvel, n);
    if (dacc) k_join_xyz<<<nb_blocks(st, n), 256, 0, s>>>(b.ax, b.ay, b.az, dacc, n);
    nb_count_launch((dpos != nullptr) + (dvel != nullptr) + (dacc != nullptr));
    NB_CHECK(cudaGetLastError());
    NB_CHECK(cudaStreamSynchronize(s));
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbGravMapCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st)
{
    if (!st) return NBODY_USER_ERROR;
    return nb_force(ctx, st, 0, 0);
}

NBodyCudaStatus nbStepSystemCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st)
{
    if (!st) return NBODY_USER_ERROR;
    NBodyCudaStatus rc = nb_force(ctx, st, 1, 1, true);
    if (!(rc & (NBODY_USER_ERROR | NBODY_UNSUPPORTED | NBODY_CUDA_ERROR))) st->step++;
    return rc;
}

NBodyCudaStatus nbRunStepsCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st, int nsteps)
{
    if (!st || nsteps < 0) return NBODY_USER_ERROR;
    NBodyCudaStatus all = NBODY_SUCCESS;
    float walkMs = 0.0f, stepMs = 0.0f;
    for (int k = 0; k < nsteps; ++k) {
        NBodyCudaStatus rc = nbStepSystemCUDA(ctx, st);
        walkMs += st->walkMs;
        stepMs += st->stepMs;
        all |= rc;
        if (rc & ~(int) NBODY_STATUS_WARNINGS_MASK) break;
    }
    st->walkMs = walkMs;
    st->stepMs = stepMs;
    st->walkLaunches = nsteps;
    return all;
}

NBodyCudaStatus nbMakeTreeCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st)
{
    if (!st) return NBODY_USER_ERROR;
    std::string why;
    NBodyCudaStatus rc = nb_check_ctx(ctx, why);
    if (rc) { g_lastError = why; return rc; }
    if (ctx->criterion == NBCUDA_EXACT) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    NbTreeBuffers& b = st->b;
    for (int attempt = 0; attempt < 4; ++attempt) {
        NbScalars init{};
        init.rsize = st->rsize;
        init.capNodes = st->capNodes;
        NB_CHECK(cudaMemcpyAsync(b.sc, &init, sizeof init, cudaMemcpyHostToDevice, st->stream));
        nb_build_tree(b, st->nbody, ctx->criterion, ctx->theta, ctx->useQuad, 0, 0.0, st->numSMs,
                      st->stream);
        nb_link_and_moments(b, st->nbody, st->capNodes, ctx->criterion, ctx->theta, ctx->useQuad,
                            st->stream);
        NB_CHECK(cudaGetLastError());
        NB_CHECK(cudaMemcpyAsync(st->scHost, b.sc, sizeof(NbScalars), cudaMemcpyDeviceToHost,
                                 st->stream));
        NB_CHECK(cudaStreamSynchronize(st->stream));
        st->rsize = st->scHost->rsize;
        if (st->scHost->status & NBODY_CELL_OVERFLOW_ERROR) {
            rc = nb_alloc_nodes(st, st->scHost->neededNodes + st->scHost->neededNodes / 4 + 64);
            if (rc) return rc;
            continue;
        }
        st->haveTree = 1;
        st->lastCriterion = ctx->criterion;
        return st->scHost->status;
    }
    return NBODY_CELL_OVERFLOW_ERROR;
}

NBodyCudaStatus nbTreeInfoCUDA(NBodyCudaState* st, NBodyCudaTreeInfo* info)
{
    if (!st || !info) return NBODY_USER_ERROR;
    const NbScalars& h = *st->scHost;
    info->rsize = st->rsize;
    info->nbody = st->nbody;
    info->nTreeBodies = st->haveTree ? h.nTree : 0;
    info->cellUsed = st->haveTree ? h.nCells : 0;
    info->maxDepth = st->haveTree ? h.maxDepth : 0;
    info->nNodes = st->haveTree ? h.nNodes : 0;
    info->step = st->step;
    info->treeIncest = st->treeIncest;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbGetTreeCUDA(NBodyCudaState* st, double* pos, double* mass, double* rcrit2,
                              double* quad, int32_t* next, int32_t* body, int32_t* depth)
{
    if (!st || !st->haveTree) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    const int nn = st->scHost->nNodes;
    NbTreeBuffers& b = st->b;
    const cudaStream_t s = st->stream;
    if (pos || mass) {
        double4* tmp = (double4*) malloc(sizeof(double4) * (size_t) (nn ? nn : 1));
        NB_CHECK(cudaMemcpyAsync(tmp, b.nodePM, sizeof(double4) * (size_t) nn, cudaMemcpyDeviceToHost, s));
        NB_CHECK(cudaStreamSynchronize(s));
        for (int k = 0; k < nn; ++k) {
            if (pos) { pos[3 * k] = tmp[k].x; pos[3 * k + 1] = tmp[k].y; pos[3 * k + 2] = tmp[k].z; }
            if (mass) mass[k] = tmp[k].w;
        }
        free(tmp);
    }
    int2* lk = (int2*) malloc(sizeof(int2) * (size_t) (nn ? nn : 1));
    NB_CHECK(cudaMemcpyAsync(lk, b.nodeLink, sizeof(int2) * (size_t) nn, cudaMemcpyDeviceToHost, s));
    if (rcrit2) NB_CHECK(cudaMemcpyAsync(rcrit2, b.nodeCrit, sizeof(double) * (size_t) nn, cudaMemcpyDeviceToHost, s));
    if (quad) NB_CHECK(cudaMemcpyAsync(quad, b.nodeQuad, 6 * sizeof(double) * (size_t) nn, cudaMemcpyDeviceToHost, s));
    if (depth) NB_CHECK(cudaMemcpyAsync(depth, b.nodeDepth, sizeof(int) * (size_t) nn, cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaStreamSynchronize(s));
    for (int k = 0; k < nn; ++k) {
        if (next) next[k] = lk[k].x;
        if (body) body[k] = lk[k].y;
        if (lk[k].y >= 0) {
            if (rcrit2) rcrit2[k] = 0.0;
            if (quad) for (int c = 0; c < 6; ++c) quad[6 * (size_t) k + c] = 0.0;
        }
    }
    free(lk);
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbExtAccelerationCUDA(const NBodyCudaPotential* pot, const double* pos,
                                      double* acc, int n, int device)
{
    if (!pot || n < 0 || (n && (!pos || !acc))) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(device));
    NBodyCudaCtx c{};
    c.potentialType = NBCUDA_POTENTIAL_DEFAULT;
    c.pot = *pot;
    std::string why;
    NBodyCudaStatus rc = nb_check_ctx(&c, why);
    if (rc) { g_lastError = why; return rc; }
    if (!n) return NBODY_SUCCESS;
    double *dp = nullptr, *da = nullptr;
    NB_CHECK(cudaMalloc((void**) &dp, 3 * sizeof(double) * (size_t) n));
    cudaError_t e = cudaMalloc((void**) &da, 3 * sizeof(double) * (size_t) n);
    if (e != cudaSuccess) { cudaFree(dp); return nb_cuda_fail(e, "cudaMalloc"); }
    e = cudaMemcpy(dp, pos, 3 * sizeof(double) * (size_t) n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        nb_launch_ext_only(dp, da, n, nb_pot_from(&c), 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(acc, da, 3 * sizeof(double) * (size_t) n, cudaMemcpyDeviceToHost);
    cudaFree(dp);
    cudaFree(da);
    if (e != cudaSuccess) return nb_cuda_fail(e, "nbExtAccelerationCUDA");
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbEmdCalcCUDA(const double* sig1, int n1, const double* sig2, int n2,
                              double* emd, int device)
{
    if (!emd || n1 < 0 || n2 < 0 || (n1 && !sig1) || (n2 && !sig2)) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(device));
    const int nb = std::max(std::max(n1, n2), 1);
    const size_t sigBytes = nb_al(24 * (size_t) nb);
    const size_t bytes = 2 * sigBytes + nb_al(nb_emd_problem_bytes(nb)) + nb_al(8);
    char* buf = nullptr;
    NB_CHECK(cudaMalloc((void**) &buf, bytes));
    double* d1 = (double*) buf;
    double* d2 = (double*) (buf + sigBytes);
    double* dOut = (double*) (buf + 2 * sigBytes);
    char* work = buf + 2 * sigBytes + nb_al(8);
    cudaError_t e = cudaSuccess;
    if (n1) e = cudaMemcpy(d1, sig1, 24 * (size_t) n1, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n2) e = cudaMemcpy(d2, sig2, 24 * (size_t) n2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        nb_launch_emd_direct(d1, n1, d2, n2, work, dOut, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(emd, dOut, sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (e != cudaSuccess) return nb_cuda_fail(e, "nbEmdCalcCUDA");
    return NBODY_SUCCESS;
}

uint64_t nbKernelLaunchesCUDA(void) { return g_launches.load(); }

NBodyCudaStatus nbLastWalkTimeCUDA(NBodyCudaState* st, double* ms, int* launches)
{
    if (!st) return NBODY_USER_ERROR;
    if (ms) *ms = st->walkMs;
    if (launches) *launches = st->walkLaunches;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbLastStepTimeCUDA(NBodyCudaState* st, double* ms)
{
    if (!st || !ms) return NBODY_USER_ERROR;
    *ms = st->stepMs;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbDirectSampleCUDA(NBodyCudaState* st, double eps2, const int32_t* targets,
                                   int count, double* acc)
{
    if (!st || count < 0 || (count && (!targets || !acc))) return NBODY_USER_ERROR;
    for (int k = 0; k < count; ++k)
        if (targets[k] < 0 || targets[k] >= st->nbody) return NBODY_USER_ERROR;
    if (!count) return NBODY_SUCCESS;
    NB_CHECK(cudaSetDevice(st->device));
    int* dt = nullptr;
    double* da = nullptr;
    NB_CHECK(cudaMalloc((void**) &dt, sizeof(int) * (size_t) count));
    cudaError_t e = cudaMalloc((void**) &da, 3 * sizeof(double) * (size_t) count);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dt, targets, sizeof(int) * (size_t) count, cudaMemcpyHostToDevice, st->stream);
    if (e == cudaSuccess) {
        nb_launch_direct_sample(st->b.px, st->b.py, st->b.pz, st->b.mass, st->nbody, dt, count,
                                eps2, da, st->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(acc, da, 3 * sizeof(double) * (size_t) count, cudaMemcpyDeviceToHost, st->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st->stream);
    cudaFree(dt);
    cudaFree(da);
    if (e != cudaSuccess) return nb_cuda_fail(e, "nbDirectSampleCUDA");
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbGravVJPCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st, const double* dAbar,
                              double* dXbar, double* dMbar)
{
    if (!st || !dAbar || !dXbar) return NBODY_USER_ERROR;
    std::string why;
    NBodyCudaStatus rc = nb_check_ctx(ctx, why);
    if (rc) { g_lastError = why; return rc; }
    if (ctx->precision != NBCUDA_PRECISION_FP64) {
        g_lastError = "the adjoint follows the FP64 walk";
        return NBODY_UNSUPPORTED;
    }
    if (!nb_pot_basic(ctx, why)) { g_lastError = "the adjoint is " + why; return NBODY_UNSUPPORTED; }
    if (ctx->criterion != st->lastCriterion || (ctx->criterion != NBCUDA_EXACT && !st->haveTree)) {
        g_lastError = "nbGravVJPCUDA needs a force evaluation with the same context first";
        return NBODY_USER_ERROR;
    }
    NB_CHECK(cudaSetDevice(st->device));
    if (ctx->criterion != NBCUDA_EXACT && st->nodeBarCap < st->capNodes) {
        cudaFree(st->nodeBar);
        st->nodeBar = nullptr;
        NB_CHECK(cudaMalloc((void**) &st->nodeBar, 10 * sizeof(double) * (size_t) st->capNodes));
        st->nodeBarCap = st->capNodes;
    }
    NbWalkParams wp{};
    wp.eps2 = ctx->eps2;
    wp.useQuad = ctx->useQuad;
    wp.n = st->nbody;
    NB_CHECK(cudaEventRecord(st->evS, st->stream));
    nb_launch_vjp(st->b, st->nodeBar, st->capNodes, st->scHost->maxDepth, ctx->criterion, wp,
                  nb_pot_from(ctx), dAbar, dXbar, dMbar, st->numSMs, st->ev0, st->ev1, st->stream);
    NB_CHECK(cudaEventRecord(st->evE, st->stream));
    NB_CHECK(cudaGetLastError());
    NB_CHECK(cudaStreamSynchronize(st->stream));
    // timings of the adjoint: walk = the walk-side kernel, step = the whole product
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, st->ev0, st->ev1);
    st->walkMs = ms;
    ms = 0.0f;
    cudaEventElapsedTime(&ms, st->evS, st->evE);
    st->stepMs = ms;
    return NBODY_SUCCESS;
}

static size_t nb_align256(size_t x) { return (x + 255) & ~(size_t) 255; }

static NBodyCudaStatus nb_save_slot(NBodyCudaState* st, NbSlot& sl)
{
    NB_CHECK(cudaSetDevice(st->device));
    const size_t n = (size_t) st->nbody;
    const size_t nodes = st->haveTree ? (size_t) st->scHost->nNodes : 0;
    auto bytesFor = [n](size_t nn) {
        return nb_align256(10 * n * sizeof(double)) + 2 * nb_align256(n * sizeof(int)) +
               nb_align256(nn * sizeof(double4)) + nb_align256(nn * sizeof(double)) +
               nb_align256(nn * sizeof(int2)) + nb_align256(6 * nn * sizeof(double)) +
               nb_align256(nn * sizeof(int)) + 256;
    };
    if (sl.bytes < bytesFor(nodes)) {
        // room for a quarter more nodes: the node count changes a little from step to step
        const size_t want = bytesFor(nodes + nodes / 4 + 1024);
        cudaFree(sl.mem);
        sl.mem = nullptr;
        sl.bytes = 0;
        NB_CHECK(cudaMalloc((void**) &sl.mem, want));
        sl.bytes = want;
    }
    char* p = sl.mem;
    auto carve = [&p](size_t bytes) { char* q = p; p += nb_align256(bytes); return q; };
    sl.body = (double*) carve(10 * n * sizeof(double));
    sl.order = (unsigned*) carve(n * sizeof(int));
    sl.bodyNode = (int*) carve(n * sizeof(int));
    sl.nodePM = (double4*) carve(nodes * sizeof(double4));
    sl.nodeCrit = (double*) carve(nodes * sizeof(double));
    sl.nodeLink = (int2*) carve(nodes * sizeof(int2));
    sl.nodeQuad = (double*) carve(6 * nodes * sizeof(double));
    sl.nodeDepth = (int*) carve(nodes * sizeof(int));
    NbTreeBuffers& b = st->b;
    const cudaStream_t s = st->stream;
    const double* src[10] = {b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.ax, b.ay, b.az, b.mass};
    for (int k = 0; k < 10; ++k)
        NB_CHECK(cudaMemcpyAsync(sl.body + k * n, src[k], n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (nodes) {
        NB_CHECK(cudaMemcpyAsync(sl.order, b.sort.idxA, n * sizeof(int), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(sl.bodyNode, b.bodyNode, n * sizeof(int), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(sl.nodePM, b.nodePM, nodes * sizeof(double4), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(sl.nodeCrit, b.nodeCrit, nodes * sizeof(double), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(sl.nodeLink, b.nodeLink, nodes * sizeof(int2), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(sl.nodeQuad, b.nodeQuad, 6 * nodes * sizeof(double), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(sl.nodeDepth, b.nodeDepth, nodes * sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
    if (st->lmcDev)
        NB_CHECK(cudaMemcpyAsync(sl.lmc, st->lmcDev, 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaStreamSynchronize(s));
    sl.sc = *st->scHost;
    sl.rsize = st->rsize;
    sl.haveTree = st->haveTree;
    sl.criterion = st->lastCriterion;
    sl.step = st->step;
    sl.treeIncest = st->treeIncest;
    sl.valid = 1;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSaveStateCUDA(NBodyCudaState* st, int slot)
{
    if (!st || slot < 0 || slot >= (1 << 16)) return NBODY_USER_ERROR;
    if ((int) st->slots.size() <= slot) st->slots.resize(slot + 1);
    return nb_save_slot(st, st->slots[slot]);
}

static NBodyCudaStatus nb_restore_slot(NBodyCudaState* st, NbSlot& sl)
{
    NB_CHECK(cudaSetDevice(st->device));
    const size_t n = (size_t) st->nbody;
    const size_t nodes = sl.haveTree ? (size_t) sl.sc.nNodes : 0;
    if (sl.haveTree && st->capNodes < sl.sc.nNodes) {
        NBodyCudaStatus rc = nb_alloc_nodes(st, sl.sc.nNodes);
        if (rc) return rc;
    }
    NbTreeBuffers& b = st->b;
    const cudaStream_t s = st->stream;
    double* dst[10] = {b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.ax, b.ay, b.az, b.mass};
    for (int k = 0; k < 10; ++k)
        NB_CHECK(cudaMemcpyAsync(dst[k], sl.body + k * n, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (nodes) {
        NB_CHECK(cudaMemcpyAsync(b.sort.idxA, sl.order, n * sizeof(int), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(b.bodyNode, sl.bodyNode, n * sizeof(int), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(b.nodePM, sl.nodePM, nodes * sizeof(double4), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(b.nodeCrit, sl.nodeCrit, nodes * sizeof(double), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(b.nodeLink, sl.nodeLink, nodes * sizeof(int2), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(b.nodeQuad, sl.nodeQuad, 6 * nodes * sizeof(double), cudaMemcpyDeviceToDevice, s));
        NB_CHECK(cudaMemcpyAsync(b.nodeDepth, sl.nodeDepth, nodes * sizeof(int), cudaMemcpyDeviceToDevice, s));
    }
    *st->scHost = sl.sc;
    st->scHost->capNodes = st->capNodes;
    NB_CHECK(cudaMemcpyAsync(b.sc, st->scHost, sizeof(NbScalars), cudaMemcpyHostToDevice, s));
    if (st->lmcDev)
        NB_CHECK(cudaMemcpyAsync(st->lmcDev, sl.lmc, 6 * sizeof(double), cudaMemcpyHostToDevice, s));
    NB_CHECK(cudaStreamSynchronize(s));
    st->rsize = sl.rsize;
    st->haveTree = sl.haveTree;
    st->lastCriterion = sl.criterion;
    st->step = sl.step;
    st->treeIncest = sl.treeIncest;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbRestoreStateCUDA(NBodyCudaState* st, int slot)
{
    if (!st || slot < 0 || slot >= (int) st->slots.size() || !st->slots[slot].valid) {
        g_lastError = "nbRestoreStateCUDA: no state saved in this slot";
        return NBODY_USER_ERROR;
    }
    return nb_restore_slot(st, st->slots[slot]);
}

NBodyCudaStatus nbReleaseStatesCUDA(NBodyCudaState* st)
{
    if (!st) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    for (NbSlot& sl : st->slots) cudaFree(sl.mem);
    st->slots.clear();
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbStepAdjointCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st, const double* dAk,
                                  double* dXbar, double* dVbar, double* dMbar, double* dAbarNext,
                                  double* dDtbar)
{
    if (!st || !dAk || !dXbar || !dVbar || !dAbarNext) return NBODY_USER_ERROR;
    std::string why;
    NBodyCudaStatus rc = nb_check_ctx(ctx, why);
    if (rc) { g_lastError = why; return rc; }
    if (ctx->precision != NBCUDA_PRECISION_FP64) {
        g_lastError = "the adjoint follows the FP64 walk";
        return NBODY_UNSUPPORTED;
    }
    if (!nb_pot_basic(ctx, why)) { g_lastError = "the adjoint is " + why; return NBODY_UNSUPPORTED; }
    if (ctx->criterion != st->lastCriterion || (ctx->criterion != NBCUDA_EXACT && !st->haveTree)) {
        g_lastError = "nbStepAdjointCUDA needs the force evaluation of the step's end state first";
        return NBODY_USER_ERROR;
    }
    NB_CHECK(cudaSetDevice(st->device));
    if (ctx->criterion != NBCUDA_EXACT && st->nodeBarCap < st->capNodes) {
        cudaFree(st->nodeBar);
        st->nodeBar = nullptr;
        NB_CHECK(cudaMalloc((void**) &st->nodeBar, 10 * sizeof(double) * (size_t) st->capNodes));
        st->nodeBarCap = st->capNodes;
    }
    if (!st->adjScratch)
        NB_CHECK(nb_alloc(&st->adjScratch, 7 * (size_t) st->capBodies));
    NbWalkParams wp{};
    wp.eps2 = ctx->eps2;
    wp.useQuad = ctx->useQuad;
    wp.n = st->nbody;
    NB_CHECK(cudaEventRecord(st->evS, st->stream));
    nb_launch_step_adjoint(st->b, st->nodeBar, st->capNodes, st->scHost->maxDepth, ctx->criterion,
                           wp, nb_pot_from(ctx), ctx->timestep, dAk, dXbar, dVbar, dMbar,
                           dAbarNext, dDtbar, st->adjScratch, st->numSMs, st->ev0, st->ev1,
                           st->stream);
    NB_CHECK(cudaEventRecord(st->evE, st->stream));
    NB_CHECK(cudaGetLastError());
    NB_CHECK(cudaStreamSynchronize(st->stream));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, st->ev0, st->ev1);
    st->walkMs = ms;
    ms = 0.0f;
    cudaEventElapsedTime(&ms, st->evS, st->evE);
    st->stepMs = ms;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbEnergyCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st, double* energy)
{
    if (!st || !energy) return NBODY_USER_ERROR;
    std::string why;
    NBodyCudaStatus rc = nb_check_ctx(ctx, why);
    if (rc) { g_lastError = why; return rc; }
    if (!nb_pot_basic(ctx, why)) { g_lastError = "the potential energy is " + why; return NBODY_UNSUPPORTED; }
    NB_CHECK(cudaSetDevice(st->device));
    NbTreeBuffers& b = st->b;
    double* dOut = st->stage;           // >= 3 doubles of device staging
    nb_launch_energy(b.px, b.py, b.pz, b.vx, b.vy, b.vz, b.mass, st->nbody, ctx->eps2,
                     nb_pot_from(ctx), dOut, st->stream);
    NB_CHECK(cudaGetLastError());
    NB_CHECK(cudaMemcpyAsync(energy, dOut, 3 * sizeof(double), cudaMemcpyDeviceToHost, st->stream));
    NB_CHECK(cudaStreamSynchronize(st->stream));
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbPeakFmaCUDA(int device, int fp64, double* tflops)
{
    if (!tflops) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(device));
    cudaDeviceProp prop;
    NB_CHECK(cudaGetDeviceProperties(&prop, device));
    *tflops = nb_fma_probe(fp64, prop.multiProcessorCount, 0);
    NB_CHECK(cudaGetLastError());
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbInteractionCountsCUDA(NBodyCudaState* st, unsigned long long* nBodyBody,
                                        unsigned long long* nBodyCell, unsigned long long* nVisit,
                                        unsigned long long* nWarpSteps)
{
    if (!st) return NBODY_USER_ERROR;
    if (nWarpSteps) *nWarpSteps = st->cWarpSteps;
    if (nBodyBody) *nBodyBody = st->cBB;
    if (nBodyCell) *nBodyCell = st->cBC;
    if (nVisit) *nVisit = st->cVisit;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetCountingCUDA(NBodyCudaState* st, int enable)
{
    if (!st) return NBODY_USER_ERROR;
    st->counting = enable != 0;
    return NBODY_SUCCESS;
}

const char* nbLastErrorCUDA(void) { return g_lastError.c_str(); }

}  // extern "C"

// =============================================================================================
// Histograms and likelihoods (kernels in nb_likelihood.cu)
// =============================================================================================
static NbHistDev nb_hist_dev(const NBodyCudaHistogramParams* hp)
{
    // nbGetHistTrig (nbody/src/nbody_coordinates.c:73-85) and the rotation of nbXYZToLambdaBeta
    const double rphi = hp->phi * M_PI / 180.0, rpsi = hp->psi * M_PI / 180.0;
    const double rth = hp->theta * M_PI / 180.0;
    const double cosphi = cos(rphi), sinphi = sin(rphi), sinpsi = sin(rpsi), cospsi = cos(rpsi);
    const double costh = cos(rth), sinth = sin(rth);
    NbHistDev h{};
    h.rot[0] = cospsi * cosphi - costh * sinphi * sinpsi;
    h.rot[1] = cospsi * sinphi + costh * cosphi * sinpsi;
    h.rot[2] = sinpsi * sinth;
    h.rot[3] = -sinpsi * cosphi - costh * sinphi * cospsi;
    h.rot[4] = -sinpsi * sinphi + costh * cosphi * cospsi;
    h.rot[5] = cospsi * sinth;
    h.rot[6] = sinth * sinphi;
    h.rot[7] = -sinth * cosphi;
    h.rot[8] = costh;
    h.sunGCDist = hp->sunGCDist;
    h.lambdaStart = hp->lambdaStart;
    h.lambdaSize = (hp->lambdaEnd - hp->lambdaStart) / (double) hp->lambdaBins;
    h.betaStart = hp->betaStart;
    h.betaSize = (hp->betaEnd - hp->betaStart) / (double) hp->betaBins;
    h.lambdaBins = hp->lambdaBins;
    h.betaBins = hp->betaBins;
    // cartesianalign (nbody/src/nbody_coordinates.c:192-224)
    const double cl = cos(M_PI - hp->lNCP), sl = sin(M_PI - hp->lNCP);
    const double cd = cos(M_PI_2 - hp->NGPdec), sd = sin(M_PI_2 - hp->NGPdec);
    const double ca = cos(hp->NGPra), sa = sin(hp->NGPra);
    h.align[0] = ca * cd * cl - sa * sl;
    h.align[1] = -ca * cd * sl - sa * cl;
    h.align[2] = ca * sd;
    h.align[3] = sa * cd * cl + ca * sl;
    h.align[4] = -sa * cd * sl + ca * cl;
    h.align[5] = sa * sd;
    h.align[6] = -sd * cl;
    h.align[7] = sd * sl;
    h.align[8] = cd;
    h.sunVel[0] = hp->sunVelx;
    h.sunVel[1] = hp->sunVely;
    h.sunVel[2] = hp->sunVelz;
    return h;
}


static NbLikeFlags nb_like_flags(const NBodyCudaHistogramParams* hp)
{
    return NbLikeFlags{hp->useBetaDisp != 0, hp->useVelDisp != 0, hp->useBetaComp != 0,
                       hp->useVlos != 0, hp->useDist != 0, hp->usePropMot != 0};
}

// Device buffers of one histogram evaluation, carved from the state's scratch block.
struct NbHistRun {
    NbHistPlan p{};
    NbDataHistDev dh{};
    NbLikeFlags f{};
    int* nbodyOf = nullptr;     // device, per dwarf
    double* out = nullptr;      // device, NB_LIKELIHOOD_TERMS per dwarf
    double* comps = nullptr;    // device, 7 x 2 x B per dwarf
};

// Plans the histograms of the dwarfs with nbodyOf[d] consecutive bodies each (one dwarf: the
// whole state) for the likelihood against data (data != NULL: the histograms its comparisons
// use) or for export (every histogram the reference builds).  Uploads the chunk table, the
// dwarf sizes and the data histogram on the state's stream.
static NBodyCudaStatus nb_hist_prepare(NBodyCudaState* st, const std::vector<int>& nbodyOf,
                                       const NBodyCudaHistogramParams* hp,
                                       const NBodyCudaDataHistogram* data, bool exportAll,
                                       NbHistRun& r)
{
    if (!hp || hp->lambdaBins < 1 || hp->betaBins < 1 || !(hp->lambdaEnd > hp->lambdaStart) ||
        !(hp->betaEnd > hp->betaStart) || hp->iterMax < 0 || hp->iterMax > 1000) {
        g_lastError = "invalid histogram parameters";
        return NBODY_USER_ERROR;
    }
    if (!st->types) { g_lastError = "body types not set"; return NBODY_USER_ERROR; }
    const int B = hp->lambdaBins * hp->betaBins;
    const NbLikeFlags f = nb_like_flags(hp);
    if (data) {
        if (data->nBins != B || !data->useBin || !data->lambda || !data->variable || !data->err) {
            g_lastError = "data histogram does not match the histogram parameters";
            return NBODY_USER_ERROR;
        }
        if (data->nRange < 0 || data->nRange > 1024 || (data->nRange > 0 && !data->emdRange)) {
            g_lastError = "data histogram: invalid EMD ranges";
            return NBODY_USER_ERROR;
        }
        if (hp->betaBins > 1 && !data->beta) {
            g_lastError = "a two-dimensional data histogram needs its beta bin centres";
            return NBODY_USER_ERROR;
        }
        if ((f.betaDisp && (!data->compVariable[0] || !data->compErr[0])) ||
            (f.velDisp && (!data->compVariable[1] || !data->compErr[1]))) {
            g_lastError = "the data histogram has no dispersion columns for an enabled comparison";
            return NBODY_USER_ERROR;
        }
        for (int k = 2; k < NB_HIST_COMPONENTS; ++k)
            if (!data->compVariable[k] != !data->compErr[k]) {
                g_lastError = "data histogram: a component has values without errors or errors "
                              "without values";
                return NBODY_USER_ERROR;
            }
    }
    // histograms 1..7 to build and the quantity each bins
    static const int kQuantity[NB_HIST_COMPONENTS] = {NB_Q_BETA, NB_Q_VLOS, NB_Q_VLOS, NB_Q_BETA,
                                                      NB_Q_DIST, NB_Q_MUDEC, NB_Q_MURA};
    bool built[NB_HIST_COMPONENTS] = {};
    if (exportAll) {
        const bool avgs = f.vlos || f.betaComp || f.dist || f.propMot;
        for (int k = 0; k < NB_HIST_COMPONENTS; ++k) built[k] = k < 2 || avgs;
    } else if (data) {
        built[0] = f.betaDisp; built[1] = f.velDisp; built[2] = f.vlos; built[3] = f.betaComp;
        built[4] = f.dist; built[5] = built[6] = f.propMot;
    }
    NbHistPlan& p = r.p;
    p = NbHistPlan{};
    p.h = nb_hist_dev(hp);
    int slotOf[NB_NQ];
    for (int q = 0; q < NB_NQ; ++q) slotOf[q] = -1;
    for (int k = 0; k < NB_HIST_COMPONENTS; ++k) {
        p.histSlot[k] = -1;
        if (!built[k]) continue;
        const int q = kQuantity[k];
        if (slotOf[q] < 0) {
            slotOf[q] = p.h.nq;
            p.h.q[p.h.nq++] = q;
        }
        p.histSlot[k] = slotOf[q];
    }
    for (int k = 0; k < p.h.nq; ++k) {
        switch (p.h.q[k]) {
        case NB_Q_BETA: p.cut[k] = hp->betaSigma; p.corr[k] = hp->betaCorrect; break;
        case NB_Q_VLOS: p.cut[k] = hp->velSigma; p.corr[k] = hp->velCorrect; break;
        case NB_Q_DIST: p.cut[k] = hp->distSigma; p.corr[k] = hp->distCorrect; break;
        default: p.cut[k] = hp->pmSigma; p.corr[k] = hp->pmCorrect; break;
        }
    }
    const int n = st->nbody;
    const int D = (int) nbodyOf.size();
    p.n = n;
    p.D = D;
    p.B = B;
    p.iterMax = hp->iterMax;
    // chunks of at most ch bodies within one dwarf
    const size_t ch = nb_hist_chunk_bodies(n, p.h.nq, B);
    std::vector<int4> chunks;
    std::vector<int> chunkFirst(D + 1);
    int first = 0;
    for (int d = 0; d < D; ++d) {
        chunkFirst[d] = (int) chunks.size();
        for (int c = first; c < first + nbodyOf[d]; c += (int) ch)
            chunks.push_back(make_int4(c, std::min(first + nbodyOf[d], c + (int) ch), d, 0));
        first += nbodyOf[d];
    }
    chunkFirst[D] = (int) chunks.size();
    if (first != n) { g_lastError = "dwarf sizes do not add up to the body count"; return NBODY_USER_ERROR; }
    p.nChunks = (int) chunks.size();
    // A data file without an EMDRange line gets the range nbReadHistogram sets
    // (nbody/src/nbody_histogram.c:1563-1567): data[0].lambda and data[lambdaBins - 1].lambda,
    // each widened by half the lambda spacing of data[0] and data[1].  With one beta bin that is
    // every bin (one range over all used bins, nRange 0 below).  With more beta bins data[1]
    // shares data[0]'s lambda and data[lambdaBins - 1] is the (lambdaBins - 1)-th bin in
    // lambda-major order, so the range is [first lambda, the lambda of that bin]: the first
    // 1/betaBins of the lambda axis; the reference compares only that part, and so does this.
    double defaultRange[2] = {0.0, 0.0};
    const bool twoDimDefault = data && hp->betaBins > 1 && data->nRange == 0 && B >= 2;
    if (twoDimDefault) {
        const double half = (data->lambda[1] - data->lambda[0]) / 2;
        defaultRange[0] = data->lambda[0] - half;
        defaultRange[1] = data->lambda[hp->lambdaBins - 1] + half;
    }
    const int nRangeUsed = twoDimDefault ? 2 : (data ? data->nRange : 0);
    const double* rangeUsed = twoDimDefault ? defaultRange : (data ? data->emdRange : nullptr);
    const size_t Dz = (size_t) D, Bz = (size_t) B, nz = (size_t) n, nq = (size_t) p.h.nq;
    const size_t QDB = std::max<size_t>(nq, 1) * Dz * Bz;
    const size_t need = nb_al(4 * Dz * Bz) + 4 * nb_al(4 * Dz) + nb_al(4 * nz) +
                        nb_al(8 * nq * nz) + nb_al(16 * chunks.size()) + nb_al(4 * (Dz + 1)) +
                        nb_al(4 * chunks.size() * Bz) + nb_al(4 * Dz * Bz) + nb_al(4 * nz) +
                        5 * nb_al(8 * QDB) + nb_al(4 * Dz) + nb_al(8 * NB_LIKELIHOOD_TERMS * Dz) +
                        nb_al(8 * Dz * NB_HIST_COMPONENTS * 2 * Bz) + nb_al(4 * Bz) +
                        (3 + 2 * NB_HIST_COMPONENTS) * nb_al(8 * Bz) +
                        nb_al(8 * (size_t) (data && nRangeUsed > 0 ? nRangeUsed : 0)) + 256;
    // two-dimensional histograms: one emdCalc problem per dwarf and lambda range
    const size_t emdProblems = data && hp->betaBins > 1
        ? Dz * (size_t) (nRangeUsed > 0 ? nRangeUsed / 2 : 1) : 0;
    const size_t emdBytes = emdProblems ? nb_al(nb_emd_problem_bytes(B)) : 0;
    const size_t needAll = need + (emdProblems ? nb_al(8 * Bz) + nb_al(8 * emdProblems) +
                                                   emdProblems * emdBytes : 0);
    NB_CHECK(cudaSetDevice(st->device));
    if (st->histScratchBytes < needAll) {
        cudaFree(st->histScratch);
        st->histScratch = nullptr;
        st->histScratchBytes = 0;
        NB_CHECK(cudaMalloc((void**) &st->histScratch, needAll));
        st->histScratchBytes = needAll;
    }
    char* cur = st->histScratch;
    auto carve = [&cur](size_t bytes) { char* q = cur; cur += nb_al(bytes); return q; };
    p.counts = (unsigned*) carve(4 * Dz * Bz);
    p.inRange = (unsigned*) carve(4 * Dz);
    p.nLight = (unsigned*) carve(4 * Dz);
    p.lastLight = (int*) carve(4 * Dz);
    p.binOf = (int*) carve(4 * nz);
    p.val = (double*) carve(8 * nq * nz);
    p.chunks = (int4*) carve(16 * chunks.size());
    p.chunkFirst = (int*) carve(4 * (Dz + 1));
    p.rows = (int*) carve(4 * chunks.size() * Bz);
    p.segStart = (int*) carve(4 * Dz * Bz);
    p.list = (int*) carve(4 * nz);
    p.sum = (double*) carve(8 * QDB);
    p.sq = (double*) carve(8 * QDB);
    p.rem = (double*) carve(8 * QDB);
    p.var = (double*) carve(8 * QDB);
    p.err = (double*) carve(8 * QDB);
    r.nbodyOf = (int*) carve(4 * Dz);
    r.out = (double*) carve(8 * NB_LIKELIHOOD_TERMS * Dz);
    r.comps = (double*) carve(8 * Dz * NB_HIST_COMPONENTS * 2 * Bz);
    const cudaStream_t s = st->stream;
    if (!chunks.empty())
        NB_CHECK(cudaMemcpyAsync(p.chunks, chunks.data(), 16 * chunks.size(),
                                 cudaMemcpyHostToDevice, s));
    NB_CHECK(cudaMemcpyAsync(p.chunkFirst, chunkFirst.data(), 4 * (Dz + 1), cudaMemcpyHostToDevice, s));
    NB_CHECK(cudaMemcpyAsync(r.nbodyOf, nbodyOf.data(), 4 * Dz, cudaMemcpyHostToDevice, s));
    r.f = f;
    r.dh = NbDataHistDev{};
    if (data) {
        NbDataHistDev& dh = r.dh;
        int* dUse = (int*) carve(4 * Bz);
        NB_CHECK(cudaMemcpyAsync(dUse, data->useBin, 4 * Bz, cudaMemcpyHostToDevice, s));
        auto up = [&](const double* src) -> const double* {
            if (!src) return nullptr;
            double* dst = (double*) carve(8 * Bz);
            cudaMemcpyAsync(dst, src, 8 * Bz, cudaMemcpyHostToDevice, s);
            return dst;
        };
        dh.useBin = dUse;
        dh.lambda = up(data->lambda);
        dh.variable = up(data->variable);
        dh.err = up(data->err);
        for (int k = 0; k < NB_HIST_COMPONENTS; ++k) {
            dh.compVar[k] = up(data->compVariable[k]);
            dh.compErr[k] = up(data->compErr[k]);
        }
        dh.massPerParticle = data->massPerParticle;
        dh.totalNum = data->totalNum;
        dh.nBins = B;
        dh.betaDispBins = data->betaDispBins;
        dh.nRange = nRangeUsed;
        dh.emdRange = nullptr;
        if (nRangeUsed > 0) {
            double* dst = (double*) carve(8 * (size_t) nRangeUsed);
            // pageable source: the copy has read it when the call returns
            cudaMemcpyAsync(dst, rangeUsed, 8 * (size_t) nRangeUsed, cudaMemcpyHostToDevice, s);
            dh.emdRange = dst;
        }
        dh.beta = nullptr;
        dh.emd2d = nullptr;
        dh.emdWork = nullptr;
        dh.emdWorkBytes = 0;
        if (emdProblems) {
            dh.beta = up(data->beta);
            dh.emd2d = (double*) carve(8 * emdProblems);
            dh.emdWork = carve(emdProblems * emdBytes);
            dh.emdWorkBytes = emdBytes;
        }
        NB_CHECK(cudaGetLastError());
    }
    return NBODY_SUCCESS;
}

// Launches the histogram passes of a prepared run (and, with data, the likelihood into r.out).
static int nb_hist_launch(NBodyCudaState* st, const int* bodyDwarf, const NbHistRun& r, bool like)
{
    NbTreeBuffers& b = st->b;
    int launches = nb_launch_hist_plan(r.p, b.px, b.py, b.pz, b.vx, b.vy, b.vz, st->types,
                                       bodyDwarf, st->numSMs, st->stream);
    if (like) {
        nb_launch_likelihood(r.p, b.mass, r.nbodyOf, r.dh, r.f, r.out, st->stream);
        ++launches;
    }
    return launches;
}

// Histograms of the dwarfs (bodyDwarf NULL: the whole state is one dwarf) and, with a data
// histogram, their likelihoods.  Host outputs, any may be NULL: counts (D x B), totals (2 per
// dwarf: bodies in range, light bodies), massPer (per dwarf), comps (7 x 2 x B per dwarf),
// out (NB_LIKELIHOOD_TERMS per dwarf).
static NBodyCudaStatus nb_hist_run(NBodyCudaState* st, const int* bodyDwarf,
                                   const std::vector<int>& nbodyOf,
                                   const NBodyCudaHistogramParams* hp,
                                   const NBodyCudaDataHistogram* data, unsigned* counts,
                                   unsigned* totals, double* massPer, double* comps, double* out)
{
    NbHistRun r;
    const bool like = data && out;
    NBodyCudaStatus rc = nb_hist_prepare(st, nbodyOf, hp, like ? data : nullptr, comps != nullptr, r);
    if (rc != NBODY_SUCCESS) return rc;
    const cudaStream_t s = st->stream;
    nb_hist_launch(st, bodyDwarf, r, like);
    const size_t D = nbodyOf.size(), B = (size_t) r.p.B;
    if (comps) nb_launch_hist_export(r.p, r.comps, s);
    NB_CHECK(cudaGetLastError());
    if (out) NB_CHECK(cudaMemcpyAsync(out, r.out, 8 * NB_LIKELIHOOD_TERMS * D, cudaMemcpyDeviceToHost, s));
    if (comps)
        NB_CHECK(cudaMemcpyAsync(comps, r.comps, 8 * D * NB_HIST_COMPONENTS * 2 * B,
                                 cudaMemcpyDeviceToHost, s));
    if (counts) NB_CHECK(cudaMemcpyAsync(counts, r.p.counts, 4 * D * B, cudaMemcpyDeviceToHost, s));
    std::vector<unsigned> inR(D), light(D);
    std::vector<int> last(D);
    NB_CHECK(cudaMemcpyAsync(inR.data(), r.p.inRange, 4 * D, cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaMemcpyAsync(light.data(), r.p.nLight, 4 * D, cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaMemcpyAsync(last.data(), r.p.lastLight, 4 * D, cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaStreamSynchronize(s));
    for (size_t d = 0; d < D; ++d) {
        if (totals) { totals[2 * d] = inR[d]; totals[2 * d + 1] = light[d]; }
        if (massPer) {
            double m = 0.0;
            if (last[d] >= 0)
                NB_CHECK(cudaMemcpy(&m, st->b.mass + last[d], sizeof(double), cudaMemcpyDeviceToHost));
            massPer[d] = m;
        }
    }
    return NBODY_SUCCESS;
}

static NBodyCudaStatus nb_set_types(NBodyCudaState* st, const int* types)
{
    if (!types) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    if (!st->types) NB_CHECK(nb_alloc(&st->types, (size_t) st->capBodies));
    if (st->nbody)
        NB_CHECK(cudaMemcpy(st->types, types, sizeof(int) * (size_t) st->nbody, cudaMemcpyHostToDevice));
    return NBODY_SUCCESS;
}

// Samples nD dwarfs into the state's bodies (dwarf k from body firsts[k]) and types.
static bool nb_component_ok(const NBodyCudaDwarfComponent& c)
{
    switch (c.type) {
    case NBCUDA_DWARF_PLUMMER:
    case NBCUDA_DWARF_GEN_HERNQUIST:
        return c.scaleLength > 0.0 && c.mass >= 0.0;
    case NBCUDA_DWARF_NFW:                           // r200 from the M200 mass
        return c.scaleLength > 0.0 && c.mass > 0.0;
    case NBCUDA_DWARF_CORED:
        return c.scaleLength > 0.0 && c.mass > 0.0 && c.r1 > 0.0 && c.rc > 0.0;
    default:
        return false;
    }
}

static bool nb_mixed_dwarf_ok(const NBodyCudaMixedDwarf& w)
{
    return w.nbody >= 1 && w.nbodyBaryon >= 0 && w.nbodyBaryon <= w.nbody &&
           nb_component_ok(w.light) && nb_component_ok(w.dark);
}

static NBodyCudaMixedDwarf nb_mixed_from_plummer(const NBodyCudaPlummerDwarf& p)
{
    NBodyCudaMixedDwarf m{};
    m.nbody = p.nbody;
    m.nbodyBaryon = p.nbodyBaryon;
    m.light.type = m.dark.type = NBCUDA_DWARF_PLUMMER;
    m.light.mass = p.massLight;
    m.light.scaleLength = p.scaleLight;
    m.dark.mass = p.massDark;
    m.dark.scaleLength = p.scaleDark;
    for (int c = 0; c < 3; ++c) { m.position[c] = p.position[c]; m.velocity[c] = p.velocity[c]; }
    m.seed = p.seed;
    return m;
}

static NBodyCudaStatus nb_generate(NBodyCudaState* st, const NBodyCudaMixedDwarf* d, int nD,
                                   const int* firsts)
{
    for (int k = 0; k < nD; ++k) {
        if (!nb_mixed_dwarf_ok(d[k])) {
            g_lastError = "invalid dwarf parameters";
            return NBODY_USER_ERROR;
        }
    }
    NB_CHECK(cudaSetDevice(st->device));
    if (!st->types) NB_CHECK(nb_alloc(&st->types, (size_t) st->capBodies));
    void* table = nullptr;
    double* scratch = nullptr;
    NB_CHECK(cudaMalloc(&table, nb_ic_table_bytes(nD)));
    cudaError_t e = cudaMalloc((void**) &scratch, sizeof(double) * 12 * (size_t) nD);
    if (e != cudaSuccess) { cudaFree(table); return nb_cuda_fail(e, "cudaMalloc"); }
    const cudaStream_t s = st->stream;
    NbScalars init{};
    init.rsize = st->rsize;
    init.capNodes = st->capNodes;
    e = cudaMemcpyAsync(st->b.sc, &init, sizeof init, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        nb_launch_ic(d, nD, firsts, table, scratch, st->b, st->types, st->nbody, st->numSMs,
                     st->b.sc, s);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(st->scHost, st->b.sc, sizeof(NbScalars),
                                              cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(table);
    cudaFree(scratch);
    if (e != cudaSuccess) return nb_cuda_fail(e, "nbGenerateDwarf");
    if (st->scHost->status & ~(int) NBODY_STATUS_WARNINGS_MASK) {
        g_lastError = "the sampler found no radius or speed for some body";
        return st->scHost->status;
    }
    return NBODY_SUCCESS;
}

extern "C" {

NBodyCudaStatus nbGenerateMixedDwarfCUDA(NBodyCudaState* st, const NBodyCudaMixedDwarf* dwarf,
                                         double treeRSize)
{
    if (!st || !dwarf || dwarf->nbody != st->nbody) return NBODY_USER_ERROR;
    NBodyCudaStatus rc = nb_reset_run(st, treeRSize);
    if (rc) return rc;
    const int first = 0;
    return nb_generate(st, dwarf, 1, &first);
}

NBodyCudaStatus nbGenerateDwarfCUDA(NBodyCudaState* st, const NBodyCudaPlummerDwarf* dwarf,
                                    double treeRSize)
{
    if (!dwarf) return NBODY_USER_ERROR;
    const NBodyCudaMixedDwarf m = nb_mixed_from_plummer(*dwarf);
    return nbGenerateMixedDwarfCUDA(st, &m, treeRSize);
}

NBodyCudaStatus nbMixedDwarfParticleMassesCUDA(const NBodyCudaMixedDwarf* dwarf, double* out)
{
    if (!dwarf || !out) return NBODY_USER_ERROR;
    if (!nb_mixed_dwarf_ok(*dwarf)) {
        g_lastError = "invalid dwarf parameters";
        return NBODY_USER_ERROR;
    }
    nb_ic_particle_masses(*dwarf, out);
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbGetBodyMassesCUDA(NBodyCudaState* st, double* mass)
{
    if (!st || !mass) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(st->device));
    if (st->nbody) {
        NB_CHECK(cudaMemcpyAsync(mass, st->b.mass, sizeof(double) * (size_t) st->nbody,
                                 cudaMemcpyDeviceToHost, st->stream));
        NB_CHECK(cudaStreamSynchronize(st->stream));
    }
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetMixedTuningCUDA(NBodyCudaState* st, int groupMax, int listCap, int blocksPerSM)
{
    if (!st || groupMax < 1 || groupMax > 64 || (listCap != 32 && listCap != 64 && listCap != 128) ||
        blocksPerSM < 0)
        return NBODY_USER_ERROR;
    st->mixGroupMax = groupMax;
    st->mixListCap = listCap;
    st->mixBlocksPerSM = blocksPerSM;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetMixedModeCUDA(NBodyCudaState* st, int exactSet)
{
    if (!st || (exactSet != 0 && exactSet != 1)) return NBODY_USER_ERROR;
    st->mixExact = exactSet;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetLMCCUDA(NBodyCudaState* st, const double* pos3, const double* vel3,
                             const double* shift, int nShift)
{
    if (!st || !pos3 || !vel3 || !shift || nShift < 2) {
        g_lastError = "nbSetLMCCUDA: position, velocity and >= 2 reflex accelerations needed";
        return NBODY_USER_ERROR;
    }
    NB_CHECK(cudaSetDevice(st->device));
    if (!st->lmcDev) NB_CHECK(cudaMalloc((void**) &st->lmcDev, 6 * sizeof(double)));
    double h[6] = {pos3[0], pos3[1], pos3[2], vel3[0], vel3[1], vel3[2]};
    NB_CHECK(cudaMemcpy(st->lmcDev, h, sizeof h, cudaMemcpyHostToDevice));
    st->lmcShift.assign(shift, shift + 3 * (size_t) nShift);
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbGetLMCCUDA(NBodyCudaState* st, double* pos3, double* vel3)
{
    if (!st || !st->lmcDev) {
        g_lastError = "nbGetLMCCUDA: no LMC set";
        return NBODY_USER_ERROR;
    }
    NB_CHECK(cudaSetDevice(st->device));
    double h[6];
    NB_CHECK(cudaMemcpyAsync(h, st->lmcDev, sizeof h, cudaMemcpyDeviceToHost, st->stream));
    NB_CHECK(cudaStreamSynchronize(st->stream));
    if (pos3) { pos3[0] = h[0]; pos3[1] = h[1]; pos3[2] = h[2]; }
    if (vel3) { vel3[0] = h[3]; vel3[1] = h[4]; vel3[2] = h[5]; }
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetTimeOriginCUDA(NBodyCudaState* st, double previousForwardTime)
{
    if (!st) return NBODY_USER_ERROR;
    st->timeOrigin = previousForwardTime;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetWalkFormCUDA(NBodyCudaState* st, int form)
{
    if (!st || form < -1 || form > 2) return NBODY_USER_ERROR;
    st->walkForm = form;
    st->walkFormChosen = -1;
    st->walkTuneStep = 0;
    for (float& ms : st->walkFormMs) ms = -1.0f;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbGetWalkFormCUDA(NBodyCudaState* st, int* form)
{
    if (!st || !form) return NBODY_USER_ERROR;
    *form = st->walkForm >= 0 ? st->walkForm : st->walkFormChosen;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetStepGraphCUDA(NBodyCudaState* st, int enable)
{
    if (!st) return NBODY_USER_ERROR;
    st->useStepGraph = enable != 0;
    if (!enable) nb_drop_step_graph(st);
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetStepCUDA(NBodyCudaState* st, int step)
{
    if (!st || step < 0) return NBODY_USER_ERROR;
    st->step = step;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbSetTypesCUDA(NBodyCudaState* st, const int* types)
{
    if (!st) return NBODY_USER_ERROR;
    return nb_set_types(st, types);
}

NBodyCudaStatus nbHistogramCUDA(NBodyCudaState* st, const NBodyCudaHistogramParams* hp,
                                unsigned int* counts, unsigned int* totals,
                                double* massPerParticle, double* comps)
{
    if (!st) return NBODY_USER_ERROR;
    return nb_hist_run(st, nullptr, {st->nbody}, hp, nullptr, counts, totals, massPerParticle,
                       comps, nullptr);
}

NBodyCudaStatus nbLikelihoodCUDA(NBodyCudaState* st, const NBodyCudaHistogramParams* hp,
                                 const NBodyCudaDataHistogram* data, double* out)
{
    if (!st || !data || !out) return NBODY_USER_ERROR;
    return nb_hist_run(st, nullptr, {st->nbody}, hp, data, nullptr, nullptr, nullptr, nullptr, out);
}

// One forward run of nbRunSystemPlain (nbody/src/nbody_plain.c:365-470): nbGravMap, steps up
// to nStep with the best-likelihood scan on the device, the final likelihood.
static NBodyCudaStatus nb_run_once(const NBodyCudaCtx* ctx, NBodyCudaState* st,
                                   const NBodyCudaRunParams* rp, NbHistRun* hr,
                                   NbBestDev& bestHost, double* finalOut)
{
    const cudaStream_t s = st->stream;
    NbBestDev init{};
    init.best[0] = 9999999.9;                       // st->bestLikelihood = DEFAULT_WORST_CASE
    init.timeEvolve = rp->timeEvolve;
    NB_CHECK(cudaMemcpyAsync(st->best, &init, sizeof init, cudaMemcpyHostToDevice, s));
    NBodyCudaStatus all = nbGravMapCUDA(ctx, st);
    if (all & ~(int) NBODY_STATUS_WARNINGS_MASK) return all;
    const bool scan = hr && rp->useBestLike;
    while (st->step < rp->nStep) {
        NBodyCudaStatus rc = nbStepSystemCUDA(ctx, st);
        all |= rc;
        if (rc & ~(int) NBODY_STATUS_WARNINGS_MASK) return all;
        if (scan && (double) st->step / (double) rp->nStep >= rp->bestLikeStart) {
            nb_hist_launch(st, nullptr, *hr, true);
            nb_launch_best_update(hr->out, st->best, 1, st->step, rp->nStep, hr->f, s);
            if (rp->keepBestBodies) {
                NbTreeBuffers& b = st->b;
                nb_launch_keep_best(st->best, nullptr, b.px, b.py, b.pz, b.vx, b.vy, b.vz,
                                    st->nbody, st->keepPos, st->keepVel, st->numSMs, s);
            }
        }
    }
    if (hr) {
        nb_hist_launch(st, nullptr, *hr, true);
        NB_CHECK(cudaMemcpyAsync(finalOut, hr->out, 8 * NB_LIKELIHOOD_TERMS,
                                 cudaMemcpyDeviceToHost, s));
    }
    NB_CHECK(cudaMemcpyAsync(&bestHost, st->best, sizeof bestHost, cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaGetLastError());
    NB_CHECK(cudaStreamSynchronize(s));
    return all;
}

NBodyCudaStatus nbRunSystemCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st,
                                const NBodyCudaRunParams* rp, const NBodyCudaHistogramParams* hp,
                                const NBodyCudaDataHistogram* data, NBodyCudaRunResult* res)
{
    if (!st || !ctx || !rp || !res || rp->nStep < 0 || rp->calibrationRuns < 0) {
        g_lastError = "nbRunSystemCUDA: invalid arguments";
        return NBODY_USER_ERROR;
    }
    if ((rp->useBestLike || rp->keepBestBodies) && (!hp || !data)) {
        g_lastError = "nbRunSystemCUDA: the best-likelihood scan needs histogram parameters and data";
        return NBODY_USER_ERROR;
    }
    if (st->step > rp->nStep) {
        g_lastError = "nbRunSystemCUDA: the state is past nStep";
        return NBODY_USER_ERROR;
    }
    NB_CHECK(cudaSetDevice(st->device));
    *res = NBodyCudaRunResult{};
    for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t) res->result[t] = res->final[t] = NAN;
    NbHistRun hr;
    const bool like = hp && data;
    if (like) {
        NBodyCudaStatus rc = nb_hist_prepare(st, {st->nbody}, hp, data, false, hr);
        if (rc != NBODY_SUCCESS) return rc;
    }
    if (!st->best) NB_CHECK(cudaMalloc((void**) &st->best, sizeof(NbBestDev)));
    if (rp->keepBestBodies && !st->keepPos) {
        NB_CHECK(nb_alloc(&st->keepPos, 3 * (size_t) st->nbody));
        NB_CHECK(nb_alloc(&st->keepVel, 3 * (size_t) st->nbody));
    }
    // nbody.c:436-447: the bar's first time origin; calibration only with an orbiting bar
    const double og = (2 * rp->bestLikeStart) / (rp->bestLikeStart + 1);
    double pft = rp->useBestLike ? rp->timeEvolve / (2 - og) : rp->timeEvolve;
    const bool bar = ctx->potentialType == NBCUDA_POTENTIAL_DEFAULT &&
                     ctx->pot.disk2.type == NBCUDA_ORBITING_BAR;
    const int runs = 1 + (bar ? rp->calibrationRuns : 0);
    if (runs > 1) {
        NBodyCudaStatus rc = nb_save_slot(st, st->runStart);
        if (rc != NBODY_SUCCESS) return rc;
    }
    NBodyCudaStatus all = NBODY_SUCCESS;
    NbBestDev best{};
    double fin[NB_LIKELIHOOD_TERMS];
    for (int i = 0; i < runs; ++i) {
        if (i > 0) {
            NBodyCudaStatus rc = nb_restore_slot(st, st->runStart);
            if (rc != NBODY_SUCCESS) return rc;
        }
        st->timeOrigin = pft;
        st->haveKeep = 0;
        all |= nb_run_once(ctx, st, rp, like ? &hr : nullptr, best, fin);
        res->runs = i + 1;
        if (all & ~(int) NBODY_STATUS_WARNINGS_MASK) break;
        if (i < runs - 1) pft = best.bestTime;          // nbody.c:508-516
    }
    res->previousForwardTime = pft;
    res->bestTime = best.bestTime;
    res->bestStep = best.bestStep;
    res->bestCount = best.count;
    st->haveKeep = rp->keepBestBodies && best.count > 0;
    for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t) res->best[t] = best.best[t];
    if (like && !(all & ~(int) NBODY_STATUS_WARNINGS_MASK)) {
        // nbody.c:308-345: clamp the final likelihood, then the best one replaces it if better
        for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t) res->final[t] = fin[t];
        double& l = res->final[0];
        const double worst = 9999999.9;
        if (l > worst || l < -1 * worst) l = worst;
        else if (l == 0.0) l = 1e-9;
        const bool useBest = rp->useBestLike && fabs(res->final[0]) > fabs(best.best[0]);
        for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t)
            res->result[t] = useBest ? best.best[t] : res->final[t];
    }
    return all;
}

NBodyCudaStatus nbGetBestBodiesCUDA(NBodyCudaState* st, double* pos, double* vel)
{
    if (!st || !st->haveKeep) {
        g_lastError = "nbGetBestBodiesCUDA: no best-likelihood bodies kept";
        return NBODY_USER_ERROR;
    }
    NB_CHECK(cudaSetDevice(st->device));
    const size_t bytes = 3 * (size_t) st->nbody * sizeof(double);
    if (pos) NB_CHECK(cudaMemcpyAsync(pos, st->keepPos, bytes, cudaMemcpyDeviceToHost, st->stream));
    if (vel) NB_CHECK(cudaMemcpyAsync(vel, st->keepVel, bytes, cudaMemcpyDeviceToHost, st->stream));
    NB_CHECK(cudaStreamSynchronize(st->stream));
    return NBODY_SUCCESS;
}

}  // extern "C"

// =============================================================================================
// Batched dwarfs (nb_batch.cu builds the forest; the walks take the forest description)
// =============================================================================================
int nb_build_forest(NbTreeBuffers& b, const NbForest& f, int n, int capNodes, int criterion,
                    double theta, int useQuad, int drift, int numSMs, cudaStream_t s,
                    const NbBatchLMC* lmc);

struct NbBatchTuning {
    int groupMax = 32;      // bodies per walk group of the mixed walk
    int listCap = 64;       // interaction-list entries per warp
    int blocksPerSM = 0;    // resident walk blocks per SM (0: as many as fit)
    int exact = 1;          // each body's own interaction set (nbBatchSetMixedModeCUDA)
};

struct NBodyCudaBatch {
    NBodyCudaState* st = nullptr;       // the bodies of all dwarfs, concatenated
    int nDwarfs = 0;
    std::vector<NBodyCudaDwarf> dwarfs;  // host parameters
    NbDwarfDev* dDwarfs = nullptr;      // device table
    NbDwarfDev* hDwarfs = nullptr;      // pinned mirror
    int* bodyDwarf = nullptr;
    NbBatchTuning tune;
    int maxWalkBlocks = 0;              // walk stacks are sized for this many blocks
    // captured step
    cudaGraphExec_t graph = nullptr;
    NBodyCudaCtx graphCtx{};
    int graphDrift = -1, graphKick = -1, graphCap = -1, graphLaunches = 0;
    NbBatchTuning graphTune;
    double lastStepMs = 0.0;
    int lastSteps = 0;
    NbBestDev* best = nullptr;          // nbBatchRunSystemCUDA: per-dwarf best-likelihood records
    bool haveKeep = false;              // keepPos/keepVel of the state hold best bodies
    double* lmcShiftDev = nullptr;      // LMC runs: every dwarf's reflex accelerations
    int nShift = 0;                     // (nShift vectors per dwarf)
    std::vector<double> lmcHost;        // the LMC states nbBatchSetLMCCUDA gave, 6 per dwarf
};

static NbForest nb_forest_of(NBodyCudaBatch* bt, const NBodyCudaCtx* ctx = nullptr)
{
    const bool lmc = ctx && ctx->lmc && bt->lmcShiftDev;
    return NbForest{bt->bodyDwarf, bt->dDwarfs, bt->nDwarfs, lmc ? bt->lmcShiftDev : nullptr,
                    lmc ? bt->nShift : 0};
}

static void nb_batch_drop_graph(NBodyCudaBatch* bt)
{
    if (bt->graph) cudaGraphExecDestroy(bt->graph);
    bt->graph = nullptr;
    bt->graphCap = -1;
}

// Walk stacks for the largest persistent grid any tuning can ask for.
static NBodyCudaStatus nb_batch_mixed_buffers(NBodyCudaBatch* bt)
{
    NBodyCudaState* st = bt->st;
    if (!bt->maxWalkBlocks) {
        int mx = 0;
        for (int cap : {32, 64, 128})
            for (int gm : {32, 64}) mx = std::max(mx, nb_mixed_walk_blocks(st->numSMs, cap, gm));
        bt->maxWalkBlocks = mx;
    }
    if (!st->mx.stacks) NB_CHECK(nb_alloc(&st->mx.stacks, nb_mixed_stack_ints(bt->maxWalkBlocks)));
    const int fit = nb_mixed_walk_blocks(st->numSMs, bt->tune.listCap, bt->tune.groupMax) / st->numSMs;
    const int per = bt->tune.blocksPerSM > 0 ? std::min(bt->tune.blocksPerSM, fit) : fit;
    st->mx.walkBlocks = std::max(1, per) * st->numSMs;
    st->mx.groupMax = bt->tune.groupMax;
    st->mx.listCap = bt->tune.listCap;
    st->mx.exact = bt->tune.exact;
    return NBODY_SUCCESS;
}

// The device work of one evaluation, enqueued on the batch's stream without any host
// synchronisation (so that it can be captured in a graph).  Returns the launches issued.
static int nb_batch_enqueue(NBodyCudaBatch* bt, const NBodyCudaCtx* ctx, int drift, int kick)
{
    NBodyCudaState* st = bt->st;
    NbTreeBuffers& b = st->b;
    const cudaStream_t s = st->stream;
    const NbForest f = nb_forest_of(bt, ctx);
    NbWalkParams wp{};
    wp.useQuad = ctx->useQuad;
    wp.kick = kick;
    wp.n = st->nbody;
    NbPot pot = nb_pot_from(ctx);
    NbBatchLMC lmc{};
    const bool withLMC = f.lmcShift != nullptr;
    if (withLMC) {                      // each dwarf's LMC: its Plummer sphere on its bodies
        pot.lmcMass = ctx->lmcMass;
        pot.lmcScale = ctx->lmcScale;
        lmc.pot = nb_pot_from(ctx);
        lmc.mass = ctx->lmcMass;
        lmc.dynaFric = ctx->lmcDynaFric;
        lmc.coulombLog = ctx->coulombLog;
    }
    int launches = nb_build_forest(b, f, st->nbody, st->capNodes, ctx->criterion, ctx->theta,
                                   ctx->useQuad, drift, st->numSMs, s, withLMC ? &lmc : nullptr);
    if (withLMC && drift) launches += 1;
    cudaEventRecord(st->ev0, s);
    if (ctx->precision == NBCUDA_PRECISION_MIXED) {
        nb_launch_walk_mixed(b, st->mx, st->capNodes, wp, pot, false, st->numSMs, s, &f);
        launches += 3;
    } else {
        nb_launch_walk_fp64(b.nodePM, b.nodeCrit, b.nodeLink, b.nodeQuad, b.sort.idxA, b.px, b.py,
                            b.pz, b.ax, b.ay, b.az, b.vx, b.vy, b.vz, wp, pot, b.sc, false, s,
                            b.walkRec, st->capNodes, &f, st->walkForm > 0 ? st->walkForm : 0);
        launches += 1;
    }
    cudaEventRecord(st->ev1, s);
    if (withLMC && kick) {              // advanceVelocities_LMC after the bodies' kick
        nb_launch_b_lmc_half(lmc, f, b.sc, 1, s);
        launches += 1;
    }
    cudaMemcpyAsync(st->scHost, b.sc, sizeof(NbScalars), cudaMemcpyDeviceToHost, s);
    return launches;
}

static bool nb_same_tuning(const NbBatchTuning& a, const NbBatchTuning& b)
{
    return a.groupMax == b.groupMax && a.listCap == b.listCap && a.blocksPerSM == b.blocksPerSM &&
           a.exact == b.exact;
}

// One evaluation of every dwarf (drift/kick: the fused halves of the leapfrog), optionally
// through a captured graph of the whole sequence.
static NBodyCudaStatus nb_batch_eval(const NBodyCudaCtx* ctx, NBodyCudaBatch* bt, int drift,
                                     int kick, bool useGraph)
{
    NBodyCudaState* st = bt->st;
    const cudaStream_t s = st->stream;
    NbTreeBuffers& b = st->b;
    const bool mixed = ctx->precision == NBCUDA_PRECISION_MIXED;
    if (ctx->lmc && (drift || kick) && st->step + 2 > bt->nShift) {
        g_lastError = "the LMC's reflex accelerations do not reach this step";
        return NBODY_USER_ERROR;
    }
    for (int attempt = 0; attempt < 4; ++attempt) {
        if (mixed) {
            NBodyCudaStatus rc = nb_batch_mixed_buffers(bt);
            if (rc) return rc;
        }
        // the capacity the build checks against and the step count (the bar's time); the
        // reset kernel keeps both
        NB_CHECK(cudaMemcpyAsync(&b.sc->capNodes, &st->capNodes, sizeof(int),
                                 cudaMemcpyHostToDevice, s));
        NB_CHECK(cudaMemcpyAsync(&b.sc->step, &st->step, sizeof(int), cudaMemcpyHostToDevice, s));
        NB_CHECK(cudaMemcpyAsync(&b.sc->timeOrigin, &st->timeOrigin, sizeof(double),
                                 cudaMemcpyHostToDevice, s));
        NB_CHECK(cudaStreamSynchronize(s));
        if (useGraph) {
            const bool same = bt->graph && bt->graphDrift == drift && bt->graphKick == kick &&
                              bt->graphCap == st->capNodes && nb_same_tuning(bt->graphTune, bt->tune) &&
                              std::memcmp(&bt->graphCtx, ctx, sizeof *ctx) == 0;
            if (!same) {
                nb_batch_drop_graph(bt);
                cudaGraph_t g = nullptr;
                NB_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                const int launches = nb_batch_enqueue(bt, ctx, drift, kick);
                NB_CHECK(cudaStreamEndCapture(s, &g));
                cudaError_t e = cudaGraphInstantiate(&bt->graph, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) { bt->graph = nullptr; return nb_cuda_fail(e, "cudaGraphInstantiate"); }
                bt->graphCtx = *ctx;
                bt->graphDrift = drift;
                bt->graphKick = kick;
                bt->graphCap = st->capNodes;
                bt->graphTune = bt->tune;
                bt->graphLaunches = launches;
            } else {
                nb_count_launch(bt->graphLaunches);
            }
            NB_CHECK(cudaEventRecord(st->evS, s));
            NB_CHECK(cudaGraphLaunch(bt->graph, s));
            NB_CHECK(cudaEventRecord(st->evE, s));
        } else {
            NB_CHECK(cudaEventRecord(st->evS, s));
            nb_batch_enqueue(bt, ctx, drift, kick);
            NB_CHECK(cudaEventRecord(st->evE, s));
        }
        NB_CHECK(cudaGetLastError());
        NB_CHECK(cudaStreamSynchronize(s));
        const NbScalars& h = *st->scHost;
        if (h.status & NBODY_CELL_OVERFLOW_ERROR) {
            // grow the node arrays and redo this evaluation (positions already drifted)
            nb_batch_drop_graph(bt);
            NBodyCudaStatus rc = nb_alloc_nodes(st, h.neededNodes + h.neededNodes / 4 + 64);
            if (rc) return rc;
            drift = 0;
            continue;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, st->evS, st->evE);
        st->stepMs = ms;
        if (!useGraph) {
            ms = 0.0f;
            cudaEventElapsedTime(&ms, st->ev0, st->ev1);
            st->walkMs = ms;
        }
        NBodyCudaStatus out = h.status;
        if (h.incest) st->treeIncest = 1;
        if (st->treeIncest)
            out |= ctx->allowIncest ? NBODY_TREE_INCEST_NONFATAL : NBODY_TREE_INCEST_FATAL;
        st->haveTree = 1;
        st->lastCriterion = ctx->criterion;
        return out;
    }
    g_lastError = "node capacity could not be grown";
    return NBODY_CELL_OVERFLOW_ERROR;
}

static NBodyCudaStatus nb_batch_check(const NBodyCudaCtx* ctx, NBodyCudaBatch* bt)
{
    if (!bt) return NBODY_USER_ERROR;
    std::string why;
    NBodyCudaStatus rc = nb_check_ctx(ctx, why);
    if (rc) { g_lastError = why; return rc; }
    if (ctx->criterion == NBCUDA_EXACT) {
        g_lastError = "batched dwarfs use a tree criterion";
        return NBODY_UNSUPPORTED;
    }
    if (ctx->lmc && !bt->lmcShiftDev) {
        g_lastError = "an LMC context needs every dwarf's LMC state (nbBatchSetLMCCUDA)";
        return NBODY_USER_ERROR;
    }
    NB_CHECK(cudaSetDevice(bt->st->device));
    return NBODY_SUCCESS;
}

// Table of the dwarfs' parameters, root sizes back at treeRSize, statuses cleared.
static NBodyCudaStatus nb_batch_reset_table(NBodyCudaBatch* bt)
{
    int first = 0;
    for (int d = 0; d < bt->nDwarfs; ++d) {
        NbDwarfDev& h = bt->hDwarfs[d];
        h = NbDwarfDev{};
        h.rsize = bt->dwarfs[d].treeRSize;
        h.eps2 = bt->dwarfs[d].eps2;
        h.dt = bt->dwarfs[d].timestep;
        h.first = first;
        h.count = bt->dwarfs[d].nbody;
        first += h.count;
        if (!bt->lmcHost.empty())
            for (int c = 0; c < 6; ++c) h.lmc[c] = bt->lmcHost[6 * (size_t) d + c];
    }
    NB_CHECK(cudaMemcpyAsync(bt->dDwarfs, bt->hDwarfs, sizeof(NbDwarfDev) * bt->nDwarfs,
                             cudaMemcpyHostToDevice, bt->st->stream));
    NB_CHECK(cudaStreamSynchronize(bt->st->stream));
    bt->st->treeIncest = 0;
    bt->st->haveTree = 0;
    return NBODY_SUCCESS;
}

extern "C" {

NBodyCudaStatus nbBatchCreateCUDA(NBodyCudaBatch** out, int device, const NBodyCudaDwarf* dwarfs,
                                  int ndwarfs)
{
    if (!out || !dwarfs || ndwarfs < 1 || ndwarfs > 65535) return NBODY_USER_ERROR;
    *out = nullptr;
    long long total = 0;
    for (int d = 0; d < ndwarfs; ++d) {
        const NBodyCudaDwarf& w = dwarfs[d];
        if (w.nbody < 2 || !(w.eps2 >= 0.0) || !(w.timestep > 0.0)) {
            g_lastError = "every dwarf needs >= 2 bodies, eps2 >= 0 and a positive time step";
            return NBODY_USER_ERROR;
        }
        if (!nb_pow2(w.treeRSize)) {
            g_lastError = "treeRSize must be a positive power of two";
            return NBODY_UNSUPPORTED;
        }
        total += w.nbody;
    }
    if (total > (1ll << 30)) { g_lastError = "too many bodies"; return NBODY_USER_ERROR; }
    NBodyCudaState* st = nullptr;
    NBodyCudaStatus rc = nbInitCUDA(&st, device, (int) total);
    if (rc) return rc;
    NBodyCudaBatch* bt = new NBodyCudaBatch();
    bt->st = st;
    bt->nDwarfs = ndwarfs;
    bt->dwarfs.assign(dwarfs, dwarfs + ndwarfs);
    cudaError_t e = cudaMalloc((void**) &bt->dDwarfs, sizeof(NbDwarfDev) * ndwarfs);
    if (e == cudaSuccess) e = cudaMallocHost((void**) &bt->hDwarfs, sizeof(NbDwarfDev) * ndwarfs);
    if (e == cudaSuccess) e = cudaMalloc((void**) &bt->bodyDwarf, sizeof(int) * (size_t) total);
    if (e == cudaSuccess) {
        std::vector<int> owner((size_t) total);
        size_t k = 0;
        for (int d = 0; d < ndwarfs; ++d)
            for (int i = 0; i < dwarfs[d].nbody; ++i) owner[k++] = d;
        e = cudaMemcpy(bt->bodyDwarf, owner.data(), sizeof(int) * (size_t) total,
                       cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) rc = nb_cuda_fail(e, "nbBatchCreateCUDA");
    if (!rc) rc = nb_batch_reset_table(bt);
    if (rc) { nbBatchDestroyCUDA(bt); return rc; }
    *out = bt;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchDestroyCUDA(NBodyCudaBatch* bt)
{
    if (!bt) return NBODY_SUCCESS;
    if (bt->st) cudaSetDevice(bt->st->device);
    nb_batch_drop_graph(bt);
    cudaFree(bt->best);
    cudaFree(bt->lmcShiftDev);
    cudaFree(bt->dDwarfs);
    cudaFree(bt->bodyDwarf);
    if (bt->hDwarfs) cudaFreeHost(bt->hDwarfs);
    if (bt->st) nbDestroyCUDA(bt->st);
    delete bt;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchSetBodiesCUDA(NBodyCudaBatch* bt, const double* pos, const double* vel,
                                     const double* mass)
{
    if (!bt) return NBODY_USER_ERROR;
    for (int i = 0; mass && i < bt->st->nbody; ++i)
        if (!(mass[i] != 0.0)) {
            g_lastError = "batched dwarfs hold massive bodies only";
            return NBODY_UNSUPPORTED;
        }
    NBodyCudaStatus rc = nbSetBodiesCUDA(bt->st, pos, vel, mass, bt->st->nbody, 4.0);
    if (rc) return rc;
    return nb_batch_reset_table(bt);
}

NBodyCudaStatus nbBatchSetBodiesDeviceCUDA(NBodyCudaBatch* bt, const double* dpos,
                                           const double* dvel, const double* dmass)
{
    if (!bt) return NBODY_USER_ERROR;
    NBodyCudaStatus rc = nbSetBodiesDeviceCUDA(bt->st, dpos, dvel, dmass, bt->st->nbody, 4.0);
    if (rc) return rc;
    return nb_batch_reset_table(bt);
}

NBodyCudaStatus nbBatchGetBodiesCUDA(NBodyCudaBatch* bt, double* pos, double* vel, double* acc)
{
    if (!bt) return NBODY_USER_ERROR;
    NBodyCudaStatus rc = nbGetBodiesCUDA(bt->st, pos, vel);
    if (!rc && acc) rc = nbGetAccelsCUDA(bt->st, acc);
    return rc;
}

NBodyCudaStatus nbBatchGetBodiesDeviceCUDA(NBodyCudaBatch* bt, double* dpos, double* dvel,
                                           double* dacc)
{
    if (!bt) return NBODY_USER_ERROR;
    return nbGetBodiesDeviceCUDA(bt->st, dpos, dvel, dacc);
}

NBodyCudaStatus nbBatchGravMapCUDA(const NBodyCudaCtx* ctx, NBodyCudaBatch* bt)
{
    NBodyCudaStatus rc = nb_batch_check(ctx, bt);
    if (rc) return rc;
    return nb_batch_eval(ctx, bt, 0, 0, false);
}

NBodyCudaStatus nbBatchRunStepsCUDA(const NBodyCudaCtx* ctx, NBodyCudaBatch* bt, int nsteps,
                                    int useGraph)
{
    NBodyCudaStatus rc = nb_batch_check(ctx, bt);
    if (rc) return rc;
    if (nsteps < 0) return NBODY_USER_ERROR;
    if (!bt->st->haveTree) {
        // the first kick needs the accelerations of the initial positions
        rc = nb_batch_eval(ctx, bt, 0, 0, false);
        if (rc & ~(int) NBODY_STATUS_WARNINGS_MASK) return rc;
    }
    double total = 0.0;
    NBodyCudaStatus out = NBODY_SUCCESS;
    for (int k = 0; k < nsteps; ++k) {
        const NBodyCudaStatus rcStep = nb_batch_eval(ctx, bt, 1, 1, useGraph != 0);
        out |= rcStep;
        total += bt->st->stepMs;
        bt->st->step++;
        if (rcStep & ~(int) NBODY_STATUS_WARNINGS_MASK) break;
    }
    bt->lastStepMs = nsteps ? total / nsteps : 0.0;
    bt->lastSteps = nsteps;
    return out;
}

NBodyCudaStatus nbBatchDwarfInfoCUDA(NBodyCudaBatch* bt, int* status, double* rsize,
                                     int* rootNode, int* nodes)
{
    if (!bt) return NBODY_USER_ERROR;
    NB_CHECK(cudaSetDevice(bt->st->device));
    NB_CHECK(cudaMemcpyAsync(bt->hDwarfs, bt->dDwarfs, sizeof(NbDwarfDev) * bt->nDwarfs,
                             cudaMemcpyDeviceToHost, bt->st->stream));
    NB_CHECK(cudaStreamSynchronize(bt->st->stream));
    for (int d = 0; d < bt->nDwarfs; ++d) {
        const NbDwarfDev& h = bt->hDwarfs[d];
        if (status) status[d] = h.status;
        if (rsize) rsize[d] = h.rsize;
        if (rootNode) rootNode[d] = h.rootNode;
        if (nodes) nodes[d] = h.rootEnd - h.rootNode;
    }
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchSetTuningCUDA(NBodyCudaBatch* bt, int groupMax, int listCap,
                                     int blocksPerSM)
{
    if (!bt || groupMax < 1 || groupMax > 64 || (listCap != 32 && listCap != 64 && listCap != 128) ||
        blocksPerSM < 0)
        return NBODY_USER_ERROR;
    bt->tune.groupMax = groupMax;
    bt->tune.listCap = listCap;
    bt->tune.blocksPerSM = blocksPerSM;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchSetWalkFormCUDA(NBodyCudaBatch* bt, int form)
{
    if (!bt || form < 0 || form > 2) return NBODY_USER_ERROR;
    bt->st->walkForm = form;
    nb_batch_drop_graph(bt);            // the captured step holds the walk kernel
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchSetMixedModeCUDA(NBodyCudaBatch* bt, int exactSet)
{
    if (!bt || (exactSet != 0 && exactSet != 1)) return NBODY_USER_ERROR;
    bt->tune.exact = exactSet;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchGetTuningCUDA(NBodyCudaBatch* bt, int* groupMax, int* listCap,
                                     int* blocksPerSM)
{
    if (!bt) return NBODY_USER_ERROR;
    if (groupMax) *groupMax = bt->tune.groupMax;
    if (listCap) *listCap = bt->tune.listCap;
    if (blocksPerSM) *blocksPerSM = bt->tune.blocksPerSM;
    return NBODY_SUCCESS;
}

// The autotuner: times the mixed walk of the batch's current state (force evaluations without
// drift or kick, so the bodies do not move) for every candidate tuning -- bodies per walk group,
// interaction-list capacity, resident blocks per SM -- keeps the fastest, and re-evaluates the
// accelerations with it.  Each candidate is evaluated twice and timed on the second run.
NBodyCudaStatus nbBatchAutotuneCUDA(const NBodyCudaCtx* ctx, NBodyCudaBatch* bt, int* groupMax,
                                    int* listCap, int* blocksPerSM, double* walkMs)
{
    NBodyCudaStatus rc = nb_batch_check(ctx, bt);
    if (rc) return rc;
    NbBatchTuning best = bt->tune;
    double bestMs = -1.0;
    if (ctx->precision == NBCUDA_PRECISION_MIXED) {
        for (int g : {24, 32, 48, 64})
            for (int l : {32, 64, 128})
                for (int b : {0, 3}) {
                    bt->tune.groupMax = g;
                    bt->tune.listCap = l;
                    bt->tune.blocksPerSM = b;
                    for (int rep = 0; rep < 2; ++rep) {
                        rc = nb_batch_eval(ctx, bt, 0, 0, false);
                        if (rc & ~(int) NBODY_STATUS_WARNINGS_MASK) { bt->tune = best; return rc; }
                    }
                    const double ms = bt->st->walkMs;
                    if (bestMs < 0.0 || ms < bestMs) { bestMs = ms; best = bt->tune; }
                }
    }
    bt->tune = best;
    rc = nb_batch_eval(ctx, bt, 0, 0, false);
    if (bestMs < 0.0) bestMs = bt->st->walkMs;
    if (groupMax) *groupMax = best.groupMax;
    if (listCap) *listCap = best.listCap;
    if (blocksPerSM) *blocksPerSM = best.blocksPerSM;
    if (walkMs) *walkMs = bestMs;
    return rc;
}

NBodyCudaStatus nbBatchSetTimeOriginCUDA(NBodyCudaBatch* bt, double previousForwardTime)
{
    if (!bt) return NBODY_USER_ERROR;
    bt->st->timeOrigin = previousForwardTime;
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchSetTypesCUDA(NBodyCudaBatch* bt, const int* types)
{
    if (!bt) return NBODY_USER_ERROR;
    return nb_set_types(bt->st, types);
}

static std::vector<int> nb_batch_sizes(const NBodyCudaBatch* bt)
{
    std::vector<int> nb(bt->nDwarfs);
    for (int d = 0; d < bt->nDwarfs; ++d) nb[d] = bt->dwarfs[d].nbody;
    return nb;
}

NBodyCudaStatus nbBatchHistogramCUDA(NBodyCudaBatch* bt, const NBodyCudaHistogramParams* hp,
                                     unsigned int* counts, unsigned int* totals,
                                     double* massPerParticle, double* comps)
{
    if (!bt) return NBODY_USER_ERROR;
    return nb_hist_run(bt->st, bt->bodyDwarf, nb_batch_sizes(bt), hp, nullptr, counts, totals,
                       massPerParticle, comps, nullptr);
}

NBodyCudaStatus nbBatchLikelihoodCUDA(NBodyCudaBatch* bt, const NBodyCudaHistogramParams* hp,
                                      const NBodyCudaDataHistogram* data, double* out)
{
    if (!bt || !data || !out) return NBODY_USER_ERROR;
    return nb_hist_run(bt->st, bt->bodyDwarf, nb_batch_sizes(bt), hp, data, nullptr, nullptr,
                       nullptr, nullptr, out);
}

NBodyCudaStatus nbBatchGenerateDwarfsCUDA(NBodyCudaBatch* bt, const NBodyCudaPlummerDwarf* dwarfs)
{
    if (!bt || !dwarfs) return NBODY_USER_ERROR;
    std::vector<NBodyCudaMixedDwarf> m(bt->nDwarfs);
    for (int d = 0; d < bt->nDwarfs; ++d) m[d] = nb_mixed_from_plummer(dwarfs[d]);
    return nbBatchGenerateMixedDwarfsCUDA(bt, m.data());
}

NBodyCudaStatus nbBatchGenerateMixedDwarfsCUDA(NBodyCudaBatch* bt, const NBodyCudaMixedDwarf* dwarfs)
{
    if (!bt || !dwarfs) return NBODY_USER_ERROR;
    std::vector<int> firsts(bt->nDwarfs);
    int first = 0;
    for (int d = 0; d < bt->nDwarfs; ++d) {
        if (dwarfs[d].nbody != bt->dwarfs[d].nbody) {
            g_lastError = "dwarf body counts do not match the batch";
            return NBODY_USER_ERROR;
        }
        firsts[d] = first;
        first += dwarfs[d].nbody;
    }
    NBodyCudaStatus rc = nb_generate(bt->st, dwarfs, bt->nDwarfs, firsts.data());
    if (rc) return rc;
    return nb_batch_reset_table(bt);
}

// Sets every dwarf's own bar time origin (origins: nDwarfs values) in the device table.
static NBodyCudaStatus nb_batch_set_origins(NBodyCudaBatch* bt, const double* origins)
{
    NB_CHECK(cudaMemcpy2DAsync(&bt->dDwarfs[0].timeOrigin, sizeof(NbDwarfDev), origins,
                               sizeof(double), sizeof(double), (size_t) bt->nDwarfs,
                               cudaMemcpyHostToDevice, bt->st->stream));
    NB_CHECK(cudaStreamSynchronize(bt->st->stream));
    return NBODY_SUCCESS;
}

// One run of the batch (nbGravMap, the steps with the scan) into bestHost / fin (per dwarf).
static NBodyCudaStatus nb_batch_run_once(const NBodyCudaCtx* ctx, NBodyCudaBatch* bt,
                                         const NBodyCudaRunParams* rp, NbHistRun* hr, bool like,
                                         int useGraph, std::vector<NbBestDev>& bestHost,
                                         std::vector<double>& fin)
{
    NBodyCudaState* st = bt->st;
    const int D = bt->nDwarfs;
    const cudaStream_t s = st->stream;
    NbBestDev init{};
    init.best[0] = 9999999.9;                       // st->bestLikelihood = DEFAULT_WORST_CASE
    init.timeEvolve = rp->timeEvolve;
    bestHost.assign(D, init);
    NB_CHECK(cudaMemcpyAsync(bt->best, bestHost.data(), sizeof(NbBestDev) * (size_t) D,
                             cudaMemcpyHostToDevice, s));
    NBodyCudaStatus all = nb_batch_eval(ctx, bt, 0, 0, false);   // nbGravMap
    const bool scan = like && rp->useBestLike;
    double total = 0.0;
    int steps = 0;
    if (!(all & ~(int) NBODY_STATUS_WARNINGS_MASK)) {
        while (st->step < rp->nStep) {
            const NBodyCudaStatus rcStep = nb_batch_eval(ctx, bt, 1, 1, useGraph != 0);
            all |= rcStep;
            total += st->stepMs;
            ++steps;
            st->step++;
            if (rcStep & ~(int) NBODY_STATUS_WARNINGS_MASK) break;
            if (scan && (double) st->step / (double) rp->nStep >= rp->bestLikeStart) {
                nb_hist_launch(st, bt->bodyDwarf, *hr, true);
                nb_launch_best_update(hr->out, bt->best, D, st->step, rp->nStep, hr->f, s);
                if (rp->keepBestBodies) {
                    NbTreeBuffers& b = st->b;
                    nb_launch_keep_best(bt->best, bt->bodyDwarf, b.px, b.py, b.pz, b.vx, b.vy,
                                        b.vz, st->nbody, st->keepPos, st->keepVel, st->numSMs, s);
                }
            }
        }
    }
    bt->lastStepMs = steps ? total / steps : 0.0;
    bt->lastSteps = steps;
    fin.assign((size_t) NB_LIKELIHOOD_TERMS * D, NAN);
    if (like && !(all & ~(int) NBODY_STATUS_WARNINGS_MASK)) {
        nb_hist_launch(st, bt->bodyDwarf, *hr, true);
        NB_CHECK(cudaMemcpyAsync(fin.data(), hr->out, 8 * fin.size(), cudaMemcpyDeviceToHost, s));
    }
    NB_CHECK(cudaMemcpyAsync(bestHost.data(), bt->best, sizeof(NbBestDev) * (size_t) D,
                             cudaMemcpyDeviceToHost, s));
    NB_CHECK(cudaGetLastError());
    NB_CHECK(cudaStreamSynchronize(s));
    return all;
}

// nbRunSystemCUDA for every dwarf of the batch at once: the steps through the batch's step
// (captured graphs when useGraph), then with the best-likelihood scan each step of the window
// one histogram pass, one likelihood and one best-record update for all dwarfs; with an
// orbiting bar the calibration runs restart the whole batch from its initial state, each dwarf
// with its own previous best time as its bar's time origin.  res[d] as nbRunSystemCUDA's for
// dwarf d.
NBodyCudaStatus nbBatchRunSystemCUDA(const NBodyCudaCtx* ctx, NBodyCudaBatch* bt,
                                     const NBodyCudaRunParams* rp,
                                     const NBodyCudaHistogramParams* hp,
                                     const NBodyCudaDataHistogram* data, int useGraph,
                                     NBodyCudaRunResult* res)
{
    if (!bt || !ctx || !rp || !res || rp->nStep < 0 || rp->calibrationRuns < 0) {
        g_lastError = "nbBatchRunSystemCUDA: invalid arguments";
        return NBODY_USER_ERROR;
    }
    NBodyCudaStatus rc = nb_batch_check(ctx, bt);
    if (rc) return rc;
    if ((rp->useBestLike || rp->keepBestBodies) && (!hp || !data)) {
        g_lastError = "nbBatchRunSystemCUDA: the best-likelihood scan needs histogram parameters and data";
        return NBODY_USER_ERROR;
    }
    NBodyCudaState* st = bt->st;
    if (st->step > rp->nStep) {
        g_lastError = "nbBatchRunSystemCUDA: the batch is past nStep";
        return NBODY_USER_ERROR;
    }
    NB_CHECK(cudaSetDevice(st->device));
    const int D = bt->nDwarfs;
    const cudaStream_t s = st->stream;
    for (int d = 0; d < D; ++d) {
        res[d] = NBodyCudaRunResult{};
        for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t) res[d].result[t] = res[d].final[t] = NAN;
    }
    NbHistRun hr;
    const bool like = hp && data;
    if (like) {
        rc = nb_hist_prepare(st, nb_batch_sizes(bt), hp, data, false, hr);
        if (rc != NBODY_SUCCESS) return rc;
    }
    if (!bt->best) NB_CHECK(cudaMalloc((void**) &bt->best, sizeof(NbBestDev) * (size_t) D));
    if (rp->keepBestBodies && !st->keepPos) {
        NB_CHECK(nb_alloc(&st->keepPos, 3 * (size_t) st->nbody));
        NB_CHECK(nb_alloc(&st->keepVel, 3 * (size_t) st->nbody));
    }
    // nbody.c:436-447: the bar's first time origin; calibration only with an orbiting bar
    const double og = (2 * rp->bestLikeStart) / (rp->bestLikeStart + 1);
    const double pft = rp->useBestLike ? rp->timeEvolve / (2 - og) : rp->timeEvolve;
    const bool bar = ctx->potentialType == NBCUDA_POTENTIAL_DEFAULT &&
                     ctx->pot.disk2.type == NBCUDA_ORBITING_BAR;
    const int runs = 1 + (bar ? rp->calibrationRuns : 0);
    std::vector<double> origin(D, 0.0);             // the first run: the shared origin pft
    rc = nb_batch_set_origins(bt, origin.data());
    if (rc) return rc;
    std::vector<NbDwarfDev> tableStart;
    if (runs > 1) {
        rc = nb_save_slot(st, st->runStart);
        if (rc != NBODY_SUCCESS) return rc;
        tableStart.resize(D);
        NB_CHECK(cudaMemcpyAsync(tableStart.data(), bt->dDwarfs, sizeof(NbDwarfDev) * (size_t) D,
                                 cudaMemcpyDeviceToHost, s));
        NB_CHECK(cudaStreamSynchronize(s));
    }
    NBodyCudaStatus all = NBODY_SUCCESS;
    std::vector<NbBestDev> bestHost;
    std::vector<double> fin;
    std::vector<double> used(D, pft);               // each dwarf's origin in the last run
    int done = 0;
    for (int i = 0; i < runs; ++i) {
        if (i > 0) {
            rc = nb_restore_slot(st, st->runStart);
            if (rc != NBODY_SUCCESS) return rc;
            NB_CHECK(cudaMemcpyAsync(bt->dDwarfs, tableStart.data(), sizeof(NbDwarfDev) * (size_t) D,
                                     cudaMemcpyHostToDevice, s));
            for (int d = 0; d < D; ++d) origin[d] = used[d] = bestHost[d].bestTime;  // nbody.c:508-516
            st->timeOrigin = 0.0;
            rc = nb_batch_set_origins(bt, origin.data());
            if (rc) return rc;
        } else {
            st->timeOrigin = pft;
        }
        bt->haveKeep = false;
        all |= nb_batch_run_once(ctx, bt, rp, like ? &hr : nullptr, like, useGraph, bestHost, fin);
        done = i + 1;
        if (all & ~(int) NBODY_STATUS_WARNINGS_MASK) break;
    }
    const bool ok = !(all & ~(int) NBODY_STATUS_WARNINGS_MASK);
    for (int d = 0; d < D; ++d) {
        NBodyCudaRunResult& r = res[d];
        const NbBestDev& b = bestHost[d];
        r.runs = done;
        r.previousForwardTime = used[d];
        r.bestTime = b.bestTime;
        r.bestStep = b.bestStep;
        r.bestCount = b.count;
        bt->haveKeep = bt->haveKeep || (rp->keepBestBodies && b.count > 0);
        for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t) r.best[t] = b.best[t];
        if (!(like && ok)) continue;
        // nbody.c:308-345: clamp the final likelihood, then the best one replaces it if better
        for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t) r.final[t] = fin[(size_t) NB_LIKELIHOOD_TERMS * d + t];
        double& l = r.final[0];
        const double worst = 9999999.9;
        if (l > worst || l < -1 * worst) l = worst;
        else if (l == 0.0) l = 1e-9;
        const bool useBest = rp->useBestLike && fabs(r.final[0]) > fabs(b.best[0]);
        for (int t = 0; t < NB_LIKELIHOOD_TERMS; ++t) r.result[t] = useBest ? b.best[t] : r.final[t];
    }
    return all;
}

// Every dwarf's LMC: pos3/vel3 3 doubles per dwarf, shift nShift vectors of 3 doubles per
// dwarf (dwarf-major), as each dwarf's reverseOrbit_LMC leaves them.
NBodyCudaStatus nbBatchSetLMCCUDA(NBodyCudaBatch* bt, const double* pos3, const double* vel3,
                                  const double* shift, int nShift)
{
    if (!bt || !pos3 || !vel3 || !shift || nShift < 2) {
        g_lastError = "nbBatchSetLMCCUDA: positions, velocities and >= 2 reflex accelerations needed";
        return NBODY_USER_ERROR;
    }
    NBodyCudaState* st = bt->st;
    NB_CHECK(cudaSetDevice(st->device));
    const int D = bt->nDwarfs;
    const size_t bytes = sizeof(double) * 3 * (size_t) nShift * D;
    if (bt->lmcShiftDev && bt->nShift != nShift) {
        cudaFree(bt->lmcShiftDev);
        bt->lmcShiftDev = nullptr;
    }
    if (!bt->lmcShiftDev) NB_CHECK(cudaMalloc((void**) &bt->lmcShiftDev, bytes));
    bt->nShift = nShift;
    NB_CHECK(cudaMemcpyAsync(bt->lmcShiftDev, shift, bytes, cudaMemcpyHostToDevice, st->stream));
    bt->lmcHost.assign(6 * (size_t) D, 0.0);
    for (int d = 0; d < D; ++d)
        for (int c = 0; c < 3; ++c) {
            bt->lmcHost[6 * (size_t) d + c] = pos3[3 * (size_t) d + c];
            bt->lmcHost[6 * (size_t) d + 3 + c] = vel3[3 * (size_t) d + c];
        }
    NB_CHECK(cudaMemcpy2DAsync(&bt->dDwarfs[0].lmc[0], sizeof(NbDwarfDev), bt->lmcHost.data(),
                               6 * sizeof(double), 6 * sizeof(double), (size_t) D,
                               cudaMemcpyHostToDevice, st->stream));
    NB_CHECK(cudaStreamSynchronize(st->stream));
    nb_batch_drop_graph(bt);
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchGetLMCCUDA(NBodyCudaBatch* bt, double* pos3, double* vel3)
{
    if (!bt || !bt->lmcShiftDev) {
        g_lastError = "nbBatchGetLMCCUDA: no LMC set";
        return NBODY_USER_ERROR;
    }
    NBodyCudaState* st = bt->st;
    NB_CHECK(cudaSetDevice(st->device));
    const int D = bt->nDwarfs;
    std::vector<double> h(6 * (size_t) D);
    NB_CHECK(cudaMemcpy2DAsync(h.data(), 6 * sizeof(double), &bt->dDwarfs[0].lmc[0],
                               sizeof(NbDwarfDev), 6 * sizeof(double), (size_t) D,
                               cudaMemcpyDeviceToHost, st->stream));
    NB_CHECK(cudaStreamSynchronize(st->stream));
    for (int d = 0; d < D; ++d)
        for (int c = 0; c < 3; ++c) {
            if (pos3) pos3[3 * (size_t) d + c] = h[6 * (size_t) d + c];
            if (vel3) vel3[3 * (size_t) d + c] = h[6 * (size_t) d + 3 + c];
        }
    return NBODY_SUCCESS;
}

// The bodies of every dwarf at its best likelihood (valid for the dwarfs whose bestCount > 0).
NBodyCudaStatus nbBatchGetBestBodiesCUDA(NBodyCudaBatch* bt, double* pos, double* vel)
{
    if (!bt || !bt->haveKeep) {
        g_lastError = "nbBatchGetBestBodiesCUDA: no best-likelihood bodies kept";
        return NBODY_USER_ERROR;
    }
    NBodyCudaState* st = bt->st;
    NB_CHECK(cudaSetDevice(st->device));
    const size_t bytes = 3 * (size_t) st->nbody * sizeof(double);
    if (pos) NB_CHECK(cudaMemcpyAsync(pos, st->keepPos, bytes, cudaMemcpyDeviceToHost, st->stream));
    if (vel) NB_CHECK(cudaMemcpyAsync(vel, st->keepVel, bytes, cudaMemcpyDeviceToHost, st->stream));
    NB_CHECK(cudaStreamSynchronize(st->stream));
    return NBODY_SUCCESS;
}

NBodyCudaStatus nbBatchLastStepTimeCUDA(NBodyCudaBatch* bt, double* stepMs)
{
    if (!bt || !stepMs) return NBODY_USER_ERROR;
    *stepMs = bt->lastSteps ? bt->lastStepMs : bt->st->stepMs;
    return NBODY_SUCCESS;
}

}  // extern "C"
