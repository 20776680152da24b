/*
 * ref_shim.c -- ctypes entry points into the reference N-body client's own CPU code.
 *
 * Test infrastructure only (the checker, never the product).  Compiled by oracle/ref.mk
 * together with the reference sources into oracle/_ref/libnbref.so; it includes the
 * reference's headers and calls its public functions unchanged:
 *   nbGravMap (nbody/src/nbody_grav.c:305), nbStepSystem (nbody/src/nbody.c:182),
 *   nbMakeTree (nbody/src/nbody_tree.c:429), nbExtAcceleration
 *   (nbody/src/nbody_potential.c:627), nbSetup (nbody/src/nbody_lua.c:612),
 *   nbCreateHistogram / nbReadHistogram / nbSystemLikelihood (nbody/src/nbody.c:217-397).
 * The mapping from the reference's NBodyCtx to the flat NBodyCudaCtx of include/nbody_b200.h
 * is the binding's own (milkywayathome_client_b200/reference_binding/nbody_cuda_ctx.h).
 */
#include "nbody_priv.h"
#include "nbody.h"
#include "nbody_lua.h"
#include "nbody_grav.h"
#include "nbody_tree.h"
#include "nbody_potential.h"
#include "nbody_histogram.h"
#include "nbody_likelihood.h"
#include "nbody_orbit_integrator.h"
#include "nbody_checkpoint.h"
#include "nbody_emd.h"
#include "nbody_defaults.h"
#include "milkyway_util.h"
#include <crlibm.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include "../include/nbody_b200.h"
#include "../milkywayathome_client_b200/reference_binding/nbody_cuda_ctx.h"

/* The reference's force walk itself (nbGravity and nbMapForceBody are file-static in
 * nbody/src/nbody_grav.c): compiled here from that source so that a bounded sample of the
 * walk can be timed; oracle/ref.mk leaves nbody_grav.o out of libnbref.so accordingly. */
#include "nbody_grav.c"
#include <omp.h>

typedef struct {
    NBodyCtx ctx;
    NBodyState st;
    NBodyFlags nbf;
    int fromLua;
} RefHandle;

/* ---- layout facts of the reference ABI ---- */
int nbref_layout(long* out, int n)
{
    long v[] = { (long) sizeof(Body), (long) offsetof(Body, bodynode.pos),
                 (long) offsetof(Body, bodynode.mass), (long) offsetof(Body, bodynode.type),
                 (long) offsetof(Body, bodynode.id), (long) offsetof(Body, vel),
                 (long) sizeof(mwvector), (long) sizeof(NBodyCell) };
    int k, m = (int) (sizeof v / sizeof v[0]);
    for (k = 0; k < n && k < m; ++k) out[k] = v[k];
    return m;
}

/* ---- NBodyCtx <-> NBodyCudaCtx ---- */
void nbref_ctx_from_flat(NBodyCtx* ctx, const NBodyCudaCtx* c)
{
    static const NBodyCtx empty = EMPTY_NBODYCTX;
    *ctx = empty;
    ctx->eps2 = c->eps2;
    ctx->theta = c->theta;
    ctx->timestep = c->timestep;
    ctx->treeRSize = c->treeRSize;
    ctx->criterion = (criterion_t) c->criterion;
    ctx->useQuad = (mwbool) c->useQuad;
    ctx->allowIncest = (mwbool) c->allowIncest;
    ctx->quietErrors = TRUE;
    ctx->potentialType = (ExternalPotentialType) c->potentialType;
    ctx->pot.sphere[0].type = (spherical_t) c->pot.sphere.type;
    ctx->pot.sphere[0].mass = c->pot.sphere.mass;
    ctx->pot.sphere[0].scale = c->pot.sphere.scale;
    ctx->pot.disk.type = (disk_t) c->pot.disk.type;
    ctx->pot.disk.mass = c->pot.disk.mass;
    ctx->pot.disk.scaleLength = c->pot.disk.scaleLength;
    ctx->pot.disk.scaleHeight = c->pot.disk.scaleHeight;
    ctx->pot.disk.patternSpeed = c->pot.disk.patternSpeed;
    ctx->pot.disk.startAngle = c->pot.disk.startAngle;
    ctx->pot.disk2.type = (disk_t) c->pot.disk2.type;
    ctx->pot.disk2.mass = c->pot.disk2.mass;
    ctx->pot.disk2.scaleLength = c->pot.disk2.scaleLength;
    ctx->pot.disk2.scaleHeight = c->pot.disk2.scaleHeight;
    ctx->pot.disk2.patternSpeed = c->pot.disk2.patternSpeed;
    ctx->pot.disk2.startAngle = c->pot.disk2.startAngle;
    ctx->pot.halo.type = (halo_t) c->pot.halo.type;
    ctx->pot.halo.vhalo = c->pot.halo.vhalo;
    ctx->pot.halo.scaleLength = c->pot.halo.scaleLength;
    ctx->pot.halo.flattenZ = c->pot.halo.flattenZ;
    ctx->pot.halo.flattenY = c->pot.halo.flattenY;
    ctx->pot.halo.flattenX = c->pot.halo.flattenX;
    ctx->pot.halo.triaxAngle = c->pot.halo.triaxAngle;
    ctx->pot.halo.c1 = c->pot.halo.c1;
    ctx->pot.halo.c2 = c->pot.halo.c2;
    ctx->pot.halo.c3 = c->pot.halo.c3;
    ctx->pot.halo.mass = c->pot.halo.mass;
    ctx->pot.halo.gamma = c->pot.halo.gamma;
    ctx->pot.halo.lambda = c->pot.halo.lambda;
    ctx->pot.halo.rho0 = c->pot.halo.rho0;
    ctx->LMC = (mwbool) c->lmc;
    ctx->LMCDynaFric = (mwbool) c->lmcDynaFric;
    ctx->LMCmass = c->lmcMass;
    ctx->LMCscale = c->lmcScale;
    ctx->coulomb_log = c->coulombLog;
}

/* the binding's own mapping (milkywayathome_client_b200/reference_binding/nbody_cuda_ctx.h) */
void nbref_ctx_to_flat(NBodyCudaCtx* c, const NBodyCtx* ctx) { nbCudaCtxFromNBodyCtx(c, ctx); }

/* ---- states built from arrays ---- */
void* nbref_state_new(const NBodyCudaCtx* c, const double* pos, const double* vel,
                      const double* mass, const int* type, int n)
{
    static const NBodyState emptyState = EMPTY_NBODYSTATE;
    RefHandle* h = (RefHandle*) calloc(1, sizeof(RefHandle));
    Body* bodies;
    int i;
    nbref_ctx_from_flat(&h->ctx, c);
    h->ctx.nStep = 0;
    h->st = emptyState;
    bodies = (Body*) mwMallocA((n > 0 ? n : 1) * sizeof(Body));
    memset(bodies, 0, (n > 0 ? n : 1) * sizeof(Body));
    for (i = 0; i < n; ++i) {
        SET_VECTOR(Pos(&bodies[i]), pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        SET_VECTOR(Vel(&bodies[i]), vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        Mass(&bodies[i]) = mass[i];
        Type(&bodies[i]) = (body_t) (type ? type[i] : 1);
        idBody(&bodies[i]) = (unsigned int) i;
    }
    setInitialNBodyState(&h->st, &h->ctx, bodies, n);
    return h;
}

int nbref_state_gravmap(void* hv)
{
    RefHandle* h = (RefHandle*) hv;
    return (int) nbGravMap(&h->ctx, &h->st);
}

int nbref_state_maketree(void* hv)
{
    RefHandle* h = (RefHandle*) hv;
    return (int) nbMakeTree(&h->ctx, &h->st);
}

/* nsteps of nbStepSystem; stops at the first fatal status as nbRunSystemPlain does. */
int nbref_state_step(void* hv, int nsteps)
{
    RefHandle* h = (RefHandle*) hv;
    int k, all = 0;
    for (k = 0; k < nsteps; ++k) {
        NBodyStatus rc = nbStepSystem(&h->ctx, &h->st);
        all |= (int) rc;
        if (nbStatusIsFatal(rc)) break;
    }
    return all;
}

void nbref_state_get(void* hv, double* pos, double* vel, double* acc, double* rsize, int* step,
                     int* incest)
{
    RefHandle* h = (RefHandle*) hv;
    int i;
    for (i = 0; i < h->st.nbody; ++i) {
        const Body* b = &h->st.bodytab[i];
        if (pos) { pos[3 * i] = X(Pos(b)); pos[3 * i + 1] = Y(Pos(b)); pos[3 * i + 2] = Z(Pos(b)); }
        if (vel) { vel[3 * i] = X(Vel(b)); vel[3 * i + 1] = Y(Vel(b)); vel[3 * i + 2] = Z(Vel(b)); }
        if (acc) {
            acc[3 * i] = X(h->st.acctab[i]);
            acc[3 * i + 1] = Y(h->st.acctab[i]);
            acc[3 * i + 2] = Z(h->st.acctab[i]);
        }
    }
    if (rsize) *rsize = h->st.tree.rsize;
    if (step) *step = (int) h->st.step;
    if (incest) *incest = h->st.treeIncest;
}

/* Masses and types of the bodies (Lua-built states). */
void nbref_state_masses(void* hv, double* mass, int* type)
{
    RefHandle* h = (RefHandle*) hv;
    int i;
    for (i = 0; i < h->st.nbody; ++i) {
        if (mass) mass[i] = Mass(&h->st.bodytab[i]);
        if (type) type[i] = Type(&h->st.bodytab[i]);
    }
}

/* st->previousForwardTime: the bar's time origin (barTime = step * timestep - this) */
void nbref_state_set_time_origin(void* hv, double t)
{
    ((RefHandle*) hv)->st.previousForwardTime = t;
}

void nbref_state_set(void* hv, const double* pos, const double* vel)
{
    RefHandle* h = (RefHandle*) hv;
    int i;
    for (i = 0; i < h->st.nbody; ++i) {
        Body* b = &h->st.bodytab[i];
        if (pos) SET_VECTOR(Pos(b), pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        if (vel) SET_VECTOR(Vel(b), vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
}

int nbref_state_nbody(void* hv) { return ((RefHandle*) hv)->st.nbody; }

static int cmp_ptr(const void* a, const void* b)
{
    const char* x = *(const char* const*) a;
    const char* y = *(const char* const*) b;
    return x < y ? -1 : (x > y);
}

static int ptr_index(const void** sorted, const int* idx, int n, const void* p)
{
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        int mid = (lo + hi) / 2;
        if ((const char*) sorted[mid] == (const char*) p) return idx[mid];
        if ((const char*) sorted[mid] < (const char*) p) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

/* Tree of the last nbMakeTree in walk (Next/More preorder) order; returns the node count.
 * Arrays as in nbGetTreeCUDA (include/nbody_b200.h); any may be NULL; cap = their length. */
int nbref_state_tree(void* hv, int cap, double* pos, double* mass, double* rcrit2, double* quad,
                     int* next, int* body, int* depth)
{
    RefHandle* h = (RefHandle*) hv;
    const NBodyNode* p;
    const void** ptrs;
    const void** sorted;
    int* order;
    int* idx;
    int n = 0, k;
    for (p = (const NBodyNode*) h->st.tree.root; p; p = isCell(p) ? More(p) : Next(p)) ++n;
    if (n > cap) return -n;
    ptrs = (const void**) malloc(sizeof(void*) * (n + 1));
    sorted = (const void**) malloc(sizeof(void*) * (n + 1));
    order = (int*) malloc(sizeof(int) * (n + 1));
    idx = (int*) malloc(sizeof(int) * (n + 1));
    k = 0;
    for (p = (const NBodyNode*) h->st.tree.root; p; p = isCell(p) ? More(p) : Next(p)) ptrs[k++] = p;
    {   /* sort pointers to map them back to walk indices */
        const void** tmp = (const void**) malloc(sizeof(void*) * (n + 1));
        for (k = 0; k < n; ++k) tmp[k] = ptrs[k];
        qsort(tmp, (size_t) n, sizeof(void*), cmp_ptr);
        for (k = 0; k < n; ++k) sorted[k] = tmp[k];
        free(tmp);
        for (k = 0; k < n; ++k) {
            int lo = 0, hi = n - 1;
            while (lo <= hi) {
                int mid = (lo + hi) / 2;
                if (sorted[mid] == ptrs[k]) { idx[mid] = k; break; }
                if ((const char*) sorted[mid] < (const char*) ptrs[k]) lo = mid + 1; else hi = mid - 1;
            }
        }
    }
    {
        /* depth by walking: a cell's children are More(c), then Next() until Next(c) */
        int* dep = (int*) calloc((size_t) n + 1, sizeof(int));
        for (k = 0; k < n; ++k) {
            const NBodyNode* q = (const NBodyNode*) ptrs[k];
            if (isCell(q)) {
                const NBodyNode* c = More(q);
                const NBodyNode* stop = Next(q);
                while (c && c != stop) {
                    int ci = ptr_index(sorted, idx, n, c);
                    if (ci >= 0) dep[ci] = dep[k] + 1;
                    c = Next(c);
                }
            }
        }
        for (k = 0; k < n; ++k) {
            const NBodyNode* q = (const NBodyNode*) ptrs[k];
            const NBodyNode* nx = Next(q);
            if (pos) { pos[3 * k] = X(Pos(q)); pos[3 * k + 1] = Y(Pos(q)); pos[3 * k + 2] = Z(Pos(q)); }
            if (mass) mass[k] = Mass(q);
            if (next) next[k] = nx ? ptr_index(sorted, idx, n, nx) : n;
            if (depth) depth[k] = dep[k];
            if (isCell(q)) {
                if (rcrit2) rcrit2[k] = Rcrit2(q);
                if (quad) {
                    if (h->ctx.useQuad) {
                        quad[6 * k + 0] = Quad(q).xx; quad[6 * k + 1] = Quad(q).xy;
                        quad[6 * k + 2] = Quad(q).xz; quad[6 * k + 3] = Quad(q).yy;
                        quad[6 * k + 4] = Quad(q).yz; quad[6 * k + 5] = Quad(q).zz;
                    } else memset(quad + 6 * k, 0, 6 * sizeof(double));
                }
                if (body) body[k] = -1;
            } else {
                if (rcrit2) rcrit2[k] = 0.0;
                if (quad) memset(quad + 6 * k, 0, 6 * sizeof(double));
                if (body) body[k] = (int) ((const Body*) q - h->st.bodytab);
            }
        }
        free(dep);
    }
    free(ptrs); free(sorted); free(order); free(idx);
    return n;
}

void nbref_state_tree_info(void* hv, double* rsize, int* cellUsed, int* maxDepth)
{
    RefHandle* h = (RefHandle*) hv;
    if (rsize) *rsize = h->st.tree.rsize;
    if (cellUsed) *cellUsed = (int) h->st.tree.cellUsed;
    if (maxDepth) *maxDepth = (int) h->st.tree.maxDepth;
}

void nbref_state_free(void* hv)
{
    RefHandle* h = (RefHandle*) hv;
    if (!h) return;
    destroyNBodyState(&h->st);
    if (h->fromLua) {
        free(h->nbf.inputFile);
        free(h->nbf.histogramFileName);
        if (h->nbf.forwardedArgs) {
            unsigned int k;
            for (k = 0; k < h->nbf.numForwardedArgs; ++k) free((void*) h->nbf.forwardedArgs[k]);
            free((void*) h->nbf.forwardedArgs);
        }
    }
    free(h);
}

/* ---- Lua-described runs (nbSetup, nbody/src/nbody_lua.c:612) ---- */
void* nbref_open_lua(const char* luaFile, const char* histFile, unsigned int seed,
                     const char* const* args, int nargs)
{
    static const NBodyState emptyState = EMPTY_NBODYSTATE;
    static const NBodyCtx emptyCtx = EMPTY_NBODYCTX;
    static const NBodyFlags emptyFlags = EMPTY_NBODY_FLAGS;
    RefHandle* h = (RefHandle*) calloc(1, sizeof(RefHandle));
    int k;
    h->ctx = emptyCtx;
    h->st = emptyState;
    h->nbf = emptyFlags;
    h->fromLua = 1;
    h->nbf.inputFile = strdup(luaFile);
    h->nbf.histogramFileName = histFile ? strdup(histFile) : NULL;
    h->nbf.setSeed = 1;
    h->nbf.seed = seed;
    h->nbf.ignoreCheckpoint = 1;
    h->nbf.numForwardedArgs = (unsigned int) nargs;
    h->nbf.forwardedArgs = (const char**) calloc((size_t) (nargs > 0 ? nargs : 1), sizeof(char*));
    for (k = 0; k < nargs; ++k) h->nbf.forwardedArgs[k] = strdup(args[k]);
    if (nbSetup(&h->ctx, &h->st, &h->nbf)) {
        nbref_state_free(h);
        return NULL;
    }
    h->ctx.quietErrors = TRUE;
    h->st.previousForwardTime = h->ctx.timeEvolve;
    /* the comparison switches nbMain copies into the state before the run (nbody.c:485-490) */
    h->st.useVelDisp = h->ctx.useVelDisp;
    h->st.useBetaDisp = h->ctx.useBetaDisp;
    h->st.useBetaComp = h->ctx.useBetaComp;
    h->st.useVlos = h->ctx.useVlos;
    h->st.useDist = h->ctx.useDist;
    h->st.usePropMot = h->ctx.usePropMot;
    /* an LMC run takes the LMC's state and the reflex accelerations that reverseOrbit_LMC
     * left behind (nbody/src/nbody_plain.c:372-385) */
    if (h->ctx.LMC && !h->st.shiftByLMC) {
        mwvector* shift;
        size_t nShift;
        mwvector x, v;
        getLMCArray(&shift, &nShift);
        setLMCShiftArray(&h->st, shift, nShift);
        getLMCPosVel(&x, &v);
        setLMCPosVel(&h->st, x, v);
    }
    return h;
}

/* Installs an LMC on the handle's state: position, velocity and n reflex accelerations
 * (3 doubles each), as nbRunSystemPlain takes them from reverseOrbit_LMC
 * (nbody/src/nbody_plain.c:372-385); the state frees the array (nbody_types.c:123). */
void nbref_handle_set_lmc(void* hv, const double* pos3, const double* vel3, const double* shift,
                          int n)
{
    RefHandle* h = (RefHandle*) hv;
    mwvector x, v;
    mwvector* arr = (mwvector*) mwCallocA((size_t) (n > 0 ? n : 1), sizeof(mwvector));
    int k;
    for (k = 0; k < n; ++k) SET_VECTOR(arr[k], shift[3 * k], shift[3 * k + 1], shift[3 * k + 2]);
    if (h->st.shiftByLMC) mwFreeA(h->st.shiftByLMC);
    setLMCShiftArray(&h->st, arr, (size_t) n);
    SET_VECTOR(x, pos3[0], pos3[1], pos3[2]);
    SET_VECTOR(v, vel3[0], vel3[1], vel3[2]);
    setLMCPosVel(&h->st, x, v);
}

/* The LMC of the handle's state: its position and velocity (pos3, vel3) and up to cap
 * reflex accelerations (3 doubles each) into shift; returns their count (0 without an LMC). */
int nbref_handle_lmc(void* hv, double* pos3, double* vel3, double* shift, int cap)
{
    RefHandle* h = (RefHandle*) hv;
    int k, n;
    pos3[0] = X(h->st.LMCpos); pos3[1] = Y(h->st.LMCpos); pos3[2] = Z(h->st.LMCpos);
    vel3[0] = X(h->st.LMCvel); vel3[1] = Y(h->st.LMCvel); vel3[2] = Z(h->st.LMCvel);
    if (!h->st.shiftByLMC) return 0;
    n = (int) h->st.nShiftLMC;
    for (k = 0; k < n && k < cap; ++k) {
        shift[3 * k] = X(h->st.shiftByLMC[k]);
        shift[3 * k + 1] = Y(h->st.shiftByLMC[k]);
        shift[3 * k + 2] = Z(h->st.shiftByLMC[k]);
    }
    return n;
}

void nbref_handle_ctx(void* hv, NBodyCudaCtx* out, int* nStep, double* timeEvolve)
{
    RefHandle* h = (RefHandle*) hv;
    nbref_ctx_to_flat(out, &h->ctx);
    if (nStep) *nStep = (int) h->ctx.nStep;
    if (timeEvolve) *timeEvolve = h->ctx.timeEvolve;
}

/* The run-loop settings of the handle's context: useBestLike, BestLikeStart and
 * calibrationRuns (nbody/include/nbody_types.h:477-512). */
void nbref_handle_run_params(void* hv, int* useBestLike, double* bestLikeStart,
                             int* calibrationRuns)
{
    RefHandle* h = (RefHandle*) hv;
    *useBestLike = (int) h->ctx.useBestLike;
    *bestLikeStart = h->ctx.BestLikeStart;
    *calibrationRuns = (int) h->ctx.calibrationRuns;
}

/* The likelihood settings of the handle's context: flags[6] = useBetaDisp, useVelDisp,
 * useBetaComp, useVlos, useDist, usePropMot; sig[8] = Beta/Vel/Dist/PM sigma cut-offs, then
 * Beta/Vel/Dist/PM corrections; *iterMax = IterMax; sun[7] = sunGCDist, sunVelx/y/z, NGPdec,
 * NGPra, lNCP (nbody/include/nbody_types.h:455-512). */
void nbref_handle_like_params(void* hv, int* flags, double* sig, int* iterMax, double* sun)
{
    RefHandle* h = (RefHandle*) hv;
    const NBodyCtx* c = &h->ctx;
    flags[0] = (int) c->useBetaDisp; flags[1] = (int) c->useVelDisp;
    flags[2] = (int) c->useBetaComp; flags[3] = (int) c->useVlos;
    flags[4] = (int) c->useDist; flags[5] = (int) c->usePropMot;
    sig[0] = c->BetaSigma; sig[1] = c->VelSigma; sig[2] = c->DistSigma; sig[3] = c->PMSigma;
    sig[4] = c->BetaCorrect; sig[5] = c->VelCorrect; sig[6] = c->DistCorrect; sig[7] = c->PMCorrect;
    *iterMax = (int) c->IterMax;
    sun[0] = c->sunGCDist; sun[1] = c->sunVelx; sun[2] = c->sunVely; sun[3] = c->sunVelz;
    sun[4] = c->NGPdec; sun[5] = c->NGPra; sun[6] = c->lNCP;
}

/* The reference's run loop without checkpoints / best-likelihood tracking:
 * nbGravMap once, then nStep x nbStepSystem (nbody/src/nbody_plain.c:366-446). */
int nbref_run(void* hv)
{
    RefHandle* h = (RefHandle*) hv;
    NBodyStatus rc = nbGravMap(&h->ctx, &h->st);
    if (nbStatusIsFatal(rc)) return (int) rc;
    while (h->st.step < h->ctx.nStep) {
        rc |= nbStepSystem(&h->ctx, &h->st);
        if (nbStatusIsFatal(rc)) break;
    }
    return (int) rc;
}

/* Final likelihood as nbReportResults computes it (nbody/src/nbody.c:217-397); out[0..9] =
 * likelihood, EMD, mass, beta, vel, betaAvg, velAvg, dist, pm_dec, pm_ra (not negated). */
int nbref_likelihood(void* hv, double* out)
{
    RefHandle* h = (RefHandle*) hv;
    HistogramParams hp;
    NBodyLikelihoodMethod method;
    MainStruct* histogram;
    MainStruct* data;
    real* arr;
    int k;
    if (!h->nbf.histogramFileName) return -1;
    if (nbGetLikelihoodInfo(&h->nbf, &hp, &method) || method == NBODY_INVALID_METHOD) return -2;
    histogram = nbCreateHistogram(&h->ctx, &h->st, &hp);
    if (!histogram) return -3;
    data = nbReadHistogram(h->nbf.histogramFileName);
    if (!data) { free(histogram); return -4; }
    arr = nbSystemLikelihood(&h->st, data, histogram, method);
    for (k = 0; k < 10; ++k) out[k] = arr[k];
    if (out[0] > DEFAULT_WORST_CASE || out[0] < -DEFAULT_WORST_CASE) out[0] = DEFAULT_WORST_CASE;
    else if (out[0] == 0.0) out[0] = DEFAULT_BEST_CASE;
    if (isnan(out[0])) out[0] = DEFAULT_WORST_CASE;
    for (k = 0; k < 8; ++k) {
        free(histogram->histograms[k]);
        free(data->histograms[k]);
    }
    free(histogram);
    free(data);
    return 0;
}

/* Points the handle's likelihood at another data histogram file (nbf.histogramFileName,
 * which nbReportResults reads when the run ends). */
void nbref_handle_set_hist(void* hv, const char* histFile)
{
    RefHandle* h = (RefHandle*) hv;
    if (h->fromLua) free(h->nbf.histogramFileName);
    h->nbf.histogramFileName = histFile ? strdup(histFile) : NULL;
    h->fromLua = 1;
}

/* ---- checkpoints (nbWriteCheckpoint / nbReadCheckpoint, nbody/src/nbody_checkpoint.c:597-672) */

/* The state's Body[] (NBCUDA_BODY_STRIDE-byte records): the host table a GPU state marshals
 * into and out of (nbMarshalBodiesCUDA). */
void* nbref_state_bodytab(void* hv) { return ((RefHandle*) hv)->st.bodytab; }

/* The step counter, root size and incest flag the checkpoint header records
 * (nbPrepareWriteCheckpointHeader), as a GPU state reports them. */
void nbref_state_set_progress(void* hv, int step, double rsize, int treeIncest)
{
    RefHandle* h = (RefHandle*) hv;
    h->st.step = (unsigned int) step;
    h->st.tree.rsize = rsize;
    h->st.treeIncest = treeIncest;
}

void nbref_state_progress(void* hv, int* step, double* rsize, int* treeIncest)
{
    RefHandle* h = (RefHandle*) hv;
    *step = (int) h->st.step;
    *rsize = h->st.tree.rsize;
    *treeIncest = h->st.treeIncest;
}

/* Writes the handle's context and state to checkpointFile through the temporary tmpFile, as
 * nbWriteCheckpoint does at a checkpoint of the run loop.  Returns nonzero on failure. */
int nbref_write_checkpoint(void* hv, const char* checkpointFile, const char* tmpFile)
{
    RefHandle* h = (RefHandle*) hv;
    free(h->st.checkpointResolved);
    h->st.checkpointResolved = NULL;
    if (nbResolveCheckpoint(&h->st, checkpointFile)) return -1;
    return nbWriteCheckpointWithTmpFile(&h->ctx, &h->st, tmpFile);
}

/* A new handle with the context and state read back from checkpointFile (nbReadCheckpoint),
 * or NULL. */
void* nbref_read_checkpoint(const char* checkpointFile)
{
    static const NBodyState emptyState = EMPTY_NBODYSTATE;
    static const NBodyCtx emptyCtx = EMPTY_NBODYCTX;
    RefHandle* h = (RefHandle*) calloc(1, sizeof(RefHandle));
    h->ctx = emptyCtx;
    h->st = emptyState;
    if (nbResolveCheckpoint(&h->st, checkpointFile) || nbReadCheckpoint(&h->ctx, &h->st)) {
        free(h->st.checkpointResolved);
        free(h);
        return NULL;
    }
    h->ctx.quietErrors = TRUE;
    return h;
}

/* The reference's EMD (emdCalc, nbody/src/nbody_emd.c:1207-1268) between two signatures of
 * (weight, lambda, beta) triples, as nbMatchEMD calls it (no lower bound). */
double nbref_emd_calc(const double* sig1, unsigned int n1, const double* sig2, unsigned int n2)
{
    return emdCalc(sig1, sig2, n1, n2, NULL);
}

/* The reference's own counts histogram of the state (nbCreateHistogram, histogram 0): per bin
 * its lambda and beta centres, normalised count, raw count and useBin; returns the bin count
 * (cap: the arrays' length) and the histogram's totalNum. */
int nbref_histogram(void* hv, int cap, double* lambda, double* beta, double* variable,
                    unsigned int* rawCount, unsigned int* totalNum)
{
    RefHandle* h = (RefHandle*) hv;
    HistogramParams hp;
    NBodyLikelihoodMethod method;
    MainStruct* hist;
    NBodyHistogram* h0;
    int k, n;
    if (nbGetLikelihoodInfo(&h->nbf, &hp, &method)) return -1;
    hist = nbCreateHistogram(&h->ctx, &h->st, &hp);
    if (!hist) return -2;
    h0 = hist->histograms[0];
    n = (int) (h0->lambdaBins * h0->betaBins);
    for (k = 0; k < n && k < cap; ++k) {
        lambda[k] = h0->data[k].lambda;
        beta[k] = h0->data[k].beta;
        variable[k] = h0->data[k].variable;
        rawCount[k] = h0->data[k].rawCount;
    }
    *totalNum = h0->totalNum;
    for (k = 0; k < 8; ++k) free(hist->histograms[k]);
    free(hist);
    return n;
}

/* ---- math pins ---- */
double nbref_pow_rn(double x, double y) { return pow_rn(x, y); }
double nbref_log_rn(double x) { return log_rn(x); }
double nbref_atan_rn(double x) { return atan_rn(x); }

void nbref_ext_accel(const NBodyCudaPotential* p, const double* pos, double* acc, int n)
{
    NBodyCudaCtx c;
    NBodyCtx ctx;
    int i;
    memset(&c, 0, sizeof c);
    c.pot = *p;
    nbref_ctx_from_flat(&ctx, &c);
    for (i = 0; i < n; ++i) {
        mwvector v, a;
        SET_VECTOR(v, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        v.w = 0.0;
        a = nbExtAcceleration(&ctx.pot, v, 0.0);
        acc[3 * i] = X(a); acc[3 * i + 1] = Y(a); acc[3 * i + 2] = Z(a);
    }
}

/* A bounded sample of one reference step for the CPU baseline: nbMakeTree on the whole
 * system, then nbGravity + nbExtAcceleration (nbMapForceBody's per-body work,
 * nbody/src/nbody_grav.c:126-176) for `count` of its bodies on all OpenMP threads.
 * Returns the tree status; times in seconds. */
int nbref_sample_step(void* hv, const int* idx, int count, double* tTree, double* tWalk)
{
    RefHandle* h = (RefHandle*) hv;
    double t0, t1, t2;
    int k;
    NBodyStatus rc;
    t0 = omp_get_wtime();
    rc = nbMakeTree(&h->ctx, &h->st);
    t1 = omp_get_wtime();
    if (!nbStatusIsFatal(rc)) {
        const Body* bodies = h->st.bodytab;
        mwvector* accels = h->st.acctab;
        mwvector zero;
        SET_VECTOR(zero, 0.0, 0.0, 0.0);
        zero.w = 0.0;
#pragma omp parallel for schedule(dynamic, 64)
        for (k = 0; k < count; ++k) {
            const Body* b = &bodies[idx[k]];
            mwvector a = nbGravity(&h->ctx, &h->st, b);
            mwvector e = mw_addv(nbExtAcceleration(&h->ctx.pot, Pos(b), 0.0),
                                 plummerAccel(Pos(b), zero, 0.0, 1.0));
            mw_incaddv(a, e);
            accels[idx[k]] = a;
        }
    }
    t2 = omp_get_wtime();
    *tTree = t1 - t0;
    *tWalk = t2 - t1;
    return (int) rc;
}

int nbref_threads(void) { return omp_get_max_threads(); }
