/*
 * nbody_b200.h -- C ABI of the B200 (sm_100a) Barnes-Hut step for the
 * Milkyway@Home N-body client.
 *
 * The library (milkywayathome_client_b200/libnbody_b200.so) replaces the
 * reference client's CPU step (nbody/src/nbody_grav.c, nbody_tree.c,
 * nbody_plain.c, nbody_potential.c) and its OpenCL twin (nbody/src/nbody_cl.c +
 * nbody/kernels/nbody_kernels.cl) on one GPU.  Every entry point takes plain
 * pointers and sizes; nothing here depends on PyTorch or on the reference's
 * headers.  The context and state the reference keeps in NBodyCtx / NBodyState
 * (nbody/include/nbody_types.h:360-521) are passed as the flat NBodyCudaCtx
 * below plus an opaque NBodyCudaState handle that owns the device copy of the
 * bodies, the tree and the accelerations.
 *
 * Status values are the reference's NBodyStatus bit mask
 * (nbody/include/nbody_types.h:541-583) with the same numeric values, so
 * nbStatusIsFatal() from the reference applies unchanged.  CUDA runtime
 * failures are reported as NBODY_CUDA_ERROR, which occupies the reference's
 * NBODY_RESERVED_ERROR_1 bit.
 *
 * Threading: each NBodyCudaState is used from one host thread at a time, as the
 * reference's NBodyState is (nbody/src/nbody.c:182-212).
 */
#ifndef NBODY_B200_H
#define NBODY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status bits: values of NBodyStatus, nbody/include/nbody_types.h:541-583 ---- */
#define NBODY_SUCCESS               0
#define NBODY_ERROR                 (1 << 1)
#define NBODY_TREE_STRUCTURE_ERROR  (1 << 3)
#define NBODY_TREE_INCEST_FATAL     (1 << 4)
#define NBODY_CAPABILITY_ERROR      (1 << 8)
#define NBODY_UNIMPLEMENTED         (1 << 10)
#define NBODY_UNSUPPORTED           (1 << 11)
#define NBODY_USER_ERROR            (1 << 12)
#define NBODY_MAX_DEPTH_ERROR       (1 << 16)
#define NBODY_CELL_OVERFLOW_ERROR   (1 << 17)
#define NBODY_CUDA_ERROR            (1 << 20)   /* NBODY_RESERVED_ERROR_1 */
#define NBODY_TREE_INCEST_NONFATAL  (1 << 24)
#define NBODY_STATUS_WARNINGS_MASK  0xFF000000u  /* NBODY_STATUS_ALL_WARNINGS */

typedef int NBodyCudaStatus;

/* ---- enumerations: same values as the reference's enums ---- */
/* criterion_t, nbody/include/nbody_types.h:171-178 */
enum { NBCUDA_TREECODE = 0, NBCUDA_SW93 = 1, NBCUDA_BH86 = 2, NBCUDA_EXACT = 3 };
/* ExternalPotentialType, nbody/include/nbody_types.h:181-186 */
enum { NBCUDA_POTENTIAL_DEFAULT = 0, NBCUDA_POTENTIAL_NONE = 1, NBCUDA_POTENTIAL_CUSTOM_LUA = 2 };
/* spherical_t, disk_t, halo_t: nbody/include/nbody_potential_types.h:30-125 */
enum { NBCUDA_NO_SPHERICAL = 0, NBCUDA_HERNQUIST_SPHERICAL = 1, NBCUDA_PLUMMER_SPHERICAL = 2 };
enum { NBCUDA_NO_DISK = 0, NBCUDA_MIYAMOTO_NAGAI_DISK = 1, NBCUDA_FREEMAN_DISK = 2,
       NBCUDA_DOUBLE_EXPONENTIAL_DISK = 3, NBCUDA_SECH2_EXPONENTIAL_DISK = 4,
       NBCUDA_ORBITING_BAR = 5 };
enum { NBCUDA_NO_HALO = 0, NBCUDA_LOGARITHMIC_HALO = 1, NBCUDA_NFW_HALO = 2,
       NBCUDA_TRIAXIAL_HALO = 3, NBCUDA_CAUSTIC_HALO = 4, NBCUDA_ALLEN_SANTILLAN_HALO = 5,
       NBCUDA_WILKINSON_EVANS_HALO = 6, NBCUDA_NFW_MASS_HALO = 7, NBCUDA_PLUMMER_HALO = 8,
       NBCUDA_HERNQUIST_HALO = 9, NBCUDA_NINKOVIC_HALO = 10 };

/* Arithmetic of the force walk. */
enum {
    NBCUDA_PRECISION_FP64  = 0,  /* drop-in: FP64, no FMA contraction, the reference's
                                    per-body opening test and summation order */
    NBCUDA_PRECISION_MIXED = 1   /* FP32 walk in leaf-cell-relative coordinates with FP64
                                    accumulation; moments, potential and leapfrog stay FP64 */
};

/* Fields of Spherical / Disk / Halo (nbody/include/nbody_potential_types.h:40-156). */
typedef struct { int type; double mass, scale; } NBodyCudaSpherical;
typedef struct { int type; double mass, scaleLength, scaleHeight, patternSpeed, startAngle; } NBodyCudaDisk;
typedef struct {
    int type;
    double vhalo, scaleLength, flattenZ, flattenY, flattenX, triaxAngle;
    double c1, c2, c3, mass, gamma, lambda, rho0;
} NBodyCudaHalo;
/* Potential (nbody/include/nbody_potential_types.h:158-165) */
typedef struct {
    NBodyCudaSpherical sphere;
    NBodyCudaDisk disk, disk2;
    NBodyCudaHalo halo;
} NBodyCudaPotential;

/* The NBodyCtx fields the step reads (nbody/include/nbody_types.h:450-521). */
typedef struct {
    double eps2;          /* softening^2 */
    double theta;         /* opening angle */
    double timestep;      /* dt */
    double treeRSize;     /* initial root size (power of two) */
    int criterion;        /* NBCUDA_TREECODE .. NBCUDA_EXACT */
    int useQuad;          /* quadrupole moments in the walk */
    int allowIncest;      /* tree incest is a warning instead of fatal */
    int potentialType;    /* NBCUDA_POTENTIAL_* */
    int precision;        /* NBCUDA_PRECISION_* (no reference counterpart) */
    int reserved;
    NBodyCudaPotential pot;
    /* the LMC as a moving Plummer sphere (ctx->LMC, LMCDynaFric, LMCmass, LMCscale,
     * coulomb_log); its position, velocity and the Milky Way's reflex accelerations are state
     * (nbSetLMCCUDA) */
    int lmc;
    int lmcDynaFric;
    double lmcMass, lmcScale, coulombLog;
} NBodyCudaCtx;

/* Layout of the reference's Body (nbody/include/nbody_types.h:103-125): pos is an
 * mwvector {x,y,z,w} at offset 0, mass at 40, type (short) at 48, id at 52, vel
 * (mwvector) at 64; sizeof(Body) == 96. */
#define NBCUDA_BODY_STRIDE      96
#define NBCUDA_BODY_POS_OFFSET   0
#define NBCUDA_BODY_MASS_OFFSET 40
#define NBCUDA_BODY_TYPE_OFFSET 48
#define NBCUDA_BODY_ID_OFFSET   52
#define NBCUDA_BODY_VEL_OFFSET  64
/* mwvector stride of st->acctab (nbody/include/nbody_types.h:367) */
#define NBCUDA_VECTOR_STRIDE    32

/* Device-resident bodies, tree and accelerations: the CUDA counterpart of the
 * st->ci / st->kernels / st->nbb slots of NBodyState (nbody_types.h:421-430). */
typedef struct NBodyCudaState NBodyCudaState;

/* Tree summary after the last tree build (NBodyTree, nbody_types.h:188-196). */
typedef struct {
    double rsize;          /* t->rsize: root side length after expandBox */
    int nbody;             /* bodies in the state */
    int nTreeBodies;       /* bodies with nonzero mass (inserted in the tree) */
    int cellUsed;          /* t->cellUsed */
    int maxDepth;          /* t->maxDepth: deepest body level */
    int nNodes;            /* cells + tree bodies, in walk (preorder) order */
    int step;              /* st->step */
    int treeIncest;        /* st->treeIncest */
} NBodyCudaTreeInfo;

/* ---- lifecycle: replaces nbInitCL / nbInitNBodyStateCL (nbody/src/nbody_types.c:258-341)
 * and destroyNBodyState's CL branch.  Allocates device buffers for nbody bodies. */
NBodyCudaStatus nbInitCUDA(NBodyCudaState** st, int device, int nbody);
void nbDestroyCUDA(NBodyCudaState* st);

/* ---- marshalling: replaces nbMarshalBodies (nbody/src/nbody_cl.c:2211-2269).
 * toDevice != 0 copies pos/vel/mass of the host Body[] (NBCUDA_BODY_STRIDE bytes apart)
 * into the device state and resets st->step and the tree root size to treeRSize;
 * toDevice == 0 writes pos and vel back into the host Body[]. */
NBodyCudaStatus nbMarshalBodiesCUDA(NBodyCudaState* st, void* bodytab, int nbody,
                                    int toDevice, double treeRSize);
/* Plain SoA host arrays (pos/vel: x0,y0,z0,x1,...; mass: n) -- the same data as above. */
NBodyCudaStatus nbSetBodiesCUDA(NBodyCudaState* st, const double* pos, const double* vel,
                                const double* mass, int nbody, double treeRSize);
NBodyCudaStatus nbGetBodiesCUDA(NBodyCudaState* st, double* pos, double* vel);
/* st->acctab after the last force evaluation: 3 doubles per body in host memory. */
NBodyCudaStatus nbGetAccelsCUDA(NBodyCudaState* st, double* acc);
/* Device-pointer variants for callers that keep the bodies in their own device
 * memory (x,y,z interleaved as above; all pointers on the state's device). */
NBodyCudaStatus nbSetBodiesDeviceCUDA(NBodyCudaState* st, const double* dpos, const double* dvel,
                                      const double* dmass, int nbody, double treeRSize);
NBodyCudaStatus nbGetBodiesDeviceCUDA(NBodyCudaState* st, double* dpos, double* dvel, double* dacc);

/* ---- the hot path ----
 * nbGravMapCUDA replaces nbGravMap (nbody/src/nbody_grav.c:305-328): builds the tree
 * (nbMakeTree, nbody/src/nbody_tree.c:429-460) unless criterion is Exact, then fills
 * the accelerations with self-gravity + nbExtAcceleration (nbody/src/nbody_potential.c:627).
 * nbStepSystemCUDA replaces nbStepSystem / nbStepSystemPlain (nbody/src/nbody.c:182-200,
 * nbody/src/nbody_plain.c:329-364): one kick-drift-kick step, st->step += 1.
 * nbRunStepsCUDA runs nsteps such steps back to back on the device and returns the OR of
 * their statuses; it stops at the first fatal status as nbRunSystemPlain does
 * (nbody/src/nbody_plain.c:410-446). */
NBodyCudaStatus nbGravMapCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st);
NBodyCudaStatus nbStepSystemCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st);
NBodyCudaStatus nbRunStepsCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st, int nsteps);

/* ---- adjoint (no counterpart in the reference) ----
 * Vector-Jacobian product of the last force evaluation with its tree frozen: given the
 * adjoint abar of every body's acceleration (device pointer, 3 doubles per body in the
 * state's body order), writes xbar_j = sum_i abar_i . d a_i / d x_j (device, 3 per body) and,
 * if dMbar is not NULL, mbar_j = sum_i abar_i . d a_i / d m_j (device, 1 per body).  Every
 * opening decision of that evaluation is kept; the accelerations depend on the bodies
 * through the cells' centres of mass, masses and quadrupoles, which the adjoint follows.
 * Call it right after nbGravMapCUDA / nbStepSystemCUDA at the positions it was evaluated
 * at, with the same context (FP64 precision). */
NBodyCudaStatus nbGravVJPCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st, const double* dAbar,
                              double* dXbar, double* dMbar);

/* Saved force evaluations for the reverse pass (no reference counterpart).  nbSaveStateCUDA
 * copies, device to device, the bodies (positions, velocities, accelerations, masses) and the
 * tree of the last force evaluation into slot `slot` (0 <= slot < 65536; storage grows on
 * demand and is kept until nbReleaseStatesCUDA or nbDestroyCUDA); nbRestoreStateCUDA makes a
 * saved evaluation the current one again, tree included, so nbGravVJPCUDA and
 * nbStepAdjointCUDA can follow it without rebuilding the tree. */
NBodyCudaStatus nbSaveStateCUDA(NBodyCudaState* st, int slot);
NBodyCudaStatus nbRestoreStateCUDA(NBodyCudaState* st, int slot);
NBodyCudaStatus nbReleaseStatesCUDA(NBodyCudaState* st);

/* Reverse of one kick-drift-kick step (the step of nbStepSystemPlain,
 * nbody/src/nbody_plain.c:329-364), no reference counterpart.  The current evaluation must be
 * the step's end state x1, v1, a1 = A(x1) (right after nbStepSystemCUDA, or restored).  With
 * h = timestep / 2, dAk the accelerations a0 at the step's start (device, 3 per body) and the
 * adjoints, all device arrays of 3 doubles per body except dMbar (1 per body) and dDtbar (one
 * double):
 *     abar = h vbar + abarNext;  (gx, gm) = nbGravVJP(abar)
 *     xbar += gx;  mbar += gm  (skipped if dMbar is NULL)
 *     dtbar += vbar.a1/2 + xbar.vh + (vbar + dt xbar).a0/2   (vh = v1 - h a1; skipped if NULL)
 *     vbar += dt xbar;  abarNext = h vbar
 * so that after it (xbar, vbar) are the adjoints of the step's start state and abarNext the
 * adjoint of a0 for the reverse of the step before.  Everything stays on the device. */
NBodyCudaStatus nbStepAdjointCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st, const double* dAk,
                                  double* dXbar, double* dVbar, double* dMbar, double* dAbarNext,
                                  double* dDtbar);

/* Total energy of the current state by FP64 direct summation, O(N^2) (no reference
 * counterpart; the energy-drift check of the walk forms): energy[0] = kinetic sum m v^2 / 2,
 * energy[1] = self-gravity -sum_{i<j} m_i m_j / sqrt(r^2 + eps2), energy[2] = sum m Phi_ext
 * for the context's potential (0 with EXTERNAL_POTENTIAL_NONE).  Host array of 3 doubles. */
NBodyCudaStatus nbEnergyCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st, double* energy);

/* ---- Lambda-Beta histograms and the likelihood on the GPU ----
 * nbCreateHistogram (nbody/src/nbody_histogram.c:671-1139) and nbSystemLikelihood
 * (nbody/src/nbody_likelihood.c:155-324) from the device-resident bodies, without copying them
 * to the host: the normalised counts; the beta and line-of-sight velocity dispersions and, when
 * a comparison needs them, the averages of the line-of-sight velocity, beta, distance and the
 * proper motions, each with IterMax passes of sigma-clipping outlier rejection (nbCalcDisp,
 * nbRemoveOutliers, nbody/src/nbody_mass.c:190-316); the EMD and cost components and the
 * comparisons (nbLikelihood, nbody_mass.c:395-469) the flags enable.  Bodies of type +1 are
 * light (they count towards totalSimulated and set massPerParticle), bodies of type < 0 are
 * ignored.  The likelihood supports one beta bin and the default EMD range (the whole
 * histogram), as the reference's runs use.  The dispersions' sums are formed in a fixed order
 * on the device (deterministic); they may differ from the reference's body-order sums by
 * rounding. */
#define NBODY_CUDA_HIST_COMPONENTS 7   /* histograms 1..7 of the reference's MainStruct */
#define NBODY_CUDA_LIKELIHOOD_TERMS 11
typedef struct {
    double phi, theta, psi;            /* Euler angles of the stream frame, degrees */
    double lambdaStart, lambdaEnd;
    double betaStart, betaEnd;
    int lambdaBins, betaBins;
    double sunGCDist;
    /* the comparisons nbSystemLikelihood adds (NBodyCtx fields of the reference; its defaults:
     * useBetaDisp 1, the others 0) */
    int useBetaDisp, useVelDisp, useBetaComp, useVlos, useDist, usePropMot;
    int iterMax;                       /* outlier-rejection passes (IterMax; default 6) */
    int reserved;
    double betaSigma, velSigma, distSigma, pmSigma;          /* cut-offs (default 2.5) */
    double betaCorrect, velCorrect, distCorrect, pmCorrect;  /* dispersion corrections (1.111) */
    double sunVelx, sunVely, sunVelz;  /* km/s (default 10.3, 229.2, 6.9) */
    double NGPdec, NGPra, lNCP;        /* radians (default d2r(27.4), d2r(192), d2r(123)) */
} NBodyCudaHistogramParams;
typedef struct {                       /* a data histogram as nbReadHistogram reads it */
    int nBins;                         /* lambdaBins * betaBins */
    unsigned int totalNum;             /* "n" */
    double massPerParticle;
    const int* useBin;                 /* host arrays of nBins entries */
    const double* lambda;              /* bin centres */
    const double* variable;            /* normalised counts */
    const double* err;                 /* count errors */
    int betaDispBins;                  /* "betaDispBins =" (0 when absent) */
    int reserved;
    /* histograms 1..7: beta dispersion, line-of-sight velocity dispersion, line-of-sight
     * velocity, beta, distance, dec and RA proper motion: values and errors of nBins entries
     * each, NULL where the file holds none */
    const double* compVariable[NBODY_CUDA_HIST_COMPONENTS];
    const double* compErr[NBODY_CUDA_HIST_COMPONENTS];
    /* the lambda ranges of the EMD ("EMDRange = {start, end, ...}", the values as strtof
     * parses them, params.EMDRange of nbody/src/nbody_histogram.c:1547-1561): nRange values,
     * pairs of inclusive bounds; nRange 0: the range nbReadHistogram gives a file without that
     * line (nbody/src/nbody_histogram.c:1563-1567) -- every bin with one beta bin; with more
     * beta bins the lambdas of bins 0 and lambdaBins - 1 in lambda-major order bound it, i.e.
     * the first 1/betaBins of the lambda axis, as the reference compares.  The
     * EMD is taken per range over its used bins, each renormalised, weighted by the range's
     * share of the data counts (nbMatchEMD, nbody/src/nbody_emd.c:1332-1402). */
    int nRange;
    int reserved2;
    const double* emdRange;
    /* bin centres in beta (nBins entries; needed when betaBins > 1, may be NULL otherwise):
     * with more than one beta bin each range's EMD is the reference's transportation-simplex
     * emdCalc over (lambda, beta) with the L2 ground distance */
    const double* beta;
} NBodyCudaDataHistogram;
/* ---- nbRunSystem: the run loop with the best-likelihood scan and the bar's calibration ----
 * The forward evolution of nbody/src/nbody.c:420-520 around nbRunSystemPlain
 * (nbody/src/nbody_plain.c:365-470) and get_likelihood (:100-237), on the device:
 *   - the bar's time origin starts at timeEvolve / (2 - s') with useBestLike (s' =
 *     2 BestLikeStart / (BestLikeStart + 1), the window start before the Lua's rescaling),
 *     else at timeEvolve;
 *   - each run: nbGravMap, then steps up to nStep; after a step with step / nStep >=
 *     BestLikeStart (with useBestLike) the likelihood against data is evaluated on the device
 *     and kept when its magnitude beats the best so far (NaN or beyond the worst case counts
 *     as the worst case, 0 as the best case), with its time step / nStep * timeEvolve;
 *   - with an orbiting bar, calibrationRuns more runs from the same initial state, each with
 *     the previous run's best time as the bar's time origin;
 *   - the result is the final state's likelihood, or the best one when the final one is worse
 *     (nbody.c:320-345).
 * The state must start at the run's first step (as nbody.c's initial state); it ends at
 * nStep.  With data NULL no likelihood is evaluated (the runs are the bare loop).  One host
 * synchronisation per step (the tree-build status), none for the scan. */
typedef struct {
    int nStep;                  /* ctx->nStep */
    int useBestLike;            /* ctx->useBestLike */
    double timeEvolve;          /* ctx->timeEvolve */
    double bestLikeStart;       /* ctx->BestLikeStart (as the context holds it) */
    int calibrationRuns;        /* ctx->calibrationRuns (used with an orbiting bar only) */
    int keepBestBodies;         /* keep the bodies of the best likelihood (nbGetBestBodiesCUDA) */
} NBodyCudaRunParams;
typedef struct {
    double result[NBODY_CUDA_LIKELIHOOD_TERMS];  /* the likelihood the reference reports */
    double final[NBODY_CUDA_LIKELIHOOD_TERMS];   /* the final state's (likelihood clamped) */
    double best[NBODY_CUDA_LIKELIHOOD_TERMS];    /* st->bestLikelihood* of the last run */
    double bestTime;                             /* st->bestLikelihood_time (0: none) */
    double previousForwardTime;                  /* the bar's time origin of the last run */
    int bestStep, bestCount;                     /* step of the best, improvements counted */
    int runs;                                    /* forward runs made */
    int reserved;
} NBodyCudaRunResult;
NBodyCudaStatus nbRunSystemCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st,
                                const NBodyCudaRunParams* rp, const NBodyCudaHistogramParams* hp,
                                const NBodyCudaDataHistogram* data, NBodyCudaRunResult* res);
/* the bodies at the best likelihood of the last nbRunSystemCUDA with keepBestBodies (the
 * reference's bestLikelihoodBodyTab, nbody/src/nbody_plain.c:226-231), host arrays of 3n */
NBodyCudaStatus nbGetBestBodiesCUDA(NBodyCudaState* st, double* pos, double* vel);

/* ---- the LMC (contexts with lmc = 1) ----
 * nbStepSystemPlain's LMC (nbody/src/nbody_plain.c:268-360): every body feels the LMC as a
 * Plummer sphere (plummerAccel, nbody/src/nbody_potential.c:145-152) at the LMC's current
 * position, and both half kicks of step k add the Milky Way's reflex acceleration
 * shift[k] / shift[k + 1] to every body; the LMC itself drifts with its velocity and is kicked
 * by the external potential plus Chandrasekhar dynamical friction (dynamicalFriction_LMC,
 * nbody/src/nbody_friction.c:85-132, with nbExtDensity, nbody/src/nbody_density.c:250-369) and
 * the same reflex accelerations, all on the device.  pos3/vel3 (st->LMCpos, st->LMCvel) and
 * shift (st->shiftByLMC, nShift >= the run's nStep + 1 vectors) are what the reference's
 * set-up (reverseOrbit_LMC, nbody/src/nbody_orbit_integrator.c:92-285) leaves. */
NBodyCudaStatus nbSetLMCCUDA(NBodyCudaState* st, const double* pos3, const double* vel3,
                             const double* shift, int nShift);
NBodyCudaStatus nbGetLMCCUDA(NBodyCudaState* st, double* pos3, double* vel3);

/* The bar's time origin, the reference's st->previousForwardTime (nbody/src/nbody.c:440-442):
 * the orbiting bar is evaluated at step * timestep - previousForwardTime (0 by default).
 * For a batch, set it on the batch's state through nbBatchSetTimeOriginCUDA. */
NBodyCudaStatus nbSetTimeOriginCUDA(NBodyCudaState* st, double previousForwardTime);

/* The step counter of a state resumed from a checkpoint: nbThawState restores st->step from
 * the checkpoint header (nbody/src/nbody_checkpoint.c:123-130), and nbMarshalBodiesCUDA's
 * copy-in resets it to 0, so a resumed run sets it after marshalling the bodies in (the
 * orbiting bar's time and the LMC's reflex accelerations are read at it). */
NBodyCudaStatus nbSetStepCUDA(NBodyCudaState* st, int step);

/* Whether nbStepSystemCUDA / nbRunStepsCUDA replay a step as one captured CUDA graph (enable
 * != 0, the default): a step's ~60 kernels are captured once per context, node capacity and
 * tuning and then launched as one graph, which removes the launch gaps that dominate small
 * systems (tens of thousands of bodies); the kernels, their order and so the results are the
 * same either way.  Steps with an orbiting bar or an LMC (whose per-step values are kernel
 * arguments) and counted evaluations are always launched directly. */
NBodyCudaStatus nbSetStepGraphCUDA(NBodyCudaState* st, int enable);

/* The FP64 force walk's form: 0 walks the union of a warp's 32 tree paths node by node (the
 * lanes whose path holds the node doing it, one broadcast load per node); 1 walks every body's
 * path in its own lane (a lane idles only once its walk is over; per-lane loads); 2 is the
 * per-lane walk that loads the next node's record as soon as the opening test has chosen it,
 * overlapping that load with the current node's arithmetic (more registers: faster for small
 * systems, slower at a million bodies).  -1 (the default) cycles twice through the three
 * forms over a state's first six uncounted FP64 tree evaluations, times the second round (the
 * first launch of each kernel also loads it) and keeps the fastest.  Every form gives every
 * body exactly its CPU walk -- same nodes, same order, same sums: the accelerations are the
 * same bit for bit.  A batch walks the union unless its form is set (nbBatchSetWalkFormCUDA);
 * the force adjoint always walks the union (it reduces each node's adjoints over the warp).
 * nbGetWalkFormCUDA reports the form in use (-1 while undecided). */
NBodyCudaStatus nbSetWalkFormCUDA(NBodyCudaState* st, int form);
NBodyCudaStatus nbGetWalkFormCUDA(NBodyCudaState* st, int* form);

/* Mixed-precision walk tuning of a single state (as nbBatchSetTuningCUDA): bodies per walk
 * group (1..64), interaction-list entries per warp (32, 64, 128), walk blocks per SM (0: max). */
NBodyCudaStatus nbSetMixedTuningCUDA(NBodyCudaState* st, int groupMax, int listCap, int blocksPerSM);
/* Interaction sets of the mixed walk.  exactSet = 1 (the default): a group of bodies walks the
 * tree together, but every body takes exactly the cells and bodies its own opening test takes
 * (the FP64 walk's set), so the mixed form's error is the FP64 walk's up to FP32 rounding.
 * exactSet = 0: every body of a group takes the group's set (cells accepted for the whole group
 * box) -- faster, never coarser per cell, but the shell of accepted cells is no longer
 * symmetric about each body and the truncation errors cancel less: a heavier error tail. */
NBodyCudaStatus nbSetMixedModeCUDA(NBodyCudaState* st, int exactSet);

/* host array of nbody types (+1 light, -1 dark) */
NBodyCudaStatus nbSetTypesCUDA(NBodyCudaState* st, const int* types);
/* host outputs, any may be NULL: counts[nBins], totals[2] = {in range, light bodies},
 * massPerParticle[1], comps[NBODY_CUDA_HIST_COMPONENTS][2][nBins] = histograms 1..7 as
 * {values, errors} (1 and 2 always; 3..7 when useVlos, useBetaComp, useDist or usePropMot is
 * set, as the reference builds them; zeros otherwise) */
NBodyCudaStatus nbHistogramCUDA(NBodyCudaState* st, const NBodyCudaHistogramParams* hp,
                                unsigned int* counts, unsigned int* totals,
                                double* massPerParticle, double* comps);
/* out[NBODY_CUDA_LIKELIHOOD_TERMS]: the reference's likelihood array (likelihood, EMD
 * component, cost component, beta dispersion, velocity dispersion, beta average,
 * line-of-sight velocity, distance, dec and RA proper motion; NaN where not compared; all NaN
 * when a comparison's data histogram is missing), then the EMD itself.  Positive; lower is
 * better. */
NBodyCudaStatus nbLikelihoodCUDA(NBodyCudaState* st, const NBodyCudaHistogramParams* hp,
                                 const NBodyCudaDataHistogram* data, double* out);

/* ---- two-component Plummer dwarf initial conditions on the GPU ----
 * The sampler of nbGenerateMixedDwarfCore (nbody/src/nbody_mixeddwarf.c:765-1026) for
 * Dwarf.plummer components: rejection sampling of radii from r^2 rho(r) and of speeds from the
 * Eddington distribution function (evaluated numerically as the reference does), isotropic
 * directions, each component recentred on its centre of mass and velocity and shifted to
 * position/velocity.  One thread per body with its own counter-based random stream: the
 * samples follow the reference's distributions, not its dSFMT stream.  Baryons (type +1) are
 * the first nbodyBaryon bodies, dark matter (type -1) the rest. */
typedef struct {
    int nbody, nbodyBaryon;
    double massLight, scaleLight;      /* comp1 */
    double massDark, scaleDark;        /* comp2 */
    double position[3], velocity[3];   /* the dwarf's centre on its orbit */
    unsigned long long seed;
} NBodyCudaPlummerDwarf;
/* fills the state's bodies and types (nbody must match the state) and resets the run like
 * nbSetBodiesCUDA with treeRSize */
NBodyCudaStatus nbGenerateDwarfCUDA(NBodyCudaState* st, const NBodyCudaPlummerDwarf* dwarf,
                                    double treeRSize);

/* Dwarf component profiles (dwarf_t, nbody/include/nbody_potential_types.h:136-152).  Einasto
 * (3) is not sampled: the reference's get_density/get_potential have no case for it. */
#define NBCUDA_DWARF_PLUMMER 0
#define NBCUDA_DWARF_NFW 1
#define NBCUDA_DWARF_GEN_HERNQUIST 2
#define NBCUDA_DWARF_CORED 4

/* One component: Dwarf.plummer / nfw / general_hernquist {mass, scaleLength} or Dwarf.cored
 * {mass, scaleLength, r1, rc} (nbody/src/nbody_lua_types/nbody_lua_dwarf.c:57-125).  For NFW
 * and cored components mass is M200; like the reference the sampler replaces it by the mass
 * inside its sampling bound 5 r200 (get_extra_nfw_mass, nbody/src/nbody_mixeddwarf.c:728-762). */
typedef struct {
    int type, reserved;
    double mass, scaleLength;
    double r1, rc;                     /* cored only */
} NBodyCudaDwarfComponent;

/* A two-component dwarf of any of those profiles (predefinedModels.mixeddwarf with comp1 =
 * light, comp2 = dark; nbGenerateMixedDwarfCore, nbody/src/nbody_mixeddwarf.c:765-1026),
 * sampled as NBodyCudaPlummerDwarf is. */
typedef struct {
    int nbody, nbodyBaryon;
    NBodyCudaDwarfComponent light, dark;
    double position[3], velocity[3];
    unsigned long long seed;
} NBodyCudaMixedDwarf;
NBodyCudaStatus nbGenerateMixedDwarfCUDA(NBodyCudaState* st, const NBodyCudaMixedDwarf* dwarf,
                                         double treeRSize);
/* the particle masses the sampler gives the two components: out[0] light, out[1] dark */
NBodyCudaStatus nbMixedDwarfParticleMassesCUDA(const NBodyCudaMixedDwarf* dwarf, double* out);
/* every body's mass (nbody doubles) */
NBodyCudaStatus nbGetBodyMassesCUDA(NBodyCudaState* st, double* mass);

/* ---- batched dwarfs (no reference counterpart: the reference runs one dwarf per process) ----
 * Many independent dwarfs stepped together.  Each dwarf is the reference's simulation (its own
 * root at the origin, root size, octree, softening and time step) and gets the same
 * accelerations, bit for bit, as a single-dwarf state (FP64 precision); every phase of the step
 * (bounding boxes, keys, sort, tree, moments, walk with the kick) is one launch over all
 * dwarfs, and nbBatchRunStepsCUDA can replay the whole step as one captured CUDA graph.
 * Bodies are concatenated dwarf after dwarf (dwarf 0's nbody bodies first) in every array;
 * all of them must be massive.  The context supplies the criterion (a tree criterion), theta,
 * quadrupoles, incest policy, potential and precision; eps2, timestep and treeRSize come from
 * each dwarf's NBodyCudaDwarf. */
typedef struct NBodyCudaBatch NBodyCudaBatch;
typedef struct {
    int nbody;           /* bodies of this dwarf, >= 2 */
    double eps2;         /* softening length squared */
    double timestep;     /* leapfrog step */
    double treeRSize;    /* initial root size, a power of two */
} NBodyCudaDwarf;
NBodyCudaStatus nbBatchCreateCUDA(NBodyCudaBatch** batch, int device, const NBodyCudaDwarf* dwarfs,
                                  int ndwarfs);
NBodyCudaStatus nbBatchDestroyCUDA(NBodyCudaBatch* batch);
/* host arrays: pos, vel 3 doubles per body, mass 1 (resets root sizes and statuses) */
NBodyCudaStatus nbBatchSetBodiesCUDA(NBodyCudaBatch* batch, const double* pos, const double* vel,
                                     const double* mass);
NBodyCudaStatus nbBatchSetBodiesDeviceCUDA(NBodyCudaBatch* batch, const double* dpos,
                                           const double* dvel, const double* dmass);
/* host arrays; any may be NULL */
NBodyCudaStatus nbBatchGetBodiesCUDA(NBodyCudaBatch* batch, double* pos, double* vel, double* acc);
NBodyCudaStatus nbBatchGetBodiesDeviceCUDA(NBodyCudaBatch* batch, double* dpos, double* dvel,
                                           double* dacc);
/* nbGravMap of every dwarf */
NBodyCudaStatus nbBatchGravMapCUDA(const NBodyCudaCtx* ctx, NBodyCudaBatch* batch);
/* nsteps kick-drift-kick steps of every dwarf (an initial nbGravMap if none was made);
 * useGraph != 0 replays one captured graph per step.  Stops at the first fatal status. */
NBodyCudaStatus nbBatchRunStepsCUDA(const NBodyCudaCtx* ctx, NBodyCudaBatch* batch, int nsteps,
                                    int useGraph);
/* per dwarf (arrays of ndwarfs, any may be NULL): sticky status bits of its tree builds, its
 * current root size, its root's node index and node count */
NBodyCudaStatus nbBatchDwarfInfoCUDA(NBodyCudaBatch* batch, int* status, double* rsize,
                                     int* rootNode, int* nodes);
/* mixed-precision walk tuning: bodies per walk group (1..64; above 32 each lane walks for two
 * bodies), interaction-list entries per warp (32, 64 or 128), resident walk blocks per SM
 * (0: as many as fit) */
NBodyCudaStatus nbBatchSetTuningCUDA(NBodyCudaBatch* batch, int groupMax, int listCap,
                                     int blocksPerSM);
/* as nbSetMixedModeCUDA, for every dwarf of the batch */
NBodyCudaStatus nbBatchSetMixedModeCUDA(NBodyCudaBatch* batch, int exactSet);
/* The FP64 walk's form for every dwarf of the batch, as nbSetWalkFormCUDA but without the
 * automatic choice: 0 (the default) the warp union, 1 per lane, 2 per lane with the next
 * record loaded early (a warp may span two dwarfs; each lane walks only its own dwarf's tree). */
NBodyCudaStatus nbBatchSetWalkFormCUDA(NBodyCudaBatch* batch, int form);
NBodyCudaStatus nbBatchGetTuningCUDA(NBodyCudaBatch* batch, int* groupMax, int* listCap,
                                     int* blocksPerSM);
/* autotuner of the mixed walk on the batch's current state: times every candidate tuning
 * (groupMax 24/32/48/64 x listCap 32/64/128 x blocksPerSM 0/3) with force evaluations that do not
 * move the bodies, keeps the fastest, re-evaluates the accelerations with it and returns it
 * (and its walk time in ms).  With FP64 precision nothing is tuned. */
NBodyCudaStatus nbBatchAutotuneCUDA(const NBodyCudaCtx* ctx, NBodyCudaBatch* batch, int* groupMax,
                                    int* listCap, int* blocksPerSM, double* walkMs);
/* histograms and likelihoods of every dwarf: types as nbSetTypesCUDA (all dwarfs' bodies),
 * counts[ndwarfs * nBins], totals[2 * ndwarfs], massPerParticle[ndwarfs], out[4 * ndwarfs] */
NBodyCudaStatus nbBatchSetTypesCUDA(NBodyCudaBatch* batch, const int* types);
NBodyCudaStatus nbBatchSetTimeOriginCUDA(NBodyCudaBatch* batch, double previousForwardTime);
/* as nbHistogramCUDA / nbLikelihoodCUDA, per dwarf: counts[ndwarfs][nBins], totals[ndwarfs][2],
 * massPerParticle[ndwarfs], comps[ndwarfs][7][2][nBins], out[ndwarfs][11] */
NBodyCudaStatus nbBatchHistogramCUDA(NBodyCudaBatch* batch, const NBodyCudaHistogramParams* hp,
                                     unsigned int* counts, unsigned int* totals,
                                     double* massPerParticle, double* comps);
NBodyCudaStatus nbBatchLikelihoodCUDA(NBodyCudaBatch* batch, const NBodyCudaHistogramParams* hp,
                                      const NBodyCudaDataHistogram* data, double* out);
/* initial conditions of every dwarf of the batch in one launch per phase (one
 * NBodyCudaPlummerDwarf per dwarf, nbody matching the batch); resets root sizes and statuses */
NBodyCudaStatus nbBatchGenerateDwarfsCUDA(NBodyCudaBatch* batch, const NBodyCudaPlummerDwarf* dwarfs);
NBodyCudaStatus nbBatchGenerateMixedDwarfsCUDA(NBodyCudaBatch* batch,
                                               const NBodyCudaMixedDwarf* dwarfs);
/* nbRunSystemCUDA for every dwarf at once (rp shared: nStep, the best-likelihood window from
 * bestLikeStart, timeEvolve): steps through the batch's step (captured graphs when useGraph),
 * each step of the window one histogram pass, likelihood and best-record update for all
 * dwarfs; res[ndwarfs] as nbRunSystemCUDA's per dwarf.  Types must be set
 * (nbBatchSetTypesCUDA).  With an orbiting bar, the calibrationRuns restart the whole batch
 * from its initial state, each dwarf with its own previous best time as its bar's origin. */
NBodyCudaStatus nbBatchRunSystemCUDA(const NBodyCudaCtx* ctx, NBodyCudaBatch* batch,
                                     const NBodyCudaRunParams* rp,
                                     const NBodyCudaHistogramParams* hp,
                                     const NBodyCudaDataHistogram* data, int useGraph,
                                     NBodyCudaRunResult* res);
/* every dwarf's bodies at its best likelihood (keepBestBodies; valid for dwarfs with
 * bestCount > 0), all bodies of the batch in order */
NBodyCudaStatus nbBatchGetBestBodiesCUDA(NBodyCudaBatch* batch, double* pos, double* vel);
/* LMC runs of a batch (a context with lmc set): every dwarf's LMC as nbSetLMCCUDA takes one --
 * pos3/vel3 3 doubles per dwarf, shift nShift reflex accelerations of 3 doubles per dwarf,
 * dwarf after dwarf.  Each dwarf's LMC moves with its own time step and bar time; set the
 * LMCs after the bodies (nbBatchSetBodiesCUDA and the generators restore the LMC states given
 * here). */
NBodyCudaStatus nbBatchSetLMCCUDA(NBodyCudaBatch* batch, const double* pos3, const double* vel3,
                                  const double* shift, int nShift);
NBodyCudaStatus nbBatchGetLMCCUDA(NBodyCudaBatch* batch, double* pos3, double* vel3);
/* mean device time of the steps of the last nbBatchRunStepsCUDA call */
NBodyCudaStatus nbBatchLastStepTimeCUDA(NBodyCudaBatch* batch, double* stepMs);

/* ---- tree introspection (parity checks of nbMakeTree) ---- */
NBodyCudaStatus nbMakeTreeCUDA(const NBodyCudaCtx* ctx, NBodyCudaState* st);
NBodyCudaStatus nbTreeInfoCUDA(NBodyCudaState* st, NBodyCudaTreeInfo* info);
/* Nodes in walk (threadTree preorder) order, nNodes entries each: pos = CoM for cells,
 * body position for bodies (3 doubles); mass; rcrit2 (0 for bodies); quad (6 doubles:
 * xx,xy,xz,yy,yz,zz; 0 for bodies); next (index of Next(), nNodes for NULL); body (index
 * of the body in the state for body nodes, -1 for cells); depth (cell level, root = 0;
 * for bodies the level of their parent cell + 1).  Any pointer may be NULL. */
NBodyCudaStatus nbGetTreeCUDA(NBodyCudaState* st, double* pos, double* mass, double* rcrit2,
                              double* quad, int32_t* next, int32_t* body, int32_t* depth);

/* ---- external potential alone: nbExtAcceleration (nbody/src/nbody_potential.c:627-762)
 * at n host positions (3 doubles each) -> n host accelerations. */
NBodyCudaStatus nbExtAccelerationCUDA(const NBodyCudaPotential* pot, const double* pos,
                                      double* acc, int n, int device);

/* nbExtAcceleration at n host positions with no device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc/cudaFree -- cudaFree waits for the
 * whole device, cudaMalloc can fail under a fixed memory budget -- such as an orbit
 * integrator evaluating a few points per step, or a process sharing the GPU with a running
 * simulation.  Positions and results go through one fixed static device array of
 * NB_NOALLOC_MAX_POINTS (65536) points (3 MiB, held by every device that loads the library
 * until exit); larger n is rejected with NBODY_USER_ERROR.  The first call on a device looks
 * up the array's address (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  The address is kept for the life of the process: a device reset
 * (cudaDeviceReset) unloads the array with the module, and calls after a reset of that
 * device are not supported.  All calls share the array: calls that overlap on the GPU race.
 * Same results as nbExtAccelerationCUDA. */
NBodyCudaStatus nbExtAccelerationNoAllocCUDA(const NBodyCudaPotential* pot, const double* pos,
                                             double* acc, int n, int device);

/* emdCalc (nbody/src/nbody_emd.c:1207-1268) on the GPU: the earth mover's distance between two
 * signatures of (weight, lambda, beta) triples (n1 and n2 of them, host arrays) with the L2
 * ground distance, by the reference's transportation simplex (the same decisions, so the same
 * value bit for bit); NaN where the reference returns EMD_INVALID.  The likelihood runs the
 * same solver on the device for two-dimensional histograms (betaBins > 1). */
NBodyCudaStatus nbEmdCalcCUDA(const double* sig1, int n1, const double* sig2, int n2,
                              double* emd, int device);

/* Number of this library's kernel launches issued since load (a launch counter for
 * benchmarks). */
uint64_t nbKernelLaunchesCUDA(void);
/* Milliseconds of device time of the force-walk kernels of the last nbGravMapCUDA /
 * nbStepSystemCUDA / nbRunStepsCUDA call (CUDA events on the launch stream), and the
 * number of walk launches they cover. */
NBodyCudaStatus nbLastWalkTimeCUDA(NBodyCudaState* st, double* ms, int* launches);
/* Milliseconds of device time of the whole last nbGravMapCUDA / nbStepSystemCUDA call (tree
 * build, walk and leapfrog; CUDA events on the state's stream); for nbRunStepsCUDA the sum
 * over its steps. */
NBodyCudaStatus nbLastStepTimeCUDA(NBodyCudaState* st, double* ms);
/* FP64 direct-summation self-gravity (the arithmetic of nbGravity_Exact,
 * nbody/src/nbody_grav.c:205-227) at `count` target bodies of the state, over all its bodies:
 * the accuracy oracle for the tree forms.  targets: host indices; acc: 3 doubles per target. */
NBodyCudaStatus nbDirectSampleCUDA(NBodyCudaState* st, double eps2, const int32_t* targets,
                                   int count, double* acc);
/* Measured FMA throughput of the device in TFLOP/s (fp64 != 0: DFMA, else FFMA; 2 flops per
 * FMA): the pipe roofline the walk kernels are reported against. */
NBodyCudaStatus nbPeakFmaCUDA(int device, int fp64, double* tflops);
/* Interaction counts of the last force evaluation (counting enabled): body-body and
 * body-cell interactions and node visits summed over all bodies (the algorithmic work of
 * the walk), and walk iterations summed over warps (32 x nWarpSteps / nVisit is the
 * fraction of lanes busy in a visit). */
NBodyCudaStatus nbInteractionCountsCUDA(NBodyCudaState* st, unsigned long long* nBodyBody,
                                        unsigned long long* nBodyCell,
                                        unsigned long long* nVisit,
                                        unsigned long long* nWarpSteps);
/* Enables (1) / disables (0) counting interactions in the walk (off by default). */
NBodyCudaStatus nbSetCountingCUDA(NBodyCudaState* st, int enable);

const char* nbLastErrorCUDA(void);

#ifdef __cplusplus
}
#endif
#endif /* NBODY_B200_H */
