/*
 * nbody_cuda.c -- the reference client's side of the B200 step.
 *
 * A maintainer adds this file to nbody/src/, compiles it into the reference's nbody library and
 * links the executable with -lnbody_b200 (include/nbody_b200.h); the dispatches that call it
 * are listed in nbody_cuda.h.  The device state hangs off the `void* nbb` slot that non-OpenCL
 * builds of NBodyState carry (nbody/include/nbody_types.h:425-429), so neither the state's
 * layout nor the checkpoint format changes; st->dirty marks host bodies that are stale while
 * the device steps (the contract of nbMarshalBodies, nbody/src/nbody_cl.c:2211-2269).
 */
#include <stdio.h>
#include <stdlib.h>

#include "nbody_priv.h"
#include "nbody_cuda.h"
#include "nbody_cuda_ctx.h"

int nbCudaRequestedDevice(void)
{
    const char* s = getenv("NBODY_CUDA_DEVICE");
    return (s && *s) ? atoi(s) : -1;
}

static NBodyStatus nbCudaStatus(NBodyCudaStatus rc, const char* what)
{
    if (nbStatusIsFatal((NBodyStatus) rc))
        mw_printf("%s failed (%d): %s\n", what, (int) rc, nbLastErrorCUDA());
    return (NBodyStatus) rc;
}

NBodyStatus nbCudaBeginRun(const NBodyCtx* ctx, NBodyState* st)
{
    const int device = nbCudaRequestedDevice();
    NBodyCudaState* cs = (NBodyCudaState*) st->nbb;
    NBodyStatus rc;

    if (device < 0)
        return NBODY_SUCCESS;
    if (!cs)
    {
        rc = nbCudaStatus(nbInitCUDA(&cs, device, (int) st->nbody), "nbInitCUDA");
        if (nbStatusIsFatal(rc))
            return rc;
        st->nbb = cs;
        mw_printf("Stepping on CUDA device %d (nbody_b200)\n", device);
    }
    rc = nbCudaStatus(nbMarshalBodiesCUDA(cs, st->bodytab, (int) st->nbody, TRUE, st->tree.rsize),
                      "nbMarshalBodiesCUDA");
    if (nbStatusIsFatal(rc))
        return rc;
    nbSetStepCUDA(cs, (int) st->step);
    nbSetTimeOriginCUDA(cs, st->previousForwardTime);
    if (ctx->LMC && st->shiftByLMC)
    {
        /* mwvector is {x, y, z, w}: the library takes 3 doubles per vector */
        const size_t n = st->nShiftLMC;
        double* shift = (double*) mwMalloc((n ? n : 1) * 3 * sizeof(double));
        double x[3], v[3];
        size_t k;
        for (k = 0; k < n; ++k)
        {
            shift[3 * k] = X(st->shiftByLMC[k]);
            shift[3 * k + 1] = Y(st->shiftByLMC[k]);
            shift[3 * k + 2] = Z(st->shiftByLMC[k]);
        }
        x[0] = X(st->LMCpos); x[1] = Y(st->LMCpos); x[2] = Z(st->LMCpos);
        v[0] = X(st->LMCvel); v[1] = Y(st->LMCvel); v[2] = Z(st->LMCvel);
        rc = nbCudaStatus(nbSetLMCCUDA(cs, x, v, shift, (int) n), "nbSetLMCCUDA");
        free(shift);
        if (nbStatusIsFatal(rc))
            return rc;
    }
    st->dirty = FALSE;
    return NBODY_SUCCESS;
}

NBodyStatus nbGravMapCUDAState(const NBodyCtx* ctx, NBodyState* st)
{
    NBodyCudaCtx c;
    nbCudaCtxFromNBodyCtx(&c, ctx);
    st->dirty = TRUE;
    return nbCudaStatus(nbGravMapCUDA(&c, (NBodyCudaState*) st->nbb), "nbGravMapCUDA");
}

NBodyStatus nbStepSystemCUDAState(const NBodyCtx* ctx, NBodyState* st)
{
    NBodyCudaCtx c;
    NBodyStatus rc;
    nbCudaCtxFromNBodyCtx(&c, ctx);
    rc = nbCudaStatus(nbStepSystemCUDA(&c, (NBodyCudaState*) st->nbb), "nbStepSystemCUDA");
    st->step++;
    st->dirty = TRUE;
    return rc;
}

NBodyStatus nbSyncBodiesFromCUDA(NBodyState* st)
{
    NBodyCudaState* cs = (NBodyCudaState*) st->nbb;
    NBodyCudaTreeInfo info;
    NBodyStatus rc;

    if (!cs || !st->dirty)
        return NBODY_SUCCESS;
    rc = nbCudaStatus(nbMarshalBodiesCUDA(cs, st->bodytab, (int) st->nbody, FALSE, 0.0),
                      "nbMarshalBodiesCUDA");
    if (nbStatusIsFatal(rc))
        return rc;
    if (nbTreeInfoCUDA(cs, &info) == NBODY_SUCCESS)
    {
        st->tree.rsize = info.rsize;
        st->treeIncest = st->treeIncest || info.treeIncest;
    }
    if (st->shiftByLMC)
    {
        double x[3], v[3];
        if (nbGetLMCCUDA(cs, x, v) == NBODY_SUCCESS)
        {
            SET_VECTOR(st->LMCpos, x[0], x[1], x[2]);
            SET_VECTOR(st->LMCvel, v[0], v[1], v[2]);
        }
    }
    st->dirty = FALSE;
    return NBODY_SUCCESS;
}

void nbDestroyStateCUDA(NBodyState* st)
{
    if (st->nbb)
    {
        nbDestroyCUDA((NBodyCudaState*) st->nbb);
        st->nbb = NULL;
    }
}
