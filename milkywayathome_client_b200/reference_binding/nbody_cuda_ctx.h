/*
 * nbody_cuda_ctx.h -- the reference's NBodyCtx as the flat NBodyCudaCtx of the B200 library.
 *
 * Reference-side code: it includes the reference's headers (NBodyCtx,
 * nbody/include/nbody_types.h:441-535) and the library's (include/nbody_b200.h).  Both the
 * binding (nbody_cuda.c, compiled into the reference executable) and the checker's shim into
 * the reference take the mapping from here, so the one mapping the tests exercise is the one
 * the binding ships.
 */
#ifndef NBODY_CUDA_CTX_H_
#define NBODY_CUDA_CTX_H_

#include <string.h>
#include "nbody_types.h"
#include "nbody_b200.h"

/* The fields the step reads: criterion, opening angle, softening, timestep, root size,
 * quadrupoles, incest handling, the external potential (sphere[0], disk, disk2, halo) and the
 * LMC settings.  The LMC's state and reflex accelerations are state, set with nbSetLMCCUDA. */
static inline void nbCudaCtxFromNBodyCtx(NBodyCudaCtx* c, const NBodyCtx* ctx)
{
    memset(c, 0, sizeof *c);
    c->eps2 = ctx->eps2;
    c->theta = ctx->theta;
    c->timestep = ctx->timestep;
    c->treeRSize = ctx->treeRSize;
    c->criterion = (int) ctx->criterion;
    c->useQuad = ctx->useQuad;
    c->allowIncest = ctx->allowIncest;
    c->potentialType = (int) ctx->potentialType;
    c->precision = NBCUDA_PRECISION_FP64;
    c->pot.sphere.type = ctx->pot.sphere[0].type;
    c->pot.sphere.mass = ctx->pot.sphere[0].mass;
    c->pot.sphere.scale = ctx->pot.sphere[0].scale;
    c->pot.disk.type = ctx->pot.disk.type;
    c->pot.disk.mass = ctx->pot.disk.mass;
    c->pot.disk.scaleLength = ctx->pot.disk.scaleLength;
    c->pot.disk.scaleHeight = ctx->pot.disk.scaleHeight;
    c->pot.disk.patternSpeed = ctx->pot.disk.patternSpeed;
    c->pot.disk.startAngle = ctx->pot.disk.startAngle;
    c->pot.disk2.type = ctx->pot.disk2.type;
    c->pot.disk2.mass = ctx->pot.disk2.mass;
    c->pot.disk2.scaleLength = ctx->pot.disk2.scaleLength;
    c->pot.disk2.scaleHeight = ctx->pot.disk2.scaleHeight;
    c->pot.disk2.patternSpeed = ctx->pot.disk2.patternSpeed;
    c->pot.disk2.startAngle = ctx->pot.disk2.startAngle;
    c->pot.halo.type = ctx->pot.halo.type;
    c->pot.halo.vhalo = ctx->pot.halo.vhalo;
    c->pot.halo.scaleLength = ctx->pot.halo.scaleLength;
    c->pot.halo.flattenZ = ctx->pot.halo.flattenZ;
    c->pot.halo.flattenY = ctx->pot.halo.flattenY;
    c->pot.halo.flattenX = ctx->pot.halo.flattenX;
    c->pot.halo.triaxAngle = ctx->pot.halo.triaxAngle;
    c->pot.halo.c1 = ctx->pot.halo.c1;
    c->pot.halo.c2 = ctx->pot.halo.c2;
    c->pot.halo.c3 = ctx->pot.halo.c3;
    c->pot.halo.mass = ctx->pot.halo.mass;
    c->pot.halo.gamma = ctx->pot.halo.gamma;
    c->pot.halo.lambda = ctx->pot.halo.lambda;
    c->pot.halo.rho0 = ctx->pot.halo.rho0;
    c->lmc = (int) ctx->LMC;
    c->lmcDynaFric = (int) ctx->LMCDynaFric;
    c->lmcMass = ctx->LMCmass;
    c->lmcScale = ctx->LMCscale;
    c->coulombLog = ctx->coulomb_log;
}

#endif /* NBODY_CUDA_CTX_H_ */
