/*
 * nbody_cuda.h -- the reference client's calls into the B200 step (nbody_cuda.c).
 *
 * The dispatches a maintainer adds beside the OpenCL ones (st->usesCL, nbody/src/nbody.c:184-189):
 *   nbRunSystemPlain (nbody/src/nbody_plain.c:366-461): nbCudaBeginRun before the first
 *     nbGravMap, nbGravMapCUDAState / nbStepSystemCUDAState instead of nbGravMap /
 *     nbStepSystemPlain when st->nbb is set, nbSyncBodiesFromCUDA before get_likelihood, before a
 *     checkpoint is written and before the final checkpoint;
 *   nbStepSystem (nbody/src/nbody.c:182-200): nbStepSystemCUDAState when st->nbb is set;
 *   destroyNBodyState (nbody/src/nbody_types.c:103): nbDestroyStateCUDA.
 */
#ifndef NBODY_CUDA_H_
#define NBODY_CUDA_H_

#include "nbody_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The GPU the run should step on: NBODY_CUDA_DEVICE=<index> in the environment; -1 (the CPU
 * step) when it is unset. */
int nbCudaRequestedDevice(void);

/* At the start of a run (and of every calibration run): with a GPU requested, creates the
 * device state in st->nbb once and marshals the host bodies in -- with the step counter, the
 * bar's time origin and the LMC of the state. */
NBodyStatus nbCudaBeginRun(const NBodyCtx* ctx, NBodyState* st);

NBodyStatus nbGravMapCUDAState(const NBodyCtx* ctx, NBodyState* st);
NBodyStatus nbStepSystemCUDAState(const NBodyCtx* ctx, NBodyState* st);

/* Host bodies (and root size, incest flag, LMC) from the device when they are stale
 * (st->dirty); a no-op for CPU states. */
NBodyStatus nbSyncBodiesFromCUDA(NBodyState* st);

void nbDestroyStateCUDA(NBodyState* st);

#ifdef __cplusplus
}
#endif

#endif /* NBODY_CUDA_H_ */
