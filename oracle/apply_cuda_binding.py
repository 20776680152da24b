"""Writes the reference's three step files with the B200 binding's dispatches added.

Test infrastructure: a recipe of oracle/ref.mk (target `cuda`).  It reads nbody.c,
nbody_plain.c and nbody_types.c from the reference checkout and writes copies into
oracle/_ref/cuda_src/ (git-ignored build output) with the one-line dispatches a maintainer adds
beside the OpenCL ones to call milkywayathome_client_b200/reference_binding/nbody_cuda.c (the
list is in nbody_cuda.h).  Every edit is anchored on text that must occur exactly once; a
reference whose text moved fails loudly instead of building a half-patched executable.

    python3 oracle/apply_cuda_binding.py <reference checkout> <output directory>
"""
import os
import sys

INCLUDE = '#include "nbody_cuda.h"\n'

EDITS = {
    "nbody_plain.c": [
        # the device state and the first force evaluation of a run (nbody_plain.c:388)
        ("    rc |= nbGravMap(ctx, st); /* Calculate accelerations for 1st step this episode */\n",
         "    rc |= nbCudaBeginRun(ctx, st);\n"
         "    if (nbStatusIsFatal(rc))\n"
         "        return rc;\n"
         "    rc |= st->nbb ? nbGravMapCUDAState(ctx, st) : nbGravMap(ctx, st); "
         "/* Calculate accelerations for 1st step this episode */\n"),
        # the step of the loop (nbody_plain.c:431-436)
        ("        if(!ctx->LMC) {\n            mwvector zero;\n",
         "        if (st->nbb)\n"
         "            rc |= nbStepSystemCUDAState(ctx, st);\n"
         "        else if(!ctx->LMC) {\n            mwvector zero;\n"),
        # host bodies before the best-likelihood histogram (nbody_plain.c:440-443)
        ("            get_likelihood(ctx, st, nbf);\n",
         "            nbSyncBodiesFromCUDA(st);\n            get_likelihood(ctx, st, nbf);\n"),
        # ... before a checkpoint is written (nbody_plain.c:60-73)
        ("    if (nbTimeToCheckpoint(ctx, st))\n    {\n",
         "    if (nbTimeToCheckpoint(ctx, st))\n    {\n        nbSyncBodiesFromCUDA(st);\n"),
        # ... and at the end of the run
        ("    return nbWriteFinalCheckpoint(ctx, st);\n",
         "    nbSyncBodiesFromCUDA(st);\n    return nbWriteFinalCheckpoint(ctx, st);\n"),
    ],
    "nbody.c": [
        # nbStepSystem (nbody.c:182-200)
        ("NBodyStatus nbStepSystem(const NBodyCtx* ctx, NBodyState* st)\n{\n",
         "NBodyStatus nbStepSystem(const NBodyCtx* ctx, NBodyState* st)\n{\n"
         "    if (st->nbb)\n        return nbStepSystemCUDAState(ctx, st);\n"),
    ],
    "nbody_types.c": [
        # destroyNBodyState (nbody_types.c:103)
        ("int destroyNBodyState(NBodyState* st)\n{\n",
         "int destroyNBodyState(NBodyState* st)\n{\n    nbDestroyStateCUDA(st);\n"),
    ],
}


def patch(text, edits, name):
    for old, new in edits:
        count = text.count(old)
        if count != 1:
            raise SystemExit("%s: anchor found %d times: %r" % (name, count, old[:60]))
        text = text.replace(old, new)
    # the binding's header after the file's first include
    first = text.index("#include")
    eol = text.index("\n", first) + 1
    return text[:eol] + INCLUDE + text[eol:]


def main(ref, out):
    os.makedirs(out, exist_ok=True)
    for name, edits in EDITS.items():
        with open(os.path.join(ref, "nbody", "src", name)) as f:
            text = f.read()
        with open(os.path.join(out, name), "w") as f:
            f.write(patch(text, edits, name))


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
