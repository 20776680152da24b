"""The Lambda-Beta histogram and EMD/cost likelihood computed on the GPU against the reference.

The reference's own Lua set-up (oracle/_ref) builds the Orphan-model dwarfs of
tests/golden/orphan_dwarf.lua, the steps run on the GPU, and the final bodies are evaluated
twice: by the reference's nbCreateHistogram + nbSystemLikelihood (through oracle/_ref) and by
nbLikelihoodCUDA from the device-resident bodies.  The EMD and cost components must agree
(the reference rounds the EMD to 1e-9); a batch of dwarfs must give each dwarf the
single-state likelihood.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
HIST = os.path.join(GOLDEN, "orphan_model_histogram_3")
CASES = [("5", "1024", "886885833"), ("4", "1024", "670828913"), ("5", "100", "670828913")]


def _orphan_params():
    from milkywayathome_client_b200 import HistogramParams
    # makeHistogram of tests/golden/orphan_dwarf.lua; the reference's default sunGCDist
    return HistogramParams(phi=128.79, theta=54.39, psi=90.70, lambdaStart=-50.0, lambdaEnd=50.0,
                           lambdaBins=34, betaStart=-15.0, betaEnd=15.0, betaBins=1,
                           sunGCDist=8.0)


def _run_case(variant, nbody, seed):
    from oracle import bindings as ob
    from milkywayathome_client_b200 import NBodyCtx, NBodyState, _lib
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"), HIST, int(seed),
                             [nbody, variant])
    c, nstep, _ = r.ctx(_lib.Ctx)
    ctx = NBodyCtx.from_struct(c, nstep)
    init = r.get()
    mass, types = r.masses()
    st = NBodyState.create(ctx, init["pos"], init["vel"], mass)
    assert st.run_steps(ctx, nstep) == 0
    st.set_types(types)
    pos, vel = st.bodies()
    r.set(pos, vel)
    return r, st, (init["pos"], init["vel"], mass, types, ctx)


@pytest.mark.parametrize("variant,nbody,seed", CASES)
def test_likelihood_matches_reference(variant, nbody, seed):
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import read_histogram
    r, st, _ = _run_case(variant, nbody, seed)
    data = read_histogram(HIST)
    params = _orphan_params()
    ref = r.likelihood()                       # likelihood, EMD component, cost, ...
    got = st.likelihood(params, data)[0]
    counts, totals, mpp = st.histogram(params)
    st.close()
    assert totals[0, 0] == counts.sum()
    assert abs(got[2] - ref[1]) <= 1e-9 * max(1.0, abs(ref[1])), (got, ref)
    assert abs(got[3] - ref[2]) <= 1e-9 * max(1.0, abs(ref[2])), (got, ref)


def test_batch_likelihood_matches_single_states():
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import NBodyBatch, read_histogram
    data = read_histogram(HIST)
    params = _orphan_params()
    singles, inputs = [], []
    for case in CASES[:2]:
        r, st, inp = _run_case(*case)
        singles.append((st.likelihood(params, data)[0], st.histogram(params)))
        p, v = st.bodies()
        inputs.append((p, v) + inp[2:])
        st.close()
    spec = [(len(m), ctx.eps2, ctx.timestep, ctx.treeRSize) for _, _, m, _, ctx in inputs]
    with NBodyBatch(spec) as bt:
        bt.set_bodies(np.concatenate([i[0] for i in inputs]), np.concatenate([i[1] for i in inputs]),
                      np.concatenate([i[2] for i in inputs]))
        bt.set_types(np.concatenate([i[3] for i in inputs]))
        out = bt.likelihood(params, data)
        counts, totals, mpp = bt.histogram(params)
    for k, (lk, (c1, t1, m1)) in enumerate(singles):
        assert np.array_equal(counts[k], c1[0])
        assert np.array_equal(totals[k], t1[0])
        assert mpp[k] == m1[0]
        assert np.array_equal(out[k], lk)
