"""The reference's golden end-to-end likelihoods with every step on the GPU.

The reference's own Lua set-up (oracle/_ref: nbSetup, its dSFMT Plummer sampler and reverse
orbit) builds the initial dwarf of tests/golden/orphan_dwarf.lua; all nStep kick-drift-kick
steps then run in libnbody_b200.so; the final bodies go back to the reference for its
histogram + EMD likelihood (nbCreateHistogram / nbSystemLikelihood).  The result must equal
the reference's golden table (nbody/tests/RunTestUnits.lua, models 4, 5 and model_triaxial)
within its own tolerance, 1e-10:
thousands of chaotic N-body steps only reproduce it if every step is bit-exact.
"""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = [("5", "100", s) for s in ("670828913", "886885833", "715144259", "430281807", "543966758")]
CASES += [("4", "100", s) for s in ("670828913", "886885833")]
CASES += [("5", "1024", "886885833"), ("4", "1024", "670828913")]
# The triaxial halo (model_triaxial): its force has no power, logarithm or trigonometric
# function (c1..c3 come over from the reference's own set-up), so it is bit-exact too.
CASES += [("triaxial", "100", s) for s in ("670828913", "886885833", "715144259")]
CASES += [("triaxial", "1024", "670828913")]


@pytest.mark.parametrize("variant,nbody,seed", CASES)
def test_golden_likelihood_through_gpu_steps(variant, nbody, seed):
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import NBodyCtx, NBodyState, _lib
    with open(os.path.join(GOLDEN, "golden_likelihoods.json")) as f:
        want = json.load(f)["models"][variant][nbody][seed]
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"),
                             os.path.join(GOLDEN, "orphan_model_histogram_3"), int(seed),
                             [nbody, variant])
    c, nstep, _ = r.ctx(_lib.Ctx)
    ctx = NBodyCtx.from_struct(c, nstep)
    init = r.get()
    mass, _ = r.masses()
    with NBodyState.create(ctx, init["pos"], init["vel"], mass) as st:
        rc = st.run_steps(ctx, nstep)
        assert rc == 0
        assert st.step_count == nstep
        pos, vel = st.bodies()
    r.set(pos, vel)
    got = r.likelihood()[0]
    assert abs(got - want) < 1e-10, (got, want)
