"""The LMC of the reference's LMC runs on the GPU, against the reference build (oracle/_ref).

The forward runs of model_LMC and model_LMC_bar take coulomb_log from the context, where it is
0, so their dynamical friction is zero and the golden tests (test_gpu_golden.py) check the LMC's
orbit bit for bit.  Here the friction is on (coulomb_log 0.470003629, the value
reverseOrbit_LMC integrates with): Chandrasekhar's formula with the potential's density and
the quadrature velocity dispersion (dynamicalFriction_LMC, nbody/src/nbody_friction.c:85-132).
Its erf and exp are the C library's in the reference and CUDA's here, so the LMC's orbit and
the bodies agree to rounding, not bit for bit.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _setup(variant, coulomb_log):
    from oracle import bindings as ob
    from milkywayathome_client_b200 import _lib
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"),
                             os.path.join(GOLDEN, "orphan_model_histogram_3"), 670828913,
                             ["1024", variant])
    c, nstep, time_evolve = r.ctx(_lib.Ctx)
    init = r.get()
    mass, types = r.masses()
    lmc = r.lmc()
    c.coulombLog = coulomb_log
    ref = ob.RefState.create(c, init["pos"], init["vel"], mass, types)
    ref.set_lmc(*lmc)
    r.close()
    return c, nstep, init, mass, types, lmc, ref


@pytest.mark.parametrize("variant", ["LMC", "LMC_bar"])
def test_lmc_with_friction_against_reference(variant):
    from milkywayathome_client_b200 import NBodyCtx, NBodyState
    c, nstep, init, mass, types, (lp, lv, shift), ref = _setup(variant, 0.470003629)
    ctx = NBodyCtx.from_struct(c, nstep)
    with NBodyState.create(ctx, init["pos"], init["vel"], mass, gravmap=False) as st:
        st.set_types(types)
        st.set_lmc(lp, lv, shift)
        assert st.gravMap(ctx) == 0
        assert st.run_steps(ctx, 100) == 0
        gpos, gvel = st.bodies()
        p, v = st.lmc()
    assert ref.gravmap() == 0 and ref.step(100) == 0
    want = ref.get()
    wp, wv, _ = ref.lmc()
    # the friction changes the LMC's velocity by ~0.1 km/s in 100 steps; agreement to rounding
    np.testing.assert_allclose(p, wp, rtol=1e-12)
    np.testing.assert_allclose(v, wv, rtol=1e-12)
    np.testing.assert_allclose(gpos, want["pos"], rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(gvel, want["vel"], rtol=1e-9, atol=1e-9)
    # and it is on: without it the LMC ends elsewhere
    _, _, _, _, _, _, ref0 = _setup(variant, 0.0)
    assert ref0.gravmap() == 0 and ref0.step(100) == 0
    assert np.abs(ref0.lmc()[1] - wv).max() > 1e3 * np.abs(v - wv).max()


def test_lmc_state_required_and_shift_bounds():
    """An LMC context without the LMC's state, or past the end of its reflex accelerations,
    is refused with an error status (no kernel runs on a missing array)."""
    from milkywayathome_client_b200 import NBodyCtx, NBodyError, NBodyState
    c, nstep, init, mass, types, (lp, lv, shift), ref = _setup("LMC", 0.0)
    ctx = NBodyCtx.from_struct(c, nstep)
    with NBodyState.create(ctx, init["pos"], init["vel"], mass, gravmap=False) as st:
        st.set_types(types)
        with pytest.raises(NBodyError):
            st.check("nbGravMap", st.gravMap(ctx))
        st.set_lmc(lp, lv, shift[:4])          # steps k = 0..2 (each takes k and k + 1)
        assert st.gravMap(ctx) == 0
        assert st.run_steps(ctx, 3) == 0
        with pytest.raises(NBodyError):
            st.check("nbStepSystem", st.step(ctx))


def test_lmc_in_the_mixed_form():
    """The mixed-precision walk with an LMC: the LMC's own orbit does not depend on the bodies,
    so it equals the FP64 run's bit for bit; the bodies agree to the mixed walk's accuracy."""
    from milkywayathome_client_b200 import NBodyCtx, NBodyState
    c, nstep, init, mass, types, (lp, lv, shift), ref = _setup("LMC", 0.470003629)
    out = {}
    for precision in ("fp64", "mixed"):
        ctx = NBodyCtx.from_struct(c, nstep).with_precision(precision)
        with NBodyState.create(ctx, init["pos"], init["vel"], mass, gravmap=False) as st:
            st.set_types(types)
            st.set_lmc(lp, lv, shift)
            assert st.gravMap(ctx) == 0
            assert st.run_steps(ctx, 50) == 0
            out[precision] = (st.bodies(), st.lmc())
    (p64, v64), (l64p, l64v) = out["fp64"]
    (pmx, vmx), (lmxp, lmxv) = out["mixed"]
    assert np.array_equal(l64p, lmxp) and np.array_equal(l64v, lmxv)
    scale = np.abs(p64).max()
    assert np.abs(pmx - p64).max() < 1e-6 * scale


@pytest.mark.parametrize("variant", ["LMC", "LMC_bar"])
def test_batch_of_lmc_dwarfs_equals_single_states(variant):
    """Three LMC-run dwarfs (three seeds, each with its own LMC orbit and reflex accelerations)
    as one batch, friction on: after 60 steps through captured graphs every body and every
    LMC equal the single-state runs bit for bit."""
    from oracle import bindings as ob
    from milkywayathome_client_b200 import NBodyBatch, NBodyCtx, NBodyState, _lib
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    dwarfs = []
    for seed in (670828913, 886885833, 430281807):
        r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"),
                                 os.path.join(GOLDEN, "orphan_model_histogram_3"), seed,
                                 ["100", variant])
        c, nstep, time_evolve = r.ctx(_lib.Ctx)
        c.coulombLog = 0.470003629
        init = r.get()
        mass, types = r.masses()
        dwarfs.append((init, mass, types, r.lmc()))
        r.close()
    ctx = NBodyCtx.from_struct(c, nstep)
    k = min(len(d[3][2]) for d in dwarfs)
    want = []
    for init, mass, types, (lp, lv, sh) in dwarfs:
        with NBodyState.create(ctx, init["pos"], init["vel"], mass, gravmap=False) as st:
            st.set_types(types)
            st.set_time_origin(time_evolve)
            st.set_lmc(lp, lv, sh[:k])
            assert st.gravMap(ctx) == 0
            assert st.run_steps(ctx, 60) == 0
            want.append((st.bodies(), st.lmc()))
    spec = [(len(d[1]), c.eps2, c.timestep, 4.0) for d in dwarfs]
    with NBodyBatch(spec) as bt:
        bt.set_bodies(np.concatenate([d[0]["pos"] for d in dwarfs]),
                      np.concatenate([d[0]["vel"] for d in dwarfs]),
                      np.concatenate([d[1] for d in dwarfs]))
        bt.set_types(np.concatenate([d[2] for d in dwarfs]))
        bt.set_time_origin(time_evolve)
        bt.set_lmc([d[3][0] for d in dwarfs], [d[3][1] for d in dwarfs],
                   np.stack([d[3][2][:k] for d in dwarfs]))
        assert bt.gravMap(ctx) == 0
        assert bt.run_steps(ctx, 60, graph=True) == 0
        pos, vel = bt.bodies()
        lp, lv = bt.lmc()
        offs = bt.offsets
    for j, ((wpos, wvel), (wlp, wlv)) in enumerate(want):
        s = slice(offs[j], offs[j + 1])
        assert np.array_equal(pos[s], wpos) and np.array_equal(vel[s], wvel), j
        assert np.array_equal(lp[j], wlp) and np.array_equal(lv[j], wlv), j
