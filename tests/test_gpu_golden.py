"""The reference's golden end-to-end likelihoods with every step on the GPU.

The reference's own Lua set-up (oracle/_ref: nbSetup, its dSFMT Plummer sampler and reverse
orbit) builds the initial dwarf of tests/golden/orphan_dwarf.lua; all nStep kick-drift-kick
steps then run in libnbody_b200.so; the final bodies go back to the reference for its
histogram + EMD likelihood (nbCreateHistogram / nbSystemLikelihood).  The result must equal
the reference's golden table (nbody/tests/RunTestUnits.lua, models 4, 5 and model_triaxial)
within its own tolerance, 1e-10:
thousands of chaotic N-body steps only reproduce it if every step is bit-exact.

nbRunSystemCUDA (the reference's run loop with its best-likelihood scan and, for the orbiting
bar, its calibration runs) is checked the same way: against the reference's own executable on
model 5 with the scan enabled, and against the golden table of model_bar.
"""
import json
import os

import numpy as np
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


def _reference_exe_likelihood(tmp_path, nbody, seed, args):
    """<search_likelihood> of the reference's own executable (negated: positive, lower better)."""
    import subprocess
    from oracle import bindings as ob
    out = subprocess.run(
        [ob.REF_EXE, "--checkpoint-interval=-1", "-g", "-f", os.path.join(GOLDEN, "orphan_dwarf.lua"),
         "-h", os.path.join(GOLDEN, "orphan_model_histogram_3"), "--seed", seed,
         "--ignore-checkpoint", nbody] + list(args), capture_output=True, text=True, timeout=600,
        cwd=str(tmp_path))
    line = [l for l in out.stderr.splitlines() + out.stdout.splitlines()
            if l.startswith("<search_likelihood>")][0]
    return -float(line.split(">")[1].split("<")[0])


def _gpu_run_system(variant, nbody, seed, options=()):
    from oracle import bindings as ob
    from milkywayathome_client_b200 import HistogramParams, NBodyCtx, NBodyState, _lib, read_histogram
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"),
                             os.path.join(GOLDEN, "orphan_model_histogram_3"), int(seed),
                             [nbody, variant] + list(options))
    c, nstep, time_evolve = r.ctx(_lib.Ctx)
    use_best, start, calib = r.run_params()
    ctx = NBodyCtx.from_struct(c, nstep)
    init = r.get()
    mass, types = r.masses()
    params = HistogramParams(**r.like_params())   # makeHistogram of orphan_dwarf.lua + the ctx
    data = read_histogram(os.path.join(GOLDEN, "orphan_model_histogram_3"))
    with NBodyState.create(ctx, init["pos"], init["vel"], mass, gravmap=not c.lmc) as st:
        st.set_types(types)
        if c.lmc:                  # the LMC's state and reflex accelerations of reverseOrbit_LMC
            st.set_lmc(*r.lmc())
        rc, res = st.run_system(ctx, nstep, time_evolve, params, data, use_best_like=use_best,
                                best_like_start=start, calibration_runs=calib,
                                keep_best_bodies=use_best)
        assert rc == 0
        assert st.step_count == nstep
        if use_best and res["best_count"] > 0:
            bpos, _ = st.best_bodies()
            assert np.all(np.isfinite(bpos))
    return res, (use_best, start, calib, nstep)


@pytest.mark.parametrize("nbody,seed", [("100", "670828913"), ("100", "715144259"),
                                        ("1024", "886885833")])
def test_best_likelihood_scan_matches_reference_executable(tmp_path, nbody, seed):
    """Model 5 (bit-exact steps) with the best-likelihood scan over the last 5% of the steps:
    nbRunSystemCUDA's result equals the reference executable's."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    want = _reference_exe_likelihood(tmp_path, nbody, seed, ["5", "bestlike"])
    res, (use_best, start, calib, nstep) = _gpu_run_system("5", nbody, seed, ["bestlike"])
    assert use_best and calib == 0 and res["runs"] == 1
    assert res["best_count"] >= 1 and res["best_step"] >= 0.95 * nstep
    assert abs(res["result"][0] - want) < 1e-10, (res, want)


RUN_VARIANTS = ("5b", "6", "8", "9", "ninkovic", "newhist1", "newhist2", "newhist3")
RUN_CASES = [(v, "100", s) for v in RUN_VARIANTS for s in ("670828913", "886885833", "715144259")]
RUN_CASES += [(v, "1024", "670828913") for v in ("4", "5", "triaxial") + RUN_VARIANTS]


@pytest.mark.parametrize("variant,nbody,seed", RUN_CASES)
def test_golden_likelihood_through_gpu_run_system(variant, nbody, seed):
    """Every step and the likelihood on the GPU (nbRunSystemCUDA with the context's comparison
    terms: the newhist models add the beta-average, line-of-sight velocity and distance
    comparisons) against the reference's golden table.  Models 6, 8 and ninkovic evaluate
    halos with logarithms and powers, correctly rounded on both sides, so every model here runs
    bit for bit like the reference and the likelihood (per-bin sums in body order) equals its
    golden value to the table's tolerance."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    with open(os.path.join(GOLDEN, "golden_likelihoods.json")) as f:
        want = json.load(f)["models"][variant][nbody][seed]
    res, (use_best, _, calib, _) = _gpu_run_system(variant, nbody, seed)
    assert not use_best and res["runs"] == 1
    assert abs(res["result"][0] - want) < 1e-10, (res["result"], want)


BAR_CASES = [("100", s) for s in ("670828913", "886885833", "715144259")] + [("1024", "670828913")]


@pytest.mark.parametrize("nbody,seed", BAR_CASES)
def test_bar_golden_through_gpu_run_system(nbody, seed):
    """model_bar: the orbiting bar, the best-likelihood window and two calibration runs, all on
    the GPU, against the reference's golden table."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    with open(os.path.join(GOLDEN, "golden_likelihoods.json")) as f:
        want = json.load(f)["models"]["bar"][nbody][seed]
    res, (use_best, start, calib, nstep) = _gpu_run_system("bar", nbody, seed)
    assert use_best and calib == 2 and res["runs"] == 3
    assert abs(res["result"][0] - want) < 1e-10, (res, want)


LMC_CASES = [(v, "100", s) for v in ("LMC", "LMC_bar") for s in ("670828913", "886885833",
                                                                 "430281807")]
LMC_CASES += [(v, "1024", "670828913") for v in ("LMC", "LMC_bar")]


@pytest.mark.parametrize("variant,nbody,seed", LMC_CASES)
def test_lmc_golden_through_gpu_run_system(variant, nbody, seed):
    """model_LMC and model_LMC_bar: the LMC as a moving Plummer sphere with dynamical friction
    (its orbit integrated beside the bodies on the GPU, the Milky Way's reflex accelerations
    added to every kick and to the LMC's own), against the reference's golden table."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    with open(os.path.join(GOLDEN, "golden_likelihoods.json")) as f:
        want = json.load(f)["models"][variant][nbody][seed]
    res, (use_best, _, calib, _) = _gpu_run_system(variant, nbody, seed)
    assert not use_best and calib == 0 and res["runs"] == 1
    assert abs(res["result"][0] - want) < 1e-10, (res["result"], want)


@pytest.mark.parametrize("variant", ["LMC", "LMC_bar"])
def test_lmc_steps_equal_reference(variant):
    """200 steps of an LMC run: every body and the LMC's position and velocity equal the
    reference's bit for bit (model_LMC; model_LMC_bar evaluates the bar's trigonometry with
    CUDA's functions, so its states agree to a few ulps instead)."""
    from oracle import bindings as ob
    from milkywayathome_client_b200 import NBodyCtx, NBodyState, _lib
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"),
                             os.path.join(GOLDEN, "orphan_model_histogram_3"), 670828913,
                             ["1024", variant])
    c, nstep, time_evolve = r.ctx(_lib.Ctx)
    assert c.lmc and c.lmcDynaFric
    ctx = NBodyCtx.from_struct(c, nstep)
    init = r.get()
    mass, types = r.masses()
    lmc_pos, lmc_vel, shift = r.lmc()
    assert len(shift) > nstep
    with NBodyState.create(ctx, init["pos"], init["vel"], mass, gravmap=False) as st:
        st.set_types(types)
        st.set_time_origin(time_evolve)
        st.set_lmc(lmc_pos, lmc_vel, shift)
        assert st.gravMap(ctx) == 0
        assert r.gravmap() == 0
        assert st.run_steps(ctx, 200) == 0
        assert r.step(200) == 0
        gpos, gvel = st.bodies()
        p, v = st.lmc()
    want = r.get()
    wp, wv, _ = r.lmc()
    if variant == "LMC":
        assert np.array_equal(gpos, want["pos"]) and np.array_equal(gvel, want["vel"])
        assert np.array_equal(p, wp) and np.array_equal(v, wv)
    else:
        np.testing.assert_allclose(gpos, want["pos"], rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(p, wp, rtol=1e-12)
        np.testing.assert_allclose(v, wv, rtol=1e-12)


@pytest.mark.parametrize("graph", [True, False])
def test_batch_run_system_with_best_likelihood_scan(graph):
    """nbBatchRunSystemCUDA on three model-5 dwarfs (three seeds) with the best-likelihood scan
    over the last 5 % of the steps and the best bodies kept: every dwarf's result, best step,
    best count and best bodies equal those of its own nbRunSystemCUDA run (FP64 batches step
    bit for bit like single states), and the final likelihood is the golden one when the scan
    is off."""
    from oracle import bindings as ob
    from milkywayathome_client_b200 import (HistogramParams, NBodyBatch, NBodyCtx, NBodyState,
                                            _lib, read_histogram)
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    seeds = ("670828913", "886885833", "715144259")
    data = read_histogram(os.path.join(GOLDEN, "orphan_model_histogram_3"))
    dwarfs = []
    for seed in seeds:
        r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"),
                                 os.path.join(GOLDEN, "orphan_model_histogram_3"), int(seed),
                                 ["100", "5", "bestlike"])
        c, nstep, time_evolve = r.ctx(_lib.Ctx)
        use_best, start, _ = r.run_params()
        init = r.get()
        mass, types = r.masses()
        dwarfs.append((c, nstep, time_evolve, start, init, mass, types,
                       HistogramParams(**r.like_params())))
    c, nstep, time_evolve, start, _, _, _, params = dwarfs[0]
    ctx = NBodyCtx.from_struct(c, nstep)
    want = []
    for c_, _, _, _, init, mass, types, _ in dwarfs:
        assert c_.timestep == c.timestep and c_.eps2 == c.eps2
        with NBodyState.create(ctx, init["pos"], init["vel"], mass) as st:
            st.set_types(types)
            rc, res = st.run_system(ctx, nstep, time_evolve, params, data, use_best_like=True,
                                    best_like_start=start, keep_best_bodies=True)
            assert rc == 0
            want.append((res, st.best_bodies()))
    spec = [(len(d[5]), c.eps2, c.timestep, 4.0) for d in dwarfs]
    with NBodyBatch(spec) as bt:
        bt.set_bodies(np.concatenate([d[4]["pos"] for d in dwarfs]),
                      np.concatenate([d[4]["vel"] for d in dwarfs]),
                      np.concatenate([d[5] for d in dwarfs]))
        bt.set_types(np.concatenate([d[6] for d in dwarfs]))
        rc, got = bt.run_system(ctx, nstep, time_evolve, params, data, use_best_like=True,
                                best_like_start=start, keep_best_bodies=True, graph=graph)
        assert rc == 0
        bpos, bvel = bt.best_bodies()
        offs = bt.offsets
    for k, ((w, (wpos, wvel)), g) in enumerate(zip(want, got)):
        assert w["best_count"] >= 1
        for key in ("best_step", "best_count", "runs"):
            assert g[key] == w[key], (k, key, g[key], w[key])
        assert g["best_time"] == w["best_time"]
        for key in ("result", "final", "best"):
            assert np.array_equal(g[key], w[key], equal_nan=True), (k, key, g[key], w[key])
        s = slice(offs[k], offs[k + 1])
        assert np.array_equal(bpos[s], wpos) and np.array_equal(bvel[s], wvel)


def test_batch_run_system_bar_calibration_runs():
    """model_bar dwarfs (three seeds) as one batch: the best-likelihood window and the two
    calibration runs, each dwarf's bar with its own time origin from its previous run's best
    time; every dwarf's result equals its own nbRunSystemCUDA run and the golden value."""
    from oracle import bindings as ob
    from milkywayathome_client_b200 import (HistogramParams, NBodyBatch, NBodyCtx, NBodyState,
                                            _lib, read_histogram)
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    seeds = ("670828913", "886885833", "715144259")
    with open(os.path.join(GOLDEN, "golden_likelihoods.json")) as f:
        golden = json.load(f)["models"]["bar"]["100"]
    data = read_histogram(os.path.join(GOLDEN, "orphan_model_histogram_3"))
    dwarfs = []
    for seed in seeds:
        r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"),
                                 os.path.join(GOLDEN, "orphan_model_histogram_3"), int(seed),
                                 ["100", "bar"])
        c, nstep, time_evolve = r.ctx(_lib.Ctx)
        use_best, start, calib = r.run_params()
        init = r.get()
        mass, types = r.masses()
        dwarfs.append((c, init, mass, types))
    assert use_best and calib == 2
    c = dwarfs[0][0]
    ctx = NBodyCtx.from_struct(c, nstep)
    params = HistogramParams(**r.like_params())
    want = []
    for _, init, mass, types in dwarfs:
        with NBodyState.create(ctx, init["pos"], init["vel"], mass) as st:
            st.set_types(types)
            rc, res = st.run_system(ctx, nstep, time_evolve, params, data, use_best_like=True,
                                    best_like_start=start, calibration_runs=calib)
            assert rc == 0 and res["runs"] == 3
            want.append(res)
    spec = [(len(d[2]), c.eps2, c.timestep, 4.0) for d in dwarfs]
    with NBodyBatch(spec) as bt:
        bt.set_bodies(np.concatenate([d[1]["pos"] for d in dwarfs]),
                      np.concatenate([d[1]["vel"] for d in dwarfs]),
                      np.concatenate([d[2] for d in dwarfs]))
        bt.set_types(np.concatenate([d[3] for d in dwarfs]))
        rc, got = bt.run_system(ctx, nstep, time_evolve, params, data, use_best_like=True,
                                best_like_start=start, calibration_runs=calib)
        assert rc == 0
    for k, (seed, w, g) in enumerate(zip(seeds, want, got)):
        assert g["runs"] == 3
        assert g["previous_forward_time"] == w["previous_forward_time"], k
        for key in ("best_step", "best_count", "best_time"):
            assert g[key] == w[key], (k, key, g[key], w[key])
        assert np.array_equal(g["result"], w["result"], equal_nan=True), (k, g["result"], w["result"])
        assert abs(g["result"][0] - golden[seed]) < 1e-10
