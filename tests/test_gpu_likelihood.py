"""The Lambda-Beta histograms and the likelihood computed on the GPU against the reference.

The reference's own Lua set-up (oracle/_ref) builds the Orphan-model dwarfs of
tests/golden/orphan_dwarf.lua, the steps run on the GPU, and the final bodies are evaluated
twice: by the reference's nbCreateHistogram + nbSystemLikelihood (through oracle/_ref) and by
nbLikelihoodCUDA from the device-resident bodies.  Every term of the reference's likelihood
array must agree (the EMD is rounded to 1e-9 by both; the dispersions' sums are formed in
another order, so they agree to rounding): the default comparisons (EMD, cost, beta
dispersion), and every comparison (velocity dispersion, line-of-sight velocity, beta average,
distance, proper motions, beta-dispersion averaging over neighbouring bins) against a data
file in the reference's extended format.  A batch of dwarfs must give each dwarf the
single-state likelihood.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
HIST = os.path.join(GOLDEN, "orphan_model_histogram_3")
LUA = os.path.join(GOLDEN, "orphan_dwarf.lua")
CASES = [("5", "1024", "886885833"), ("4", "1024", "670828913"), ("5", "100", "670828913")]
WORST, BEST = 9999999.9, 1e-9
ALL = dict(useVelDisp=True, useBetaComp=True, useVlos=True, useDist=True, usePropMot=True)


def _orphan_params(**flags):
    from milkywayathome_client_b200 import HistogramParams
    # makeHistogram of tests/golden/orphan_dwarf.lua; the reference's default sunGCDist
    return HistogramParams(phi=128.79, theta=54.39, psi=90.70, lambdaStart=-50.0, lambdaEnd=50.0,
                           lambdaBins=34, betaStart=-15.0, betaEnd=15.0, betaBins=1,
                           sunGCDist=8.0, **flags)


def _clamped(x):
    """The worst/best-case clamps the reference applies to the likelihood itself."""
    if np.isnan(x) or x > WORST or x < -WORST:
        return WORST
    return BEST if x == 0.0 else x


def _assert_terms(got, ref):
    got = np.array(got[:10], dtype=float)
    got[0] = _clamped(got[0])
    for k in range(10):
        if np.isnan(ref[k]):
            assert np.isnan(got[k]), (k, got, ref)
        else:
            assert abs(got[k] - ref[k]) <= 1e-9 * max(1.0, abs(ref[k])), (k, got, ref)


def _run_case(variant, nbody, seed, extra=(), hist=HIST):
    from oracle import bindings as ob
    from milkywayathome_client_b200 import NBodyCtx, NBodyState, _lib
    r = ob.RefState.open_lua(LUA, hist, int(seed), [nbody, variant] + list(extra))
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
    assert np.isfinite(ref[3])                 # the beta-dispersion term is compared
    _assert_terms(got, ref)


@pytest.mark.parametrize("ranges", ["{-40,-10.3,10.3,40}", "{-30,0}", "{-45,-20,-15,5,12,48}",
                                    "{-50,50}", "{-40,-10}"])
def test_emd_ranges_match_reference(tmp_path, ranges):
    """A data file with an EMDRange line: the EMD per lambda range, each renormalised and
    weighted by its share of the data counts, rescaled by the integer ratio of all data counts
    to those in the ranges (nbMatchEMD, nbody/src/nbody_emd.c:1332-1427)."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import read_histogram
    path = tmp_path / "ranged_histogram"
    path.write_text(open(HIST).read().replace("betaBins = 1\n",
                                              "betaBins = 1\nEMDRange = %s\n" % ranges))
    r, st, _ = _run_case("5", "1024", "886885833", hist=str(path))
    data = read_histogram(str(path))
    assert data.emdRange is not None
    ref = r.likelihood()
    got = st.likelihood(_orphan_params(), data)[0]
    full = st.likelihood(_orphan_params(), read_histogram(HIST))[0]
    st.close()
    _assert_terms(got, ref)
    if ranges != "{-50,50}":
        assert got[1] != full[1]               # the ranges change the EMD term


@pytest.mark.parametrize("beta_disp_bins", [0, 3, 4])
def test_every_comparison_term_matches_reference(tmp_path, beta_disp_bins):
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import data_from_counts, read_histogram, write_histogram
    seed = "886885833"
    r, st, _ = _run_case("5", "1024", seed, ["allterms"])
    params = _orphan_params(**ALL)
    # the Orphan data file has no proper-motion columns: the reference's NaN array
    got = st.likelihood(params, read_histogram(HIST))[0]
    ref = r.likelihood()
    assert np.all(np.isnan(got[:10])) and ref[0] == WORST and np.all(np.isnan(ref[1:]))
    # a data file in the extended format from the GPU's own histograms, perturbed so that
    # every comparison contributes
    counts, totals, mpp, comps = st.histogram(params, components=True)
    assert np.any(comps[0, 4, 1] > 0) and np.any(comps[0, 5, 1] > 0)   # averages were built
    data = data_from_counts(params, counts[0], totals[0, 1], mpp[0], comps[0])
    rng = np.random.default_rng(5)
    data.components = [(c[0] * (1.0 + 0.05 * rng.standard_normal(len(c[0]))) + 0.01,
                        np.abs(c[1]) + 0.02) for c in data.components]
    data.betaDispBins = beta_disp_bins
    path = str(tmp_path / "hist_all")
    write_histogram(path, params, data)
    data2 = read_histogram(path)
    assert data2.betaDispBins == beta_disp_bins and all(c is not None for c in data2.components)
    pos, vel = st.bodies()
    r2 = ob.RefState.open_lua(LUA, path, int(seed), ["1024", "5", "allterms"])
    r2.set(pos, vel)
    ref2 = r2.likelihood()
    got2 = st.likelihood(params, data2)[0]
    st.close()
    assert np.all(np.isfinite(ref2))
    _assert_terms(got2, ref2)


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
        assert np.array_equal(out[k], lk, equal_nan=True)


# ---- two-dimensional histograms (betaBins > 1): the EMD by the transportation simplex ----
def _orphan_params_2d(beta_bins, **flags):
    from milkywayathome_client_b200 import HistogramParams
    return HistogramParams(phi=128.79, theta=54.39, psi=90.70, lambdaStart=-50.0, lambdaEnd=50.0,
                           lambdaBins=34, betaStart=-15.0, betaEnd=15.0, betaBins=beta_bins,
                           sunGCDist=8.0, **flags)


def _random_data_2d(params, seed, fill=0.6):
    """A data histogram over the two-dimensional grid: seeded counts in a fraction of the bins,
    a few bins unused."""
    from milkywayathome_client_b200 import data_from_counts
    rng = np.random.default_rng(seed)
    counts = rng.integers(1, 40, params.nbins) * (rng.uniform(size=params.nbins) < fill)
    data = data_from_counts(params, counts, int(counts.sum()) * 3, 2.5e-3)
    data.useBin[rng.choice(params.nbins, size=3, replace=False)] = 0
    return data


@pytest.mark.parametrize("beta_bins,ranges", [(2, None), (3, None), (5, None),
                                              (4, "{-40,-10.3,10.3,40}")])
def test_two_dimensional_likelihood_matches_reference(tmp_path, beta_bins, ranges):
    """betaBins > 1: each lambda range's EMD is the reference's transportation-simplex emdCalc
    over (lambda, beta) (nbMatchEMD, nbody/src/nbody_emd.c:1278-1427), solved on the GPU by the
    same decisions; every likelihood term agrees with the reference's nbSystemLikelihood."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import read_histogram, write_histogram
    params = _orphan_params_2d(beta_bins)
    data = _random_data_2d(params, 100 + beta_bins)
    path = str(tmp_path / "hist2d")
    write_histogram(path, params, data)
    if ranges:
        text = open(path).read()
        open(path, "w").write(text.replace("betaBins = %d\n" % beta_bins,
                                           "betaBins = %d\nEMDRange = %s\n" % (beta_bins, ranges)))
    r, st, _ = _run_case("5", "1024", "886885833", ["beta%d" % beta_bins], hist=path)
    counts, _, _ = st.histogram(params)
    assert np.count_nonzero(counts[0]) > 10            # a stream over many (lambda, beta) bins
    ref = r.likelihood()
    got = st.likelihood(params, read_histogram(path))[0]
    st.close()
    assert np.isfinite(ref[1]) and ref[1] > 0.0
    _assert_terms(got, ref)


def test_emd_on_the_gpu_matches_reference_emdcalc():
    """nbEmdCalcCUDA (the device solver, one block per problem) against the reference's emdCalc
    on grid signatures with ties, zero weights and unequal totals: bit for bit."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import emd
    rng = np.random.default_rng(77)
    for k in range(40):
        lb, bb = int(rng.integers(4, 30)), int(rng.integers(2, 6))
        li = np.repeat(np.arange(lb), bb)
        bi = np.tile(np.arange(bb), lb)
        sig = []
        for _ in range(2):
            c = rng.integers(1, 50, lb * bb) * (rng.uniform(size=lb * bb) < 0.5)
            w = c / max(c.sum(), 1)
            sig.append(np.stack([w, (li + 0.5) * (300.0 / lb) - 150.0, (bi + 0.5) * (30.0 / bb) - 15.0], 1))
        if k % 5 == 0:
            sig[1][:, 0] *= 1.3                          # unequal totals: the dummy node
        want, got = ob.ref_emd(sig[0], sig[1]), emd(sig[0], sig[1])
        assert np.float64(got).view(np.uint64) == np.float64(want).view(np.uint64), (k, got, want)
