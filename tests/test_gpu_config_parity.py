"""Parity on the benchmark's own configurations, against the reference built from its sources
(oracle/_ref).

(a) The CPU-runnable two-component dwarf: tests/golden/config0_dwarf.lua builds 20,000 bodies
    with the reference's own Lua set-up and sampler (the sample workunit's Plummer+Plummer
    dwarf on its orbit point, its potential, TreeCode theta = 1.0 with quadrupoles, dt and eps2
    from the reference's formulas).  200 GPU steps against 200 of the reference's nbStepSystem
    (nbody/src/nbody.c:182-200): positions, velocities and accelerations bit for bit; then the
    Lambda-Beta histogram and every likelihood term (nbSystemLikelihood) to 1e-9 against a data
    histogram of the initial state.
(b) The 1M dwarf of the benchmark (N = 1,048,576 sampled on the GPU, seed 1000): one tree build
    and one force evaluation at theta = 0.5 and 1.0 against nbMakeTree / nbGravMap
    (nbody/src/nbody_tree.c:429-460, nbody/src/nbody_grav.c:305-328): the node count, depth,
    root size and every node's centre of mass, mass, rcrit2, quadrupole, Next link, body and
    depth bit for bit, and every acceleration bit for bit.
"""
import os

import numpy as np
import pytest

from conftest import bits_equal

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CONFIG0 = os.path.join(GOLDEN, "config0_dwarf.lua")
TREE_KEYS = ("pos", "mass", "rcrit2", "quad", "next", "body", "depth")


def _need_ref():
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    return ob


def test_config0_200_steps_and_likelihood(tmp_path):
    ob = _need_ref()
    from milkywayathome_client_b200 import (HistogramParams, NBodyCtx, NBodyState, _lib,
                                            data_from_counts, read_histogram, write_histogram)
    r = ob.RefState.open_lua(CONFIG0, None, 270828913, [])
    c, nstep, _ = r.ctx(_lib.Ctx)
    ctx = NBodyCtx.from_struct(c, nstep)
    assert c.theta == 1.0 and c.useQuad == 1 and r.nbody == 20000
    init = r.get()
    mass, types = r.masses()
    assert int((types > 0).sum()) == 10000
    params = HistogramParams(lambdaStart=-150.0, lambdaEnd=150.0, lambdaBins=50, betaStart=-15.0,
                             betaEnd=15.0, betaBins=1, **r.like_params())
    with NBodyState.create(ctx, init["pos"], init["vel"], mass) as st:
        st.set_types(types)
        # the data: the initial state's own histogram, in the reference's file format
        counts, totals, mpp, comps = st.histogram(params, components=True)
        data = data_from_counts(params, counts[0], totals[0, 1], mpp[0], comps[0])
        path = str(tmp_path / "config0_initial_hist")
        write_histogram(path, params, data)
        r.set_histogram_file(path)
        assert r.gravmap() == 0
        assert r.step(200) == 0
        want = r.get()
        assert st.run_steps(ctx, 200) == 0
        p, v = st.bodies()
        a = st.accels()
        assert st.step_count == 200 == want["step"]
        assert st.tree_info().rsize == want["rsize"]
        got = st.likelihood(params, read_histogram(path))[0]
    assert bits_equal(p, want["pos"]) and bits_equal(v, want["vel"]) and bits_equal(a, want["acc"])
    ref = r.likelihood()
    r.close()
    assert np.isfinite(ref[0]) and np.isfinite(ref[1])
    for k in range(10):
        if np.isnan(ref[k]):
            assert np.isnan(got[k]), (k, got, ref)
        else:
            assert abs(got[k] - ref[k]) <= 1e-9 * max(1.0, abs(ref[k])), (k, got, ref)


@pytest.fixture(scope="module")
def dwarf_1m():
    from milkywayathome_client_b200 import models
    return models.sampled_dwarf(1048576, seed=1000)


@pytest.mark.parametrize("theta", [0.5, 1.0])
def test_1m_tree_and_gravmap_bitexact(dwarf_1m, theta):
    ob = _need_ref()
    from milkywayathome_client_b200 import NBodyCtx, NBodyState, models
    pos, vel, mass, types = dwarf_1m
    n = len(mass)
    ctx = NBodyCtx(potential=models.sample_workunit_potential(), **models.dwarf_config(n, theta=theta))
    r = ob.RefState.create(ctx.struct, pos, vel, mass, types)
    assert r.maketree() == 0
    want = r.tree()
    with NBodyState.create(ctx, pos, vel, mass, gravmap=False) as st:
        assert st.makeTree(ctx) == 0
        info = st.tree_info()
        got = st.tree()
        assert info.nNodes == want["nNodes"] and info.maxDepth == want["maxDepth"]
        assert info.cellUsed == want["cellUsed"] and info.rsize == want["rsize"]
        for k in TREE_KEYS:
            if k in ("next", "body", "depth"):
                assert np.array_equal(got[k], want[k]), k
            else:
                assert bits_equal(got[k], want[k]), k
        del got, want
        assert r.gravmap() == 0
        acc = r.get()["acc"]
        assert st.gravMap(ctx) == 0
        assert bits_equal(st.accels(), acc)
    r.close()
