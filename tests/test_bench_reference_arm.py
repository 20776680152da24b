"""The benchmark's reference arm and CPU-baseline leg (bench.RefStepper) step the reference's
own code -- nbGravMap once, then whole nbStepSystem steps -- with no sampling: after k steps
its state is the reference's after k steps, and the C restatement it falls back to (where the
reference build is absent) lands on the same state bit for bit.  Both arms print the same
`config`.  CPU only."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_ref_stepper_takes_whole_reference_steps():
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    import bench
    from milkywayathome_client_b200 import models
    pos, vel, mass, typ = models.plummer_plummer_dwarf(3000, seed=3)
    ctx, _ = bench.bench_ctx(3000, 0.5)
    ref = bench.RefStepper(ctx, pos, vel, mass, typ)
    assert ref.kind == "reference" and ref.status == 0
    secs = [ref.step(1) for _ in range(3)]
    assert all(s > 0 for s in secs) and ref.status == 0
    got = ref.r.get()
    ref.close()
    assert got["step"] == 3
    # the oracle's C restatement (the fallback) reaches the same state
    rc, p, v, a, _ = ob.steps(ctx.struct, pos, vel, mass, ctx.treeRSize, 3)
    assert rc == 0
    for x, y in ((got["pos"], p), (got["vel"], v), (got["acc"], a)):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))


def test_port_stepper_matches_one_call_run():
    import bench
    from oracle import bindings as ob
    from milkywayathome_client_b200 import models
    pos, vel, mass, typ = models.plummer_plummer_dwarf(2000, seed=4)
    ctx, _ = bench.bench_ctx(2000, 0.7)
    st = bench.RefStepper.__new__(bench.RefStepper)
    st.ob, st.ctx, st.kind, st.n = ob, ctx, "port", 2000
    st.cores = 1
    st.status, st.pos, st.vel, st.acc, st.rsize = ob.steps(ctx.struct, pos, vel, mass,
                                                            ctx.treeRSize, 0)
    st.mass = np.ascontiguousarray(mass)
    st.step(1)
    st.step(1)
    rc, p, v, a, rs = ob.steps(ctx.struct, pos, vel, mass, ctx.treeRSize, 2)
    assert st.status == rc == 0 and st.rsize == rs
    assert np.array_equal(st.pos, p) and np.array_equal(st.vel, v) and np.array_equal(st.acc, a)


def test_both_arms_print_the_same_config():
    import bench
    a = bench.bench_config(1048576, 0.5)
    b = bench.bench_config(1048576, 0.5)
    assert a == b and a["n_bodies"] == 1048576 and a["theta"] == 0.5
    assert a["eps2"] == bench.bench_ctx(1048576, 0.5)[0].eps2
