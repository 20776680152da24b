"""The benchmark's reference arm and CPU-baseline leg (bench.RefStepper) step the reference's
own code -- nbGravMap once, then whole nbStepSystem steps -- with no sampling: after k steps
its state is the reference's after k steps, and the C restatement it falls back to (where the
reference build is absent) lands on the same state bit for bit.  Both arms print the same
`config`.  The timed arm settles the FP64 walk's automatic form before timing.  CPU only."""
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


class _FakeState:
    """Stands in for NBodyState: the walk form is chosen after `decide_after` evaluations."""

    def __init__(self, decide_after):
        self.evaluations = 0
        self.decide_after = decide_after

    def walk_form(self):
        return 1 if self.evaluations >= self.decide_after else -1

    def gravMap(self, ctx):
        self.evaluations += 1
        return 0

    def check(self, what, rc):
        assert rc == 0, what


def test_walk_form_is_settled_before_timed_steps():
    """bench settles the FP64 walk's automatic form with untimed force evaluations, only for
    FP64 tree walks, and never loops past its bound."""
    import bench
    from milkywayathome_client_b200 import NBodyCtx, models
    ctx = NBodyCtx(potential=models.sample_workunit_potential(), **models.dwarf_config(4096))
    st = _FakeState(decide_after=2)
    bench.settle_walk_form(st, ctx)
    assert st.evaluations == 2 and st.walk_form() == 1
    st = _FakeState(decide_after=0)
    bench.settle_walk_form(st, ctx)
    assert st.evaluations == 0
    st = _FakeState(decide_after=100)
    bench.settle_walk_form(st, ctx)
    assert st.evaluations == 8
    st = _FakeState(decide_after=2)
    bench.settle_walk_form(st, ctx.with_precision("mixed"))
    assert st.evaluations == 0
    assert set(bench.WALK_FORM_NAMES) == {0, 1, 2}
