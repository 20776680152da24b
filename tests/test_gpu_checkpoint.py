"""A GPU-resident state through the reference's own checkpoint files.

The reference checkpoints by writing its context and state, the host Body[] included, with
nbWriteCheckpoint and resumes with nbReadCheckpoint (nbody/src/nbody_checkpoint.c:597-672);
nbody/tests/CheckpointTest.lua requires a resumed run to equal an uninterrupted one.  A GPU run
checkpoints the same way: the device bodies are marshalled out into the host Body[]
(nbMarshalBodiesCUDA), the step counter and root size go into the state the header records,
the reference writes the file; resuming reads it with the reference's reader, marshals the
bodies in, restores the step counter (nbSetStepCUDA) and recomputes the accelerations, as
nbRunSystemPlain does before its first step (nbody/src/nbody_plain.c:388).  The resumed GPU
run, and the reference resuming the same file on the CPU, must both equal the uninterrupted
GPU run bit for bit.
"""
import numpy as np
import pytest

from conftest import bits_equal, make_ctx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("criterion,theta", [("TreeCode", 0.7), ("SW93", 1.0)])
def test_checkpoint_round_trip_bitexact(dwarf_small, tmp_path, criterion, theta):
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import NBodyCtx, NBodyState, _lib
    pos, vel, mass, typ = dwarf_small
    n = len(mass)
    ctx = make_ctx(n, theta=theta, criterion=criterion)
    path, tmp = str(tmp_path / "nbody_checkpoint"), str(tmp_path / "nbody_checkpoint_tmp")
    with NBodyState.create(ctx, pos, vel, mass) as a:
        assert a.run_steps(ctx, 12) == 0
        # checkpoint: the GPU bodies into a reference state's Body[], then the reference writer
        r = ob.RefState.create(ctx.struct, pos, vel, mass, typ)
        tab = r.bodytab()
        a.marshal_bodies(tab, to_device=False)
        info = a.tree_info()
        r.set_progress(info.step, info.rsize, info.treeIncest)
        r.write_checkpoint(path, tmp)
        r.close()
        # the uninterrupted run goes on
        assert a.run_steps(ctx, 9) == 0
        p_a, v_a = a.bodies()
        acc_a = a.accels()
        rs_a = a.tree_info().rsize
        assert a.step_count == 21

    r2 = ob.RefState.read_checkpoint(path)
    c2, _, _ = r2.ctx(_lib.Ctx)
    step, rsize, incest = r2.progress()
    assert (step, rsize, incest) == (12, info.rsize, 0)
    assert (c2.eps2, c2.theta, c2.timestep, c2.criterion, c2.useQuad) == (
        ctx.eps2, ctx.theta, ctx.timestep, ctx.criterion, ctx.useQuad)
    ctx2 = NBodyCtx.from_struct(c2)
    tab2 = r2.bodytab()
    assert bits_equal(tab2["mass"], mass) and np.array_equal(tab2["type"], typ)
    with NBodyState(n) as b:
        b.marshal_bodies(tab2, to_device=True, treeRSize=rsize)
        b.set_step(step)
        assert b.gravMap(ctx2) == 0
        assert b.run_steps(ctx2, 9) == 0
        assert b.step_count == 21
        assert b.tree_info().rsize == rs_a
        p_b, v_b = b.bodies()
        acc_b = b.accels()
    assert bits_equal(p_b, p_a) and bits_equal(v_b, v_a) and bits_equal(acc_b, acc_a)

    # the reference resumes the same file on the CPU (nbGravMap, then nbStepSystem)
    assert r2.gravmap() == 0
    assert r2.step(9) == 0
    want = r2.get()
    r2.close()
    assert want["step"] == 21
    assert bits_equal(want["pos"], p_a) and bits_equal(want["vel"], v_a)
    assert bits_equal(want["acc"], acc_a)

