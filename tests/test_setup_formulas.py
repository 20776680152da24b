"""The set-up formulas the benchmark and the batched workload use on the host, pinned to the
reference's own Lua set-up (oracle/_ref, built from the reference's sources): the
two-component timestep of the sample workunit with nbCorrectTimestep's correction, and
calculateEps2 (nbCalculateVirial's Gauss-Legendre integral, eps = 0.98 r_v N^-0.26) at the
body counts of the CPU-runnable dwarf (20,000), the 1M dwarf and the 8M dwarf.

tests/golden/config0_dwarf.lua evaluates calculateEps2 at its second argument while sampling
only its first, so the 1M and 8M softenings are read without sampling those dwarfs.
Both are compared bit for bit: the timestep takes the same IEEE operations and C library pow
on both sides; the restatement of the integral forms its terms in the reference's operation
order and sums them one after another as the reference's loop does (its powers come from
numpy's pow rather than crlibm's pow_rn, which agree on every term here).
"""
import os

import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CONFIG0 = os.path.join(GOLDEN, "config0_dwarf.lua")


@pytest.mark.parametrize("n_eps,theta,nsteps", [(20000, 1.0, 200), (1048576, 0.5, 100),
                                                (8388608, 0.5, 50)])
def test_dwarf_config_matches_reference_lua(n_eps, theta, nsteps):
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import _lib, models
    from milkywayathome_client_b200.nbody import NBodyCtx
    r = ob.RefState.open_lua(CONFIG0, None, 1, ["64", str(n_eps), repr(theta), str(nsteps)])
    c, nstep, time_evolve = r.ctx(_lib.Ctx)
    r.close()
    cfg = models.dwarf_config(n_eps, theta=theta)
    ctx = NBodyCtx(timeEvolve=nsteps * cfg["timestep"], **cfg)
    assert time_evolve == nsteps * cfg["timestep"]
    assert ctx.nStep == nstep
    assert ctx.timestep == c.timestep
    assert c.theta == theta and c.criterion == ctx.criterion and c.useQuad == 1
    assert cfg["eps2"] == c.eps2


def test_sample_workunit_potential_matches_reference_lua():
    """The benchmark's potential is the sample workunit's (vhalo 74.61 kpc/Gyr = 73 km/s)."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    import ctypes
    from milkywayathome_client_b200 import _lib, models
    r = ob.RefState.open_lua(CONFIG0, None, 1, ["64"])
    c, _, _ = r.ctx(_lib.Ctx)
    r.close()
    want = models.sample_workunit_potential()
    assert ctypes.sizeof(c.pot) == ctypes.sizeof(want)
    assert bytes(c.pot) == bytes(want)
