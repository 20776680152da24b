"""nbEnergyCUDA (the energy-drift oracle of the walk forms) against a numpy FP64 restatement."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _phi_ext_numpy(pot, x):
    """Miyamoto-Nagai + logarithmic halo + Hernquist bulge potential (a = -grad Phi)."""
    X, Y, Z = x[:, 0], x[:, 1], x[:, 2]
    r = np.maximum(np.sqrt(X * X + Y * Y + Z * Z), 2.0 ** -8)
    d = pot.disk
    azp = d.scaleLength + np.sqrt(Z * Z + d.scaleHeight ** 2)
    phi = -d.mass / np.sqrt(X * X + Y * Y + azp * azp)
    h = pot.halo
    phi += h.vhalo ** 2 * np.log(h.scaleLength ** 2 + X * X + Y * Y + (Z / h.flattenZ) ** 2)
    s = pot.sphere
    phi += -s.mass / (r + s.scale)
    return phi


def test_energy_matches_numpy_direct_sum():
    from milkywayathome_client_b200 import NBodyCtx, NBodyState, milky_way_potential, models
    n = 2048
    pos, vel, mass, _ = models.plummer_plummer_dwarf(n, seed=21)
    cfg = models.dwarf_config(n, theta=0.5)
    ctx = NBodyCtx(potential=milky_way_potential(), **cfg)
    with NBodyState.create(ctx, pos, vel, mass) as st:
        kin, self_pot, ext = st.energy(ctx)
    kin_ref = 0.5 * np.sum(mass * np.sum(vel * vel, axis=1))
    d = pos[None, :, :] - pos[:, None, :]
    r = np.sqrt(np.sum(d * d, axis=2) + cfg["eps2"])
    np.fill_diagonal(r, np.inf)
    self_ref = -0.5 * np.sum(mass[:, None] * mass[None, :] / r)
    ext_ref = np.sum(mass * _phi_ext_numpy(ctx.struct.pot, pos))
    assert abs(kin - kin_ref) <= 1e-12 * abs(kin_ref)
    assert abs(self_pot - self_ref) <= 1e-11 * abs(self_ref)
    assert abs(ext - ext_ref) <= 1e-12 * abs(ext_ref)


def test_energy_is_conserved_by_small_steps():
    """A direct-summation run with a quarter of the default step keeps the total energy to
    1e-8 (the oracle's leapfrog drifts by 8e-10 over the same run; the external potential
    dominates the total)."""
    from milkywayathome_client_b200 import NBodyCtx, NBodyState, milky_way_potential, models
    n = 1024
    pos, vel, mass, _ = models.plummer_plummer_dwarf(n, seed=22)
    cfg = models.dwarf_config(n, theta=0.5, criterion="Exact")
    cfg["timestep"] *= 0.25
    ctx = NBodyCtx(potential=milky_way_potential(), **cfg)
    with NBodyState.create(ctx, pos, vel, mass) as st:
        e0 = sum(st.energy(ctx))
        st.check("nbRunSteps", st.run_steps(ctx, 40))
        e1 = sum(st.energy(ctx))
    assert abs(e1 - e0) <= 1e-8 * abs(e0)
