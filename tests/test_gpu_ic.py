"""The GPU two-component dwarf sampler (nbGenerateDwarfCUDA) against the reference's own
mixed-dwarf sampler (nbGenerateMixedDwarfCore through oracle/_ref, tests/golden/
two_component_dwarf.lua).  The random streams differ, so the check is statistical: two-sample
Kolmogorov-Smirnov tests on the radii and speeds of each component about its centre, plus the
exact recentring onto the orbit position and velocity and the reference's particle masses.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
POS = np.array([-21.6, -10.4, 23.2])
VEL = np.array([-150.0, 80.0, 100.0])


def _components(pos, vel, mass, nb):
    out = []
    for sel in (slice(0, nb), slice(nb, len(mass))):
        m = mass[sel]
        cm = (m[:, None] * pos[sel]).sum(0) / m.sum()
        cv = (m[:, None] * vel[sel]).sum(0) / m.sum()
        out.append((cm, cv, np.linalg.norm(pos[sel] - cm, axis=1),
                    np.linalg.norm(vel[sel] - cv, axis=1), m))
    return out


@pytest.mark.parametrize("params", [(12.0, 0.2, 0.2, 0.2), (30.0, 0.3, 0.4, 0.5)])
def test_sampler_matches_reference_distributions(params):
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from scipy.stats import ks_2samp
    from milkywayathome_client_b200 import NBodyCtx, NBodyState
    mass_l, rscale_l, rr, mr = params
    n, nb = 6000, 3000
    rscale_d = rscale_l / rr * (1.0 - rr)
    mass_d = mass_l / mr * (1.0 - mr)
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "two_component_dwarf.lua"), None, 4242,
                             [str(n), str(nb), repr(mass_l), repr(rscale_l), repr(mass_d),
                              repr(rscale_d)])
    g = r.get()
    rmass, rtypes = r.masses()
    ctx = NBodyCtx(timestep=1e-4, eps2=1e-6, theta=0.5)
    with NBodyState.generate(ctx, n, seed=99, nbody_baryon=nb, mass_l=mass_l, rscale_l=rscale_l,
                             light_r_ratio=rr, light_mass_ratio=mr, position=POS, velocity=VEL,
                             gravmap=False) as st:
        pos, vel = st.bodies()
    assert np.all(rtypes[:nb] == 1) and np.all(rtypes[nb:] == -1)
    ref = _components(g["pos"], g["vel"], rmass, nb)
    gpu = _components(pos, vel, rmass, nb)      # the same particle masses (mass / count)
    for (rcm, rcv, rr_, rv, rm), (gcm, gcv, gr, gv, gm) in zip(ref, gpu):
        np.testing.assert_allclose(gcm, POS, rtol=0, atol=1e-9)
        np.testing.assert_allclose(gcv, VEL, rtol=0, atol=1e-9)
        assert ks_2samp(rr_, gr).pvalue > 1e-3, ks_2samp(rr_, gr)
        assert ks_2samp(rv, gv).pvalue > 1e-3, ks_2samp(rv, gv)


def test_batch_generation_matches_single_sampler():
    from scipy.stats import ks_2samp
    from milkywayathome_client_b200 import NBodyBatch, NBodyCtx, NBodyState
    from milkywayathome_client_b200.nbody import plummer_dwarf_struct
    specs = [(5000, 11, 12.0, 0.2, 0.2, 0.2, (-20.0, 5.0, 3.0)),
             (3001, 12, 30.0, 0.3, 0.4, 0.5, (10.0, -4.0, 30.0)),
             (7777, 13, 3.0, 0.15, 0.25, 0.05, (0.0, 40.0, -8.0))]
    dw = [plummer_dwarf_struct(n, s, None, m, r, rr, mr, p, (10.0, 20.0, 30.0))
          for n, s, m, r, rr, mr, p in specs]
    with NBodyBatch([(n, 1e-4, 1e-4, 4.0) for n, *_ in specs]) as bt:
        bt.generate(dw)
        pos, vel = bt.bodies()
        offs = bt.offsets
    ctx = NBodyCtx(timestep=1e-4, eps2=1e-6, theta=0.5)
    for k, (n, s, m, r, rr, mr, p) in enumerate(specs):
        bp = pos[offs[k]:offs[k + 1]]
        nb = n // 2
        np.testing.assert_allclose(bp[:nb].mean(0), p, atol=1e-9)     # equal particle masses
        np.testing.assert_allclose(bp[nb:].mean(0), p, atol=1e-9)
        with NBodyState.generate(ctx, n, seed=s + 100, mass_l=m, rscale_l=r, light_r_ratio=rr,
                                 light_mass_ratio=mr, position=p, gravmap=False) as st:
            sp, _ = st.bodies()
        for sel in (slice(0, nb), slice(nb, n)):
            a = np.linalg.norm(bp[sel] - p, axis=1)
            b = np.linalg.norm(sp[sel] - p, axis=1)
            assert ks_2samp(a, b).pvalue > 1e-3


PROFILE_CASES = [("plummer", "nfw", 12.0, 0.2, 40.0, 0.8, 0.0, 0.0),
                 ("plummer", "general_hernquist", 12.0, 0.2, 48.0, 0.8, 0.0, 0.0),
                 ("plummer", "cored", 12.0, 0.2, 40.0, 0.8, 0.3, 0.2),
                 ("general_hernquist", "nfw", 12.0, 0.2, 40.0, 0.8, 0.0, 0.0)]


def _component(kind, mass, scale, r1, rc):
    from milkywayathome_client_b200 import Dwarf
    if kind == "cored":
        return Dwarf.cored(mass, scale, r1, rc)
    return getattr(Dwarf, kind)(mass, scale)


@pytest.mark.parametrize("case", PROFILE_CASES, ids=lambda c: c[0] + "-" + c[1])
def test_profiles_match_reference_distributions(case):
    """NFW, general Hernquist and cored components (nbGenerateMixedDwarfCUDA) against the
    reference's sampler: the same particle masses bit for bit (the NFW/cored mass reset), the
    exact recentring, and two-sample KS tests of radii and speeds per component."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from scipy.stats import ks_2samp
    from milkywayathome_client_b200 import NBodyCtx, NBodyState
    tl, td, ml, al, md, ad, r1, rc = case
    n, nb = 4000, 2000
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "two_component_dwarf.lua"), None, 4242,
                             [str(n), str(nb), repr(ml), repr(al), repr(md), repr(ad), tl, td,
                              repr(r1), repr(rc)])
    g = r.get()
    rmass, rtypes = r.masses()
    ctx = NBodyCtx(timestep=1e-4, eps2=1e-6, theta=0.5)
    with NBodyState.generate_mixed(ctx, n, 77, _component(tl, ml, al, r1, rc),
                                   _component(td, md, ad, r1, rc), nbody_baryon=nb,
                                   position=POS, velocity=VEL, gravmap=False) as st:
        pos, vel = st.bodies()
        gmass = st.masses()
    assert np.array_equal(gmass, rmass)
    for (rcm, rcv, *_), (gcm, gcv, *_) in zip(_components(g["pos"], g["vel"], rmass, nb),
                                              _components(pos, vel, gmass, nb)):
        np.testing.assert_allclose(gcm, POS, rtol=0, atol=1e-9)
        np.testing.assert_allclose(gcv, VEL, rtol=0, atol=1e-9)
    # radii and speeds about each component's coordinate-wise median: the Hernquist and NFW
    # tails reach the sampling bound, which moves a sample's centre of mass by a good fraction
    # of the core radius (and differently in the two samples)
    for sel in (slice(0, nb), slice(nb, n)):
        for a, b in ((g["pos"][sel], pos[sel]), (g["vel"][sel], vel[sel])):
            ra = np.linalg.norm(a - np.median(a, axis=0), axis=1)
            rb = np.linalg.norm(b - np.median(b, axis=0), axis=1)
            assert ks_2samp(ra, rb).pvalue > 1e-3, ks_2samp(ra, rb)


def test_batch_of_mixed_profiles():
    """A batch of dwarfs of different profiles in one launch per phase: each dwarf's masses and
    centres as its single-state sample gives them."""
    from milkywayathome_client_b200 import (NBodyBatch, mixed_dwarf_particle_masses,
                                            mixed_dwarf_struct)
    specs = [(3000, c) for c in PROFILE_CASES]
    dw = [mixed_dwarf_struct(n, 5 + k, _component(c[0], c[2], c[3], c[6], c[7]),
                             _component(c[1], c[4], c[5], c[6], c[7]), n // 3,
                             (10.0 * k, -3.0, 4.0), (1.0, 2.0, 3.0 * k))
          for k, (n, c) in enumerate(specs)]
    with NBodyBatch([(n, 1e-4, 1e-4, 4.0) for n, _ in specs]) as bt:
        bt.generate(dw)
        pos, vel = bt.bodies()
        offs = bt.offsets
    for k, (n, c) in enumerate(specs):
        bp, bv = pos[offs[k]:offs[k + 1]], vel[offs[k]:offs[k + 1]]
        nb = n // 3
        ml, md = mixed_dwarf_particle_masses(dw[k])
        assert np.all(np.isfinite(bp)) and np.all(np.isfinite(bv))
        np.testing.assert_allclose(bp[:nb].mean(0), (10.0 * k, -3.0, 4.0), atol=1e-9)
        np.testing.assert_allclose(bp[nb:].mean(0), (10.0 * k, -3.0, 4.0), atol=1e-9)
        np.testing.assert_allclose(bv[nb:].mean(0), (1.0, 2.0, 3.0 * k), atol=1e-9)
        assert ml > 0 and md > 0
