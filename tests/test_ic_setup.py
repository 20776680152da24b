"""The dwarf sampler's per-component set-up on the host (no GPU): the particle masses that
nbMixedDwarfParticleMassesCUDA reports -- after the NFW and cored components' mass reset to
the mass inside the sampling bound 5 r200 (get_extra_nfw_mass, nbody/src/nbody_mixeddwarf.c:
728-762) -- equal the masses the reference's own sampler gives its bodies (oracle/_ref through
tests/golden/two_component_dwarf.lua), bit for bit."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASES = [("plummer", "plummer", 12.0, 0.2, 48.0, 0.8, 0.0, 0.0),
         ("plummer", "nfw", 12.0, 0.2, 40.0, 0.8, 0.0, 0.0),
         ("nfw", "nfw", 5.0, 0.3, 60.0, 1.5, 0.0, 0.0),
         ("plummer", "general_hernquist", 12.0, 0.2, 48.0, 0.8, 0.0, 0.0),
         ("plummer", "cored", 12.0, 0.2, 40.0, 0.8, 0.3, 0.2),
         ("cored", "cored", 8.0, 0.5, 40.0, 0.8, 1.5, 0.4)]


def _component(kind, mass, scale, r1, rc):
    from milkywayathome_client_b200 import Dwarf
    if kind == "cored":
        return Dwarf.cored(mass, scale, r1, rc)
    return getattr(Dwarf, kind)(mass, scale)


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0] + "-" + c[1])
def test_particle_masses_equal_reference(case):
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    from milkywayathome_client_b200 import mixed_dwarf_particle_masses, mixed_dwarf_struct
    tl, td, ml, al, md, ad, r1, rc = case
    n, nb = 200, 80
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "two_component_dwarf.lua"), None, 9,
                             [str(n), str(nb), repr(ml), repr(al), repr(md), repr(ad), tl, td,
                              repr(r1), repr(rc)])
    mass, types = r.masses()
    d = mixed_dwarf_struct(n, 1, _component(tl, ml, al, r1, rc), _component(td, md, ad, r1, rc), nb)
    light, dark = mixed_dwarf_particle_masses(d)
    assert np.all(mass[:nb] == light) and np.all(mass[nb:] == dark)
    assert np.all(types[:nb] == 1) and np.all(types[nb:] == -1)


def test_invalid_components_rejected():
    from milkywayathome_client_b200 import (Dwarf, NBodyError, mixed_dwarf_particle_masses,
                                            mixed_dwarf_struct)
    bad = [Dwarf.nfw(0.0, 1.0), Dwarf.cored(10.0, 1.0, 0.0, 0.2), Dwarf.plummer(1.0, 0.0)]
    for comp in bad:
        with pytest.raises(NBodyError):
            mixed_dwarf_particle_masses(mixed_dwarf_struct(10, 1, Dwarf.plummer(1.0, 0.2), comp))
    einasto = Dwarf._make(3, 1.0, 1.0)
    with pytest.raises(NBodyError):
        mixed_dwarf_particle_masses(mixed_dwarf_struct(10, 1, einasto, Dwarf.plummer(1.0, 0.2)))
