"""Pins of the oracle (CPU only).

1. The reference built from its own sources (oracle/_ref) reproduces the reference's golden
   end-to-end likelihoods (nbody/tests/RunTestUnits.lua) on tests/golden/orphan_dwarf.lua.
2. The C restatement (oracle/nbody_oracle.c) equals that build bit for bit: trees, forces,
   trajectories, the external potential and the correctly rounded powers.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import bits_equal, make_ctx

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def ref_or_skip():
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present; run `make -f oracle/ref.mk`")
    return ob


def golden():
    with open(os.path.join(GOLDEN, "golden_likelihoods.json")) as f:
        return json.load(f)


def test_body_layout_matches_header():
    ob = ref_or_skip()
    lay = np.zeros(8, dtype=np.int64)
    ob.ref().nbref_layout(lay.ctypes.data, 8)
    # sizeof(Body), pos, mass, type, id, vel offsets, sizeof(mwvector), sizeof(NBodyCell)
    assert list(lay[:7]) == [96, 0, 40, 48, 52, 64, 32]


@pytest.mark.parametrize("variant,seed", [("5", "670828913"), ("5", "886885833"),
                                          ("4", "715144259"), ("4", "543966758"),
                                          ("triaxial", "670828913"), ("LMC", "430281807"),
                                          ("LMC_bar", "886885833")])
def test_reference_build_reproduces_golden_likelihood(variant, seed):
    """The from-source reference reproduces RunTestUnits.lua's table (|diff| < 1e-10)."""
    ob = ref_or_skip()
    want = golden()["models"][variant]["100"][seed]
    r = ob.RefState.open_lua(os.path.join(GOLDEN, "orphan_dwarf.lua"),
                             os.path.join(GOLDEN, "orphan_model_histogram_3"), int(seed),
                             ["100", variant])
    assert r.run() == 0
    got = r.likelihood()[0]
    assert abs(got - want) < 1e-10


def test_reference_executable_golden():
    """The reference's own executable (milkyway_nbody) on the same input prints the golden."""
    ob = ref_or_skip()
    out = subprocess.run(
        [ob.REF_EXE, "--checkpoint-interval=-1", "-g", "-f", os.path.join(GOLDEN, "orphan_dwarf.lua"),
         "-h", os.path.join(GOLDEN, "orphan_model_histogram_3"), "--seed", "670828913",
         "--ignore-checkpoint", "100", "5"], capture_output=True, text=True, timeout=300,
        cwd=os.environ.get("TMPDIR", "/tmp"))
    line = [l for l in out.stderr.splitlines() + out.stdout.splitlines()
            if l.startswith("<search_likelihood>")][0]
    got = -float(line.split(">")[1].split("<")[0])
    assert abs(got - golden()["models"]["5"]["100"]["670828913"]) < 1e-10


CONFIGS = [dict(theta=0.5), dict(theta=1.0, criterion="SW93"), dict(theta=0.6, criterion="BH86"),
           dict(theta=0.0), dict(theta=0.7, useQuad=False), dict(theta=0.5, criterion="Exact")]


@pytest.mark.parametrize("cfg", CONFIGS, ids=str)
def test_oracle_equals_reference(dwarf_small, cfg):
    ob = ref_or_skip()
    pos, vel, mass, typ = dwarf_small
    ctx = make_ctx(len(mass), **cfg)
    r = ob.RefState.create(ctx.struct, pos, vel, mass, typ)
    assert r.gravmap() == 0
    want = r.get()
    rc, acc, rsize, incest = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    assert rc == 0 and rsize == want["rsize"] and bits_equal(acc, want["acc"])
    if cfg.get("criterion") != "Exact":
        rt = r.tree()
        ot = ob.tree(ctx.struct, pos, mass, ctx.treeRSize)
        assert ot["nNodes"] == rt["nNodes"] and ot["maxDepth"] == rt["maxDepth"]
        assert rt["cellUsed"] == int((ot["body"] < 0).sum())
        for k in ("next", "body", "depth"):
            assert np.array_equal(ot[k], rt[k]), k
        for k in ("pos", "mass", "rcrit2", "quad"):
            assert bits_equal(ot[k], rt[k]), k


def test_oracle_trajectory_equals_reference(dwarf_small):
    ob = ref_or_skip()
    pos, vel, mass, typ = dwarf_small
    ctx = make_ctx(len(mass), theta=0.8)
    r = ob.RefState.create(ctx.struct, pos, vel, mass, typ)
    assert r.gravmap() == 0 and r.step(15) == 0
    want = r.get()
    rc, p, v, a, rs = ob.steps(ctx.struct, pos, vel, mass, ctx.treeRSize, 15)
    assert rc == 0
    assert bits_equal(p, want["pos"]) and bits_equal(v, want["vel"]) and bits_equal(a, want["acc"])


def test_oracle_incest_and_structure_errors_match_reference():
    ob = ref_or_skip()
    rng = np.random.default_rng(3)
    pos = rng.normal(size=(300, 3))
    vel = np.zeros_like(pos)
    mass = np.ones(300)
    mass[5] = 0.0                                    # test particle: incest
    ctx = make_ctx(300, allowIncest=True)
    r = ob.RefState.create(ctx.struct, pos, vel, mass)
    rc_ref = r.gravmap()
    rc, acc, _, incest = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    assert rc == rc_ref == (1 << 24) and bits_equal(acc, r.get()["acc"])
    pos2 = pos.copy()
    pos2[9] = pos2[4]                                # coincident: structure error
    mass2 = np.ones(300)
    r2 = ob.RefState.create(ctx.struct, pos2, vel, mass2)
    assert r2.gravmap() == ob.grav_map(ctx.struct, pos2, mass2, ctx.treeRSize)[0] == (1 << 3)


def test_powers_are_correctly_rounded():
    """The double-double x^1.5 and x^3 equal crlibm's correctly rounded pow_rn."""
    ob = ref_or_skip()
    rng = np.random.default_rng(0)
    xs = np.exp(rng.uniform(np.log(1e-6), np.log(1e6), 200000))
    o, r = ob.oracle(), ob.ref()
    bad15 = [x for x in xs if o.or_pow_1p5(x) != r.nbref_pow_rn(x, 1.5)]
    bad3 = [x for x in xs if o.or_pow_3(x) != r.nbref_pow_rn(x, 3.0)]
    assert not bad15 and not bad3


def test_external_potential_equals_reference():
    ob = ref_or_skip()
    from milkywayathome_client_b200 import nbody
    rng = np.random.default_rng(2)
    pos = rng.normal(scale=25.0, size=(50000, 3))
    pos[:3] = [[0, 0, 0], [1e-3, 0, 0], [0, 0, 1e-9]]
    for pot in (nbody.milky_way_potential(),
                nbody.Potential.create(spherical=nbody.Spherical.plummer(1.52954402e5, 0.7),
                                       disk=nbody.Disk.miyamotoNagai(4.45865888e5, 6.5, 0.26),
                                       halo=nbody.Halo.logarithmic(73, 12, 1))):
        assert bits_equal(ob.ext_accel(pot, pos), ob.ref_ext_accel(pot, pos))
    nfw = nbody.Potential.create(spherical=nbody.Spherical.hernquist(1.5e5, 0.7),
                                 halo=nbody.Halo.nfw(155, 22.25))
    assert bits_equal(ob.ext_accel(nfw, pos), ob.ref_ext_accel(nfw, pos))
