"""GPU parity: the CUDA step against the oracle (the reference's algorithm restated in C,
itself pinned bit-for-bit to the reference built from its sources).

Bar: bit-exact for the tree (cell set, body-to-leaf map, counts, centres of mass, rcrit2,
quadrupoles, walk links) and for FP64 accelerations and trajectories -- the CUDA FP64 path
uses the reference's operation order without FMA contraction and correctly rounded
powers and logarithms (the NFW halo's log included).
"""
import numpy as np
import pytest

from conftest import bits_equal, make_ctx

pytestmark = pytest.mark.gpu

TREE_KEYS = ("pos", "mass", "rcrit2", "quad", "next", "body", "depth")

CONFIGS = [
    dict(theta=0.5, criterion="TreeCode", useQuad=True),
    dict(theta=1.0, criterion="TreeCode", useQuad=True),
    dict(theta=0.7, criterion="TreeCode", useQuad=False),
    dict(theta=1.0, criterion="SW93", useQuad=True),
    dict(theta=0.6, criterion="BH86", useQuad=True),
    dict(theta=0.0, criterion="TreeCode", useQuad=True),
]


def _gpu_state(ctx, pos, vel, mass):
    from milkywayathome_client_b200 import NBodyState
    return NBodyState.create(ctx, pos, vel, mass, gravmap=False)


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "%s-%g-q%d" % (c["criterion"], c["theta"], c["useQuad"]))
def test_tree_bitexact(dwarf_small, cfg):
    from oracle import bindings as ob
    pos, vel, mass, _ = dwarf_small
    ctx = make_ctx(len(mass), **cfg)
    want = ob.tree(ctx.struct, pos, mass, ctx.treeRSize)
    assert want["status"] == 0
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.makeTree(ctx) == 0
        info = st.tree_info()
        got = st.tree()
    assert info.nNodes == want["nNodes"]
    assert info.rsize == want["rsize"]
    assert info.maxDepth == want["maxDepth"]
    assert info.cellUsed == int((want["body"] < 0).sum())
    for k in TREE_KEYS:
        if k in ("next", "body", "depth"):
            assert np.array_equal(got[k], want[k]), k
        else:
            assert bits_equal(got[k], want[k]), k


@pytest.mark.parametrize("cfg", CONFIGS + [dict(theta=0.5, criterion="Exact", useQuad=False)],
                         ids=lambda c: "%s-%g-q%d" % (c["criterion"], c["theta"], c["useQuad"]))
def test_gravmap_bitexact(dwarf_small, cfg):
    from oracle import bindings as ob
    pos, vel, mass, _ = dwarf_small
    ctx = make_ctx(len(mass), **cfg)
    rc, acc, rsize, incest = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.gravMap(ctx) == rc == 0
        got = st.accels()
    assert bits_equal(got, acc)


@pytest.mark.parametrize("potential", ["none", "plummer-bulge", "nfw"])
def test_gravmap_potentials(dwarf_small, potential):
    from oracle import bindings as ob
    from milkywayathome_client_b200 import nbody
    pos, vel, mass, _ = dwarf_small
    pots = {
        "none": None,
        "plummer-bulge": nbody.Potential.create(
            spherical=nbody.Spherical.plummer(mass=1.52954402e5, scale=0.7),
            disk=nbody.Disk.miyamotoNagai(mass=4.45865888e5, scaleLength=6.5, scaleHeight=0.26),
            halo=nbody.Halo.logarithmic(vhalo=73, scaleLength=12, flattenZ=1)),
        "nfw": nbody.Potential.create(
            spherical=nbody.Spherical.hernquist(mass=1.52954402e5, scale=0.7),
            disk=nbody.Disk.miyamotoNagai(mass=4.45865888e5, scaleLength=6.5, scaleHeight=0.26),
            halo=nbody.Halo.nfw(vhalo=155, scaleLength=22.25)),
    }
    ctx = make_ctx(len(mass), potential=pots[potential])
    rc, acc, _, _ = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.gravMap(ctx) == rc == 0
        got = st.accels()
    assert bits_equal(got, acc)


def test_steps_bitexact(dwarf_small):
    """20 kick-drift-kick steps: positions, velocities and accelerations stay bit-exact."""
    from oracle import bindings as ob
    pos, vel, mass, _ = dwarf_small
    ctx = make_ctx(len(mass), theta=0.7)
    rc, p_want, v_want, a_want, rs = ob.steps(ctx.struct, pos, vel, mass, ctx.treeRSize, 20)
    assert rc == 0
    from milkywayathome_client_b200 import NBodyState
    with NBodyState.create(ctx, pos, vel, mass) as st:
        assert st.run_steps(ctx, 20) == 0
        p, v = st.bodies()
        a = st.accels()
        assert st.step_count == 20
        assert st.tree_info().rsize == rs
    assert bits_equal(p, p_want) and bits_equal(v, v_want) and bits_equal(a, a_want)


def test_larger_dwarf_bitexact():
    """40,000 bodies (deeper tree, long equal-key runs in the sort): accelerations bit-exact."""
    from oracle import bindings as ob
    from milkywayathome_client_b200 import models
    pos, vel, mass, _ = models.plummer_plummer_dwarf(40000, seed=5)
    ctx = make_ctx(len(mass), theta=0.5)
    rc, acc, _, _ = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.gravMap(ctx) == rc == 0
        assert bits_equal(st.accels(), acc)


def test_against_reference_build(dwarf_small):
    """Directly against the reference's own nbGravMap / nbStepSystem (compiled from its sources)."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    pos, vel, mass, typ = dwarf_small
    ctx = make_ctx(len(mass), theta=1.0, criterion="SW93")
    r = ob.RefState.create(ctx.struct, pos, vel, mass, typ)
    assert r.gravmap() == 0
    assert r.step(10) == 0
    want = r.get()
    from milkywayathome_client_b200 import NBodyState
    with NBodyState.create(ctx, pos, vel, mass) as st:
        assert st.run_steps(ctx, 10) == 0
        p, v = st.bodies()
        a = st.accels()
    assert bits_equal(p, want["pos"]) and bits_equal(v, want["vel"]) and bits_equal(a, want["acc"])


# ---- edge cases the reference's tree code has ----
def test_massless_bodies_are_not_in_the_tree():
    """Test particles (mass 0) are skipped by nbMakeTree (nbody_tree.c:440); they still get
    forces, never meet themselves in the walk, and so raise tree incest."""
    from oracle import bindings as ob
    from milkywayathome_client_b200 import models, NBodyState
    pos, vel, mass, _ = models.plummer_plummer_dwarf(1000, seed=2)
    mass = mass.copy()
    mass[::7] = 0.0
    ctx = make_ctx(len(mass), theta=0.6, allowIncest=True)
    rc, acc, _, incest = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    assert incest == 1 and rc == (1 << 24)
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.gravMap(ctx) == rc
        assert st.tree_info().nTreeBodies == int((mass != 0).sum())
        assert bits_equal(st.accels(), acc)
    ctx_fatal = make_ctx(len(mass), theta=0.6, allowIncest=False)
    with _gpu_state(ctx_fatal, pos, vel, mass) as st:
        assert st.gravMap(ctx_fatal) == (1 << 4)        # NBODY_TREE_INCEST_FATAL


@pytest.mark.parametrize("n", [1, 2, 3, 33])
def test_tiny_systems(n):
    from oracle import bindings as ob
    rng = np.random.default_rng(n)
    pos = rng.normal(size=(n, 3))
    vel = rng.normal(size=(n, 3))
    mass = rng.uniform(0.5, 1.5, n)
    ctx = make_ctx(max(n, 2), theta=0.8)
    want = ob.tree(ctx.struct, pos, mass, ctx.treeRSize)
    rc, acc, _, _ = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.gravMap(ctx) == rc
        got = st.tree()
        assert st.tree_info().nNodes == want["nNodes"]
        for k in TREE_KEYS:
            assert np.array_equal(got[k], want[k]), k
        assert bits_equal(st.accels(), acc)


def test_coincident_bodies_structure_error():
    """Two bodies at the same point cannot be separated: NBODY_TREE_STRUCTURE_ERROR
    (nbLoadBody's qsize <= REAL_EPSILON check, nbody_tree.c:256-264)."""
    from oracle import bindings as ob
    rng = np.random.default_rng(0)
    pos = rng.normal(size=(50, 3))
    pos[17] = pos[3]
    vel = np.zeros_like(pos)
    mass = np.ones(50)
    ctx = make_ctx(50)
    rc, _, _, _ = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    assert rc == (1 << 3)
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.gravMap(ctx) == rc


def test_deep_chain_grows_node_storage():
    """Pairs that part only ~40 levels down create long chains of single-child cells; the
    node arrays (sized 2N+64 up front) grow and the build is redone transparently."""
    from oracle import bindings as ob
    rng = np.random.default_rng(4)
    base = rng.normal(size=(6, 3))
    pos = np.concatenate([base, base + 1e-11])
    vel = np.zeros_like(pos)
    mass = np.ones(len(pos))
    ctx = make_ctx(len(pos), theta=0.5)
    want = ob.tree(ctx.struct, pos, mass, ctx.treeRSize)
    assert want["status"] == 0 and want["nNodes"] > 2 * len(pos) + 64
    rc, acc, _, _ = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.gravMap(ctx) == rc == 0
        got = st.tree()
        for k in TREE_KEYS:
            assert np.array_equal(got[k], want[k]), k
        assert bits_equal(st.accels(), acc)


def test_root_size_grows_and_persists():
    """expandBox only ever doubles t->rsize (nbody_tree.c:172-175): a body flung far out grows
    the root, and the root stays large when it comes back."""
    from oracle import bindings as ob
    rng = np.random.default_rng(9)
    pos = rng.normal(size=(200, 3))
    vel = np.zeros_like(pos)
    mass = np.ones(200)
    ctx = make_ctx(200)
    far = pos.copy()
    far[0] = [300.0, 0.0, 0.0]
    with _gpu_state(ctx, far, vel, mass) as st:
        assert st.gravMap(ctx) == 0
        assert st.tree_info().rsize == 1024.0
        st.set_bodies(pos, vel, mass, 1024.0)
        assert st.gravMap(ctx) == 0
        rc, acc, rs, _ = ob.grav_map(ctx.struct, pos, mass, 1024.0)
        assert rs == 1024.0 and bits_equal(st.accels(), acc)


def test_ext_acceleration_bitexact():
    from oracle import bindings as ob
    from milkywayathome_client_b200 import ext_acceleration, nbody
    rng = np.random.default_rng(1)
    pos = rng.normal(scale=20.0, size=(20000, 3))
    pos[:5] = [[0, 0, 0], [1e-3, 0, 0], [0, 0, 2e-3], [300, -200, 100], [1e-9, 1e-9, 1e-9]]
    for pot in (nbody.milky_way_potential(),
                nbody.Potential.create(spherical=nbody.Spherical.plummer(1.5e5, 0.7),
                                       disk=nbody.Disk.miyamotoNagai(4.4e5, 6.5, 0.26),
                                       disk2=nbody.Disk.miyamotoNagai(1e5, 3.0, 0.5))):
        assert bits_equal(ext_acceleration(pot, pos), ob.ext_accel(pot, pos))


def test_marshal_reference_body_records(dwarf_small):
    """nbMarshalBodiesCUDA reads and writes the reference's 96-byte Body records."""
    from milkywayathome_client_b200 import NBodyState
    pos, vel, mass, typ = dwarf_small
    n = len(mass)
    rec = np.zeros(n, dtype=[("pos", "f8", 4), ("next", "u8"), ("mass", "f8"), ("type", "i2"),
                             ("pad", "i2"), ("id", "u4"), ("pad2", "u8"), ("vel", "f8", 4)])
    assert rec.itemsize == 96
    rec["pos"][:, :3] = pos
    rec["vel"][:, :3] = vel
    rec["mass"] = mass
    rec["type"] = typ
    rec["id"] = np.arange(n)
    ctx = make_ctx(n)
    with NBodyState(n) as st:
        st.marshal_bodies(rec, to_device=True, treeRSize=4.0)
        p, v = st.bodies()
        assert bits_equal(p, pos) and bits_equal(v, vel)
        assert st.step(ctx) == 0
        p2, v2 = st.bodies()
        st.marshal_bodies(rec, to_device=False)
    assert bits_equal(rec["pos"][:, :3], p2) and bits_equal(rec["vel"][:, :3], v2)
    assert np.array_equal(rec["id"], np.arange(n)) and bits_equal(rec["mass"], mass)


def test_mixed_precision_error_vs_direct_summation(dwarf_small):
    """The mixed form (FP32 group walk, FP64 accumulation).  In its default exact-set mode every
    body takes exactly the cells and bodies of its own opening test, so its accelerations are
    the FP64 walk's up to FP32 rounding and its error against FP64 direct summation equals the
    FP64 walk's at every percentile (within 1 %, max included).  In the group mode every body
    takes its group's set: never coarser per cell, but the accepted shell is no longer
    symmetric about each body, so the median drops while the tail may grow (bounded)."""
    from milkywayathome_client_b200 import NBodyState
    pos, vel, mass, _ = dwarf_small
    ctx = make_ctx(len(mass), theta=0.5, potential=None)
    ctxm = ctx.with_precision("mixed")
    with _gpu_state(ctx, pos, vel, mass) as st:
        direct = st.direct_sample(ctx.eps2, np.arange(len(mass)))
        assert st.gravMap(ctx) == 0
        a64 = st.accels()
        assert st.gravMap(ctxm) == 0
        a32 = st.accels()
        st.set_mixed_mode(False)
        assert st.gravMap(ctxm) == 0
        ag = st.accels()
    norm = np.linalg.norm(direct, axis=1)
    e64 = np.linalg.norm(a64 - direct, axis=1) / norm
    e32 = np.linalg.norm(a32 - direct, axis=1) / norm
    eg = np.linalg.norm(ag - direct, axis=1) / norm
    # exact sets: the FP64 walk's accelerations up to FP32 rounding, body by body
    assert np.max(np.linalg.norm(a32 - a64, axis=1) / norm) < 1e-5
    for q in (50, 90, 99, 100):
        assert np.percentile(e32, q) <= 1.01 * np.percentile(e64, q), q
    # group mode: a lower median, a bounded tail
    assert np.percentile(eg, 50) <= np.percentile(e64, 50)
    assert eg.max() < 3e-2


def test_mixed_precision_step_runs_and_stays_close(dwarf_small):
    """Ten mixed-precision steps track the FP64 trajectory closely (positions within 1e-5
    of the dwarf's size after ten steps: the two forms differ by the Barnes-Hut error, not
    by a systematic drift)."""
    from milkywayathome_client_b200 import NBodyState
    pos, vel, mass, _ = dwarf_small
    ctx = make_ctx(len(mass), theta=0.5)
    ctxm = ctx.with_precision("mixed")
    with NBodyState.create(ctx, pos, vel, mass) as s64, NBodyState.create(ctxm, pos, vel, mass) as s32:
        assert s64.run_steps(ctx, 10) == 0
        assert s32.run_steps(ctxm, 10) == 0
        p64, _ = s64.bodies()
        p32, _ = s32.bodies()
    scale = np.abs(pos - pos.mean(0)).max()
    assert np.abs(p32 - p64).max() < 1e-5 * scale


def test_mixed_flags_test_particles_as_incest():
    from milkywayathome_client_b200 import models
    pos, vel, mass, _ = models.plummer_plummer_dwarf(1000, seed=2)
    mass = mass.copy()
    mass[::9] = 0.0
    ctx = make_ctx(len(mass), theta=0.6, allowIncest=True, precision="mixed")
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.gravMap(ctx) == (1 << 24)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_graph_equals_direct_launches(dwarf_small, precision):
    """Whole steps are replayed as one captured CUDA graph by default (nbSetStepGraphCUDA); the
    same steps launched kernel by kernel give the same bodies and accelerations bit for bit."""
    from milkywayathome_client_b200 import NBodyState
    pos, vel, mass, _ = dwarf_small
    ctx = make_ctx(len(mass), theta=0.7, precision=precision)
    with NBodyState.create(ctx, pos, vel, mass) as a, NBodyState.create(ctx, pos, vel, mass) as b:
        b.set_step_graph(False)
        for k in range(8):
            assert a.step(ctx) == 0 and b.step(ctx) == 0
        assert a.run_steps(ctx, 5) == 0 and b.run_steps(ctx, 5) == 0
        pa, va = a.bodies()
        pb, vb = b.bodies()
        assert bits_equal(pa, pb) and bits_equal(va, vb) and bits_equal(a.accels(), b.accels())
        assert a.step_count == b.step_count == 13


@pytest.mark.parametrize("cfg", [dict(theta=0.5, criterion="TreeCode", useQuad=True),
                                 dict(theta=1.0, criterion="SW93", useQuad=True),
                                 dict(theta=0.7, criterion="TreeCode", useQuad=False)],
                         ids=lambda c: "%s-%g-q%d" % (c["criterion"], c["theta"], c["useQuad"]))
def test_union_and_per_lane_walks_are_bit_equal(dwarf_small, cfg):
    """The FP64 walk's forms (nbSetWalkFormCUDA): the warp-union walk, the per-lane walk with
    and without the early load of the next record, and the automatic choice among them all give
    each body its CPU walk -- the oracle's accelerations bit for bit, and the same interaction
    counts."""
    from oracle import bindings as ob
    pos, vel, mass, _ = dwarf_small
    ctx = make_ctx(len(mass), **cfg)
    rc, acc, _, _, cnt = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize, counts=True)
    steps = {}
    for form in (0, 1, 2):
        with _gpu_state(ctx, pos, vel, mass) as st:
            st.set_walk_form(form)
            st.set_counting(True)
            assert st.gravMap(ctx) == rc == 0
            stats = st.walk_stats()
            assert bits_equal(st.accels(), acc), form
            assert tuple(stats[:3]) == tuple(cnt), form
            steps[form] = stats[3]
            assert st.walk_form() == form
    # the per-lane walks run fewer warp iterations than the union walk
    assert steps[1] == steps[2] < steps[0]
    # automatic: the first six evaluations cycle twice through the forms, then one is kept
    with _gpu_state(ctx, pos, vel, mass) as st:
        assert st.walk_form() == -1
        for _ in range(7):
            assert st.gravMap(ctx) == 0
            assert bits_equal(st.accels(), acc)
        assert st.walk_form() in (0, 1, 2)


@pytest.mark.parametrize("form", [0, 1, 2])
def test_negative_mass_bodies(dwarf_small, form):
    """Bodies of negative mass (nothing in the reference forbids them): the tree, its moments
    and both walk forms still give the oracle's status and accelerations bit for bit."""
    from oracle import bindings as ob
    pos, vel, mass, _ = dwarf_small
    mass = mass.copy()
    mass[::97] *= -0.5
    ctx = make_ctx(len(mass), theta=0.6, allowIncest=True)
    rc, acc, _, _ = ob.grav_map(ctx.struct, pos, mass, ctx.treeRSize)
    with _gpu_state(ctx, pos, vel, mass) as st:
        st.set_walk_form(form)
        assert st.gravMap(ctx) == rc
        if rc == 0:
            assert bits_equal(st.accels(), acc)
