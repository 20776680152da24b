"""Batched dwarfs (nbBatch*CUDA): every dwarf of a batch must evolve exactly as it does alone.

The FP64 batch is compared bit for bit with single-dwarf NBodyState runs of the same dwarfs
(gravMap, then steps through a captured graph and without one); the mixed batch against the
single-dwarf mixed form.  The dwarfs differ in size (sizes not multiples of 32, so warps
straddle dwarf boundaries), parameters, softening and time step, and sit at different
distances from the origin, so their root sizes differ.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch_dwarfs():
    from milkywayathome_client_b200 import models
    specs = [  # nbody, baryon mass, baryon radius, radius ratio, mass ratio, centre
        (3001, 12.0, 0.2, 0.2, 0.2, (-21.6, -10.4, 23.2)),
        (4096, 30.0, 0.3, 0.4, 0.5, (5.0, 3.0, -2.0)),
        (2050, 3.0, 0.15, 0.25, 0.05, (60.0, -40.0, 10.0)),
        (6143, 80.0, 0.45, 0.15, 0.9, (-1.0, 0.5, 0.25)),
        (37, 1.0, 0.1, 0.5, 0.5, (0.0, 0.0, 120.0)),
    ]
    out = []
    for k, (n, m, r, rr, mr, c) in enumerate(specs):
        pos, vel, mass, _ = models.plummer_plummer_dwarf(n, seed=100 + k, mass_l=m, rscale_l=r,
                                                        light_r_ratio=rr, light_mass_ratio=mr)
        pos = pos + np.asarray(c)
        cfg = models.dwarf_config(n, theta=0.5, mass_l=m, rscale_l=r, light_r_ratio=rr,
                                  light_mass_ratio=mr)
        out.append((pos, vel, mass, cfg))
    return out


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64),
                          np.ascontiguousarray(b).view(np.uint64))


def _run_single(pot, dwarfs, precision, steps):
    from milkywayathome_client_b200 import NBodyCtx, NBodyState
    res = []
    for pos, vel, mass, cfg in dwarfs:
        ctx = NBodyCtx(potential=pot, precision=precision, **cfg)
        with NBodyState.create(ctx, pos, vel, mass) as st:
            a0 = st.accels()
            st.check("nbRunSteps", st.run_steps(ctx, steps))
            p, v = st.bodies()
            res.append((a0, p, v, st.accels(), st.tree_info().rsize))
    return res


def _run_batch(pot, dwarfs, precision, steps, graph, walk_form=0):
    from milkywayathome_client_b200 import NBodyBatch, NBodyCtx
    cfg0 = dwarfs[0][3]
    ctx = NBodyCtx(potential=pot, precision=precision, **cfg0)
    spec = [(len(m), cfg["eps2"], cfg["timestep"], 4.0) for _, _, m, cfg in dwarfs]
    with NBodyBatch(spec) as bt:
        if walk_form:
            bt.set_walk_form(walk_form)
        bt.set_bodies(np.concatenate([d[0] for d in dwarfs]), np.concatenate([d[1] for d in dwarfs]),
                      np.concatenate([d[2] for d in dwarfs]))
        bt.check("nbBatchGravMap", bt.gravMap(ctx))
        a0 = bt.accels()
        bt.check("nbBatchRunSteps", bt.run_steps(ctx, steps, graph=graph))
        p, v = bt.bodies()
        a1 = bt.accels()
        status, rsize, root, nodes = bt.dwarf_info()
        offs = bt.offsets
    out = []
    for k in range(len(dwarfs)):
        s = slice(offs[k], offs[k + 1])
        out.append((a0[s], p[s], v[s], a1[s], rsize[k]))
    return out, status, root, nodes


@pytest.mark.parametrize("graph,walk_form", [(False, 0), (True, 0), (False, 1), (True, 1),
                                             (True, 2)])
def test_fp64_batch_matches_single_dwarfs_bit_for_bit(graph, walk_form):
    """Every FP64 walk form; with the walks per lane a warp that spans two dwarfs has each lane
    walk its own dwarf's tree."""
    from milkywayathome_client_b200 import milky_way_potential
    dwarfs = _batch_dwarfs()
    pot = milky_way_potential()
    want = _run_single(pot, dwarfs, "fp64", 4)
    got, status, root, nodes = _run_batch(pot, dwarfs, "fp64", 4, graph, walk_form)
    assert np.all(status == 0)
    assert root[0] == 0 and np.all(np.diff(root) == nodes[:-1])
    for k, (w, g) in enumerate(zip(want, got)):
        for name, a, b in zip(("a0", "pos", "vel", "a4"), w[:4], g[:4]):
            assert _same(a, b), (k, name, np.abs(a - b).max())
        assert w[4] == g[4]


def test_mixed_batch_matches_single_dwarfs():
    from milkywayathome_client_b200 import milky_way_potential
    dwarfs = _batch_dwarfs()
    pot = milky_way_potential()
    want = _run_single(pot, dwarfs, "mixed", 3)
    got, status, _, _ = _run_batch(pot, dwarfs, "mixed", 3, True)
    assert np.all(status == 0)
    for k, (w, g) in enumerate(zip(want, got)):
        for name, a, b in zip(("a0", "pos", "vel", "a3"), w[:4], g[:4]):
            scale = np.abs(a).max()
            assert np.abs(a - b).max() <= 1e-12 * scale, (k, name, np.abs(a - b).max() / scale)


def test_batch_rejects_bad_input():
    from milkywayathome_client_b200 import NBodyBatch, NBodyError
    with pytest.raises(NBodyError):
        NBodyBatch([(1, 1e-3, 1e-3, 4.0)])                 # a dwarf needs >= 2 bodies
    with pytest.raises(NBodyError):
        NBodyBatch([(10, 1e-3, 1e-3, 3.0)])                # root size not a power of two
    with NBodyBatch([(4, 1e-3, 1e-3, 4.0)]) as bt:
        with pytest.raises(NBodyError):                    # massless bodies
            bt.set_bodies(np.zeros((4, 3)), np.zeros((4, 3)), np.array([1.0, 0.0, 1.0, 1.0]))


def test_autotune_picks_a_candidate_and_leaves_its_accelerations():
    from milkywayathome_client_b200 import NBodyBatch, NBodyCtx, milky_way_potential
    dwarfs = _batch_dwarfs()
    ctx = NBodyCtx(potential=milky_way_potential(), precision="mixed", **dwarfs[0][3])
    spec = [(len(m), cfg["eps2"], cfg["timestep"], 4.0) for _, _, m, cfg in dwarfs]
    cat = lambda k: np.concatenate([d[k] for d in dwarfs])
    with NBodyBatch(spec) as bt:
        bt.set_bodies(cat(0), cat(1), cat(2))
        bt.check("nbBatchGravMap", bt.gravMap(ctx))
        g, l, b, ms = bt.autotune(ctx)
        assert g in (24, 32, 48, 64) and l in (32, 64, 128) and b in (0, 3) and ms > 0
        assert bt.tuning() == (g, l, b)
        tuned = bt.accels()
        pos0, _ = bt.bodies()
    assert _same(pos0, cat(0))                      # the autotuner does not move the bodies
    with NBodyBatch(spec) as bt2:
        bt2.set_bodies(cat(0), cat(1), cat(2))
        bt2.set_tuning(g, l, b)
        bt2.check("nbBatchGravMap", bt2.gravMap(ctx))
        assert _same(bt2.accels(), tuned)
