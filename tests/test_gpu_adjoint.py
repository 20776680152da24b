"""The adjoint of the step (no reference counterpart), checked three ways on the GPU:

1. nbGravVJPCUDA against central differences of nbGravMapCUDA's accelerations
   (directional derivative, tree frozen by a small enough step);
2. a 50-step run of 2,048 bodies with the Exact criterion against FP64 direct summation
   differentiated by torch autograd (same arithmetic, so agreement to rounding);
3. the full parameters -> soft-histogram loss (6 dwarf + 6 orbit parameters) with the tree
   (TreeCode, quadrupoles) against central finite differences of the GPU forward (relative
   step 1e-6) and against the direct-summation autograd reference.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ctx(n, criterion="TreeCode", theta=0.5, potential=True):
    from milkywayathome_client_b200 import NBodyCtx, milky_way_potential, models
    cfg = models.dwarf_config(n, theta=theta, criterion=criterion)
    return NBodyCtx(potential=milky_way_potential() if potential else None, **cfg)


def _dwarf(n, seed=3):
    from milkywayathome_client_b200 import models
    pos, vel, mass, _ = models.plummer_plummer_dwarf(n, seed=seed)
    dev = torch.device("cuda:0")
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    return t(pos), t(vel), t(mass)


@pytest.mark.parametrize("criterion", ["TreeCode", "SW93", "Exact"])
def test_force_vjp_matches_central_differences(criterion):
    from milkywayathome_client_b200.adjoint import DeviceState
    n = 2048
    x, v, m = _dwarf(n)
    ctx = _ctx(n, criterion=criterion)
    ds = DeviceState(n, x.device)
    g = torch.Generator(device="cpu").manual_seed(0)
    abar = torch.randn((n, 3), generator=g, dtype=torch.float64).to(x.device)
    d = torch.randn((n, 3), generator=g, dtype=torch.float64).to(x.device)
    ds.set(x, v, m, ctx.treeRSize)
    ds.gravmap(ctx)
    xbar, mbar = ds.vjp(ctx, abar)
    eps = 1e-7
    vals = []
    for sgn in (1.0, -1.0):
        ds.set(x + sgn * eps * d, v, m, ctx.treeRSize)
        ds.gravmap(ctx)
        vals.append(ds.get()[2])
    fd = ((vals[0] - vals[1]) * abar).sum().item() / (2 * eps)
    ad = (xbar * d).sum().item()
    assert abs(fd - ad) <= 1e-5 * abs(ad)
    # mass direction
    dm = torch.rand(n, generator=g, dtype=torch.float64).to(x.device) * m
    vals = []
    for sgn in (1.0, -1.0):
        ds.set(x, v, m + sgn * 1e-6 * dm, ctx.treeRSize)
        ds.gravmap(ctx)
        vals.append(ds.get()[2])
    fd_m = ((vals[0] - vals[1]) * abar).sum().item() / (2e-6)
    ad_m = (mbar * dm).sum().item()
    assert abs(fd_m - ad_m) <= 1e-5 * abs(ad_m)
    ds.close()


def test_exact_run_gradient_matches_direct_sum_autograd():
    from milkywayathome_client_b200 import adjoint
    n, steps = 2048, 50
    ctx = _ctx(n, criterion="Exact")
    x0, v0, m = _dwarf(n, seed=5)
    dt0 = torch.tensor(ctx.timestep, dtype=torch.float64, device=x0.device)
    g = torch.Generator(device="cpu").manual_seed(1)
    wx = torch.randn((n, 3), generator=g, dtype=torch.float64).to(x0.device)
    wv = torch.randn((n, 3), generator=g, dtype=torch.float64).to(x0.device)

    def loss_of(fwd):
        xs, vs, ms, dts = (t.clone().requires_grad_(True) for t in (x0, v0, m, dt0))
        xN, vN = fwd(xs, vs, ms, dts)
        L = (xN * wx).sum() + 1e-2 * (vN * wv).sum()
        L.backward()
        return L.item(), [t.grad for t in (xs, vs, ms, dts)]

    L_gpu, g_gpu = loss_of(lambda x, v, mm, dt: adjoint.run(ctx, x, v, mm, dt, steps, every=16))
    L_ref, g_ref = loss_of(lambda x, v, mm, dt: adjoint.direct_run_torch(
        x, v, mm, dt, steps, ctx.eps2, ctx.struct.pot))
    assert abs(L_gpu - L_ref) <= 1e-10 * abs(L_ref)
    for a, b in zip(g_gpu, g_ref):
        err = (a - b).abs().max().item()
        assert err <= 1e-8 * b.abs().max().item()


def test_parameter_gradients_tree_vs_fd_and_direct():
    from milkywayathome_client_b200 import adjoint
    n, steps = 2048, 50
    dev = torch.device("cuda:0")
    ctx = _ctx(n, criterion="TreeCode", theta=0.5)
    draws = adjoint.DwarfDraws(n, seed=7, device=dev)
    params = torch.tensor([0.025, 4.0, 0.2, 0.2, 12.0, 0.2], dtype=torch.float64, device=dev)
    orbit = torch.tensor([218.0, 53.5, 28.6, -156.0, 79.0, 107.0], dtype=torch.float64, device=dev)
    target = adjoint.model_histogram(ctx, params * 1.05, orbit, draws, steps).detach()

    def loss(p, o, forward=None):
        h = adjoint.model_histogram(ctx, p, o, draws, steps, every=16, forward=forward)
        return ((h - target) ** 2).sum()

    p = params.clone().requires_grad_(True)
    o = orbit.clone().requires_grad_(True)
    L = loss(p, o)
    L.backward()
    grad = torch.cat([p.grad, o.grad]).cpu().numpy()

    # central finite differences of the GPU forward, relative step 1e-6
    fd = np.zeros(12)
    base = torch.cat([params, orbit])
    with torch.no_grad():
        for k in range(12):
            step = 1e-6 * abs(base[k].item())
            vals = []
            for sgn in (1.0, -1.0):
                b = base.clone()
                b[k] += sgn * step
                vals.append(loss(b[:6], b[6:]).item())
            fd[k] = (vals[0] - vals[1]) / (2 * step)
    scale = np.abs(fd).max()
    assert np.all(np.abs(grad - fd) <= 2e-3 * scale + 1e-3 * np.abs(fd)), (grad, fd)

    # FP64 direct summation through torch autograd (a different force approximation: the
    # tree's gradients agree with it to the Barnes-Hut error level)
    p2 = params.clone().requires_grad_(True)
    o2 = orbit.clone().requires_grad_(True)
    L2 = loss(p2, o2, forward=lambda x0, v0, m, dt: adjoint.direct_run_torch(
        x0, v0, m, dt, steps, ctx.eps2, ctx.struct.pot))
    L2.backward()
    grad_ref = torch.cat([p2.grad, o2.grad]).cpu().numpy()
    assert np.abs(grad - grad_ref).max() <= 5e-2 * np.abs(grad_ref).max()


def test_saved_state_restores_bodies_and_tree():
    """nbRestoreStateCUDA brings back a saved evaluation exactly: bodies bit for bit, and the
    force VJP on the restored tree equals the one taken right after the evaluation (up to the
    order of the node-adjoint atomics)."""
    from milkywayathome_client_b200.adjoint import DeviceState
    n = 4096
    x, v, m = _dwarf(n, seed=9)
    ctx = _ctx(n)
    ds = DeviceState(n, x.device)
    ds.set(x, v, m, ctx.treeRSize)
    ds.gravmap(ctx)
    ds.step(ctx)
    saved = ds.get()
    info = ds.st.tree_info()
    ds.save(3)
    abar = torch.randn((n, 3), dtype=torch.float64, device=x.device,
                       generator=torch.Generator(device=x.device).manual_seed(2))
    gx_a, gm_a = ds.vjp(ctx, abar)
    for _ in range(3):
        ds.step(ctx)
    ds.restore(3)
    for a, b in zip(saved, ds.get()):
        assert torch.equal(a, b)
    assert ds.st.tree_info().nNodes == info.nNodes
    gx_b, gm_b = ds.vjp(ctx, abar)
    assert torch.allclose(gx_a, gx_b, rtol=1e-12, atol=1e-12 * gx_a.abs().max().item())
    assert torch.allclose(gm_a, gm_b, rtol=1e-12, atol=1e-12 * gm_a.abs().max().item())
    with pytest.raises(Exception):
        ds.restore(7)
    ds.close()
