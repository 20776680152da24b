"""Differentiable N-body runs: a torch.autograd.Function over the CUDA step and its adjoint.

No counterpart in the reference (it has no adjoint).  The forward pass runs nsteps
kick-drift-kick steps of the FP64 drop-in step on the GPU (nbStepSystemCUDA), keeping a
checkpoint (positions, velocities, root size) every K steps.  The backward pass walks the
segments in reverse: it recomputes the states of one segment from its checkpoint, saving
each state's bodies and tree in HBM (nbSaveStateCUDA), then runs the reverse leapfrog step
by step on the device (nbRestoreStateCUDA + nbStepAdjointCUDA: the vector-Jacobian product
of the forces with that state's tree frozen -- tidal tensor of the walk, the cells' moment
adjoints, the external potential's Jacobian -- and the reverse kicks and drift).

Around it, torch code that is differentiable end to end:
  * dwarf_ics       -- a seeded two-component Plummer dwarf as a function of the 6 dwarf
                       parameters (fixed random draws, reparameterised);
  * reverse_orbit   -- the reference's reverse orbit integration (nbReverseOrbit,
                       nbody/src/nbody_orbit_integrator.c:44-86) of the 6 orbit coordinates;
  * lambda_beta     -- nbXYZToLambdaBeta (nbody/src/nbody_coordinates.c:129-164);
  * soft_histogram  -- Gaussian-kernel soft binning of the baryons in (Lambda, Beta).
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from .models import PI_4_3, SUN_GC_DIST
from .nbody import NBodyCtx, NBodyError, NBodyState, status_is_fatal

DWARF_PARAMS = ("t_forward", "time_ratio", "r_baryon", "radius_ratio", "m_baryon", "mass_ratio")
ORBIT_PARAMS = ("l", "b", "r", "vx", "vy", "vz")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _sync():
    torch.cuda.current_stream().synchronize()


class DeviceState:
    """An NBodyState fed from and read into device torch tensors (float64, (n,3) / (n,))."""

    def __init__(self, n, device):
        self.st = NBodyState(n, device.index if device.index is not None else 0)
        self.lib = self.st.lib
        self.n = n
        self.device = device

    def close(self):
        self.st.close()

    def set(self, x, v, m, rsize):
        _sync()
        rc = self.lib.nbSetBodiesDeviceCUDA(self.st._h, _ptr(x), _ptr(v), _ptr(m), self.n, float(rsize))
        NBodyState.check("nbSetBodiesDeviceCUDA", rc)

    def get(self):
        x = torch.empty((self.n, 3), dtype=torch.float64, device=self.device)
        v = torch.empty_like(x)
        a = torch.empty_like(x)
        rc = self.lib.nbGetBodiesDeviceCUDA(self.st._h, _ptr(x), _ptr(v), _ptr(a))
        NBodyState.check("nbGetBodiesDeviceCUDA", rc)
        return x, v, a

    def rsize(self):
        return self.st.tree_info().rsize

    def gravmap(self, ctx):
        return NBodyState.check("nbGravMap", self.st.gravMap(ctx))

    def step(self, ctx):
        return NBodyState.check("nbStepSystem", self.st.step(ctx))

    def maketree(self, ctx):
        """Rebuild the tree at the current positions (nothing to build for Exact)."""
        if ctx.criterion == _lib.EXACT:
            return 0
        return NBodyState.check("nbMakeTree", self.st.makeTree(ctx))

    def accel(self):
        a = torch.empty((self.n, 3), dtype=torch.float64, device=self.device)
        rc = self.lib.nbGetBodiesDeviceCUDA(self.st._h, None, None, _ptr(a))
        NBodyState.check("nbGetBodiesDeviceCUDA", rc)
        return a

    def save(self, slot):
        NBodyState.check("nbSaveStateCUDA", self.lib.nbSaveStateCUDA(self.st._h, slot))

    def restore(self, slot):
        NBodyState.check("nbRestoreStateCUDA", self.lib.nbRestoreStateCUDA(self.st._h, slot))

    def step_adjoint(self, ctx, ak, xbar, vbar, mbar, abar_next, dtbar):
        """Reverse of the step whose end state is current (nbStepAdjointCUDA); updates the
        adjoint tensors in place."""
        _sync()
        rc = self.lib.nbStepAdjointCUDA(ctypes.byref(ctx.struct), self.st._h, _ptr(ak), _ptr(xbar),
                                        _ptr(vbar), _ptr(mbar), _ptr(abar_next), _ptr(dtbar))
        NBodyState.check("nbStepAdjointCUDA", rc)

    def vjp(self, ctx, abar):
        abar = abar.contiguous()
        xbar = torch.empty((self.n, 3), dtype=torch.float64, device=self.device)
        mbar = torch.empty((self.n,), dtype=torch.float64, device=self.device)
        _sync()
        rc = self.lib.nbGravVJPCUDA(ctypes.byref(ctx.struct), self.st._h, _ptr(abar), _ptr(xbar),
                                    _ptr(mbar))
        NBodyState.check("nbGravVJPCUDA", rc)
        return xbar, mbar


# Device states kept between runs, one per (bodies, device): a state keeps its buffers and the
# saved trees of its last backward pass allocated, so repeated runs (an optimisation loop)
# allocate nothing after the first.  release_states() frees them.
_POOL = {}


def _acquire(n, device):
    ds = _POOL.pop((n, device.index or 0), None)
    return ds if ds is not None else DeviceState(n, device)


def _release(ds):
    key = (ds.n, ds.device.index or 0)
    old = _POOL.pop(key, None)
    if old is not None:
        old.close()
    _POOL[key] = ds


def release_states():
    """Free the device states (and their saved trees) kept between runs."""
    for ds in _POOL.values():
        ds.close()
    _POOL.clear()


class _Run(torch.autograd.Function):
    """(x0, v0, m, dt) -> (xN, vN) through nsteps GPU steps; see the module docstring."""

    @staticmethod
    def forward(fctx, x0, v0, m, dt, nbctx, nsteps, every, stats):
        n = x0.shape[0]
        ds = _acquire(n, x0.device)
        ctx = NBodyCtx.from_struct(nbctx.struct)
        ctx.struct.timestep = float(dt)
        x0c, v0c, mc = x0.detach().contiguous(), v0.detach().contiguous(), m.detach().contiguous()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _sync()
        ev0.record()
        ds.set(x0c, v0c, mc, ctx.treeRSize)
        ds.gravmap(ctx)
        ckpts = [(x0c.clone(), v0c.clone(), ctx.treeRSize)]
        fwd_ms = 0.0
        for k in range(nsteps):
            if k and k % every == 0:
                x, v, _ = ds.get()
                ckpts.append((x, v, ds.rsize()))
            ds.step(ctx)
            fwd_ms += ds.st.step_time_ms()
        xN, vN, _ = ds.get()
        ev1.record()
        ev1.synchronize()
        fctx.ds = ds
        fctx.ctx = ctx
        fctx.ckpts = ckpts
        fctx.nsteps = nsteps
        fctx.every = every
        fctx.stats = stats
        if stats is not None:
            stats["forward_step_ms"] = ev0.elapsed_time(ev1) / max(nsteps, 1)
            stats["forward_step_device_ms"] = fwd_ms / max(nsteps, 1)
        fctx.save_for_backward(mc)
        if not any(fctx.needs_input_grad[:4]):
            fctx.ds = None                # no backward pass will come
            _release(ds)
        return xN, vN

    @staticmethod
    def backward(fctx, gx, gv):
        (m,) = fctx.saved_tensors
        ds, ctx, ckpts = fctx.ds, fctx.ctx, fctx.ckpts
        nsteps, every = fctx.nsteps, fctx.every
        like = ckpts[0][0]
        xbar = gx.detach().clone().contiguous() if gx is not None else torch.zeros_like(like)
        vbar = gv.detach().clone().contiguous() if gv is not None else torch.zeros_like(like)
        mbar = torch.zeros_like(m)
        dtbar = torch.zeros((), dtype=torch.float64, device=m.device)
        abar_next = torch.zeros_like(like)        # adjoint of a_{k+1} from the step after it
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _sync()
        ev0.record()
        rev_calls = 0
        rec_ms = rev_ms = rev_walk_ms = 0.0       # device times of the parts, summed
        for s in range(len(ckpts) - 1, -1, -1):
            k0 = s * every
            k1 = min(k0 + every, nsteps)
            x0, v0, rs0 = ckpts[s]
            # recompute the segment; slot j keeps the evaluation (bodies + tree) of state k0 + j
            ds.set(x0, v0, m, rs0)
            ds.gravmap(ctx)
            ds.save(0)
            acc = [ds.accel()]
            for j in range(k0, k1):
                ds.step(ctx)
                rec_ms += ds.st.step_time_ms()
                ds.save(j - k0 + 1)
                acc.append(ds.accel())
            # reverse steps k1-1 .. k0 on the saved trees (nbStepAdjointCUDA)
            for k in range(k1 - 1, k0 - 1, -1):
                ds.restore(k - k0 + 1)
                ds.step_adjoint(ctx, acc[k - k0], xbar, vbar, mbar, abar_next, dtbar)
                rev_ms += ds.st.step_time_ms()
                rev_walk_ms += ds.st.walk_time_ms()[0]
                rev_calls += 1
        # a_0 = A(x_0) feeds the first kick: slot 0 of the first segment holds it
        ds.restore(0)
        gx0, gm0 = ds.vjp(ctx, abar_next)
        xbar = xbar + gx0
        mbar = mbar + gm0
        ev1.record()
        ev1.synchronize()
        if fctx.stats is not None:
            fctx.stats["adjoint_step_ms"] = ev0.elapsed_time(ev1) / max(nsteps, 1)
            fctx.stats["vjp_calls"] = rev_calls + 1
            fctx.stats["recompute_step_device_ms"] = rec_ms / max(nsteps, 1)
            fctx.stats["reverse_step_device_ms"] = rev_ms / max(rev_calls, 1)
            fctx.stats["vjp_walk_device_ms"] = rev_walk_ms / max(rev_calls, 1)
        _release(ds)
        return xbar, vbar, mbar, dtbar, None, None, None, None


def run(nbctx, x0, v0, m, dt, nsteps, every=32, stats=None):
    """Differentiable run of nsteps FP64 GPU steps (checkpoints every `every` steps)."""
    return _Run.apply(x0, v0, m, dt, nbctx, nsteps, every, stats)


# ---------------------------------------------------------------------------------------
# differentiable set-up and loss (torch)
class DwarfDraws:
    """The seeded random numbers of one dwarf realisation, independent of the parameters."""

    def __init__(self, nbody, seed, device, n_baryon=None):
        rng = np.random.default_rng(seed)
        self.n = nbody
        self.nb = nbody // 2 if n_baryon is None else n_baryon
        umax = (1.0 + 1.0 / 50.0 ** 2) ** -1.5
        u = rng.uniform(1e-12, umax, nbody)
        z = rng.uniform(-1.0, 1.0, (2, nbody))
        phi = rng.uniform(0.0, 2.0 * math.pi, (2, nbody))
        from .models import _df_speed_fraction
        q = _df_speed_fraction(rng, nbody)
        t = lambda a: torch.tensor(a, dtype=torch.float64, device=device)
        self.shape = t(1.0 / np.sqrt(u ** (-2.0 / 3.0) - 1.0))   # r / a
        s = np.sqrt(1.0 - z * z)
        self.dir_pos = t(np.stack([s[0] * np.cos(phi[0]), s[0] * np.sin(phi[0]), z[0]], 1))
        self.dir_vel = t(np.stack([s[1] * np.cos(phi[1]), s[1] * np.sin(phi[1]), z[1]], 1))
        self.q = t(q)
        self.is_baryon = torch.zeros(nbody, dtype=torch.bool, device=device)
        self.is_baryon[:self.nb] = True


def dwarf_ics(params, draws):
    """Positions, velocities and masses of the dwarf (centred, at rest) as a function of
    (r_baryon, radius_ratio, m_baryon, mass_ratio) = params[2:6]: the two-component
    Plummer+Plummer sampler of models.plummer_plummer_dwarf with its draws held fixed."""
    a_b, xr, M_b, xm = params[2], params[3], params[4], params[5]
    a_d = a_b / xr * (1.0 - xr)
    M_d = M_b / xm * (1.0 - xm)
    b = draws.is_baryon
    a = torch.where(b, a_b, a_d)
    r = a * draws.shape
    pos = r[:, None] * draws.dir_pos
    phi = -(M_b / torch.sqrt(r * r + a_b * a_b)) - (M_d / torch.sqrt(r * r + a_d * a_d))
    vel = (draws.q * torch.sqrt(-2.0 * phi))[:, None] * draws.dir_vel
    nb, nd = draws.nb, draws.n - draws.nb
    mass = torch.where(b, M_b / max(nb, 1), M_d / max(nd, 1))
    mtot = mass.sum()
    pos = pos - (mass[:, None] * pos).sum(0) / mtot
    vel = vel - (mass[:, None] * vel).sum(0) / mtot
    return pos, vel, mass


def ext_accel_torch(pot, x):
    """nbExtAcceleration for MN disks, Hernquist/Plummer bulge, logarithmic/NFW halo."""
    X, Y, Z = x[..., 0], x[..., 1], x[..., 2]
    absv = torch.sqrt(Z * Z + (Y * Y + X * X))
    r = torch.clamp(absv, min=0.00390625)
    ax = torch.zeros_like(X); ay = torch.zeros_like(X); az = torch.zeros_like(X)
    for d in (pot.disk, pot.disk2):
        if d.type == _lib.MIYAMOTO_NAGAI_DISK:
            zp = torch.sqrt(Z * Z + d.scaleHeight ** 2)
            azp = d.scaleLength + zp
            rth = (X * X + Y * Y + azp * azp) ** 1.5
            ax = ax - d.mass * X / rth
            ay = ay - d.mass * Y / rth
            az = az - d.mass * Z * azp / (zp * rth)
    h = pot.halo
    if h.type == _lib.LOGARITHMIC_HALO:
        denom = h.scaleLength ** 2 + X * X + Y * Y + (Z / h.flattenZ) ** 2
        k = -2.0 * h.vhalo * h.vhalo / denom
        ax, ay, az = ax + k * X, ay + k * Y, az + k * Z / (h.flattenZ ** 2)
    elif h.type == _lib.NFW_HALO:
        a = h.scaleLength
        M = h.vhalo ** 2 * a / 0.2162165954
        c = (-M / (r * r)) * (torch.log((a + r) / a) / r - 1.0 / (a + r))
        ax, ay, az = ax + c * X, ay + c * Y, az + c * Z
    s = pot.sphere
    if s.type == _lib.HERNQUIST_SPHERICAL:
        c = -s.mass / (r * (s.scale + r) ** 2)
        ax, ay, az = ax + c * X, ay + c * Y, az + c * Z
    elif s.type == _lib.PLUMMER_SPHERICAL:
        c = -s.mass / torch.sqrt(s.scale ** 2 + r * r) ** 3
        ax, ay, az = ax + c * X, ay + c * Y, az + c * Z
    return torch.stack([ax, ay, az], -1)


def lbr_to_cartesian(l_deg, b_deg, r, sun_gc_dist=SUN_GC_DIST):
    l, b = l_deg * (math.pi / 180.0), b_deg * (math.pi / 180.0)
    return torch.stack([r * torch.cos(b) * torch.cos(l) - sun_gc_dist,
                        r * torch.cos(b) * torch.sin(l), r * torch.sin(b)])


def reverse_orbit(pot, pos, vel, tstop, dt):
    """nbReverseOrbit (nbody/src/nbody_orbit_integrator.c:44-86): leapfrog of the dwarf's
    centre backwards in the external potential for tstop; returns its start position and
    velocity.  The step count is fixed by the values of tstop and dt (a whole number, not
    differentiated): the gradient with respect to tstop flows only through the step length
    tstop / nsteps."""
    value = lambda t: float(t.detach()) if torch.is_tensor(t) else float(t)
    nsteps = int(math.floor(value(tstop) / value(dt))) + 1
    dtr = tstop / nsteps
    x, v = pos, -vel
    acc = ext_accel_torch(pot, x)
    for _ in range(nsteps):
        v = v + 0.5 * dtr * acc
        x = x + dtr * v
        acc = ext_accel_torch(pot, x)
        v = v + 0.5 * dtr * acc
    return x, -v


def lambda_beta(x, phi=128.79, theta=54.39, psi=90.70, sun_gc_dist=SUN_GC_DIST):
    """nbXYZToLambdaBeta (nbody/src/nbody_coordinates.c:129-164), degrees."""
    d2r = math.pi / 180.0
    cph, sph = math.cos(phi * d2r), math.sin(phi * d2r)
    cps, sps = math.cos(psi * d2r), math.sin(psi * d2r)
    cth, sth = math.cos(theta * d2r), math.sin(theta * d2r)
    X = x[:, 0] + sun_gc_dist
    Y, Z = x[:, 1], x[:, 2]
    tx = (cps * cph - cth * sph * sps) * X + (cps * sph + cth * cph * sps) * Y + sps * sth * Z
    ty = (-sps * cph - cth * sph * cps) * X + (-sps * sph + cth * cph * cps) * Y + cps * sth * Z
    tz = sth * sph * X - sth * cph * Y + cth * Z
    rr = torch.sqrt(tx * tx + ty * ty + tz * tz)
    return torch.atan2(ty, tx) / d2r, torch.asin(-tz / rr) / d2r


def soft_histogram(lam, beta, weight, bins=50, lam_range=(-150.0, 150.0),
                   beta_range=(-15.0, 15.0), width_bins=1.0):
    """Gaussian-kernel soft binning: every body spreads its weight over the bins with a
    Gaussian of sigma = width_bins x bin width in Lambda, and is counted in the single Beta
    bin through the same Gaussian's integral over [beta_lo, beta_hi]."""
    lo, hi = lam_range
    bw = (hi - lo) / bins
    sig = width_bins * bw
    edges = lo + bw * torch.arange(bins + 1, dtype=lam.dtype, device=lam.device)
    cdf = 0.5 * (1.0 + torch.erf((edges[None, :] - lam[:, None]) / (sig * math.sqrt(2.0))))
    w_lam = cdf[:, 1:] - cdf[:, :-1]
    b0, b1 = beta_range
    w_beta = 0.5 * (torch.erf((b1 - beta) / (sig * math.sqrt(2.0))) -
                    torch.erf((b0 - beta) / (sig * math.sqrt(2.0))))
    h = (weight[:, None] * w_beta[:, None] * w_lam).sum(0)
    return h / h.sum().clamp_min(1e-300)


def model_histogram(nbctx, params, orbit, draws, nsteps, every=32, pot=None, stats=None,
                    forward=None):
    """Parameters -> final baryon (Lambda, Beta) soft histogram.  params: 6 dwarf parameters
    (t_forward, time_ratio, r_baryon, radius_ratio, m_baryon, mass_ratio); orbit: (l, b, r,
    vx, vy, vz) of the dwarf's present position.  forward(x0, v0, m, dt) -> (xN, vN) defaults
    to the GPU run (`run`)."""
    pot = pot if pot is not None else nbctx.struct.pot
    t_fwd, ratio = params[0], params[1]
    dt = t_fwd / nsteps
    centre = lbr_to_cartesian(orbit[0], orbit[1], orbit[2])
    x_c, v_c = reverse_orbit(pot, centre, orbit[3:6], t_fwd / ratio, dt)
    pos, vel, mass = dwarf_ics(params, draws)
    x0 = (pos + x_c).contiguous()
    v0 = (vel + v_c).contiguous()
    if forward is None:
        xN, vN = run(nbctx, x0, v0, mass, dt, nsteps, every, stats)
    else:
        xN, vN = forward(x0, v0, mass, dt)
    lam, beta = lambda_beta(xN[draws.is_baryon])
    return soft_histogram(lam, beta, mass[draws.is_baryon])


def direct_run_torch(x0, v0, m, dt, nsteps, eps2, pot):
    """FP64 direct-summation N-body run in plain torch (autograd reference): the arithmetic
    of nbGravity_Exact (nbody/src/nbody_grav.c:205-227) + nbExtAcceleration + KDK."""
    def accel(x):
        d = x[None, :, :] - x[:, None, :]             # d[i, j] = x_j - x_i
        s = (d * d).sum(-1) + eps2
        a = ((m[None, :] / (s * torch.sqrt(s)))[..., None] * d).sum(1)
        return a + ext_accel_torch(pot, x)
    h = 0.5 * dt
    x, v = x0, v0
    a = accel(x)
    for _ in range(nsteps):
        v = v + h * a
        x = x + dt * v
        a = accel(x)
        v = v + h * a
    return x, v
