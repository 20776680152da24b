"""Set-up helpers: the reference's timestep/softening formulas and a seeded synthetic
two-component Plummer dwarf with the shapes and sizes of the reference's dwarf models.

These run once per simulation on the host (they are the reference's Lua set-up, not the
step).  The dwarf sampler is synthetic: positions follow each component's Plummer profile
exactly; speeds are drawn from the isotropic Plummer distribution function
f(E) ~ (-E)^{7/2} evaluated in the combined potential of both components, which keeps the
dwarf close to equilibrium.  It is not the reference's Eddington-inversion sampler
(nbGenerateMixedDwarfCore, nbody/src/nbody_mixeddwarf.c:765-1026) and does not reproduce
its random stream; parity with the reference is established on identical input arrays.
"""
import math

import numpy as np

# PI_4_3 of the reference (milkyway/include/milkyway_math_supplemental.h:195), the constant its
# Lua set-up sees as pi_4_3; 4.0 * math.pi / 3.0 rounds one ulp lower
PI_4_3 = 4.188790204786390984616857844372670512262892532500141
SUN_GC_DIST = 8.0   # ctx.sunGCDist default (nbody/include/nbody_defaults.h)


def calculate_timestep(mass, r0):
    """calculateTimestep (nbody/src/nbody_lua_models.c:139-142)."""
    return (1.0 / 10.0) ** 2 * math.sqrt((PI_4_3 * r0 ** 3) / mass)


def two_component_timestep(mass_l, rscale_l, mass_d, rscale_d):
    """get_timestep of the two-component sample workunit
    (nbody/sample_workunits/for_developers.lua:165-199)."""
    mass_enc_d = mass_d * rscale_l ** 3 * (rscale_l ** 2 + rscale_d ** 2) ** (-1.5)
    mass_enc_l = mass_l * rscale_d ** 3 * (rscale_l ** 2 + rscale_d ** 2) ** (-1.5)
    s1 = rscale_l ** 3 / (mass_enc_d + mass_l)
    s2 = rscale_d ** 3 / (mass_enc_l + mass_d)
    return (1.0 / 100.0) * (PI_4_3 * min(s1, s2)) ** (1.0 / 2.0)


def calculate_virial(a_b, a_d, M_b, M_d, n=100000):
    """nbCalculateVirial (nbody/src/nbody_virial.c:38-103): 5-point Gauss-Legendre on n
    panels out to 1000 scale radii, the terms formed in the reference's operation order and
    summed one after another as its loop does (numpy's pow stands in for crlibm's pow_rn,
    so the result may differ from the reference's in the last bits)."""
    w = np.array([0.2369268850561891, 0.4786286704993665, 0.5688888888888889,
                  0.4786286704993665, 0.2369268850561891])
    x = np.array([-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831,
                  0.9061798459386640])
    upper = 1000.0 * a_b if a_b > a_d else 1000.0 * a_d
    width = (upper - 0.0) / (n * 1.0)
    i = np.arange(n, dtype=np.float64)
    a1 = 0.0 + i * width
    b1 = 0.0 + (i + 1.0) * width
    r = width * x[None, :] / 2.0 + ((a1 + b1) / 2.0)[:, None]
    dens = 3.0 / 4.0 / math.pi * (M_b / a_b ** 3.0 * (1.0 + r * r / a_b / a_b) ** -2.5 +
                                  M_d / a_d ** 3.0 * (1.0 + r * r / a_d / a_d) ** -2.5)
    integ = 1.0 / 4.0 / math.pi * (M_b / a_b * r * r * (1.0 + r * r / a_b / a_b) ** -0.5 +
                                   M_d / a_d * r * r * (1.0 + r * r / a_d / a_d) ** -0.5)
    terms = (w[None, :] * dens * integ * width / 2.0).ravel()
    integral = 0.0
    for t in terms.tolist():
        integral += t
    M_tot = M_b + M_d
    return M_tot * M_tot / 16.0 / math.pi / math.pi / integral


def calculate_eps2(nbody, a_b, a_d, M_b, M_d):
    """calculateEps2 (nbody/src/nbody_lua_models.c:158-169): eps = 0.98 r_v N^-0.26."""
    eps = calculate_virial(a_b, a_d, M_b, M_d) * 0.98 * float(nbody) ** -0.26
    eps2 = (eps * eps) / 1.0
    return eps2 if eps2 > np.finfo(np.float64).eps else float(np.finfo(np.float64).eps)


def sample_workunit_potential():
    """The potential of the two-component sample workunit
    (nbody/sample_workunits/for_developers.lua:150-162): Hernquist bulge, Miyamoto-Nagai disk
    and a logarithmic halo of vhalo = 74.61 kpc/Gyr (73 km/s)."""
    from .nbody import milky_way_potential
    return milky_way_potential(vhalo=74.61)


def lbr_to_cartesian(l_deg, b_deg, r, sun_gc_dist=SUN_GC_DIST):
    """lbrToCartesian with the Sun at (-sunGCDist, 0, 0)."""
    l, b = math.radians(l_deg), math.radians(b_deg)
    return np.array([r * math.cos(b) * math.cos(l) - sun_gc_dist,
                     r * math.cos(b) * math.sin(l), r * math.sin(b)])


def _plummer_radii(rng, n, a, rmax_factor=50.0):
    umax = (1.0 + 1.0 / rmax_factor ** 2) ** -1.5     # mass fraction inside rmax
    u = rng.uniform(1e-12, umax, n)
    return a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)


def _unit_vectors(rng, n):
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    s = np.sqrt(1.0 - z * z)
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)


def _df_speed_fraction(rng, n):
    """q = v / v_esc with density q^2 (1 - q^2)^{7/2} (rejection, Aarseth et al. 1974)."""
    out = np.empty(n)
    filled = 0
    while filled < n:
        k = max(2 * (n - filled), 1024)
        q = rng.uniform(0.0, 1.0, k)
        y = rng.uniform(0.0, 0.1, k)
        q = q[y < q * q * (1.0 - q * q) ** 3.5]
        take = min(len(q), n - filled)
        out[filled:filled + take] = q[:take]
        filled += take
    return out


def plummer_plummer_dwarf(nbody, seed=0, mass_l=12.0, rscale_l=0.2, light_r_ratio=0.2,
                          light_mass_ratio=0.2, n_baryon=None, position=None, velocity=None):
    """Seeded two-component Plummer+Plummer dwarf (baryons first, then dark matter).

    Parameters follow the sample workunit (for_developers.lua:460-478): the dark component
    has radius rscale_l/light_r_ratio*(1-light_r_ratio) and mass
    mass_l/light_mass_ratio*(1-light_mass_ratio).  Returns pos (n,3), vel (n,3), mass (n,),
    type (n,) with +1 for baryons and -1 for dark matter (the reference's ignore flag)."""
    rng = np.random.default_rng(seed)
    if n_baryon is None:
        n_baryon = nbody // 2
    n_dark = nbody - n_baryon
    dwarf_mass = mass_l / light_mass_ratio
    rscale_t = rscale_l / light_r_ratio
    rscale_d = rscale_t * (1.0 - light_r_ratio)
    mass_d = dwarf_mass * (1.0 - light_mass_ratio)
    r = np.concatenate([_plummer_radii(rng, n_baryon, rscale_l), _plummer_radii(rng, n_dark, rscale_d)])
    pos = r[:, None] * _unit_vectors(rng, nbody)
    phi = -(mass_l / np.sqrt(r * r + rscale_l ** 2)) - (mass_d / np.sqrt(r * r + rscale_d ** 2))
    v = _df_speed_fraction(rng, nbody) * np.sqrt(-2.0 * phi)
    vel = v[:, None] * _unit_vectors(rng, nbody)
    mass = np.concatenate([np.full(n_baryon, mass_l / max(n_baryon, 1)),
                           np.full(n_dark, mass_d / max(n_dark, 1))])
    typ = np.concatenate([np.ones(n_baryon, np.int32), -np.ones(n_dark, np.int32)])
    # centre the sample, then place it on the orbit
    cm = (mass[:, None] * pos).sum(0) / mass.sum()
    cv = (mass[:, None] * vel).sum(0) / mass.sum()
    pos -= cm
    vel -= cv
    if position is None:
        position = lbr_to_cartesian(218.0, 53.5, 28.6)
    if velocity is None:
        velocity = np.array([-156.0, 79.0, 107.0])
    pos += np.asarray(position, dtype=np.float64)
    vel += np.asarray(velocity, dtype=np.float64)
    return pos, vel, mass, typ


# the present-day orbit point of the sample workunits' dwarf: (l, b, r) in deg, deg, kpc and
# the velocity the Lua set-up gives Vector.create
SAMPLE_ORBIT = ((218.0, 53.5, 28.6), (-156.0, 79.0, 107.0))


def sampled_dwarf(nbody, seed, device=0, mass_l=12.0, rscale_l=0.2, light_r_ratio=0.2,
                  light_mass_ratio=0.2, position=None, velocity=None):
    """The sample workunit's two-component Plummer dwarf (half baryons) sampled on the GPU by
    the library's port of the reference's sampler (nbGenerateDwarfCUDA: nbGenerateMixedDwarfCore,
    nbody/src/nbody_mixeddwarf.c:765-1026, with a counter-based stream per body), recentred and
    placed on the orbit point (by default SAMPLE_ORBIT, no reverse orbit).  The same seed gives
    the same bodies bit for bit on every run.  Returns host arrays pos (n,3), vel (n,3),
    mass (n,) and type (n,): +1 for the baryons (the first nbody // 2), -1 for dark matter."""
    from .nbody import NBodyState, plummer_dwarf_struct
    import ctypes
    if position is None:
        position = lbr_to_cartesian(*SAMPLE_ORBIT[0])
    if velocity is None:
        velocity = np.asarray(SAMPLE_ORBIT[1], dtype=np.float64)
    d = plummer_dwarf_struct(nbody, seed, None, mass_l, rscale_l, light_r_ratio,
                             light_mass_ratio, position, velocity)
    with NBodyState(nbody, device) as st:
        st.check("nbGenerateDwarf", st.lib.nbGenerateDwarfCUDA(st._h, ctypes.byref(d), 4.0))
        pos, vel = st.bodies()
        mass = st.masses()
    nb = int(d.nbodyBaryon)
    typ = np.concatenate([np.ones(nb, np.int32), -np.ones(nbody - nb, np.int32)])
    return pos, vel, mass, typ


def dwarf_config(nbody, theta=1.0, criterion="TreeCode", useQuad=True, mass_l=12.0,
                 rscale_l=0.2, light_r_ratio=0.2, light_mass_ratio=0.2):
    """Context settings of the two-component sample workunit at nbody bodies: dt from the
    two-component formula, eps2 from calculateEps2."""
    rscale_d = rscale_l / light_r_ratio * (1.0 - light_r_ratio)
    mass_d = mass_l / light_mass_ratio * (1.0 - light_mass_ratio)
    dt = two_component_timestep(mass_l, rscale_l, mass_d, rscale_d)
    eps2 = calculate_eps2(nbody, rscale_l, rscale_d, mass_l, mass_d)
    return dict(timestep=dt, eps2=eps2, theta=theta, criterion=criterion, useQuad=useQuad,
                treeRSize=4.0)


# ---- batched uneven dwarfs ----
def dwarf_parameter_draws(ndwarfs, seed, nmin=4096, nmax=65536):
    """Seeded parameter sets of the batched-dwarfs workload: N log-uniform in [nmin, nmax];
    forward time U[3.5, 4.5] Gyr, baryon scale radius U[0.1, 0.5] kpc, radius ratio U[0.1, 0.5],
    baryon mass U[1, 100] SMU, mass ratio U[0.01, 0.95]."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(nmin), math.log(nmax), ndwarfs)).astype(np.int64)
    return [dict(nbody=int(n[k]), t_forward=float(rng.uniform(3.5, 4.5)),
                 rscale_l=float(rng.uniform(0.1, 0.5)), light_r_ratio=float(rng.uniform(0.1, 0.5)),
                 mass_l=float(rng.uniform(1.0, 100.0)), light_mass_ratio=float(rng.uniform(0.01, 0.95)))
            for k in range(ndwarfs)]


def reverse_orbits(potential, pos, vel, tstops, dt, device=0):
    """nbReverseOrbit (nbody/src/nbody_orbit_integrator.c:44-86) of many orbit centres at once:
    leapfrog backwards for each tstop with nsteps = floor(tstop / dt) + 1 steps of
    tstop / nsteps, the potential evaluated on the GPU (nbExtAccelerationNoAllocCUDA: one small
    call per step, no allocation; more than 65,536 orbit centres are evaluated in chunks of
    65,536 per step)."""
    from .nbody import ext_acceleration
    pos = np.array(pos, dtype=np.float64).reshape(-1, 3)
    vel = -np.array(vel, dtype=np.float64).reshape(-1, 3)
    tstops = np.asarray(tstops, dtype=np.float64)
    nsteps = np.floor(tstops / dt).astype(np.int64) + 1
    dtr = (tstops / nsteps)[:, None]
    acc = ext_acceleration(potential, pos, device, no_alloc=True)
    for k in range(int(nsteps.max())):
        live = (k < nsteps)[:, None]
        v = vel + 0.5 * dtr * acc
        x = pos + dtr * v
        a = ext_acceleration(potential, x, device, no_alloc=True)
        v = v + 0.5 * dtr * a
        pos = np.where(live, x, pos)
        vel = np.where(live, v, vel)
        acc = np.where(live, a, acc)
    return pos, -vel


def batched_dwarfs(draws, potential, seed=0, orbit_dt=1e-3, device=0, nsteps=None,
                   orbit=((218.0, 53.5, 28.6), (-156.0, 79.0, 107.0))):
    """Initial conditions of a batch: every draw of dwarf_parameter_draws becomes a
    two-component Plummer dwarf started on the shared orbit t_forward back from the present-day
    position, with its own softening (calculateEps2) and time step: the two-component formula,
    or, with nsteps, t_forward / nsteps (as nbCorrectTimestep sets it for a run of nsteps
    steps over the evolution time).  Returns a list of dicts: pos, vel, mass, types, eps2,
    timestep, params."""
    (l, b, r), v0 = orbit
    p0 = lbr_to_cartesian(l, b, r)
    tf = [d["t_forward"] for d in draws]
    starts, vstarts = reverse_orbits(potential, np.tile(p0, (len(draws), 1)),
                                     np.tile(np.asarray(v0, dtype=np.float64), (len(draws), 1)),
                                     tf, orbit_dt, device)
    out = []
    for k, d in enumerate(draws):
        pos, vel, mass, typ = plummer_plummer_dwarf(
            d["nbody"], seed=seed + k, mass_l=d["mass_l"], rscale_l=d["rscale_l"],
            light_r_ratio=d["light_r_ratio"], light_mass_ratio=d["light_mass_ratio"],
            position=starts[k], velocity=vstarts[k])
        cfg = dwarf_config(d["nbody"], mass_l=d["mass_l"], rscale_l=d["rscale_l"],
                           light_r_ratio=d["light_r_ratio"], light_mass_ratio=d["light_mass_ratio"])
        dt = d["t_forward"] / nsteps if nsteps else cfg["timestep"]
        out.append(dict(pos=pos, vel=vel, mass=mass, types=typ, eps2=cfg["eps2"],
                        timestep=dt, params=d))
    return out


def batched_dwarf_structs(draws, potential, seed=0, orbit_dt=1e-3, device=0, nsteps=None,
                          orbit=((218.0, 53.5, 28.6), (-156.0, 79.0, 107.0))):
    """As batched_dwarfs, for the GPU sampler: returns the batch spec [(nbody, eps2, timestep,
    treeRSize)] and one NBodyCudaPlummerDwarf per draw (nbBatchGenerateDwarfsCUDA samples the
    bodies on the device with the reference's two-component algorithm)."""
    from .nbody import plummer_dwarf_struct
    (l, b, r), v0 = orbit
    p0 = lbr_to_cartesian(l, b, r)
    starts, vstarts = reverse_orbits(potential, np.tile(p0, (len(draws), 1)),
                                     np.tile(np.asarray(v0, dtype=np.float64), (len(draws), 1)),
                                     [d["t_forward"] for d in draws], orbit_dt, device)
    spec, structs = [], []
    for k, d in enumerate(draws):
        cfg = dwarf_config(d["nbody"], mass_l=d["mass_l"], rscale_l=d["rscale_l"],
                           light_r_ratio=d["light_r_ratio"], light_mass_ratio=d["light_mass_ratio"])
        dt = d["t_forward"] / nsteps if nsteps else cfg["timestep"]
        spec.append((d["nbody"], cfg["eps2"], dt, 4.0))
        structs.append(plummer_dwarf_struct(d["nbody"], seed + k, None, d["mass_l"], d["rscale_l"],
                                            d["light_r_ratio"], d["light_mass_ratio"], starts[k],
                                            vstarts[k]))
    return spec, structs
