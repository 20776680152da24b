"""Host-side mirror of the reference's N-body step interface, running on the B200 library.

Names, argument meaning and error behaviour follow the reference's own plugin seam for the
step -- the Lua types and methods the reference's tests drive (NBodyCtx.create,
Potential.create with Spherical/Disk/Halo, NBodyState.create, state:step;
nbody/src/nbody_lua_types/*.c) and the C entry points behind them (nbGravMap,
nbStepSystem, nbRunSystem; nbody/src/nbody_grav.c:305, nbody/src/nbody.c:182-212).
Statuses are the reference's NBodyStatus bit masks.  All arithmetic happens in the CUDA
library (libnbody_b200.so); this module only marshals numpy arrays through the C ABI.
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import (CRITERIA, PRECISION_FP64, PRECISION_MIXED, POTENTIAL_DEFAULT, POTENTIAL_NONE,
                   status_is_fatal, status_names)


class NBodyError(RuntimeError):
    """A fatal NBodyStatus returned by the library."""

    def __init__(self, what, status):
        detail = _lib.last_error() if status & _lib.NBODY_CUDA_ERROR else ""
        super().__init__("%s failed: %s%s" % (what, "|".join(status_names(status)),
                                              (" (" + detail + ")") if detail else ""))
        self.status = status


# ---- potential components (nbody/src/nbody_lua_types/nbody_lua_{spherical,disk,halo}.c) ----
class Spherical:
    @staticmethod
    def hernquist(mass, scale):
        return _lib.Spherical(_lib.HERNQUIST_SPHERICAL, mass, scale)

    @staticmethod
    def plummer(mass, scale):
        return _lib.Spherical(_lib.PLUMMER_SPHERICAL, mass, scale)

    @staticmethod
    def none(mass=0.0):
        return _lib.Spherical(_lib.NO_SPHERICAL, mass, 0.0)


class Disk:
    @staticmethod
    def miyamotoNagai(mass, scaleLength, scaleHeight):
        return _lib.Disk(_lib.MIYAMOTO_NAGAI_DISK, mass, scaleLength, scaleHeight, 0.0, 0.0)

    @staticmethod
    def orbitingBar(mass, scaleLength, patternSpeed, startAngle):
        """The softened needle bar (disk2 only), rotating at patternSpeed (rad/Gyr)."""
        return _lib.Disk(_lib.ORBITING_BAR, mass, scaleLength, 0.0, patternSpeed, startAngle)

    @staticmethod
    def none(mass=0.0):
        return _lib.Disk(_lib.NO_DISK, mass, 0.0, 0.0, 0.0, 0.0)


class Halo:
    @staticmethod
    def logarithmic(vhalo, scaleLength, flattenZ):
        h = _lib.Halo()
        h.type, h.vhalo, h.scaleLength, h.flattenZ = _lib.LOGARITHMIC_HALO, vhalo, scaleLength, flattenZ
        return h

    @staticmethod
    def nfw(vhalo, scaleLength):
        h = _lib.Halo()
        h.type, h.vhalo, h.scaleLength = _lib.NFW_HALO, vhalo, scaleLength
        return h

    @staticmethod
    def caustic(vhalo=0.0, scaleLength=0.0):
        """Halo.caustic{vhalo, scaleLength}: the field takes the reference's fixed flow tables;
        the two parameters are carried but unused, as in the reference."""
        h = _lib.Halo()
        h.type, h.vhalo, h.scaleLength = _lib.CAUSTIC_HALO, vhalo, scaleLength
        return h

    @staticmethod
    def triaxial(vhalo, scaleLength, flattenX, flattenY, flattenZ, triaxAngle):
        """Triaxial logarithmic halo; c1..c3 as nbCheckParams derives them
        (nbody/src/nbody_check_params.c:182-194)."""
        h = _lib.Halo()
        h.type, h.vhalo, h.scaleLength = _lib.TRIAXIAL_HALO, vhalo, scaleLength
        h.flattenX, h.flattenY, h.flattenZ, h.triaxAngle = flattenX, flattenY, flattenZ, triaxAngle
        phi = triaxAngle * math.pi / 180.0
        cp, sp = math.cos(phi), math.sin(phi)
        cps, sps = cp * cp, sp * sp
        qxs, qys = flattenX * flattenX, flattenY * flattenY
        h.c1 = (cps / qxs) + (sps / qys)
        h.c2 = (cps / qys) + (sps / qxs)
        h.c3 = math.sin(2.0 * phi) * ((qys - qxs) / (qxs * qys))
        return h

    @staticmethod
    def _mass_halo(kind, mass, scaleLength, **extra):
        h = _lib.Halo()
        h.type, h.mass, h.scaleLength = kind, mass, scaleLength
        for k, v in extra.items():
            setattr(h, k, v)
        return h

    @staticmethod
    def allenSantillan(mass, scaleLength, gamma, lambda_):
        return Halo._mass_halo(_lib.ALLEN_SANTILLAN_HALO, mass, scaleLength, gamma=gamma,
                               lambda_=lambda_)

    @staticmethod
    def wilkinsonEvans(mass, scaleLength):
        return Halo._mass_halo(_lib.WILKINSON_EVANS_HALO, mass, scaleLength)

    @staticmethod
    def nfwMass(mass, scaleLength):
        return Halo._mass_halo(_lib.NFW_MASS_HALO, mass, scaleLength)

    @staticmethod
    def plummer(mass, scaleLength):
        return Halo._mass_halo(_lib.PLUMMER_HALO, mass, scaleLength)

    @staticmethod
    def hernquist(mass, scaleLength):
        return Halo._mass_halo(_lib.HERNQUIST_HALO, mass, scaleLength)

    @staticmethod
    def ninkovic(rho0, scaleLength, lambda_):
        return Halo._mass_halo(_lib.NINKOVIC_HALO, 0.0, scaleLength, rho0=rho0, lambda_=lambda_)

    @staticmethod
    def none(mass=0.0):
        h = _lib.Halo()
        h.type, h.mass = _lib.NO_HALO, mass
        return h


class Potential:
    """Potential.create{spherical, disk, disk2, halo} (nbody_lua_potential.c)."""

    @staticmethod
    def create(spherical=None, disk=None, disk2=None, halo=None):
        p = _lib.Potential()
        p.sphere = spherical if spherical is not None else Spherical.none()
        p.disk = disk if disk is not None else Disk.none()
        p.disk2 = disk2 if disk2 is not None else Disk.none()
        p.halo = halo if halo is not None else Halo.none()
        return p


def milky_way_potential(vhalo=73.0):
    """The Miyamoto-Nagai + Hernquist + logarithmic-halo potential of the sample workunits
    (nbody/sample_workunits/for_developers.lua:150-162)."""
    return Potential.create(
        spherical=Spherical.hernquist(mass=1.52954402e5, scale=0.7),
        disk=Disk.miyamotoNagai(mass=4.45865888e5, scaleLength=6.5, scaleHeight=0.26),
        disk2=Disk.none(mass=3.0e5),
        halo=Halo.logarithmic(vhalo=vhalo, scaleLength=12.0, flattenZ=1.0))


class NBodyCtx:
    """NBodyCtx.create{...} (nbody/src/nbody_lua_types/nbody_lua_nbodyctx.c:84-221): the
    settings of a run.  nStep = ceil(timeEvolve / timestep) and the timestep is corrected to
    timeEvolve / nStep as the reference does (nbCorrectTimestep, nbody/src/nbody_util.c:26-30)."""

    def __init__(self, timestep, eps2, theta=0.0, criterion="TreeCode", useQuad=True,
                 timeEvolve=None, treeRSize=4.0, allowIncest=False, potential=None,
                 precision="fp64", LMC=False, LMCmass=0.0, LMCscale=1.0, LMCDynaFric=False,
                 coulomb_log=0.0):
        crit = CRITERIA[criterion.lower()] if isinstance(criterion, str) else int(criterion)
        self.nStep = 0
        if timeEvolve is not None and timeEvolve > 0.0:
            self.nStep = int(math.ceil(timeEvolve / timestep))
            timestep = timeEvolve / self.nStep
        self.timeEvolve = timeEvolve
        c = _lib.Ctx()
        c.eps2, c.theta, c.timestep, c.treeRSize = eps2, theta, timestep, treeRSize
        c.criterion, c.useQuad, c.allowIncest = crit, int(bool(useQuad)), int(bool(allowIncest))
        if potential is None:
            c.potentialType = POTENTIAL_NONE
        else:
            c.potentialType = POTENTIAL_DEFAULT
            c.pot = potential
        c.precision = {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}[precision]
        # the LMC (its state and reflex accelerations: NBodyState.set_lmc)
        c.lmc, c.lmcDynaFric = int(bool(LMC)), int(bool(LMCDynaFric))
        c.lmcMass, c.lmcScale, c.coulombLog = float(LMCmass), float(LMCscale), float(coulomb_log)
        self._c = c

    @classmethod
    def from_struct(cls, c, nStep=0):
        self = cls.__new__(cls)
        self._c = _lib.Ctx()
        ctypes.pointer(self._c)[0] = c
        self.nStep = nStep
        self.timeEvolve = c.timestep * nStep if nStep else None
        return self

    def with_precision(self, precision):
        other = NBodyCtx.from_struct(self._c, self.nStep)
        other._c.precision = {"fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}[precision]
        return other

    def __getattr__(self, name):
        c = self.__dict__.get("_c")
        if c is not None and name in dict(_lib.Ctx._fields_):
            return getattr(c, name)
        raise AttributeError(name)

    @property
    def struct(self):
        return self._c


def plummer_dwarf_struct(nbody, seed, nbody_baryon=None, mass_l=12.0, rscale_l=0.2,
                         light_r_ratio=0.2, light_mass_ratio=0.2, position=None, velocity=None):
    """NBodyCudaPlummerDwarf with the parameterisation of the sample workunits
    (for_developers.lua: dark radius rscale_l / light_r_ratio * (1 - light_r_ratio), dark mass
    mass_l / light_mass_ratio * (1 - light_mass_ratio))."""
    d = _lib.PlummerDwarf()
    d.nbody = int(nbody)
    d.nbodyBaryon = int(nbody // 2 if nbody_baryon is None else nbody_baryon)
    d.massLight, d.scaleLight = mass_l, rscale_l
    d.massDark = mass_l / light_mass_ratio * (1.0 - light_mass_ratio)
    d.scaleDark = rscale_l / light_r_ratio * (1.0 - light_r_ratio)
    pos = np.zeros(3) if position is None else np.asarray(position, dtype=np.float64)
    vel = np.zeros(3) if velocity is None else np.asarray(velocity, dtype=np.float64)
    for c in range(3):
        d.position[c], d.velocity[c] = float(pos[c]), float(vel[c])
    d.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return d


class Dwarf:
    """The components of a two-component dwarf, as the reference's Lua Dwarf.plummer, nfw,
    general_hernquist and cored (nbody/src/nbody_lua_types/nbody_lua_dwarf.c:57-125): for nfw
    and cored, mass is M200 (the sampler takes the mass inside its bound 5 r200 instead)."""

    @staticmethod
    def _make(kind, mass, scaleLength, r1=0.0, rc=0.0):
        c = _lib.DwarfComponent()
        c.type, c.mass, c.scaleLength, c.r1, c.rc = kind, float(mass), float(scaleLength), float(r1), float(rc)
        return c

    @staticmethod
    def plummer(mass, scaleLength):
        return Dwarf._make(_lib.DWARF_PLUMMER, mass, scaleLength)

    @staticmethod
    def nfw(mass, scaleLength):
        return Dwarf._make(_lib.DWARF_NFW, mass, scaleLength)

    @staticmethod
    def general_hernquist(mass, scaleLength):
        return Dwarf._make(_lib.DWARF_GEN_HERNQUIST, mass, scaleLength)

    @staticmethod
    def cored(mass, scaleLength, r1, rc):
        return Dwarf._make(_lib.DWARF_CORED, mass, scaleLength, r1, rc)


def mixed_dwarf_struct(nbody, seed, comp1, comp2, nbody_baryon=None, position=None, velocity=None):
    """NBodyCudaMixedDwarf: predefinedModels.mixeddwarf{nbody, nbody_baryon, comp1 (light),
    comp2 (dark), position, velocity} with the GPU sampler's seed."""
    d = _lib.MixedDwarf()
    d.nbody = int(nbody)
    d.nbodyBaryon = int(nbody // 2 if nbody_baryon is None else nbody_baryon)
    d.light, d.dark = comp1, comp2
    pos = np.zeros(3) if position is None else np.asarray(position, dtype=np.float64)
    vel = np.zeros(3) if velocity is None else np.asarray(velocity, dtype=np.float64)
    for c in range(3):
        d.position[c], d.velocity[c] = float(pos[c]), float(vel[c])
    d.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return d


def mixed_dwarf_particle_masses(dwarf):
    """(light, dark) particle masses the sampler assigns (nbMixedDwarfParticleMassesCUDA)."""
    out = np.zeros(2)
    NBodyState.check("nbMixedDwarfParticleMasses",
                     _lib.load().nbMixedDwarfParticleMassesCUDA(ctypes.byref(dwarf), _lib.ptr(out)))
    return float(out[0]), float(out[1])


class NBodyState:
    """Device-resident N-body state: NBodyState.create(ctx, bodies) and state:step(ctx)
    (nbody/src/nbody_lua_types/nbody_lua_nbodystate.c:60-147) over the CUDA library.

    Bodies are given as arrays: pos (n,3), vel (n,3), mass (n,), float64.  Like the reference
    binding, create() evaluates the initial accelerations (nbGravMap) so that step() is a full
    kick-drift-kick."""

    def __init__(self, nbody, device=0):
        self.lib = _lib.load()
        self.nbody = int(nbody)
        self.device = device
        h = ctypes.c_void_p()
        rc = self.lib.nbInitCUDA(ctypes.byref(h), device, self.nbody)
        if rc:
            raise NBodyError("nbInitCUDA", rc)
        self._h = h

    @classmethod
    def create(cls, ctx, pos, vel, mass, device=0, gravmap=True):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
        mass = np.ascontiguousarray(mass, dtype=np.float64).reshape(-1)
        st = cls(len(mass), device)
        st.set_bodies(pos, vel, mass, ctx.treeRSize)
        if gravmap:
            st.check("nbGravMap", st.gravMap(ctx))
        return st

    # -- lifecycle --
    def close(self):
        if getattr(self, "_h", None):
            self.lib.nbDestroyCUDA(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def check(what, rc):
        if status_is_fatal(rc):
            raise NBodyError(what, rc)
        return rc

    @classmethod
    def generate(cls, ctx, nbody, seed, nbody_baryon=None, mass_l=12.0, rscale_l=0.2,
                 light_r_ratio=0.2, light_mass_ratio=0.2, position=None, velocity=None,
                 device=0, gravmap=True):
        """A two-component Plummer dwarf sampled on the GPU (nbGenerateDwarfCUDA) with the
        parameters of plummer_plummer_dwarf, then nbGravMap."""
        st = cls(nbody, device)
        d = plummer_dwarf_struct(nbody, seed, nbody_baryon, mass_l, rscale_l, light_r_ratio,
                                 light_mass_ratio, position, velocity)
        st.check("nbGenerateDwarf", st.lib.nbGenerateDwarfCUDA(st._h, ctypes.byref(d),
                                                                float(ctx.treeRSize)))
        if gravmap:
            st.check("nbGravMap", st.gravMap(ctx))
        return st

    @classmethod
    def generate_mixed(cls, ctx, nbody, seed, comp1, comp2, nbody_baryon=None, position=None,
                       velocity=None, device=0, gravmap=True):
        """A two-component dwarf of any of the reference's profiles (Dwarf.*) sampled on the
        GPU (nbGenerateMixedDwarfCUDA), then nbGravMap."""
        st = cls(nbody, device)
        d = mixed_dwarf_struct(nbody, seed, comp1, comp2, nbody_baryon, position, velocity)
        st.check("nbGenerateMixedDwarf", st.lib.nbGenerateMixedDwarfCUDA(
            st._h, ctypes.byref(d), float(ctx.treeRSize)))
        if gravmap:
            st.check("nbGravMap", st.gravMap(ctx))
        return st

    def masses(self):
        """Every body's mass (nbGetBodyMassesCUDA)."""
        m = np.empty(self.nbody)
        self.check("nbGetBodyMasses", self.lib.nbGetBodyMassesCUDA(self._h, _lib.ptr(m)))
        return m

    def set_mixed_tuning(self, group_max=32, list_cap=64, blocks_per_sm=0):
        """Mixed-precision walk tuning (nbSetMixedTuningCUDA)."""
        self.check("nbSetMixedTuning", self.lib.nbSetMixedTuningCUDA(
            self._h, int(group_max), int(list_cap), int(blocks_per_sm)))

    def set_lmc(self, position, velocity, shift):
        """The LMC of an LMC run (nbSetLMCCUDA): its position and velocity and the Milky Way's
        reflex accelerations shift (k, 3), as the reference's reverseOrbit_LMC leaves them."""
        p = np.ascontiguousarray(position, dtype=np.float64).reshape(3)
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(3)
        sh = np.ascontiguousarray(shift, dtype=np.float64).reshape(-1, 3)
        self.check("nbSetLMC", self.lib.nbSetLMCCUDA(self._h, _lib.ptr(p), _lib.ptr(v),
                                                     _lib.ptr(sh), len(sh)))

    def lmc(self):
        """The LMC's current position and velocity (nbGetLMCCUDA)."""
        p, v = np.empty(3), np.empty(3)
        self.check("nbGetLMC", self.lib.nbGetLMCCUDA(self._h, _lib.ptr(p), _lib.ptr(v)))
        return p, v

    def set_mixed_mode(self, exact=True):
        """Mixed walk interaction sets (nbSetMixedModeCUDA): exact=True (default) gives every
        body its own FP64 interaction set; False lets a group share its box's set (faster,
        heavier error tail)."""
        self.check("nbSetMixedMode", self.lib.nbSetMixedModeCUDA(self._h, int(bool(exact))))

    def set_time_origin(self, previous_forward_time):
        """The orbiting bar's time origin (the reference's st->previousForwardTime)."""
        self.check("nbSetTimeOrigin", self.lib.nbSetTimeOriginCUDA(self._h,
                                                                  float(previous_forward_time)))

    def set_walk_form(self, form=-1):
        """The FP64 walk's form (nbSetWalkFormCUDA): 0 the warp union, 1 per lane, 2 per lane
        with the next node's record loaded early, -1 chosen by timing the three over the first
        evaluations; the accelerations are the same bit for bit."""
        self.check("nbSetWalkForm", self.lib.nbSetWalkFormCUDA(self._h, int(form)))

    def walk_form(self):
        """The FP64 walk form in use (-1 while the automatic choice is undecided)."""
        f = ctypes.c_int()
        self.check("nbGetWalkForm", self.lib.nbGetWalkFormCUDA(self._h, ctypes.byref(f)))
        return f.value

    def set_step_graph(self, enable=True):
        """Whole steps replayed as one captured CUDA graph (nbSetStepGraphCUDA; the default)."""
        self.check("nbSetStepGraph", self.lib.nbSetStepGraphCUDA(self._h, int(bool(enable))))

    def set_step(self, step):
        """The step counter of a state resumed from a checkpoint (nbSetStepCUDA)."""
        self.check("nbSetStep", self.lib.nbSetStepCUDA(self._h, int(step)))

    # -- marshalling (nbMarshalBodies) --
    def set_bodies(self, pos, vel, mass, treeRSize=4.0):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        rc = self.lib.nbSetBodiesCUDA(self._h, _lib.ptr(pos), _lib.ptr(vel), _lib.ptr(mass),
                                      self.nbody, float(treeRSize))
        self.check("nbSetBodiesCUDA", rc)

    def marshal_bodies(self, bodytab, to_device, treeRSize=4.0):
        """bodytab: a writable buffer of n reference Body records (96 bytes each)."""
        buf = (ctypes.c_char * (96 * self.nbody)).from_buffer(bodytab)
        rc = self.lib.nbMarshalBodiesCUDA(self._h, ctypes.addressof(buf), self.nbody,
                                          int(bool(to_device)), float(treeRSize))
        self.check("nbMarshalBodiesCUDA", rc)

    def bodies(self, out=None):
        """(pos, vel) of every body; out: two C-contiguous float64 (n,3) arrays to fill (page-
        locked ones make the copy a direct DMA)."""
        if out is None:
            pos, vel = np.empty((self.nbody, 3)), np.empty((self.nbody, 3))
        else:
            pos, vel = out
            for a in out:
                assert a.dtype == np.float64 and a.flags.c_contiguous and a.shape == (self.nbody, 3)
        self.check("nbGetBodiesCUDA", self.lib.nbGetBodiesCUDA(self._h, _lib.ptr(pos), _lib.ptr(vel)))
        return pos, vel

    def accels(self):
        acc = np.empty((self.nbody, 3))
        self.check("nbGetAccelsCUDA", self.lib.nbGetAccelsCUDA(self._h, _lib.ptr(acc)))
        return acc

    # -- the step (nbGravMap / nbStepSystem / run loop) --
    def gravMap(self, ctx):
        return self.lib.nbGravMapCUDA(ctypes.byref(ctx.struct), self._h)

    def step(self, ctx):
        return self.lib.nbStepSystemCUDA(ctypes.byref(ctx.struct), self._h)

    def run_steps(self, ctx, nsteps):
        return self.lib.nbRunStepsCUDA(ctypes.byref(ctx.struct), self._h, int(nsteps))

    def run_system(self, ctx, nstep, time_evolve, params=None, data=None, use_best_like=False,
                   best_like_start=0.95, calibration_runs=0, keep_best_bodies=False):
        """The reference's forward evolution (nbRunSystemCUDA: nbody.c's calibration runs
        around nbRunSystemPlain with its best-likelihood scan): steps to nstep from the current
        step; with params and data, the likelihood of the result.  Returns (status, dict) with
        result / final / best (histogram.TERMS arrays), best_time, best_step, best_count,
        previous_forward_time and runs."""
        rp = _lib.RunParams(int(nstep), int(bool(use_best_like)), float(time_evolve),
                            float(best_like_start), int(calibration_runs),
                            int(bool(keep_best_bodies)))
        res = _lib.RunResult()
        hp = params.struct() if params is not None else None
        dh = data.struct() if data is not None else None
        rc = self.lib.nbRunSystemCUDA(ctypes.byref(ctx.struct), self._h, ctypes.byref(rp),
                                      ctypes.byref(hp) if hp is not None else None,
                                      ctypes.byref(dh) if dh is not None else None,
                                      ctypes.byref(res))
        out = {"result": np.array(res.result[:]), "final": np.array(res.final[:]),
               "best": np.array(res.best[:]), "best_time": res.bestTime,
               "best_step": res.bestStep, "best_count": res.bestCount,
               "previous_forward_time": res.previousForwardTime, "runs": res.runs}
        return rc, out

    def best_bodies(self):
        """Positions and velocities (n, 3) at the best likelihood of the last run_system with
        keep_best_bodies (the reference's bestLikelihoodBodyTab)."""
        pos = np.empty((self.nbody, 3))
        vel = np.empty((self.nbody, 3))
        self.check("nbGetBestBodiesCUDA",
                   self.lib.nbGetBestBodiesCUDA(self._h, _lib.ptr(pos), _lib.ptr(vel)))
        return pos, vel

    def makeTree(self, ctx):
        return self.lib.nbMakeTreeCUDA(ctypes.byref(ctx.struct), self._h)

    # -- introspection --
    def tree_info(self):
        info = _lib.TreeInfo()
        self.check("nbTreeInfoCUDA", self.lib.nbTreeInfoCUDA(self._h, ctypes.byref(info)))
        return info

    def tree(self):
        n = self.tree_info().nNodes
        out = {"pos": np.empty((n, 3)), "mass": np.empty(n), "rcrit2": np.empty(n),
               "quad": np.empty((n, 6)), "next": np.empty(n, np.int32),
               "body": np.empty(n, np.int32), "depth": np.empty(n, np.int32)}
        rc = self.lib.nbGetTreeCUDA(self._h, *[_lib.ptr(out[k]) for k in
                                               ("pos", "mass", "rcrit2", "quad", "next", "body",
                                                "depth")])
        self.check("nbGetTreeCUDA", rc)
        return out

    @property
    def step_count(self):
        return self.tree_info().step

    def walk_time_ms(self):
        ms = ctypes.c_double()
        n = ctypes.c_int()
        self.lib.nbLastWalkTimeCUDA(self._h, ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value

    def step_time_ms(self):
        """Device time of the whole last gravMap / step / run_steps call."""
        ms = ctypes.c_double()
        self.lib.nbLastStepTimeCUDA(self._h, ctypes.byref(ms))
        return ms.value

    def energy(self, ctx):
        """(kinetic, self-gravity, external) energy of the current state, FP64 direct sum."""
        out = (ctypes.c_double * 3)()
        self.check("nbEnergy", self.lib.nbEnergyCUDA(ctypes.byref(ctx.struct), self._h, out))
        return tuple(out)

    # -- Lambda-Beta histogram and likelihood (nbCreateHistogram / nbSystemLikelihood) --
    def set_types(self, types):
        t = np.ascontiguousarray(types, dtype=np.int32)
        assert len(t) == self.nbody
        rc = getattr(self.lib, self._fn("SetTypes"))(self._h, _lib.ptr(t))
        self.check("%s(types)" % self._kind, rc)

    def histogram(self, params, components=False):
        """counts (ndwarfs, nBins), totals (ndwarfs, 2) = (in range, light), massPerParticle;
        with components=True also histograms 1..7 (ndwarfs, 7, 2, nBins) as (values, errors):
        the beta and line-of-sight velocity dispersions and, when params compare averages, the
        averages (zeros where not built)."""
        nd = getattr(self, "ndwarfs", 1)
        counts = np.zeros((nd, params.nbins), dtype=np.uint32)
        totals = np.zeros((nd, 2), dtype=np.uint32)
        mpp = np.zeros(nd)
        comps = np.zeros((nd, _lib.HIST_COMPONENTS, 2, params.nbins)) if components else None
        hp = params.struct()
        self.check("histogram", getattr(self.lib, self._fn("Histogram"))(
            self._h, ctypes.byref(hp), _lib.ptr(counts), _lib.ptr(totals), _lib.ptr(mpp),
            _lib.ptr(comps) if components else None))
        if components:
            return counts, totals, mpp, comps
        return counts, totals, mpp

    def likelihood(self, params, data):
        """(ndwarfs, 11): the reference's likelihood array -- likelihood, EMD component, cost
        component, beta dispersion, velocity dispersion, beta average, line-of-sight velocity,
        distance, dec and RA proper motion (NaN where not compared) -- then the EMD itself
        (histogram.TERMS).  Positive; lower is better."""
        nd = getattr(self, "ndwarfs", 1)
        out = np.zeros((nd, _lib.LIKELIHOOD_TERMS))
        hp = params.struct()
        dh = data.struct()
        self.check("likelihood", getattr(self.lib, self._fn("Likelihood"))(
            self._h, ctypes.byref(hp), ctypes.byref(dh), _lib.ptr(out)))
        return out

    _kind = "nbState"

    @staticmethod
    def _fn(name):
        return "nb%sCUDA" % name

    def direct_sample(self, eps2, targets):
        """FP64 direct-sum self-gravity at the given body indices (accuracy oracle)."""
        targets = np.ascontiguousarray(targets, dtype=np.int32)
        acc = np.empty((len(targets), 3))
        rc = self.lib.nbDirectSampleCUDA(self._h, float(eps2), _lib.ptr(targets), len(targets),
                                         _lib.ptr(acc))
        self.check("nbDirectSampleCUDA", rc)
        return acc

    def set_counting(self, enable):
        self.lib.nbSetCountingCUDA(self._h, int(bool(enable)))

    def interaction_counts(self):
        """(body-body, body-cell, visits) of the last force evaluation with counting on."""
        return self.walk_stats()[:3]

    def walk_stats(self):
        """(body-body, body-cell, visits, warp iterations) of the last counted evaluation."""
        v = [ctypes.c_ulonglong() for _ in range(4)]
        self.lib.nbInteractionCountsCUDA(self._h, *[ctypes.byref(x) for x in v])
        return tuple(x.value for x in v)


class NBodyBatch:
    """Many independent dwarfs stepped together on one GPU (nbBatch*CUDA): every phase of the
    step is one launch over all dwarfs, and run_steps can replay each step as one captured CUDA
    graph.  No counterpart in the reference, which runs one dwarf per process; each dwarf here
    gets the same accelerations as an NBodyState holding it alone.

    dwarfs: a list of (nbody, eps2, timestep, treeRSize).  Bodies are concatenated arrays,
    dwarf 0's bodies first: pos (N,3), vel (N,3), mass (N,)."""

    def __init__(self, dwarfs, device=0):
        self.lib = _lib.load()
        arr = (_lib.Dwarf * len(dwarfs))()
        for k, (nb, eps2, dt, rsize) in enumerate(dwarfs):
            arr[k].nbody, arr[k].eps2, arr[k].timestep, arr[k].treeRSize = int(nb), eps2, dt, rsize
        self.counts = np.array([int(d[0]) for d in dwarfs], dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)])
        self.nbody = int(self.offsets[-1])
        self.ndwarfs = len(dwarfs)
        self.device = device
        h = ctypes.c_void_p()
        rc = self.lib.nbBatchCreateCUDA(ctypes.byref(h), device, arr, len(dwarfs))
        if rc:
            raise NBodyError("nbBatchCreateCUDA", rc)
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.nbBatchDestroyCUDA(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    check = staticmethod(NBodyState.check)

    def set_bodies(self, pos, vel, mass):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        assert len(mass) == self.nbody
        self.check("nbBatchSetBodiesCUDA", self.lib.nbBatchSetBodiesCUDA(
            self._h, _lib.ptr(pos), _lib.ptr(vel), _lib.ptr(mass)))

    def bodies(self):
        pos = np.empty((self.nbody, 3))
        vel = np.empty((self.nbody, 3))
        self.check("nbBatchGetBodiesCUDA", self.lib.nbBatchGetBodiesCUDA(
            self._h, _lib.ptr(pos), _lib.ptr(vel), None))
        return pos, vel

    def accels(self):
        acc = np.empty((self.nbody, 3))
        self.check("nbBatchGetBodiesCUDA", self.lib.nbBatchGetBodiesCUDA(
            self._h, None, None, _lib.ptr(acc)))
        return acc

    def gravMap(self, ctx):
        return self.lib.nbBatchGravMapCUDA(ctypes.byref(ctx.struct), self._h)

    def run_steps(self, ctx, nsteps, graph=True):
        return self.lib.nbBatchRunStepsCUDA(ctypes.byref(ctx.struct), self._h, int(nsteps),
                                            int(bool(graph)))

    def dwarf_info(self):
        """Per dwarf: status bits, root size, root node index, node count."""
        st = np.zeros(self.ndwarfs, dtype=np.int32)
        rs = np.zeros(self.ndwarfs)
        root = np.zeros(self.ndwarfs, dtype=np.int32)
        nodes = np.zeros(self.ndwarfs, dtype=np.int32)
        self.check("nbBatchDwarfInfoCUDA", self.lib.nbBatchDwarfInfoCUDA(
            self._h, _lib.ptr(st), _lib.ptr(rs), _lib.ptr(root), _lib.ptr(nodes)))
        return st, rs, root, nodes

    def set_tuning(self, group_max=32, list_cap=64, blocks_per_sm=0):
        self.check("nbBatchSetTuningCUDA", self.lib.nbBatchSetTuningCUDA(
            self._h, int(group_max), int(list_cap), int(blocks_per_sm)))

    def set_walk_form(self, form=0):
        """nbBatchSetWalkFormCUDA: the FP64 walk's form for every dwarf (0 warp union, 1 per
        lane, 2 per lane loading the next record early); the accelerations are the same bit
        for bit."""
        self.check("nbBatchSetWalkFormCUDA", self.lib.nbBatchSetWalkFormCUDA(self._h, int(form)))

    def set_mixed_mode(self, exact=True):
        """nbBatchSetMixedModeCUDA: as NBodyState.set_mixed_mode for every dwarf."""
        self.check("nbBatchSetMixedModeCUDA",
                   self.lib.nbBatchSetMixedModeCUDA(self._h, int(bool(exact))))

    def autotune(self, ctx):
        """nbBatchAutotuneCUDA: (groupMax, listCap, blocksPerSM, walk ms) of the fastest."""
        g, l, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = ctypes.c_double()
        self.check("nbBatchAutotune", self.lib.nbBatchAutotuneCUDA(
            ctypes.byref(ctx.struct), self._h, ctypes.byref(g), ctypes.byref(l), ctypes.byref(b),
            ctypes.byref(ms)))
        return g.value, l.value, b.value, ms.value

    def tuning(self):
        g, l, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.nbBatchGetTuningCUDA(self._h, ctypes.byref(g), ctypes.byref(l), ctypes.byref(b))
        return g.value, l.value, b.value

    def step_time_ms(self):
        ms = ctypes.c_double()
        self.lib.nbBatchLastStepTimeCUDA(self._h, ctypes.byref(ms))
        return ms.value

    def generate(self, dwarfs):
        """Sample every dwarf on the GPU in one launch per phase (nbBatchGenerateDwarfsCUDA):
        dwarfs is a list of plummer_dwarf_struct()s or mixed_dwarf_struct()s matching the
        batch's sizes."""
        if dwarfs and isinstance(dwarfs[0], _lib.MixedDwarf):
            arr = (_lib.MixedDwarf * len(dwarfs))(*dwarfs)
            self.check("nbBatchGenerateMixedDwarfs",
                       self.lib.nbBatchGenerateMixedDwarfsCUDA(self._h, arr))
            return
        arr = (_lib.PlummerDwarf * len(dwarfs))(*dwarfs)
        self.check("nbBatchGenerateDwarfs", self.lib.nbBatchGenerateDwarfsCUDA(self._h, arr))

    def run_system(self, ctx, nstep, time_evolve, params=None, data=None, use_best_like=False,
                   best_like_start=0.95, calibration_runs=0, keep_best_bodies=False, graph=True):
        """NBodyState.run_system for every dwarf at once (nbBatchRunSystemCUDA): returns
        (status, [dict per dwarf]) with the keys of NBodyState.run_system."""
        rp = _lib.RunParams(int(nstep), int(bool(use_best_like)), float(time_evolve),
                            float(best_like_start), int(calibration_runs),
                            int(bool(keep_best_bodies)))
        res = (_lib.RunResult * self.ndwarfs)()
        hp = params.struct() if params is not None else None
        dh = data.struct() if data is not None else None
        rc = self.lib.nbBatchRunSystemCUDA(ctypes.byref(ctx.struct), self._h, ctypes.byref(rp),
                                           ctypes.byref(hp) if hp is not None else None,
                                           ctypes.byref(dh) if dh is not None else None,
                                           int(bool(graph)), res)
        out = [{"result": np.array(r.result[:]), "final": np.array(r.final[:]),
                "best": np.array(r.best[:]), "best_time": r.bestTime, "best_step": r.bestStep,
                "best_count": r.bestCount, "previous_forward_time": r.previousForwardTime,
                "runs": r.runs} for r in res]
        return rc, out

    def set_lmc(self, positions, velocities, shifts):
        """Every dwarf's LMC (nbBatchSetLMCCUDA): positions and velocities (ndwarfs, 3), reflex
        accelerations (ndwarfs, k, 3)."""
        p = np.ascontiguousarray(positions, dtype=np.float64).reshape(self.ndwarfs, 3)
        v = np.ascontiguousarray(velocities, dtype=np.float64).reshape(self.ndwarfs, 3)
        sh = np.ascontiguousarray(shifts, dtype=np.float64).reshape(self.ndwarfs, -1, 3)
        self.check("nbBatchSetLMC", self.lib.nbBatchSetLMCCUDA(self._h, _lib.ptr(p), _lib.ptr(v),
                                                               _lib.ptr(sh), sh.shape[1]))

    def lmc(self):
        """Every dwarf's LMC position and velocity, (ndwarfs, 3) each (nbBatchGetLMCCUDA)."""
        p, v = np.empty((self.ndwarfs, 3)), np.empty((self.ndwarfs, 3))
        self.check("nbBatchGetLMC", self.lib.nbBatchGetLMCCUDA(self._h, _lib.ptr(p), _lib.ptr(v)))
        return p, v

    def best_bodies(self):
        """Every dwarf's bodies at its best likelihood (nbBatchGetBestBodiesCUDA)."""
        n = int(self.offsets[-1])
        pos, vel = np.empty((n, 3)), np.empty((n, 3))
        self.check("nbBatchGetBestBodies", self.lib.nbBatchGetBestBodiesCUDA(
            self._h, _lib.ptr(pos), _lib.ptr(vel)))
        return pos, vel

    def set_time_origin(self, previous_forward_time):
        self.check("nbBatchSetTimeOrigin", self.lib.nbBatchSetTimeOriginCUDA(
            self._h, float(previous_forward_time)))

    _kind = "nbBatch"
    set_types = NBodyState.set_types
    histogram = NBodyState.histogram
    likelihood = NBodyState.likelihood

    @staticmethod
    def _fn(name):
        return "nbBatch%sCUDA" % name


NO_ALLOC_MAX_POINTS = 65536       # the static staging area of nbExtAccelerationNoAllocCUDA


def ext_acceleration(potential, pos, device=0, no_alloc=False):
    """nbExtAcceleration (nbody/src/nbody_potential.c:627) at many positions, on the GPU.
    no_alloc: through nbExtAccelerationNoAllocCUDA (no device allocation per call: the form
    for loops of small calls such as orbit integration); that entry point takes at most
    NO_ALLOC_MAX_POINTS (65,536) positions per call, so more positions are evaluated in
    consecutive chunks of that size."""
    lib = _lib.load()
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    acc = np.empty_like(pos)
    if not no_alloc:
        rc = lib.nbExtAccelerationCUDA(ctypes.byref(potential), _lib.ptr(pos), _lib.ptr(acc),
                                       len(pos), device)
        NBodyState.check("nbExtAcceleration", rc)
        return acc
    for lo in range(0, len(pos), NO_ALLOC_MAX_POINTS):
        p, a = pos[lo:lo + NO_ALLOC_MAX_POINTS], acc[lo:lo + NO_ALLOC_MAX_POINTS]
        rc = lib.nbExtAccelerationNoAllocCUDA(ctypes.byref(potential), _lib.ptr(p), _lib.ptr(a),
                                              len(p), device)
        NBodyState.check("nbExtAccelerationNoAlloc", rc)
    return acc


def emd(sig1, sig2, device=0):
    """emdCalc (nbody/src/nbody_emd.c:1207-1268) of two signatures, (n, 3) arrays of (weight,
    lambda, beta) rows, on the GPU (nbEmdCalcCUDA): the reference's transportation simplex with
    the L2 ground distance; NaN where the reference's is invalid."""
    lib = _lib.load()
    a = np.ascontiguousarray(sig1, dtype=np.float64).reshape(-1, 3)
    b = np.ascontiguousarray(sig2, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(1)
    NBodyState.check("nbEmdCalc", lib.nbEmdCalcCUDA(_lib.ptr(a), len(a), _lib.ptr(b), len(b),
                                                    _lib.ptr(out), device))
    return float(out[0])


def peak_fma_tflops(fp64=True, device=0):
    """Measured DFMA (fp64) or FFMA throughput of the device, TFLOP/s."""
    out = ctypes.c_double()
    rc = _lib.load().nbPeakFmaCUDA(device, int(bool(fp64)), ctypes.byref(out))
    NBodyState.check("nbPeakFmaCUDA", rc)
    return out.value


def kernel_launches():
    """Kernel launches issued by libnbody_b200.so since it was loaded."""
    return int(_lib.load().nbKernelLaunchesCUDA())
