"""ctypes bindings of the oracle -- TEST INFRASTRUCTURE ONLY.

Two checkers live under oracle/:
  * liboracle_nbody.so  -- nbody_oracle.c, the plain-C restatement of the reference's step;
  * _ref/libnbref.so    -- the reference's own CPU code compiled from its sources plus
                           ref_shim.c (present where oracle/ref.mk was run).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle_nbody.so")
REF_LIB = os.path.join(HERE, "_ref", "libnbref.so")
REF_EXE = os.path.join(HERE, "_ref", "milkyway_nbody")

_dp = ctypes.POINTER(ctypes.c_double)
# the reference's Body record (nbody/include/nbody_types.h:103-125), 96 bytes
BODY_DTYPE = np.dtype([("pos", "f8", 4), ("next", "u8"), ("mass", "f8"), ("type", "i2"),
                       ("pad", "i2"), ("id", "u4"), ("pad2", "u8"), ("vel", "f8", 4)])
_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def build_oracle():
    """Compile liboracle_nbody.so (make -C oracle)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "liboracle_nbody.so"], check=True)
    return ORACLE_LIB


_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            build_oracle()
        lib = ctypes.CDLL(ORACLE_LIB)
        lib.or_grav_map.restype = ctypes.c_int
        lib.or_grav_map.argtypes = [_vp, _vp, _vp, ctypes.c_int, _dp, _vp, _ip, _vp]
        lib.or_step.restype = ctypes.c_int
        lib.or_step.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int, _dp, _vp, ctypes.c_int, _ip]
        lib.or_tree.restype = ctypes.c_int
        lib.or_tree.argtypes = [_vp, _vp, _vp, ctypes.c_int, _dp, ctypes.c_int] + [_vp] * 7 + [_ip, _ip]
        lib.or_ext_accel.restype = None
        lib.or_ext_accel.argtypes = [_vp, _vp, _vp, ctypes.c_int]
        lib.or_pow_1p5.restype = ctypes.c_double
        lib.or_pow_1p5.argtypes = [ctypes.c_double]
        lib.or_sample_step.restype = ctypes.c_int
        lib.or_sample_step.argtypes = [_vp, _vp, _vp, ctypes.c_int, _dp, _vp, ctypes.c_int, _vp, _dp, _dp]
        lib.or_threads.restype = ctypes.c_int
        lib.or_threads.argtypes = []
        lib.or_pow_3.restype = ctypes.c_double
        lib.or_pow_3.argtypes = [ctypes.c_double]
        _oracle = lib
    return _oracle


def ref_available():
    return os.path.exists(REF_LIB)


def ref():
    """The reference's own code (oracle/_ref/libnbref.so); None when it was not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            return None
        lib = ctypes.CDLL(REF_LIB)
        sig = {
            "nbref_layout": (ctypes.c_int, [_vp, ctypes.c_int]),
            "nbref_state_new": (_vp, [_vp, _vp, _vp, _vp, _vp, ctypes.c_int]),
            "nbref_state_gravmap": (ctypes.c_int, [_vp]),
            "nbref_state_maketree": (ctypes.c_int, [_vp]),
            "nbref_state_step": (ctypes.c_int, [_vp, ctypes.c_int]),
            "nbref_state_get": (None, [_vp, _vp, _vp, _vp, _dp, _ip, _ip]),
            "nbref_state_set": (None, [_vp, _vp, _vp]),
            "nbref_state_masses": (None, [_vp, _vp, _vp]),
            "nbref_state_nbody": (ctypes.c_int, [_vp]),
            "nbref_state_tree": (ctypes.c_int, [_vp, ctypes.c_int] + [_vp] * 7),
            "nbref_state_tree_info": (None, [_vp, _dp, _ip, _ip]),
            "nbref_state_free": (None, [_vp]),
            "nbref_open_lua": (_vp, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint,
                                     ctypes.POINTER(ctypes.c_char_p), ctypes.c_int]),
            "nbref_handle_ctx": (None, [_vp, _vp, _ip, _dp]),
            "nbref_run": (ctypes.c_int, [_vp]),
            "nbref_handle_run_params": (None, [_vp, _ip, _dp, _ip]),
            "nbref_handle_like_params": (None, [_vp, _vp, _vp, _ip, _vp]),
            "nbref_likelihood": (ctypes.c_int, [_vp, _vp]),
            "nbref_handle_lmc": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int]),
            "nbref_handle_set_lmc": (None, [_vp, _vp, _vp, _vp, ctypes.c_int]),
            "nbref_pow_rn": (ctypes.c_double, [ctypes.c_double, ctypes.c_double]),
            "nbref_log_rn": (ctypes.c_double, [ctypes.c_double]),
            "nbref_atan_rn": (ctypes.c_double, [ctypes.c_double]),
            "nbref_ext_accel": (None, [_vp, _vp, _vp, ctypes.c_int]),
            "nbref_sample_step": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _dp, _dp]),
            "nbref_threads": (ctypes.c_int, []),
            "nbref_handle_set_hist": (None, [_vp, ctypes.c_char_p]),
            "nbref_state_bodytab": (_vp, [_vp]),
            "nbref_state_set_progress": (None, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
            "nbref_state_progress": (None, [_vp, _ip, _dp, _ip]),
            "nbref_write_checkpoint": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_char_p]),
            "nbref_read_checkpoint": (_vp, [ctypes.c_char_p]),
            "nbref_emd_calc": (ctypes.c_double, [_vp, ctypes.c_uint, _vp, ctypes.c_uint]),
            "nbref_histogram": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp,
                                               ctypes.POINTER(ctypes.c_uint)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _ref = lib
    return _ref


# ---- oracle (restatement) helpers ----
def grav_map(ctx, pos, mass, rsize, counts=False):
    """or_grav_map: returns (status, acc, rsize, incest[, (bb, bc, visits)])."""
    lib = oracle()
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    acc = np.zeros((len(mass), 3))
    rs = ctypes.c_double(rsize)
    inc = ctypes.c_int(0)
    cnt = np.zeros(3, dtype=np.uint64)
    rc = lib.or_grav_map(ctypes.byref(ctx), _p(pos), _p(mass), len(mass), ctypes.byref(rs),
                         _p(acc), ctypes.byref(inc), _p(cnt) if counts else None)
    out = (rc, acc, rs.value, inc.value)
    return out + ((int(cnt[0]), int(cnt[1]), int(cnt[2])),) if counts else out


def steps(ctx, pos, vel, mass, rsize, nsteps):
    """Initial or_grav_map then nsteps of or_step; returns (status, pos, vel, acc, rsize)."""
    lib = oracle()
    pos = np.array(pos, dtype=np.float64, order="C")
    vel = np.array(vel, dtype=np.float64, order="C")
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    acc = np.zeros((len(mass), 3))
    rs = ctypes.c_double(rsize)
    inc = ctypes.c_int(0)
    rc = lib.or_grav_map(ctypes.byref(ctx), _p(pos), _p(mass), len(mass), ctypes.byref(rs),
                         _p(acc), ctypes.byref(inc), None)
    if nsteps:
        rc |= lib.or_step(ctypes.byref(ctx), _p(pos), _p(vel), _p(mass), len(mass),
                          ctypes.byref(rs), _p(acc), nsteps, ctypes.byref(inc))
    return rc, pos, vel, acc, rs.value


def tree(ctx, pos, mass, rsize):
    lib = oracle()
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    cap = 4 * len(mass) + 64
    while True:
        out = {"pos": np.empty((cap, 3)), "mass": np.empty(cap), "rcrit2": np.empty(cap),
               "quad": np.empty((cap, 6)), "next": np.empty(cap, np.int32),
               "body": np.empty(cap, np.int32), "depth": np.empty(cap, np.int32)}
        rs = ctypes.c_double(rsize)
        md = ctypes.c_int(0)
        st = ctypes.c_int(0)
        n = lib.or_tree(ctypes.byref(ctx), _p(pos), _p(mass), len(mass), ctypes.byref(rs), cap,
                        *[_p(out[k]) for k in ("pos", "mass", "rcrit2", "quad", "next", "body",
                                               "depth")], ctypes.byref(md), ctypes.byref(st))
        if n < 0:
            cap = -n
            continue
        res = {k: v[:n] for k, v in out.items()}
        res.update(status=st.value, rsize=rs.value, maxDepth=md.value, nNodes=n)
        return res


def sample_step(ctx, pos, mass, rsize, idx):
    """or_sample_step: (status, t_tree, t_walk, acc_of_sample)."""
    lib = oracle()
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    acc = np.zeros((len(idx), 3))
    rs, tt, tw = ctypes.c_double(rsize), ctypes.c_double(), ctypes.c_double()
    rc = lib.or_sample_step(ctypes.byref(ctx), _p(pos), _p(mass), len(mass), ctypes.byref(rs),
                            _p(idx), len(idx), _p(acc), ctypes.byref(tt), ctypes.byref(tw))
    return rc, tt.value, tw.value, acc


def ext_accel(potential, pos):
    lib = oracle()
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    acc = np.empty_like(pos)
    lib.or_ext_accel(ctypes.byref(potential), _p(pos), _p(acc), len(pos))
    return acc


# ---- the reference itself ----
class RefState:
    """A reference NBodyState built from arrays (or from a Lua model via open_lua)."""

    def __init__(self, handle):
        self.lib = ref()
        self.h = handle
        if not handle:
            raise RuntimeError("reference state creation failed")

    @classmethod
    def create(cls, ctx, pos, vel, mass, types=None):
        lib = ref()
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        t = None if types is None else np.ascontiguousarray(types, dtype=np.int32)
        return cls(lib.nbref_state_new(ctypes.byref(ctx), _p(pos), _p(vel), _p(mass), _p(t),
                                       len(mass)))

    @classmethod
    def open_lua(cls, lua_file, hist_file, seed, args=()):
        lib = ref()
        arr = (ctypes.c_char_p * max(len(args), 1))(*[a.encode() for a in args])
        h = lib.nbref_open_lua(lua_file.encode(), hist_file.encode() if hist_file else None,
                               seed, arr, len(args))
        return cls(h)

    def close(self):
        if self.h:
            self.lib.nbref_state_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nbody(self):
        return self.lib.nbref_state_nbody(self.h)

    def gravmap(self):
        return self.lib.nbref_state_gravmap(self.h)

    def maketree(self):
        return self.lib.nbref_state_maketree(self.h)

    def step(self, n=1):
        return self.lib.nbref_state_step(self.h, n)

    def run(self):
        return self.lib.nbref_run(self.h)

    def get(self):
        n = self.nbody
        pos, vel, acc = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        rs, stp, inc = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
        self.lib.nbref_state_get(self.h, _p(pos), _p(vel), _p(acc), ctypes.byref(rs),
                                 ctypes.byref(stp), ctypes.byref(inc))
        return dict(pos=pos, vel=vel, acc=acc, rsize=rs.value, step=stp.value, incest=inc.value)

    def set_time_origin(self, t):
        self.lib.nbref_state_set_time_origin.argtypes = [ctypes.c_void_p, ctypes.c_double]
        self.lib.nbref_state_set_time_origin(self.h, float(t))

    def set(self, pos=None, vel=None):
        self.lib.nbref_state_set(self.h, _p(None if pos is None else np.ascontiguousarray(pos, dtype=np.float64)),
                                 _p(None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)))

    def masses(self):
        n = self.nbody
        m = np.empty(n)
        t = np.empty(n, np.int32)
        self.lib.nbref_state_masses(self.h, _p(m), _p(t))
        return m, t

    def tree(self):
        cap = 4 * self.nbody + 64
        while True:
            out = {"pos": np.empty((cap, 3)), "mass": np.empty(cap), "rcrit2": np.empty(cap),
                   "quad": np.empty((cap, 6)), "next": np.empty(cap, np.int32),
                   "body": np.empty(cap, np.int32), "depth": np.empty(cap, np.int32)}
            n = self.lib.nbref_state_tree(self.h, cap, *[_p(out[k]) for k in (
                "pos", "mass", "rcrit2", "quad", "next", "body", "depth")])
            if n < 0:
                cap = -n
                continue
            res = {k: v[:n] for k, v in out.items()}
            rs, cu, md = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
            self.lib.nbref_state_tree_info(self.h, ctypes.byref(rs), ctypes.byref(cu), ctypes.byref(md))
            res.update(rsize=rs.value, cellUsed=cu.value, maxDepth=md.value, nNodes=n)
            return res

    def sample_step(self, idx):
        """nbMakeTree + the walk for the bodies in idx; returns (status, t_tree, t_walk) s."""
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        tt, tw = ctypes.c_double(), ctypes.c_double()
        rc = self.lib.nbref_sample_step(self.h, _p(idx), len(idx), ctypes.byref(tt), ctypes.byref(tw))
        return rc, tt.value, tw.value

    def ctx(self, ctx_type):
        c = ctx_type()
        ns, te = ctypes.c_int(), ctypes.c_double()
        self.lib.nbref_handle_ctx(self.h, ctypes.byref(c), ctypes.byref(ns), ctypes.byref(te))
        return c, ns.value, te.value

    def run_params(self):
        """(useBestLike, BestLikeStart, calibrationRuns) of the context."""
        u, c = ctypes.c_int(), ctypes.c_int()
        b = ctypes.c_double()
        self.lib.nbref_handle_run_params(self.h, ctypes.byref(u), ctypes.byref(b), ctypes.byref(c))
        return bool(u.value), b.value, c.value

    def like_params(self):
        """The context's likelihood settings as HistogramParams keyword arguments."""
        flags = np.zeros(6, np.int32)
        sig = np.zeros(8)
        sun = np.zeros(7)
        it = ctypes.c_int()
        self.lib.nbref_handle_like_params(self.h, _p(flags), _p(sig), ctypes.byref(it), _p(sun))
        names = ("useBetaDisp", "useVelDisp", "useBetaComp", "useVlos", "useDist", "usePropMot")
        kw = {k: bool(v) for k, v in zip(names, flags)}
        kw.update(zip(("BetaSigma", "VelSigma", "DistSigma", "PMSigma", "BetaCorrect",
                       "VelCorrect", "DistCorrect", "PMCorrect"), (float(x) for x in sig)))
        kw.update(zip(("sunGCDist", "sunVelx", "sunVely", "sunVelz", "NGPdec", "NGPra", "lNCP"),
                      (float(x) for x in sun)))
        kw["IterMax"] = it.value
        return kw

    def lmc(self):
        """(position, velocity, shift (k, 3)) of the state's LMC; shift is empty without one."""
        p, v = np.zeros(3), np.zeros(3)
        n = self.lib.nbref_handle_lmc(self.h, _p(p), _p(v), None, 0)
        sh = np.zeros((max(n, 1), 3))
        self.lib.nbref_handle_lmc(self.h, _p(p), _p(v), _p(sh), n)
        return p, v, sh[:n]

    def set_lmc(self, position, velocity, shift):
        """Installs an LMC (position, velocity, reflex accelerations (k, 3)) on the state."""
        p = np.ascontiguousarray(position, dtype=np.float64).reshape(3)
        v = np.ascontiguousarray(velocity, dtype=np.float64).reshape(3)
        sh = np.ascontiguousarray(shift, dtype=np.float64).reshape(-1, 3)
        self.lib.nbref_handle_set_lmc(self.h, _p(p), _p(v), _p(sh), len(sh))

    def set_histogram_file(self, path):
        """The data histogram the next likelihood() compares with."""
        self.lib.nbref_handle_set_hist(self.h, path.encode() if path else None)

    def bodytab(self):
        """The state's Body[] as a numpy record view (96-byte records, the reference's layout):
        pos, next, mass, type, id, vel."""
        n = self.nbody
        buf = (ctypes.c_char * (96 * n)).from_address(self.lib.nbref_state_bodytab(self.h))
        return np.frombuffer(buf, dtype=BODY_DTYPE, count=n)

    def set_progress(self, step, rsize, tree_incest=0):
        self.lib.nbref_state_set_progress(self.h, int(step), float(rsize), int(tree_incest))

    def progress(self):
        """(step, tree root size, treeIncest) of the state."""
        stp, rs, inc = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        self.lib.nbref_state_progress(self.h, ctypes.byref(stp), ctypes.byref(rs), ctypes.byref(inc))
        return stp.value, rs.value, inc.value

    def write_checkpoint(self, path, tmp):
        rc = self.lib.nbref_write_checkpoint(self.h, path.encode(), tmp.encode())
        if rc:
            raise RuntimeError("nbWriteCheckpoint failed: %d" % rc)

    @classmethod
    def read_checkpoint(cls, path):
        return cls(ref().nbref_read_checkpoint(path.encode()))

    def histogram(self):
        """The reference's counts histogram of the state: dict of lambda, beta, variable,
        rawCount (per bin) and totalNum."""
        cap = 1 << 16
        lam, beta, var = np.zeros(cap), np.zeros(cap), np.zeros(cap)
        raw = np.zeros(cap, np.uint32)
        tot = ctypes.c_uint()
        n = self.lib.nbref_histogram(self.h, cap, _p(lam), _p(beta), _p(var), _p(raw), ctypes.byref(tot))
        if n < 0:
            raise RuntimeError("nbref_histogram failed: %d" % n)
        return dict(lambda_=lam[:n], beta=beta[:n], variable=var[:n], rawCount=raw[:n],
                    totalNum=tot.value)

    def likelihood(self):
        out = np.zeros(10)
        rc = self.lib.nbref_likelihood(self.h, _p(out))
        if rc:
            raise RuntimeError("nbref_likelihood failed: %d" % rc)
        return out


def ref_emd(sig1, sig2):
    """The reference's emdCalc of two (n, 3) signatures of (weight, lambda, beta) rows."""
    a = np.ascontiguousarray(sig1, dtype=np.float64).reshape(-1, 3)
    b = np.ascontiguousarray(sig2, dtype=np.float64).reshape(-1, 3)
    return ref().nbref_emd_calc(_p(a), len(a), _p(b), len(b))


def ref_ext_accel(potential, pos):
    lib = ref()
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    acc = np.empty_like(pos)
    lib.nbref_ext_accel(ctypes.byref(potential), _p(pos), _p(acc), len(pos))
    return acc
