"""Lambda-Beta histograms: parameters, the reference's histogram file format, data histograms.

HistogramParams mirrors the Lua HistogramParams.create{...} of the reference
(nbody/src/nbody_lua_types/nbody_lua_histogram_params.c) together with the NBodyCtx fields
that select and tune the likelihood's comparisons (useBetaDisp ... usePropMot, the sigma
cut-offs, dispersion corrections and IterMax, the Sun's velocity and the NGP angles;
defaults of nbody/include/nbody_defaults.h).  read_histogram parses a histogram file as
nbReadHistogram does (nbody/src/nbody_histogram.c:1140-1571): the `<histogram>` block, its
`n =`, `massPerParticle =`, `totalSimulated =`, `lambdaBins =`, `betaBins =`,
`betaDispBins =` and `hasPM =` lines, a `!` line marking the extended format, then one row
per bin: useBin, lambda, beta, then value and error of the normalised counts and of
histograms 1..2 (the default format) or 1..5 (extended) or 1..7 (extended with proper
motions).  data_from_counts makes the same data histogram from a simulation's counts and
comparison histograms, as nbNormalizeHistogram does (:626-661), for a histogram produced by
a simulation (the likelihood target of a parameter fit).
"""
import ctypes
import math
import re
from dataclasses import dataclass, field

import numpy as np

from . import _lib


COMPONENTS = ("betaDisp", "velDisp", "vlos", "betaAvg", "dist", "muDec", "muRA")
TERMS = ("likelihood", "emd_component", "cost", "beta_disp", "vel_disp", "beta_avg", "vlos",
         "distance", "pm_dec", "pm_ra", "emd")


@dataclass
class HistogramParams:
    phi: float = 128.79
    theta: float = 54.39
    psi: float = 90.70
    lambdaStart: float = -50.0
    lambdaEnd: float = 50.0
    lambdaBins: int = 34
    betaStart: float = -15.0
    betaEnd: float = 15.0
    betaBins: int = 1
    sunGCDist: float = 8.0
    # likelihood comparisons and their outlier rejection (NBodyCtx of the reference)
    useBetaDisp: bool = True
    useVelDisp: bool = False
    useBetaComp: bool = False
    useVlos: bool = False
    useDist: bool = False
    usePropMot: bool = False
    IterMax: int = 6
    BetaSigma: float = 2.5
    VelSigma: float = 2.5
    DistSigma: float = 2.5
    PMSigma: float = 2.5
    BetaCorrect: float = 1.111
    VelCorrect: float = 1.111
    DistCorrect: float = 1.111
    PMCorrect: float = 1.111
    sunVelx: float = 10.3
    sunVely: float = 229.2
    sunVelz: float = 6.9
    NGPdec: float = 27.4 * math.pi / 180.0
    NGPra: float = 192 * math.pi / 180.0
    lNCP: float = 123 * math.pi / 180.0

    def struct(self):
        h = _lib.HistParams()
        for f in ("phi", "theta", "psi", "lambdaStart", "lambdaEnd", "betaStart", "betaEnd",
                  "sunGCDist", "sunVelx", "sunVely", "sunVelz", "NGPdec", "NGPra", "lNCP"):
            setattr(h, f, float(getattr(self, f)))
        h.lambdaBins, h.betaBins = int(self.lambdaBins), int(self.betaBins)
        for f in ("useBetaDisp", "useVelDisp", "useBetaComp", "useVlos", "useDist", "usePropMot"):
            setattr(h, f, int(bool(getattr(self, f))))
        h.iterMax = int(self.IterMax)
        h.betaSigma, h.velSigma = float(self.BetaSigma), float(self.VelSigma)
        h.distSigma, h.pmSigma = float(self.DistSigma), float(self.PMSigma)
        h.betaCorrect, h.velCorrect = float(self.BetaCorrect), float(self.VelCorrect)
        h.distCorrect, h.pmCorrect = float(self.DistCorrect), float(self.PMCorrect)
        return h

    def builds_averages(self):
        """Whether histograms 3..7 are built (nbCreateHistogram, :783-828)."""
        return bool(self.useVlos or self.useBetaComp or self.useDist or self.usePropMot)

    @property
    def nbins(self):
        return self.lambdaBins * self.betaBins

    def centres(self):
        """Bin centres (lambda, beta) in bin order (lambda-major), as nbNormalizeHistogram."""
        ls = (self.lambdaEnd - self.lambdaStart) / self.lambdaBins
        bs = (self.betaEnd - self.betaStart) / self.betaBins
        lam = np.repeat((np.arange(self.lambdaBins) + 0.5) * ls + self.lambdaStart, self.betaBins)
        beta = np.tile((np.arange(self.betaBins) + 0.5) * bs + self.betaStart, self.lambdaBins)
        return lam, beta


@dataclass
class DataHistogram:
    totalNum: int
    massPerParticle: float
    totalSimulated: int
    useBin: np.ndarray
    lambda_: np.ndarray
    beta: np.ndarray
    variable: np.ndarray
    err: np.ndarray
    # histograms 1..7 (COMPONENTS order): (values, errors) or None where the file has none
    components: list = field(default_factory=lambda: [None] * 7)
    betaDispBins: int = 0
    # "EMDRange = {...}": the EMD's lambda ranges as pairs of bounds (None: every bin)
    emdRange: np.ndarray = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nbins(self):
        return len(self.variable)

    def struct(self):
        """NBodyCudaDataHistogram over this histogram's arrays (kept alive by the object)."""
        dp = ctypes.POINTER(ctypes.c_double)
        use = np.ascontiguousarray(self.useBin, dtype=np.int32)
        lam = np.ascontiguousarray(self.lambda_, dtype=np.float64)
        beta = np.ascontiguousarray(self.beta, dtype=np.float64)
        var = np.ascontiguousarray(self.variable, dtype=np.float64)
        err = np.ascontiguousarray(self.err, dtype=np.float64)
        keep = [use, lam, beta, var, err]
        d = _lib.DataHist()
        d.nBins = len(var)
        d.totalNum = int(self.totalNum)
        d.massPerParticle = float(self.massPerParticle)
        d.useBin = use.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        d.lambda_ = lam.ctypes.data_as(dp)
        d.beta = beta.ctypes.data_as(dp)
        d.variable = var.ctypes.data_as(dp)
        d.err = err.ctypes.data_as(dp)
        d.betaDispBins = int(self.betaDispBins)
        for k, comp in enumerate(self.components):
            if comp is None:
                d.compVariable[k] = dp()
                d.compErr[k] = dp()
                continue
            v = np.ascontiguousarray(comp[0], dtype=np.float64)
            e = np.ascontiguousarray(comp[1], dtype=np.float64)
            if len(v) != len(var) or len(e) != len(var):
                raise ValueError("component %s has %d/%d bins, expected %d"
                                 % (COMPONENTS[k], len(v), len(e), len(var)))
            keep += [v, e]
            d.compVariable[k] = v.ctypes.data_as(dp)
            d.compErr[k] = e.ctypes.data_as(dp)
        d.nRange = 0
        if self.emdRange is not None:
            rng = np.ascontiguousarray(self.emdRange, dtype=np.float64)
            keep.append(rng)
            d.nRange = len(rng)
            d.emdRange = rng.ctypes.data_as(dp)
        self._keep = keep
        return d


_libc = None


def _strtof(text):
    """The C library's strtof (decimal to the nearest float, then exactly to double)."""
    global _libc
    if _libc is None:
        _libc = ctypes.CDLL(None)
        _libc.strtof.restype = ctypes.c_float
        _libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    return float(_libc.strtof(text.encode(), None))


def parse_emd_range(value):
    """params.EMDRange as nbReadHistogram reads an "EMDRange = {...}" line
    (nbody/src/nbody_histogram.c:1290-1301 and 1547-1561): the first token without white space
    after the brace, cut at any of {}()[], and space, each piece parsed by strtof."""
    v = value.strip()
    if not v.startswith("{"):
        return None
    words = v[1:].split()
    token = words[0] if words else ""
    return np.array([_strtof(t) for t in re.split(r"[{}()\[\], ]", token) if t])


def read_histogram(path):
    """A reference histogram file (nbReadHistogram): counts and comparison histograms."""
    header = {}
    rows = []
    inside = False
    extended = False
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            if s.startswith("<histogram>"):
                inside = True
                continue
            if s.startswith("</histogram>"):
                break
            if not inside:
                continue
            if s.startswith("!"):
                extended = True
                continue
            if "=" in s:
                k, v = (t.strip() for t in s.split("=", 1))
                header[k] = v
                continue
            rows.append([float(t) for t in s.split()])
    has_pm = int(header.get("hasPM", 0)) == 1
    ncols = (19 if has_pm else 15) if extended else 9
    rows = np.array(rows)
    if rows.ndim != 2 or rows.shape[1] != ncols:
        raise ValueError("%s: expected %d columns per bin, got %s" % (path, ncols, rows.shape))
    ncomp = (ncols - 5) // 2
    comps = [None] * 7
    for k in range(ncomp):
        comps[k] = (rows[:, 5 + 2 * k].copy(), rows[:, 6 + 2 * k].copy())
    return DataHistogram(totalNum=int(header["n"]), massPerParticle=float(header["massPerParticle"]),
                         totalSimulated=int(header.get("totalSimulated", 0)),
                         useBin=rows[:, 0].astype(np.int32), lambda_=rows[:, 1], beta=rows[:, 2],
                         variable=rows[:, 3], err=rows[:, 4], components=comps,
                         betaDispBins=int(header.get("betaDispBins", 0)),
                         emdRange=(parse_emd_range(header["EMDRange"])
                                   if "EMDRange" in header else None))


def write_histogram(path, params, data):
    """The <histogram> block as nbPrintHistogram writes it (nbody/src/nbody_histogram.c:516-599):
    counts and histograms 1..2, or all of 1..7 when the averages are present; a nonzero
    betaDispBins is written as the `betaDispBins =` line nbReadHistogram reads."""
    full = all(c is not None for c in data.components)
    with open(path, "w") as f:
        f.write("<histogram>\n")
        f.write("n = %u\n" % data.totalNum)
        f.write("massPerParticle = %12.15f\n" % data.massPerParticle)
        f.write("totalSimulated = %u\n" % data.totalSimulated)
        f.write("lambdaBins = %u\n" % params.lambdaBins)
        f.write("betaBins = %u\n" % params.betaBins)
        if data.betaDispBins:
            f.write("betaDispBins = %u\n" % data.betaDispBins)
        if data.emdRange is not None:         # float values, written to parse back exactly
            f.write("EMDRange = {%s}\n" % ",".join(repr(float(np.float32(v)))
                                                    for v in data.emdRange))
        if full:
            f.write("hasPM = 1\n!\n")
        ncomp = 7 if full else 2
        for i in range(data.nbins):
            vals = [data.variable[i], data.err[i]]
            for k in range(ncomp):
                comp = data.components[k]
                vals += [comp[0][i], comp[1][i]] if comp is not None else [0.0, 0.0]
            f.write("%d %12.15f %12.15f " % (int(data.useBin[i]), data.lambda_[i], data.beta[i]) +
                    " ".join("%12.15f" % v for v in vals) + "\n")
            if i % params.betaBins == params.betaBins - 1:
                f.write("\n")
        f.write("</histogram>\n")


def normalized_error(n, total_histogram, total_simulated):
    """nbNormalizedHistogramError (nbody/src/nbody_histogram.c:60-64): binomial errors."""
    if n == 0:
        return math.sqrt((1.0 / total_simulated) * (1.0 - 1.0 / total_simulated)) / total_histogram
    rn = float(n)
    return math.sqrt(rn * (rn / total_simulated) * (1.0 - rn / total_simulated)) / total_histogram


def data_from_counts(params, counts, total_simulated, mass_per_particle, components=None):
    """A data histogram from a simulation's counts (nbNormalizeHistogram) and, optionally, its
    comparison histograms (an array (7, 2, nBins) of values and errors, as
    NBodyState.histogram(components=True) returns them; histograms the simulation did not
    build are left out)."""
    counts = np.asarray(counts, dtype=np.int64)
    total = int(counts.sum())
    lam, beta = params.centres()
    var = counts / float(total) if total else np.zeros(len(counts))
    # the reference indexes the error by the lambda index (data[i].rawCount, :652), which is
    # the bin index when there is one beta bin
    li = np.repeat(np.arange(params.lambdaBins), params.betaBins)
    err = np.array([normalized_error(int(counts[i]), float(total), float(total_simulated))
                    for i in li])
    comps = [None] * 7
    if components is not None:
        components = np.asarray(components, dtype=np.float64)
        built = 7 if params.builds_averages() else 2
        for k in range(built):
            comps[k] = (components[k, 0].copy(), components[k, 1].copy())
    return DataHistogram(totalNum=total, massPerParticle=float(mass_per_particle),
                         totalSimulated=int(total_simulated),
                         useBin=np.ones(len(counts), dtype=np.int32), lambda_=lam, beta=beta,
                         variable=var, err=err, components=comps)
