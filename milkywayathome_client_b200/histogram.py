"""Lambda-Beta histograms: parameters, the reference's histogram file format, data histograms.

HistogramParams mirrors the Lua HistogramParams.create{...} of the reference
(nbody/src/nbody_lua_types/nbody_lua_histogram_params.c); read_histogram parses the
normalised-counts columns of a histogram file as nbReadHistogram does
(nbody/src/nbody_histogram.c:1140-1571: the `<histogram>` block, its `n =`,
`massPerParticle =`, `totalSimulated =`, `lambdaBins =`, `betaBins =` lines, then one row per
bin: useBin, lambda, beta, normalised count, count error, ...); data_from_counts makes the
same data histogram from counts, as nbNormalizeHistogram does (:626-661), for a histogram
produced by a simulation (the likelihood target of a parameter fit).
"""
import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib


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

    def struct(self):
        h = _lib.HistParams()
        for f in ("phi", "theta", "psi", "lambdaStart", "lambdaEnd", "betaStart", "betaEnd",
                  "sunGCDist"):
            setattr(h, f, float(getattr(self, f)))
        h.lambdaBins, h.betaBins = int(self.lambdaBins), int(self.betaBins)
        return h

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
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nbins(self):
        return len(self.variable)

    def struct(self):
        """NBodyCudaDataHistogram over this histogram's arrays (kept alive by the object)."""
        use = np.ascontiguousarray(self.useBin, dtype=np.int32)
        lam = np.ascontiguousarray(self.lambda_, dtype=np.float64)
        var = np.ascontiguousarray(self.variable, dtype=np.float64)
        err = np.ascontiguousarray(self.err, dtype=np.float64)
        self._keep = [use, lam, var, err]
        d = _lib.DataHist()
        d.nBins = len(var)
        d.totalNum = int(self.totalNum)
        d.massPerParticle = float(self.massPerParticle)
        d.useBin = use.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        d.lambda_ = lam.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.variable = var.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.err = err.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        return d


def read_histogram(path):
    """The normalised-counts histogram of a reference histogram file."""
    header = {}
    rows = []
    inside = False
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
            if "=" in s:
                k, v = (t.strip() for t in s.split("=", 1))
                header[k] = v
                continue
            if s.startswith("!"):
                continue
            rows.append([float(t) for t in s.split()])
    rows = np.array(rows)
    return DataHistogram(totalNum=int(header["n"]), massPerParticle=float(header["massPerParticle"]),
                         totalSimulated=int(header.get("totalSimulated", 0)),
                         useBin=rows[:, 0].astype(np.int32), lambda_=rows[:, 1], beta=rows[:, 2],
                         variable=rows[:, 3], err=rows[:, 4])


def normalized_error(n, total_histogram, total_simulated):
    """nbNormalizedHistogramError (nbody/src/nbody_histogram.c:60-64): binomial errors."""
    if n == 0:
        return math.sqrt((1.0 / total_simulated) * (1.0 - 1.0 / total_simulated)) / total_histogram
    rn = float(n)
    return math.sqrt(rn * (rn / total_simulated) * (1.0 - rn / total_simulated)) / total_histogram


def data_from_counts(params, counts, total_simulated, mass_per_particle):
    """A data histogram from a simulation's counts (nbNormalizeHistogram)."""
    counts = np.asarray(counts, dtype=np.int64)
    total = int(counts.sum())
    lam, beta = params.centres()
    var = counts / float(total) if total else np.zeros(len(counts))
    # the reference indexes the error by the lambda index (data[i].rawCount, :652), which is
    # the bin index when there is one beta bin
    li = np.repeat(np.arange(params.lambdaBins), params.betaBins)
    err = np.array([normalized_error(int(counts[i]), float(total), float(total_simulated))
                    for i in li])
    return DataHistogram(totalNum=total, massPerParticle=float(mass_per_particle),
                         totalSimulated=int(total_simulated),
                         useBin=np.ones(len(counts), dtype=np.int32), lambda_=lam, beta=beta,
                         variable=var, err=err)
