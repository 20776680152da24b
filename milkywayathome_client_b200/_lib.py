"""ctypes view of the C ABI in include/nbody_b200.h (libnbody_b200.so).

The library is the product: every force evaluation and step runs in its sm_100a kernels.
There is no CPU fallback -- if the shared library is missing or cannot be loaded, loading
raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnbody_b200.so")

# NBodyStatus bits (nbody/include/nbody_types.h:541-583)
NBODY_SUCCESS = 0
NBODY_ERROR = 1 << 1
NBODY_TREE_STRUCTURE_ERROR = 1 << 3
NBODY_TREE_INCEST_FATAL = 1 << 4
NBODY_CAPABILITY_ERROR = 1 << 8
NBODY_UNIMPLEMENTED = 1 << 10
NBODY_UNSUPPORTED = 1 << 11
NBODY_USER_ERROR = 1 << 12
NBODY_MAX_DEPTH_ERROR = 1 << 16
NBODY_CELL_OVERFLOW_ERROR = 1 << 17
NBODY_CUDA_ERROR = 1 << 20
NBODY_TREE_INCEST_NONFATAL = 1 << 24
NBODY_STATUS_ALL_WARNINGS = 0xFF000000

STATUS_NAMES = {
    NBODY_ERROR: "NBODY_ERROR", NBODY_TREE_STRUCTURE_ERROR: "NBODY_TREE_STRUCTURE_ERROR",
    NBODY_TREE_INCEST_FATAL: "NBODY_TREE_INCEST_FATAL",
    NBODY_CAPABILITY_ERROR: "NBODY_CAPABILITY_ERROR", NBODY_UNIMPLEMENTED: "NBODY_UNIMPLEMENTED",
    NBODY_UNSUPPORTED: "NBODY_UNSUPPORTED", NBODY_USER_ERROR: "NBODY_USER_ERROR",
    NBODY_MAX_DEPTH_ERROR: "NBODY_MAX_DEPTH_ERROR",
    NBODY_CELL_OVERFLOW_ERROR: "NBODY_CELL_OVERFLOW_ERROR", NBODY_CUDA_ERROR: "NBODY_CUDA_ERROR",
    NBODY_TREE_INCEST_NONFATAL: "NBODY_TREE_INCEST_NONFATAL",
}


def status_is_fatal(rc):
    """nbStatusIsFatal (nbody/include/nbody_types.h:582)."""
    return (rc & ~NBODY_STATUS_ALL_WARNINGS & 0xFFFFFFFF) != 0


def status_names(rc):
    return [name for bit, name in sorted(STATUS_NAMES.items()) if rc & bit] or ["NBODY_SUCCESS"]


# criterion_t (nbody/include/nbody_types.h:171-178)
TREECODE, SW93, BH86, EXACT = 0, 1, 2, 3
CRITERIA = {"treecode": TREECODE, "sw93": SW93, "bh86": BH86, "exact": EXACT}
# ExternalPotentialType
POTENTIAL_DEFAULT, POTENTIAL_NONE, POTENTIAL_CUSTOM_LUA = 0, 1, 2
# spherical_t / disk_t / halo_t (nbody/include/nbody_potential_types.h)
NO_SPHERICAL, HERNQUIST_SPHERICAL, PLUMMER_SPHERICAL = 0, 1, 2
NO_DISK, MIYAMOTO_NAGAI_DISK = 0, 1
NO_HALO, LOGARITHMIC_HALO, NFW_HALO, TRIAXIAL_HALO, CAUSTIC_HALO = 0, 1, 2, 3, 4
ALLEN_SANTILLAN_HALO, WILKINSON_EVANS_HALO, NFW_MASS_HALO = 5, 6, 7
PLUMMER_HALO, HERNQUIST_HALO, NINKOVIC_HALO = 8, 9, 10
ORBITING_BAR = 5
PRECISION_FP64, PRECISION_MIXED = 0, 1


class Spherical(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("mass", ctypes.c_double), ("scale", ctypes.c_double)]


class Disk(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("mass", ctypes.c_double),
                ("scaleLength", ctypes.c_double), ("scaleHeight", ctypes.c_double),
                ("patternSpeed", ctypes.c_double), ("startAngle", ctypes.c_double)]


class Halo(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int)] + [(f, ctypes.c_double) for f in (
        "vhalo", "scaleLength", "flattenZ", "flattenY", "flattenX", "triaxAngle",
        "c1", "c2", "c3", "mass", "gamma", "lambda_", "rho0")]


class Potential(ctypes.Structure):
    _fields_ = [("sphere", Spherical), ("disk", Disk), ("disk2", Disk), ("halo", Halo)]


class Dwarf(ctypes.Structure):
    _fields_ = [("nbody", ctypes.c_int), ("eps2", ctypes.c_double),
                ("timestep", ctypes.c_double), ("treeRSize", ctypes.c_double)]


class PlummerDwarf(ctypes.Structure):
    _fields_ = [("nbody", ctypes.c_int), ("nbodyBaryon", ctypes.c_int),
                ("massLight", ctypes.c_double), ("scaleLight", ctypes.c_double),
                ("massDark", ctypes.c_double), ("scaleDark", ctypes.c_double),
                ("position", ctypes.c_double * 3), ("velocity", ctypes.c_double * 3),
                ("seed", ctypes.c_uint64)]


DWARF_PLUMMER, DWARF_NFW, DWARF_GEN_HERNQUIST, DWARF_CORED = 0, 1, 2, 4   # NBCUDA_DWARF_*


class DwarfComponent(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("reserved", ctypes.c_int),
                ("mass", ctypes.c_double), ("scaleLength", ctypes.c_double),
                ("r1", ctypes.c_double), ("rc", ctypes.c_double)]


class MixedDwarf(ctypes.Structure):
    _fields_ = [("nbody", ctypes.c_int), ("nbodyBaryon", ctypes.c_int),
                ("light", DwarfComponent), ("dark", DwarfComponent),
                ("position", ctypes.c_double * 3), ("velocity", ctypes.c_double * 3),
                ("seed", ctypes.c_uint64)]


HIST_COMPONENTS = 7       # NBODY_CUDA_HIST_COMPONENTS
LIKELIHOOD_TERMS = 11     # NBODY_CUDA_LIKELIHOOD_TERMS


class HistParams(ctypes.Structure):
    _fields_ = [("phi", ctypes.c_double), ("theta", ctypes.c_double), ("psi", ctypes.c_double),
                ("lambdaStart", ctypes.c_double), ("lambdaEnd", ctypes.c_double),
                ("betaStart", ctypes.c_double), ("betaEnd", ctypes.c_double),
                ("lambdaBins", ctypes.c_int), ("betaBins", ctypes.c_int),
                ("sunGCDist", ctypes.c_double),
                ("useBetaDisp", ctypes.c_int), ("useVelDisp", ctypes.c_int),
                ("useBetaComp", ctypes.c_int), ("useVlos", ctypes.c_int),
                ("useDist", ctypes.c_int), ("usePropMot", ctypes.c_int),
                ("iterMax", ctypes.c_int), ("reserved", ctypes.c_int),
                ("betaSigma", ctypes.c_double), ("velSigma", ctypes.c_double),
                ("distSigma", ctypes.c_double), ("pmSigma", ctypes.c_double),
                ("betaCorrect", ctypes.c_double), ("velCorrect", ctypes.c_double),
                ("distCorrect", ctypes.c_double), ("pmCorrect", ctypes.c_double),
                ("sunVelx", ctypes.c_double), ("sunVely", ctypes.c_double),
                ("sunVelz", ctypes.c_double), ("NGPdec", ctypes.c_double),
                ("NGPra", ctypes.c_double), ("lNCP", ctypes.c_double)]


class DataHist(ctypes.Structure):
    _fields_ = [("nBins", ctypes.c_int), ("totalNum", ctypes.c_uint),
                ("massPerParticle", ctypes.c_double),
                ("useBin", ctypes.POINTER(ctypes.c_int)),
                ("lambda_", ctypes.POINTER(ctypes.c_double)),
                ("variable", ctypes.POINTER(ctypes.c_double)),
                ("err", ctypes.POINTER(ctypes.c_double)),
                ("betaDispBins", ctypes.c_int), ("reserved", ctypes.c_int),
                ("compVariable", ctypes.POINTER(ctypes.c_double) * HIST_COMPONENTS),
                ("compErr", ctypes.POINTER(ctypes.c_double) * HIST_COMPONENTS),
                ("nRange", ctypes.c_int), ("reserved2", ctypes.c_int),
                ("emdRange", ctypes.POINTER(ctypes.c_double)),
                ("beta", ctypes.POINTER(ctypes.c_double))]


class RunParams(ctypes.Structure):
    _fields_ = [("nStep", ctypes.c_int), ("useBestLike", ctypes.c_int),
                ("timeEvolve", ctypes.c_double), ("bestLikeStart", ctypes.c_double),
                ("calibrationRuns", ctypes.c_int), ("keepBestBodies", ctypes.c_int)]


class RunResult(ctypes.Structure):
    _fields_ = [("result", ctypes.c_double * LIKELIHOOD_TERMS),
                ("final", ctypes.c_double * LIKELIHOOD_TERMS),
                ("best", ctypes.c_double * LIKELIHOOD_TERMS),
                ("bestTime", ctypes.c_double), ("previousForwardTime", ctypes.c_double),
                ("bestStep", ctypes.c_int), ("bestCount", ctypes.c_int),
                ("runs", ctypes.c_int), ("reserved", ctypes.c_int)]


class Ctx(ctypes.Structure):
    """NBodyCudaCtx: the NBodyCtx fields the step reads."""
    _fields_ = [("eps2", ctypes.c_double), ("theta", ctypes.c_double),
                ("timestep", ctypes.c_double), ("treeRSize", ctypes.c_double),
                ("criterion", ctypes.c_int), ("useQuad", ctypes.c_int),
                ("allowIncest", ctypes.c_int), ("potentialType", ctypes.c_int),
                ("precision", ctypes.c_int), ("reserved", ctypes.c_int),
                ("pot", Potential),
                ("lmc", ctypes.c_int), ("lmcDynaFric", ctypes.c_int),
                ("lmcMass", ctypes.c_double), ("lmcScale", ctypes.c_double),
                ("coulombLog", ctypes.c_double)]


class TreeInfo(ctypes.Structure):
    _fields_ = [("rsize", ctypes.c_double), ("nbody", ctypes.c_int),
                ("nTreeBodies", ctypes.c_int), ("cellUsed", ctypes.c_int),
                ("maxDepth", ctypes.c_int), ("nNodes", ctypes.c_int), ("step", ctypes.c_int),
                ("treeIncest", ctypes.c_int)]


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p
_ull = ctypes.POINTER(ctypes.c_ulonglong)

# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("nbInitCUDA", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int]),
    ("nbDestroyCUDA", None, [_vp]),
    ("nbMarshalBodiesCUDA", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    ("nbSetBodiesCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_double]),
    ("nbGetBodiesCUDA", ctypes.c_int, [_vp, _vp, _vp]),
    ("nbGetAccelsCUDA", ctypes.c_int, [_vp, _vp]),
    ("nbSetBodiesDeviceCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_double]),
    ("nbGetBodiesDeviceCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("nbGravMapCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp]),
    ("nbStepSystemCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp]),
    ("nbRunStepsCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp, ctypes.c_int]),
    ("nbMakeTreeCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp]),
    ("nbGravVJPCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp, _vp, _vp, _vp]),
    ("nbEnergyCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp, _dp]),
    ("nbBatchCreateCUDA", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                         ctypes.POINTER(Dwarf), ctypes.c_int]),
    ("nbBatchDestroyCUDA", ctypes.c_int, [_vp]),
    ("nbBatchSetBodiesCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("nbBatchSetBodiesDeviceCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("nbBatchGetBodiesCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("nbBatchGetBodiesDeviceCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("nbBatchGravMapCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp]),
    ("nbBatchRunStepsCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp, ctypes.c_int, ctypes.c_int]),
    ("nbBatchDwarfInfoCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    ("nbBatchSetTuningCUDA", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("nbBatchGetTuningCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("nbBatchAutotuneCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp, _vp, _vp, _vp, _dp]),
    ("nbBatchLastStepTimeCUDA", ctypes.c_int, [_vp, _dp]),
    ("nbSetTypesCUDA", ctypes.c_int, [_vp, _vp]),
    ("nbSetTimeOriginCUDA", ctypes.c_int, [_vp, ctypes.c_double]),
    ("nbSetStepCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbSetStepGraphCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbSetWalkFormCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbGetWalkFormCUDA", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    ("nbSetMixedTuningCUDA", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("nbBatchSetTimeOriginCUDA", ctypes.c_int, [_vp, ctypes.c_double]),
    ("nbGenerateDwarfCUDA", ctypes.c_int, [_vp, ctypes.POINTER(PlummerDwarf), ctypes.c_double]),
    ("nbBatchGenerateDwarfsCUDA", ctypes.c_int, [_vp, ctypes.POINTER(PlummerDwarf)]),
    ("nbGenerateMixedDwarfCUDA", ctypes.c_int, [_vp, ctypes.POINTER(MixedDwarf), ctypes.c_double]),
    ("nbBatchGenerateMixedDwarfsCUDA", ctypes.c_int, [_vp, ctypes.POINTER(MixedDwarf)]),
    ("nbBatchRunSystemCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    ("nbBatchGetBestBodiesCUDA", ctypes.c_int, [_vp, _vp, _vp]),
    ("nbBatchSetLMCCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int]),
    ("nbBatchGetLMCCUDA", ctypes.c_int, [_vp, _vp, _vp]),
    ("nbMixedDwarfParticleMassesCUDA", ctypes.c_int, [ctypes.POINTER(MixedDwarf), _vp]),
    ("nbGetBodyMassesCUDA", ctypes.c_int, [_vp, _vp]),
    ("nbHistogramCUDA", ctypes.c_int, [_vp, ctypes.POINTER(HistParams), _vp, _vp, _vp, _vp]),
    ("nbLikelihoodCUDA", ctypes.c_int, [_vp, ctypes.POINTER(HistParams), ctypes.POINTER(DataHist),
                                        _vp]),
    ("nbBatchSetTypesCUDA", ctypes.c_int, [_vp, _vp]),
    ("nbBatchHistogramCUDA", ctypes.c_int, [_vp, ctypes.POINTER(HistParams), _vp, _vp, _vp, _vp]),
    ("nbBatchLikelihoodCUDA", ctypes.c_int, [_vp, ctypes.POINTER(HistParams),
                                             ctypes.POINTER(DataHist), _vp]),
    ("nbRunSystemCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp, ctypes.POINTER(RunParams),
                                       ctypes.POINTER(HistParams), ctypes.POINTER(DataHist),
                                       ctypes.POINTER(RunResult)]),
    ("nbGetBestBodiesCUDA", ctypes.c_int, [_vp, _vp, _vp]),
    ("nbSetMixedModeCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbSetLMCCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int]),
    ("nbGetLMCCUDA", ctypes.c_int, [_vp, _vp, _vp]),
    ("nbBatchSetMixedModeCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbBatchSetWalkFormCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbSaveStateCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbRestoreStateCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbReleaseStatesCUDA", ctypes.c_int, [_vp]),
    ("nbStepAdjointCUDA", ctypes.c_int, [ctypes.POINTER(Ctx), _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("nbTreeInfoCUDA", ctypes.c_int, [_vp, ctypes.POINTER(TreeInfo)]),
    ("nbGetTreeCUDA", ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("nbEmdCalcCUDA", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int]),
    ("nbExtAccelerationCUDA", ctypes.c_int,
     [ctypes.POINTER(Potential), _vp, _vp, ctypes.c_int, ctypes.c_int]),
    ("nbExtAccelerationNoAllocCUDA", ctypes.c_int,
     [ctypes.POINTER(Potential), _vp, _vp, ctypes.c_int, ctypes.c_int]),
    ("nbKernelLaunchesCUDA", ctypes.c_uint64, []),
    ("nbLastWalkTimeCUDA", ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_int)]),
    ("nbLastStepTimeCUDA", ctypes.c_int, [_vp, _dp]),
    ("nbDirectSampleCUDA", ctypes.c_int, [_vp, ctypes.c_double, _vp, ctypes.c_int, _vp]),
    ("nbPeakFmaCUDA", ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dp]),
    ("nbInteractionCountsCUDA", ctypes.c_int, [_vp, _ull, _ull, _ull, _ull]),
    ("nbSetCountingCUDA", ctypes.c_int, [_vp, ctypes.c_int]),
    ("nbLastErrorCUDA", ctypes.c_char_p, []),
]

_lib = None


def load(path=LIB_PATH):
    """Load libnbody_b200.so (raises OSError/FileNotFoundError when it is absent)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            "%s is missing: build it with `python -m milkywayathome_client_b200.build`" % path)
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


def last_error():
    return load().nbLastErrorCUDA().decode(errors="replace")


def ptr(a):
    """Address of a numpy array's data (None passes NULL)."""
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)
