"""The 2-D earth mover's distance (milkywayathome_client_b200/csrc/nb_emd.cuh), host build, no
GPU: bit for bit against the reference's own emdCalc (nbody/src/nbody_emd.c:1207-1268,
oracle/_ref).

The header uses only IEEE +, -, *, / and sqrt, so the host build computes what the device
computes.  The reference's transportation simplex stops at a basis within a tolerance of the
optimum, so equal results need the same decisions in the same order; the cases are the
signatures nbMatchEMD builds -- normalised weights on the (lambda, beta) bin centres of a
regular grid, where many ground distances tie -- with zero-weight bins, unequal totals (the
dummy node), one-row and one-column problems, and the invalid inputs the reference rejects.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    "milkywayathome_client_b200", "csrc")
SRC = r'''
#include <vector>
#include "nb_emd.cuh"
extern "C" double emd_host(const double* s1, int n1, const double* s2, int n2)
{
    std::vector<char> buf(nb_emd_work_bytes(n1, n2) + 64);
    NbEmdWork w = nb_emd_carve(buf.data(), n1, n2);
    NbEmdScalars sc;
    return nb_emd_calc(NbEmdSerial(), s1, n1, s2, n2, w, sc);
}
'''


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("emd")
    src = d / "emd.cpp"
    src.write_text(SRC)
    so = d / "libemd.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I",
                    CSRC, str(src), "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    lib.emd_host.restype = ctypes.c_double
    lib.emd_host.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    return lib


def _emd(lib, a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return lib.emd_host(a.ctypes.data, len(a), b.ctypes.data, len(b))


def _grid_signature(rng, lam_bins, beta_bins, fill, lam=(-150.0, 150.0), beta=(-15.0, 15.0)):
    """nbMatchEMD's signature of a histogram: count / total on the bin centres (lambda-major)."""
    ls = (lam[1] - lam[0]) / lam_bins
    bs = (beta[1] - beta[0]) / beta_bins
    li = np.repeat(np.arange(lam_bins), beta_bins)
    bi = np.tile(np.arange(beta_bins), lam_bins)
    counts = rng.integers(1, 60, lam_bins * beta_bins) * (rng.uniform(size=lam_bins * beta_bins) < fill)
    total = max(int(counts.sum()), 1)
    w = (counts / float(total)) * total / (1.0 * total)
    return np.stack([w, (li + 0.5) * ls + lam[0], (bi + 0.5) * bs + beta[0]], axis=1)


def _need_ref():
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    return ob


@pytest.mark.parametrize("lam_bins,beta_bins,fill", [(10, 2, 0.9), (20, 3, 0.5), (12, 5, 0.7),
                                                     (34, 2, 0.3), (50, 4, 0.25), (8, 8, 1.0)])
def test_emd_matches_reference_bit_for_bit(lib, lam_bins, beta_bins, fill):
    ob = _need_ref()
    rng = np.random.default_rng(lam_bins * 100 + beta_bins)
    for _ in range(25):
        a = _grid_signature(rng, lam_bins, beta_bins, fill)
        b = _grid_signature(rng, lam_bins, beta_bins, fill)
        want, got = ob.ref_emd(a, b), _emd(lib, a, b)
        assert np.isnan(want) == np.isnan(got)
        if not np.isnan(want):
            assert np.float64(got).view(np.uint64) == np.float64(want).view(np.uint64), (got, want)


def test_emd_unequal_totals_dummy_node(lib):
    """Totals that differ by more than 1e-5 of the supply get a zero-cost dummy node on the
    short side; the EMD divides by the larger total."""
    ob = _need_ref()
    rng = np.random.default_rng(5)
    for scale in (0.5, 0.9, 1.2, 3.0, 1.0 + 2e-5, 1.0 + 5e-6):
        a = _grid_signature(rng, 15, 3, 0.6)
        b = _grid_signature(rng, 15, 3, 0.6)
        b[:, 0] *= scale
        want, got = ob.ref_emd(a, b), _emd(lib, a, b)
        assert np.float64(got).view(np.uint64) == np.float64(want).view(np.uint64), (scale, got, want)


def test_emd_random_points_and_degenerate_shapes(lib):
    ob = _need_ref()
    rng = np.random.default_rng(11)
    cases = []
    for n1, n2 in ((1, 7), (7, 1), (1, 1), (2, 2), (5, 9), (30, 17), (60, 60)):
        a = np.stack([rng.uniform(0.1, 1.0, n1), rng.uniform(-50, 50, n1), rng.uniform(-5, 5, n1)], 1)
        b = np.stack([rng.uniform(0.1, 1.0, n2), rng.uniform(-50, 50, n2), rng.uniform(-5, 5, n2)], 1)
        a[:, 0] /= a[:, 0].sum()
        b[:, 0] /= b[:, 0].sum()
        cases.append((a, b))
    for a, b in cases:
        want, got = ob.ref_emd(a, b), _emd(lib, a, b)
        assert np.float64(got).view(np.uint64) == np.float64(want).view(np.uint64), (len(a), len(b))


def test_emd_invalid_inputs_are_nan(lib):
    """No positive weight on a side, or a negative weight: the reference's EMD_INVALID."""
    ob = _need_ref()
    a = np.array([[0.5, 0.0, 0.0], [0.5, 1.0, 0.0]])
    for b in (np.array([[0.0, 0.0, 0.0]]), np.array([[-0.5, 0.0, 0.0], [1.5, 1.0, 1.0]])):
        assert np.isnan(ob.ref_emd(a, b)) and np.isnan(_emd(lib, a, b))


def test_emd_one_beta_bin_is_the_1d_transport_cost(lib):
    """With one beta bin the points lie on the lambda axis: the EMD is the 1-D transport cost
    sum |F1 - F2| dlambda that the one-beta-bin likelihood evaluates in closed form."""
    rng = np.random.default_rng(3)
    for _ in range(10):
        a = _grid_signature(rng, 40, 1, 0.8)
        b = _grid_signature(rng, 40, 1, 0.8)
        lam = a[:, 1]
        closed = float(np.sum(np.abs(np.cumsum(a[:, 0]) - np.cumsum(b[:, 0]))[:-1] * np.diff(lam)))
        assert abs(_emd(lib, a, b) - closed) < 1e-9
