"""Correctly rounded log and pow (milkywayathome_client_b200/csrc/nb_crmath.cuh), no GPU.

The header uses only IEEE +, -, *, /, fma and sqrt, so a host build of it computes what the
device computes, bit for bit.  Its results are compared with Python's decimal module (60
digits, then rounded once to a double): the correctly rounded values that crlibm's log_rn and
pow_rn, the reference's mw_log and mw_pow, return.
"""
import ctypes
import os
import random
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    "milkywayathome_client_b200", "csrc")
SRC = r'''
#include "nb_crmath.cuh"
extern "C" void cr_log(const double* x, int n, double* out)
{ for (int i = 0; i < n; ++i) out[i] = nb_log_rn(x[i]); }
extern "C" void cr_pow(const double* x, const double* y, int n, double* out)
{ for (int i = 0; i < n; ++i) out[i] = nb_pow_rn(x[i], y[i]); }
'''


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("crmath")
    src = d / "crmath.cpp"
    src.write_text(SRC)
    so = d / "libcrmath.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I", CSRC,
                    str(src), "-o", str(so)], check=True)
    return ctypes.CDLL(str(so))


def _call(lib, name, *arrays):
    arrays = [np.ascontiguousarray(a, dtype=np.float64) for a in arrays]
    out = np.empty(len(arrays[0]))
    ptrs = [a.ctypes.data_as(ctypes.c_void_p) for a in arrays]
    getattr(lib, name)(*ptrs[:1], *([ptrs[1]] if len(ptrs) > 1 else []), ctypes.c_int(len(out)),
                       out.ctypes.data_as(ctypes.c_void_p))
    return out


def _rn(d):
    return float(d)          # Decimal -> double: correctly rounded


def test_ln2_constant():
    getcontext().prec = 60
    hi, lo = 6.93147180559945286227e-01, 2.31904681384629955842e-17
    err = abs(Decimal(hi) + Decimal(lo) - Decimal(2).ln())
    assert err < Decimal(2) ** -106


def test_log_is_correctly_rounded(lib):
    getcontext().prec = 60
    rng = random.Random(7)
    xs = [1.0 + rng.random() * 10 ** rng.uniform(0, 4) for _ in range(6000)]       # NFW: ar/a
    xs += [10 ** rng.uniform(-300, 300) for _ in range(4000)]
    xs += [1.0 + rng.uniform(-1e-6, 1e-6) for _ in range(2000)]                      # near 1
    xs += [2.0 ** k for k in range(-1070, 1020, 37)] + [5e-324, 1.5, 0.75, 3.0, 1e308]
    got = _call(lib, "cr_log", xs)
    want = [_rn(Decimal(x).ln()) for x in xs]
    bad = [(x, g, w) for x, g, w in zip(xs, got, want) if g != w]
    assert not bad, bad[:5]


def test_log_special_values(lib):
    got = _call(lib, "cr_log", [0.0, -1.0, float("inf"), 1.0])
    assert got[0] == -np.inf and np.isnan(got[1]) and got[2] == np.inf and got[3] == 0.0


def test_pow_is_correctly_rounded(lib):
    getcontext().prec = 60
    rng = random.Random(11)
    xs, ys = [], []
    for _ in range(8000):
        xs.append(10 ** rng.uniform(-4, 4))
        ys.append(rng.choice([rng.uniform(-3, 3), 1.0, 2.0, 0.5, 1.5, 3.0, -1.0, 0.0,
                              rng.uniform(0.5, 2.5)]))
    got = _call(lib, "cr_pow", xs, ys)
    want = [_rn((Decimal(y) * Decimal(x).ln()).exp()) if y not in (0.0, 1.0)
            else (1.0 if y == 0.0 else x) for x, y in zip(xs, ys)]
    bad = [(x, y, g, w) for x, y, g, w in zip(xs, ys, got, want) if g != w]
    assert not bad, bad[:5]


def test_equal_to_the_reference_crlibm(lib):
    """The same inputs through crlibm's log_rn and pow_rn of the reference build (oracle/_ref)."""
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    ref = ob.ref()
    rng = random.Random(3)
    xs = [1.0 + rng.random() * 10 ** rng.uniform(0, 4) for _ in range(5000)]
    xs += [10 ** rng.uniform(-300, 300) for _ in range(5000)]
    got = _call(lib, "cr_log", xs)
    assert all(g == ref.nbref_log_rn(x) for g, x in zip(got, xs))
    px = [10 ** rng.uniform(-4, 4) for _ in range(5000)]
    py = [rng.uniform(-3, 3) for _ in range(5000)]
    got = _call(lib, "cr_pow", px, py)
    assert all(g == ref.nbref_pow_rn(x, y) for g, x, y in zip(got, px, py))
