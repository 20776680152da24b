"""Correctly rounded log, pow, sin, cos and atan (milkywayathome_client_b200/csrc/nb_crmath.cuh),
no GPU.

The header uses only IEEE +, -, *, /, fma and sqrt, so a host build of it computes what the
device computes, bit for bit.  Its results are compared with Python's decimal module (60
digits, then rounded once to a double): the correctly rounded values that crlibm's log_rn and
pow_rn, the reference's mw_log and mw_pow, return (and its atan_rn, mw_atan).  sin and cos are
checked the same way; the reference's are the C library's, which round correctly but for about
0.1 % of the arguments (glibc 2.39).
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
extern "C" void cr_sin(const double* x, int n, double* out)
{ for (int i = 0; i < n; ++i) out[i] = nb_sin_rn(x[i]); }
extern "C" void cr_cos(const double* x, int n, double* out)
{ for (int i = 0; i < n; ++i) out[i] = nb_cos_rn(x[i]); }
extern "C" void cr_sincos(const double* x, int n, double* out)
{ for (int i = 0; i < n; ++i) { double s, c; nb_sincos_rn(x[i], s, c); out[i] = s + 2.0 * c; } }
extern "C" void cr_atan(const double* x, int n, double* out)
{ for (int i = 0; i < n; ++i) out[i] = nb_atan_rn(x[i]); }
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


def _dec_pi():
    def arctan_inv(n):
        x = Decimal(1) / n
        x2, s, t, k, sign = x * x, Decimal(0), x, 1, 1
        while t > Decimal(10) ** -75:
            s += sign * t / k
            t *= x2
            k += 2
            sign = -sign
        return s
    return 16 * arctan_inv(5) - 4 * arctan_inv(239)


def _dec_sincos(x, pi):
    """(sin x, cos x) by Taylor series after reducing x modulo 2 pi, 80 digits."""
    x = Decimal(x)
    r = x - (x / (2 * pi)).to_integral_value() * 2 * pi
    out = []
    for t, n in ((r, 1), (Decimal(1), 0)):
        s = Decimal(0)
        while t and abs(t) > Decimal(10) ** -75 * abs(s + t):
            s += t
            t = -t * r * r / ((n + 1) * (n + 2))
            n += 2
        out.append(s)
    return out


def _dec_atan(x, pi):
    """atan x: three halvings x -> x / (1 + sqrt(1 + x^2)), then the series, 80 digits."""
    x = Decimal(x)
    neg, x = x < 0, abs(x)
    inv = x > 1
    if inv:
        x = 1 / x
    for _ in range(3):
        x = x / (1 + (1 + x * x).sqrt())
    s, t, k, x2, sign = Decimal(0), x, 1, x * x, 1
    while t > Decimal(10) ** -75:
        s += sign * t / k
        t *= x2
        k += 2
        sign = -sign
    s *= 8
    if inv:
        s = pi / 2 - s
    return -s if neg else s


def test_sin_cos_are_correctly_rounded(lib):
    getcontext().prec = 80
    pi = _dec_pi()
    rng = random.Random(13)
    xs = [rng.uniform(-1200, 1200) for _ in range(3000)]          # the bar's angles
    xs += [rng.uniform(-2, 2) for _ in range(2000)]
    xs += [10 ** rng.uniform(-9, 8) * rng.choice([-1, 1]) for _ in range(2000)]
    xs += [0.0, -0.0, 1e-300, 7.4e-9, 1.5e-8, 0.7853981633974483, 1.5707963267948966, 3.141592653589793]
    want = [_dec_sincos(x, pi) for x in xs]
    s, c = _call(lib, "cr_sin", xs), _call(lib, "cr_cos", xs)
    bad = [(x, g, float(w[0])) for x, g, w in zip(xs, s, want) if g != float(w[0])]
    assert not bad, bad[:5]
    bad = [(x, g, float(w[1])) for x, g, w in zip(xs, c, want) if g != float(w[1])]
    assert not bad, bad[:5]
    both = _call(lib, "cr_sincos", xs)
    assert np.array_equal(both, s + 2.0 * c)


def test_sin_cos_agree_with_the_c_library_on_most_arguments(lib):
    """The reference's bar takes the C library's sin and cos: they agree with the correctly
    rounded values on all but a small fraction of the bar's angles."""
    rng = np.random.default_rng(1)
    xs = rng.uniform(-1200, 1200, 50000)
    s, c = _call(lib, "cr_sin", xs), _call(lib, "cr_cos", xs)
    assert (s != np.sin(xs)).mean() < 0.01 and (c != np.cos(xs)).mean() < 0.01
    assert np.max(np.abs(s - np.sin(xs))) <= np.max(np.spacing(np.abs(s)))


def test_atan_is_correctly_rounded(lib):
    getcontext().prec = 80
    pi = _dec_pi()
    rng = random.Random(17)
    xs = [rng.uniform(-30, 30) for _ in range(3000)]
    xs += [10 ** rng.uniform(-9, 19) * rng.choice([-1, 1]) for _ in range(3000)]
    xs += [0.0, -0.0, 7.4e-9, 7.5e-9, 1.0, -1.0, 1.2e18, 1e300, float("inf"), -float("inf")]
    got = _call(lib, "cr_atan", xs)
    want = [float(_dec_atan(x, pi)) if np.isfinite(x) else float(np.arctan(x)) for x in xs]
    bad = [(x, g, w) for x, g, w in zip(xs, got, want) if g != w]
    assert not bad, bad[:5]
    assert np.isnan(_call(lib, "cr_atan", [float("nan")])[0])


def test_atan_equal_to_the_reference_crlibm(lib):
    from oracle import bindings as ob
    if not ob.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    ref = ob.ref()
    rng = random.Random(19)
    xs = [rng.uniform(-30, 30) for _ in range(5000)]
    xs += [10 ** rng.uniform(-12, 20) * rng.choice([-1, 1]) for _ in range(5000)]
    got = _call(lib, "cr_atan", xs)
    assert all(g == ref.nbref_atan_rn(x) for g, x in zip(got, xs))
