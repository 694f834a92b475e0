"""Error bound of the Newton-Raphson reciprocal and square root the residual
kernels use instead of the XU-pipe FP64 divide/sqrt (csrc/zj_math.h): within
2 ulp of the correctly rounded result (numpy's IEEE division and sqrt) on
2^20 log-uniform samples of each function's domain; and of the viscosity
law's x^0.7 (series log and exp): within 2 ulp of numpy's x**0.7."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = r'''
#include "zj_math.h"
extern "C" void rcp_n(const double* x, double* y, long n) { for (long i = 0; i < n; ++i) y[i] = zj::zj_rcp(x[i]); }
extern "C" void sqrt_n(const double* x, double* y, long n) { for (long i = 0; i < n; ++i) y[i] = zj::zj_sqrt(x[i]); }
extern "C" void pow07_n(const double* x, double* y, long n) { for (long i = 0; i < n; ++i) y[i] = zj::zj_pow07(x[i]); }
'''


@pytest.fixture(scope="module")
def mathlib(tmp_path_factory):
    d = tmp_path_factory.mktemp("zjmath")
    (d / "m.cpp").write_text(SRC)
    so = d / "m.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-mfma", "-I",
                    os.path.join(ROOT, "zhijian_b200", "csrc"), str(d / "m.cpp"), "-o", str(so)],
                   check=True)
    lib = C.CDLL(str(so))
    for f in (lib.rcp_n, lib.sqrt_n, lib.pow07_n):
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_long]
    return lib


def ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def run(f, x):
    y = np.empty_like(x)
    f(x.ctypes.data, y.ctypes.data, x.size)
    return y


def test_rcp_within_2ulp(mathlib):
    rng = np.random.default_rng(0)
    x = 10.0 ** rng.uniform(-300, 300, 1 << 20)
    x = np.concatenate([x, [1.0, 2.0, 0.5, 3.0, 1e-10, 1.4, 0.01, 100.0]])
    assert ulps(run(mathlib.rcp_n, x), 1.0 / x).max() <= 2


def test_sqrt_within_2ulp(mathlib):
    rng = np.random.default_rng(1)
    x = 10.0 ** rng.uniform(-300, 300, 1 << 20)
    x = np.concatenate([x, [1.0, 2.0, 4.0, 1e-10, 0.25, 1e300, 5e-324 * 2 ** 60]])
    assert ulps(run(mathlib.sqrt_n, x), np.sqrt(x)).max() <= 2


def test_sqrt_special_values(mathlib):
    x = np.array([0.0, np.inf, np.nan, -1.0])
    y = run(mathlib.sqrt_n, x)
    assert y[0] == 0.0 and y[1] == np.inf and np.isnan(y[2]) and np.isnan(y[3])


def test_pow07_within_2ulp(mathlib):
    rng = np.random.default_rng(2)
    x = 10.0 ** rng.uniform(-300, 300, 1 << 20)
    t = rng.uniform(0.01, 100.0, 1 << 20)                 # temperatures of the solver's cases
    edge = [1.0, 2.0, 0.5, 1.4142135623730951, np.nextafter(1.4142135623730951, 2.0),
            np.nextafter(1.4142135623730951, 0.0), 0.7071067811865476, 10.0, 1024.0, 2.0 ** -1022,
            1.7976931348623157e308, 7.94, 1.0 / (1.4 * 0.09), 8.5e4, 300.0]
    x = np.concatenate([x, t, edge])
    ref = x ** 0.7
    got = run(mathlib.pow07_n, x)
    assert ulps(got, ref).max() <= 2
    assert run(mathlib.pow07_n, np.array([1.0]))[0] == 1.0
    sp = np.array([0.0, -1.0, np.inf, np.nan, 5e-324])
    got = run(mathlib.pow07_n, sp)
    assert got[0] == 0.0 and np.isnan(got[1]) and got[2] == np.inf and np.isnan(got[3]) and got[4] == 5e-324 ** 0.7
