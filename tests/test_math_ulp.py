"""The step's own exp (Cody-Waite reduction + Taylor series) and cube root
(exponent split + Newton), compiled for the host from the device source,
against numpy's exp and cbrt (the platform libm): error in units in the last
place over the ranges the step uses them.

exp: the BGK factor exp(-dt/tc) (collision35) takes arguments in
[-745, 0]; the whole double range is checked too.  cbrt: the Cardano roots of
the realizability cubics (rootsR, rootsR_X_Y) take any finite argument.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "hyqmom.jl_b200", "csrc")


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = tmp_path_factory.mktemp("shim_ulp") / "libshim.so"
    subprocess.check_call(["/usr/bin/g++", "-O2", "-std=c++17", "-fno-fast-math", "-ffp-contract=off", "-fPIC", "-shared",
                           "-I", CSRC, "-o", str(out), os.path.join(HERE, "host_device_shim.cpp")])
    return ctypes.CDLL(str(out))


def run(shim, name, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    dp = ctypes.POINTER(ctypes.c_double)
    getattr(shim, name)(x.ctypes.data_as(dp), y.ctypes.data_as(dp), ctypes.c_longlong(x.size))
    return y


def ulps(a, b):
    """|a - b| in units in the last place of b (same-sign finite values)."""
    return np.abs(np.ascontiguousarray(a).view(np.int64) - np.ascontiguousarray(b).view(np.int64))


def test_hexp_within_one_ulp(shim):
    rng = np.random.default_rng(0)
    x = np.concatenate([-rng.uniform(0, 2, 200000), -np.exp(rng.uniform(np.log(1e-12), np.log(745.0), 200000)),
                        rng.uniform(-708, 709, 200000), [0.0, -0.0, -1e-300, 1e-300, -708.39, 709.7]])
    y = run(shim, "sh_hexp_n", x)
    ref = np.exp(x)
    normal = ref > 4.0 * 2.2250738585072014e-308  # results clear of the subnormal range
    u = ulps(y[normal], ref[normal])
    print("hexp: max %d ulp, %.4f%% of arguments off by one" % (u.max(), 100 * np.mean(u > 0)))
    assert u.max() <= 1
    # results at the bottom of the range (scaled into the subnormals by one
    # ldexp): within an ulp of the smallest normal
    sub = ~normal
    assert np.all(np.abs(y[sub] - ref[sub]) <= 2.0 * 2.220446049250313e-16 * 4.0 * 2.2250738585072014e-308)


def test_hexp_special_values(shim):
    x = np.array([np.nan, np.inf, -np.inf, 710.0, -746.0])
    y = run(shim, "sh_hexp_n", x)
    assert np.isnan(y[0]) and y[1] == np.inf and y[2] == 0.0 and y[3] == np.inf and y[4] == 0.0


def test_hcbrt_within_one_ulp(shim):
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-10, 10, 200000), np.exp(rng.uniform(-700, 700, 200000)) * rng.choice([-1, 1], 200000)])
    y = run(shim, "sh_hcbrt_n", x)
    u = ulps(np.abs(y), np.abs(np.cbrt(x)))
    print("hcbrt: max %d ulp, %.4f%% of arguments off by one" % (u.max(), 100 * np.mean(u > 0)))
    assert u.max() <= 1
    assert np.all(np.sign(y) == np.sign(x))
    z = run(shim, "sh_hcbrt_n", np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 27.0, -8.0]))
    assert z[0] == 0.0 and z[2] == np.inf and z[3] == -np.inf and np.isnan(z[4]) and z[5] == 3.0 and z[6] == -2.0
