"""The device per-cell code, compiled for the host with g++ (strict IEEE, no
contraction), is bit-identical to the oracle on evolved crossing-jet states.

The CUDA build uses the same source with -fmad=false and IEEE division and
square root, so this pins GPU-vs-oracle agreement without a GPU; the GPU
parity tests then check the CUDA build itself."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol
from hyqmom import ic

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "hyqmom.jl_b200", "csrc")


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = tmp_path_factory.mktemp("shim") / "libshim.so"
    subprocess.check_call(["/usr/bin/g++", "-O2", "-std=c++17", "-fno-fast-math", "-ffp-contract=off", "-fPIC", "-shared",
                           "-I", CSRC, "-o", str(out), os.path.join(HERE, "host_device_shim.cpp")])
    return ctypes.CDLL(str(out))


@pytest.fixture(scope="module")
def states():
    p = ic.with_jets(ic.default_params(Nx=12, Ny=12, Nz=12, Ma=0.0, Kn=1.0, CFL=0.7, dtmax=1e-2, tmax=10.0, nnmax=100), "crossing")
    M = ic.initial_state(p)
    pp = dict(p, **ic.grid_spacing(p))
    t, out = 0.0, []
    for s in range(24):
        _, t, _ = ol.step(M, pp, t)
        if s % 6 == 5:
            out.append(np.array(M).reshape(-1, 35, order="F"))
    return np.concatenate(out)


def P(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def test_per_cell_functions_bitwise(shim, states):
    for c in range(states.shape[0]):
        m = np.ascontiguousarray(states[c])
        o = [np.zeros(35) for _ in range(4)]
        shim.sh_flux(P(m), 0, ctypes.c_double(0.0), *[P(x) for x in o])
        for a, b in zip(o, ol.flux_closure35(m, 0, 0.0)):
            assert np.array_equal(a, b, equal_nan=True), c
        r = np.zeros(35)
        shim.sh_realized(P(m), 0, ctypes.c_double(0.0), P(r))  # the closure without the flux work
        assert np.array_equal(r, o[3], equal_nan=True), c
        for ax in (1, 2, 3):
            v, Mr = np.zeros(2), np.zeros(35)
            shim.sh_eig(P(m), ax, 0, ctypes.c_double(0.0), 1, P(v), P(Mr))
            rv = ol.eigenvalues6z(m, 0, 0.0, True) if ax == 3 else ol.eigenvalues6(m, ax, 0, 0.0)
            assert np.array_equal(v, np.array(rv[:2]), equal_nan=True) and np.array_equal(Mr, rv[2], equal_nan=True), (c, ax)
        mom = np.ascontiguousarray(m[[0, 1, 2, 3, 4]])
        v = np.zeros(2)
        shim.sh_closure(P(mom), P(v))
        assert np.array_equal(v, np.array(ol.closure_and_eigenvalues(mom)[1:]), equal_nan=True)
        mm = m.copy()
        shim.sh_coll(P(mm), ctypes.c_double(3e-3), ctypes.c_double(1.0), 1)
        assert np.array_equal(mm, ol.collision35(m, 3e-3, 1.0), equal_nan=True)


def jacobians(states, seed=5):
    """Flux Jacobians of every x and y slice of the evolved states, plus
    perturbed copies (random entries zeroed, scaled, made NaN)."""
    SL = [[0, 5, 9, 12, 14, 1, 6, 10, 13, 2, 7, 11, 3, 8, 4], list(range(15)),
          [0, 15, 19, 22, 24, 1, 16, 20, 23, 2, 17, 21, 3, 18, 4]]
    rng = np.random.default_rng(seed)
    out = []
    for m in states:
        for sl in SL:
            out.append(ol.vec_fn("hyqo_jacobian6", m[sl], 36))
    base = np.array(out)
    extra = []
    for J in base[rng.choice(len(base), 400, replace=False)]:
        K = J.copy()
        K[rng.integers(0, 36, size=rng.integers(1, 6))] = 0.0
        extra.append(K)
        extra.append(J * 10.0 ** rng.uniform(-150, 150))
        K = J.copy()
        K[rng.integers(0, 36)] = np.nan
        extra.append(K)
    # late-time Jacobians: round-off-sized entries in the first column (and
    # sometimes the last) leave dgebal nothing to isolate (pattern 0)
    for J in base[rng.choice(len(base), 400, replace=False)]:
        K = J.copy()
        scale = np.max(np.abs(J[np.isfinite(J)])) if np.isfinite(J).any() else 1.0
        for r in rng.choice([2, 4, 5], size=rng.integers(1, 4), replace=False):
            K[6 * r] = scale * 10.0 ** rng.uniform(-19, -12) * rng.choice([-1, 1])
        if rng.random() < 0.3:
            K[6 * 2 + 5] = scale * 10.0 ** rng.uniform(-19, -12)
        extra.append(K)
    extra.append(np.zeros(36))
    extra.append(np.eye(6).ravel())
    return np.concatenate([base, np.array(extra)])


def test_fast_eigen_path_is_bitwise_general(shim, states):
    """The register-resident path for the permutation dgebal usually finds on
    flux Jacobians gives the general eig_real<6> results bit for bit (the
    other patterns are recognised and left to the general code)."""
    seen = {-1: 0, 0: 0, 1: 0}
    out = np.zeros(25)
    for A in jacobians(states):
        shim.sh_eig6_both(P(np.ascontiguousarray(A)), P(out))
        seen[int(out[24])] += 1
        assert np.array_equal(out[:12], out[12:24], equal_nan=True), (A, out)
    assert seen[1] > 100 and seen[0] > 300, seen


def test_kernel_parts_defer_or_agree(shim, states):
    """The step kernels run the eigenvalue functions in parts: the pattern-1
    register path first, the general code on the cells it left, and the
    correction last, from the planes the earlier part reported.  On every cell (the evolved states and copies whose first
    Jacobian column carries round-off-sized entries) each part either leaves
    the cell to a later one or gives the complete function's results bit for
    bit; the flag variants likewise."""
    rng = np.random.default_rng(11)
    cells = [np.ascontiguousarray(m) for m in states]
    for m in states[rng.choice(len(states), 200, replace=False)]:
        k = m.copy()
        k[rng.choice([16, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34], 2, replace=False)] *= 1.0 + 1e-15
        cells.append(np.ascontiguousarray(k))
    shim.sh_eig_part.restype = ctypes.c_int
    shim.sh_eig_flags.restype = ctypes.c_int
    seen = {(g, st): 0 for g in (0, 1) for st in (0, 1, 2)}
    for m in cells:
        for ax in (1, 2, 3):
            v, Mr = np.zeros(2), np.zeros(35)
            shim.sh_eig(P(m), ax, 0, ctypes.c_double(0.0), 1, P(v), P(Mr))
            for gen in (0, 1):
                v2, Mr2, planes = np.zeros(2), np.zeros(35), ctypes.c_int(-1)
                st = shim.sh_eig_part(P(m), ax, 0, ctypes.c_double(0.0), 1, gen, P(v2), P(Mr2), ctypes.byref(planes))
                seen[(gen, st)] += 1
                assert st in (0, 1, 2) and not (gen and st == 1)
                if st == 2 and planes.value:
                    v2, Mr2 = np.zeros(2), np.zeros(35)
                    shim.sh_eig_corrected(P(m), ax, planes.value, 0, ctypes.c_double(0.0), P(v2), P(Mr2))
                    st = 0
                if st == 0:
                    assert np.array_equal(v, v2, equal_nan=True) and np.array_equal(Mr, Mr2, equal_nan=True), (ax, gen)
            if ax < 3:
                full = shim.sh_eig_flags(P(m), ax, 0)
                f = shim.sh_eig_flags(P(m), ax, 1)
                assert f == -1 or f == full
                assert shim.sh_eig_flags(P(m), ax, 2) == full
    assert seen[(0, 0)] > 100 and seen[(0, 1)] > 100 and seen[(1, 0)] > 100 and seen[(1, 2)] > 0, seen


def test_z_stage_reuses_the_y_stage_vw_speeds(shim, states):
    """The y stage parks the speeds of its VW-plane Jacobian; the z stage,
    given the y stage's output, uses them instead of solving that Jacobian
    again and gets the same bits as solving it (or ignores a NaN pair)."""
    shim.sh_yz_park.restype = ctypes.c_int
    used = 0
    for m in states:
        m = np.ascontiguousarray(m)
        out = np.zeros(74)
        used += shim.sh_yz_park(P(m), 1, P(out))
        assert np.array_equal(out[:37], out[37:], equal_nan=True)
    assert used > len(states) // 2, used


def test_reciprocal_division_is_ieee_division(shim):
    """div_by (the HLL star state's division through a shared reciprocal,
    with Markstein's correction) equals the IEEE quotient bit for bit."""
    shim.sh_div_check.restype = ctypes.c_longlong
    shim.sh_div_check.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_ulonglong]
    assert shim.sh_div_check(20_000_000, 40, 12345) == 0
    assert shim.sh_div_check(5_000_000, 300, 777) == 0
