"""The reference's own property tests of the per-cell functions, on this code.

test/test_eigenvalue_ordering.jl and test/test_z_eigenvalue_fix.jl of the
reference check eigenvalues6_hyperbolic_3D, eigenvalues6z_hyperbolic_3D and
closure_and_eigenvalues on Gaussian moment sets (InitializeM4_35) for their
ordering, symmetry, bounds and high-Mach stability; test/test_closures.jl and
test/test_realizability.jl check the closure's output, its mass and the
realizability_S2 projection; test/test_numerical_schemes.jl the HLL update
of a row and the BGK collision; test/test_moment_conversions.jl and
test/test_realizability_bounds.jl the moments of Gaussians;
test/test_numerical_accuracy.jl determinism, mirror symmetry of the speeds
and tiny or large states; test/test_initialization.jl InitializeM4_35; test/test_initial_conditions.jl the IC regions
(here on the host IC module, hyqmom.ic).  The same cases and the same assertions run here
on the oracle; the device code compiled for the host and the GPU's per-cell
entry points must give the oracle's numbers bit for bit on the wave-speed
cases.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "hyqmom.jl_b200", "csrc")
SQ3 = np.sqrt(3.0)


def gaussian(u, v, w, rho=1.0, T=1.0):
    """InitializeM4_35(rho, u, v, w, T, 0, 0, T, 0, T) (isotropic Gaussian)."""
    return ol.initialize_m4_35(rho, u, v, w, T, 0.0, 0.0, T, 0.0, T)


def speeds(M, Ma):
    """(x, y, z) extreme speeds of the oracle, flag2D = 0, positivity on."""
    x = ol.eigenvalues6(M, 1, 0, Ma)[:2]
    y = ol.eigenvalues6(M, 2, 0, Ma)[:2]
    z = ol.eigenvalues6z(M, 0, Ma)[:2]
    return x, y, z


# (u, v, w, Ma) of the eigenvalue cases of the reference's property tests
CASES = {
    "ordering": (5.0, 3.0, -2.0, 6.0),
    "symmetric": (50.0, 50.0, 50.0, SQ3 * 50.0),
    "bounded": (10.0, 0.0, 0.0, 10.0),
    "high_mach": (100.0, 0.0, 0.0, 100.0),
    "rest": (0.0, 0.0, 0.0, 0.0),
    "sign_pos": (20.0, 0.0, 0.0, 20.0),
    "sign_neg": (-20.0, 0.0, 0.0, 20.0),
    "z_consistency": (10.0, 5.0, 15.0, float(np.sqrt(10.0 ** 2 + 5.0 ** 2 + 15.0 ** 2))),
    "z_fix": (40.0, 40.0, -40.0, 70.0),
    "z_high_mach": (150.0 / SQ3, 150.0 / SQ3, -150.0 / SQ3, 150.0),
    "mirror_pos": (5.0, 0.0, 0.0, 5.0),
    "mirror_neg": (-5.0, 0.0, 0.0, 5.0),
    "large": (1000.0, 0.0, 0.0, 1000.0),
}


def test_eigenvalue_ordering_properties():
    """test/test_eigenvalue_ordering.jl, each testset's assertions."""
    # eigenvalues sorted correctly
    for lo, hi in speeds(gaussian(5.0, 3.0, -2.0), 6.0):
        assert lo <= hi
    # symmetric flow: the three directions within 10 %
    (xl, xh), (yl, yh), (zl, zh) = speeds(gaussian(50.0, 50.0, 50.0), SQ3 * 50.0)
    for a, b in ((xh, yh), (xh, zh), (yh, zh), (xl, yl), (xl, zl), (yl, zl)):
        assert np.isclose(a, b, rtol=0.1, atol=0.0)
    # bounded by the flow velocity and the sound speed
    u, c = 10.0, 1.0
    lo, hi = ol.eigenvalues6(gaussian(u, 0.0, 0.0), 1, 0, 10.0)[:2]
    assert u < hi < 5.0 * (abs(u) + c)
    assert -5.0 * (abs(u) + c) < lo < u
    # high Mach number: finite, not pathological
    lo, hi = ol.eigenvalues6(gaussian(100.0, 0.0, 0.0), 1, 0, 100.0)[:2]
    assert np.isfinite(lo) and np.isfinite(hi) and abs(hi) < 1e4 and abs(lo) < 1e4
    # at rest: symmetric about zero, of the order of the sound speed
    lo, hi = ol.eigenvalues6(gaussian(0.0, 0.0, 0.0), 1, 0, 0.0)[:2]
    assert abs(lo + hi) < 1.0 and abs(hi) < 5.0
    # sign consistency
    assert ol.eigenvalues6(gaussian(20.0, 0.0, 0.0), 1, 0, 20.0)[1] > 0.0
    assert ol.eigenvalues6(gaussian(-20.0, 0.0, 0.0), 1, 0, 20.0)[0] < 0.0
    # z consistent with x and y
    u, v, w, Ma = CASES["z_consistency"]
    sp = speeds(gaussian(u, v, w), Ma)
    assert all(np.isfinite(s).all() for s in sp)
    mx = [abs(s[1]) for s in sp]
    assert max(mx) / min(mx) < 10.0


def test_closure_eigenvalues_bounded_by_velocity():
    """test/test_eigenvalue_ordering.jl, "1D closure eigenvalues"."""
    rho, u, T = 1.0, 5.0, 1.0
    mom = [rho, rho * u, rho * (u * u + T), rho * (u ** 3 + 3 * u * T), rho * (u ** 4 + 6 * u * u * T + 3 * T * T)]
    _, lo, hi = ol.closure_and_eigenvalues(mom)
    assert np.isfinite(lo) and np.isfinite(hi) and lo <= hi
    assert hi > u and lo < u


def test_z_eigenvalue_regression_properties():
    """test/test_z_eigenvalue_fix.jl: the WV Jacobian's moment ordering keeps
    the z speeds physical (the reference's bug gave ~3.3e5)."""
    u, v, w, Ma = CASES["z_fix"]
    (xl, xh), (yl, yh), (zl, zh) = speeds(gaussian(u, v, w), Ma)
    assert np.isfinite(zl) and np.isfinite(zh)
    assert abs(zh) < 5000.0 and abs(zl) < 5000.0 and abs(zh) < 5.0 * abs(Ma)
    assert abs(xh) < 5000.0 and abs(yh) < 5000.0
    mx = [abs(xh), abs(yh), abs(zh)]
    if min(mx) > 1.0:
        assert max(mx) / min(mx) < 10.0
    u, v, w, Ma = CASES["z_high_mach"]
    zl, zh = ol.eigenvalues6z(gaussian(u, v, w), 0, Ma)[:2]
    assert np.isfinite(zh) and abs(zh) < 1e4 and abs(zh) < 50.0 * Ma


def test_closure_properties():
    """test/test_closures.jl, each testset's assertions."""
    _, lo, hi = ol.closure_and_eigenvalues([1.0, 0.1, 1.2, 0.15, 3.5])
    assert np.isfinite(lo) and np.isfinite(hi) and lo <= hi
    # the closure's output is finite (3-D and 2-D mode) and keeps the mass
    for rho, (u, v, w), T, flag2D, Ma in ((1.0, (0.1, 0.0, 0.0), 1.0, 0, 2.0), (0.8, (0.0, 0.1, 0.0), 1.2, 1, 0.5)):
        M4 = gaussian(u, v, w, rho=rho, T=T)
        for out in ol.flux_closure35(M4, flag2D, Ma):
            assert out.shape == (35,) and np.isfinite(out).all()
    M4 = gaussian(0.0, 0.0, 0.0, rho=2.0, T=1.5)
    assert abs(ol.flux_closure35(M4, 0, 2.0)[3][0] - M4[0]) <= 1e-10
    # eigenvalues along each axis (axis 3 is the y pair, as in the
    # reference's compute_eigenvalues_for_axis) and in 2-D mode
    lo, hi = ol.eigenvalues6(gaussian(0.1, 0.2, 0.3), 1, 0, 2.0)[:2]
    assert np.isfinite(lo) and np.isfinite(hi) and lo <= hi
    M4 = gaussian(0.2, -0.1, 0.05, T=0.8)
    for axis in (1, 2, 3):
        for flag2D in (0, 1):
            lo, hi = ol.eigenvalues6(M4, axis, flag2D, 1.5)[:2]
            assert np.isfinite(lo) and np.isfinite(hi) and lo <= hi
    assert ol.eigenvalues6(M4, 3, 0, 1.5)[:2] == ol.eigenvalues6(M4, 2, 0, 1.5)[:2]


def test_realizability_S2_properties():
    """test/test_realizability.jl: realizability_S2 basic, Gaussian moments
    unchanged, finiteness near the corner."""
    tol = 1e-10
    for corr in ((0.5, 0.3, 0.4), (-0.8, -0.6, -0.7), (0.99, 0.98, 0.97)):
        r = ol.realizability_S2(*corr)
        assert np.isfinite(r).all() and all(abs(x) <= 1.0 + tol for x in r[:3]) and r[3] >= 0.0
    r = ol.realizability_S2(0.0, 0.0, 0.0)
    assert r[0] == 0.0 and r[1] == 0.0 and r[2] == 0.0 and np.isfinite(r[3])
    assert np.isfinite(ol.realizability_S2(1.5, 1.5, 1.5)).all()
    _, S4 = ol.m2cs4_35(gaussian(0.0, 0.0, 0.0))
    S110, S101, S011 = S4[6], S4[16], S4[25]
    r = ol.realizability_S2(S110, S101, S011)
    assert abs(r[0] - S110) <= tol and abs(r[1] - S101) <= tol and abs(r[2] - S011) <= tol


def test_numerical_schemes_properties():
    """test/test_numerical_schemes.jl: pas_HLL on a uniform row (the
    reference's 5 moments become the step's 35), collision35 keeps the mass
    and moves a perturbed moment."""
    Nx = 10
    M = np.ones((Nx, 35))
    Mp = ol.pas_hll(M, 0.1 * M, 0.01, 0.1, -np.ones(Nx), np.ones(Nx))
    assert Mp.shape == M.shape and np.isfinite(Mp).all()
    M = gaussian(0.1, 0.2, 0.3)
    for dt, Kn in ((0.001, 0.01), (0.01, 0.001)):  # the reference test passes (Kn, dt) positionally
        Mn = ol.collision35(M, dt, Kn)
        assert Mn.shape == (35,) and np.isfinite(Mn).all() and abs(Mn[0] - M[0]) <= 1e-10
    M = gaussian(0.0, 0.0, 0.0)
    M[10] += 0.1  # the reference's M[11] (1-based)
    assert abs(ol.collision35(M, 0.1, 0.01)[10] - M[10]) > 0.0


def test_moment_conversion_properties():
    """test/test_moment_conversions.jl: M2CS4_35 of Gaussians (variances T,
    S400 = S040 = S004 = 3, correlations within [-1, 1]), finite for
    correlated covariances, InitializeM4_35 with correlations."""
    tol = 1e-10
    T = 1.5
    C4, S4 = ol.m2cs4_35(gaussian(0.1, 0.2, 0.3, T=T))
    assert abs(C4[2] - T) <= tol and abs(C4[9] - T) <= tol and abs(C4[19] - T) <= tol
    assert abs(S4[4] - 3.0) <= tol and abs(S4[14] - 3.0) <= tol and abs(S4[24] - 3.0) <= tol
    _, S4 = ol.m2cs4_35(gaussian(0.0, 0.0, 0.0))
    assert all(abs(S4[k]) <= 1.0 + tol for k in (6, 16, 25))
    M = ol.initialize_m4_35(1.5, 0.3, -0.2, 0.4, 1.2, 0.3, -0.1, 1.5, 0.2, 1.8)
    C4, S4 = ol.m2cs4_35(M)
    assert abs(M[0] - 1.5) <= tol and np.isfinite(C4).all() and np.isfinite(S4).all()
    for r in (0.0, 0.3, 0.6, 0.9, -0.3, -0.6):
        M = ol.initialize_m4_35(1.0, 0.0, 0.0, 0.0, 1.0, r, r, 1.0, r, 1.0)
        assert M.shape == (35,) and np.isfinite(M).all() and abs(M[0] - 1.0) <= tol


def test_realizability_bounds_properties():
    """test/test_realizability_bounds.jl: InitializeM4_35 moments (density,
    variances, Cauchy-Schwarz, fourth moments, ordering, zero velocity) and
    the 1-D closure's fifth moment."""
    M = gaussian(10.0, 5.0, -3.0, rho=1.5)
    assert M[0] > 0 and M[0] == 1.5
    T = 2.0
    M = gaussian(10.0, 5.0, -3.0, T=T)
    for k, vel in ((2, 10.0), (9, 5.0), (19, -3.0)):  # M200, M020, M002
        var = M[k] - vel ** 2
        assert var > 0 and abs(var - T) <= 1e-10 * T
    M = gaussian(10.0, 5.0, 0.0)
    assert M[6] ** 2 <= M[2] * M[9] and M[16] ** 2 <= M[2] * M[19] and M[25] ** 2 <= M[9] * M[19]
    M = gaussian(5.0, 0.0, 0.0)
    assert np.isfinite(M).all() and M[4] > 0 and M[14] > 0 and M[24] > 0
    M = gaussian(10.0, 0.0, 0.0)
    assert M[1] / M[0] > 1.0 and M[2] / M[1] > 1.0
    M = gaussian(0.0, 0.0, 0.0)
    assert abs(M[0] - 1.0) <= 1e-12 and all(abs(M[k]) <= 1e-10 for k in (1, 5, 15))
    assert all(abs(M[k] - 1.0) <= 1e-12 for k in (2, 9, 19))
    u, T = 5.0, 1.0
    Mp, lo, hi = ol.closure_and_eigenvalues([1.0, u, u * u + T, u ** 3 + 3 * u * T, u ** 4 + 6 * u * u * T + 3 * T * T])
    assert Mp >= 0 and np.isfinite(Mp) and np.isfinite(lo) and np.isfinite(hi)


def test_numerical_accuracy_properties():
    """test/test_numerical_accuracy.jl: small perturbations stay small,
    tiny and large states stay finite, the speeds are deterministic and
    mirror-symmetric (max at +u = -min at -u), convex mixtures of Gaussians
    keep a positive density and variance."""
    M1 = gaussian(5.0, 0.0, 0.0)
    M2 = ol.initialize_m4_35(1.0 + 1e-14, 5.0, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0, 0.0, 1.0)
    assert np.max(np.abs(M2 - M1)) < 1e-10
    for M in (gaussian(0.0, 0.0, 0.0, rho=1e-10), gaussian(1000.0, 0.0, 0.0)):
        assert np.isfinite(M).all() and M[0] > 0
    M = gaussian(10.0, 0.0, 0.0)
    a, b = ol.eigenvalues6(M, 1, 0, 10.0)[:2], ol.eigenvalues6(M, 1, 0, 10.0)[:2]
    assert a == b
    lo_p, hi_p = ol.eigenvalues6(gaussian(5.0, 0.0, 0.0), 1, 0, 5.0)[:2]
    lo_n, hi_n = ol.eigenvalues6(gaussian(-5.0, 0.0, 0.0), 1, 0, 5.0)[:2]
    assert np.isclose(hi_p, -lo_n, rtol=1e-10, atol=0.0) and np.isclose(lo_p, -hi_n, rtol=1e-10, atol=0.0)
    M1, M2 = gaussian(3.0, 0.0, 0.0), gaussian(7.0, 0.0, 0.0, rho=1.5)
    Mm = 0.6 * M1 + 0.4 * M2
    assert Mm[0] > 0 and np.isfinite(Mm).all() and Mm[2] / Mm[0] - (Mm[1] / Mm[0]) ** 2 > 0


def test_initial_condition_region_properties():
    """test/test_initial_conditions.jl: CubicRegion's default temperature,
    region_to_moments (density kept, finite with correlations) and
    cell_overlaps_cube (strict overlap; an infinite background overlaps
    everything), with the reference's cases."""
    from hyqmom import ic
    inf = float("inf")
    assert ic.CubicRegion((0.0, 0.0, 0.0), (0.1, 0.1, 0.1), 1.0, (0.0, 0.0, 0.0)).temperature == 1.0
    region = ic.CubicRegion((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 1.0, (0.0, 0.0, 0.0), 1.0)
    Mr = ic.region_to_moments(region, 0.0, 0.0, 0.0)
    assert len(Mr) == 35 and np.isfinite(Mr).all() and np.isclose(Mr[0], 1.0)
    moving = ic.CubicRegion((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 2.0, (1.0, 0.5, 0.0), 0.5)
    Mr = ic.region_to_moments(moving, 0.0, 0.0, 0.0)
    assert len(Mr) == 35 and np.isfinite(Mr).all() and np.isclose(Mr[0], 2.0)
    assert np.isfinite(ic.region_to_moments(region, 0.1, 0.2, 0.3)).all()
    cube = ic.CubicRegion((0.0, 0.0, 0.0), (0.2, 0.2, 0.2), 1.0, (0.0, 0.0, 0.0), 1.0)
    cs = (0.1, 0.1, 0.1)
    assert ic.cell_overlaps_cube((0.0, 0.0, 0.0), cs, cube)
    assert ic.cell_overlaps_cube((0.05, 0.05, 0.05), cs, cube)
    assert ic.cell_overlaps_cube((0.15, 0.0, 0.0), cs, cube)
    assert not ic.cell_overlaps_cube((0.5, 0.0, 0.0), cs, cube)
    assert not ic.cell_overlaps_cube((0.0, 0.5, 0.0), cs, cube)
    background = ic.CubicRegion((0.0, 0.0, 0.0), (inf, inf, inf), 0.01, (0.0, 0.0, 0.0), 1.0)
    assert ic.cell_overlaps_cube((100.0, 100.0, 100.0), cs, background)


def test_initialization_properties():
    """test/test_initialization.jl: InitializeM4_35's mean, variances,
    correlation, kurtosis 3 and vanishing odd standardized moments."""
    tol = 1e-10
    rho, u, v, w, T = 1.5, 0.1, 0.2, 0.3, 2.0
    M = ol.initialize_m4_35(rho, u, v, w, T, 0.0, 0.0, T, 0.0, T)
    assert abs(M[0] - rho) <= tol and abs(M[1] / M[0] - u) <= tol and abs(M[5] / M[0] - v) <= tol and abs(M[15] / M[0] - w) <= tol
    _, S4 = ol.m2cs4_35(M)
    assert all(abs(S4[k] - 3.0) <= tol for k in (4, 14, 24))
    C200, C020, C002, C110, C101, C011 = 1.0, 1.5, 2.0, 0.5, 0.3, 0.6
    C4, S4 = ol.m2cs4_35(ol.initialize_m4_35(1.0, 0.0, 0.0, 0.0, C200, C110, C101, C020, C011, C002))
    assert abs(C4[2] - C200) <= tol and abs(C4[9] - C020) <= tol and abs(C4[19] - C002) <= tol
    assert abs(S4[6] - C110 / np.sqrt(C200 * C020)) <= tol
    assert abs(ol.initialize_m4_35(3.0, 0.0, 0.0, 0.0, 1.5, 0.0, 0.0, 1.5, 0.0, 1.5)[0] - 3.0) <= tol
    _, S4 = ol.m2cs4_35(gaussian(0.0, 0.0, 0.0))
    odd = [4, 8, 9, 11, 13, 18, 19, 21, 23, 24, 27, 28, 29, 30, 31, 32, 33, 34]  # the reference's 1-based list
    assert all(abs(S4[k - 1]) < tol for k in odd)
    M = gaussian(0.5, -0.3, 0.1, rho=2.0)
    C4, _ = ol.m2cs4_35(M)
    assert M[0] > 0 and np.isfinite(M).all() and C4[2] > 0 and C4[9] > 0 and C4[19] > 0
    # test/test_conservation.jl, "Symmetry preservation": equal velocities give
    # equal second moments
    M = gaussian(5.0, 5.0, 5.0)
    assert np.isclose(M[2], M[9], rtol=1e-10, atol=0.0) and np.isclose(M[2], M[19], rtol=1e-10, atol=0.0)


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = tmp_path_factory.mktemp("shim_props") / "libshim.so"
    subprocess.check_call(["/usr/bin/g++", "-O2", "-std=c++17", "-fno-fast-math", "-ffp-contract=off", "-fPIC", "-shared",
                           "-I", CSRC, "-o", str(out), os.path.join(HERE, "host_device_shim.cpp")])
    return ctypes.CDLL(str(out))


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def test_device_code_on_host_gives_the_oracle_speeds(shim):
    """The device source compiled for the host, on every case and axis: the
    oracle's speeds and realized moments, bit for bit."""
    for name, (u, v, w, Ma) in CASES.items():
        M = np.ascontiguousarray(gaussian(u, v, w))
        for axis in (1, 2, 3):
            vv, Mr = np.zeros(2), np.zeros(35)
            shim.sh_eig(_p(M), ctypes.c_int(axis), ctypes.c_int(0), ctypes.c_double(Ma), ctypes.c_int(1), _p(vv), _p(Mr))
            lo, hi, Mo = ol.eigenvalues6z(M, 0, Ma) if axis == 3 else ol.eigenvalues6(M, axis, 0, Ma)
            assert vv[0] == lo and vv[1] == hi, (name, axis, vv, lo, hi)
            assert np.array_equal(Mr, Mo), (name, axis)


@pytest.mark.gpu
def test_gpu_cells_give_the_oracle_speeds():
    """hyq_cells_eigenvalues on all cases at once (one cell each): the
    oracle's speeds and realized moments, bit for bit."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hyqmom import _lib
    lib = _lib.load()
    names = list(CASES)
    for Ma in sorted({c[3] for c in CASES.values()}):
        rows = [n for n in names if CASES[n][3] == Ma]
        states = np.array([gaussian(*CASES[n][:3]) for n in rows])
        n = len(rows)
        dM = torch.tensor(np.ascontiguousarray(states.T), dtype=torch.float64, device="cuda")
        for axis in (1, 2, 3):
            v = torch.empty(2, n, dtype=torch.float64, device="cuda")
            Mr = torch.empty_like(dM)
            assert lib.hyq_cells_eigenvalues(dM.data_ptr(), n, axis, 0, Ma, 1, v.data_ptr(), Mr.data_ptr(), None) == 0
            torch.cuda.synchronize()
            gv, gM = v.cpu().numpy(), Mr.cpu().numpy().T
            for k, name in enumerate(rows):
                lo, hi, Mo = ol.eigenvalues6z(states[k], 0, Ma) if axis == 3 else ol.eigenvalues6(states[k], axis, 0, Ma)
                assert gv[0, k] == lo and gv[1, k] == hi, (name, axis)
                assert np.array_equal(gM[k], Mo), (name, axis)
