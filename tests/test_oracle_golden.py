"""The CPU oracle against the reference's own golden data.

* generated closed forms vs the reference's expressions (tests/golden/autogen.npz)
* MATLAB unit goldens used by the reference's test/test_golden_files.jl
  (tolerance GOLDEN_TOL = 1e-10 there, test/test_golden_files.jl:15)
* end-to-end Nz=1 goldens test/goldenfiles/mpi_1rank_*.bin read by
  test/test_mpi.jl:114-141 (the reference's bar is abs 1e-6 / rel 1e-4,
  test/test_mpi.jl:35-36; the oracle is held to abs 1e-12 here).
"""
import os

import numpy as np
import pytest

import oracle_lib as ol
from hyqmom import ic

GOLD = os.path.join(os.path.dirname(__file__), "golden")
GOLDEN_TOL = 1e-10


@pytest.fixture(scope="module")
def ag():
    return np.load(os.path.join(GOLD, "autogen.npz"))


@pytest.fixture(scope="module")
def mat():
    return np.load(os.path.join(GOLD, "matlab_unit.npz"))


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def test_delta2star3D_is_reference(ag):
    for a, E in zip(ag["d2_in"], ag["d2_E"]):
        assert rel(ol.vec_fn("hyqo_delta2star3D", a, 36).reshape(6, 6), E) < 1e-11


def test_bounds_are_reference(ag):
    for a, lb, bm in zip(ag["d2_in"], ag["lb_S220"], ag["bound_minor1"]):
        g = dict(zip(["300", "400", "110", "210", "310", "120", "220", "030", "130", "040", "101", "201", "301", "102", "202",
                      "003", "103", "004", "011", "111", "211", "021", "121", "031", "012", "112", "013", "022"], a))
        o = ol.vec_fn("hyqo_lower_bound_S220", [g[k] for k in ["011", "012", "021", "101", "102", "110", "111", "120", "201", "210"]], 3)
        assert rel(o, lb) < 1e-11
        o = ol.vec_fn("hyqo_bound_minor1", [g[k] for k in ["003", "011", "012", "021", "030", "101", "102", "110", "111", "120",
                                                           "201", "210", "300"]], 12)
        assert rel(o, bm) < 1e-11


def test_jacobian6_is_reference(ag):
    errs = [rel(ol.vec_fn("hyqo_jacobian6", a, 36).reshape(6, 6), J) for a, J in zip(ag["jac_in"], ag["jac_J"])]
    assert np.median(errs) < 1e-13
    assert max(errs) < 1e-8


def test_L3_sign_and_value(ag):
    for a, o in zip(ag["L3_in"], ag["L3_out"]):
        v = ol.delta2starchol_L3(a)
        assert np.sign(v) == np.sign(o)
        assert abs(v - o) <= 1e-11 * max(1.0, abs(o))


@pytest.mark.parametrize("name,key", [("hyqo_rootsR", "rootsR"), ("hyqo_rootsR_X_Y", "rXY")])
def test_cubic_roots(ag, name, key):
    for a, re, im in zip(ag[key + "_in"], ag[key + "_re"], ag[key + "_im"]):
        r, i = ol.roots(name, a)
        if np.all(np.isfinite(re)):
            R1, R2 = np.sort_complex(re + 1j * im), np.sort_complex(r + 1j * i)
            assert np.max(np.abs(R1 - R2)) < 1e-9 * max(1.0, np.max(np.abs(R1)))
        else:  # three real roots: the reference's fast-math Cardano form is NaN
            assert not np.any(np.isfinite(r))


def test_moment_conversions_are_reference(ag):
    for a, o in zip(ag["m4c_in"], ag["m4c_out"]):
        assert rel(ol.vec_fn("hyqo_m4toc4", a, 35), o) < 1e-11


def test_matlab_initialization(mat):
    for case in ("case1", "case2", "case3"):
        p = "test_initialization_golden." + case
        rho, u, v, w, T = (float(mat[f"{p}.input.{k}"].ravel()[0]) for k in ("rho", "u", "v", "w", "T"))
        corr = mat[f"{p}.input.corr"].ravel()
        C200 = C020 = C002 = T
        M = ol.initialize_m4_35(rho, u, v, w, C200, corr[0] * np.sqrt(C200 * C020), corr[1] * np.sqrt(C200 * C002), C020,
                                corr[2] * np.sqrt(C020 * C002), C002)
        np.testing.assert_allclose(M, mat[p + ".output"].ravel(), atol=GOLDEN_TOL, rtol=0)


def test_matlab_moment_conversions(mat):
    p = "test_moment_conversions_golden.gaussian"
    rho, u, v, w, T = (float(mat[f"{p}.input.{k}"].ravel()[0]) for k in ("rho", "u", "v", "w", "T"))
    M = ol.initialize_m4_35(rho, u, v, w, T, 0, 0, T, 0, T)
    C, S = ol.m2cs4_35(M)
    np.testing.assert_allclose(M, mat[p + ".output.M"].ravel(), atol=GOLDEN_TOL, rtol=0)
    np.testing.assert_allclose(C, mat[p + ".output.C4"].ravel(), atol=GOLDEN_TOL, rtol=0)
    np.testing.assert_allclose(S, mat[p + ".output.S4"].ravel(), atol=GOLDEN_TOL, rtol=0)
    p = "test_moment_conversions_golden.correlated"
    g = {k: float(mat[f"{p}.input.{k}"].ravel()[0]) for k in ("rho", "u", "v", "w", "C200", "C110", "C101", "C020", "C011", "C002")}
    M = ol.initialize_m4_35(g["rho"], g["u"], g["v"], g["w"], g["C200"], g["C110"], g["C101"], g["C020"], g["C011"], g["C002"])
    C, S = ol.m2cs4_35(M)
    np.testing.assert_allclose(M, mat[p + ".output.M"].ravel(), atol=GOLDEN_TOL, rtol=0)
    np.testing.assert_allclose(C, mat[p + ".output.C4"].ravel(), atol=GOLDEN_TOL, rtol=0)
    np.testing.assert_allclose(S, mat[p + ".output.S4"].ravel(), atol=GOLDEN_TOL, rtol=0)


def test_matlab_realizability_S2(mat):
    for c in (1, 2, 3):
        p = f"test_realizability_golden.S2_case{c}"
        o = ol.realizability_S2(*(float(mat[f"{p}.input.{k}"].ravel()[0]) for k in ("S110", "S101", "S011")))
        exp = [float(mat[f"{p}.output.{k}"].ravel()[0]) for k in ("S110r", "S101r", "S011r", "S2r")]
        np.testing.assert_allclose(o, exp, atol=GOLDEN_TOL, rtol=0)


def test_matlab_closure_1d(mat):
    p = "test_closures_golden.closure_1d"
    Mp, vmin, vmax = ol.closure_and_eigenvalues(mat[p + ".input"].ravel())
    assert abs(Mp - mat[p + ".output.Mp"].ravel()[0]) < GOLDEN_TOL
    assert abs(vmin - mat[p + ".output.vpmin"].ravel()[0]) < 1e-5  # golden stored to 6 digits
    assert abs(vmax - mat[p + ".output.vpmax"].ravel()[0]) < 1e-5


def test_matlab_flux_and_eigenvalues(mat):
    p = "test_flux_eigenvalues_golden.flux_basic"
    Fx, Fy, Fz, Mr = ol.flux_closure35(mat[p + ".input"].ravel(), 1, 0.5)
    for got, k in ((Fx, "Fx"), (Fy, "Fy"), (Fz, "Fz"), (Mr, "M_real")):
        np.testing.assert_allclose(got, mat[f"{p}.output.{k}"].ravel(), atol=GOLDEN_TOL, rtol=0)
    p = "test_flux_eigenvalues_golden.eigenvalues"
    M = mat[p + ".input"].ravel()
    vx = ol.eigenvalues6(M, 1, 1, 0.5)
    vy = ol.eigenvalues6(M, 2, 1, 0.5)
    assert abs(vx[0] - mat[p + ".output.v6min_x"].ravel()[0]) < 1e-5
    assert abs(vx[1] - mat[p + ".output.v6max_x"].ravel()[0]) < 1e-5
    assert abs(vy[0] - mat[p + ".output.v6min_y"].ravel()[0]) < 1e-5
    assert abs(vy[1] - mat[p + ".output.v6max_y"].ravel()[0]) < 1e-5


def test_matlab_pas_hll(mat):
    p = "test_numerical_schemes_golden.pas_hll"
    Mp = ol.pas_hll(mat[p + ".input.M"], mat[p + ".input.F"], float(mat[p + ".input.dt"].ravel()[0]),
                    float(mat[p + ".input.dx"].ravel()[0]), mat[p + ".input.vpmin"].ravel(), mat[p + ".input.vpmax"].ravel())
    np.testing.assert_allclose(Mp, mat[p + ".output"], atol=GOLDEN_TOL, rtol=0)


def test_matlab_collision(mat):
    p = "test_collision_golden.basic"
    out = ol.collision35(mat[p + ".input.M"].ravel(), float(mat[p + ".input.dt"].ravel()[0]), float(mat[p + ".input.Kn"].ravel()[0]))
    np.testing.assert_allclose(out, mat[p + ".output"].ravel(), atol=GOLDEN_TOL, rtol=0)


def test_matlab_check2d(mat):
    p = "test_diagnostics_golden.check2d"
    names = ("S30", "S40", "S11", "S21", "S31", "S12", "S22", "S03", "S13", "S04")
    out = ol.check2d([float(mat[f"{p}.input.{k}"].ravel()[0]) for k in names])
    exp = [float(mat[f"{p}.output.{k}"].ravel()[0]) for k in names]
    np.testing.assert_allclose(out, exp, atol=GOLDEN_TOL, rtol=0)


@pytest.mark.parametrize("name", ["small", "medium"])
def test_end_to_end_nz1_golden(name):
    g = np.load(os.path.join(GOLD, f"mpi_1rank_{name}.npz"))
    Np, tmax = int(g["Np"]), float(g["tmax"])
    params = ic.run_simulation_params(Nx=Np, Ny=Np, Nz=1, tmax=tmax, Kn=1.0, Ma=0.0, flag2D=0, CFL=0.5)
    M = ic.initial_state(params)
    grid = ic.grid_spacing(params)
    p = dict(params, **grid)
    t, nn = 0.0, 0
    while t < tmax and nn < params["nnmax"]:
        _, t, _ = ol.step(M, p, t)
        nn += 1
    assert nn == int(g["steps"])
    assert t == float(g["tfinal"])
    np.testing.assert_allclose(M[:, :, 0, :], g["M"], atol=1e-12, rtol=0)
