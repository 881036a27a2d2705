"""The learned wave-speed path on the host (no GPU):

* the certified characteristic-polynomial solve (hyq_charpoly.cuh, compiled
  with g++ from the device source) against the LAPACK-path eigen-solve of the
  oracle on flux Jacobians of evolved crossing-jet states: every certified
  Jacobian is one whose eigenvalues the reference calls real, and its extreme
  eigenvalues agree to 1e-13 relative (FP64 throughout);
* seeds near the extremes cut the solve's polynomial evaluations;
* the host FP64 reference of the network's backward pass against finite
  differences, and the Gaussian-mixture moment sampler against the
  reference's own Gaussian moments (InitializeM4_35).
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol
from hyqmom import ic, wavenet

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "hyqmom.jl_b200", "csrc")
SLICES = ([0, 5, 9, 12, 14, 1, 6, 10, 13, 2, 7, 11, 3, 8, 4], [0, 15, 19, 22, 24, 1, 16, 20, 23, 2, 17, 21, 3, 18, 4])
EPS = 2.220446049250313e-16
_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = tmp_path_factory.mktemp("shim_cp") / "libshim.so"
    subprocess.check_call(["/usr/bin/g++", "-O2", "-std=c++17", "-fno-fast-math", "-ffp-contract=off", "-fPIC", "-shared",
                           "-I", CSRC, "-o", str(out), os.path.join(HERE, "host_device_shim.cpp")])
    return ctypes.CDLL(str(out))


@pytest.fixture(scope="module")
def jacobians():
    """Flux Jacobians (x planes) of the realized moments of a 14^3 crossing-jet
    run at Ma=1, Kn=0.01 (CFL 0.5), sampled at steps 10, 20, 30."""
    p = ic.with_jets(ic.default_params(Nx=14, Ny=14, Nz=14, Ma=1.0, Kn=0.01, CFL=0.5, tmax=10.0, nnmax=100), "crossing")
    M = np.asfortranarray(ic.initial_state(p))
    pp = dict(p, **ic.grid_spacing(p))
    t, out = 0.0, []
    lib = ol.load()
    rng = np.random.default_rng(0)
    for s in range(30):
        _, t, _ = ol.step(M, pp, t)
        if s % 10 == 9:
            S = np.array(M).reshape(-1, 35, order="F")
            for c in rng.choice(len(S), 500, replace=False):
                _, _, _, Mr = ol.flux_closure35(S[c].copy(), 0, 1.0)
                for sl in SLICES:
                    a = np.ascontiguousarray(Mr[sl])
                    J = np.zeros(36)
                    lib.hyqo_jacobian6(_p(a), _p(J))
                    out.append(J)
    return np.array(out)


def cp_extremes(shim, J, lo=np.nan, hi=np.nan, margin=0.0):
    out = np.zeros(4)
    A = np.ascontiguousarray(J, dtype=np.float64)
    shim.sh_cp_extremes(_p(A), ctypes.c_double(lo), ctypes.c_double(hi), ctypes.c_double(margin), _p(out))
    return bool(out[0]), out[1], out[2], int(out[3])


def test_charpoly_is_det_of_jacobian(shim, jacobians):
    for J in jacobians[::37]:
        c = np.zeros(7)
        shim.sh_cp_charpoly(_p(np.ascontiguousarray(J)), _p(c))
        # numpy forms the polynomial from computed eigenvalues: compare against
        # the coefficients' overall magnitude (a formula error is O(1))
        ref = np.real(np.poly(J.reshape(6, 6)))[::-1]
        assert np.max(np.abs(c - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))


def test_certified_extremes_match_lapack_path(shim, jacobians):
    """Certified => the reference's complex test passes and the extremes agree
    to 1e-13 relative; most developed-flow Jacobians certify."""
    ncert = 0
    worst = 0.0
    for J in jacobians:
        ok, lo, hi, _ = cp_extremes(shim, J)
        wr, wi, info = ol.eig6(J.reshape(6, 6).copy())
        if not ok:
            continue
        ncert += 1
        assert info == 0
        assert np.max(np.abs(wi)) <= 1000 * EPS, "certified a Jacobian the LAPACK path calls complex"
        scale = np.max(np.abs(wr))
        worst = max(worst, abs(lo - wr.min()) / scale, abs(hi - wr.max()) / scale)
    assert worst < 1e-13, worst
    assert ncert > 0.9 * len(jacobians), (ncert, len(jacobians))


def test_uncertifiable_jacobians_are_refused(shim):
    """A double eigenvalue, a complex pair and non-finite entries are left to
    the LAPACK path."""
    def companion(roots_poly):
        # J with the unit rows of jacobian6 whose characteristic polynomial is
        # prod (lam - r): a block companion matrix
        c = np.real(np.poly(roots_poly))[::-1]  # c0..c6, monic
        J = np.zeros((6, 6))
        J[0, 1] = J[1, 2] = J[3, 4] = 1.0
        # rows 2, 4, 5 chosen so that det(lam I - J) = the polynomial: put the
        # whole polynomial in row 5 of a companion in (v0, v3, v5) coordinates
        # by the substitution v3 = lam^3 v0, v5 = lam^5 v0
        J[2, 3] = 1.0          # lam^3 v0 = v3
        J[4, 5] = 1.0          # lam^2 v3 = v5  (v5 = lam^5 v0)
        J[5, 0:3] = -c[0:3]    # lam v5 = -(c0 v0 + c1 v1 + c2 v2 + c3 v3 + c4 v4 + c5 v5)
        J[5, 3:6] = -c[3:6]
        return J.ravel()
    good = companion([-2.0, -1.1, -0.3, 0.4, 1.2, 2.5])
    ok, lo, hi, _ = cp_extremes(shim, good)
    assert ok and abs(lo + 2.0) < 1e-12 and abs(hi - 2.5) < 1e-12
    assert not cp_extremes(shim, companion([-2.0, -1.0, 0.5, 0.5, 1.0, 2.0]))[0]
    assert not cp_extremes(shim, companion([-2.0, -1.0, 0.5 + 0.2j, 0.5 - 0.2j, 1.0, 2.0]))[0]
    bad = good.copy()
    bad[14] = np.nan
    assert not cp_extremes(shim, bad)[0]


def test_seeds_cut_the_evaluations(shim, jacobians):
    """Starting from the true extremes (moved out by a small margin) costs
    fewer polynomial evaluations than starting from the root bound, and
    changes the extremes by round-off only."""
    plain, seeded = [], []
    for J in jacobians[::3]:
        ok0, lo0, hi0, n0 = cp_extremes(shim, J)
        if not ok0:
            continue
        wr, _, _ = ol.eig6(J.reshape(6, 6).copy())
        ok1, lo1, hi1, n1 = cp_extremes(shim, J, wr.min(), wr.max(), 0.02)
        assert ok1
        scale = np.max(np.abs(wr))
        assert abs(lo1 - lo0) <= 1e-14 * scale * 8 and abs(hi1 - hi0) <= 1e-14 * scale * 8
        plain.append(n0)
        seeded.append(n1)
    assert np.mean(seeded) < 0.9 * np.mean(plain), (np.mean(seeded), np.mean(plain))


def test_reference_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = wavenet.init_params(1).astype(np.float64)
    S = rng.normal(size=(5, 35))
    T = rng.normal(size=(5, 6))
    g, _ = wavenet.reference_gradients(p, S, T, 1.0, emulate=False)
    # the parameters are FP32 numbers, so the FP64 loss below sees the same
    # network at the unperturbed point
    for idx in (wavenet.P_W1 + 7, wavenet.P_B1 + 3, wavenet.P_W2 + 1000, wavenet.P_W3 + 77, wavenet.P_W4 + 5, wavenet.P_B4 + 2):
        h = 1e-3
        qp, qm = p.copy(), p.copy()
        qp[idx] += h
        qm[idx] -= h
        fd = (loss_f64(qp, S, T) - loss_f64(qm, S, T)) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-4 * max(1.0, abs(fd)), (idx, fd, g[idx])


def loss_f64(q, S, T):
    """0.5 * SSE of the FP64 network with parameters q (no FP32 rounding)."""
    W1 = q[wavenet.P_W1:wavenet.P_B1].reshape(128, 35)
    b1 = q[wavenet.P_B1:wavenet.P_W2]
    W2 = q[wavenet.P_W2:wavenet.P_B2].reshape(128, 128)
    b2 = q[wavenet.P_B2:wavenet.P_W3]
    W3 = q[wavenet.P_W3:wavenet.P_B3].reshape(128, 128)
    b3 = q[wavenet.P_B3:wavenet.P_W4]
    W4 = q[wavenet.P_W4:wavenet.P_B4].reshape(6, 128)
    b4 = q[wavenet.P_B4:]
    h = S
    for W, b in ((W1, b1), (W2, b2), (W3, b3)):
        z = h @ W.T + b
        h = z / (1.0 + np.exp(-z))
    y = h @ W4.T + b4
    return 0.5 * np.sum((y - T) ** 2)


def test_gaussian_moments_match_initialize_m4_35():
    rng = np.random.default_rng(5)
    for _ in range(5):
        mu = rng.normal(size=3)
        A = rng.normal(size=(3, 5)) / np.sqrt(5.0)
        C = A @ A.T
        got = wavenet.gaussian_raw_moments(mu[None, :], C[None, :, :])[:, 0]
        ref = ol.initialize_m4_35(1.0, mu[0], mu[1], mu[2], C[0, 0], C[0, 1], C[0, 2], C[1, 1], C[1, 2], C[2, 2])
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_mixture_moments_are_realizable():
    rng = np.random.default_rng(6)
    M = wavenet.mixture_moments(2000, rng, Ma=1.0)
    assert np.allclose(M[0], 1.0)
    for i2, i1 in ((2, 1), (9, 5), (19, 15)):
        assert np.all(M[i2] - M[i1] ** 2 > 0)
    # a mixture is a measure: its 2nd-order moment matrix is positive definite
    for c in range(0, 2000, 97):
        m = M[:, c]
        mom = np.array([[m[0], m[1], m[5], m[15]], [m[1], m[2], m[6], m[16]], [m[5], m[6], m[9], m[25]],
                        [m[15], m[16], m[25], m[19]]])
        assert np.linalg.eigvalsh(mom).min() > 0
