"""Rare branches of the reference's algorithm are exercised and agree.

The oracle built with branch-hit counters (oracle/liboracle_branches.so)
runs phase [A]'s per-cell sequence (Flux_closure35_and_realizable_3D, then
eigenvalues6_hyperbolic_3D x and y, then eigenvalues6z_hyperbolic_3D) on the
states of branch_states.py; every counted branch must be taken at least
once: edge_corner_correction, the flag220
repeats, the complex-eigenvalue corrections (x/y and z), the three-real-root
NaN of rootsR and rootsR_X_Y, and eigenvalues6z's re-realization.

The faces case of realizable_3D (S2 <= S2min, src/realizability/
realizable_3D.jl:79-142) cannot be reached through
Flux_closure35_and_realizable_3D: every state with |S_ij| >= 1 goes to
edge_corner_correction first, and realizability_S2 contracts (S110, S101,
S011) by 0.9999 before the test, which leaves S2 = 1 + 2 x^3 P - x^2 Q far
above 1e-12 (x = 0.9999 times the bisection root, where Y' < 0).  It is
exercised by calling realizable_3D itself on correlations at a corner of the
elliptope scaled out by 1 / 0.9999 (where the contraction lands S2 on 0), the
device source (compiled for the host) against the oracle, bit for bit.  The GPU
test runs the same states through the device's per-cell phase [A] and
requires the oracle's results (FP64, 1e-12 relative per moment field; the
two are bit-identical in practice), so the device takes the same branches.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol
from branch_states import branch_states, negative_variance_rows

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BRANCH_LIB = os.path.join(ROOT, "oracle", "liboracle_branches.so")
NAMES = ["faces", "edge_corner", "flag220_repeat", "complex_xy", "complex_z", "rootsR_nan", "rootsR_X_Y_nan", "rerealize_z"]
_dp = ctypes.POINTER(ctypes.c_double)


def branch_lib():
    if not os.path.exists(BRANCH_LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return ctypes.CDLL(BRANCH_LIB)


def phase_a_oracle(lib, m, Ma=1.0):
    """Phase [A] per cell on the instrumented oracle: returns (Mr, v[6])."""
    def p(a):
        return a.ctypes.data_as(_dp)
    m = np.ascontiguousarray(m, dtype=np.float64)
    Fx, Fy, Fz, a = (np.zeros(35) for _ in range(4))
    lib.hyqo_flux_closure35(p(m), ctypes.c_int(0), ctypes.c_double(Ma), p(Fx), p(Fy), p(Fz), p(a))
    v = np.zeros(6)
    b, c, d = np.zeros(35), np.zeros(35), np.zeros(35)
    vv = np.zeros(2)
    lib.hyqo_eigenvalues6(p(a), ctypes.c_int(1), ctypes.c_int(0), ctypes.c_double(Ma), p(vv), p(b))
    v[0:2] = vv
    lib.hyqo_eigenvalues6(p(b), ctypes.c_int(2), ctypes.c_int(0), ctypes.c_double(Ma), p(vv), p(c))
    v[2:4] = vv
    lib.hyqo_eigenvalues6z(p(c), ctypes.c_int(0), ctypes.c_double(Ma), ctypes.c_int(1), p(vv), p(d))
    v[4:6] = vv
    return d, v


@pytest.fixture(scope="module")
def states():
    return branch_states()


def test_states_take_every_counted_branch(states):
    lib = branch_lib()
    out = (ctypes.c_longlong * 8)()
    lib.hyqo_branch_counts(out, 1)
    for s in states:
        phase_a_oracle(lib, s)
    # the z function directly on the unrealized negative-variance states
    for s in states[negative_variance_rows(states)]:
        m = np.ascontiguousarray(s)
        vv, r = np.zeros(2), np.zeros(35)
        lib.hyqo_eigenvalues6z(m.ctypes.data_as(_dp), ctypes.c_int(0), ctypes.c_double(1.0), ctypes.c_int(1), vv.ctypes.data_as(_dp),
                               r.ctypes.data_as(_dp))
    lib.hyqo_branch_counts(out, 1)
    hits = dict(zip(NAMES, list(out)))
    print("branch hits over", len(states), "states:", hits)
    # the faces case is unreachable through the closure (module docstring);
    # test_faces_case_device_source_matches_oracle takes it directly
    assert hits["faces"] == 0
    assert all(v > 0 for k, v in hits.items() if k != "faces"), hits


def test_uninstrumented_oracle_counts_nothing():
    lib = ol.load()
    out = (ctypes.c_longlong * 8)()
    lib.hyqo_branch_counts(out, 0)
    assert list(out) == [0] * 8


@pytest.mark.gpu
def test_device_phase_a_matches_oracle_on_branch_states(states):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hyqmom import _lib
    lib = _lib.load()
    n = states.shape[0]
    dM = torch.tensor(np.ascontiguousarray(states.T), dtype=torch.float64, device="cuda")
    outs = [torch.empty_like(dM) for _ in range(4)]
    vp = torch.empty(6, n, dtype=torch.float64, device="cuda")
    assert lib.hyq_cells_phase_A(dM.data_ptr(), n, 0, 1.0, 1, *[o.data_ptr() for o in outs], vp.data_ptr(), None) == 0
    torch.cuda.synchronize()
    got_M = outs[3].cpu().numpy().T
    olib = branch_lib()
    ref = [phase_a_oracle(olib, s) for s in states]
    ref_M = np.array([r[0] for r in ref])
    # phase [A]'s realized state: the closure of the corrected moments (the
    # device's Mr output), compared per moment field
    fx = np.array([ol.flux_closure35(r, 0, 1.0)[3] for r in ref_M])
    scale = np.maximum(np.max(np.abs(fx), axis=0), 1e-300)
    rel = np.max(np.where(np.isnan(fx) & np.isnan(got_M), 0.0, np.abs(got_M - fx)), axis=0) / scale
    assert np.nanmax(rel) <= 1e-12, np.nanmax(rel)
    assert np.array_equal(np.isnan(got_M), np.isnan(fx))


@pytest.mark.gpu
def test_device_z_eigenvalues_match_oracle_on_negative_variance(states):
    """eigenvalues6z on unrealized states with a negative variance (its
    re-realization branch): device per-cell entry against the oracle."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hyqmom import _lib
    lib = _lib.load()
    rows = states[negative_variance_rows(states)]
    n = rows.shape[0]
    assert n > 0
    dM = torch.tensor(np.ascontiguousarray(rows.T), dtype=torch.float64, device="cuda")
    v = torch.empty(2, n, dtype=torch.float64, device="cuda")
    Mr = torch.empty_like(dM)
    assert lib.hyq_cells_eigenvalues(dM.data_ptr(), n, 3, 0, 1.0, 1, v.data_ptr(), Mr.data_ptr(), None) == 0
    torch.cuda.synchronize()
    gv, gM = v.cpu().numpy().T, Mr.cpu().numpy().T
    for c in range(n):
        a, b, r = ol.eigenvalues6z(rows[c], 0, 1.0, True)
        assert np.array_equal(np.array([gv[c, 0], gv[c, 1]]), np.array([a, b]), equal_nan=True), (c, gv[c], a, b)
        assert np.array_equal(gM[c], r, equal_nan=True)


def face_inputs(n=24, seed=4):
    """28-sets (s300, s400, s110, ...) with (S110, S101, S011) = v_i v_j /
    0.9999 for a sign vector v and Gaussian-like other moments."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        v = rng.choice([-1.0, 1.0], 3)
        a = {k: 0.0 for k in ["s300", "s400", "s110", "s210", "s310", "s120", "s220", "s030", "s130", "s040", "s101", "s201", "s301",
                               "s102", "s202", "s003", "s103", "s004", "s011", "s111", "s211", "s021", "s121", "s031", "s012", "s112",
                               "s013", "s022"]}
        c = {"s110": v[0] * v[1], "s101": v[0] * v[2], "s011": v[1] * v[2]}
        for k, x in c.items():
            a[k] = x / 0.9999 * (1 + 1e-14 * rng.normal())
        a["s400"] = a["s040"] = a["s004"] = 3.0 + rng.uniform(0, 0.5)
        a["s220"] = 1 + 2 * c["s110"] ** 2
        a["s202"] = 1 + 2 * c["s101"] ** 2
        a["s022"] = 1 + 2 * c["s011"] ** 2
        a["s310"] = a["s130"] = 3 * c["s110"]
        a["s301"] = a["s103"] = 3 * c["s101"]
        a["s031"] = a["s013"] = 3 * c["s011"]
        a["s211"] = c["s011"] + 2 * c["s110"] * c["s101"]
        a["s121"] = c["s101"] + 2 * c["s110"] * c["s011"]
        a["s112"] = c["s110"] + 2 * c["s101"] * c["s011"]
        out.append(np.array(list(a.values())))
    return out


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = tmp_path_factory.mktemp("shim_br") / "libshim.so"
    here = os.path.dirname(os.path.abspath(__file__))
    subprocess.check_call(["/usr/bin/g++", "-O2", "-std=c++17", "-fno-fast-math", "-ffp-contract=off", "-fPIC", "-shared", "-I",
                           os.path.join(ROOT, "hyqmom.jl_b200", "csrc"), "-o", str(out), os.path.join(here, "host_device_shim.cpp")])
    return ctypes.CDLL(str(out))


def test_faces_case_device_source_matches_oracle(shim):
    lib = branch_lib()
    cnt = (ctypes.c_longlong * 8)()
    lib.hyqo_branch_counts(cnt, 1)
    for a in face_inputs():
        ref = np.ascontiguousarray(a.copy())
        flag = ctypes.c_int()
        lib.hyqo_realizable_3d(ref.ctypes.data_as(_dp), ctypes.byref(flag))
        dev = np.ascontiguousarray(a.copy())
        dflag = shim.sh_realizable_3d(dev.ctypes.data_as(_dp))
        assert dflag == flag.value
        assert np.array_equal(dev, ref, equal_nan=True)
    lib.hyqo_branch_counts(cnt, 1)
    assert cnt[0] > 0, list(cnt)
