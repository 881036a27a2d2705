"""ctypes access to the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is test infrastructure: a scalar C++ restatement of the
reference's serial time step.  Only tests, ``__graft_entry__.smoke()`` and the
bench's CPU-baseline leg load it, and only as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_lib = None


def _p(a):
    return a.ctypes.data_as(_dp)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    lib = ctypes.CDLL(LIB_PATH)
    lib.hyqo_step.restype = ctypes.c_double
    lib.hyqo_step.argtypes = [ctypes.c_int] * 3 + [_dp] + [ctypes.c_double] * 2 + [ctypes.c_int] + \
        [ctypes.c_double] * 6 + [ctypes.c_int, _dp, _dp]
    lib.hyqo_delta2starchol_L3.restype = ctypes.c_double
    lib.hyqo_eig6.restype = ctypes.c_int
    lib.hyqo_step_begin.restype = ctypes.c_void_p
    lib.hyqo_step_begin.argtypes = [ctypes.c_int] * 3 + [_dp] + [ctypes.c_double] * 2 + [ctypes.c_int] + \
        [ctypes.c_double] * 6 + [ctypes.c_int, _dp]
    lib.hyqo_step_end.restype = ctypes.c_double
    lib.hyqo_step_end.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, _dp]
    lib.hyqo_set_threads.argtypes = [ctypes.c_int]
    lib.hyqo_set_threads.restype = None
    _lib = lib
    return lib


def f64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def initialize_m4_35(rho, u, v, w, C200, C110, C101, C020, C011, C002):
    out = np.zeros(35)
    load().hyqo_initialize_m4_35(*[ctypes.c_double(float(x)) for x in (rho, u, v, w, C200, C110, C101, C020, C011, C002)], _p(out))
    return out


def m2cs4_35(M):
    M = f64(M)
    C, S = np.zeros(35), np.zeros(35)
    load().hyqo_m2cs4_35(_p(M), _p(C), _p(S))
    return C, S


def flux_closure35(M, flag2D, Ma):
    M = f64(M)
    o = [np.zeros(35) for _ in range(4)]
    load().hyqo_flux_closure35(_p(M), ctypes.c_int(flag2D), ctypes.c_double(Ma), *[_p(x) for x in o])
    return tuple(o)


def eigenvalues6(M, axis, flag2D, Ma):
    M = f64(M)
    v, Mr = np.zeros(2), np.zeros(35)
    load().hyqo_eigenvalues6(_p(M), ctypes.c_int(axis), ctypes.c_int(flag2D), ctypes.c_double(Ma), _p(v), _p(Mr))
    return v[0], v[1], Mr


def eigenvalues6z(M, flag2D, Ma, positivity=True):
    M = f64(M)
    v, Mr = np.zeros(2), np.zeros(35)
    load().hyqo_eigenvalues6z(_p(M), ctypes.c_int(flag2D), ctypes.c_double(Ma), ctypes.c_int(int(positivity)), _p(v), _p(Mr))
    return v[0], v[1], Mr


def closure_and_eigenvalues(mom):
    mom = f64(mom)
    out = np.zeros(3)
    load().hyqo_closure_and_eigenvalues(_p(mom), _p(out))
    return tuple(out)


def collision35(M, dt, Kn, positivity=True):
    M = f64(M)
    out = np.zeros(35)
    load().hyqo_collision35(_p(M), ctypes.c_double(dt), ctypes.c_double(Kn), ctypes.c_int(int(positivity)), _p(out))
    return out


def pas_hll(M, F, dt, dx, vpmin, vpmax):
    M = np.asfortranarray(M, dtype=np.float64)
    F = np.asfortranarray(F, dtype=np.float64)
    Mp = np.zeros_like(M, order="F")
    vpmin, vpmax = f64(vpmin), f64(vpmax)
    load().hyqo_pas_hll(ctypes.c_int(M.shape[0]), M.ctypes.data_as(_dp), F.ctypes.data_as(_dp), ctypes.c_double(dt),
                        ctypes.c_double(dx), _p(vpmin), _p(vpmax), Mp.ctypes.data_as(_dp))
    return Mp


def realizability_S2(S110, S101, S011):
    out = np.zeros(4)
    load().hyqo_realizability_S2(ctypes.c_double(S110), ctypes.c_double(S101), ctypes.c_double(S011), _p(out))
    return tuple(out)


def check2d(s10):
    s = f64(s10).copy()
    load().hyqo_check2d(_p(s))
    return s


def vec_fn(name, inp, nout):
    inp = f64(inp)
    out = np.zeros(nout)
    getattr(load(), name)(_p(inp), _p(out))
    return out


def roots(name, inp):
    inp = f64(inp)
    re, im = np.zeros(3), np.zeros(3)
    getattr(load(), name)(_p(inp), _p(re), _p(im))
    return re, im


def delta2starchol_L3(a):
    a = f64(a)
    return load().hyqo_delta2starchol_L3(_p(a))


def eig6(A):
    A = f64(A)
    wr, wi = np.zeros(6), np.zeros(6)
    info = load().hyqo_eig6(_p(A), _p(wr), _p(wi))
    return wr, wi, info


def c5tom5(M000, u, v, w, Ccube):
    Ccube = f64(Ccube)
    out = np.zeros(216)
    load().hyqo_c5tom5(ctypes.c_double(M000), ctypes.c_double(u), ctypes.c_double(v), ctypes.c_double(w), _p(Ccube), _p(out))
    return out


def s4toc4_r(C2, Scube):
    C2, Scube = f64(C2), f64(Scube)
    out = np.zeros(216)
    load().hyqo_s4toc4_r(_p(C2), _p(Scube), _p(out))
    return out


def step(M, params, t):
    """One serial step on M (Nx,Ny,Nz,35) Fortran-ordered, in place.
    Returns (dt, t_new, vmax)."""
    assert M.flags["F_CONTIGUOUS"] and M.dtype == np.float64
    Nx, Ny, Nz, _ = M.shape
    tt = np.array([t], dtype=np.float64)
    vm = np.zeros(1)
    p = params
    dt = load().hyqo_step(Nx, Ny, Nz, M.ctypes.data_as(_dp), p["Kn"], p["Ma"], int(p["flag2D"]), p["CFL"], p["dtmax"],
                          p["tmax"], p["dx"], p["dy"], p["dz"], int(p.get("positivity", True)), _p(tt), _p(vm))
    return dt, float(tt[0]), float(vm[0])


def step_begin(M, params):
    """Phase [A] of a step on M in place; returns (work handle, local vmax)."""
    assert M.flags["F_CONTIGUOUS"] and M.dtype == np.float64
    Nx, Ny, Nz, _ = M.shape
    vm = np.zeros(1)
    p = params
    w = load().hyqo_step_begin(Nx, Ny, Nz, M.ctypes.data_as(_dp), p["Kn"], p["Ma"], int(p["flag2D"]), p["CFL"], p["dtmax"],
                               p["tmax"], p["dx"], p["dy"], p["dz"], int(p.get("positivity", True)), _p(vm))
    return w, float(vm[0])


def step_end(work, M, vmax, t):
    """The rest of the step with the (global) vmax; returns (dt, t_new)."""
    tt = np.array([t], dtype=np.float64)
    dt = load().hyqo_step_end(ctypes.c_void_p(work), M.ctypes.data_as(_dp), float(vmax), _p(tt))
    return dt, float(tt[0])


def count_ops_stages(M, params, dt):
    """Per-kernel FP64 op counts of the staged step, summed over cells (9)."""
    M = np.asfortranarray(M, dtype=np.float64)
    Nx, Ny, Nz, _ = M.shape
    out = np.zeros(9)
    p = params
    load().hyqo_count_ops_stages(Nx, Ny, Nz, M.ctypes.data_as(_dp), ctypes.c_double(p["Kn"]), ctypes.c_double(p["Ma"]),
                                 int(p["flag2D"]), int(p.get("positivity", True)), ctypes.c_double(dt), _p(out))
    return out


def count_ops(M, params, dt):
    M = np.asfortranarray(M, dtype=np.float64)
    Nx, Ny, Nz, _ = M.shape
    out = np.zeros(3)
    p = params
    load().hyqo_count_ops(Nx, Ny, Nz, M.ctypes.data_as(_dp), ctypes.c_double(p["Kn"]), ctypes.c_double(p["Ma"]),
                          int(p["flag2D"]), int(p.get("positivity", True)), ctypes.c_double(dt), _p(out))
    return out


def _field_rel(a, b):
    a = a.reshape(-1, 35)
    b = b.reshape(-1, 35)
    return float(np.max(np.max(np.abs(a - b), axis=0) / np.maximum(np.max(np.abs(b), axis=0), 1e-300)))


def one_ulp_spread(M, pp, t, trials=3, seed=0):
    """The oracle's own one-step spread at state M: the largest field-relative
    difference between its step from M and its steps from M with every entry
    moved by one ulp (random direction), over `trials` perturbations."""
    A = np.asfortranarray(M.copy())
    step(A, pp, t)
    rng = np.random.default_rng(seed)
    worst = 0.0
    for _ in range(trials):
        flat = np.array(M, order="F").reshape(-1, order="F")
        up = rng.random(flat.size) < 0.5
        flat = np.where(up, np.nextafter(flat, np.inf), np.nextafter(flat, -np.inf))
        B = np.asfortranarray(flat.reshape(M.shape, order="F"))
        step(B, pp, t)
        worst = max(worst, _field_rel(B, A))
    return worst



def step_end_hll(work, M, vmax, t):
    """The rest of the step stopped after the HLL combination: M becomes the
    state phases [E]+[F] start from; returns (dt, t_new)."""
    lib = load()
    lib.hyqo_step_end_hll.restype = ctypes.c_double
    tt = np.array([t], dtype=np.float64)
    dt = lib.hyqo_step_end_hll(ctypes.c_void_p(work), M.ctypes.data_as(_dp), ctypes.c_double(vmax), _p(tt))
    return dt, float(tt[0])


def phase_EF(M, params, dt):
    """Phases [E]+[F] in place on a post-HLL state M with the step's dt."""
    assert M.flags["F_CONTIGUOUS"] and M.dtype == np.float64
    Nx, Ny, Nz, _ = M.shape
    p = params
    load().hyqo_phase_EF(Nx, Ny, Nz, M.ctypes.data_as(_dp), ctypes.c_double(p["Kn"]), ctypes.c_double(p["Ma"]), int(p["flag2D"]),
                         int(p.get("positivity", True)), ctypes.c_double(dt))


def post_hll_spread(M, pp, t, trials=6, seed=0):
    """The oracle's own spread in the part of its step after the wave speeds:
    the largest field-relative difference between phases [E]+[F] on its HLL
    output from M and on that output with every entry moved by one ulp
    (random direction), over `trials` perturbations."""
    A = np.asfortranarray(M.copy())
    w, vm = step_begin(A, pp)
    dt, _ = step_end_hll(w, A, vm, t)
    base = A.copy(order="F")
    phase_EF(base, pp, dt)
    rng = np.random.default_rng(seed)
    worst = 0.0
    for _ in range(trials):
        flat = A.reshape(-1, order="F")
        up = rng.random(flat.size) < 0.5
        B = np.asfortranarray(np.where(up, np.nextafter(flat, np.inf), np.nextafter(flat, -np.inf)).reshape(A.shape, order="F"))
        phase_EF(B, pp, dt)
        worst = max(worst, _field_rel(B, base))
    return worst
