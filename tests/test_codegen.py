"""Generated code: the closed-form jacobian6 shared by the CUDA path and the
oracle is current with its generator and agrees with forward-mode
differentiation of the same closure."""
import filecmp
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle_lib as ol
from hyqmom import ic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GEN = os.path.join(ROOT, "hyqmom.jl_b200", "codegen", "gen_jacobian6.py")


def test_generated_jacobian_is_current(tmp_path):
    pytest.importorskip("sympy")
    subprocess.check_call([sys.executable, GEN, str(tmp_path)], timeout=300)
    fresh = os.path.join(tmp_path, "gen_jacobian6.inc")
    for dst in (os.path.join(ROOT, "hyqmom.jl_b200", "csrc", "gen_jacobian6.inc"), os.path.join(ROOT, "oracle", "gen_jacobian6.inc")):
        assert filecmp.cmp(fresh, dst, shallow=False), dst


def slices(n=300, seed=3):
    """15-moment (x, y) slices of Gaussian-mixture states in jacobian6 order."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        k = rng.integers(1, 4)
        m = np.zeros(35)
        for w in rng.dirichlet(np.ones(k)) * (0.01 + rng.random()):
            mu = rng.normal(0, 1.5, size=3)
            A = rng.normal(size=(3, 3))
            Cv = A @ A.T / 3 + 0.1 * np.eye(3)
            m += ic.gaussian_moments(w, *mu, Cv[0, 0], Cv[0, 1], Cv[0, 2], Cv[1, 1], Cv[1, 2], Cv[2, 2])
        E = {e: i for i, e in enumerate(ic.E35)}
        out.append([m[E[(a, b, 0)]] for (a, b) in [(0, 0), (0, 1), (0, 2), (0, 3), (0, 4), (1, 0), (1, 1), (1, 2), (1, 3),
                                                    (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (4, 0)]])
    return np.array(out)


def test_closed_form_matches_dual_numbers():
    errs = []
    for a in slices():
        J = ol.vec_fn("hyqo_jacobian6", a, 36)
        Jd = ol.vec_fn("hyqo_jacobian6_ad", a, 36)
        errs.append(np.max(np.abs(J - Jd)) / np.max(np.abs(Jd)))
    assert np.median(errs) < 1e-14 and max(errs) < 1e-11
