"""Device diagnostics of the step against host computations from the oracle:

* the first-step vmax breakdown (src/simulation_runner.jl:404-470): the
  largest |wave speed| along x, y and z at step 1 and the worst cell, against
  phase [A]'s per-cell speeds from the oracle;
* MaxDiff (src/simulation_runner.jl:562-637), the diagonal symmetry measure,
  at the reference's cadence (nn % symmetry_check_interval == 0 or nn == 1),
  against the formula evaluated on the host from the same state.
"""
import numpy as np
import pytest

import oracle_lib as ol
from hyqmom import ic

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def host_maxdiff(M):
    Nd = min(M.shape[0], M.shape[1])
    diag = np.array([M[i, i, 0, :5] for i in range(Nd)])
    out = []
    for m in range(5):
        a, b = diag[:, m], diag[::-1, m]
        d = a + b if m % 2 else a - b
        out.append(abs(np.max(d) / (np.linalg.norm(d) + 1.0)))
    return max(out)


def test_first_step_breakdown_matches_oracle_speeds():
    need_gpu()
    from hyqmom.runner import Solver
    p = ic.with_jets(ic.default_params(Nx=8, Ny=8, Nz=6, Ma=1.0, Kn=1.0, CFL=0.5, tmax=10.0, nnmax=10), "crossing")
    M0 = ic.initial_state(p)
    s = Solver(p)
    try:
        s.set_state(M0)
        s.advance(1)
        st = s.stats()
    finally:
        s.close()
    cells = M0.reshape(-1, 35, order="F")
    v = np.zeros((cells.shape[0], 6))
    for c, m in enumerate(cells):
        _, _, _, a = ol.flux_closure35(m, 0, p["Ma"])
        vx0, vx1, b = ol.eigenvalues6(a, 1, 0, p["Ma"])
        vy0, vy1, b2 = ol.eigenvalues6(b, 2, 0, p["Ma"])
        vz0, vz1, b3 = ol.eigenvalues6z(b2, 0, p["Ma"], True)
        _, _, _, r = ol.flux_closure35(b3, 0, p["Ma"])
        e = [ol.closure_and_eigenvalues(r[idx]) for idx in ([0, 1, 2, 3, 4], [0, 5, 9, 12, 14], [0, 15, 19, 22, 24])]
        v[c] = [min(e[0][1], vx0), max(e[0][2], vx1), min(e[1][1], vy0), max(e[1][2], vy1), min(e[2][1], vz0), max(e[2][2], vz1)]
    a = np.abs(v)
    ref = [a[:, 0:2].max(), a[:, 2:4].max(), a[:, 4:6].max()]
    assert list(st["vmax_first"]) == ref, (st["vmax_first"], ref)
    assert max(ref) == st["vmax"]
    worst = np.argmax(a.max(axis=1))
    assert st["worst_cell"] == worst
    assert st["worst_dir"] == int(np.argmax([a[worst, 0:2].max(), a[worst, 2:4].max(), a[worst, 4:6].max()]))


def test_maxdiff_at_the_reference_cadence():
    need_gpu()
    from hyqmom.runner import Solver
    p = ic.with_jets(ic.default_params(Nx=12, Ny=12, Nz=4, Ma=1.0, Kn=1.0, CFL=0.5, tmax=10.0, nnmax=20, symmetry_check_interval=4),
                     "crossing")
    s = Solver(p)
    try:
        s.set_state(ic.initial_state(p))
        seen = []
        for k in range(1, 10):
            s.advance(1)
            st = s.stats()
            seen.append(st["maxdiff_step"])
            if st["maxdiff_step"] == k:
                ref = host_maxdiff(s.get_state())
                assert abs(st["maxdiff"] - ref) <= 1e-12 * max(1.0, ref), (k, st["maxdiff"], ref)
        assert seen == [1, 1, 1, 4, 4, 4, 4, 8, 8], seen
    finally:
        s.close()
