"""Batched independent domains (hyq_batch): every member of one batch, with
its own grid, parameters and dt, matches the same domain stepped alone."""
import numpy as np
import pytest

from hyqmom import ic

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hyqmom import _lib
    return _lib.load()


def field_rel(a, b):
    a = np.asarray(a).reshape(-1, 35)
    b = np.asarray(b).reshape(-1, 35)
    scale = np.maximum(np.max(np.abs(b), axis=0), 1e-300)
    return float(np.max(np.max(np.abs(a - b), axis=0) / scale))


def members():
    a = ic.with_jets(ic.default_params(Nx=12, Ny=10, Nz=8, Ma=1.0, Kn=1.0, CFL=0.5, tmax=10.0, nnmax=6), "crossing")
    b = ic.with_jets(ic.default_params(Nx=16, Ny=16, Nz=12, Ma=0.5, Kn=0.1, CFL=0.5, tmax=10.0, nnmax=4), "triple-jet")
    c = ic.run_simulation_params(Nx=14, Ny=12, Nz=6, tmax=0.02, Kn=1.0, Ma=1.0, CFL=0.5)
    c["nnmax"] = 100
    return [a, b, c]


def test_batch_members_match_single_runs():
    cuda()
    from hyqmom.runner import BatchSolver, Solver
    ps = members()
    ref = []
    for p in ps:
        s = Solver(p)
        try:
            s.set_state(ic.initial_state(p))
            s.advance(12)
            ref.append((s.get_state(), s.stats()))
        finally:
            s.close()
    b = BatchSolver(ps)
    try:
        for m, p in zip(b.members, ps):
            m.set_state(ic.initial_state(p))
        b.advance(3)                  # three one-step replays
        ndone, nfailed = b.advance(9)  # one eight-step replay and one one-step replay
        assert nfailed == 0
        for m, (Mref, sref) in zip(b.members, ref):
            st = m.stats()
            assert st["nn"] == sref["nn"] and st["t"] == sref["t"]
            assert field_rel(m.get_state(), Mref) < 1e-12
        # members stop at their own limits: 6 and 4 steps, and tmax = 0.02
        assert [m.stats()["nn"] for m in b.members][:2] == [6, 4]
        assert ndone == sum(bool(m.stats()["done"]) for m in b.members)
    finally:
        b.close()
