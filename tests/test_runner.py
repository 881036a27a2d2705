"""The host mirror of the reference's entry points over the CUDA step
(src/simulation_runner.jl:63-757, :994-1011): return tuples, the
snapshot key layout and cadence, and the snapshots' standardized and central
fields (hyq_get_SC, compute_standardized_field / compute_central_field,
src/utils/compute_standardized_field.jl:16-66) against the oracle."""
import numpy as np
import pytest

import oracle_lib as ol
from hyqmom import ic

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def crossing(n=12, nnmax=9, tmax=10.0):
    return ic.with_jets(ic.default_params(Nx=n, Ny=n, Nz=n, Ma=1.0, Kn=1.0, CFL=0.5, tmax=tmax, nnmax=nnmax), "crossing")


def test_simulation_runner_returns_reference_tuple():
    need_gpu()
    from hyqmom.runner import simulation_runner
    p = crossing()
    M, t, nn, grid = simulation_runner(p)
    assert M.shape == (12, 12, 12, 35) and nn == 9
    Mo = np.asfortranarray(ic.initial_state(p))
    pp = dict(p, **ic.grid_spacing(p))
    to = 0.0
    for _ in range(9):
        _, to, _ = ol.step(Mo, pp, to)
    assert np.array_equal(M, Mo) and t == to
    assert set(grid) >= {"x", "y", "z", "dx", "dy", "dz", "xm", "ym", "zm"}
    assert len(grid["x"]) == 13 and len(grid["xm"]) == 12


def test_snapshots_layout_and_cadence(tmp_path):
    """Snapshot 1 is the IC; then every `interval` steps and at the end
    (nn % interval == 0 || done), each with M, t, step, S and C."""
    need_gpu()
    from hyqmom.runner import run_simulation_with_snapshots
    p = crossing(nnmax=7)
    p["snapshot_filename"] = str(tmp_path / "snaps.jld2")
    fname, grid = run_simulation_with_snapshots(p, snapshot_interval=3)
    assert fname.endswith(".npz")
    z = np.load(fname)
    n = int(z["meta/n_snapshots"])
    steps = [int(z["snapshots/%06d/step" % k]) for k in range(1, n + 1)]
    assert steps == [0, 3, 6, 7]
    assert int(z["meta/snapshot_interval"]) == 3
    for k in range(1, n + 1):
        for f in ("M", "S", "C"):
            assert z["snapshots/%06d/%s" % (k, f)].shape == (12, 12, 12, 35)
    assert np.array_equal(z["snapshots/000001/M"], ic.initial_state(p))
    assert float(z["snapshots/000001/t"]) == 0.0
    assert np.array_equal(z["grid/xm"], grid["xm"])


def test_get_SC_matches_oracle():
    need_gpu()
    from hyqmom.runner import Solver
    p = crossing()
    s = Solver(p)
    try:
        s.set_state(ic.initial_state(p))
        s.advance(5)
        M = s.get_state()
        S, C = s.get_SC()
    finally:
        s.close()
    cells = M.reshape(-1, 35, order="F")
    Sg, Cg = S.reshape(-1, 35, order="F"), C.reshape(-1, 35, order="F")
    for c in range(0, cells.shape[0], 7):
        Co, So = ol.m2cs4_35(cells[c])
        assert np.array_equal(Cg[c], Co) and np.array_equal(Sg[c], So), c
