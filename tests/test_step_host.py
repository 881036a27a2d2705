"""hyq_step_host (one step on a host state with the copies overlapped with
the per-cell phases, slab by slab) gives the same state as hyq_advance."""
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


def case():
    return ic.with_jets(ic.default_params(Nx=24, Ny=20, Nz=16, Ma=1.0, Kn=1.0, CFL=0.5, tmax=10.0, nnmax=100), "crossing")


@pytest.mark.parametrize("nslabs,pinned,inplace", [(5, True, True), (1, False, False), (10_000, True, False)])
def test_step_host_matches_advance(nslabs, pinned, inplace):
    cuda()
    from hyqmom.runner import Solver
    p = case()
    M0 = ic.initial_state(p)
    shape = M0.shape
    a = Solver(p)
    try:
        a.set_state(M0)
        a.advance(3)
        Mref, sref = a.get_state(), a.stats()
    finally:
        a.close()
    if pinned:
        buf = torch.empty(M0.size, dtype=torch.float64).pin_memory().numpy()
        Min = buf.reshape(shape, order="F")
    else:
        Min = np.empty(shape, dtype=np.float64, order="F")
    Min[...] = M0
    Mout = Min if inplace else np.empty(shape, dtype=np.float64, order="F")
    b = Solver(p)
    try:
        b.set_state(M0)
        for k in range(3):
            t, nn, done = b.step_host(Min, Mout, nslabs=nslabs)
            if not inplace:
                Min[...] = Mout
        assert nn == sref["nn"] == 3 and t == sref["t"] and not done
        assert np.array_equal(Mout, Mref)
        assert np.array_equal(b.get_state(), Mref)   # the device state is left equal to M_out
    finally:
        b.close()
