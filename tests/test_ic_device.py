"""The initial condition generated on the device (hyq_set_state_ic) against
the host builder ic.initial_state (which the reference's Nz=1 goldens pin):
the tables reproduce it on the host, and the device fill reproduces it bit
for bit (src/initial_conditions.jl:152-217, :281-302;
src/simulation_runner.jl:200-271)."""
import numpy as np
import pytest

from hyqmom import ic


def cases():
    return [ic.with_jets(ic.default_params(Nx=10, Ny=12, Nz=8, Ma=1.0), "crossing"),
            ic.with_jets(ic.default_params(Nx=9, Ny=7, Nz=5, Ma=2.0, r110=0.3, r011=-0.2), "triple-jet"),
            ic.with_jets(ic.default_params(Nx=16, Ny=16, Nz=1, Ma=0.5), "crossing2D"),
            ic.default_params(Nx=10, Ny=12, Nz=8, Ma=1.0),
            ic.run_simulation_params(Nx=20, Ny=20, Nz=1, Ma=1.0)]


def emulate(p):
    """The device kernel's per-cell rule on the host."""
    xm, ym, zm, dx, dy, dz, bg, regs, moms = ic.ic_tables(p)
    M = np.empty((p["Nx"], p["Ny"], p["Nz"], 35), order="F")
    for i in range(p["Nx"]):
        for j in range(p["Ny"]):
            for k in range(p["Nz"]):
                use = -1
                for r, (kind, every, lo, hi, idx) in enumerate(regs):
                    if kind == 1:
                        inn = idx[0] <= i <= idx[1] and idx[2] <= j <= idx[3] and idx[4] <= k <= idx[5]
                    elif every:
                        inn = True
                    else:
                        inn = all(max(x - d / 2.0, lo[q]) < min(x + d / 2.0, hi[q])
                                  for q, (x, d) in enumerate(((xm[i], dx), (ym[j], dy), (zm[k], dz))))
                    if inn:
                        use = r
                M[i, j, k] = bg if use < 0 else moms[use]
    return M


@pytest.mark.parametrize("q", range(5))
def test_tables_reproduce_host_ic(q):
    p = cases()[q]
    assert np.array_equal(emulate(p), ic.initial_state(p))


@pytest.mark.gpu
@pytest.mark.parametrize("q", range(5))
def test_device_ic_matches_host_ic(q):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hyqmom.runner import Solver
    p = dict(cases()[q], tmax=1.0, nnmax=10)
    s = Solver(p)
    try:
        s.set_state_ic()
        M = s.get_state()
        st = s.stats()
    finally:
        s.close()
    assert np.array_equal(M, ic.initial_state(p))
    assert st["nn"] == 0 and st["t"] == 0.0
