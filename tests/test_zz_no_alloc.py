"""hyq_step_noalloc: the allocation-free step on a caller-owned device state,
called through the C-ABI, against the context path (hyq_create/hyq_advance)
for three calls in a row; and its cell-count limit.

Both paths run the same kernels in the same order, so the states must agree
bit for bit (the tolerance of the step's parity tests, 1e-12 relative, is
implied).  The context path keeps its eigenvalue stages' dense-mode counters
across steps while each allocation-free call starts them from zero; the
dense and listed code paths give identical bits, which three calls cover."""
import ctypes
import os

import numpy as np
import pytest

from hyqmom import _lib, ic

torch = pytest.importorskip("torch")


def params_struct(p, device=0):
    xmin, xmax, ymin, ymax, zmin, zmax = ic.extents(p)
    return _lib.HyqParams(Nx=p["Nx"], Ny=p["Ny"], Nz=p["Nz"], flag2D=int(p["flag2D"]),
                          positivity=int(bool(p.get("positivity", True))), device=device, nnmax=int(p["nnmax"]),
                          tmax=float(p["tmax"]), Kn=float(p["Kn"]), Ma=float(p["Ma"]), CFL=float(p["CFL"]),
                          dtmax=float(p["dtmax"]), xmin=xmin, xmax=xmax, ymin=ymin, ymax=ymax, zmin=zmin, zmax=zmax)


def field_rel(a, b):
    a = np.asarray(a).reshape(-1, 35)
    b = np.asarray(b).reshape(-1, 35)
    scale = np.maximum(np.max(np.abs(b), axis=0), 1e-300)
    return float(np.max(np.max(np.abs(a - b), axis=0) / scale))


def crossing(Nx, Ny, Nz):
    return ic.with_jets(ic.default_params(Nx=Nx, Ny=Ny, Nz=Nz, Ma=1.0, Kn=1.0, CFL=0.5, tmax=10.0, nnmax=100), "crossing")


@pytest.mark.gpu
def test_noalloc_step_matches_context_step():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hyqmom.runner import Solver
    lib = _lib.load()
    p = crossing(20, 18, 16)  # 5,760 cells
    M0 = ic.initial_state(p)

    s = Solver(p)
    ref = []
    try:
        s.set_state(M0)
        for _ in range(3):
            s.advance(1)
            ref.append((s.get_state(), s.stats()))
    finally:
        s.close()

    hp = params_struct(p)
    dM = torch.tensor(np.ravel(M0, order="F"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = _lib.HyqStats()
    st.t, st.nn = 0.0, 0
    free = []
    for k in range(3):
        rc = lib.hyq_step_noalloc(ctypes.byref(hp), ctypes.c_void_p(dM.data_ptr()), ctypes.byref(st), None)
        assert rc == 0, lib.hyq_last_error(None).decode()
        free.append(torch.cuda.mem_get_info()[0])
        got = dM.cpu().numpy().reshape(p["Nx"], p["Ny"], p["Nz"], 35, order="F")
        Mref, sref = ref[k]
        assert st.nn == sref["nn"] == k + 1 and st.status == 0 and not st.done
        assert st.t == sref["t"] and st.dt == sref["dt"] and st.vmax == sref["vmax"]
        assert np.array_equal(got, Mref), field_rel(got, Mref)
    # the later calls find the scratch set up and allocate nothing
    assert free[2] == free[1] == free[0]


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="library not built")
def test_noalloc_rejects_grids_above_the_limit():
    """Checked on the host before any CUDA call, so this runs without a GPU."""
    lib = _lib.load()
    p = crossing(128, 128, 2)  # 32,768 cells > HYQ_NOALLOC_MAX_CELLS
    assert p["Nx"] * p["Ny"] * p["Nz"] > _lib.NOALLOC_MAX_CELLS
    st = _lib.HyqStats()
    rc = lib.hyq_step_noalloc(ctypes.byref(params_struct(p)), ctypes.c_void_p(16), ctypes.byref(st), None)
    assert rc == -1
    msg = lib.hyq_last_error(None).decode()
    assert "at most %d" % _lib.NOALLOC_MAX_CELLS in msg
