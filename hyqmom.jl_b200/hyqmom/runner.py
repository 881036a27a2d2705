"""Host mirror of the reference's entry points over the CUDA step.

    simulation_runner(params)                      src/simulation_runner.jl:63-759
    run_simulation(; Nx, Ny, Nz, tmax, ...)        src/simulation_runner.jl:816-944
    run_simulation_with_snapshots(params; interval) src/simulation_runner.jl:994-1011

Same parameter names, same return tuples.  The IC is built on the host (as in
the reference), every time step runs on the GPU through libhyqmom_b200.so.
"""
import ctypes
import time

import numpy as np

from . import _lib
from . import ic as _ic
from .snapshots import SnapshotWriter


def params_struct(p, device=0, mode="plain"):
    """hyq_params of a reference-style parameter dict; mode: "plain" (the
    reference's eigenvalue path), "learned" or "certified"."""
    xmin, xmax, ymin, ymax, zmin, zmax = _ic.extents(p)
    return _lib.HyqParams(Nx=p["Nx"], Ny=p["Ny"], Nz=p["Nz"], flag2D=int(p["flag2D"]),
                          positivity=int(bool(p.get("positivity", True))), device=device, nnmax=int(p["nnmax"]),
                          tmax=float(p["tmax"]), Kn=float(p["Kn"]), Ma=float(p["Ma"]), CFL=float(p["CFL"]),
                          dtmax=float(p["dtmax"]), xmin=xmin, xmax=xmax, ymin=ymin, ymax=ymax, zmin=zmin, zmax=zmax,
                          mode=_lib.MODES[mode] if isinstance(mode, str) else int(mode),
                          symmetry_check_interval=int(p.get("symmetry_check_interval", 0) or 0))


class Solver:
    """One simulation domain on one GPU (a hyq_ctx).

    mode: "plain" (the reference's LAPACK-path eigen-solves), "learned" (the
    wave-speed network seeds a certified characteristic-polynomial solve;
    `net` is the network, a hyqmom.wavenet.WaveNet or None for the packaged
    one) or "certified" (the certified solve without the network)."""

    def __init__(self, params, device=0, _handle=None, mode="plain", net=None):
        lib = _lib.load()
        p = params
        self._owns = _handle is None
        self.mode = mode
        self.device = device
        if _handle is None:
            hp = params_struct(p, device, mode)
            h = ctypes.c_void_p()
            rc = lib.hyq_create(ctypes.byref(hp), ctypes.byref(h))
            if rc != 0:
                raise _lib.HyqError(f"{_lib.ERRORS.get(rc, rc)}: {lib.hyq_last_error(None).decode()}")
        else:
            h = ctypes.c_void_p(_handle)
        self._lib, self._h, self.params = lib, h, dict(p)
        self.shape = (p["Nx"], p["Ny"], p["Nz"], 35)
        if mode == "learned" and _handle is None:
            from . import wavenet
            self.set_wavespeed_net(net if net is not None else wavenet.load_default())

    def set_wavespeed_net(self, net):
        """Upload the wave-speed network (a hyqmom.wavenet.WaveNet)."""
        w = np.ascontiguousarray(net.params, dtype=np.float32)
        assert w.size == _lib.NET_PARAMS
        self._chk(self._lib.hyq_set_wavespeed_net(self._h, w.ctypes.data, float(net.margin)))

    def set_variant(self, kernel, variant):
        """Launch variant of a kernel ("hll"; hyq_set_variant): the same bits,
        another launch shape."""
        self._chk(self._lib.hyq_set_variant(self._h, _KERNELS[kernel], int(variant)))

    def close(self):
        if self._h:
            if self._owns:
                self._lib.hyq_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise _lib.HyqError(f"{_lib.ERRORS.get(rc, rc)}: {self._lib.hyq_last_error(self._h).decode()}")

    # state ----------------------------------------------------------------
    def set_state(self, M):
        M = np.asfortranarray(M, dtype=np.float64)
        assert M.shape == self.shape
        self._chk(self._lib.hyq_set_state(self._h, M.ctypes.data))

    def set_state_ic(self, params=None, tables=None):
        """Generate the initial condition of `params` (default: the solver's)
        on the device (hyq_set_state_ic); equal bit for bit to ic.initial_state.
        tables: ic.ic_tables output to use instead (a slab's layers)."""
        p = self.params if params is None else params
        xm, ym, zm, dx, dy, dz, bg, regions, moments = tables if tables is not None else _ic.ic_tables(p)
        n = len(regions)
        arr = (_lib.HyqIcRegion * max(n, 1))()
        for q, (kind, every, lo, hi, idx) in enumerate(regions):
            arr[q].kind, arr[q].everywhere = kind, every
            for a in range(3):
                arr[q].lo[a], arr[q].hi[a] = lo[a], hi[a]
            arr[q].i0, arr[q].i1, arr[q].j0, arr[q].j1, arr[q].k0, arr[q].k1 = idx
        xm, ym, zm = (np.ascontiguousarray(a, dtype=np.float64) for a in (xm, ym, zm))
        bg = np.ascontiguousarray(bg, dtype=np.float64)
        mom = np.ascontiguousarray(np.array(moments, dtype=np.float64).reshape(-1)) if n else np.zeros(1)
        self._chk(self._lib.hyq_set_state_ic(self._h, xm.ctypes.data, ym.ctypes.data, zm.ctypes.data, float(dx), float(dy), float(dz),
                                             bg.ctypes.data, n, ctypes.cast(arr, ctypes.c_void_p), mom.ctypes.data))

    def get_state(self):
        M = np.empty(self.shape, dtype=np.float64, order="F")
        self._chk(self._lib.hyq_get_state(self._h, M.ctypes.data))
        return M

    def set_state_device(self, ptr):
        self._chk(self._lib.hyq_set_state_device(self._h, ctypes.c_void_p(ptr)))

    def get_state_device(self, ptr):
        self._chk(self._lib.hyq_get_state_device(self._h, ctypes.c_void_p(ptr)))

    def get_SC(self):
        S = np.empty(self.shape, dtype=np.float64, order="F")
        C = np.empty(self.shape, dtype=np.float64, order="F")
        self._chk(self._lib.hyq_get_SC(self._h, S.ctypes.data, C.ctypes.data))
        return S, C

    def set_clock(self, t, nn):
        self._chk(self._lib.hyq_set_clock(self._h, float(t), int(nn)))

    # stepping --------------------------------------------------------------
    def advance(self, max_steps):
        t = ctypes.c_double()
        nn = ctypes.c_int64()
        done = ctypes.c_int32()
        self._chk(self._lib.hyq_advance(self._h, int(max_steps), ctypes.byref(t), ctypes.byref(nn), ctypes.byref(done)))
        return t.value, nn.value, bool(done.value)

    def advance_async(self, max_steps):
        self._chk(self._lib.hyq_advance_async(self._h, int(max_steps)))

    def step_host(self, M_in, M_out=None, nslabs=8):
        """One step on a host state (Fortran-ordered (Nx,Ny,Nz,35) float64),
        the copies overlapped with the per-cell phases; returns (t, nn, done).
        M_out defaults to M_in (updated in place)."""
        M_out = M_in if M_out is None else M_out
        for a in (M_in, M_out):
            assert a.shape == self.shape and a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
        t = ctypes.c_double()
        nn = ctypes.c_int64()
        done = ctypes.c_int32()
        self._chk(self._lib.hyq_step_host(self._h, M_in.ctypes.data, M_out.ctypes.data, int(nslabs), ctypes.byref(t),
                                          ctypes.byref(nn), ctypes.byref(done)))
        return t.value, nn.value, bool(done.value)

    def synchronize(self):
        self._chk(self._lib.hyq_synchronize(self._h))

    def stats(self):
        st = _lib.HyqStats()
        self._chk(self._lib.hyq_stats_get(self._h, ctypes.byref(st)))
        return dict(t=st.t, dt=st.dt, vmax=st.vmax, nn=st.nn, done=bool(st.done), status=st.status,
                    stage_cells=st.stage_cells, fallback_cells=st.fallback_cells, dense_mask=st.dense_mask,
                    vmax_first=tuple(st.vmax_first), worst_cell=st.worst_cell, worst_dir=st.worst_dir, maxdiff=st.maxdiff,
                    maxdiff_step=st.maxdiff_step)

    def reset_counters(self):
        self._chk(self._lib.hyq_reset_counters(self._h))

    @property
    def stream(self):
        return self._lib.hyq_stream(self._h)


_KERNELS = {"hll": _lib.KERNEL_HLL, "corr": _lib.KERNEL_CORR}


def variant_count(kernel):
    """Number of launch variants of a kernel ("hll", "corr")."""
    return int(_lib.load().hyq_variant_count(_KERNELS[kernel]))


class BatchSolver:
    """Independent domains stepped together (a hyq_batch): one CUDA graph
    replay advances every member that is not done by one step of its own dt.
    ``members[i]`` is a Solver view of member i (state, clock, stats)."""

    def __init__(self, params_list, device=0, mode="plain", net=None):
        lib = _lib.load()
        n = len(params_list)
        arr = (_lib.HyqParams * n)(*[params_struct(p, device, mode) for p in params_list])
        h = ctypes.c_void_p()
        rc = lib.hyq_batch_create(arr, n, ctypes.byref(h))
        if rc != 0:
            raise _lib.HyqError(f"{_lib.ERRORS.get(rc, rc)}: {lib.hyq_last_error(None).decode()}")
        self._lib, self._h = lib, h
        self.members = [Solver(p, device, _handle=lib.hyq_batch_member(h, i)) for i, p in enumerate(params_list)]
        if mode == "learned":
            from . import wavenet
            net = net if net is not None else wavenet.load_default()
            for m in self.members:
                m.set_wavespeed_net(net)

    def close(self):
        if self._h:
            for m in self.members:
                m.close()
            self._lib.hyq_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.members)

    def _chk(self, rc):
        if rc != 0:
            raise _lib.HyqError(f"{_lib.ERRORS.get(rc, rc)}: {self._lib.hyq_last_error(None).decode()}")

    def advance(self, max_steps):
        """Returns (members done, members stopped by a non-finite wave speed)."""
        nd, nf = ctypes.c_int32(), ctypes.c_int32()
        self._chk(self._lib.hyq_batch_advance(self._h, int(max_steps), ctypes.byref(nd), ctypes.byref(nf)))
        return nd.value, nf.value

    def advance_async(self, max_steps):
        self._chk(self._lib.hyq_batch_advance_async(self._h, int(max_steps)))

    @property
    def stream(self):
        return self._lib.hyq_batch_stream(self._h)

    @property
    def schedule(self):
        """"fused" (one launch per kernel for all members) or "branches"."""
        return "fused" if self._lib.hyq_batch_schedule(self._h) == _lib.BATCH_FUSED else "branches"

    def set_schedule(self, schedule):
        self._chk(self._lib.hyq_batch_set_schedule(self._h, _lib.BATCH_FUSED if schedule == "fused" else _lib.BATCH_BRANCHES))

    def set_variant(self, kernel, variant):
        """Launch variant of a kernel for every member ("hll" or "corr";
        hyq_batch_set_variant): the same bits, another launch shape."""
        self._chk(self._lib.hyq_batch_set_variant(self._h, _KERNELS[kernel], int(variant)))


def _runner_params(params):
    p = dict(params)
    p.setdefault("positivity", True)
    p.setdefault("nnmax", 20000000)
    return p


def print_first_step_diagnostics(p, st):
    """The reference's FIRST STEP DIAGNOSTICS block (src/simulation_runner.jl:404-470)
    from the device's first-step breakdown."""
    g = _ic.grid_spacing(p)
    dx, dy, dz = g["dx"], g["dy"], g["dz"]
    vmax = max(st["vmax_first"]) if not any(v != v for v in st["vmax_first"]) else float("nan")
    hmin = min(dx, dy, dz)
    print("\n  === FIRST STEP DIAGNOSTICS ===")
    print("  vmax breakdown:")
    for name, v in zip("xyz", st["vmax_first"]):
        print("    v%s_max = %.6e" % (name, v))
    print("    vmax (global) = %.6e" % vmax)
    print("  Grid spacing:\n    dx = %.6e, dy = %.6e, dz = %.6e\n    min(dx,dy,dz) = %.6e" % (dx, dy, dz, hmin))
    print("  Time step calculation:\n    CFL = %.6f\n    dtmax = %.6e\n    Kn = %.6e" % (p["CFL"], p["dtmax"], p["Kn"]))
    print("    CFL*min(dx,dy,dz)/vmax = %.6e" % (p["CFL"] * hmin / vmax))
    print("    dt (final) = %.6e" % min(p["CFL"] * hmin / vmax, min(p["dtmax"], p["Kn"])))
    if vmax > 100.0 or vmax != vmax:
        c = st["worst_cell"]
        i, j, k = c % p["Nx"], (c // p["Nx"]) % p["Ny"], c // (p["Nx"] * p["Ny"])
        print("  WARNING: vmax = %.6e (unusually large or invalid)" % vmax)
        print("  Worst cell: (%d,%d,%d) in %s-direction" % (i + 1, j + 1, k + 1, "xyz"[st["worst_dir"]]))
    print("  ==============================\n")


def simulation_runner(params, device=0, verbose=False, chunk=64):
    """Reference ``simulation_runner(params)`` for one rank.

    Returns ``(M_final, final_time, time_steps, grid)`` or, when
    ``params['snapshot_interval'] > 0``, ``(snapshot_filename, grid)``.
    """
    p = _runner_params(params)
    interval = int(p.get("snapshot_interval", 0) or 0)
    grid_out = _ic.grid(p)
    M0 = _ic.initial_state(p)
    solver = Solver(p, device=device)
    try:
        solver.set_state(M0)
        writer = None
        if interval > 0:
            # the reference's default name (src/simulation_runner.jl:283-289);
            # the writer stores it as .npz (see snapshots.py)
            fname = p.get("snapshot_filename") or "snapshots_Nx%d_Ny%d_Nz%d_Kn%.2f_Ma%.2f_tmax%.4f.jld2" % (
                p["Nx"], p["Ny"], p["Nz"], p["Kn"], p["Ma"], p["tmax"])
            writer = SnapshotWriter(fname, p, interval)
            S, C = solver.get_SC()
            writer.write(M0, 0.0, 0, S, C)
        t0 = time.time()
        done = False
        t, nn = 0.0, 0
        # verbose: one step at a time, printed as the reference prints them
        step_block = 1 if verbose else (interval if interval > 0 else chunk)
        sym = int(p.get("symmetry_check_interval", 0) or 0)
        while not done:
            t, nn, done = solver.advance(step_block)
            if verbose:
                st = solver.stats()
                if nn == 1:
                    print_first_step_diagnostics(p, st)
                line = "Step %4d: t = %.4f, dt = %.4e, wall = %.4f s" % (nn, t, st["dt"], time.time() - t0)
                if sym > 0 and st["maxdiff_step"] == nn:
                    line += ", MaxDiff = %.3e" % st["maxdiff"]
                print(line)
            if writer is not None and (nn % interval == 0 or done):
                S, C = solver.get_SC()
                writer.write(solver.get_state(), t, nn, S, C)
        if writer is not None:
            writer.close(grid_out)
            return writer.filename, grid_out
        return solver.get_state(), t, nn, grid_out
    finally:
        solver.close()


def run_simulation(Np=None, Nx=20, Ny=20, Nz=1, tmax=0.1, num_workers=1, verbose=True, Kn=1.0, Ma=0.0, flag2D=0, CFL=0.5,
                   homogeneous_z=True, debug_output=False, device=0, **_unused):
    """Reference ``run_simulation`` (src/simulation_runner.jl:816-944); returns the result dict."""
    if Np is not None:
        Nx = Ny = Np
    p = _ic.run_simulation_params(Nx=Nx, Ny=Ny, Nz=Nz, tmax=tmax, Kn=Kn, Ma=Ma, flag2D=flag2D, CFL=CFL,
                                  homogeneous_z=homogeneous_z, debug_output=debug_output)
    M, t, nn, g = simulation_runner(p, device=device, verbose=False)
    if verbose:
        print("Simulation complete! Final time: %s Time steps: %d" % (t, nn))
    return {"M": M, "final_time": t, "time_steps": nn, "xm": g["xm"], "ym": g["ym"], "zm": g["zm"], "Nx": Nx, "Ny": Ny,
            "Nz": Nz, "tmax": tmax}


def run_simulation_with_snapshots(params, snapshot_interval=2, device=0):
    """Reference ``run_simulation_with_snapshots`` (src/simulation_runner.jl:994-1011)."""
    p = dict(params)
    p["snapshot_interval"] = snapshot_interval
    result = simulation_runner(p, device=device)
    if snapshot_interval > 0:
        return result
    return None, result[3]
