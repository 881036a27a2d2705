"""Launch-shape autotuner for the step's kernels, kept per device.

Some kernels of the step have several launch shapes (hyq_variant_count):
the HLL sweep's cells per block and moment groups, the fused batch's
correction-pass blocks per member, and the batch schedule itself (fused
member-table launches or the members' graphs as branches).  Every choice
gives the same bits, so the tuner only times them: on the caller's own
workload, from the same state, with CUDA events on the stream the work runs
on.  The state and clock are put back after each trial, so tuning leaves the
run where it was.

Choices are kept in a JSON file (HYQMOM_TUNE_CACHE, default
~/.cache/hyqmom/tune.json) under the device (name, SM count, compute
capability, library ABI) and a workload key (grid sizes and path), and read
back instead of timing again.
"""
import json
import os

from . import _lib

CACHE_ENV = "HYQMOM_TUNE_CACHE"
HLL_SLOT = 6  # hyq_advance_timed slot of the HLL sweep


def cache_path():
    return os.environ.get(CACHE_ENV) or os.path.join(os.path.expanduser("~"), ".cache", "hyqmom", "tune.json")


def device_key(device=0):
    import torch
    pr = torch.cuda.get_device_properties(device)
    return f"{pr.name}|sm{pr.multi_processor_count}|cc{pr.major}.{pr.minor}|abi{_lib.load().hyq_abi_version()}"


def load_cache(path=None):
    path = path or cache_path()
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(data, path=None):
    path = path or cache_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _lookup(dev, key, path):
    return load_cache(path).get(dev, {}).get(key)


def _store(dev, key, choice, path):
    data = load_cache(path)
    data.setdefault(dev, {})[key] = choice
    save_cache(data, path)


def solver_key(p, mode):
    return f"solver|{p['Nx']}x{p['Ny']}x{p['Nz']}|{mode}"


def batch_key(params_list, mode):
    grids = ",".join(f"{p['Nx']}x{p['Ny']}x{p['Nz']}" for p in params_list)
    import hashlib
    return f"batch|{len(params_list)}|{mode}|{hashlib.sha1(grids.encode()).hexdigest()[:16]}"


class _Snapshot:
    """A solver's device state and clock, to put back after each trial."""

    def __init__(self, solver):
        import torch
        st = solver.stats()
        self.solver, self.t, self.nn = solver, st["t"], st["nn"]
        n = 35 * solver.shape[0] * solver.shape[1] * solver.shape[2]
        self.buf = torch.empty(n, dtype=torch.float64, device=f"cuda:{solver.device}")
        solver.get_state_device(self.buf.data_ptr())
        solver.synchronize()

    def restore(self):
        self.solver.set_state_device(self.buf.data_ptr())
        self.solver.set_clock(self.t, self.nn)
        self.solver.synchronize()


def tune_solver(solver, mode="plain", steps=1, reps=2, path=None, use_cache=True, log=None):
    """Pick the HLL sweep's launch variant for one context: the variant with
    the least HLL time over `reps` x `steps` steps from the current state
    (hyq_advance_timed).  Returns {"hll": variant, "ms": {variant: ms}}."""
    import ctypes
    dev = device_key(solver.device)
    key = solver_key(solver.params, mode)
    if use_cache:
        hit = _lookup(dev, key, path)
        if hit is not None:
            solver.set_variant("hll", hit["hll"])
            return dict(hit, cached=True)
    snap = _Snapshot(solver)
    nvar = int(solver._lib.hyq_variant_count(_lib.KERNEL_HLL))
    times = {}
    for v in range(nvar):
        solver.set_variant("hll", v)
        best = float("inf")
        for _ in range(reps):
            snap.restore()
            ms = (ctypes.c_float * 11)()
            solver._chk(solver._lib.hyq_advance_timed(solver._h, int(steps), ms))
            best = min(best, ms[HLL_SLOT] / steps)
        times[v] = best
        if log:
            log(f"hll variant {v}: {best:.3f} ms")
    snap.restore()
    choice = min(times, key=times.get)
    solver.set_variant("hll", choice)
    out = {"hll": choice, "ms": {str(k): v for k, v in times.items()}}
    _store(dev, key, out, path)
    return dict(out, cached=False)


def _time_batch(batch, snaps, steps):
    import torch
    for s in snaps:
        s.restore()
    stream = torch.cuda.ExternalStream(batch.stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.advance_async(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def tune_batch(batch, params_list, mode="plain", steps=1, path=None, use_cache=True, log=None):
    """Pick the batch schedule, the HLL variant and (fused) the correction
    passes' blocks per member by coordinate search: each candidate times
    `steps` replays from the same states of all members.  Returns the choice
    {"schedule", "hll", "corr", "ms": {...}}."""
    import torch
    dev = device_key(batch.members[0].device)
    key = batch_key(params_list, mode)
    if use_cache:
        hit = _lookup(dev, key, path)
        if hit is not None:
            apply_batch(batch, hit)
            return dict(hit, cached=True)
    snaps = [_Snapshot(m) for m in batch.members]
    torch.cuda.synchronize()
    trials = {}

    def trial(schedule, hll, corr):
        batch.set_schedule(schedule)
        batch.set_variant("hll", hll)
        if schedule == "fused":
            batch.set_variant("corr", corr)
        ms = _time_batch(batch, snaps, steps)
        trials[f"{schedule}/hll{hll}/corr{corr}"] = ms
        if log:
            log(f"{schedule} hll {hll} corr {corr}: {ms:.3f} ms/step")
        return ms

    best = {"schedule": "fused", "hll": 0, "corr": 0}
    scheds = ["fused", "branches"]
    try:
        batch.set_schedule("fused")
    except _lib.HyqError:
        scheds = ["branches"]
        best["schedule"] = "branches"
    if len(scheds) > 1:
        t = {s: trial(s, 0, 0) for s in scheds}
        best["schedule"] = min(t, key=t.get)
    nh = int(batch._lib.hyq_variant_count(_lib.KERNEL_HLL))
    t = {v: trial(best["schedule"], v, 0) for v in range(nh)}
    best["hll"] = min(t, key=t.get)
    if best["schedule"] == "fused":
        nc = int(batch._lib.hyq_variant_count(_lib.KERNEL_CORR))
        t = {v: trial("fused", best["hll"], v) for v in range(nc)}
        best["corr"] = min(t, key=t.get)
    for s in snaps:
        s.restore()
    apply_batch(batch, best)
    out = dict(best, ms=trials)
    _store(dev, key, out, path)
    return dict(out, cached=False)


def apply_batch(batch, choice):
    batch.set_schedule(choice["schedule"])
    batch.set_variant("hll", int(choice["hll"]))
    if choice["schedule"] == "fused":
        batch.set_variant("corr", int(choice["corr"]))
