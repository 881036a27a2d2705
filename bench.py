"""Throughput of the HyQMOM explicit step on B200: cell-steps/s.

A "step" is one time step of simulation_runner over the whole grid.  Default
workload: crossing jets 256 x 256 x 128 (8,388,608 cells, 2.35 GB of FP64
state), Ma=1, Kn=0.01, the run's own 500 steps from the initial condition.
CFL is 0.5, not the named 0.7: at 0.7 the x+y+z-2M update of this scheme
drives a jet-corner cell non-realizable and a flux Jacobian non-finite at
step 2 (observed in the CPU restatement of the reference and on the GPU,
which agree bit for bit; the reference's eigvals would throw there).

The run advances on the learned path (HYQ_MODE_LEARNED).  --steps K steps
spread evenly over the 500 (steps 500/K, 2*500/K, ..., 500) are timed, each
from the run's own state, on three paths from that same state: plain (the
reference's LAPACK-path eigen-solves), certified (the characteristic-
polynomial solve from bound starts) and learned (seeded by the wave-speed
network); the steps between them are untimed.  `value` is the learned path's
cell-steps/s.  The state exceeds L2 (126 MB), so no flush is needed between
timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c5|c2|c2s|c1|c4] [--impl reference]

Multi-GPU: independent replicas (one domain per rank, no data-path
collective); value = all ranks' cell-steps / max-over-ranks time.
--impl reference: the CPU restatement of the reference's step (the oracle,
OpenMP on all host cores) on bounded samples of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hyqmom.jl_b200"))

import numpy as np  # noqa: E402

METRIC = "cell-steps/s on 1 B200: plain eig vs learned warm-start, <=1e-8 rel vs FP64 ref"
UNIT = "cell-steps/s"
B_ALG = 2 * 35 * 8  # bytes per cell-step: state read once, written once

# The step's kernels in launch order (hyq_advance_timed slots); an eigenvalue
# stage slot holds its kernel and the passes over the cells it listed.
LAUNCHES_PER_STEP = {"plain": 24, "certified": 24, "learned": 25}
STAGE_KERNELS = {k: f"k_{p}_eig+k_{p}_fix+k_{p}_corr ({k[-1]})" for k, p in
                 (("A2_eig_x", "A"), ("A3_eig_y", "A"), ("A4_eig_z", "A"), ("E2_eig_x", "E"), ("E3_eig_y", "E"))}
KERNELS = ["A1_closure", "A2_eig_x", "A3_eig_y", "A4_eig_z", "A5_flux_speeds", "cfl", "hll",
           "E1_closure", "E2_eig_x", "E3_eig_y", "E4_closure_bgk"]
# DRAM bytes (read + write) per cell of each timed slot of the learned path
# (an eigenvalue stage: its kernel and passes; A1: the closure and the
# network), from ncu captures of steps 151-152 of crossing jets 128 x 128 x 64
# (Ma=1, Kn=0.01), scaled to a launch by its cells; the HLL slot per launch
# variant.
TRAFFIC_PER_CELL = {"A1_closure": 1356.1, "A2_eig_x": 831.4, "A3_eig_y": 853.4, "A4_eig_z": 1818.4, "A5_flux_speeds": 2845.4,
                    "E1_closure": 1055.0, "E2_eig_x": 663.4, "E3_eig_y": 652.5, "E4_closure_bgk": 1953.7}
TRAFFIC_HLL = {0: 1732.6, 1: 1540.5, 2: 1514.4, 3: 1540.1, 4: 1514.9, 5: 1739.5, 6: 1743.6, 7: 1715.1, 8: 1544.4, 9: 1506.7}
TRAFFIC_SOURCE = ("ncu dram__bytes_read+write per cell, learned path, steps 151-152 of crossing jets 128x128x64 (Ma=1, Kn=0.01), "
                  "scaled to this launch's cells")
MODES = ("plain", "certified", "learned")
E2E_SLABS = 6


RUN_STEPS = {"c5": 500, "c5s": 500, "c3": 200, "c2": 200, "c2s": 200, "c1": 100}


def workload(name="c5"):
    """Crossing jets (the reference's IC generator): c5 256x256x128 Ma=1
    Kn=0.01 (the headline, 500 steps); c5s the c5 case on 128x128x64
    (profiling captures); c3 160x160x80 Ma=1 Kn=0.1 (the learned path's
    evaluation case, 200 steps); c2 160x160x80 Ma=1 Kn=1 (200 steps);
    c2s the c2 case on 96x96x48 (profiling captures); c1 20^3 Ma=0 Kn=1.
    CFL 0.5 for c5/c2/c2s: at the named 0.7 the scheme turns a flux Jacobian
    non-finite within a few steps of this IC (the reference's eigvals throws
    there); c1 keeps 0.7."""
    from hyqmom import ic
    if name == "c5":
        p = ic.default_params(Nx=256, Ny=256, Nz=128, Ma=1.0, Kn=0.01, CFL=0.5, tmax=1e9, nnmax=1000000)
    elif name == "c5s":
        p = ic.default_params(Nx=128, Ny=128, Nz=64, Ma=1.0, Kn=0.01, CFL=0.5, tmax=1e9, nnmax=1000000)
    elif name == "c3":
        p = ic.default_params(Nx=160, Ny=160, Nz=80, Ma=1.0, Kn=0.1, CFL=0.5, tmax=1e9, nnmax=1000000)
    elif name == "c2":
        p = ic.default_params(Nx=160, Ny=160, Nz=80, Ma=1.0, Kn=1.0, CFL=0.5, tmax=1e9, nnmax=1000000)
    elif name == "c2s":
        p = ic.default_params(Nx=96, Ny=96, Nz=48, Ma=1.0, Kn=1.0, CFL=0.5, tmax=1e9, nnmax=1000000)
    elif name == "c1":
        p = ic.default_params(Nx=20, Ny=20, Nz=20, Ma=0.0, Kn=1.0, CFL=0.7, tmax=1e9, nnmax=1000000)
    else:
        raise ValueError(name)
    return ic.with_jets(p, "crossing")


def timed_steps(run_steps, k):
    """The k step numbers timed within a run of run_steps steps, evenly spread
    and ending at the last step (run_steps / k, 2 run_steps / k, ...)."""
    k = max(1, min(int(k), run_steps))
    return [int(round((q + 1) * run_steps / k)) for q in range(k)]


def sample_slab(p, nz=8):
    """A bounded sample of the workload: an nz-layer z-slab through the jets."""
    from hyqmom import ic
    M = ic.initial_state(p)
    z0 = p["Nz"] // 2 - nz // 2
    return np.asfortranarray(M[:, :, z0:z0 + nz, :])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self._stop = index, [], threading.Event()

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in self.rows for q in range(4) if len(r) > 3 + q and r[3 + q].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def fp64_peak_tflops(torch):
    """Measured FP64 FMA throughput of this GPU (dense double matmul: the
    non-tensor FP64 ceiling of B200 is the same DFMA pipe cuBLAS DGEMM uses)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def measured_hbm_gbs():
    """The measured HBM copy bandwidth of this pool's B200s, when recorded."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return None


def slab_of(M, nz):
    """An nz-layer z-slab through the middle (the jets) of a state."""
    z0 = M.shape[2] // 2 - nz // 2
    return np.array(M[:, :, z0:z0 + nz, :], order="F")


def cpu_baseline(p, slabs, what=None, threads=None):
    """The oracle (CPU restatement of the reference's step, OpenMP): one step
    on each of `slabs` [(step, state)], slabs of the run's states at
    spread-out steps (the same array listed again is stepped again).
    threads: OpenMP threads (default all host threads; 1 = serial)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    from hyqmom import ic
    lib = ol.load()
    lib.hyqo_set_threads(int(threads or os.cpu_count() or 1))
    cells = el = 0.0
    try:
        for _, M in slabs:
            q = dict(p, Nz=M.shape[2], **ic.grid_spacing(p))
            Mw = np.array(M, order="F")
            t0 = time.perf_counter()
            ol.step(Mw, q, 0.0)
            el += time.perf_counter() - t0
            cells += Mw.shape[0] * Mw.shape[1] * Mw.shape[2]
        cores = int(lib.hyqo_num_threads())
    finally:
        lib.hyqo_set_threads(int(os.cpu_count() or 1))
    M = slabs[0][1]
    return {"value": cells / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{what or 'one step of a z-slab through the jets of the run state at each of steps %s' % [k for k, _ in slabs]}"
                      f" ({M.shape[0]}x{M.shape[1]}x{M.shape[2]} cells, {int(cells)} cell-steps, {el:.1f} s), "
                      f"oracle C++ restatement, {'serial' if cores == 1 else 'OpenMP'}"}


def run_reference(args, rank, world):
    """The oracle on the host cores: each step one oracle step of a z-slab
    of the workload's initial condition (the reference arm has no GPU run to
    draw later states from; the IC's steps are the cheapest of the run, so
    this rate is optimistic for the CPU)."""
    if rank != 0:
        return
    p = workload(args.config)
    from hyqmom import ic
    M0 = ic.initial_state(p)
    n = max(1, min(args.steps, 3))
    slab = slab_of(M0, 8)
    base = cpu_baseline(p, [(k, slab) for k in range(n)], f"steps 1-{n} of a z-slab through the jets of the initial condition")
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference crossing-jets IC generator)",
            "config": {"workload": f"crossing jets {p['Nx']}x{p['Ny']}x{p['Nz']} Ma={p['Ma']} Kn={p['Kn']} CFL={p['CFL']}",
                       "sample": base["sample"]},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Julia CPU path unavailable (no julia in the image); timed: the oracle restatement on IC slabs"}
    print(json.dumps(line), flush=True)


def max_over_ranks(ms, dist=None, device="cpu"):
    """The slowest rank's time (every rank gets it); ms itself with one rank."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, cells, steps, ms):
    """Whole-job cell-steps/s of `world` replicas that each advanced `cells`
    cells by `steps` steps in `ms` (the max over ranks)."""
    return world * cells * steps / (ms * 1e-3)


def run_gpu(args, rank, world, local_rank):
    import ctypes
    import torch
    torch.cuda.set_device(local_rank)
    from hyqmom import ic
    from hyqmom.runner import Solver
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    p = workload(args.config)
    cells = p["Nx"] * p["Ny"] * p["Nz"]
    run_steps = RUN_STEPS[args.config]
    marks = timed_steps(run_steps, args.steps)
    shape = (p["Nx"], p["Ny"], p["Nz"], 35)
    sol = {m: Solver(p, device=local_rank, mode=m) for m in MODES}
    traj = sol["learned"]
    streams = {m: torch.cuda.ExternalStream(sol[m].stream) for m in MODES}
    buf = torch.empty(35 * cells, dtype=torch.float64, device="cuda")  # the state before a timed step
    Mh_flat = torch.empty(35 * cells, dtype=torch.float64).pin_memory()
    Mh = Mh_flat.numpy().reshape(shape, order="F")
    Mh_out_flat = torch.empty(35 * cells, dtype=torch.float64).pin_memory()
    Mh_out = Mh_out_flat.numpy().reshape(shape, order="F")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def restore(s, t, nn):
        s.set_state_device(buf.data_ptr())
        s.set_clock(t, nn)
        s.synchronize()

    def time_graph_step(m):
        st = streams[m]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        sol[m].advance_async(1)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1)

    # the initial condition generated on the device (the reference's region fill)
    traj.set_state_ic()
    # warm-up: the first W steps of the run (untimed), every path once
    for m in MODES:
        if m != "learned":
            sol[m].set_state_ic()
            sol[m].advance(1)
    traj.advance(max(1, min(args.warmup, marks[0] - 1)))
    # the HLL sweep's launch shape, timed on this workload (same bits in every
    # shape) and used by all three paths
    from hyqmom import autotune
    tune = autotune.tune_solver(sol["plain"], use_cache=False)
    for m in MODES:
        sol[m].set_variant("hll", tune["hll"])
    ms = {m: [] for m in MODES}
    kern = {m: np.zeros(len(KERNELS)) for m in MODES}
    e2e_s = 0.0
    slabs = []
    fb = {"certified": [0, 0], "learned": [0, 0]}
    barrier()
    sampler = ClockSampler(local_rank)
    with sampler:
        for q, step in enumerate(marks):
            st = traj.stats()
            if st["nn"] < step - 1:
                traj.advance(step - 1 - st["nn"])
            st = traj.stats()
            assert st["status"] == 0 and st["nn"] == step - 1, f"run stopped early: {st}"
            t, nn = st["t"], st["nn"]
            traj.get_state_device(buf.data_ptr())
            traj.synchronize()
            # the step on every path from the same state (CUDA events on each
            # context's stream, graph replay)
            for m in ("plain", "certified"):
                restore(sol[m], t, nn)
                sol[m].reset_counters()
                ms[m].append(time_graph_step(m))
                if m in fb:
                    sm = sol[m].stats()
                    fb[m][0] += sm["fallback_cells"]
                    fb[m][1] += sm["stage_cells"]
            # per-kernel device times of the same step (individual launches)
            for m in MODES:
                restore(sol[m], t, nn)
                kms = (ctypes.c_float * len(KERNELS))()
                sol[m]._chk(sol[m]._lib.hyq_advance_timed(sol[m]._h, 1, kms))
                kern[m] += np.array(kms[:])
            # the run itself: the learned step (graph replay) ...
            restore(traj, t, nn)
            traj.reset_counters()
            ms["learned"].append(time_graph_step("learned"))
            sm = traj.stats()
            fb["learned"][0] += sm["fallback_cells"]
            fb["learned"][1] += sm["stage_cells"]
            # ... and end to end through the public API from a pinned host
            # state: upload, step, download (hyq_step_host); the device state
            # is again the step's result, from which the run continues
            Mh_flat.copy_(buf)
            if q % max(1, len(marks) // 4) == 0:
                slabs.append((step - 1, slab_of(Mh, 2)))
            restore(traj, t, nn)
            t0 = time.perf_counter()
            traj.step_host(Mh, Mh_out, nslabs=E2E_SLABS)
            e2e_s += time.perf_counter() - t0
    barrier()
    st = traj.stats()
    assert st["status"] == 0 and st["nn"] == marks[-1], f"run stopped early: {st}"
    k = len(marks)
    tot = {m: max_over_ranks(float(np.sum(ms[m])), dist, "cuda") for m in MODES}
    value = {m: replica_throughput(world, cells, k, tot[m]) for m in MODES}
    e2e = {"value": world * cells * k / e2e_s, "unit": UNIT, "h2d_bytes_per_step": Mh_flat.numel() * 8,
           "d2h_bytes_per_step": Mh_flat.numel() * 8, "api": f"hyq_step_host (learned path), {E2E_SLABS} slabs, pinned host state"}
    for s_ in sol.values():
        s_.close()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    fp64 = fp64_peak_tflops(torch)
    # algorithmic FP64 operations of the plain path on the timed steps'
    # states (oracle op counter on 2-layer z-slabs through the jets)
    F_alg, F_kernel = count_ops_on(p, slabs)
    per_kernel = {m: {KERNELS[i]: round(float(kern[m][i] / k), 3) for i in range(len(KERNELS))} for m in MODES}
    lk = {KERNELS[i]: kern["learned"][i] / k for i in range(len(KERNELS))}
    dom = max((x for x in KERNELS if x not in ("cfl", "hll")), key=lambda x: lk[x])
    ach = F_kernel[dom] * cells / (lk[dom] * 1e-3) / 1e12
    step_ms = tot["learned"] / k
    step_tflops = F_alg * cells / (step_ms * 1e-3) / 1e12
    per_cell = TRAFFIC_HLL.get(tune["hll"]) if dom == "hll" else TRAFFIC_PER_CELL.get(dom)
    traffic = per_cell * cells if per_cell else None
    roof = {"bound": "fp64", "achieved": ach, "peak": fp64, "unit": "TFLOP/s", "frac": ach / fp64, "traffic": traffic,
            "traffic_source": TRAFFIC_SOURCE if traffic else None,
            "peak_source": "measured in this run: FP64 DGEMM 8192^3 (cuBLAS via torch), best of 3",
            "dominant_kernel": STAGE_KERNELS.get(dom, "k_" + dom) + ", learned path", "f_alg_per_cell": F_kernel[dom],
            "note": ("achieved = the plain path's FP64 op count of this kernel (oracle counter on the timed steps' states) x cells / "
                     "the learned path's mean launch time; built with -fmad=false, so an FMA-free kernel tops out at peak/2"),
            "step": {"f_alg_per_cell": F_alg, "achieved": step_tflops, "frac": step_tflops / fp64,
                     "hbm_achieved_gbs": B_ALG * cells / (step_ms * 1e-3) / 1e9}}
    hbm_peak = measured_hbm_gbs()
    if hbm_peak:
        roof["step"]["hbm_peak_gbs"] = hbm_peak
        roof["step"]["hbm_frac"] = roof["step"]["hbm_achieved_gbs"] / hbm_peak
        roof["step"]["hbm_peak_source"] = "MEASURED_PEAKS.json (copy bandwidth)"
    modes = {m: {"value": value[m], "ms_per_step": tot[m] / k, "kernels_ms": per_kernel[m],
                 "launches_per_step": LAUNCHES_PER_STEP[m]} for m in MODES}
    for m in fb:
        modes[m]["fallback_rate"] = fb[m][0] / max(1, fb[m][1])
        modes[m]["fallback_cells"], modes[m]["stage_cells"] = fb[m]
    modes["learned"]["over_plain"] = value["learned"] / value["plain"]
    modes["learned"]["over_certified"] = value["learned"] / value["certified"]
    line = {"metric": METRIC, "value": value["learned"], "unit": UNIT, "n_gpus": world, "steps": k, "warmup": args.warmup,
            "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference crossing-jets IC generator)",
            "config": {"workload": f"crossing jets {p['Nx']}x{p['Ny']}x{p['Nz']} Ma={p['Ma']} Kn={p['Kn']} CFL={p['CFL']}, "
                                   f"{run_steps}-step run, learned wave-speed path",
                       "cells": cells, "parallelism": f"replicas x{world}", "run_steps": run_steps, "timed_steps": marks,
                       "timing": "each timed step from the run's own state; plain and certified paths timed from the same state",
                       "l2": f"state {cells * 35 * 8 / 1e6:.0f} MB > L2 (126 MB), no flush needed", "steps_done": st["nn"],
                       "autotune": {"hll_variant": tune["hll"], "hll_ms": tune["ms"]}},
            "modes": modes,
            "gpu_launches": LAUNCHES_PER_STEP["learned"] * k, "e2e": e2e, "roofline": roof, "clocks": sampler.summary()}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p, slabs)
        line["cpu_baseline_serial"] = cpu_baseline(p, slabs[:1], threads=1)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def count_ops_on(p, slabs):
    """(F_alg, per-kernel F): the oracle's FP64 op counter (plain path) on
    the slabs, averaged per cell."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    from hyqmom import ic
    names = [k for k in KERNELS if k not in ("cfl", "hll")]
    tot, stages, n = 0.0, np.zeros(len(names)), 0
    hll = 0.0
    for _, M in slabs:
        q = dict(p, Nz=M.shape[2], **ic.grid_spacing(p))
        c = M.shape[0] * M.shape[1] * M.shape[2]
        out = ol.count_ops(np.array(M, order="F"), q, 1e-3) / np.array([c, c, 1.0])
        st = ol.count_ops_stages(np.array(M, order="F"), q, 1e-3)[:len(names)] / c
        tot += float(out.sum())
        hll += float(out[2])
        stages += st
        n += 1
    F = {k: float(v / n) for k, v in zip(names, stages)}
    F["cfl"] = 1.0
    F["hll"] = hll / n
    return tot / n, F


def run_slabs(args, rank, world, local_rank):
    """One domain split into z-slabs over the ranks (hyqmom.slabs; ghost
    exchange and the dt all-reduce over NCCL): the workload's steps W+1 ..
    W+K on the learned path, strong scaling (the whole grid over N GPUs)."""
    import torch
    import torch.distributed as dist
    from hyqmom import slabs
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    p = workload(args.config)
    cells = p["Nx"] * p["Ny"] * p["Nz"]
    eng = slabs.GpuSlab(p, world, rank, device=local_rank, mode="learned")
    eng.set_initial_condition()
    d = dist if world > 1 else None

    def buf(shape):
        return torch.zeros(shape, dtype=torch.float64, device="cuda")

    for _ in range(args.warmup):
        slabs.step(eng, rank, world, eng.layout, d, buf)
    torch.cuda.synchronize()
    if d is not None:
        d.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        slabs.step(eng, rank, world, eng.layout, d, buf)
    e1.record()
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), d, "cuda")
    st = eng.stats()
    eng.close()
    if rank == 0:
        line = {"metric": METRIC, "value": cells * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference crossing-jets IC generator)",
                "config": {"workload": f"crossing jets {p['Nx']}x{p['Ny']}x{p['Nz']} Ma={p['Ma']} Kn={p['Kn']} CFL={p['CFL']}, "
                                       f"learned wave-speed path, z-slabs over {world} GPUs",
                           "cells": cells, "parallelism": f"z-slabs x{world}", "timed_steps": f"{args.warmup + 1}-{args.warmup + args.steps}",
                           "steps_done": st["nn"]},
                "gpu_launches": (LAUNCHES_PER_STEP["learned"] + 4) * args.steps}
        print(json.dumps(line), flush=True)
    if d is not None:
        d.destroy_process_group()


def batch_workload(n=64, seed=0, CFL=0.5):
    """Sweep of independent domains: grids uniform from 16^3 to 96x96x48,
    Ma ~ U[0, 2], Kn log-uniform in [1e-3, 1], crossing and triple-jet ICs
    alternating, 100 steps each, seed-fixed.  CFL 0.5 as for the single-domain
    workload."""
    from hyqmom import ic
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        Nx, Ny = (int(v) for v in rng.integers(16, 97, size=2))
        Nz = int(rng.integers(16, 49))
        Ma = float(rng.uniform(0.0, 2.0))
        Kn = float(10 ** rng.uniform(-3.0, 0.0))
        p = ic.default_params(Nx=Nx, Ny=Ny, Nz=Nz, Ma=Ma, Kn=Kn, CFL=CFL, tmax=1e9, nnmax=100)
        out.append(ic.with_jets(p, "crossing" if i % 2 == 0 else "triple-jet"))
    return out


def run_batch(args, rank, world, local_rank):
    """Batched sweep: every domain advanced together (one graph replay per
    step; the schedule and launch variants picked by the autotuner, which
    times them from the same states and keeps the choice per device) against
    the same domains advanced one at a time."""
    import torch
    torch.cuda.set_device(local_rank)
    from hyqmom import autotune
    from hyqmom.runner import BatchSolver
    ps = batch_workload()
    cells = [p["Nx"] * p["Ny"] * p["Nz"] for p in ps]
    mode = args.batch_mode
    b = BatchSolver(ps, device=local_rank, mode=mode)

    def reset():
        # every member's initial condition generated on the device
        for m in b.members:
            m.set_state_ic()

    def nn_all():
        return [m.stats()["nn"] for m in b.members]

    reset()
    b.advance(args.warmup)
    tune = autotune.tune_batch(b, ps, mode=mode, steps=1, use_cache=False, log=lambda m: print(m, file=sys.stderr, flush=True))
    n0 = nn_all()
    stream = torch.cuda.ExternalStream(b.stream)
    sampler = ClockSampler(local_rank)
    with sampler:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        b.advance_async(args.steps)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    n1 = nn_all()
    work = sum(c * (x1 - x0) for c, x0, x1 in zip(cells, n0, n1))
    failed = sum(1 for m in b.members if m.stats()["status"] > 0)
    value = work / (ms * 1e-3)

    # the same domains one at a time: each member's own step graph on its own
    # stream, members in sequence, device time summed
    reset()
    for m in b.members:
        m.advance(args.warmup)
    seq_ms = 0.0
    for m in b.members:
        st = torch.cuda.ExternalStream(m.stream)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(st)
        m.advance_async(args.steps)
        f1.record(st)
        f1.synchronize()
        seq_ms += f0.elapsed_time(f1)
    seq_value = work / (seq_ms * 1e-3)
    b.close()
    per_step = LAUNCHES_PER_STEP[mode] if tune["schedule"] == "fused" else LAUNCHES_PER_STEP[mode] * len(ps)
    if mode == "learned" and tune["schedule"] == "fused":
        per_step += len(ps) - 1  # the network runs once per member
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference crossing / triple-jet IC generator, seed 0)",
            "config": {"workload": f"batched sweep of {len(ps)} domains, 16^3..96x96x48, Ma U[0,2], Kn logU[1e-3,1], CFL 0.5, "
                                   f"{mode} eigenvalue path",
                       "cells_total": sum(cells), "domains_failed": failed, "one_at_a_time_value": seq_value,
                       "batched_over_one_at_a_time": value / seq_value, "l2": "state of all domains > L2",
                       "autotune": {"schedule": tune["schedule"], "hll_variant": tune["hll"], "corr_variant": tune["corr"],
                                    "trials_ms_per_step": tune["ms"]},
                       "timed_steps": f"{args.warmup + 1}-{args.warmup + args.steps} of each member (members stop at their own limits)"},
            "gpu_launches": per_step * args.steps, "clocks": sampler.summary()}
    print(json.dumps(line), flush=True)


def run_profile_case(args, local_rank):
    """A fixed sequence of launches for ncu captures (no timing): the
    workload on one path from its initial condition, `before` steps, then
    `after` more; or (hll) one step per HLL launch variant from the state
    after `before` steps, checking that every variant gives the same bits."""
    import torch
    from hyqmom import ic
    from hyqmom.runner import Solver, variant_count
    torch.cuda.set_device(local_rank)
    p = workload(args.config)
    mode, before, after = args.profile[0], int(args.profile[1]), int(args.profile[2])
    s = Solver(p, device=local_rank, mode="plain" if mode == "hll" else mode)
    s.set_state(ic.initial_state(p))
    s.advance(before)
    if mode != "hll":
        s.advance(after)
        print(json.dumps({"profile": mode, "config": args.config, "stats": s.stats()}), flush=True)
        s.close()
        return
    st = s.stats()
    buf = torch.empty(35 * p["Nx"] * p["Ny"] * p["Nz"], dtype=torch.float64, device="cuda")
    s.get_state_device(buf.data_ptr())
    s.synchronize()
    ref, same = None, []
    for v in range(variant_count("hll")):
        s.set_variant("hll", v)
        s.set_state_device(buf.data_ptr())
        s.set_clock(st["t"], st["nn"])
        s.synchronize()
        s.advance(1)
        M = s.get_state()
        ref = M if ref is None else ref
        same.append(bool(np.array_equal(M, ref)))
    s.close()
    print(json.dumps({"profile": "hll", "config": args.config, "variants_same_bits": same}), flush=True)
    if not all(same):
        raise SystemExit("HLL variants differ")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20, help="steps timed, spread evenly over the run")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c5", choices=["c1", "c2", "c2s", "c3", "c4", "c5", "c5s"])
    ap.add_argument("--profile", nargs=3, metavar=("MODE", "BEFORE", "AFTER"),
                    help="launch sequence for ncu captures: MODE plain|certified|learned|hll")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-mode", default="plain", choices=["plain", "certified", "learned"],
                    help="--config c4: the members' eigenvalue path")
    ap.add_argument("--decompose", default="replicas", choices=["replicas", "slabs"],
                    help="N > 1: independent replicas (default) or one domain split into z-slabs")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.profile:
        return run_profile_case(args, local_rank)
    if args.config == "c4":
        return run_batch(args, rank, world, local_rank)
    if args.decompose == "slabs":
        return run_slabs(args, rank, world, local_rank)
    run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
