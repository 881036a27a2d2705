"""Throughput of the HyQMOM explicit step on B200: cell-steps/s.

A "step" is one time step of simulation_runner over the whole grid.  Default
workload: crossing jets 160 x 160 x 80 (2,048,000 cells, 573 MB of FP64
state), Ma=1, Kn=1, plain eigen-solve, 200 steps from the initial condition
(the timed steps always start from the IC: a step's cost grows ~7x over the
run as the flow develops, so a window of early steps would not represent
it).  The state (573 MB) and the flux buffers exceed L2 (126 MB), so no L2
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--from-step S] [--impl reference]

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

# FP64 operations per cell-step of the plain path (oracle op counter, +,-,*,/
# and sqrt/cbrt/exp counted 1 each), crossing jets 160x160x80 Ma=1 Kn=1,
# averaged over the 200-step run: counted on a 160x160x4 slab through the
# jets of the state at steps 0, 25, ..., 175; recomputed by
# `python bench.py --count-ops` (needs the GPU for the states).
F_ALG = 92682.1
B_ALG = 2 * 35 * 8  # bytes per cell-step: state read once, written once

# The step's kernels in launch order (hyq_advance_timed slots) and their FP64
# operations per cell from the same count (CFL: one max per cell; HLL: three
# sweeps of 18 ops per moment plus the 4-op combination).
E2E_SLABS = 4
LAUNCHES_PER_STEP = 21  # the eleven timed kernels and the two passes over listed cells of A2-A4, E2, E3
# the launches of an eigenvalue stage (one hyq_advance_timed slot)
STAGE_KERNELS = {k: f"k_{p}_eig+k_{p}_fix+k_{p}_corr ({k[-1]})" for k, p in
                 (("A2_eig_x", "A"), ("A3_eig_y", "A"), ("A4_eig_z", "A"), ("E2_eig_x", "E"), ("E3_eig_y", "E"))}
KERNELS = ["A1_closure", "A2_eig_x", "A3_eig_y", "A4_eig_z", "A5_flux_speeds", "cfl", "hll",
           "E1_closure", "E2_eig_x", "E3_eig_y", "E4_closure_bgk"]
# DRAM bytes (read + write) per cell from ncu captures on the 96x96x48 case of
# the same workload (profiles/step_kernels_crossing96x96x48.md), scaled to a
# launch by its cells (the local-memory traffic per cell does not depend on
# the grid size): the eigenvalue stages A2-A4 from step 151 (dense mode, the
# late part of the run that dominates it), the closure and HLL kernels from
# the first step.
TRAFFIC_PER_CELL = {"A1_closure": 3221.0, "A2_eig_x": 3531.0, "A3_eig_y": 3546.0, "A4_eig_z": 4028.0, "A5_flux_speeds": 4487.0,
                    "hll": 1609.0, "E1_closure": 3211.0, "E4_closure_bgk": 3951.0}
TRAFFIC_SOURCE = ("ncu dram__bytes_read+write per cell on 96x96x48 (eigenvalue stages: all three kernels at step 151; "
                  "closures: first step), scaled to this launch's cells")
F_KERNEL = {"A1_closure": 11800.8, "A2_eig_x": 8014.9, "A3_eig_y": 8022.6, "A4_eig_z": 8494.7, "A5_flux_speeds": 13804.2,
            "cfl": 1.0, "hll": 2030.0, "E1_closure": 11811.2, "E2_eig_x": 8050.8, "E3_eig_y": 8050.3, "E4_closure_bgk": 12602.6}


def workload(name="c2"):
    from hyqmom import ic
    if name == "c2":
        # CFL 0.5: at the named CFL 0.7 the reference scheme's x+y+z-2M update
        # empties a jet-corner cell in step 1 (density 0.004, negative
        # variance), the CFL speed jumps 20x and a flux Jacobian turns NaN a
        # few steps later (the reference's eigvals throws there); 0.5 is the
        # largest of {0.3, 0.5, 0.7} that runs
        p = ic.default_params(Nx=160, Ny=160, Nz=80, Ma=1.0, Kn=1.0, CFL=0.5, tmax=1e9, nnmax=1000000)
    elif name == "c5":
        p = ic.default_params(Nx=256, Ny=256, Nz=128, Ma=1.0, Kn=0.01, CFL=0.5, tmax=1e9, nnmax=1000000)
    elif name == "c2s":
        # the same case on 96 x 96 x 48 cells: profiling captures (ncu)
        p = ic.default_params(Nx=96, Ny=96, Nz=48, Ma=1.0, Kn=1.0, CFL=0.5, tmax=1e9, nnmax=1000000)
    elif name == "c1":
        p = ic.default_params(Nx=20, Ny=20, Nz=20, Ma=0.0, Kn=1.0, CFL=0.7, tmax=1e9, nnmax=1000000)
    else:
        raise ValueError(name)
    return ic.with_jets(p, "crossing")


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


def slab_of(M, nz):
    """An nz-layer z-slab through the middle (the jets) of a state."""
    z0 = M.shape[2] // 2 - nz // 2
    return np.array(M[:, :, z0:z0 + nz, :], order="F")


def cpu_baseline(p, slabs, what=None):
    """The oracle (CPU restatement, OpenMP, all host threads): one step on each
    of `slabs` [(step, state)], slabs of the run's states at spread-out steps
    (the same array listed again is stepped again)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    from hyqmom import ic
    cells = el = 0.0
    for _, M in slabs:
        q = dict(p, Nz=M.shape[2], **ic.grid_spacing(p))
        t0 = time.perf_counter()
        ol.step(M, q, 0.0)
        el += time.perf_counter() - t0
        cells += M.shape[0] * M.shape[1] * M.shape[2]
    M = slabs[0][1]
    return {"value": cells / el, "unit": UNIT, "cores": int(ol.load().hyqo_num_threads()), "kind": "port",
            "sample": f"{what or 'one step of a z-slab through the jets of the run state at each of steps %s' % [k for k, _ in slabs]}"
                      f" ({M.shape[0]}x{M.shape[1]}x{M.shape[2]} cells, {int(cells)} cell-steps, {el:.1f} s), "
                      f"oracle C++ restatement, OpenMP"}


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
    M0 = ic.initial_state(p)
    s = Solver(p, device=local_rank)
    stream = torch.cuda.ExternalStream(s.stream)
    s.set_state(M0)
    s.advance(args.warmup)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # the timed steps: S+1..S+K of the run from the initial condition
    # (set_state resets t and nn; S = --from-step, 0 by default)
    def restart():
        s.set_state(M0)
        if args.from_step:
            s.advance(args.from_step)

    restart()
    barrier()
    sampler = ClockSampler(local_rank)
    with sampler:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.advance_async(args.steps)
        e1.record(stream)
        e1.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    st = s.stats()
    assert st["status"] == 0 and st["nn"] == args.from_step + args.steps, f"steps did not all run: {st}"
    ms = max_over_ranks(ms, dist, "cuda")
    value = replica_throughput(world, cells, args.steps, ms)

    # per-kernel device time over the same steps (individual launches, CUDA
    # events on the context stream)
    import ctypes
    restart()
    kms = (ctypes.c_float * len(KERNELS))()
    s._chk(s._lib.hyq_advance_timed(s._h, args.steps, kms))
    kern = {k: kms[i] / args.steps for i, k in enumerate(KERNELS)}

    # end to end through the public API over the same steps: each step uploads
    # the host state (pinned) and downloads the result (hyq_step_host, the
    # copies overlapped slab by slab with the per-cell phases).  Slabs of the
    # state at four points of the run are kept (outside the timing) for the
    # CPU baseline.
    restart()
    Mh_flat = torch.empty(35 * cells, dtype=torch.float64).pin_memory()
    Mh = Mh_flat.numpy().reshape(M0.shape, order="F")
    s._chk(s._lib.hyq_get_state(s._h, ctypes.c_void_p(Mh_flat.data_ptr())))
    marks = sorted({(args.steps * q) // 4 for q in range(4)})  # offsets into the timed steps
    slabs = []
    e2e_s = 0.0
    for k in range(args.steps):
        if k in marks:
            slabs.append((args.from_step + k, slab_of(Mh, 8)))
        t0 = time.perf_counter()
        s.step_host(Mh, nslabs=E2E_SLABS)
        e2e_s += time.perf_counter() - t0
    e2e = {"value": world * cells * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": Mh_flat.numel() * 8,
           "d2h_bytes_per_step": Mh_flat.numel() * 8, "api": f"hyq_step_host, {E2E_SLABS} slabs, pinned host state"}
    s.close()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    fp64 = fp64_peak_tflops(torch)
    # roofline of the dominant kernel: its algorithmic FP64 ops per launch over
    # its mean launch time; the FP64 peak is a measured DGEMM (an FMA counts 2)
    dom = max((k for k in KERNELS if k not in ("cfl", "hll")), key=lambda k: kern[k])
    ach = F_KERNEL[dom] * cells / (kern[dom] * 1e-3) / 1e12
    per_kernel = {k: {"ms": round(kern[k], 3), "tflops": round(F_KERNEL[k] * cells / (kern[k] * 1e-3) / 1e12, 3)}
                  for k in KERNELS if k not in ("cfl",)}
    step_tflops = F_ALG * cells / (ms / args.steps * 1e-3) / 1e12
    traffic = TRAFFIC_PER_CELL[dom] * cells if dom in TRAFFIC_PER_CELL else None
    roof = {"bound": "fp64", "achieved": ach, "peak": fp64, "unit": "TFLOP/s", "frac": ach / fp64, "traffic": traffic,
            "traffic_source": TRAFFIC_SOURCE,
            "peak_source": "measured in this run: FP64 DGEMM 8192^3 (cuBLAS via torch), best of 3",
            "dominant_kernel": STAGE_KERNELS.get(dom, "k_" + dom), "f_alg_per_cell": F_KERNEL[dom],
            "note": "built with -fmad=false: every counted op is one FP64 pipe instruction, so an FMA-free kernel tops out at peak/2",
            "step": {"f_alg_per_cell": F_ALG, "achieved": step_tflops, "frac": step_tflops / fp64,
                     "hbm_achieved_gbs": B_ALG * cells / (ms / args.steps * 1e-3) / 1e9},
            "kernels": per_kernel}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference crossing-jets IC generator)",
            "config": {"workload": f"crossing jets {p['Nx']}x{p['Ny']}x{p['Nz']} Ma={p['Ma']} Kn={p['Kn']} CFL={p['CFL']}, plain eig",
                       "cells": cells, "parallelism": f"replicas x{world}",
                       "timed_steps": f"{args.from_step + 1}-{args.from_step + args.steps} from the initial condition",
                       "l2": f"state {cells * 35 * 8 / 1e6:.0f} MB > L2 (126 MB), no flush needed",
                       "steps_done": st["nn"]},
            "gpu_launches": LAUNCHES_PER_STEP * args.steps, "e2e": e2e, "roofline": roof, "clocks": sampler.summary()}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p, slabs)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


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
    step) against the same domains advanced one at a time."""
    import torch
    torch.cuda.set_device(local_rank)
    from hyqmom import ic
    from hyqmom.runner import BatchSolver
    ps = batch_workload()
    cells = [p["Nx"] * p["Ny"] * p["Nz"] for p in ps]
    M0 = [ic.initial_state(p) for p in ps]
    b = BatchSolver(ps, device=local_rank)

    def reset():
        for m, M in zip(b.members, M0):
            m.set_state(M)

    def nn_all():
        return [m.stats()["nn"] for m in b.members]

    reset()
    b.advance(args.warmup)
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
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference crossing / triple-jet IC generator, seed 0)",
            "config": {"workload": f"batched sweep of {len(ps)} domains, 16^3..96x96x48, Ma U[0,2], Kn logU[1e-3,1], CFL 0.5",
                       "cells_total": sum(cells), "domains_failed": failed, "one_at_a_time_value": seq_value,
                       "batched_over_one_at_a_time": value / seq_value, "l2": "state of all domains > L2"},
            "gpu_launches": LAUNCHES_PER_STEP * args.steps * len(ps), "clocks": sampler.summary()}
    print(json.dumps(line), flush=True)


def count_ops(args):
    """F_ALG and F_KERNEL: the oracle's FP64 op counter on a 160x160x4 z-slab
    through the jets of the workload's state at steps 0, 25, ..., 175 of the
    run (states from the GPU step, which is bit-identical to the oracle's),
    averaged over the samples."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    from hyqmom import ic
    from hyqmom.runner import Solver
    p = workload("c2")
    s = Solver(p)
    s.set_state(ic.initial_state(p))
    names = [k for k in KERNELS if k not in ("cfl", "hll")]
    tot, stages, samples = np.zeros(3), np.zeros(len(names)), []
    for k in range(0, args.steps, 25):
        s.advance(k - s.stats()["nn"])
        M = slab_of(s.get_state(), 4)
        q = dict(p, Nz=M.shape[2], **ic.grid_spacing(p))
        cells = M.shape[0] * M.shape[1] * M.shape[2]
        out = ol.count_ops(M, q, 1e-3) / np.array([cells, cells, 1.0])
        st = ol.count_ops_stages(M, q, 1e-3)[:len(names)] / cells
        tot, stages = tot + out, stages + st
        samples.append({"step": k, "F": round(float(out[0] + out[1] + out[2]), 1)})
        print(json.dumps(samples[-1]), flush=True)
    s.close()
    n = len(samples)
    print(json.dumps({"samples": n, "F_alg": round(float(tot.sum() / n), 1), "hll_ops_per_cell": float(tot[2] / n),
                      "per_kernel": {k: round(float(v / n), 1) for k, v in zip(names, stages)}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--from-step", type=int, default=0, help="untimed steps from the initial condition before the timed ones")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c1", "c2", "c2s", "c4", "c5"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--count-ops", action="store_true")
    args = ap.parse_args()
    if args.count_ops:
        return count_ops(args)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.config == "c4":
        return run_batch(args, rank, world, local_rank)
    run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
