"""bench.py's CPU legs: the reference arm prints one JSON line with the keys
the benchmark contract asks for, and the CPU baseline times the oracle on the
slabs it is given.  Both run the oracle only (no GPU)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == bench.UNIT and d["metric"] == bench.METRIC
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_cpu_baseline_steps_each_given_slab():
    from hyqmom import ic
    p = bench.workload("c2s")
    M = ic.initial_state(p)
    a, b = bench.slab_of(M, 2), bench.slab_of(M, 2)
    assert a.shape == (p["Nx"], p["Ny"], 2, 35) and a.flags["F_CONTIGUOUS"]
    base = bench.cpu_baseline(p, [(0, a), (7, b)])
    assert base["value"] > 0 and base["unit"] == bench.UNIT
    assert "[0, 7]" in base["sample"] and "OpenMP" in base["sample"]
    # each slab was stepped on a copy: the caller's states are unchanged
    assert np.array_equal(a, bench.slab_of(M, 2)) and np.array_equal(a, b)
    serial = bench.cpu_baseline(p, [(0, a)], threads=1)
    assert serial["cores"] == 1 and "serial" in serial["sample"]


def test_timed_steps_spread_over_the_run():
    assert bench.timed_steps(500, 20) == list(range(25, 501, 25))
    assert bench.timed_steps(500, 1) == [500]
    assert bench.timed_steps(200, 3) == [67, 133, 200]
    assert bench.timed_steps(10, 50) == list(range(1, 11))


def test_traffic_tables_cover_every_slot_and_launch_variant():
    """The roofline's DRAM-traffic tables have an entry for every timed slot
    with per-cell kernels and for every HLL launch variant the library offers
    (the autotuner may pick any of them on the bench's workload)."""
    from hyqmom import _lib
    lib = _lib.load()
    per_cell = set(bench.KERNELS) - {"cfl", "hll"}
    assert set(bench.TRAFFIC_PER_CELL) == per_cell
    assert set(bench.TRAFFIC_HLL) == set(range(lib.hyq_variant_count(_lib.KERNEL_HLL)))
    assert all(v > bench.B_ALG / 2 for v in bench.TRAFFIC_PER_CELL.values())
