"""HyQMOM explicit time step on NVIDIA B200 (sm_100a).

Python host mirror of the reference's public entry points
(``simulation_runner``, ``run_simulation``, ``run_simulation_with_snapshots``,
src/simulation_runner.jl) over the C-ABI library ``libhyqmom_b200.so``.
"""
from . import ic  # noqa: F401
