"""HyQMOM explicit time step on NVIDIA B200 (sm_100a).

Python host mirror of the reference's public entry points
(``simulation_runner``, ``run_simulation``, ``run_simulation_with_snapshots``,
src/simulation_runner.jl) over the C-ABI library ``libhyqmom_b200.so``.
"""
from . import ic  # noqa: F401
from .ic import CubicRegion, run_simulation_params, default_params, jet_configuration, with_jets  # noqa: F401


def __getattr__(name):
    # the runner needs the CUDA library; import it lazily so that the host-only
    # pieces (parameters, grid, IC) work without a GPU build
    if name in ("simulation_runner", "run_simulation", "run_simulation_with_snapshots", "Solver"):
        from . import runner
        return getattr(runner, name)
    raise AttributeError(name)
