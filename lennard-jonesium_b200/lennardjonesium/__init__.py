"""B200 engine for lennard-jonesium's NVE hot path.

The package keeps the reference's import name and entry points
(src/python/lennardjonesium/__init__.py:1-8): run, run_sweep,
SweepConfiguration, SeedGenerator, Configuration, Simulation, SimulationPool.
Simulations run on a CUDA engine reached through the C ABI of include/lj_gpu.h;
GpuSystem exposes that engine directly.
"""

from lennardjonesium.engine import GpuSystem, initial_condition, autotune, window_stats_host, THERMO_FIELDS
from lennardjonesium.simulation import SeedGenerator, Configuration, Simulation, SimulationPool
from lennardjonesium.orchestration import run, run_sweep, SweepConfiguration, SweepResult, RunResult

_ADJOINT = ("AdjointNVE", "DifferentiableNVE", "nve_observables")


def __getattr__(name):
    # the differentiable engine imports torch; load it on first use only
    if name in _ADJOINT:
        from lennardjonesium import adjoint
        return getattr(adjoint, name)
    raise AttributeError(f"module 'lennardjonesium' has no attribute {name!r}")
