"""B200 engine for lennard-jonesium's NVE hot path.

The package keeps the reference's import name and entry points
(src/python/lennardjonesium/__init__.py:1-8): run, run_sweep,
SweepConfiguration, SeedGenerator, Configuration, Simulation, SimulationPool.
Simulations run on a CUDA engine reached through the C ABI of include/lj_gpu.h;
GpuSystem exposes that engine directly.
"""

from lennardjonesium.engine import GpuSystem, initial_condition, autotune, THERMO_FIELDS
from lennardjonesium.simulation import SeedGenerator, Configuration, Simulation, SimulationPool
from lennardjonesium.orchestration import run, run_sweep, SweepConfiguration, SweepResult, RunResult
