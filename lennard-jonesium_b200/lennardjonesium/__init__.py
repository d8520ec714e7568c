"""B200 engine for lennard-jonesium's NVE hot path.

The package keeps the reference's import name and entry points
(src/python/lennardjonesium/__init__.py:1-8) over a CUDA engine reached
through the C ABI of include/lj_gpu.h.
"""

from lennardjonesium.engine import GpuSystem, initial_condition, THERMO_FIELDS
