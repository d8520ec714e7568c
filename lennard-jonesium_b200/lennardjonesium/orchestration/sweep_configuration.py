"""A (temperature, density) sweep: the fields and defaults of the reference's
SweepConfiguration (src/python/lennardjonesium/orchestration/sweep_configuration.py:34-136)."""

import itertools
import pathlib
from dataclasses import dataclass, field

from lennardjonesium.tools import INIParsable, DictParsable, linspace, divide


@dataclass
class SweepConfiguration(INIParsable, DictParsable):
    @dataclass
    class _System:
        temperature_start: float = 0.1
        temperature_stop: float = 1.0
        temperature_steps: int = 10
        density_start: float = 0.1
        density_stop: float = 1.0
        density_steps: int = 10
        particle_count: int = 100
        cutoff_distance: float = 2.5
        time_delta: float = 0.005

    @dataclass
    class _Templates:
        directory: str = "T_{temperature:f}/d_{density:f}"
        run_config_file: str = "run.ini"
        phase_name: str = "(T={temperature:f}, d={density:f}) {name}"

    @dataclass
    class _Equilibration:
        name: str = "Equilibration Phase"
        tolerance: float = 0.05
        sample_size: int = 50
        adjustment_interval: int = 200
        steady_state_time: int = 1000
        timeout: int = 5000

    @dataclass
    class _Observation:
        name: str = "Observation Phase"
        tolerance: float = 0.10
        sample_size: int = 50
        observation_interval: int = 200
        observation_count: int = 20

    @dataclass
    class _Filenames:
        event_log: str = "events.log"
        thermodynamic_log: str = "thermodynamics.csv"
        observation_log: str = "observations.csv"
        snapshot_log: str = "snapshots.csv"

    system: _System = field(default_factory=_System)
    templates: _Templates = field(default_factory=_Templates)
    equilibration: _Equilibration = field(default_factory=_Equilibration)
    observation: _Observation = field(default_factory=_Observation)
    filenames: _Filenames = field(default_factory=_Filenames)

    def sweep_range(self, chunk_count=1, chunk_index=0):
        """(temperature, density) pairs of one chunk: the T x rho product, T outer."""
        s = self.system
        ts = linspace(s.temperature_start, s.temperature_stop, s.temperature_steps, endpoint=True)
        ds = linspace(s.density_start, s.density_stop, s.density_steps, endpoint=True)
        yield from divide(chunk_count, itertools.product(ts, ds))[chunk_index]

    def simulation_dir(self, temperature, density):
        return pathlib.Path(self.templates.directory.format(temperature=temperature, density=density))

    def simulation_dir_range(self, chunk_count=1, chunk_index=0):
        return (self.simulation_dir(t, d) for t, d in self.sweep_range(chunk_count, chunk_index))
