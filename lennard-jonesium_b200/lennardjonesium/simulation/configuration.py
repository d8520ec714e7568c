"""Run configuration: the fields and defaults of the reference's Configuration
(src/python/lennardjonesium/simulation/configuration.py:30-75, api/configuration.hpp:35-102),
plus the engine's precision and device."""

from dataclasses import dataclass, field

from lennardjonesium.tools import INIParsable, DictParsable
from lennardjonesium.simulation.seed_generator import SeedGenerator


@dataclass
class Configuration(INIParsable, DictParsable):
    @dataclass
    class _System:
        temperature: float = 0.8
        density: float = 1.0
        particle_count: int = 100
        cutoff_distance: float = 2.5
        time_delta: float = 0.005
        random_seed: int = SeedGenerator.default_seed()

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
    class _Filepaths:
        event_log: str = "events.log"
        thermodynamic_log: str = "thermodynamics.csv"
        observation_log: str = "observations.csv"
        snapshot_log: str = "snapshots.csv"

    @dataclass
    class _Engine:
        precision: str = "fp64"   # "fp64" (the drop-in) or "mixed"
        device: int = 0

    system: _System = field(default_factory=_System)
    equilibration: _Equilibration = field(default_factory=_Equilibration)
    observation: _Observation = field(default_factory=_Observation)
    filepaths: _Filepaths = field(default_factory=_Filepaths)
    engine: _Engine = field(default_factory=_Engine)
