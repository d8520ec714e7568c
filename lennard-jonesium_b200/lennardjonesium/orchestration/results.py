"""RunResult / SweepResult: what the event logs say about finished runs.

Same fields and classification as the reference's
src/python/lennardjonesium/orchestration/run_result.py:31-127 and sweep_result.py:29-83.
"""

import pathlib
from dataclasses import dataclass
from enum import Enum, auto

from lennardjonesium.simulation import Configuration


class SimulationStatus(Enum):
    completed = auto()
    equilibration_aborted = auto()
    observation_aborted = auto()


class RunResult:
    def __init__(self, config_filepath):
        config_filepath = pathlib.Path(config_filepath)
        cfg = Configuration.from_file(config_filepath)
        log = pathlib.Path(cfg.filepaths.event_log)
        if not log.is_absolute():
            log = config_filepath.parent / log
        self.simulation_status = None
        self.equilibration_started = self.equilibration_completed = self.equilibration_time_steps = None
        self.observation_started = self.observation_completed = self.observation_time_steps = None
        self.total_time_steps = 0
        self.temperature_adjustments = []
        self.observations_recorded = []
        with open(log) as fh:
            for line in fh:
                if line.strip():
                    self._event(line.rstrip("\n"))

    def _event(self, line):
        step_text, what = line.split(": ", 1)
        step = int(step_text)
        self.total_time_steps = step
        if what.startswith("Phase started"):
            if self.equilibration_started is None:
                self.equilibration_started = step
            else:
                self.observation_started = step
        elif what.startswith("Phase complete"):
            if self.equilibration_completed is None:
                self.equilibration_completed = step
                self.equilibration_time_steps = step - self.equilibration_started
            else:
                self.observation_completed = step
                self.observation_time_steps = step - self.observation_started
                self.simulation_status = SimulationStatus.completed
        elif what.startswith("Temperature"):
            self.temperature_adjustments.append(step)
        elif what.startswith("Observation"):
            self.observations_recorded.append(step)
        elif what.startswith("Simulation aborted"):
            self.simulation_status = (SimulationStatus.equilibration_aborted if self.equilibration_completed is None
                                      else SimulationStatus.observation_aborted)


class SweepResult:
    @dataclass
    class _SimulationResult:
        simulation_dir: pathlib.Path
        event_data: RunResult

    def __init__(self, sweep_config_file, chunk_count=1, chunk_index=0):
        from lennardjonesium.orchestration.sweep_configuration import SweepConfiguration
        sweep_config_file = pathlib.Path(sweep_config_file)
        self.completed, self.equilibration_aborted, self.observation_aborted = [], [], []
        buckets = {SimulationStatus.completed: self.completed,
                   SimulationStatus.equilibration_aborted: self.equilibration_aborted,
                   SimulationStatus.observation_aborted: self.observation_aborted}
        cfg = SweepConfiguration.from_file(sweep_config_file)
        for sim_dir in cfg.simulation_dir_range(chunk_count, chunk_index):
            rr = RunResult(sweep_config_file.parent / sim_dir / cfg.templates.run_config_file)
            if rr.simulation_status in buckets:
                buckets[rr.simulation_status].append(self._SimulationResult(sim_dir, rr))
