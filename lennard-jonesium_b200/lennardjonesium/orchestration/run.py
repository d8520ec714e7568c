"""run(): one simulation from a config file, as the reference's
src/python/lennardjonesium/orchestration/run.py:35-107 (same arguments and
file handling); the simulation itself runs on the GPU engine."""

import os
import pathlib
import time
from copy import deepcopy
from types import BuiltinFunctionType, FunctionType

from lennardjonesium.simulation import Configuration, Simulation
from lennardjonesium.orchestration.results import RunResult


def _seed(value, default):
    if isinstance(value, bool):
        return default
    if isinstance(value, int):
        return value
    if isinstance(value, (FunctionType, BuiltinFunctionType)) or callable(value):
        return value()
    return default


def run(config_file, echo_status=True, random_seed=None, config_object=None):
    """Run the simulation described by config_file (or config_object, which then
    overwrites config_file).  random_seed: None keeps the file's seed, an int sets
    it, a callable supplies one.  The config file is (re)written with the seed
    used; output paths are relative to its folder.  Returns a RunResult."""
    path = pathlib.Path(config_file).resolve()
    if not path.is_file() and config_object is None:
        raise ValueError("config_object must be given if config_file is not an existing file")
    cfg = Configuration.from_file(path) if config_object is None else deepcopy(config_object)
    cfg.system.random_seed = _seed(random_seed, cfg.system.random_seed)
    path.parent.mkdir(parents=True, exist_ok=True)
    cfg.write(path)
    if echo_status:
        s = cfg.system
        print(f"==== Lennard-Jones simulation (B200 engine, {cfg.engine.precision}) ====\n"
              f"T = {s.temperature}, density = {s.density}, N = {s.particle_count}, dt = {s.time_delta}, "
              f"seed = {s.random_seed}\nphases: {cfg.equilibration.name}; {cfg.observation.name}", flush=True)
    cwd = os.getcwd()
    os.chdir(path.parent)
    try:
        sim = Simulation(cfg)
        t0 = time.perf_counter()
        sim.run(echo=echo_status)
        elapsed = time.perf_counter() - t0
    finally:
        os.chdir(cwd)
    result = RunResult(path)
    if echo_status:
        n = max(result.total_time_steps, 1)
        print(f"{result.total_time_steps} time steps in {elapsed:.3f} s "
              f"({1e3 * elapsed / n:.3f} ms per step, {n / elapsed:.1f} steps/s)", flush=True)
    return result
