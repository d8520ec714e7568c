"""run_sweep(): a grid of (temperature, density) simulations, as the reference's
src/python/lennardjonesium/orchestration/run_sweep.py:37-139 (same arguments,
folders and per-run config files).

batched=True (the default) runs every point whose box holds at least 3 cells
of edge >= cutoff per axis on one batched GPU engine (lj_sim_run_batch: one
launch per kernel for all systems, CUDA graphs per chunk of steps); the rest,
and every point when batched=False, run through a SimulationPool of
thread_count workers, one GPU context each (the reference's parallelism)."""

import os
import pathlib
import time
from copy import deepcopy

from lennardjonesium.simulation import Configuration, Simulation, SimulationPool, run_batched, fits_batched
from lennardjonesium.orchestration.results import SweepResult
from lennardjonesium.orchestration.run import _seed
from lennardjonesium.orchestration.sweep_configuration import SweepConfiguration


def _run_configuration(sweep_cfg, temperature, density):
    cfg = Configuration()
    s = cfg.system
    s.temperature, s.density = temperature, density
    s.particle_count = sweep_cfg.system.particle_count
    s.cutoff_distance = sweep_cfg.system.cutoff_distance
    s.time_delta = sweep_cfg.system.time_delta
    fmt = sweep_cfg.templates.phase_name
    for dst, src in ((cfg.equilibration, sweep_cfg.equilibration), (cfg.observation, sweep_cfg.observation)):
        for key, value in vars(src).items():
            setattr(dst, key, value)
        dst.name = fmt.format(temperature=temperature, density=density, name=src.name)
    for key in vars(cfg.filepaths):
        setattr(cfg.filepaths, key, getattr(sweep_cfg.filenames, key))
    return cfg


def _create_simulations(sweep_cfg, random_seed=None, chunk_count=1, chunk_index=0):
    sims = []
    for temperature, density in sweep_cfg.sweep_range(chunk_count, chunk_index):
        sim_dir = sweep_cfg.simulation_dir(temperature, density)
        run_file = sim_dir / sweep_cfg.templates.run_config_file
        cfg = _run_configuration(sweep_cfg, temperature, density)
        if random_seed is None and run_file.is_file():
            cfg.system.random_seed = Configuration.from_file(run_file).system.random_seed
        else:
            cfg.system.random_seed = _seed(random_seed, cfg.system.random_seed)
        run_file.parent.mkdir(parents=True, exist_ok=True)
        cfg.write(run_file)
        for key in vars(cfg.filepaths):  # paths relative to the sweep folder for the run itself
            setattr(cfg.filepaths, key, str(sim_dir / getattr(cfg.filepaths, key)))
        sims.append(Simulation(cfg))
    return sims


def run_sweep(sweep_config_file, echo_status=True, polling_interval=0.5, thread_count=4, random_seed=None,
              chunk_count=1, chunk_index=0, sweep_config_object=None, batched=True):
    """Run every (T, rho) point of the sweep (one chunk of it); returns a SweepResult."""
    path = pathlib.Path(sweep_config_file).resolve()
    if not path.is_file() and sweep_config_object is None:
        raise ValueError("sweep_config_object must be given if sweep_config_file is not an existing file")
    if sweep_config_object is None:
        sweep_cfg = SweepConfiguration.from_file(path)
    else:
        sweep_cfg = deepcopy(sweep_config_object)
        path.parent.mkdir(parents=True, exist_ok=True)
        sweep_cfg.write(path)
    cwd = os.getcwd()
    os.chdir(path.parent)
    try:
        sims = _create_simulations(sweep_cfg, random_seed, chunk_count, chunk_index)
        together = [s for s in sims if batched and fits_batched(s.configuration)]
        alone = [s for s in sims if not (batched and fits_batched(s.configuration))]
        if echo_status:
            print(f"==== Lennard-Jones sweep (B200 engine): {len(together)} runs batched, {len(alone)} runs on "
                  f"{thread_count} threads ====", flush=True)
        t0 = time.perf_counter()
        if together:
            run_batched(together)
        pool = SimulationPool(thread_count)
        for sim in alone:
            pool.push(sim)
        while echo_status and alone:
            st = pool.status()
            print(f"queued {st.waiting}, running {st.running}, completed {st.completed}, "
                  f"{time.perf_counter() - t0:.1f} s", end="\r", flush=True)
            if st.completed == len(alone):
                print(flush=True)
                break
            time.sleep(polling_interval)
        pool.wait()
        pool.close()
        elapsed = time.perf_counter() - t0
        if pool.errors:
            raise pool.errors[0]
    finally:
        os.chdir(cwd)
    result = SweepResult(path, chunk_count, chunk_index)
    if echo_status:
        print(f"completed {len(result.completed)}, aborted in equilibration {len(result.equilibration_aborted)}, "
              f"aborted in observation {len(result.observation_aborted)}; {elapsed:.3f} s", flush=True)
    return result
