"""Simulation and SimulationPool over the engine's lj_sim_run.

Mirrors the reference's Cython classes (src/python/lennardjonesium/simulation/
_simulation.pyx:42-117, _simulation_pool.pyx:36-108): a Simulation runs one
configuration to completion and writes its four output files; a
SimulationPool runs pushed simulations on worker threads.  ctypes releases the
GIL during lj_sim_run, so pool workers run their GPU contexts concurrently.
"""

import ctypes
import queue
import threading
from typing import NamedTuple

from lennardjonesium import _native as nat
from lennardjonesium.simulation.configuration import Configuration

_PRECISION = {"fp64": nat.LJ_PRECISION_FP64, "mixed": nat.LJ_PRECISION_MIXED}


def _sim_config(cfg):
    c = nat.SimConfig()
    s, e, o, f = cfg.system, cfg.equilibration, cfg.observation, cfg.filepaths
    c.temperature, c.density = float(s.temperature), float(s.density)
    c.particle_count, c.random_seed = int(s.particle_count), int(s.random_seed) & 0xFFFFFFFF
    c.cutoff_distance, c.time_delta = float(s.cutoff_distance), float(s.time_delta)
    c.eq_name, c.eq_tolerance = e.name.encode(), float(e.tolerance)
    c.eq_sample_size, c.eq_adjustment_interval = int(e.sample_size), int(e.adjustment_interval)
    c.eq_steady_state_time, c.eq_timeout = int(e.steady_state_time), int(e.timeout)
    c.ob_name, c.ob_tolerance = o.name.encode(), float(o.tolerance)
    c.ob_sample_size, c.ob_observation_interval = int(o.sample_size), int(o.observation_interval)
    c.ob_observation_count = int(o.observation_count)
    c.event_log, c.thermodynamic_log = f.event_log.encode(), f.thermodynamic_log.encode()
    c.observation_log, c.snapshot_log = f.observation_log.encode(), f.snapshot_log.encode()
    c.precision = _PRECISION[cfg.engine.precision]
    c.device = int(cfg.engine.device)
    return c


class Simulation:
    """One Lennard-Jones NVE simulation described by a Configuration."""

    def __init__(self, configuration=None):
        if configuration is None:
            configuration = Configuration()
        if not isinstance(configuration, Configuration):
            raise TypeError("Argument must be of type Configuration")
        self.configuration = configuration
        self.result = None

    def run(self, *, echo=True, delay=0.05):
        """Run to completion (rerunning overwrites the output files); echo prints events live."""
        c = _sim_config(self.configuration)
        r = nat.SimResult()
        status = nat.lib().lj_sim_run(ctypes.byref(c), 1 if echo else 0, ctypes.byref(r))
        nat.check(status)
        self.result = {"time_steps": r.time_steps, "outcome": r.outcome, "observations": r.observations,
                       "seconds": r.seconds}
        return self.result

    def _pair(self, separation):
        out = (ctypes.c_double * 3)()
        nat.check(nat.lib().lj_pair_along_z(float(self.configuration.system.cutoff_distance),
                                            float(separation), out))
        return out

    def potential(self, separation):
        return self._pair(separation)[0]

    def virial(self, separation):
        return self._pair(separation)[1]

    def force(self, separation):
        return self._pair(separation)[2]


def run_batched(simulations, echo=False):
    """Run several Simulations on one batched GPU engine (lj_sim_run_batch): all
    systems step together, each with its own control protocol and output files.
    They must share cutoff and time step, and every box edge must be at least
    3 cutoffs.  Returns the per-simulation results."""
    if not simulations:
        return []
    n = len(simulations)
    cfgs = (nat.SimConfig * n)(*[_sim_config(sim.configuration) for sim in simulations])
    res = (nat.SimResult * n)()
    nat.check(nat.lib().lj_sim_run_batch(cfgs, n, 1 if echo else 0, res))
    out = []
    for sim, r in zip(simulations, res):
        sim.result = {"time_steps": r.time_steps, "outcome": r.outcome, "observations": r.observations,
                      "seconds": r.seconds}
        out.append(sim.result)
    return out


def fits_batched(configuration):
    """True when the run's cubic box holds >= 3 cells of edge >= cutoff per axis."""
    from lennardjonesium.engine import lattice_side
    s = configuration.system
    return lattice_side(s.particle_count, s.density) >= 3 * s.cutoff_distance


class SimulationPool:
    """Worker threads that run pushed Simulations (api/simulation_pool.cpp:35-101)."""

    Status = NamedTuple("Status", [("queued", int), ("waiting", int), ("started", int), ("running", int),
                                   ("completed", int)])

    def __init__(self, thread_count=4):
        if not isinstance(thread_count, int):
            raise TypeError("Thread count must be an integer")
        self._q = queue.Queue()
        self._lock = threading.Lock()
        self._queued = self._started = self._completed = 0
        self.errors = []
        self._workers = [threading.Thread(target=self._work, daemon=True) for _ in range(thread_count)]
        for w in self._workers:
            w.start()

    def _work(self):
        while True:
            sim = self._q.get()
            if sim is None:
                self._q.task_done()
                return
            with self._lock:
                self._started += 1
            try:
                sim.run(echo=False)
            except Exception as exc:  # reported through .errors, the run's files show how far it got
                with self._lock:
                    self.errors.append(exc)
            finally:
                with self._lock:
                    self._completed += 1
                self._q.task_done()

    def push(self, simulation):
        if not isinstance(simulation, Simulation):
            raise TypeError("Argument must be of type Simulation")
        with self._lock:
            self._queued += 1
        self._q.put(simulation)

    def status(self):
        with self._lock:
            return self.Status(self._queued, self._queued - self._started, self._started,
                               self._started - self._completed, self._completed)

    def wait(self):
        self._q.join()

    def close(self):
        for _ in self._workers:
            self._q.put(None)
        for w in self._workers:
            w.join()
