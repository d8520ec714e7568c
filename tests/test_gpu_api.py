"""The drop-in Python entry points on the GPU: lj.run(), lj.run_sweep(), Simulation.

The reference's own seeded run (notebooks/quick_single_run/data) is reproduced
through lj.run(): the event log byte for byte, the per-step thermodynamics to
1e-12 before the first rescale and within chaos growth after, the observations,
and the snapshot file's shape.
"""

import csv
import pathlib

import numpy as np
import pytest

import ljref

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"


def _rows(path, skip):
    with open(path) as fh:
        return [list(map(float, r)) for r in list(csv.reader(fh))[skip:] if r]


def test_run_reproduces_reference_seeded_run(tmp_path, golden):
    import lennardjonesium as lj
    cfg = lj.Configuration.from_file(GOLDEN / "quick_single_run_run.ini")
    result = lj.run(tmp_path / "run.ini", echo_status=False, config_object=cfg)
    assert (tmp_path / "events.log").read_text() == (GOLDEN / "quick_single_run_events.log").read_text()
    assert result.total_time_steps == 1600 and result.temperature_adjustments == [50, 100]
    thermo = np.array(_rows(tmp_path / "thermodynamics.csv", 1))
    assert thermo.shape == (1600, 8)
    head = golden["thermo_head"]
    assert np.array_equal(thermo[:200, 0], head[:, 0]) and np.array_equal(thermo[:200, 1], head[:, 1])
    rel = np.abs(thermo[:49, 2:] - head[:49, 2:]) / np.abs(head[:49, 2:])
    assert rel.max() < 1e-12
    te = golden["thermo_te"]
    assert (np.abs(thermo[:, 4] - te) / np.abs(te)).max() < 1e-8
    obs = np.array(_rows(tmp_path / "observations.csv", 1))
    ref_obs = golden["observations"]
    assert obs.shape == ref_obs.shape == (20, 7)
    assert np.array_equal(obs[:, 0], ref_obs[:, 0])
    # temperature, density, total energy, pressure: the first observations to 1e-9,
    # all of them to 1e-6 (by step 1600 chaos has grown the trajectory difference
    # to ~1e-7 in window averages); the fluctuation-based specific heat and the
    # regression slope D amplify it further, so they are held to 1e-4
    assert np.allclose(obs[:4, 1:5], ref_obs[:4, 1:5], rtol=1e-9)
    assert np.allclose(obs[:, 1:5], ref_obs[:, 1:5], rtol=1e-6)
    assert np.allclose(obs[:, 5:], ref_obs[:, 5:], rtol=1e-4, atol=1e-6)
    snap = np.array(_rows(tmp_path / "snapshots.csv", 2))
    assert snap.shape == (500, 11) and np.all(snap[:, 0] == 1600)
    # final positions: 1600 chaotic steps grow the 1e-16 summation-order
    # differences to ~1e-6 (measured 2.6e-6); the force parity at this exact state
    # is covered by test_gpu_parity.py::test_golden_snapshot
    assert np.abs(snap[:, 2:5] - golden["snapshot_xvf"][:, 0:3]).max() < 1e-4


def test_simulation_reference_python_test_config(tmp_path):
    """tests/python/lennardjonesium/simulation/test_simulation.py:14-48 (N=100,
    seed 17, 2 cells per axis): observations.csv holds observation_count + 1 lines,
    and the event log equals the CPU oracle's."""
    import lennardjonesium as lj
    cfg = lj.Configuration()
    s = cfg.system
    s.temperature, s.density, s.particle_count, s.cutoff_distance, s.random_seed = 0.6, 1.0, 100, 2.0, 17
    e = cfg.equilibration
    e.name, e.tolerance, e.sample_size, e.adjustment_interval, e.steady_state_time, e.timeout = (
        "Test Simulation Eq Phase", 0.10, 20, 100, 500, 5000)
    o = cfg.observation
    o.name, o.tolerance, o.sample_size, o.observation_interval, o.observation_count = (
        "Test Simulation Ob Phase", 0.10, 20, 100, 19)
    for k in vars(cfg.filepaths):
        setattr(cfg.filepaths, k, str(tmp_path / getattr(cfg.filepaths, k)))
    sim = lj.Simulation(cfg)
    sim.run(echo=False)
    lines = (tmp_path / "observations.csv").read_text().splitlines()
    events = (tmp_path / "events.log").read_text()
    oc = ljref.SimConfig(0.6, 1.0, 100, 17, 2.0, 0.005, 0.10, 20, 100, 500, 5000, 0.10, 20, 100, 19)
    _, ref_events, _ = ljref.simulate(oc)
    ref_events = (ref_events.replace("Equilibration Phase", "Test Simulation Eq Phase")
                  .replace("Observation Phase", "Test Simulation Ob Phase"))
    assert events == ref_events
    if "aborted" not in events:
        assert len(lines) == o.observation_count + 1


def test_run_sweep_small_grid(tmp_path):
    import lennardjonesium as lj
    sc = lj.SweepConfiguration()
    sc.system.temperature_start, sc.system.temperature_stop, sc.system.temperature_steps = 0.8, 1.2, 2
    sc.system.density_start, sc.system.density_stop, sc.system.density_steps = 0.5, 0.8, 2
    sc.system.particle_count = 108
    sc.equilibration.adjustment_interval, sc.equilibration.steady_state_time = 50, 100
    sc.equilibration.timeout, sc.equilibration.tolerance = 1000, 0.2
    sc.observation.observation_interval, sc.observation.observation_count = 50, 3
    sc.observation.tolerance = 0.5
    res = lj.run_sweep(tmp_path / "sweep.ini", echo_status=False, thread_count=2, random_seed=11,
                       sweep_config_object=sc)
    n = len(res.completed) + len(res.equilibration_aborted) + len(res.observation_aborted)
    assert n == 4
    for r in res.completed:
        assert len(r.event_data.observations_recorded) == 3
    # every run folder holds its own run.ini with the seed used and the four files
    for t, d in sc.sweep_range():
        folder = tmp_path / sc.simulation_dir(t, d)
        assert lj.Configuration.from_file(folder / "run.ini").system.random_seed == 11
        for name in ("events.log", "thermodynamics.csv", "observations.csv", "snapshots.csv"):
            assert (folder / name).is_file()


def _fmt(v):
    import ctypes
    from lennardjonesium import _native as nat
    buf = ctypes.create_string_buffer(40)
    assert nat.lib().lj_format_double(float(v), buf, 40) == 0
    return buf.value.decode()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_trajectory_frames_equal_downloads(tmp_path, precision):
    """Each trajectory frame, written by the background writer while the GPU
    steps on, is byte for byte the snapshot rows of lj_gpu_download_state at
    that step (steps 10, 20, 30 with every = 10; the 7 steps after the last
    frame add none)."""
    from lennardjonesium import GpuSystem
    N = 500
    x, v, L = ljref.initial_state(N, 0.5, 0.8, 117208264)
    path = tmp_path / "trajectory.csv"
    want = ["TimeStep,ParticleID,Position,Position,Position,Velocity,Velocity,Velocity,Force,Force,Force",
            "TimeStep,ParticleID,X,Y,Z,X,Y,Z,X,Y,Z"]
    with GpuSystem(N, L, precision=precision) as g:
        g.upload(x, v=v)
        g.trajectory_open(path, 10)
        for step in (10, 20, 30):
            g.step(10, record=False)
            st = g.download()
            for i in range(N):
                vals = [st[k][i, q] for k in ("x", "v", "F") for q in range(3)]
                want.append(",".join([str(step), str(i)] + [_fmt(a) for a in vals]))
        g.step_async(7)
        g.synchronize()
        assert g.trajectory_close() == 3
    assert path.read_text() == "\n".join(want) + "\n"


def test_trajectory_frame_of_a_large_system(tmp_path):
    """A frame of 42 592 atoms, more than one formatting block of 32 768 rows (the
    blocks are formatted on parallel threads and written in row order), is byte
    for byte the snapshot rows of lj_gpu_download_state at that step."""
    from lennardjonesium import GpuSystem
    N = 4 * 22 ** 3
    x, v, L = ljref.initial_state(N, 1.0, 0.8442, 11)
    path = tmp_path / "trajectory.csv"
    with GpuSystem(N, L) as g:
        g.upload(x, v=v)
        g.trajectory_open(path, 5)
        g.step(5, record=False)
        st = g.download()
        assert g.trajectory_close() == 1
    lines = path.read_text().split("\n")
    assert len(lines) == 2 + N + 1 and lines[-1] == ""
    for i in range(N):
        vals = [st[k][i, q] for k in ("x", "v", "F") for q in range(3)]
        assert lines[2 + i] == ",".join(["5", str(i)] + [_fmt(a) for a in vals]), i


def test_equilibration_reaches_a_new_temperature():
    """tests/cpp/integration/test_system_equilibration.cpp, loose phase: N = 100 at
    rho 0.8, rc 2.0 (two list cells per axis), started at T 0.3 and driven to 0.8
    by the equilibration rule (every 100 steps, rescale to the target when the
    mean T of the last 50 steps is off by >= 10 %; done after 5000 steps without
    a rescale).  The temperature then measured as the mean of 20 samples 5
    steps apart is within 10 % of 0.8."""
    from lennardjonesium import GpuSystem
    x, v, L = ljref.initial_state(100, 0.3, 0.8, 5489)
    with GpuSystem(100, L, cutoff=2.0) as g:
        g.upload(x, v=v)
        steady = 0
        for _ in range(500):  # the reference's timeout: 50 000 steps
            recs = g.step(100)
            if abs(recs[-50:, 5].mean() / 0.8 - 1.0) >= 0.10:
                g.set_temperature(0.8)
                steady = 0
            else:
                steady += 100
                if steady >= 5000:
                    break
        assert steady >= 5000
        T = np.mean([g.step(5)[-1, 5] for _ in range(20)])
    assert abs(T / 0.8 - 1.0) < 0.10
