"""The drop-in Python layer on CPU: configuration files, sweep ranges, event-log
parsing, the pair functions and the CSV number format (no GPU calls)."""

import ctypes
import math
import pathlib

import numpy as np
import pytest

import ljref

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"


def test_configuration_ini_round_trip(tmp_path):
    # tests/python/lennardjonesium/simulation/test_configuration.py:13-55
    from lennardjonesium import Configuration
    cfg = Configuration()
    cfg.system.temperature = 0.6
    cfg.system.particle_count = 123
    cfg.equilibration.name = "Eq"
    cfg.engine.precision = "mixed"
    f = tmp_path / "run.ini"
    cfg.write(f)
    back = Configuration.from_file(f)
    assert back == cfg
    assert isinstance(back.system.particle_count, int) and isinstance(back.system.temperature, float)


def test_configuration_dict_round_trip():
    from lennardjonesium import Configuration
    cfg = Configuration()
    d = cfg.to_dict()
    d["system"]["density"] = 0.75
    d["observation"]["extra_key"] = 1  # unknown keys are ignored
    back = Configuration.from_dict(d)
    assert back.system.density == 0.75 and not hasattr(back.observation, "extra_key")


def test_reference_run_ini_is_readable():
    from lennardjonesium import Configuration
    cfg = Configuration.from_file(GOLDEN / "quick_single_run_run.ini")
    assert cfg.system.particle_count == 500 and cfg.system.random_seed == 117208264
    assert cfg.equilibration.adjustment_interval == 50 and cfg.observation.tolerance == 0.2
    assert cfg.engine.precision == "fp64"


def test_sweep_range_and_chunks():
    from lennardjonesium import SweepConfiguration
    s = SweepConfiguration()
    s.system.temperature_start, s.system.temperature_stop, s.system.temperature_steps = 0.5, 2.0, 8
    s.system.density_start, s.system.density_stop, s.system.density_steps = 0.05, 1.0, 8
    pts = list(s.sweep_range())
    assert len(pts) == 64 and pts[0] == (0.5, 0.05) and pts[1][0] == 0.5 and pts[8][0] != 0.5
    assert pts[-1][0] == pytest.approx(2.0) and pts[-1][1] == pytest.approx(1.0)
    chunks = [list(s.sweep_range(5, k)) for k in range(5)]
    assert [len(c) for c in chunks] == [13, 13, 13, 13, 12] and sum(chunks, []) == pts
    assert str(s.simulation_dir(0.5, 0.05)) == "T_0.500000/d_0.050000"


def test_run_result_parses_reference_events(tmp_path):
    from lennardjonesium import Configuration, RunResult
    from lennardjonesium.orchestration import SimulationStatus
    cfg = Configuration.from_file(GOLDEN / "quick_single_run_run.ini")
    cfg.write(tmp_path / "run.ini")
    (tmp_path / "events.log").write_text((GOLDEN / "quick_single_run_events.log").read_text())
    r = RunResult(tmp_path / "run.ini")
    assert r.simulation_status == SimulationStatus.completed
    assert r.temperature_adjustments == [50, 100]
    assert r.equilibration_started == 0 and r.equilibration_completed == 600
    assert r.observation_started == 600 and r.observation_completed == 1600
    assert len(r.observations_recorded) == 20 and r.total_time_steps == 1600


def test_pair_functions_match_oracle():
    from lennardjonesium import Simulation, Configuration
    cfg = Configuration()
    cfg.system.cutoff_distance = 2.5
    sim = Simulation(cfg)
    for r in (0.95, 1.0, 2 ** (1 / 6), 1.7, 2.49, 2.6):
        V, W, Fz = ljref.pair_along_z(r, 2.5)
        assert sim.potential(r) == pytest.approx(V, rel=1e-14, abs=1e-300)
        assert sim.virial(r) == pytest.approx(W, rel=1e-14, abs=1e-300)
        assert sim.force(r) == pytest.approx(Fz, rel=1e-14, abs=1e-300)


def _fmt(x):
    from lennardjonesium import _native as nat
    buf = ctypes.create_string_buffer(64)
    assert nat.lib().lj_format_double(x, buf, 64) == 0
    return buf.value.decode()


def test_csv_number_format_matches_reference_files():
    """Every number in the reference's thermodynamics.csv re-formats to the same text."""
    text = (GOLDEN / "quick_single_run_events.log").read_text()  # noqa: F841 (presence)
    rng = np.random.default_rng(2)
    vals = np.concatenate([rng.normal(size=200) * 10.0 ** rng.integers(-9, 20, size=200),
                           [0.005, 3.7500000000000003e-05, 0.0001498634676421689, 7.999999999999852, 1600.0,
                            -2339.506585898019, 1e16, 1e15, 0.0001, 1e-05, 123456789012345.6]])
    for x in vals:
        s = _fmt(float(x))
        assert float(s) == x
        want = repr(float(x))
        if want.endswith(".0"):
            want = want[:-2]
        assert s == want, (x, s, want)
