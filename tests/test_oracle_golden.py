"""Pin the CPU oracle against the reference's committed run data.

notebooks/quick_single_run/data of bniehoff/lennard-jonesium (run.ini:1-28):
N=500, rho=0.8, T=0.5, rc=2.5, dt=0.005, seed 117208264.  The fixtures in
tests/golden were extracted by tests/golden/make_golden.py.
"""

import numpy as np
import pytest

import ljref

RUN = dict(T=0.5, rho=0.8, N=500, rc=2.5, dt=0.005, seed=117208264)


@pytest.fixture(scope="module")
def side():
    _, _, L = ljref.initial_state(RUN["N"], RUN["T"], RUN["rho"], RUN["seed"])
    return L


def test_box_side(side):
    # tools/cubic_lattice.cpp:43-58: 5 cells per side, scale cbrt((500/125)/0.8)
    assert side == pytest.approx(5 * (5.0) ** (1 / 3), rel=1e-15)


def test_snapshot_forces_pe_virial(golden, side):
    """Single-step known answer: F, PE and W recomputed from the step-1600 positions."""
    snap = golden["snapshot_xvf"]
    last = golden["thermo_tail"][0]  # TimeStep, Time, KE, PE, TE, W, T, MSD
    F, pe, w = ljref.forces(snap[:, 0:3], side, RUN["rc"])
    assert pe == pytest.approx(last[3], rel=1e-12)
    assert w == pytest.approx(last[5], rel=1e-12)
    scale = np.abs(snap[:, 6:9]).max()
    assert np.abs(F[:, :3] - snap[:, 6:9]).max() <= 1e-12 * scale
    ke = 0.5 * np.sum(snap[:, 3:6] ** 2)
    assert ke == pytest.approx(last[2], rel=1e-13)


def _config():
    return ljref.SimConfig(RUN["T"], RUN["rho"], RUN["N"], RUN["seed"], RUN["rc"], RUN["dt"],
                           0.1, 50, 50, 500, 2000, 0.2, 50, 50, 20)


@pytest.fixture(scope="module")
def seeded_run():
    return ljref.simulate(_config())


def test_seeded_trajectory_head(golden, seeded_run):
    """The seeded init plus the control protocol reproduce the first 200 rows."""
    thermo, _, _ = seeded_run
    head = golden["thermo_head"]
    ours = thermo[:200]
    assert np.allclose(ours[:, 0], head[:, 1], rtol=1e-13, atol=0)
    rel = np.abs(ours[:, 1:7] - head[:, 2:8]) / np.abs(head[:, 2:8])
    assert rel.max() < 1e-13


def test_seeded_events_log(seeded_run):
    """The event stream (rescales at 50 and 100, phase changes) is byte-identical."""
    _, events, _ = seeded_run
    with open(__file__.replace("test_oracle_golden.py", "golden/quick_single_run_events.log")) as fh:
        assert events == fh.read()


def test_total_energy_trace(golden, seeded_run):
    """All 1600 rows of TE agree; chaos only amplifies rounding late in the run."""
    thermo, _, _ = seeded_run
    te = golden["thermo_te"]
    assert thermo.shape[0] == te.shape[0] == 1600
    rel = np.abs(thermo[:, 3] - te) / np.abs(te)
    assert rel[:900].max() < 1e-13
    assert rel.max() < 1e-9


def test_initial_temperature_and_momentum():
    x, v, L = ljref.initial_state(RUN["N"], RUN["T"], RUN["rho"], RUN["seed"])
    ke = 0.5 * np.sum(v[:, :3] ** 2)
    assert (2.0 / 3.0) * ke / RUN["N"] == pytest.approx(RUN["T"], rel=1e-14)
    assert np.abs(v[:, :3].sum(axis=0)).max() < 1e-12
    com = x[:, :3].mean(axis=0)
    ang = np.cross(x[:, :3] - com, v[:, :3]).sum(axis=0)
    assert np.abs(ang).max() < 1e-10
