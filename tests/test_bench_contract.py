"""The benchmark's arithmetic on the CPU: the timed step count, the roofline's
algorithmic work per atom-step and the clock summary's rejection fields.

The algorithmic flops are the reference's half-shell count F = 9 C + 30 P
(C candidate tests per atom over the 27-cell stencil counted once per pair, P
kept pairs): at N = 1 048 576, rho = 0.8442, rc = 2.5 the box edge is
107.494156 with 42 cells per axis, C = 190.6, P = 27.63 and F = 2544.
"""

import math
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, str(ROOT))
    import bench as b
    return b


def test_timed_steps_are_whole_graph_launches(bench):
    assert bench.timed_step_count(20) == 320
    assert bench.timed_step_count(320) == 320
    assert bench.timed_step_count(1000) == 1024
    for k in (1, 33, 500, 4097):
        n = bench.timed_step_count(k)
        assert n % bench.GRAPH_STEPS == 0 and n >= max(k, bench.MIN_TIMED_STEPS)


def test_algorithmic_flops_of_the_1m_atom_workload(bench):
    N, rho, rc = 4 * 64 ** 3, 0.8442, 2.5
    L = (N / rho) ** (1.0 / 3.0)
    assert L == pytest.approx(107.494156, abs=1e-6)
    assert math.floor(L / rc) == 42
    F, C, P = bench.alg_flops_per_atom_step(N, L, rc, rho)
    assert C == pytest.approx(190.6, abs=0.05)
    assert P == pytest.approx(27.63, abs=0.01)
    assert F == pytest.approx(2544, abs=1)


def test_clock_summary_reports_throttle_reasons(bench):
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1965, 1965, 720.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    s = c.summary()
    assert s == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    c.lines = []
    assert c.summary()["samples"] == 0
