"""Edge cases at the drop-in boundary: a single atom (no pairs at all), pairs
at and just inside the cutoff, a neighbour list too small for its system, and
a non-finite energy (two atoms at one point).

The engine's error convention replaces the reference's asserts with status
codes: a list that overflows its capacity is truncated on the device (no
entry is written past it) and reported as LJ_ERR_CAPACITY; a non-finite
energy or virial is reported as LJ_ERR_NONFINITE.
"""

import numpy as np
import pytest

import ljref

pytestmark = pytest.mark.gpu


def test_single_atom_moves_ballistically():
    from lennardjonesium import GpuSystem
    x = np.array([[9.9, 0.05, 5.0]])
    v = np.array([[1.5, -0.7, 0.2]])
    with GpuSystem(1, 10.0) as g:
        g.upload(x, v=v)
        pe, w = g.compute_forces()
        assert pe == 0.0 and w == 0.0
        assert not g.download()["F"].any()
        th = g.step(40)  # crosses the x face: wrapped, displacement unwrapped
        st = g.download()
    ref = ljref.State(x, v=v)
    rth = ljref.run_steps(ref, 10.0, 0.005, 40)
    for k, a in (("x", ref.x), ("v", ref.v), ("d", ref.d)):
        assert np.array_equal(st[k][:, :3], a[:, :3]), k
    # the records' sums differ from the oracle's only in FMA contraction
    assert np.array_equal(th[:, 0], rth[:, 0])
    assert np.allclose(th, rth, rtol=1e-14, atol=0.0)
    assert st["x"][0, 0] < 1.0  # it wrapped


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pairs_at_the_cutoff(precision):
    """r = rc exactly is outside (r^2 < rc^2, particle_pair_filter.cpp:183);
    one ulp inside is a pair whose V and W are ~0 by the spline."""
    from lennardjonesium import GpuSystem
    rc = 2.5
    for r, inside in ((rc, False), (np.nextafter(rc, 0.0), True), (rc * 1.01, False)):
        x = np.array([[5.0, 5.0, 0.5], [5.0, 5.0, 0.5 + r]])  # 0.5 + r and r are exact
        with GpuSystem(2, 12.0, precision=precision) as g:
            g.upload(x)
            pe, w = g.compute_forces()
            F = g.download()["F"]
            npairs = g.debug_pairs()[0].shape[0]
        Fo, peo, wo = ljref.forces(x, 12.0, rc)
        assert npairs == (1 if inside else 0)  # each unordered pair once
        if precision == "fp64":
            assert abs(pe - peo) <= 1e-15 and abs(w - wo) <= 1e-14
            assert np.abs(F[:, :3] - Fo[:, :3]).max() <= 1e-14
        else:
            assert abs(pe - peo) < 1e-7 and abs(w - wo) < 1e-6
            assert np.abs(F[:, :3] - Fo[:, :3]).max() < 1e-6
        if not inside:
            assert pe == 0.0 and w == 0.0 and not F.any()


def test_capacity_overflow_is_reported():
    from lennardjonesium import GpuSystem, _native as nat
    x, v, L = ljref.initial_state(4000, 1.0, 0.8442, 12)
    with GpuSystem(4000, L, capacity=8) as g:  # ~80 candidates per atom, room for 8
        g.upload(x, v=v)
        with pytest.raises(nat.LJError) as e:
            g.step(1)
        assert e.value.status == nat.LJ_ERR_CAPACITY
    # the same system with the default capacity steps normally
    with GpuSystem(4000, L) as g:
        g.upload(x, v=v)
        g.step(1)
        assert g.stats()["max_neighbors"] <= g.stats()["neighbor_capacity"]


def test_nonfinite_energy_is_reported():
    from lennardjonesium import GpuSystem, _native as nat
    x = np.array([[4.0, 4.0, 4.0], [4.0, 4.0, 4.0], [1.0, 6.0, 2.0]])
    with GpuSystem(3, 10.0) as g:
        g.upload(x)
        with pytest.raises(nat.LJError) as e:
            g.compute_forces()
        assert e.value.status == nat.LJ_ERR_NONFINITE
