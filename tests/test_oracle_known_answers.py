"""The reference's unit known answers, checked on the CPU oracle.

Each test cites the reference test it restates (tests/cpp/lennardjonesium/...).
The same cases run through the GPU library in tests/test_gpu_known_answers.py.
"""

import math

import numpy as np
import pytest

import ljref

# engine/test_particle_pair_filter.cpp:59-91: box 10, rc 2, 10 atoms, 8 pairs
PAIR_POSITIONS = np.array([
    [0, 0, 0], [1, 1, 1], [1, 9, 9], [9, 1, 9], [9, 9, 1],
    [5, 5, 5], [4, 4, 4], [4, 6, 6], [6, 4, 6], [6, 6, 4]], dtype=float)
PAIR_EXPECTED = [  # (separation, first, second)
    ((-1, -1, -1), 0, 1), ((-1, 1, 1), 0, 2), ((1, -1, 1), 0, 3), ((1, 1, -1), 0, 4),
    ((1, 1, 1), 5, 6), ((1, -1, -1), 5, 7), ((-1, 1, -1), 5, 8), ((-1, -1, 1), 5, 9)]


def canonical_pairs(pi, pj, sep):
    """Unordered, sign-aware pair set (particle_pair_filter.cpp:37-48)."""
    out = set()
    for i, j, s in zip(pi, pj, sep):
        s = tuple(np.round(np.asarray(s, dtype=float), 9))
        if i > j:
            i, j, s = j, i, tuple(-c for c in s)
        out.add((int(i), int(j), s))
    return out


def separations(x, L, pi, pj, codes):
    img = np.stack([codes // 9 - 1, (codes // 3) % 3 - 1, codes % 3 - 1], axis=1)
    return (x[pi] - x[pj]) - img * np.asarray(L)


@pytest.mark.parametrize("naive", [False, True])
def test_pair_filter_known_pairs(naive):
    pi, pj, codes, _ = ljref.pairs(PAIR_POSITIONS, 10.0, 2.0, naive=naive)
    got = canonical_pairs(pi, pj, separations(PAIR_POSITIONS, 10.0, pi, pj, codes))
    want = canonical_pairs([p[1] for p in PAIR_EXPECTED], [p[2] for p in PAIR_EXPECTED],
                           [p[0] for p in PAIR_EXPECTED])
    assert got == want


@pytest.mark.parametrize("L,rc", [(1.0, 0.3), (1.0, 0.48), (1.0, 0.67), (1.0, 0.9),
                                  ((1.0, 1.3, 0.7), 0.31), (5.0, 1.2)])
def test_cell_filter_equals_naive_filter(L, rc):
    """Stencil completeness (tools/test_cell_list_array.cpp:117-244) as a pair-set
    identity on 1^3, 2^3, 3^3 and anisotropic grids: the cell-list filter finds
    exactly the naive filter's (i, j, image) triples with bit-identical r^2."""
    rng = np.random.default_rng(7)
    Lv = np.broadcast_to(np.asarray(L, dtype=float), (3,))
    x = rng.random((60, 3)) * Lv
    a = ljref.pairs(x, Lv, rc)
    b = ljref.pairs(x, Lv, rc, naive=True)

    def key(pi, pj, codes, r2):
        s = set()
        for i, j, c, r in zip(pi, pj, codes, r2):
            if i > j:
                i, j, c = j, i, 26 - c
            s.add((int(i), int(j), int(c), float(r)))
        return s

    ka, kb = key(*a), key(*b)
    assert len(ka) == len(a[0]) and ka == kb


def test_cell_shape():
    assert list(ljref.cell_shape(8.549879733383484, 2.5)) == [3, 3, 3]
    assert list(ljref.cell_shape(1.0, 0.67)) == [1, 1, 1]
    assert list(ljref.cell_shape((10.0, 5.0, 2.5), 2.5)) == [4, 2, 1]


def test_binning_order_and_offsets():
    rng = np.random.default_rng(3)
    x = rng.random((200, 3)) * 10.0
    cell_of, offsets, members = ljref.bin_atoms(x, 10.0, 2.5)
    assert offsets[0] == 0 and offsets[-1] == 200
    ratio = 4 / 10.0
    c = np.floor(x * ratio).astype(int)
    assert np.array_equal(cell_of, (c[:, 0] * 4 + c[:, 1]) * 4 + c[:, 2])
    for k in range(64):
        seg = members[offsets[k]:offsets[k + 1]]
        assert np.all(np.diff(seg) > 0) and np.all(cell_of[seg] == k)


# engine/test_short_range_force_calculation.cpp:18-166 (mock constant force, strength -10)
@pytest.mark.parametrize("z0,z1", [(0.2, 0.6), (0.8, 1.2), (2.8, 0.2)])
def test_mock_force_two_particles(z0, z1):
    x = np.array([[0.2, 0.2, z0], [0.2, 0.2, z1]])
    F, pe, w = ljref.forces(x, 3.0, rc=1.0, kind=ljref.FORCE_CONSTANT, strength=-10.0)
    assert np.allclose(F[0, :3], [0, 0, 10.0]) and np.allclose(F[1, :3], [0, 0, -10.0])
    assert pe == pytest.approx(-6.0) and w == pytest.approx(-4.0)


def test_mock_force_l_shape():
    x = np.array([[0.6, 0.6, 0.2], [1.4, 0.6, 0.2], [0.6, 1.4, 0.2]])
    F, pe, w = ljref.forces(x, 3.0, rc=1.0, kind=ljref.FORCE_CONSTANT, strength=-10.0)
    assert np.allclose(F[:, :3], [[10, 10, 0], [-10, 0, 0], [0, -10, 0]])
    assert pe == pytest.approx(-4.0) and w == pytest.approx(-16.0)


# engine/test_velocity_verlet_integrator.cpp:25-239 (dt = 1, 4 steps)
@pytest.mark.parametrize("gravity,periodic", [(False, False), (True, False), (False, True),
                                              (True, True)])
def test_velocity_verlet_exact(gravity, periodic):
    v = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    F = np.array([[0, 0, -1.0], [0, 0, -1.0]]) if gravity else np.zeros((2, 3))
    st = ljref.State(np.zeros((2, 3)), v=v, F=F)
    ljref.run_steps(st, 3.0, 1.0, 4, kind=ljref.FORCE_NONE, periodic=periodic, record=False)
    z = -8.0 if gravity else 0.0
    want_x = np.array([[4.0, 0, z], [0, 4.0, z]])
    want_d = want_x.copy()
    if periodic:
        want_x = np.array([[1.0, 0, 1.0 if gravity else 0.0], [0, 1.0, 1.0 if gravity else 0.0]])
    assert np.array_equal(st.x[:, :3], want_x)
    assert np.array_equal(st.d[:, :3], want_d)
    assert np.array_equal(st.v[:, :3], [[1.0, 0, -4.0 if gravity else 0], [0, 1.0, -4.0 if gravity else 0]])
    assert st.t == 4.0


def test_periodic_wrap():
    # engine/test_periodic_boundary_condition.cpp:12-42: box 1.5 wraps to 0.2
    x = np.array([[1.7, 0, 0], [0, 3.2, 0], [0, 0, -4.3]])
    st = ljref.State(x)
    ljref.run_steps(st, 1.5, 0.0, 1, kind=ljref.FORCE_NONE, periodic=True, record=False)
    assert st.x[0, 0] == pytest.approx(0.2) and st.x[1, 1] == pytest.approx(0.2)
    assert st.x[2, 2] == pytest.approx(0.2)


def test_lennard_jones_shape():
    # physics/test_lennard_jones_force.cpp:13-157 with rc = 4.5
    rc, d, tol = 4.5, 0.025, 0.002
    well = 2 ** (1 / 6)
    V, W, Fz = ljref.pair_along_z(1 - d, rc)
    assert V > 0 and W > 0 and Fz > 0
    V, W, Fz = ljref.pair_along_z(1 + d, rc)
    assert V < 0 and W > 0 and Fz > 0
    V, W, Fz = ljref.pair_along_z(well, rc)
    assert abs(V + 1) < tol and abs(W) < tol and abs(Fz) < tol
    V, W, Fz = ljref.pair_along_z(well + d, rc)
    assert V < 0 and W < 0 and Fz < 0
    V, W, Fz = ljref.pair_along_z(rc - d, rc)
    assert abs(V) < tol and abs(W) < tol and abs(Fz) < tol
    assert list(ljref.pair_along_z(rc + d, rc)) == [0.0, 0.0, 0.0]


def test_spline_vanishes_at_cutoff():
    rc = 2.5
    a, b = ljref.spline(rc)
    r6 = rc ** -6
    assert 4 * r6 * (r6 - 1) + a == pytest.approx(0.0, abs=1e-15)
    assert 24 * r6 * (2 * r6 - 1) - 2 * b == pytest.approx(0.0, abs=1e-15)


def test_measurements_four_atom_cube():
    # physics/test_measurements.cpp:15-100: rotating 4-atom cube, KE = 4, T = (8/3)/4
    x = np.array([[0, 0, 0], [0, 0, 2], [2, 2, 0], [2, 2, 2]], dtype=float)
    v = np.array([[1, -1, 0], [1, -1, 0], [-1, 1, 0], [-1, 1, 0]], dtype=float)
    st = ljref.State(x, v=v)
    th = ljref.run_steps(st, 100.0, 0.0, 1, kind=ljref.FORCE_NONE, periodic=False)
    assert th[0, 1] == pytest.approx(4.0) and th[0, 5] == pytest.approx(8 / 3 / 4)


def test_set_temperature():
    rng = np.random.default_rng(0)
    v = np.zeros((50, 4))
    v[:, :3] = rng.normal(size=(50, 3))
    v = ljref.set_temperature(v, 1.7)
    assert (2 / 3) * 0.5 * np.sum(v ** 2) / 50 == pytest.approx(1.7, rel=1e-14)


def test_rdf_ideal_lattice_peak():
    """FCC lattice: the first peak holds 12 neighbours per atom at a/sqrt(2)."""
    x, _, L = ljref.initial_state(256, 1.0, 0.8442, 1)
    nbins, rmax = 200, 4.0 if L / 2 >= 4.0 else L / 2
    h = ljref.rdf(x, L, nbins, rmax)
    a = L / 4
    r1 = a / math.sqrt(2)
    b1 = int(r1 * nbins / rmax)
    assert h[b1] == 256 * 12
    assert h[:b1].sum() == 0


@pytest.mark.parametrize("N,rho,rmax,threads", [(2048, 0.8442, 3.0, 1), (4000, 0.8, 4.0, 3), (6912, 0.3, 5.0, 4)])
def test_rdf_cells_equals_all_pairs(N, rho, rmax, threads):
    """The O(N) cell-list RDF (used at sizes where the all-pairs one is too slow)
    counts exactly the all-pairs histogram, on any number of threads."""
    x, _, L = ljref.initial_state(N, 1.0, rho, 3)
    rng = np.random.default_rng(N)
    x[:, :3] = np.mod(x[:, :3] + rng.uniform(-0.3, 0.3, size=(N, 3)), L)
    assert L / 3 >= rmax
    assert np.array_equal(ljref.rdf_cells(x, L, 200, rmax, threads=threads), ljref.rdf(x, L, 200, rmax))
