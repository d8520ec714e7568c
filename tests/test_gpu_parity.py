"""GPU path vs the CPU oracle, through the C ABI.

Tolerances (FP64 path):
  * cell assignment, cell offsets, cell members, neighbour-pair set: bit-exact
    (pairs compared as (i, j, image, r^2) with r^2 bit patterns equal);
  * per-atom forces: |F_gpu - F_ref| <= 1e-12 * S_i per component, where S_i is
    the sum of |f_ij| over atom i's pairs (the scale the summation order acts on);
  * PE and virial: 1e-12 relative;
  * integration with no force calculation: bit-exact;
  * RDF histogram: bit-exact.
"""

import numpy as np
import pytest

import ljref

pytestmark = pytest.mark.gpu

FCC_CASES = [  # N, T, rho, seed, rc
    (864, 0.722, 0.8442, 5489, 2.5),
    (500, 0.5, 0.8, 117208264, 2.5),
    (100, 0.6, 1.0, 17, 2.0),       # 2 cells per axis (the reference's Python test config)
    (4000, 1.2, 0.8, 7, 2.5),
    (4000, 1.2, 0.8, 7, 4.5),       # 3 list cells of ~5.7 sigma per axis: the largest cell edges
]


def gpu_system(N, L, **kw):
    from lennardjonesium import GpuSystem
    return GpuSystem(N, L, **kw)


def perturbed_fcc(N, T, rho, seed, amp=0.15):
    x, v, L = ljref.initial_state(N, T, rho, seed)
    rng = np.random.default_rng(seed)
    x[:, :3] = np.mod(x[:, :3] + rng.uniform(-amp, amp, size=(N, 3)), L)
    return x, v, L


def pair_key(i, j, img, r2):
    return set(zip(i.tolist(), j.tolist(), img.tolist(), r2.view(np.int64).tolist()))


def oracle_pair_key(x, L, rc):
    pi, pj, pc, pr = ljref.pairs(x, L, rc)
    swap = pi > pj
    i = np.where(swap, pj, pi)
    j = np.where(swap, pi, pj)
    c = np.where(swap, 26 - pc, pc)
    return pair_key(i, j, c, pr)


def assert_forces(F, Fref, Sabs, tol=1e-12):
    err = np.abs(F[:, :3] - Fref[:, :3])
    bound = tol * np.maximum(Sabs, 1e-300)[:, None]
    assert np.all(err <= bound), f"max excess {(err / bound).max()}"


@pytest.mark.parametrize("case", FCC_CASES)
def test_forces_pe_virial(case):
    N, T, rho, seed, rc = case
    x, _, L = perturbed_fcc(N, T, rho, seed)
    Fref, pe, w = ljref.forces(x, L, rc)
    S = ljref.force_abs_sum(x, L, rc)
    with gpu_system(N, L, cutoff=rc) as g:
        g.upload(x)
        gpe, gw = g.compute_forces()
        F = g.download()["F"]
    assert gpe == pytest.approx(pe, rel=1e-12)
    assert gw == pytest.approx(w, rel=1e-12)
    assert_forces(F, Fref, S)


def test_golden_snapshot(golden):
    """Forces, PE and W at step 1600 of the reference's own run."""
    snap = golden["snapshot_xvf"]
    last = golden["thermo_tail"][0]
    _, _, L = ljref.initial_state(500, 0.5, 0.8, 117208264)
    with gpu_system(500, L) as g:
        g.upload(snap[:, 0:3], v=snap[:, 3:6])
        pe, w = g.compute_forces()
        st = g.download()
        m = g.measure()
    assert pe == pytest.approx(last[3], rel=1e-12)
    assert w == pytest.approx(last[5], rel=1e-12)
    assert np.abs(st["F"][:, :3] - snap[:, 6:9]).max() <= 1e-12 * np.abs(snap[:, 6:9]).max()
    assert m[1] == pytest.approx(last[2], rel=1e-13)


@pytest.mark.parametrize("case", FCC_CASES)
def test_pair_set_bit_exact(case):
    N, T, rho, seed, rc = case
    x, _, L = perturbed_fcc(N, T, rho, seed)
    with gpu_system(N, L, cutoff=rc) as g:
        g.upload(x)
        got = pair_key(*g.debug_pairs())
    want = oracle_pair_key(x, L, rc)
    assert len(got) == len(want) and got == want


@pytest.mark.parametrize("L,rc,N", [(10.0, 2.0, 10), (1.6, 1.2, 12), (3.0, 1.2, 40), (5.0, 1.2, 60),
                                    ((4.0, 7.5, 2.6), 1.2, 50)])
def test_pair_set_small_and_anisotropic_boxes(L, rc, N):
    """1, 2 and 3+ cells per axis: explicit images vs minimum image."""
    rng = np.random.default_rng(N)
    Lv = np.broadcast_to(np.asarray(L, dtype=float), (3,))
    x = rng.random((N, 3)) * Lv
    if N == 10:
        from test_oracle_known_answers import PAIR_POSITIONS
        x = PAIR_POSITIONS
    with gpu_system(N, Lv, cutoff=rc) as g:
        g.upload(x)
        got = pair_key(*g.debug_pairs())
        Fg = g.download()["F"]
        g.compute_forces()
        Fg = g.download()["F"]
    assert got == oracle_pair_key(x, Lv, rc)
    Fref, _, _ = ljref.forces(x, Lv, rc)
    assert_forces(Fg, Fref, ljref.force_abs_sum(x, Lv, rc))


@pytest.mark.parametrize("case", FCC_CASES[:3])
def test_cells_bit_exact(case):
    N, T, rho, seed, rc = case
    x, _, L = perturbed_fcc(N, T, rho, seed)
    with gpu_system(N, L, cutoff=rc) as g:
        g.upload(x)
        shape, cell_of, offsets, members = g.debug_cells()
    rcell, roff, rmem = ljref.bin_atoms(x, L, rc)
    assert list(shape) == list(ljref.cell_shape(L, rc))
    assert np.array_equal(cell_of, rcell)
    assert np.array_equal(offsets, roff)
    assert np.array_equal(members, rmem)


@pytest.mark.parametrize("gravity,periodic", [(False, False), (True, False), (False, True), (True, True)])
def test_velocity_verlet_exact(gravity, periodic):
    # engine/test_velocity_verlet_integrator.cpp:25-239
    v = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    F = np.array([[0, 0, -1.0], [0, 0, -1.0]]) if gravity else np.zeros((2, 3))
    with gpu_system(2, 3.0, dt=1.0, force="none", periodic=periodic) as g:
        g.upload(np.zeros((2, 3)), v=v, F=F)
        g.step(4)
        st = g.download()
    ref = ljref.State(np.zeros((2, 3)), v=v, F=F)
    ljref.run_steps(ref, 3.0, 1.0, 4, kind=ljref.FORCE_NONE, periodic=periodic, record=False)
    for k, a in (("x", ref.x), ("v", ref.v), ("d", ref.d)):
        assert np.array_equal(st[k][:, :3], a[:, :3]), k
    assert st["t"] == 4.0


def test_periodic_wrap():
    x = np.array([[1.7, 0, 0], [0, 3.2, 0], [0, 0, -4.3]])
    with gpu_system(3, 1.5, dt=0.0, force="none") as g:
        g.upload(x)
        g.step(1)
        st = g.download()
    ref = ljref.State(x)
    ljref.run_steps(ref, 1.5, 0.0, 1, kind=ljref.FORCE_NONE, periodic=True, record=False)
    assert np.array_equal(st["x"][:, :3], ref.x[:, :3])
    assert st["x"][0, 0] == pytest.approx(0.2)


@pytest.mark.parametrize("z0,z1", [(0.2, 0.6), (0.8, 1.2), (2.8, 0.2)])
def test_mock_force_two_particles(z0, z1):
    # engine/test_short_range_force_calculation.cpp:18-112
    x = np.array([[0.2, 0.2, z0], [0.2, 0.2, z1]])
    with gpu_system(2, 3.0, cutoff=1.0, force="constant", strength=-10.0) as g:
        g.upload(x)
        pe, w = g.compute_forces()
        F = g.download()["F"]
    assert np.allclose(F[0, :3], [0, 0, 10.0]) and np.allclose(F[1, :3], [0, 0, -10.0])
    assert pe == pytest.approx(-6.0) and w == pytest.approx(-4.0)


def test_mock_force_l_shape():
    x = np.array([[0.6, 0.6, 0.2], [1.4, 0.6, 0.2], [0.6, 1.4, 0.2]])
    with gpu_system(3, 3.0, cutoff=1.0, force="constant", strength=-10.0) as g:
        g.upload(x)
        pe, w = g.compute_forces()
        F = g.download()["F"]
    assert np.allclose(F[:, :3], [[10, 10, 0], [-10, 0, 0], [0, -10, 0]])
    assert pe == pytest.approx(-4.0) and w == pytest.approx(-16.0)


@pytest.mark.parametrize("r", [0.975, 1.025, 2 ** (1 / 6), 2 ** (1 / 6) + 0.025, 4.475, 4.525])
def test_lennard_jones_shape(r):
    """physics/test_lennard_jones_force.cpp:13-157 through the GPU: two atoms along z, rc 4.5."""
    x = np.array([[7.0, 7.0, 7.0 + r], [7.0, 7.0, 7.0]])
    with gpu_system(2, 14.0, cutoff=4.5) as g:
        g.upload(x)
        pe, w = g.compute_forces()
        F = g.download()["F"]
    V, W, Fz = ljref.pair_along_z(r, 4.5)
    # near the well bottom V, W and F pass through ~0: the tolerance is 1e-12 of
    # the size of the terms that cancel there (4 r^-12 + 4 r^-6 for V, 48 r^-12 + 24 r^-6 for W)
    sV, sW = 4 * r ** -12 + 4 * r ** -6, 48 * r ** -12 + 24 * r ** -6
    assert abs(pe - V) <= 1e-12 * sV
    assert abs(w - W) <= 1e-12 * sW
    assert abs(F[0, 2] - Fz) <= 1e-12 * sW / r and abs(F[1, 2] + Fz) <= 1e-12 * sW / r
    assert np.sign(F[0, 2]) == np.sign(Fz) or abs(Fz) < 1e-12 * sW


def test_seeded_run_matches_reference_rows(golden):
    """From the seeded init, steps 1..49 reproduce the reference's thermodynamics.csv
    (before the first temperature rescale at step 50)."""
    x, v, L = ljref.initial_state(500, 0.5, 0.8, 117208264)
    with gpu_system(500, L) as g:
        g.upload(x, v=v)
        th = g.step(49)
    head = golden["thermo_head"][:49]
    assert np.array_equal(th[:, 0], head[:, 1])  # time accumulates t += dt exactly
    rel = np.abs(th[:, 1:7] - head[:, 2:8]) / np.abs(head[:, 2:8])
    assert rel.max() < 1e-12


def test_trajectory_vs_oracle():
    """N = 864 (4*6^3, rho 0.8442, T 0.722): 100 steps; chaos amplifies only summation-order rounding."""
    x, v, L = ljref.initial_state(864, 0.722, 0.8442, 5489)
    ref = ljref.State(x, v=v)
    rth = ljref.run_steps(ref, L, 0.005, 100)
    with gpu_system(864, L) as g:
        g.upload(x, v=v)
        th = g.step(100)
        st = g.download()
        stats = g.stats()
    rel = np.abs(th[:, 1:] - rth[:, 1:]) / np.abs(rth[:, 1:])
    assert rel.max() < 1e-9
    assert np.abs(st["x"] - ref.x).max() < 1e-10
    assert 1 <= stats["list_builds"] < 100  # the skin criterion skips most rebuilds


def test_energy_conservation_fp64():
    """N = 864 for 2000 steps.  Melting from the FCC lattice raises TE by ~1e-3 in the
    first ~200 steps in the reference algorithm too (the oracle shows the same
    transient); after it, TE is flat and the GPU's trace follows the oracle's."""
    x, v, L = ljref.initial_state(864, 0.722, 0.8442, 5489)
    ref = ljref.State(x, v=v)
    rte = ljref.run_steps(ref, L, 0.005, 2000)[:, 3]
    with gpu_system(864, L) as g:
        g.upload(x, v=v)
        th = g.step(2000)
    te = th[:, 3]
    E = abs(te[0])
    assert np.abs(te[-200:].mean() - te[400:600].mean()) / E < 2e-4
    assert abs(te[-500:].mean() - rte[-500:].mean()) / E < 2e-4
    assert np.abs(te[:200] - rte[:200]).max() / E < 1e-9


def test_set_temperature_and_scale():
    x, v, L = ljref.initial_state(864, 0.722, 0.8442, 5489)
    with gpu_system(864, L) as g:
        g.upload(x, v=v)
        g.step(10)
        T0 = g.measure()[5]
        measured = g.set_temperature(1.5)
        assert measured == pytest.approx(T0, rel=1e-15)
        assert g.measure()[5] == pytest.approx(1.5, rel=1e-14)
        g.scale_velocities(2.0)
        assert g.measure()[5] == pytest.approx(6.0, rel=1e-14)


def test_upload_download_roundtrip():
    rng = np.random.default_rng(1)
    N = 3000
    arrs = [rng.random((N, 3)) * 14.0 for _ in range(4)]
    with gpu_system(N, 14.0) as g:
        g.upload(*arrs, t=1.25, pe=-3.0, virial=2.0)
        g.compute_forces()  # re-sorts the atoms on the device
        st = g.download()
    assert np.array_equal(st["x"][:, :3], arrs[0])
    assert np.array_equal(st["v"][:, :3], arrs[1])
    assert np.array_equal(st["d"][:, :3], arrs[2])
    assert st["t"] == 1.25


@pytest.mark.parametrize("N,rho,rmax", [(864, 0.8442, 4.0), (4000, 0.8, 4.0), (2048, 0.3, 5.0)])
def test_rdf_bit_exact(N, rho, rmax):
    x, _, L = perturbed_fcc(N, 1.0, rho, 11, amp=0.3)
    rmax = min(rmax, L / 2)
    with gpu_system(N, L) as g:
        g.upload(x)
        h = g.rdf(200, rmax)
    assert np.array_equal(h, ljref.rdf(x, L, 200, rmax))


def test_rdf_accumulates_on_the_device():
    """Samples added on the device along a run equal the sum of single-sample
    histograms of the same positions, each bit-exact with the oracle; a sample
    with other bins is refused until a reset."""
    from lennardjonesium._native import LJError
    x, v, L = ljref.initial_state(4000, 1.2, 0.8, 7)
    with gpu_system(4000, L) as g:
        g.upload(x, v=v)
        total = np.zeros(150, dtype=np.uint64)
        for k in range(4):
            g.step(25, record=False)
            g.rdf_accumulate(150, 4.0)
            h = g.rdf(150, 4.0)  # a single sample leaves the accumulation alone
            assert np.array_equal(h, ljref.rdf(g.download()["x"], L, 150, 4.0))
            total += h
        acc, n = g.rdf_read()
        assert n == 4 and np.array_equal(acc, total)
        with pytest.raises(LJError):
            g.rdf_accumulate(100, 4.0)
        g.rdf_reset()
        g.rdf_accumulate(100, 4.0)
        acc, n = g.rdf_read()
        assert n == 1 and np.array_equal(acc, g.rdf(100, 4.0))


@pytest.mark.parametrize("per_pair", [False, True])
def test_mixed_precision_force_error(per_pair):
    """Mixed path (FP32 pair arithmetic) vs FP64: stated bounds, with 8-pair FP32
    sums into the FP64 accumulators and with every pair added in FP64."""
    x, v, L = perturbed_fcc(4000, 1.2, 0.8, 7)
    with gpu_system(4000, L) as g:
        g.upload(x)
        pe64, w64 = g.compute_forces()
        F64 = g.download()["F"]
    with gpu_system(4000, L, precision="mixed", mixed_per_pair=per_pair) as g:
        g.upload(x)
        pe32, w32 = g.compute_forces()
        F32 = g.download()["F"]
    # stated bounds: per-atom error <= 1e-5 of the atom's sum of |pair force|
    # (FP32 cell-local coordinates carry ~2.4e-7 absolute rounding, which the
    # r^-13 repulsion amplifies ~13x; plus FP32 pair arithmetic and 8-neighbour
    # chunk sums), RMS error <= 2e-5 of the RMS force, PE within 1e-6 and W (a sum
    # of large terms of both signs) within 1e-5 relative
    S = ljref.force_abs_sum(x, L, 2.5)
    err = np.sqrt(np.sum((F32 - F64)[:, :3] ** 2, axis=1))
    assert np.all(err <= 1e-5 * S)
    rms = np.sqrt(np.mean(np.sum(F64[:, :3] ** 2, axis=1)))
    assert np.sqrt(np.mean(err ** 2)) / rms < 2e-5
    assert abs(pe32 - pe64) / abs(pe64) < 1e-6
    assert abs(w32 - w64) / abs(w64) < 1e-5


def test_mixed_precision_energy_drift():
    x, v, L = ljref.initial_state(864, 0.722, 0.8442, 5489)
    with gpu_system(864, L, precision="mixed") as g:
        g.upload(x, v=v)
        th = g.step(2000)
    te = th[:, 3]
    assert np.abs(te[-200:].mean() - te[200:400].mean()) / abs(te[0]) < 2e-4


def test_full_size_properties():
    """At the 1M-atom benchmark size (N = 1 048 576): size-independent properties."""
    from lennardjonesium import initial_condition
    N = 4 * 64 ** 3
    x, v, L = initial_condition(N, 1.0, 0.8442, 5489)
    with gpu_system(N, L) as g:
        g.upload(x, v=v)
        th = g.step(20)
        st = g.download()
        shape, cell_of, offsets, members = g.debug_cells()
    F = st["F"][:, :3]
    rmsF = np.sqrt(np.mean(np.sum(F ** 2, axis=1)))
    assert np.abs(F.sum(axis=0)).max() < 1e-9 * rmsF * N  # Newton's third law
    assert np.abs(st["v"][:, :3].sum(axis=0)).max() < 1e-8  # momentum stays zero
    assert list(shape) == [42, 42, 42] and offsets[-1] == N
    assert np.array_equal(np.sort(members), np.arange(N))
    assert np.all(np.diff(offsets) >= 0)
    te = th[:, 3]
    assert np.abs(te - te[0]).max() / abs(te[0]) < 5e-4  # lattice-melting transient only
    assert np.all(np.isfinite(th))
    # full-size single-step parity: forces at the step-20 positions vs the oracle
    Fref, pe, w = ljref.forces(st["x"], L, 2.5)
    S = ljref.force_abs_sum(st["x"], L, 2.5)
    assert_forces(st["F"], Fref, S)
    assert st["pe"] == pytest.approx(pe, rel=1e-12) and st["virial"] == pytest.approx(w, rel=1e-12)


def test_full_size_pair_set_checksums():
    """Bit-exact pair set at N = 1 048 576, compared through order-free checksums
    (count, sums of ids, of id products and of the r^2 bit patterns)."""
    from lennardjonesium import initial_condition
    N = 4 * 64 ** 3
    x, v, L = initial_condition(N, 1.0, 0.8442, 5489)
    with gpu_system(N, L) as g:
        g.upload(x, v=v)
        g.step(30)
        x = g.download()["x"]
        gi, gj, gc, gr = g.debug_pairs()
    pi, pj, pc, pr = ljref.pairs(x, L, 2.5)
    swap = pi > pj
    oi, oj = np.where(swap, pj, pi), np.where(swap, pi, pj)
    oc = np.where(swap, 26 - pc, pc)

    def sums(i, j, c, r2):
        i = i.astype(np.uint64)
        j = j.astype(np.uint64)
        return (len(i), int(i.sum()), int(j.sum()), int((i * np.uint64(N) + j).sum()),
                int((c.astype(np.uint64) * (i + np.uint64(7))).sum()), int(r2.view(np.uint64).sum()))
    assert sums(gi, gj, gc, gr) == sums(oi, oj, oc, pr)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_steps_equal_direct_launches(precision):
    """Steps run as CUDA graphs (conditional rebuild node) and steps launched one
    kernel at a time give bit-identical records and state: every reduction has a
    fixed order and the within-cell order is deterministic."""
    x, v, L = ljref.initial_state(4000, 1.2, 0.8, 7)
    with gpu_system(4000, L, precision=precision) as a, gpu_system(4000, L, precision=precision) as b:
        a.upload(x, v=v)
        b.upload(x, v=v)
        ra = a.step(72)           # two launches of the 32-step graph, one of the 8-step graph
        b.step_timed(72)          # direct launches with per-phase events
        rb = b.step(1)            # one more step on both to compare a record
        ra1 = a.step(1)
        sa, sb = a.download(), b.download()
        assert a.stats()["list_builds"] == b.stats()["list_builds"]
    assert np.array_equal(ra1, rb)
    for k in ("x", "v", "d", "F"):
        assert np.array_equal(sa[k], sb[k]), k
    assert np.all(np.isfinite(ra))


@pytest.mark.parametrize("skin,block,precision", [(0.15, 64, "fp64"), (0.5, 256, "fp64"), (0.7, 128, "fp64"), (0.4, 64, "mixed")])
def test_tuning_parameters_keep_parity(skin, block, precision):
    """Every autotuner candidate computes the same physics: bit-exact pair sets and
    FP64 forces within the parity tolerance at other skins and block sizes."""
    N, T, rho, seed, rc = FCC_CASES[3]
    x, v, L = perturbed_fcc(N, T, rho, seed)
    with gpu_system(N, L, skin=skin, force_block=block, precision=precision) as g:
        g.upload(x)
        assert pair_key(*g.debug_pairs()) == oracle_pair_key(x, L, rc)
        pe, w = g.compute_forces()
        F = g.download()["F"]
        g.upload(x, v=v)
        th = g.step(50)
    Fref, pe_ref, w_ref = ljref.forces(x, L, rc)
    if precision == "fp64":
        assert_forces(F, Fref, ljref.force_abs_sum(x, L, rc))
        assert pe == pytest.approx(pe_ref, rel=1e-12)
    assert np.all(np.isfinite(th))


def test_autotune_returns_a_candidate():
    from lennardjonesium import autotune
    x, v, L = ljref.initial_state(4000, 1.2, 0.8, 7)
    kw, ms = autotune(4000, L, x, v, steps=24)
    assert kw["force_block"] in (64, 128, 256) and 0.0 <= kw["skin"] <= 0.7 and ms > 0


@pytest.mark.parametrize("per_pair", [False, True])
def test_mixed_full_size_force_error(per_pair):
    """N = 1 048 576 (4 * 64^3 FCC, rho = 0.8442, perturbed): the mixed forces
    against the FP64 path (itself at 1e-12 of the oracle), both accumulation modes."""
    from lennardjonesium import initial_condition
    N = 4 * 64 ** 3
    x, v, L = initial_condition(N, 1.0, 0.8442, 5489)
    rng = np.random.default_rng(5489)
    x[:, :3] = np.mod(x[:, :3] + 0.08 * rng.standard_normal((N, 3)), L)
    with gpu_system(N, L) as g:
        g.upload(x)
        pe64, w64 = g.compute_forces()
        F64 = g.download()["F"]
    with gpu_system(N, L, precision="mixed", mixed_per_pair=per_pair) as g:
        g.upload(x)
        pe32, w32 = g.compute_forces()
        F32 = g.download()["F"]
    S = ljref.force_abs_sum(x, L, 2.5)
    err = np.sqrt(np.sum((F32 - F64)[:, :3] ** 2, axis=1))
    assert np.all(err <= 1e-5 * S)
    rms = np.sqrt(np.mean(np.sum(F64[:, :3] ** 2, axis=1)))
    assert np.sqrt(np.mean(err ** 2)) / rms < 2e-5
    assert abs(pe32 - pe64) / abs(pe64) < 1e-6
    assert abs(w32 - w64) / abs(w64) < 1e-5


def _anisotropic_lattice(n=(12, 16, 24), a=1.0772, amp=0.1, seed=12):
    """A perturbed simple-cubic lattice in an anisotropic box (rho ~ 0.8)."""
    g = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), axis=-1).reshape(-1, 3)
    L = np.array(n, dtype=float) * a
    rng = np.random.default_rng(seed)
    x = np.mod((g + 0.5) * a + rng.uniform(-amp, amp, size=g.shape), L)
    return x, L


def test_anisotropic_box_both_paths_and_rdf():
    """An anisotropic box of 4608 atoms (12 x 16 x 24 cells of the lattice): the
    FP64 pair set bit-exact and forces at 1e-12, the mixed path within its
    bounds, the RDF bit-exact, all against the oracle."""
    x, L = _anisotropic_lattice()
    N = x.shape[0]
    with gpu_system(N, L) as g:
        g.upload(x)
        assert pair_key(*g.debug_pairs()) == oracle_pair_key(x, L, 2.5)
        pe64, w64 = g.compute_forces()
        F64 = g.download()["F"]
        h = g.rdf(160, 4.0)
    Fref, pe, w = ljref.forces(x, L, 2.5)
    S = ljref.force_abs_sum(x, L, 2.5)
    assert_forces(F64, Fref, S)
    assert pe64 == pytest.approx(pe, rel=1e-12) and w64 == pytest.approx(w, rel=1e-12)
    assert np.array_equal(h, ljref.rdf(x, L, 160, 4.0))
    with gpu_system(N, L, precision="mixed") as g:
        g.upload(x)
        pe32, w32 = g.compute_forces()
        F32 = g.download()["F"]
    err = np.sqrt(np.sum((F32 - F64)[:, :3] ** 2, axis=1))
    assert np.all(err <= 1e-5 * S)
    assert abs(pe32 - pe64) / abs(pe64) < 1e-6 and abs(w32 - w64) / abs(w64) < 1e-5


def test_measurement_rotating_cube():
    """physics/test_measurements.cpp: four atoms on a cube rotating about z,
    KE = 4 and T = (8/3) / 4, measured on the GPU (no force calculation)."""
    x = np.array([[0, 0, 0], [0, 0, 2], [2, 2, 0], [2, 2, 2]], dtype=float)
    v = np.array([[1, -1, 0], [1, -1, 0], [-1, 1, 0], [-1, 1, 0]], dtype=float)
    with gpu_system(4, 10.0, force="none", periodic=False) as g:
        g.upload(x, v=v)
        m = g.measure()
    assert m[1] == 4.0 and m[5] == pytest.approx(8 / 3 / 4, rel=1e-15)
    assert m[2] == 0.0 and m[4] == 0.0 and m[6] == 0.0
