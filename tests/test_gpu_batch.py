"""The batched engine (lj_batch_*) against single-system runs.

Every block and every cell of the batched launch belongs to one system, the
rebuilds are gated per system and the reductions follow the single-system
order, so a batched run must reproduce each system run alone bit for bit.
"""

import ctypes
import filecmp
import pathlib

import numpy as np
import pytest

import ljref

pytestmark = pytest.mark.gpu

SYSTEMS = [  # N, T, rho, seed: uneven sizes and densities (each box >= 3 cutoffs)
    (500, 0.5, 0.8, 117208264),
    (864, 0.722, 0.8442, 5489),
    (2048, 1.5, 0.3, 3),
    (4000, 1.2, 0.8, 7),
    (4 * 9 ** 3, 2.0, 0.05, 11),
]


def _table(states, L, skin=-1.0):
    from lennardjonesium import _native as nat
    n = len(states)
    systems = (nat.BatchSystem * n)()
    for s, ((x, v), box) in enumerate(zip(states, L)):
        systems[s].particle_count = x.shape[0]
        for k in range(3):
            systems[s].box[k] = box
        systems[s].time_delta = 0.005
        systems[s].skin = skin
    return systems


def _batch(states, L, skin=-1.0, force_block=0, list_tile=0):
    from lennardjonesium import _native as nat
    lib = nat.lib()
    n = len(states)
    systems = _table(states, L, skin)
    b = ctypes.c_void_p()
    nat.check(lib.lj_batch_create(systems, n, 2.5, 0, ctypes.byref(b)))
    if force_block:
        nat.check(lib.lj_batch_set_force_block(b, force_block))
    if list_tile:
        nat.check(lib.lj_batch_set_list_tile(b, list_tile))
    for s, (x, v) in enumerate(states):
        nat.check(lib.lj_batch_upload_system(b, s, x.ctypes.data_as(ctypes.c_void_p),
                                             v.ctypes.data_as(ctypes.c_void_p), 4))
    return lib, b


def _download(lib, b, s, N):
    x, v, F = (np.zeros((N, 4)) for _ in range(3))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.lj_batch_download_system(b, s, P(x), P(v), P(F), 4) == 0
    return x, v, F


def test_batch_equals_single_systems():
    from lennardjonesium import GpuSystem
    states, L = [], []
    for N, T, rho, seed in SYSTEMS:
        x, v, box = ljref.initial_state(N, T, rho, seed)
        states.append((x, v))
        L.append(box)
    lib, b = _batch(states, L)
    steps = 203  # graph chunks of 8 plus a remainder
    recs = np.zeros((steps, len(SYSTEMS), 7))
    assert lib.lj_batch_step(b, steps, recs.ctypes.data_as(ctypes.c_void_p)) == 0
    builds = (ctypes.c_longlong * len(SYSTEMS))()
    lib.lj_batch_info(b, None, builds, None)
    for s, ((x, v), box) in enumerate(zip(states, L)):
        with GpuSystem(x.shape[0], box) as g:
            g.upload(x, v=v)
            ref = g.step(steps)
            st = g.download()
            assert g.stats()["list_builds"] == builds[s]
        assert np.array_equal(recs[:, s, :], ref), f"system {s}"
        bx, bv, bF = _download(lib, b, s, x.shape[0])
        assert np.array_equal(bx, st["x"]) and np.array_equal(bv, st["v"]) and np.array_equal(bF, st["F"])
    lib.lj_batch_destroy(b)


def test_batch_set_temperature_and_inactive():
    states, L = [], []
    for N, T, rho, seed in SYSTEMS[:3]:
        x, v, box = ljref.initial_state(N, T, rho, seed)
        states.append((x, v))
        L.append(box)
    lib, b = _batch(states, L)
    recs = np.zeros((20, 3, 7))
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.lj_batch_step(b, 20, P(recs)) == 0
    measured = ctypes.c_double()
    assert lib.lj_batch_set_temperature(b, 1, 1.7, ctypes.byref(measured)) == 0
    assert measured.value == pytest.approx(recs[-1, 1, 5], rel=1e-14)
    m = np.zeros((3, 7))
    assert lib.lj_batch_measure(b, P(m)) == 0
    assert m[1, 5] == pytest.approx(1.7, rel=1e-14)
    frozen = _download(lib, b, 2, states[2][0].shape[0])
    assert lib.lj_batch_set_active(b, 2, 0) == 0
    assert lib.lj_batch_step(b, 16, P(np.zeros((16, 3, 7)))) == 0
    after = _download(lib, b, 2, states[2][0].shape[0])
    assert all(np.array_equal(p, q) for p, q in zip(frozen, after))
    lib.lj_batch_destroy(b)


def test_run_sweep_batched_equals_thread_pool(tmp_path):
    """The batched sweep writes byte-identical files to the one-context-per-run path."""
    import lennardjonesium as lj
    sc = lj.SweepConfiguration()
    sc.system.temperature_start, sc.system.temperature_stop, sc.system.temperature_steps = 0.7, 1.5, 3
    sc.system.density_start, sc.system.density_stop, sc.system.density_steps = 0.3, 0.9, 3
    sc.system.particle_count = 500
    sc.equilibration.adjustment_interval, sc.equilibration.steady_state_time = 50, 150
    sc.equilibration.timeout, sc.equilibration.tolerance = 1000, 0.05
    sc.observation.observation_interval, sc.observation.observation_count = 50, 4
    sc.observation.tolerance = 0.3
    runs = {}
    for mode in ("batched", "pool"):
        d = tmp_path / mode
        runs[mode] = lj.run_sweep(d / "sweep.ini", echo_status=False, thread_count=3, random_seed=29,
                                  sweep_config_object=sc, batched=(mode == "batched"))
    for t, rho in sc.sweep_range():
        sub = sc.simulation_dir(t, rho)
        for name in ("events.log", "thermodynamics.csv", "observations.csv", "snapshots.csv"):
            a, p = tmp_path / "batched" / sub / name, tmp_path / "pool" / sub / name
            assert filecmp.cmp(a, p, shallow=False), f"{sub}/{name}"
    assert len(runs["batched"].completed) == len(runs["pool"].completed)


def _host_stats(records, N, rho):
    from lennardjonesium import _native as nat
    r = np.ascontiguousarray(records, dtype=np.float64)
    o = nat.Observation()
    assert nat.lib().lj_window_stats_host(r.ctypes.data_as(ctypes.c_void_p), r.shape[0], N, rho,
                                          ctypes.byref(o)) == 0
    return np.array([getattr(o, f) for f, _ in o._fields_])


def test_batch_window_statistics_on_device():
    """ThermodynamicAnalyzer results of 64 systems computed on the device from the
    batch's record ring equal the host restatement over the same records to 1e-12."""
    from lennardjonesium import _native as nat
    rng = np.random.default_rng(64)
    states, L, sizes, rhos = [], [], [], []
    for k in range(64):
        n = int(rng.integers(5, 9))
        rho = float(rng.uniform(0.3, 1.0))
        x, v, box = ljref.initial_state(4 * n ** 3, float(rng.uniform(0.5, 2.0)), rho, 100 + k)
        states.append((x, v))
        L.append(box)
        sizes.append(4 * n ** 3)
        rhos.append(rho)
    lib, b = _batch(states, L)
    try:
        W = 200
        recs = np.zeros((250, 64, 7))
        assert lib.lj_batch_step(b, 250, recs.ctypes.data_as(ctypes.c_void_p)) == 0
        obs = (nat.Observation * 64)()
        dens = np.array(rhos)
        assert lib.lj_batch_window_stats(b, W, dens.ctypes.data_as(ctypes.c_void_p), obs) == 0
        assert lib.lj_batch_window_stats(b, 300, dens.ctypes.data_as(ctypes.c_void_p), obs) == nat.LJ_ERR_ARG
        assert lib.lj_batch_window_stats(b, W, dens.ctypes.data_as(ctypes.c_void_p), obs) == 0
    finally:
        lib.lj_batch_destroy(b)
    for s in range(64):
        want = _host_stats(recs[-W:, s, :], sizes[s], rhos[s])
        got = np.array([getattr(obs[s], f) for f, _ in obs[s]._fields_])
        assert np.all(np.abs(got - want) <= 1e-12 * np.abs(want)), (s, got, want)


def test_context_window_statistics_on_device():
    from lennardjonesium import GpuSystem
    from lennardjonesium import _native as nat
    x, v, L = ljref.initial_state(4000, 1.2, 0.8, 7)
    with GpuSystem(4000, L) as g:
        g.upload(x, v=v)
        recs = g.step(1300)  # the ring holds the last 1024 records
        o = nat.Observation()
        for W in (2, 500, 1024):
            assert nat.lib().lj_gpu_window_stats(g._ctx, W, 0.8, ctypes.byref(o)) == 0
            got = np.array([getattr(o, f) for f, _ in o._fields_])
            want = _host_stats(recs[-W:], 4000, 0.8)
            assert np.all(np.abs(got - want) <= 1e-12 * np.abs(want)), (W, got, want)
        assert nat.lib().lj_gpu_window_stats(g._ctx, 1025, 0.8, ctypes.byref(o)) == nat.LJ_ERR_ARG


def test_window_stats_through_the_python_api():
    """GpuSystem.window_stats (device) equals window_stats_host over the records
    step() returned, to 1e-12."""
    from lennardjonesium import GpuSystem, window_stats_host
    x, v, L = ljref.initial_state(4000, 1.2, 0.8, 7)
    with GpuSystem(4000, L) as g:
        g.upload(x, v=v)
        recs = g.step(600)
        dev = g.window_stats(500, 0.8)
    host = window_stats_host(recs[-500:], 4000, 0.8)
    assert dev.keys() == host.keys()
    for k in host:
        assert abs(dev[k] - host[k]) <= 1e-12 * abs(host[k]), (k, dev[k], host[k])


def test_batch_chunk_loop_bound():
    """A chunk launch runs its device-side loop under an iteration bound: with the
    bound set below the chunk's 8 iterations the launch stops early and the call
    returns LJ_ERR_TIMEOUT; with the default bound the same batch steps on, and
    its records then equal a single-system run of the steps it really took."""
    from lennardjonesium import GpuSystem
    from lennardjonesium import _native as nat
    N, T, rho, seed = SYSTEMS[1]
    x, v, box = ljref.initial_state(N, T, rho, seed)
    lib, b = _batch([(x, v)], [box])
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    try:
        assert lib.lj_batch_set_iteration_limit(b, 3) == 0
        assert lib.lj_batch_step(b, 64, None) == nat.LJ_ERR_TIMEOUT
        assert b"iteration bound" in lib.lj_batch_last_error(b)
        assert lib.lj_batch_set_iteration_limit(b, 0) == 0
        assert lib.lj_batch_upload_system(b, 0, P(x), P(v), 4) == 0
        recs = np.zeros((64, 1, 7))
        assert lib.lj_batch_step(b, 64, P(recs)) == 0
    finally:
        lib.lj_batch_destroy(b)
    with GpuSystem(N, box) as g:
        g.upload(x, v=v)
        ref = g.step(64)
    assert np.array_equal(recs[:, 0, :], ref)


@pytest.mark.parametrize("skin,block,tile", [(0.4, 64, 2), (0.2, 256, 8)])
def test_tuned_batch_equals_single_systems(skin, block, tile):
    """A batch run with another skin, pair-kernel block size and list-build tile
    (autotuner candidates) equals single-system runs with the same skin and
    block size bit for bit."""
    from lennardjonesium import GpuSystem
    states, L = [], []
    for N, T, rho, seed in SYSTEMS[:4]:
        x, v, box = ljref.initial_state(N, T, rho, seed)
        states.append((x, v))
        L.append(box)
    lib, b = _batch(states, L, skin=skin, force_block=block, list_tile=tile)
    recs = np.zeros((90, len(states), 7))
    try:
        assert lib.lj_batch_step(b, 90, recs.ctypes.data_as(ctypes.c_void_p)) == 0
    finally:
        lib.lj_batch_destroy(b)
    for s, ((x, v), box) in enumerate(zip(states, L)):
        with GpuSystem(x.shape[0], box, skin=skin, force_block=block) as g:
            g.upload(x, v=v)
            ref = g.step(90)
        assert np.array_equal(recs[:, s, :], ref), f"system {s}"


def test_batch_autotune_returns_a_candidate():
    from lennardjonesium import _native as nat
    states, L = [], []
    for N, T, rho, seed in SYSTEMS[:3]:
        x, v, box = ljref.initial_state(N, T, rho, seed)
        states.append((x, v))
        L.append(box)
    x = np.concatenate([a for a, _ in states])
    v = np.concatenate([b for _, b in states])
    best = nat.BatchTuning()
    rc = nat.lib().lj_batch_autotune(_table(states, L), len(states), 2.5, 0, x.ctypes.data_as(ctypes.c_void_p),
                                     v.ctypes.data_as(ctypes.c_void_p), 4, 16, ctypes.byref(best))
    assert rc == 0
    assert best.skin in (0.2, 0.3, 0.4, 0.5) and best.force_block in (64, 128, 256) and best.ms_per_step > 0
    assert best.list_cells_per_block in (2, 4, 8)


def test_batch_anisotropic_system_equals_single():
    """A batch holding an anisotropic box beside a cubic one: each system evolves
    bit for bit as it does alone."""
    from lennardjonesium import GpuSystem
    from lennardjonesium import _native as nat
    rng = np.random.default_rng(21)
    n = (8, 10, 13)
    a = 1.0772
    g = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), axis=-1).reshape(-1, 3)
    La = np.array(n, dtype=float) * a
    xa = np.zeros((g.shape[0], 4))
    xa[:, :3] = np.mod((g + 0.5) * a + rng.uniform(-0.1, 0.1, size=g.shape), La)
    va = np.zeros_like(xa)
    va[:, :3] = rng.normal(0.0, 1.0, size=(g.shape[0], 3))
    va[:, :3] -= va[:, :3].mean(axis=0)
    xc, vc, Lc = ljref.initial_state(864, 0.722, 0.8442, 5489)
    systems = (nat.BatchSystem * 2)()
    for s, (x, box) in enumerate(((xa, La), (xc, np.full(3, Lc)))):
        systems[s].particle_count = x.shape[0]
        for k in range(3):
            systems[s].box[k] = box[k]
        systems[s].time_delta = 0.005
        systems[s].skin = -1.0
    lib = nat.lib()
    b = ctypes.c_void_p()
    nat.check(lib.lj_batch_create(systems, 2, 2.5, 0, ctypes.byref(b)))
    P = lambda q: q.ctypes.data_as(ctypes.c_void_p)
    recs = np.zeros((120, 2, 7))
    try:
        for s, (x, v) in enumerate(((xa, va), (xc, vc))):
            nat.check(lib.lj_batch_upload_system(b, s, P(x), P(v), 4))
        assert lib.lj_batch_step(b, 120, P(recs)) == 0
    finally:
        lib.lj_batch_destroy(b)
    for s, (x, v, box) in enumerate(((xa, va, La), (xc, vc, Lc))):
        with GpuSystem(x.shape[0], box) as gs:
            gs.upload(x, v=v)
            ref = gs.step(120)
        assert np.array_equal(recs[:, s, :], ref), f"system {s}"
