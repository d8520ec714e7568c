"""Python face of the GPU engine: one system on one GPU behind the C ABI.

``GpuSystem`` mirrors the reference's engine plugin points
(src/cpp/lennardjonesium/engine/integrator.hpp:34-102 and
force_calculation.hpp:63-79): ``step`` is ``Integrator::operator()(n)``
followed by a ``ThermodynamicMeasurement`` per step, ``compute_forces`` is
``ShortRangeForceCalculation::operator()``.  State arrays are numpy (N, 3)
or (N, 4) float64 in atom-id order, as the reference's ``SystemState``.
"""

import ctypes

import numpy as np

from lennardjonesium import _native as nat

THERMO_FIELDS = ("time", "kinetic_energy", "potential_energy", "total_energy", "virial",
                 "temperature", "mean_square_displacement")


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _as4(a, N):
    if a is None:
        return None
    a = np.asarray(a, dtype=np.float64)
    if a.shape != (N, 3) and a.shape != (N, 4):
        raise ValueError(f"expected shape ({N}, 3) or ({N}, 4), got {a.shape}")
    out = np.zeros((N, 4))
    out[:, :3] = a[:, :3]
    return out


def window_stats_host(records, particle_count, density):
    """The same analysis as GpuSystem.window_stats on records the caller holds
    ((n, 7) step records, oldest first), in the reference's summation order."""
    r = np.ascontiguousarray(records, dtype=np.float64)
    o = nat.Observation()
    nat.check(nat.lib().lj_window_stats_host(_p(r), r.shape[0], int(particle_count), float(density),
                                             ctypes.byref(o)))
    return {f: getattr(o, f) for f, _ in o._fields_}


def lattice_side(N, density):
    """Edge of the cubic box engine::InitialCondition builds (tools/cubic_lattice.cpp:43-58)."""
    import math
    cells = math.ceil(N / 4)
    per_side = math.ceil(round(cells ** (1 / 3), 12))
    return per_side * ((N / per_side ** 3) / density) ** (1 / 3)


def initial_condition(N, temperature, density, seed):
    """engine::InitialCondition: FCC positions, seeded MB velocities (N, 4), box edge."""
    x = np.zeros((N, 4))
    v = np.zeros((N, 4))
    side = np.zeros(1)
    nat.check(nat.lib().lj_initial_condition(N, temperature, density, seed, _p(x), _p(v), _p(side)))
    return x, v, float(side[0])


def autotune(N, box, x, v, steps=100, **kw):
    """Project autotuner (lj_gpu_autotune): the fastest (skin, force_block) for
    this system and state, as GpuSystem keyword arguments, plus its ms per step."""
    base = _params(N, box, **kw)
    best = nat.Params()
    ms = ctypes.c_double()
    xs, vs = _as4(x, N), _as4(v, N) if v is not None else None
    nat.check(nat.lib().lj_gpu_autotune(ctypes.byref(base), _p(xs), _p(vs), 4, int(steps), ctypes.byref(best),
                                        ctypes.byref(ms)))
    return {"skin": best.skin, "force_block": best.force_block,
            "mixed_per_pair": bool(best.mixed_per_pair)}, ms.value


def _params(N, box, cutoff=2.5, dt=0.005, precision="fp64", force="lj", strength=0.0, periodic=True, device=0,
            skin=None, capacity=0, force_block=0, mixed_per_pair=False):
    L = nat.lib()
    p = nat.Params()
    L.lj_gpu_default_params(ctypes.byref(p))
    p.particle_count = int(N)
    b = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,))
    for k in range(3):
        p.box[k] = float(b[k])
    p.cutoff_distance = float(cutoff)
    p.time_delta = float(dt)
    p.precision = {"fp64": nat.LJ_PRECISION_FP64, "mixed": nat.LJ_PRECISION_MIXED}[precision]
    p.force_kind = {"none": nat.LJ_FORCE_NONE, "lj": nat.LJ_FORCE_LJ, "constant": nat.LJ_FORCE_CONSTANT}[force]
    p.force_strength = float(strength)
    p.periodic = 1 if periodic else 0
    p.device = int(device)
    p.skin = -1.0 if skin is None else float(skin)
    p.neighbor_capacity = int(capacity)
    p.force_block = int(force_block)
    p.mixed_per_pair = 1 if mixed_per_pair else 0
    return p


class GpuSystem:
    """One periodic LJ system resident on a GPU (a context of include/lj_gpu.h).

    N, box: atom count and box edge (a scalar or three edges); cutoff, dt: rc
    and the time step.  precision: "fp64" (the drop-in path) or "mixed" (FP32
    pair arithmetic, FP64 accumulation and integration).  force: "lj", "constant"
    (the reference's test mock, with `strength`) or "none".  skin: Verlet skin
    (None: 0.3); capacity: list entries per atom (0: density-based);
    force_block: atoms per pair-kernel block (64, 128, 256; 0: 128).  Mixed path
    only: mixed_per_pair adds every pair force in FP64 instead of FP32 sums of
    8 pairs.  Every call raises LJError on a non-zero status."""

    def __init__(self, N, box, cutoff=2.5, dt=0.005, precision="fp64", force="lj", strength=0.0,
                 periodic=True, device=0, skin=None, capacity=0, force_block=0, mixed_per_pair=False):
        L = nat.lib()
        p = _params(N, box, cutoff=cutoff, dt=dt, precision=precision, force=force, strength=strength,
                    periodic=periodic, device=device, skin=skin, capacity=capacity, force_block=force_block,
                    mixed_per_pair=mixed_per_pair)
        b = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,))
        self.N = int(N)
        self.box = b.copy()
        self.params = p
        self._ctx = ctypes.c_void_p()
        nat.check(L.lj_gpu_create(ctypes.byref(p), ctypes.byref(self._ctx)))

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self._ctx:
            nat.lib().lj_gpu_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status):
        nat.check(status, self._ctx)

    # -- state ------------------------------------------------------------
    def upload(self, x, v=None, d=None, F=None, t=0.0, pe=0.0, virial=0.0):
        N = self.N
        arrs = [_as4(a, N) for a in (x, v, d, F)]
        self._check(nat.lib().lj_gpu_upload_state(self._ctx, *[_p(a) for a in arrs], 4, t, pe, virial))

    def download(self):
        N = self.N
        x, v, d, F = (np.zeros((N, 4)) for _ in range(4))
        t, pe, w = (ctypes.c_double() for _ in range(3))
        self._check(nat.lib().lj_gpu_download_state(self._ctx, _p(x), _p(v), _p(d), _p(F), 4,
                                                    ctypes.byref(t), ctypes.byref(pe), ctypes.byref(w)))
        return dict(x=x, v=v, d=d, F=F, t=t.value, pe=pe.value, virial=w.value)

    # -- physics ------------------------------------------------------------
    def compute_forces(self):
        pe, w = ctypes.c_double(), ctypes.c_double()
        self._check(nat.lib().lj_gpu_compute_forces(self._ctx, ctypes.byref(pe), ctypes.byref(w)))
        return pe.value, w.value

    def step(self, n=1, record=True):
        out = np.zeros((n, 7)) if record else None
        self._check(nat.lib().lj_gpu_step(self._ctx, int(n), _p(out)))
        return out

    def step_async(self, n):
        """Enqueue n steps on the context's stream without waiting."""
        self._check(nat.lib().lj_gpu_step_async(self._ctx, int(n)))

    def synchronize(self):
        self._check(nat.lib().lj_gpu_synchronize(self._ctx))

    @property
    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        return nat.lib().lj_gpu_stream(self._ctx)

    def step_timed(self, n):
        """Run n steps with CUDA-event timing of each phase; returns a dict of totals."""
        t = nat.PhaseTimes()
        self._check(nat.lib().lj_gpu_step_timed(self._ctx, int(n), ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in t._fields_}

    def measure(self):
        out = np.zeros(7)
        self._check(nat.lib().lj_gpu_measure(self._ctx, _p(out)))
        return out

    def scale_velocities(self, factor):
        self._check(nat.lib().lj_gpu_scale_velocities(self._ctx, float(factor)))

    def set_temperature(self, target):
        m = ctypes.c_double()
        self._check(nat.lib().lj_gpu_set_temperature(self._ctx, float(target), ctypes.byref(m)))
        return m.value

    # -- inspection -----------------------------------------------------------
    def debug_cells(self):
        shape = np.zeros(3, dtype=np.int32)
        self._check(nat.lib().lj_gpu_debug_cells(self._ctx, _p(shape), None, None, None))
        nc = int(np.prod(shape))
        cell_of = np.zeros(self.N, dtype=np.int32)
        offsets = np.zeros(nc + 1, dtype=np.int32)
        members = np.zeros(self.N, dtype=np.int32)
        self._check(nat.lib().lj_gpu_debug_cells(self._ctx, _p(shape), _p(cell_of), _p(offsets),
                                                 _p(members)))
        return shape, cell_of, offsets, members

    def debug_pairs(self):
        L = nat.lib()
        n = L.lj_gpu_debug_pairs(self._ctx, 0, None, None, None, None)
        if n < 0:
            self._check(-n)
        i, j, img = (np.zeros(n, dtype=np.int32) for _ in range(3))
        r2 = np.zeros(n)
        m = L.lj_gpu_debug_pairs(self._ctx, n, _p(i), _p(j), _p(img), _p(r2))
        if m < 0:
            self._check(-m)
        return i, j, img, r2

    def rdf(self, nbins, rmax):
        """Histogram of the current positions (ordered pairs, nbins bins on [0, rmax))."""
        h = np.zeros(nbins, dtype=np.uint64)
        self._check(nat.lib().lj_gpu_rdf(self._ctx, int(nbins), float(rmax), _p(h)))
        return h

    def rdf_accumulate(self, nbins, rmax):
        """Add the current positions' histogram to the device accumulator, without
        waiting for it (no allocation after the first sample)."""
        self._check(nat.lib().lj_gpu_rdf_accumulate(self._ctx, int(nbins), float(rmax)))
        self._rdf_bins = int(nbins)

    def rdf_read(self):
        """(summed histogram, number of samples) of the accumulator."""
        n = ctypes.c_longlong()
        h = np.zeros(getattr(self, "_rdf_bins", 0), dtype=np.uint64)
        self._check(nat.lib().lj_gpu_rdf_read(self._ctx, _p(h) if len(h) else None, ctypes.byref(n)))
        return (h, n.value) if n.value else (np.zeros(0, dtype=np.uint64), 0)

    def rdf_reset(self):
        self._check(nat.lib().lj_gpu_rdf_reset(self._ctx))

    def trajectory_open(self, path, every):
        """Write a frame (snapshot format) every `every` steps to `path` while stepping."""
        self._check(nat.lib().lj_gpu_trajectory_open(self._ctx, str(path).encode(), int(every)))

    def trajectory_close(self):
        """Flush and close the trajectory; returns the number of frames written."""
        n = ctypes.c_longlong()
        self._check(nat.lib().lj_gpu_trajectory_close(self._ctx, ctypes.byref(n)))
        return n.value

    def window_stats(self, sample_size, density):
        """ThermodynamicAnalyzer result (physics/analyzers.cpp:44-159) over the last
        sample_size step records, computed on the device from the record ring:
        temperature, density, total_energy, pressure, specific_heat,
        diffusion_coefficient."""
        o = nat.Observation()
        self._check(nat.lib().lj_gpu_window_stats(self._ctx, int(sample_size), float(density), ctypes.byref(o)))
        return {f: getattr(o, f) for f, _ in o._fields_}

    def stats(self):
        s = nat.Stats()
        self._check(nat.lib().lj_gpu_get_stats(self._ctx, ctypes.byref(s)))
        return {f: (list(getattr(s, f)) if f == "list_cells" else getattr(s, f)) for f, _ in s._fields_}
