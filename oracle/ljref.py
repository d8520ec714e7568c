"""ctypes wrapper around the CPU oracle (``ljref.cpp``).

TEST INFRASTRUCTURE ONLY: imported by the tests, the smoke check and the CPU
baseline leg of the benchmark.  The GPU library never imports this module.

Arrays follow the reference's ``SystemState`` layout: 4 x N doubles per vector,
column-major (x0, y0, z0, 0, x1, ...), i.e. numpy shape (N, 4).
"""

import ctypes
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
FORCE_NONE, FORCE_LJ, FORCE_CONSTANT = 0, 1, 2

_libs = {}


def build():
    """Compile both oracle variants with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib(fast=False):
    name = "libljref_fast.so" if fast else "libljref.so"
    if name not in _libs:
        path = HERE / "build" / name
        if not path.exists():
            build()
        L = ctypes.CDLL(str(path))
        d, i, u, ll = ctypes.c_double, ctypes.c_int, ctypes.c_uint, ctypes.c_longlong
        P = ctypes.c_void_p
        L.ljref_pair_along_z.argtypes = [i, d, d, d, P]
        L.ljref_spline.argtypes = [d, P]
        L.ljref_initial_state.argtypes = [i, d, d, u, P, P, P]
        L.ljref_cell_shape.argtypes = [P, d, P]
        L.ljref_bin.argtypes = [i, P, i, P, d, P, P, P]
        L.ljref_pairs.argtypes = [i, i, P, i, P, d, ll, P, P, P, P]
        L.ljref_pairs.restype = ll
        L.ljref_forces.argtypes = [i, P, P, i, d, d, P, P, P]
        L.ljref_force_abs_sum.argtypes = [i, P, P, d, P]
        L.ljref_run_steps.argtypes = [i, P, P, P, P, P, P, P, P, d, i, i, d, d, i, P]
        L.ljref_set_temperature.argtypes = [i, P, d]
        L.ljref_rdf.argtypes = [i, P, i, P, i, d, P]
        L.ljref_rdf_cells.argtypes = [i, P, i, P, i, d, i, P]
        L.ljref_simulate.argtypes = [P, ll, P, P, i, P]
        L.ljref_simulate.restype = ll
        L.ljref_bench.argtypes = [i, d, d, u, d, d, i, i, i, P]
        _libs[name] = L
    return _libs[name]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _box(L):
    b = np.ascontiguousarray(np.broadcast_to(np.asarray(L, dtype=np.float64), (3,)))
    return b


def as4(x):
    """(N, 3) or (N, 4) -> contiguous (N, 4) float64 with a zero 4th column."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros((x.shape[0], 4))
    out[:, :3] = x[:, :3]
    return out


def pair_along_z(r, rc=2.5, kind=FORCE_LJ, strength=0.0):
    out = np.zeros(3)
    lib().ljref_pair_along_z(kind, rc, strength, r, _p(out))
    return out  # V, W, Fz


def spline(rc):
    out = np.zeros(2)
    lib().ljref_spline(rc, _p(out))
    return out


def initial_state(N, T, density, seed):
    x = np.zeros((N, 4))
    v = np.zeros((N, 4))
    side = np.zeros(1)
    rc = lib().ljref_initial_state(N, T, density, seed, _p(x), _p(v), _p(side))
    assert rc == 0
    return x, v, float(side[0])


def cell_shape(L, rc):
    s = np.zeros(3, dtype=np.int32)
    lib().ljref_cell_shape(_p(_box(L)), rc, _p(s))
    return s


def bin_atoms(x, L, rc):
    x = as4(x)
    N = x.shape[0]
    shape = cell_shape(L, rc)
    nc = int(np.prod(shape))
    cell_of = np.zeros(N, dtype=np.int32)
    offsets = np.zeros(nc + 1, dtype=np.int32)
    members = np.zeros(N, dtype=np.int32)
    lib().ljref_bin(N, _p(x), 4, _p(_box(L)), rc, _p(cell_of), _p(offsets), _p(members))
    return cell_of, offsets, members


def pairs(x, L, rc, naive=False):
    """Reference pair set as arrays (i, j, image_code, r2), in the reference's order."""
    x = as4(x)
    N = x.shape[0]
    box = _box(L)
    n = lib().ljref_pairs(1 if naive else 0, N, _p(x), 4, _p(box), rc, 0, None, None, None, None)
    pi = np.zeros(n, dtype=np.int32)
    pj = np.zeros(n, dtype=np.int32)
    pc = np.zeros(n, dtype=np.int32)
    pr = np.zeros(n)
    lib().ljref_pairs(1 if naive else 0, N, _p(x), 4, _p(box), rc, n, _p(pi), _p(pj), _p(pc), _p(pr))
    return pi, pj, pc, pr


def forces(x, L, rc=2.5, kind=FORCE_LJ, strength=0.0):
    x = as4(x)
    N = x.shape[0]
    F = np.zeros((N, 4))
    pe = np.zeros(1)
    w = np.zeros(1)
    lib().ljref_forces(N, _p(x), _p(_box(L)), kind, rc, strength, _p(F), _p(pe), _p(w))
    return F, float(pe[0]), float(w[0])


def force_abs_sum(x, L, rc=2.5):
    x = as4(x)
    out = np.zeros(x.shape[0])
    lib().ljref_force_abs_sum(x.shape[0], _p(x), _p(_box(L)), rc, _p(out))
    return out


class State:
    """Mutable 4 x N state mirroring the reference's SystemState."""

    def __init__(self, x, v=None, d=None, F=None, t=0.0, pe=0.0, vir=0.0):
        self.x = as4(x)
        N = self.x.shape[0]
        self.v = as4(v) if v is not None else np.zeros((N, 4))
        self.d = as4(d) if d is not None else np.zeros((N, 4))
        self.F = as4(F) if F is not None else np.zeros((N, 4))
        self.t, self.pe, self.vir = t, pe, vir

    @property
    def N(self):
        return self.x.shape[0]


def run_steps(state, L, dt, nsteps, rc=2.5, kind=FORCE_LJ, strength=0.0, periodic=True,
              record=True):
    t = np.array([state.t])
    pe = np.array([state.pe])
    w = np.array([state.vir])
    thermo = np.zeros((nsteps, 7)) if record else None
    lib().ljref_run_steps(state.N, _p(state.x), _p(state.v), _p(state.d), _p(state.F), _p(t),
                          _p(pe), _p(w), _p(_box(L)), dt, 1 if periodic else 0, kind, rc,
                          strength, nsteps, _p(thermo) if record else None)
    state.t, state.pe, state.vir = float(t[0]), float(pe[0]), float(w[0])
    return thermo


def set_temperature(v, target):
    v = np.ascontiguousarray(v, dtype=np.float64)
    lib().ljref_set_temperature(v.shape[0], _p(v), target)
    return v


def rdf(x, L, nbins, rmax):
    x = as4(x)
    hist = np.zeros(nbins, dtype=np.uint64)
    lib().ljref_rdf(x.shape[0], _p(x), 4, _p(_box(L)), nbins, rmax, _p(hist))
    return hist


def rdf_cells(x, L, nbins, rmax, threads=None):
    """ljref.rdf's histogram in O(N) through a cell list of edge >= rmax (boxes of
    at least 3 such cells per axis), on `threads` host threads (default: all)."""
    x = as4(x)
    hist = np.zeros(nbins, dtype=np.uint64)
    t = cpu_count() if threads is None else int(threads)
    rc = lib().ljref_rdf_cells(x.shape[0], _p(x), 4, _p(_box(L)), nbins, rmax, t, _p(hist))
    if rc != 0:
        raise ValueError("rdf_cells needs at least 3 cells of edge rmax per axis")
    return hist


class SimConfig(ctypes.Structure):
    _fields_ = [
        ("temperature", ctypes.c_double), ("density", ctypes.c_double),
        ("particle_count", ctypes.c_int), ("random_seed", ctypes.c_uint),
        ("cutoff_distance", ctypes.c_double), ("time_delta", ctypes.c_double),
        ("eq_tolerance", ctypes.c_double), ("eq_sample_size", ctypes.c_int),
        ("eq_adjustment_interval", ctypes.c_int), ("eq_steady_state_time", ctypes.c_int),
        ("eq_timeout", ctypes.c_int),
        ("ob_tolerance", ctypes.c_double), ("ob_sample_size", ctypes.c_int),
        ("ob_observation_interval", ctypes.c_int), ("ob_observation_count", ctypes.c_int),
    ]


def simulate(cfg, max_steps=100000):
    """Run the reference control protocol; returns (thermo[n,7], events_text, snapshot[N,9])."""
    thermo = np.zeros((max_steps, 7))
    ev = ctypes.create_string_buffer(1 << 20)
    snap = np.zeros((cfg.particle_count, 9))
    n = lib().ljref_simulate(ctypes.byref(cfg), max_steps, _p(thermo), ev, len(ev), _p(snap))
    assert n >= 0, "thermo buffer too small"
    return thermo[:n], ev.value.decode(), snap


def bench(N, T, density, seed, rc, dt, warm, steps, replicas, fast=True):
    """Seconds for `steps` VV steps on `replicas` concurrent threads (max over threads)."""
    sec = np.zeros(1)
    lib(fast).ljref_bench(N, T, density, seed, rc, dt, warm, steps, replicas, _p(sec))
    return float(sec[0])


def cpu_count():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1
