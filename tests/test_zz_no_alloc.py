"""The allocation-free RDF entry point (lj_gpu_rdf_noalloc) against lj_gpu_rdf and the oracle.

lj_gpu_rdf_noalloc serves callers that may not call cudaMalloc (an application
whose GPU memory belongs to its own pool allocator, or an analysis hook in a
time-critical loop).  It takes device buffers the caller owns and takes its
cell-list scratch from a fixed array inside the library, which every call
shares.  This test calls it through the C ABI twice in a row on each case
(the second call must not see the first call's leftovers) and requires the
same histogram as the allocating entry point, bit for bit (the tolerance the
RDF tests use).  The file is named to be collected last.
"""

import ctypes

import numpy as np
import pytest

import ljref

pytestmark = pytest.mark.gpu

CASES = [  # N, rho, nbins, rmax: the first uses all pairs, the others the cell list
    (864, 0.8442, 200, 4.0),
    (4000, 0.8, 200, 4.0),
    (32000, 0.8442, 300, 3.5),
]


def _positions(N, rho, seed):
    x, _, L = ljref.initial_state(N, 1.0, rho, seed)
    rng = np.random.default_rng(seed)
    x[:, :3] = np.mod(x[:, :3] + rng.uniform(-0.3, 0.3, size=(N, 3)), L)
    return x, L


def _noalloc(x, box, nbins, rmax, stream):
    """Call lj_gpu_rdf_noalloc on device copies of x; returns (status, histogram)."""
    import torch
    from lennardjonesium import _native as nat
    pos = torch.from_numpy(np.ascontiguousarray(x)).to("cuda")
    hist = torch.full((nbins,), -1, dtype=torch.int64, device="cuda")  # stale contents
    boxv = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,)).copy()
    rc = nat.lib().lj_gpu_rdf_noalloc(ctypes.c_void_p(pos.data_ptr()), x.shape[0],
                                      boxv.ctypes.data_as(ctypes.c_void_p), nbins, rmax,
                                      ctypes.c_void_p(hist.data_ptr()), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, hist.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("N,rho,nbins,rmax", CASES)
def test_rdf_noalloc_matches_rdf(N, rho, nbins, rmax):
    import torch
    from lennardjonesium import GpuSystem
    from lennardjonesium import _native as nat

    L = nat.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for call, seed in enumerate((3, 4)):
        x, box = _positions(N, rho, seed)
        rmax_c = min(rmax, box / 2)
        with GpuSystem(N, box) as g:
            g.upload(x)
            want = g.rdf(nbins, rmax_c)
        pos = torch.from_numpy(np.ascontiguousarray(x)).to("cuda")
        hist = torch.full((nbins,), -1, dtype=torch.int64, device="cuda")  # stale contents
        boxv = np.full(3, box)
        rc = L.lj_gpu_rdf_noalloc(ctypes.c_void_p(pos.data_ptr()), N, boxv.ctypes.data_as(ctypes.c_void_p),
                                  nbins, rmax_c, ctypes.c_void_p(hist.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        got = hist.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want), f"call {call}"
        assert got.sum() > 0
        # and straight against the oracle's textbook histogram
        assert np.array_equal(got, ljref.rdf(x, box, nbins, rmax_c)), f"call {call} vs oracle"


def test_rdf_noalloc_coarsens_a_grid_beyond_its_cell_limit():
    """1000 atoms in a box of 60 with rmax 1.5 make 40^3 = 64000 cells of edge
    rmax, more than the array's 32768: the call runs on coarser cells and still
    counts exactly the oracle's histogram, twice in a row."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    for call in range(2):
        x = np.zeros((1000, 4))
        x[:, :3] = rng.uniform(0.0, 60.0, size=(1000, 3))
        rc, got = _noalloc(x, 60.0, 100, 1.5, stream)
        assert rc == 0, f"call {call}: status {rc}"
        assert np.array_equal(got, ljref.rdf(x, 60.0, 100, 1.5)), f"call {call}"


def test_rdf_noalloc_rejects_sizes_beyond_its_limit():
    import torch
    from lennardjonesium import _native as nat

    L = nat.lib()
    pos = torch.zeros((131073, 4), dtype=torch.float64, device="cuda")
    hist = torch.zeros(16, dtype=torch.int64, device="cuda")
    boxv = np.full(3, 60.0)
    rc = L.lj_gpu_rdf_noalloc(ctypes.c_void_p(pos.data_ptr()), 131073, boxv.ctypes.data_as(ctypes.c_void_p), 16,
                              4.0, ctypes.c_void_p(hist.data_ptr()), None)
    assert rc == nat.LJ_ERR_ARG
    rc = L.lj_gpu_rdf_noalloc(ctypes.c_void_p(pos.data_ptr()), 1000, boxv.ctypes.data_as(ctypes.c_void_p), 20000,
                              4.0, ctypes.c_void_p(hist.data_ptr()), None)
    assert rc == nat.LJ_ERR_ARG
    # rmax beyond half the box, a misaligned histogram and a tiny rmax whose
    # cell count would overflow an int: rejected, or (the last) run on a
    # coarse grid, before any kernel starts
    rc = L.lj_gpu_rdf_noalloc(ctypes.c_void_p(pos.data_ptr()), 1000, boxv.ctypes.data_as(ctypes.c_void_p), 16,
                              30.5, ctypes.c_void_p(hist.data_ptr()), None)
    assert rc == nat.LJ_ERR_ARG
    rc = L.lj_gpu_rdf_noalloc(ctypes.c_void_p(pos.data_ptr()), 1000, boxv.ctypes.data_as(ctypes.c_void_p), 8,
                              4.0, ctypes.c_void_p(hist.data_ptr() + 4), None)
    assert rc == nat.LJ_ERR_ARG
    rc = L.lj_gpu_rdf_noalloc(ctypes.c_void_p(pos.data_ptr()), 1000, boxv.ctypes.data_as(ctypes.c_void_p), 16,
                              1e-12, ctypes.c_void_p(hist.data_ptr()), None)
    torch.cuda.synchronize()
    # 1000 coincident atoms: every ordered pair at r = 0 < rmax, all in bin 0
    h = hist.cpu().numpy().view(np.uint64)
    assert rc == 0 and int(h[0]) == 1000 * 999 and int(h[1:].sum()) == 0
