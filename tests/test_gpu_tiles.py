"""The mixed path's two pair kernels: neighbour-list gathers from global
memory (tile_cells = 0) and shared-memory tiles (lj_tile.cuh).

Every tile shape reads the same pair set in the same order and evaluates the
same FP32 expressions, so per-atom forces are bit-identical across tile shapes
and between staged tiles and tiles read from global memory (a staging array
too small for the window); only the block partition of the energy sums
changes.  Both kernels meet the mixed path's stated bound against FP64.
"""

import numpy as np
import pytest

import ljref

pytestmark = pytest.mark.gpu


def _perturbed(N, T, rho, seed, amp=0.05):
    x, v, L = ljref.initial_state(N, T, rho, seed)
    rng = np.random.default_rng(seed)
    x[:, :3] = np.mod(x[:, :3] + amp * rng.standard_normal((N, 3)), L)
    return x, v, L


def _forces(x, L, **kw):
    from lennardjonesium import GpuSystem
    with GpuSystem(x.shape[0], L, **kw) as g:
        g.upload(x)
        pe, w = g.compute_forces()
        F = g.download()["F"]
        st = g.stats()
    return F, pe, w, st


@pytest.mark.parametrize("N,rho", [(4000, 0.8), (4 * 12 ** 3, 0.8442), (4 * 9 ** 3, 0.3)])
def test_tile_shapes_and_global_fallback_agree(N, rho):
    x, v, L = _perturbed(N, 1.0, rho, 11)
    F0, pe0, w0, st0 = _forces(x, L, precision="mixed", tile_cells=4)
    assert st0["tile_cells"] >= 1 and 0 < st0["max_staged"] <= st0["tile_capacity"]
    for cells in (1, 2, 3, 6, 8):
        F, pe, w, st = _forces(x, L, precision="mixed", tile_cells=cells)
        assert np.array_equal(F, F0), cells
        assert pe == pytest.approx(pe0, rel=1e-13) and w == pytest.approx(w0, rel=1e-12)
    # a staging array smaller than every window: all tiles read global memory
    F, pe, w, st = _forces(x, L, precision="mixed", tile_cells=4, tile_capacity=16)
    assert st["max_staged"] > st["tile_capacity"] == 16
    assert np.array_equal(F, F0)
    assert pe == pytest.approx(pe0, rel=1e-13)
    # the global-gather kernel: same pairs, the column offset applied per pair
    # (a different FP32 rounding of the separation): within the mixed bound
    F, pe, w, st = _forces(x, L, precision="mixed")
    assert st["tile_cells"] == 0
    S = ljref.force_abs_sum(x, L, 2.5)
    assert np.all(np.sqrt(np.sum((F - F0)[:, :3] ** 2, axis=1)) <= 1e-5 * S)
    assert pe == pytest.approx(pe0, rel=1e-6)


@pytest.mark.parametrize("tile_cells", [0, 6])
def test_mixed_full_size_force_error(tile_cells):
    """N = 1 048 576 (4 * 64^3 FCC, rho = 0.8442, perturbed): the mixed forces
    of both kernels against the FP64 path (itself at 1e-12 of the oracle)."""
    N = 4 * 64 ** 3
    x, v, L = _perturbed(N, 1.0, 0.8442, 5489, amp=0.08)
    F64, pe64, w64, _ = _forces(x, L)
    F32, pe32, w32, st = _forces(x, L, precision="mixed", tile_cells=tile_cells)
    assert st["max_staged"] <= st["tile_capacity"]
    S = ljref.force_abs_sum(x, L, 2.5)
    err = np.sqrt(np.sum((F32 - F64)[:, :3] ** 2, axis=1))
    assert np.all(err <= 1e-5 * S)
    rms = np.sqrt(np.mean(np.sum(F64[:, :3] ** 2, axis=1)))
    assert np.sqrt(np.mean(err ** 2)) / rms < 2e-5
    assert abs(pe32 - pe64) / abs(pe64) < 1e-6
    assert abs(w32 - w64) / abs(w64) < 1e-5


def test_tiled_steps_follow_fp64():
    """200 steps of the tiled mixed path stay on the FP64 trajectory's energy
    (3 cells per axis: every tile is one cell, windows wrap in z)."""
    from lennardjonesium import GpuSystem
    x, v, L = ljref.initial_state(864, 0.722, 0.8442, 5489)
    out = {}
    for prec in ("fp64", "mixed"):
        with GpuSystem(864, L, precision=prec, tile_cells=4 if prec == "mixed" else 0) as g:
            g.upload(x, v=v)
            out[prec] = g.step(200)
            if prec == "mixed":
                assert g.stats()["tile_cells"] == 1
    te64, te32 = out["fp64"][:, 3], out["mixed"][:, 3]
    assert np.max(np.abs(te32 - te64)) / abs(te64[0]) < 1e-5
