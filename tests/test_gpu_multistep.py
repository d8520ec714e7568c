"""Multi-step acceptance criteria, on the GPU through the C ABI.

Trajectories of a chaotic system diverge after a few hundred steps whatever the
arithmetic, so multi-step runs are judged on what survives the divergence:

  * energy conservation: after an equilibration that discards the melting
    transient of the FCC start, the total energy E changes by at most
    |dE / E| <= 1e-4 over 10^4 steps, both as the endpoint difference and as
    a least-squares slope times 10^4 steps, on the FP64 and the mixed path at
    N = 1 048 576 (4 * 64^3, rho 0.8442, T 1.0, dt 0.005);
  * thermodynamic averages: over a production window, the means of the
    temperature T, the potential energy per atom U = PE / N and the
    instantaneous virial pressure P = rho (T + W / 3N) (the estimator of
    src/cpp/lennardjonesium/physics/analyzers.cpp:70-75 applied per step) agree
    within their 2-sigma error bars (the bars overlap: |a - b| <= 2 sigma_a +
    2 sigma_b, sigma the block-averaged standard error of each mean), GPU FP64
    vs the CPU oracle and mixed vs FP64, at N = 864 (4 * 6^3, rho 0.8442,
    T 0.722) and N = 4000 (4 * 10^3, rho 0.8, T 1.2).  Runs from the same
    start decorrelate within a few hundred steps, so the pairs of means behave
    as independent samples: overlapping 2-sigma bars fail by chance with
    probability ~0.5 % per comparison, where a 2-sigma bound on the
    difference alone would fail one of these twelve comparisons ~40 % of the
    time whenever a change of rounding reshuffles the trajectories;
  * the 4 000 000-atom system (4 * 100^3, rho 0.8, T 0.9, dt 0.004): single-step
    forces within 1e-12 of each atom's sum of |pair forces|, PE and virial
    within 1e-12 relative of the oracle, the RDF (200 bins to 4 sigma)
    bit-exact against the oracle's histogram, and the mixed path's forces
    within its stated bounds (1e-5 of the sum of |pair forces|, PE 1e-6 and
    virial 1e-5 relative).
"""

import concurrent.futures as cf

import numpy as np
import pytest

import ljref

pytestmark = pytest.mark.gpu


def gpu_system(N, L, **kw):
    from lennardjonesium import GpuSystem
    return GpuSystem(N, L, **kw)


def block_mean_and_error(series, blocks=20):
    """Mean of a time series and the standard error of that mean from the
    spread of `blocks` consecutive block means (blocks longer than the
    correlation time make the block means independent)."""
    n = len(series) // blocks * blocks
    b = np.asarray(series[:n]).reshape(blocks, -1).mean(axis=1)
    return float(b.mean()), float(b.std(ddof=1) / np.sqrt(blocks))


def observables(th, N, rho):
    """Per-step T, U = PE / N and P = rho (T + W / 3N) from records
    {t, KE, PE, TE, W, T, MSD}."""
    T = th[:, 5]
    return {"T": T, "U": th[:, 2] / N, "P": rho * (T + th[:, 4] / (3.0 * N))}


def assert_same_averages(a, b, what):
    for k in ("T", "U", "P"):
        ma, ea = block_mean_and_error(a[k])
        mb, eb = block_mean_and_error(b[k])
        bound = 2.0 * (ea + eb)
        assert abs(ma - mb) <= bound, f"{what} <{k}>: {ma} +- {2 * ea:.3g} vs {mb} +- {2 * eb:.3g} (2 sigma)"


def drift(te):
    """|dE/E| over the series: endpoint difference and fitted slope times its length."""
    E0 = abs(te[0])
    n = len(te)
    slope = np.polyfit(np.arange(n, dtype=np.float64), te, 1)[0]
    return abs(te[-1] - te[0]) / E0, abs(slope) * n / E0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_energy_drift_full_size(precision):
    from lennardjonesium import initial_condition
    N = 4 * 64 ** 3
    x, v, L = initial_condition(N, 1.0, 0.8442, 5489)
    with gpu_system(N, L, precision=precision) as g:
        g.upload(x, v=v)
        g.step(1000, record=False)  # equilibration: the lattice melts
        te = g.step(10000)[:, 3]
    end, fit = drift(te)
    assert np.all(np.isfinite(te))
    assert end <= 1e-4, f"endpoint |dE/E| {end:.3g}"
    assert fit <= 1e-4, f"fitted |dE/E| over 1e4 steps {fit:.3g}"


# N, T, rho, seed, equilibration steps, production steps
AVERAGE_CASES = [(864, 0.722, 0.8442, 5489, 1000, 8000), (4000, 1.2, 0.8, 7, 1000, 5000)]


@pytest.mark.parametrize("case", AVERAGE_CASES, ids=["N864", "N4000"])
def test_thermodynamic_averages(case):
    N, T, rho, seed, eq, prod = case
    x, v, L = ljref.initial_state(N, T, rho, seed)

    def oracle_run():
        st = ljref.State(x, v=v)
        return ljref.run_steps(st, L, 0.005, eq + prod)[eq:]

    # the oracle runs on a host thread (its C code releases the GIL) while the GPU runs
    with cf.ThreadPoolExecutor(1) as pool:
        fut = pool.submit(oracle_run)
        runs = {}
        for prec in ("fp64", "mixed"):
            with gpu_system(N, L, precision=prec) as g:
                g.upload(x, v=v)
                runs[prec] = g.step(eq + prod)[eq:]
        ref = fut.result()
    obs = {k: observables(th, N, rho) for k, th in runs.items()}
    oref = observables(ref, N, rho)
    for th in list(runs.values()) + [ref]:
        assert np.all(np.isfinite(th))
    assert_same_averages(obs["fp64"], oref, "GPU FP64 vs oracle")
    assert_same_averages(obs["mixed"], obs["fp64"], "mixed vs FP64")


def test_four_million_atoms_forces_and_rdf():
    from lennardjonesium import initial_condition
    n = 100
    N = 4 * n ** 3
    x, v, L = initial_condition(N, 0.9, 0.8, 2718)
    with gpu_system(N, L, dt=0.004) as g:
        g.upload(x, v=v)
        g.step(20)
        st = g.download()
        h = g.rdf(200, 4.0)
    xs = st["x"]
    with cf.ThreadPoolExecutor(2) as pool:
        f_forces = pool.submit(ljref.forces, xs, L, 2.5)
        f_abs = pool.submit(ljref.force_abs_sum, xs, L, 2.5)
        Fref, pe, w = f_forces.result()
        S = f_abs.result()
    err = np.abs(st["F"][:, :3] - Fref[:, :3])
    bound = 1e-12 * np.maximum(S, 1e-300)[:, None]
    assert np.all(err <= bound), f"max excess {(err / bound).max()}"
    assert st["pe"] == pytest.approx(pe, rel=1e-12)
    assert st["virial"] == pytest.approx(w, rel=1e-12)
    assert np.array_equal(h, ljref.rdf_cells(xs, L, 200, 4.0))
    # config 5 runs the mixed path: its forces at the same positions, within the stated bounds
    with gpu_system(N, L, dt=0.004, precision="mixed") as g:
        g.upload(xs)
        pe32, w32 = g.compute_forces()
        F32 = g.download()["F"]
    e32 = np.sqrt(np.sum((F32 - Fref)[:, :3] ** 2, axis=1))
    assert np.all(e32 <= 1e-5 * S)
    assert abs(pe32 - pe) / abs(pe) < 1e-6 and abs(w32 - w) / abs(w) < 1e-5
