"""The differentiable NVE engine (lj_adj_*) on the GPU.

Workload of the gradient checks: N = 4000 (4 * 10^3 FCC), rho = 0.8, T = 1.2,
rc = 2.5 sigma, dt = 0.005, 200 steps, FP64, checkpoints every 20 steps; the
loss is the time-averaged total PE plus the virial pressure.  The adjoint
gradient is checked against central finite differences (h = 1e-6) to 1e-4
relative, and against the FP64 torch.autograd reference gradient of
tests/adjoint_reference.py.
"""

import numpy as np
import pytest

import ljref

pytestmark = pytest.mark.gpu

N, RHO, T, STEPS, K, DT = 4000, 0.8, 1.2, 200, 20, 0.005
H = 1e-6


@pytest.fixture(scope="module")
def system():
    x, v, L = ljref.initial_state(N, T, RHO, 4000)
    return x[:, :3].copy(), v[:, :3].copy(), L


@pytest.fixture(scope="module")
def engine(system):
    from lennardjonesium import AdjointNVE
    x, v, L = system
    with AdjointNVE(N, L, STEPS, checkpoint_every=K, time_delta=DT) as e:
        yield e


def test_forward_matches_oracle_trajectory():
    from lennardjonesium import AdjointNVE
    x, v, L = ljref.initial_state(500, 1.2, 0.8, 5)
    steps = 60
    st = ljref.State(x, v)
    st.F, st.pe, st.vir = ljref.forces(x, L)  # F_0 = F(x_0)
    thermo = ljref.run_steps(st, L, DT, steps)
    with AdjointNVE(500, L, steps, checkpoint_every=7, time_delta=DT) as e:
        pe_avg, p_avg, series = e.forward(x, v)
    # series: PE, W, KE, P; oracle thermo: time, KE, PE, TE, virial, T, MSD
    assert np.allclose(series[:, 0], thermo[:, 2], rtol=1e-10, atol=0)
    assert np.allclose(series[:, 1], thermo[:, 4], rtol=1e-10, atol=0)
    assert np.allclose(series[:, 2], thermo[:, 1], rtol=1e-10, atol=0)
    assert pe_avg == pytest.approx(thermo[:, 2].mean(), rel=1e-10)


def _fd(engine, x, v, fn):
    """Central difference of fn's perturbation of (x, v, eps, sigma)."""
    vals = []
    for s in (+H, -H):
        xs, vs, eps, sig = fn(s)
        engine.set_potential(eps, sig)
        pe, p, _ = engine.forward(xs, vs)
        vals.append((pe, p))
    engine.set_potential(1.0, 1.0)
    return [(vals[0][q] - vals[1][q]) / (2 * H) for q in range(2)]


@pytest.mark.parametrize("weights", [(1.0, 0.0), (0.0, 1.0), (1.0, 1.0)])
def test_gradient_vs_central_differences(system, engine, weights):
    x, v, L = system
    engine.set_potential(1.0, 1.0)
    engine.forward(x, v)
    g = engine.backward(*weights)
    rng = np.random.default_rng(17)
    dx = rng.standard_normal(x.shape)
    dx /= np.linalg.norm(dx)  # unit directions: h is the length of the step
    dv = rng.standard_normal(v.shape)
    dv /= np.linalg.norm(dv)
    i = int(np.argmax(np.abs(g["x0"]).sum(1)))  # the most sensitive atom
    ex = np.zeros_like(x)
    ex[i] = g["x0"][i] / np.linalg.norm(g["x0"][i])
    cases = {
        "epsilon": (lambda s: (x, v, 1.0 + s, 1.0), g["epsilon"]),
        "sigma": (lambda s: (x, v, 1.0, 1.0 + s), g["sigma"]),
        "x0 random direction": (lambda s: (x + s * dx, v, 1.0, 1.0), float((g["x0"] * dx).sum())),
        "x0 one atom": (lambda s: (x + s * ex, v, 1.0, 1.0), float((g["x0"] * ex).sum())),
        "v0 random direction": (lambda s: (x, v + s * dv, 1.0, 1.0), float((g["v0"] * dv).sum())),
    }
    report, bad = [], False
    for name, (fn, ad) in cases.items():
        fpe, fp = _fd(engine, x, v, fn)
        fd = weights[0] * fpe + weights[1] * fp
        rel = abs(ad - fd) / abs(fd)
        bad |= not rel <= 1e-4
        report.append(f"{name}: adjoint {ad!r} central difference {fd!r} rel {rel:.2e}")
    assert not bad, "\n".join(report)


def test_gradient_vs_fp64_autograd_reference(system, engine):
    import torch
    import adjoint_reference as ar
    x, v, L = system
    engine.set_potential(1.0, 1.0)
    pe, p, series = engine.forward(x, v)
    g = engine.backward(1.0, 1.0)
    dev = torch.device("cuda:0")
    x0 = torch.from_numpy(x).to(dev).requires_grad_(True)
    v0 = torch.from_numpy(v).to(dev).requires_grad_(True)
    eps = torch.tensor(1.0, dtype=torch.float64, device=dev, requires_grad=True)
    sig = torch.tensor(1.0, dtype=torch.float64, device=dev, requires_grad=True)
    out, rows = ar.observables(x0, v0, eps, sig, L, STEPS, dt=DT, per_step_checkpoint=True)
    gx, gv, ge, gs = torch.autograd.grad(out[0] + out[1], (x0, v0, eps, sig))
    out = out.detach().cpu().numpy()
    assert out[0] == pytest.approx(pe, rel=1e-10)
    assert out[1] == pytest.approx(p, rel=1e-9)
    assert g["epsilon"] == pytest.approx(float(ge), rel=1e-7)
    assert g["sigma"] == pytest.approx(float(gs), rel=1e-7)
    for mine, ref in ((g["x0"], gx), (g["v0"], gv)):
        ref = ref.cpu().numpy()
        assert np.linalg.norm(mine - ref) <= 1e-7 * np.linalg.norm(ref)


def test_checkpoint_interval_does_not_change_the_gradient(system):
    from lennardjonesium import AdjointNVE
    x, v, L = system
    steps = 40
    ref = None
    for k in (1, 7, 40, 100):
        with AdjointNVE(N, L, steps, checkpoint_every=k, time_delta=DT) as e:
            out = e.forward(x, v)[:2]
            g = e.backward(1.0, 1.0)
        if ref is None:
            ref = (out, g)
            continue
        assert out == ref[0]
        assert g["epsilon"] == ref[1]["epsilon"] and g["sigma"] == ref[1]["sigma"]
        assert np.array_equal(g["x0"], ref[1]["x0"]) and np.array_equal(g["v0"], ref[1]["v0"])


def test_autograd_function(system):
    import torch
    import lennardjonesium as lj
    x, v, L = system
    steps = 30
    x0 = torch.from_numpy(x).cuda().requires_grad_(True)
    v0 = torch.from_numpy(v).cuda()
    eps = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    engine = lj.AdjointNVE(N, L, steps, checkpoint_every=10, time_delta=DT)
    out = lj.nve_observables(x0, v0, eps, sig, L, steps, engine=engine)
    assert out.shape == (2,) and out.device == x0.device
    loss = 2.0 * out[0] - 3.0 * out[1]
    # another forward pass on the same engine in between: backward replays its inputs
    engine.forward(x + 0.01, v)
    loss.backward()
    assert x0.grad is not None and v0.grad is None
    engine.set_potential(1.0, 1.0)
    engine.forward(x, v)
    g = engine.backward(2.0, -3.0)
    assert np.array_equal(x0.grad.cpu().numpy(), g["x0"])
    assert float(eps.grad) == g["epsilon"] and float(sig.grad) == g["sigma"]
    engine.close()


def test_argument_errors():
    from lennardjonesium import AdjointNVE
    from lennardjonesium._native import LJError
    with pytest.raises(LJError):
        AdjointNVE(100, 6.0, 10)  # 2 cells of edge 2.5 per axis: below the 3 the stencil needs
    with pytest.raises(LJError):
        AdjointNVE(500, 8.55, 10, cutoff_sigma=1.0)  # rc^2 <= 2^(1/3)
    with AdjointNVE(500, 8.55, 10) as e:
        with pytest.raises(LJError):
            e.backward()  # no forward pass yet
        with pytest.raises(LJError):
            e.set_potential(1.0, 1.2)  # 8.55 / (2.5 * 1.2) < 3 cells
