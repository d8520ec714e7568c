"""Pins the FP64 reference gradient (tests/adjoint_reference.py) on the CPU.

Its trajectory at epsilon = sigma = 1 is the oracle's (which the golden
vectors pin), and its autograd gradient is the derivative of its own output
(central differences).  The GPU adjoint is then checked against it in
test_gpu_adjoint.py.
"""

import numpy as np
import pytest
import torch

import adjoint_reference as ar
import ljref


def _state(N, T, rho, seed):
    x, v, L = ljref.initial_state(N, T, rho, seed)
    return x, v, L


def test_reference_trajectory_matches_oracle():
    x, v, L = _state(500, 1.2, 0.8, 5)
    steps = 25
    st = ljref.State(x, v)
    st.F, st.pe, st.vir = ljref.forces(x, L)  # F_0 = F(x_0)
    thermo = ljref.run_steps(st, L, 0.005, steps)
    out, rows = ar.observables(torch.from_numpy(x[:, :3]), torch.from_numpy(v[:, :3]), 1.0, 1.0, L, steps)
    rows = rows.numpy()
    # oracle thermo columns: time, KE, PE, TE, virial, T, MSD
    assert np.allclose(rows[:, 0], thermo[:, 2], rtol=1e-11, atol=0)
    assert np.allclose(rows[:, 1], thermo[:, 4], rtol=1e-11, atol=0)
    assert np.allclose(rows[:, 2], thermo[:, 1], rtol=1e-11, atol=0)
    rho = 500 / L ** 3
    assert np.allclose(rows[:, 3], rho * (thermo[:, 5] + thermo[:, 4] / 1500), rtol=1e-11)
    assert float(out[0]) == pytest.approx(thermo[:, 2].mean(), rel=1e-11)


def test_reference_gradient_is_the_derivative():
    x, v, L = _state(108, 1.2, 0.8, 9)
    steps = 12
    x0 = torch.from_numpy(x[:, :3]).requires_grad_(True)
    v0 = torch.from_numpy(v[:, :3]).requires_grad_(True)
    eps = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    out, _ = ar.observables(x0, v0, eps, sig, L, steps)
    loss = out[0] + out[1]
    gx, gv, ge, gs = torch.autograd.grad(loss, (x0, v0, eps, sig))
    rng = np.random.default_rng(3)
    dx = torch.from_numpy(rng.standard_normal((108, 3)))
    dv = torch.from_numpy(rng.standard_normal((108, 3)))
    h = 1e-6

    def f(dxs=0.0, dvs=0.0, de=0.0, ds=0.0):
        with torch.no_grad():
            o, _ = ar.observables(x0 + dxs * dx, v0 + dvs * dv, 1.0 + de, 1.0 + ds, L, steps)
        return float(o[0] + o[1])

    checks = [
        ((f(de=h) - f(de=-h)) / (2 * h), float(ge)),
        ((f(ds=h) - f(ds=-h)) / (2 * h), float(gs)),
        ((f(dxs=h) - f(dxs=-h)) / (2 * h), float((gx * dx).sum())),
        ((f(dvs=h) - f(dvs=-h)) / (2 * h), float((gv * dv).sum())),
    ]
    for fd, ad in checks:
        assert ad == pytest.approx(fd, rel=1e-5)
