"""FP64 reference gradient for the differentiable NVE engine (test infrastructure).

A plain PyTorch restatement of the same trajectory, all pairs under the
minimum image, differentiated by torch.autograd: velocity Verlet of
src/cpp/lennardjonesium/engine/integrator.cpp:62-88 starting from
F_0 = F(x_0), the LJ spline of physics/lennard_jones_force.cpp:68-121 with an
energy scale epsilon and a length scale sigma (cutoff = cutoff_sigma * sigma),
and the time averages over steps 1..M of the total potential energy and of the
virial pressure rho (T + W / 3N) (physics/analyzers.cpp:73-75).  It shares no
code with the CUDA engine; it is the checker, never the product path.
"""

import torch
from torch.utils.checkpoint import checkpoint


def pair_terms(q, eps, sigma, uc):
    """V and W = -r V'(r) at q = r^2."""
    rcm6 = 1.0 / uc ** 6
    alpha = -4.0 * rcm6 * (rcm6 - 1.0)
    beta = 12.0 * rcm6 * (2.0 * rcm6 - 1.0)
    s6 = (sigma * sigma / q) ** 3
    x = q / (uc * uc * sigma * sigma)
    V = eps * (4.0 * s6 * (s6 - 1.0) + alpha + beta * (x - 1.0))
    W = eps * (48.0 * s6 * s6 - 24.0 * s6 - 2.0 * beta * x)
    return V, W


def forces(x, L, eps, sigma, uc):
    """(F, PE, W) over all pairs within the cutoff (minimum image)."""
    N = x.shape[0]
    r = x[:, None, :] - x[None, :, :]
    r = r - L * torch.round(r / L)
    q = (r * r).sum(-1)
    rc = uc * sigma
    mask = (q < rc * rc) & ~torch.eye(N, dtype=torch.bool, device=x.device)
    qs = torch.where(mask, q, torch.ones_like(q))
    V, W = pair_terms(qs, eps, sigma, uc)
    V = torch.where(mask, V, torch.zeros_like(V))
    W = torch.where(mask, W, torch.zeros_like(W))
    F = ((W / qs)[:, :, None] * r).sum(1)
    return F, 0.5 * V.sum(), 0.5 * W.sum()


def _step(x, v, F, L, eps, sigma, uc, dt):
    h = v + 0.5 * dt * F
    x = x + dt * h
    x = x - torch.floor(x / L) * L
    F, pe, w = forces(x, L, eps, sigma, uc)
    v = h + 0.5 * dt * F
    return x, v, F, pe, w


def observables(x0, v0, eps, sigma, L, steps, dt=0.005, uc=2.5, per_step_checkpoint=False):
    """tensor([PE_avg, P_avg]) and the per-step series (PE, W, KE, P)."""
    N = x0.shape[0]
    L = torch.as_tensor(L, dtype=torch.float64, device=x0.device)
    rho = N / torch.prod(L.expand(3))
    x, v = x0, v0
    F, _, _ = forces(x, L, eps, sigma, uc)
    pes, ps, rows = [], [], []
    for _ in range(steps):
        if per_step_checkpoint:
            x, v, F, pe, w = checkpoint(_step, x, v, F, L, eps, sigma, uc, dt, use_reentrant=False)
        else:
            x, v, F, pe, w = _step(x, v, F, L, eps, sigma, uc, dt)
        ke = 0.5 * (v * v).sum()
        T = (2.0 / 3.0) * ke / N
        P = rho * (T + w / (3.0 * N))
        pes.append(pe)
        ps.append(P)
        rows.append(torch.stack([pe, w, ke, P]).detach())
    out = torch.stack([torch.stack(pes).mean(), torch.stack(ps).mean()])
    return out, torch.stack(rows)
