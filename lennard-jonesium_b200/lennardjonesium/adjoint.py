"""Differentiable NVE on the GPU: gradients of time-averaged observables.

AdjointNVE wraps the lj_adj_* entry points of include/lj_gpu.h: velocity
Verlet (src/cpp/lennardjonesium/engine/integrator.cpp:62-88) over the LJ
spline of physics/lennard_jones_force.cpp:68-121 generalised to an energy
scale epsilon and a length scale sigma (cutoff = cutoff_sigma * sigma), and a
hand-written discrete adjoint (reverse velocity Verlet with one force
Hessian-vector product per step, checkpoints every k steps, segments
recomputed).  DifferentiableNVE exposes it as a torch.autograd.Function whose
output is the pair (PE_avg, P_avg): the time averages over steps 1..M of the
total potential energy and of the virial pressure (physics/analyzers.cpp:73-75).
Gradients flow to the initial positions and velocities, epsilon and sigma.
"""

import ctypes

import numpy as np
import torch

from lennardjonesium import _native as nat


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class AdjointNVE:
    """One differentiable-NVE context: N atoms in a periodic box, M steps.

    forward(x0, v0) runs the trajectory and returns (PE_avg, P_avg, series)
    with series[n] = (PE, W, KE, P) of state n + 1; backward(w_pe, w_p)
    returns the gradient of w_pe * PE_avg + w_p * P_avg at the last forward
    pass as a dict with keys x0, v0 (N x 3 arrays), epsilon and sigma.
    """

    def __init__(self, N, box, steps, checkpoint_every=20, time_delta=0.005, epsilon=1.0, sigma=1.0,
                 cutoff_sigma=2.5, device=0):
        box = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,))
        self._lib = nat.lib()
        p = nat.AdjParams()
        p.particle_count = int(N)
        for k in range(3):
            p.box[k] = float(box[k])
        p.time_delta = float(time_delta)
        p.steps = int(steps)
        p.checkpoint_every = int(checkpoint_every)
        p.epsilon, p.sigma, p.cutoff_sigma = float(epsilon), float(sigma), float(cutoff_sigma)
        p.device = int(device)
        self._ctx = ctypes.c_void_p()
        status = self._lib.lj_adj_create(ctypes.byref(p), ctypes.byref(self._ctx))
        if status != nat.LJ_OK:
            msg = self._lib.lj_adj_last_error(self._ctx).decode() if self._ctx else ""
            if self._ctx:
                self._lib.lj_adj_destroy(self._ctx)
            self._ctx = None
            raise nat.LJError(status, msg or self._lib.lj_gpu_status_string(status).decode())
        self.N, self.box, self.steps = int(N), box.copy(), int(steps)
        self.epsilon, self.sigma = float(epsilon), float(sigma)
        self.generation = 0  # bumped by every forward pass and potential change

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.lj_adj_destroy(self._ctx)
            self._ctx = None

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
        if status != nat.LJ_OK:
            msg = self._lib.lj_adj_last_error(self._ctx).decode()
            raise nat.LJError(status, msg or self._lib.lj_gpu_status_string(status).decode())

    def set_potential(self, epsilon, sigma):
        if (float(epsilon), float(sigma)) != (self.epsilon, self.sigma):
            self._check(self._lib.lj_adj_set_potential(self._ctx, float(epsilon), float(sigma)))
            self.epsilon, self.sigma = float(epsilon), float(sigma)
            self.generation += 1

    def forward(self, x0, v0):
        x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64)[:, :3])
        v = np.ascontiguousarray(np.asarray(v0, dtype=np.float64)[:, :3])
        if x.shape != (self.N, 3) or v.shape != (self.N, 3):
            raise ValueError(f"expected ({self.N}, 3) positions and velocities")
        out = np.zeros(2)
        series = np.zeros((self.steps, 4))
        self._check(self._lib.lj_adj_forward(self._ctx, _p(x), _p(v), 3, _p(out), _p(series)))
        self.generation += 1
        return float(out[0]), float(out[1]), series

    def backward(self, w_pe=1.0, w_p=1.0):
        dx = np.zeros((self.N, 3))
        dv = np.zeros((self.N, 3))
        de = np.zeros(1)
        ds = np.zeros(1)
        self._check(self._lib.lj_adj_backward(self._ctx, float(w_pe), float(w_p), _p(dx), _p(dv), 3, _p(de),
                                              _p(ds)))
        return {"x0": dx, "v0": dv, "epsilon": float(de[0]), "sigma": float(ds[0])}


class DifferentiableNVE(torch.autograd.Function):
    """(x0, v0, epsilon, sigma, engine) -> tensor([PE_avg, P_avg]).

    x0, v0: (N, 3) float64 tensors on any device; epsilon, sigma: float64
    scalar tensors or Python floats.  The backward pass is the engine's
    adjoint; if the engine ran another forward pass or changed its potential
    in between, the stored inputs are replayed first.
    """

    @staticmethod
    def forward(ctx, x0, v0, epsilon, sigma, engine):
        eps = float(epsilon)
        sig = float(sigma)
        engine.set_potential(eps, sig)
        xn = x0.detach().to("cpu", torch.float64).numpy()
        vn = v0.detach().to("cpu", torch.float64).numpy()
        pe, p, _ = engine.forward(xn, vn)
        ctx.engine = engine
        ctx.generation = engine.generation
        ctx.replay = (xn.copy(), vn.copy(), eps, sig)
        ctx.devices = (x0.device, v0.device)
        ctx.param_kinds = tuple(
            (t.device, t.dtype) if isinstance(t, torch.Tensor) else None for t in (epsilon, sigma))
        return torch.tensor([pe, p], dtype=torch.float64, device=x0.device)

    @staticmethod
    def backward(ctx, grad):
        engine = ctx.engine
        if engine.generation != ctx.generation:
            xn, vn, eps, sig = ctx.replay
            engine.set_potential(eps, sig)
            engine.forward(xn, vn)
            ctx.generation = engine.generation
        w = grad.detach().to("cpu", torch.float64).tolist()
        g = engine.backward(w[0], w[1])
        need = ctx.needs_input_grad
        gx = torch.from_numpy(g["x0"]).to(ctx.devices[0]) if need[0] else None
        gv = torch.from_numpy(g["v0"]).to(ctx.devices[1]) if need[1] else None
        out = [gx, gv]
        for name, kind, req in (("epsilon", ctx.param_kinds[0], need[2]), ("sigma", ctx.param_kinds[1], need[3])):
            out.append(torch.tensor(g[name], dtype=kind[1], device=kind[0]) if (req and kind) else None)
        return (*out, None)


def nve_observables(x0, v0, epsilon, sigma, box, steps, time_delta=0.005, checkpoint_every=20, cutoff_sigma=2.5,
                    engine=None, device=0):
    """Differentiable (PE_avg, P_avg) of an M-step NVE run from (x0, v0).

    Builds an AdjointNVE for the run unless one is passed in; reuse one engine
    across calls of the same N, box and step count.
    """
    if engine is None:
        engine = AdjointNVE(x0.shape[0], box, steps, checkpoint_every, time_delta, float(epsilon), float(sigma),
                            cutoff_sigma, device)
    return DifferentiableNVE.apply(x0, v0, epsilon, sigma, engine)
