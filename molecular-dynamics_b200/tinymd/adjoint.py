"""Differentiable form: a torch.autograd.Function over the md_adjoint_* C ABI.

    sim = tinymd.Simulation(lib, *tinymd.setup_particles("default", (16, 16, 16)), temp=1.44)
    configure(lib, steps=200, reneigh=20, dt=0.005, cutoff=2.5, skin=0.3, precision=1)
    v0 = torch.tensor(initial_velocities(lib, sim), requires_grad=True)
    eps = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    sigma = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    loss = TrajectoryLoss.apply(v0, eps, sigma, lib)
    loss.backward()          # v0.grad, eps.grad, sigma.grad

The loss is L = (1/N) sum_i |x_T,i - x_0,i|^2 (unwrapped) + U(x_T)/N over a
velocity-Verlet LJ trajectory with exact periodic ghosts, starting from the
positions given to md_initialize_grid.  The forward pass runs on the GPU in
the configured precision and keeps one checkpoint per reneighbour interval;
the backward pass recomputes each interval and runs the hand-written
Hessian-vector-product adjoint kernels over the same neighbour lists.
"""
import ctypes

import numpy as np
import torch

from . import check, ptr


def configure(lib, steps, reneigh=20, dt=0.005, cutoff=2.5, skin=0.3, precision=1, shifted_energy=False):
    """Trajectory and loss settings; shifted_energy selects U shifted to zero at the
    cutoff (continuous in eps and sigma) instead of the reference's unshifted U."""
    if lib.md_adjoint_configure(steps, reneigh, dt, cutoff, skin, precision) != 0:
        check(lib)
        raise RuntimeError("md_adjoint_configure failed")
    lib.md_adjoint_set_loss(1 if shifted_energy else 0)


def initial_velocities(lib, sim):
    """The velocities of the grid's locals (reference order) after md_create_velocity."""
    _, _, v, _ = sim.arrays()
    return v


def times(lib):
    """(forward ms, backward ms) of the last passes, device time."""
    f, b = ctypes.c_double(), ctypes.c_double()
    lib.md_adjoint_times(ctypes.byref(f), ctypes.byref(b))
    return f.value, b.value


def loss_value(lib, v0, eps, sigma):
    """Forward pass only (no gradient state kept for the caller)."""
    v = np.ascontiguousarray(np.asarray(v0, dtype=np.float64))
    out = ctypes.c_double()
    if lib.md_adjoint_forward(ptr(v), float(eps), float(sigma), ctypes.byref(out)) != 0:
        check(lib)
        raise RuntimeError("md_adjoint_forward failed")
    return out.value


class TrajectoryLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, v0, eps, sigma, lib):
        v = np.ascontiguousarray(v0.detach().to("cpu", torch.float64).numpy())
        out = ctypes.c_double()
        if lib.md_adjoint_forward(ptr(v), float(eps), float(sigma), ctypes.byref(out)) != 0:
            check(lib)
            raise RuntimeError("md_adjoint_forward failed")
        ctx.lib = lib
        ctx.shape = tuple(v0.shape)
        ctx.device = v0.device
        return torch.tensor(out.value, dtype=torch.float64, device=v0.device)

    @staticmethod
    def backward(ctx, grad_out):
        gv = np.zeros(ctx.shape)
        ge, gs = ctypes.c_double(), ctypes.c_double()
        if ctx.lib.md_adjoint_backward(ptr(gv), ctypes.byref(ge), ctypes.byref(gs)) != 0:
            check(ctx.lib)
            raise RuntimeError("md_adjoint_backward failed")
        g = grad_out.to(torch.float64)
        return (g * torch.from_numpy(gv).to(ctx.device), g * ge.value, g * gs.value, None)
