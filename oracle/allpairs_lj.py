"""FP64 all-pairs LJ trajectory in torch -- TEST INFRASTRUCTURE ONLY (the adjoint oracle).

Naive O(N^2) forces with minimum-image periodic boundaries and the hard cutoff
of the reference's LJ closure (core/runtime.impala:188-201; the same force form
as naive/main.cpp:24-46), velocity-Verlet with unit masses
(core/compute.impala:97-116), and the trajectory loss of the differentiable
form: mean squared (unwrapped) displacement plus potential energy per atom.
torch.autograd through this function is the reference the hand-written
adjoint kernels are checked against.
"""
import torch


def pair_terms(x, box, eps, sigma, rc):
    d = x[:, None, :] - x[None, :, :]
    d = d - box * torch.round(d / box)
    r2 = (d * d).sum(-1)
    n = x.shape[0]
    mask = (r2 < rc * rc) & ~torch.eye(n, dtype=torch.bool, device=x.device)
    r2s = torch.where(mask, r2, torch.ones_like(r2))
    sr2 = 1.0 / r2s
    sr6 = sr2 ** 3 * sigma ** 6
    f = torch.where(mask, 48.0 * eps * sr6 * (sr6 - 0.5) * sr2, torch.zeros_like(r2))
    e = torch.where(mask, 4.0 * eps * sr6 * (sr6 - 1.0), torch.zeros_like(r2))
    return d, f, e


def forces(x, box, eps, sigma, rc):
    d, f, _ = pair_terms(x, box, eps, sigma, rc)
    return (f[..., None] * d).sum(1)


def energy(x, box, eps, sigma, rc, shifted=False):
    d, f, e = pair_terms(x, box, eps, sigma, rc)
    u = 0.5 * e.sum()
    if shifted:  # each pair inside the cutoff shifted by its value at the cutoff
        src6 = (sigma / rc) ** 6
        inside = (f != 0).sum() * 0.5
        u = u - inside * 4.0 * eps * (src6 * src6 - src6)
    return u


def trajectory_loss(x0, v0, eps, sigma, box, dt, steps, rc=2.5, shifted=False):
    x = x0
    v = v0
    f = forces(x, box, eps, sigma, rc)
    for _ in range(steps):
        v = v + 0.5 * dt * f
        x = x + dt * v
        f = forces(x, box, eps, sigma, rc)
        v = v + 0.5 * dt * f
    n = x0.shape[0]
    return ((x - x0) ** 2).sum() / n + energy(x, box, eps, sigma, rc, shifted) / n
