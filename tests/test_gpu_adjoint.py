"""The differentiable form on the GPU: hand-written adjoint kernels vs FP64 autograd and FD.

The trajectory is velocity-Verlet LJ with lists frozen per reneighbour segment;
the loss is MSD + U(x_T)/N.  Two loss energies: the reference's unshifted pair
energy (the loss jumps when a pair crosses the cutoff, so central differences
of it are not derivatives once pairs can cross between theta +- h) and the
energy shifted to zero at the cutoff (continuous).  The adjoint is checked
exactly against torch autograd of an all-pairs trajectory for both, and against
central differences on the continuous loss at steps where no cutoff crossing
moves between theta +- h (the truncated force itself jumps at the cutoff).
"""
import os
import sys

import numpy as np
import pytest
import torch

import tinymd
from tinymd import adjoint
from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import allpairs_lj  # noqa: E402

pytestmark = pytest.mark.gpu


def setup(product, cells):
    parts = tinymd.setup_particles("default", cells, lib=product)
    sim = tinymd.Simulation(product, *parts, temp=1.44)
    v0 = adjoint.initial_velocities(product, sim)
    return sim, parts, v0


def adjoint_grads(product, v0, eps=1.0, sigma=1.0):
    v = torch.tensor(v0, requires_grad=True)
    e = torch.tensor(eps, dtype=torch.float64, requires_grad=True)
    s = torch.tensor(sigma, dtype=torch.float64, requires_grad=True)
    loss = adjoint.TrajectoryLoss.apply(v, e, s, product)
    loss.backward()
    return float(loss.detach()), v.grad.numpy(), float(e.grad), float(s.grad)


@pytest.mark.parametrize("shifted", [False, True])
def test_adjoint_matches_allpairs_autograd(product, shifted):
    """4x4x4 cells (256 atoms), 50 steps, FP64, lists rebuilt every 5 steps (within the 0.3 skin,
    so the list trajectory is the all-pairs one): adjoint kernels vs torch autograd."""
    sim, parts, v0 = setup(product, (4, 4, 4))
    try:
        adjoint.configure(product, steps=50, reneigh=5, dt=0.005, precision=0, shifted_energy=shifted)
        loss, gv, ge, gs = adjoint_grads(product, v0)
    finally:
        sim.close()
    m, x, _, world, _ = parts
    box = torch.tensor(world[1::2] - world[0::2], dtype=torch.float64)
    vt = torch.tensor(v0, requires_grad=True)
    et = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    st = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    lt = allpairs_lj.trajectory_loss(torch.tensor(x), vt, et, st, box, 0.005, 50, shifted=shifted)
    lt.backward()
    assert loss == pytest.approx(float(lt.detach()), rel=1e-10)
    assert ge == pytest.approx(float(et.grad), rel=1e-8)
    assert gs == pytest.approx(float(st.grad), rel=1e-8)
    ref = vt.grad.numpy()
    assert np.max(np.abs(gv - ref)) <= 1e-8 * np.max(np.abs(ref))


def _fd_eps(product, v0, h):
    return (adjoint.loss_value(product, v0, 1 + h, 1.0) - adjoint.loss_value(product, v0, 1 - h, 1.0)) / (2 * h)


def _fd_sigma(product, v0, h):
    return (adjoint.loss_value(product, v0, 1.0, 1 + h) - adjoint.loss_value(product, v0, 1.0, 1 - h)) / (2 * h)


def _worst_velocity_error(product, v0, gv, h, count=32, seed=2024):
    """Max relative error over `count` seeded initial-velocity components, each normalised by
    max(|FD|, 1e-3 max|grad|) so components with a near-zero derivative do not dominate."""
    rng = np.random.default_rng(seed)
    scale = np.max(np.abs(gv))
    worst = 0.0
    for k in rng.choice(v0.size, count, replace=False):
        i, d = divmod(int(k), 3)
        vp, vm = v0.copy(), v0.copy()
        vp[i, d] += h
        vm[i, d] -= h
        fd = (adjoint.loss_value(product, vp, 1.0, 1.0) - adjoint.loss_value(product, vm, 1.0, 1.0)) / (2 * h)
        worst = max(worst, abs(gv[i, d] - fd) / max(abs(fd), 1e-3 * scale))
    return worst


def test_adjoint_matches_central_differences_16k_10_steps(product):
    """16x16x16 cells (16,384 atoms), 10 steps: the FP64-forward adjoint against central
    differences of the FP64 forward on the continuous (shifted) loss, to 1e-4 relative:
    eps and sigma at h = 1e-6, 32 seeded initial-velocity components at h = 1e-4 (their
    derivatives are ~1e-5 after 10 steps, so at smaller h the roundoff of the loss,
    ~1e-16 |L| / h, is no longer negligible; over 10 steps a perturbation of 1e-4 moves
    almost no cutoff crossing into another step).  The mixed-forward adjoint agrees with
    the FP64-forward one to 1e-5 (eps, sigma) and 1e-4 of the largest velocity gradient."""
    sim, parts, v0 = setup(product, (16, 16, 16))
    try:
        adjoint.configure(product, steps=10, reneigh=5, dt=0.005, precision=1, shifted_energy=True)
        _, gv1, ge1, gs1 = adjoint_grads(product, v0)
        adjoint.configure(product, steps=10, reneigh=5, dt=0.005, precision=0, shifted_energy=True)
        _, gv0, ge0, gs0 = adjoint_grads(product, v0)
        assert ge1 == pytest.approx(ge0, rel=1e-5) and gs1 == pytest.approx(gs0, rel=1e-5)
        assert np.max(np.abs(gv1 - gv0)) <= 1e-4 * np.max(np.abs(gv0))
        assert ge0 == pytest.approx(_fd_eps(product, v0, 1e-6), rel=1e-4)
        assert gs0 == pytest.approx(_fd_sigma(product, v0, 1e-6), rel=1e-4)
        worst = _worst_velocity_error(product, v0, gv0, 1e-4)
        assert worst <= 1e-4, worst
    finally:
        sim.close()


def test_adjoint_matches_central_differences_16k_200_steps(product):
    """16x16x16 cells (16,384 atoms), 200 steps of dt 0.005, lists fixed per 20-step segment.

    The reference's LJ force is truncated, not shifted: it jumps by about 0.039 eps/sigma when a
    pair crosses rc, so the discrete trajectory map is piecewise smooth.  The adjoint is the exact
    derivative of the smooth piece (the pathwise gradient).  A central difference over theta +- h
    also picks up every crossing that the perturbation moves into another step; their number grows
    like h, so for h large enough to contain any they add an h-independent bias (1.6 % on dL/deps
    at h = 1e-4 .. 1e-2 here) and for smaller h a few isolated jumps.  The FP64 forward is
    deterministic bit for bit, so each check below uses a step at which no crossing lands in the
    window: eps at h = 1e-8 and 32 seeded velocity components at h = 1e-7, both to 1e-4 relative
    against the FP64-forward adjoint.  sigma rescales every pair distance, so some crossing moves
    at every h down to 1e-8; it is checked by the 10-step case and exactly against all-pairs
    autograd.  The mixed-forward adjoint differentiates a different trajectory (FP32 pair forces,
    ~1e-5 relative, amplified by 200 chaotic steps): its eps and sigma gradients agree with the
    FP64-forward ones to 1e-5 and its per-component velocity gradients to 1e-3 of the largest
    (about 2e-4 measured; how close depends on the FP32 summation order of the forward)."""
    sim, parts, v0 = setup(product, (16, 16, 16))
    try:
        adjoint.configure(product, steps=200, reneigh=20, dt=0.005, precision=1, shifted_energy=True)
        _, gv1, ge1, gs1 = adjoint_grads(product, v0)
        fwd_ms, bwd_ms = adjoint.times(product)
        adjoint.configure(product, steps=200, reneigh=20, dt=0.005, precision=0, shifted_energy=True)
        _, gv0, ge0, gs0 = adjoint_grads(product, v0)
        assert ge1 == pytest.approx(ge0, rel=1e-5) and gs1 == pytest.approx(gs0, rel=1e-5)
        assert np.max(np.abs(gv1 - gv0)) <= 1e-3 * np.max(np.abs(gv0))
        fd_e = _fd_eps(product, v0, 1e-8)
        assert ge0 == pytest.approx(fd_e, rel=1e-4)
        worst = _worst_velocity_error(product, v0, gv0, 1e-7)
        assert worst <= 1e-4, worst
        print(f"adjoint 16k x 200 (mixed forward): forward {fwd_ms:.2f} ms, backward {bwd_ms:.2f} ms, "
              f"ratio {bwd_ms / fwd_ms:.2f}; dL/deps {ge0:.8f} (FD {fd_e:.8f}), worst v rel err {worst:.2e}")
    finally:
        sim.close()


def test_reference_loss_fd_at_several_steps(product):
    """The unshifted loss at 256 atoms: central differences at h = 1e-4, 1e-5, 1e-6 against the adjoint.
    A pair crossing the cutoff between theta +- h adds 4 eps (rc^-12 - rc^-6) / (N 2h) to the estimate;
    at least the smallest step agrees to 1e-4."""
    sim, parts, v0 = setup(product, (4, 4, 4))
    try:
        adjoint.configure(product, steps=50, reneigh=5, dt=0.005, precision=0, shifted_energy=False)
        loss, gv, ge, gs = adjoint_grads(product, v0)
        rows = []
        for h in (1e-4, 1e-5, 1e-6):
            fe = (adjoint.loss_value(product, v0, 1 + h, 1.0) - adjoint.loss_value(product, v0, 1 - h, 1.0)) / (2 * h)
            fs = (adjoint.loss_value(product, v0, 1.0, 1 + h) - adjoint.loss_value(product, v0, 1.0, 1 - h)) / (2 * h)
            rows.append((h, fe, fs))
        print("adjoint", ge, gs, "FD", rows)
        h, fe, fs = rows[-1]
        assert ge == pytest.approx(fe, rel=1e-4) and gs == pytest.approx(fs, rel=1e-4)
    finally:
        sim.close()
