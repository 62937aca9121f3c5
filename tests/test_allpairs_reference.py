"""The adjoint's oracle (oracle/allpairs_lj.py, torch FP64 all-pairs LJ): autograd vs central differences."""
import os
import sys

import numpy as np
import pytest
import torch

import tinymd
from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import allpairs_lj  # noqa: E402


def lattice(product, cells=(4, 4, 4)):
    m, x, v, world, rank = tinymd.setup_particles("default", cells, lib=product)
    box = torch.tensor(world[1::2] - world[0::2], dtype=torch.float64)
    vv = v - v.mean(0)
    vv *= np.sqrt(1.44 / ((vv ** 2).sum() / (3 * len(m) - 3)))
    return torch.tensor(x), torch.tensor(vv), box


def test_lattice_energy_matches_oracle(product):
    x, v, box = lattice(product)
    u = allpairs_lj.energy(x, box, 1.0, 1.0, 2.5) / x.shape[0]
    assert float(u) == pytest.approx(-6.773317807608419, rel=1e-12)


def test_autograd_matches_central_differences(product):
    """10 steps at 256 atoms: no pair crosses the cutoff between theta +- h here."""
    x, v, box = lattice(product)
    steps, dt, h = 10, 0.005, 1e-4
    v0 = v.clone().requires_grad_(True)
    eps = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    loss = allpairs_lj.trajectory_loss(x, v0, eps, sig, box, dt, steps)
    loss.backward()
    with torch.no_grad():
        def L(vv=v, e=1.0, s=1.0):
            return float(allpairs_lj.trajectory_loss(x, vv, e, s, box, dt, steps))
        fd_e = (L(e=1 + h) - L(e=1 - h)) / (2 * h)
        fd_s = (L(s=1 + h) - L(s=1 - h)) / (2 * h)
        assert float(eps.grad) == pytest.approx(fd_e, rel=1e-5)
        assert float(sig.grad) == pytest.approx(fd_s, rel=1e-5)
        scale = float(v0.grad.abs().max())
        rng = np.random.default_rng(7)
        for k in rng.choice(v.numel(), 6, replace=False):
            i, d = divmod(int(k), 3)
            vp, vm = v.clone(), v.clone()
            vp[i, d] += h
            vm[i, d] -= h
            fd = (L(vv=vp) - L(vv=vm)) / (2 * h)
            assert abs(float(v0.grad[i, d]) - fd) <= 1e-5 * scale
