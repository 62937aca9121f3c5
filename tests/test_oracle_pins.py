"""Pins of the CPU oracle (CPU only): known answers and the reference's own code.

The reference ships no tests or golden vectors for this path, so the oracle is
pinned by (a) the analytic FCC lattice energy and neighbour shells, (b)
miniMD's published thermo output for the same lattice, RNG and integrator
(results/single_gpu_v100.txt:38-39: T, U, P at steps 0 and 100 for 64x64x32
unit cells, dt 0.001), which the restatement reproduces to every printed
digit with exact periodic ghosts, and (c) the reference's own full-list LJ
kernel core/force_lj.cpp (compiled from the reference tree into oracle/_ref, or
its committed golden output when the tree is absent).
"""
import ctypes
import os

import numpy as np
import pytest

import tinymd
from conftest import GOLDEN
from helpers import make_sim, rel_err

MINIMD_LATTICE = (4.0 / 0.8442) ** (1.0 / 3.0)  # miniMD derives the lattice constant from the density


def thermo(lib, n, volume, half=False):
    t = np.zeros(2)
    lib.oracle_last_thermo(tinymd.ptr(t))
    w = 1.0 if half else 0.5
    temp = lib.oracle_temperature()
    dof = 3.0 * n - 3.0
    return temp, t[0] * w / n, (temp * dof + t[1] * w) / (3.0 * volume)


def fcc_energy_per_atom(a, rc=2.5):
    basis = np.array([[0, 0, 0], [.5, .5, 0], [.5, 0, .5], [0, .5, .5]])
    r = np.arange(-3, 4)
    cells = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 1, 3)
    d = np.linalg.norm((cells + basis[None]).reshape(-1, 3) * a, axis=1)
    d = d[(d > 0) & (d < rc)]
    return 0.5 * np.sum(4 * (d ** -12 - d ** -6)), len(d)


def test_lattice_energy_and_shells(product, oracle):
    sim = make_sim(oracle, setup_lib=product, cells=(8, 8, 8))
    try:
        n = sim.n
        vol = sim.world[1] * sim.world[3] * sim.world[5]
        T, U, P = thermo(oracle, n, vol)
        u_ref, n25 = fcc_energy_per_atom(1.6796)
        assert T == pytest.approx(1.44, rel=1e-12)
        assert U == pytest.approx(u_ref, rel=1e-12)
        assert n25 == 54
        lists = tinymd.neighbor_lists(oracle, n)
        assert all(len(l) == 78 for l in lists)  # 12 + 6 + 24 + 12 + 24 within 2.8
        _, _, f = tinymd.full_state(oracle)
        assert np.abs(f).max() < 1e-10  # a perfect lattice is in equilibrium
    finally:
        sim.close()


@pytest.mark.slow
def test_minimd_published_thermo(product, oracle):
    """results/single_gpu_v100.txt:38-39 (miniMD, 64x64x32 unit cells, dt 0.001)."""
    oracle.oracle_set_ghost_mode(1)
    try:
        m, x, v, world, rank = tinymd.setup_particles("default", (64, 64, 32), MINIMD_LATTICE, lib=product)
        sim = tinymd.Simulation(oracle, m, x, v, world, rank, temp=1.44)
        vol = (world[1] - world[0]) * (world[3] - world[2]) * (world[5] - world[4])
        T0, U0, P0 = thermo(oracle, sim.n, vol)
        assert sim.n == 524288
        assert (f"{T0:.6e}", f"{U0:.6e}", f"{P0:.6e}") == ("1.440000e+00", "-6.773368e+00", "-5.019672e+00")
        sim.step(0.001, 100)
        T, U, P = thermo(oracle, sim.n, vol)
        assert (f"{T:.6e}", f"{U:.6e}", f"{P:.6e}") == ("7.192753e-01", "-5.698859e+00", "2.176028e-01")
        sim.close()
    finally:
        oracle.oracle_set_ghost_mode(0)


def test_half_list_semantics(product, oracle):
    """Reference half lists: j < i only, never a ghost; corrected mode equals the full-list force.

    Compared with exact periodic ghosts: the reference's lagged edge/corner
    ghosts make pair forces asymmetric, which no Newton-third-law half list
    can reproduce."""
    oracle.oracle_set_ghost_mode(1)
    full = make_sim(oracle, setup_lib=product, cells=(6, 6, 6))
    full.step(0.005, 10)
    x, v, ffull = tinymd.full_state(oracle)
    lfull = tinymd.neighbor_lists(oracle, full.n)
    n = full.n
    m0, x0, v0 = full._keep
    full.close()
    for mode in (0, 1):
        oracle.oracle_set_half_mode(mode)
        sim = make_sim(oracle, setup_lib=product, cells=(6, 6, 6), half=True)
        sim.step(0.005, 10)
        lh = tinymd.neighbor_lists(oracle, n)
        for i, l in enumerate(lh):
            assert set(l) <= set(lfull[i])
            if mode == 0:
                assert np.all(l < i)
        _, _, fh = tinymd.full_state(oracle)
        if mode == 1:
            assert rel_err(fh, ffull) < 1e-9
        else:
            assert rel_err(fh, ffull) > 1e-3  # boundary pairs are missing
        sim.close()
    oracle.oracle_set_half_mode(0)
    oracle.oracle_set_ghost_mode(0)


def test_exact_ghosts_are_periodic_images(product, oracle):
    oracle.oracle_set_ghost_mode(1)
    try:
        sim = make_sim(oracle, setup_lib=product, cells=(6, 6, 6))
        sim.step(0.005, 13)
        x, _, _ = tinymd.full_state(oracle)
        src, pbc, root, tsh = tinymd.ghost_info(oracle)
        L = sim.world[1::2] - sim.world[0::2]
        np.testing.assert_array_equal(x[sim.n:], x[root] + tsh * L)
        sim.close()
    finally:
        oracle.oracle_set_ghost_mode(0)


def test_lagged_ghosts_follow_two_phase_update(product, oracle):
    """comm/comm.impala:334-388: a chained ghost holds its source's previous value."""
    sim = make_sim(oracle, setup_lib=product, cells=(6, 6, 6))
    n = sim.n
    src, pbc, root, tsh = tinymd.ghost_info(oracle)
    L = sim.world[1::2] - sim.world[0::2]
    x_prev, _, _ = tinymd.full_state(oracle)
    sim.step(0.005, 1)
    x, _, _ = tinymd.full_state(oracle)
    for g in range(len(src)):
        s = src[g]
        expect = (x[s] if s < n else x_prev[s]) + pbc[g] * L
        np.testing.assert_array_equal(x[n + g], expect)
    sim.close()


def _reference_force(refsetup, x_all, lists, n):
    cap = max(len(l) for l in lists)
    nb = np.zeros((n, cap), dtype=np.int32)
    for i, l in enumerate(lists):
        nb[i, :len(l)] = l
    num = np.array([len(l) for l in lists], dtype=np.int32)
    f = np.zeros_like(x_all)
    fn = refsetup.compute_fullneigh
    fn.argtypes = [ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
    fn(n, 6.25, tinymd.ptr(np.ascontiguousarray(x_all)), tinymd.ptr(f), tinymd.ptr(nb), tinymd.ptr(num), cap)
    return f[:n]


def test_oracle_force_equals_reference_force_lj(product, oracle, refsetup):
    """core/force_lj.cpp (the reference's native kernel, sigma = eps = 1) vs the oracle, bit for bit."""
    sim = make_sim(oracle, setup_lib=product, cells=(4, 4, 4))
    sim.step(0.005, 7)
    x, _, f = tinymd.full_state(oracle)
    lists = tinymd.neighbor_lists(oracle, sim.n)
    fref = _reference_force(refsetup, x, lists, sim.n)
    sim.close()
    np.testing.assert_array_equal(f, fref)


def test_oracle_force_equals_golden_reference_output(product, oracle):
    path = os.path.join(GOLDEN, "force_lj_4x4x4_step7.npz")
    g = np.load(path)
    sim = make_sim(oracle, setup_lib=product, cells=(4, 4, 4))
    sim.step(0.005, 7)
    x, _, f = tinymd.full_state(oracle)
    sim.close()
    np.testing.assert_array_equal(x, g["positions"])
    np.testing.assert_array_equal(f, g["forces"])
