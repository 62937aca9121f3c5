"""Edge cases of the timestep on the GPU against the oracle: storage growth and an atom outside
the cell grid.

The reference grows its capacities on overflow and redoes the step
(core/grid.impala:183-213, core/neighborlist.impala:74-76); so do the library and the
oracle.  An atom outside the rank box extended by one cell is in no cell
(core/grid.impala:302); the library keeps it in an outside bucket, gives it an empty
list and latches MD_ERR_OUT_OF_GRID (5), a warning.
"""
import numpy as np
import pytest

import tinymd
from helpers import make_sim

pytestmark = pytest.mark.gpu


def run_both(product, oracle, steps, **kw):
    p = make_sim(product, setup_lib=product, **kw)
    o = make_sim(oracle, setup_lib=product, **kw)
    try:
        for chunk in range(steps // 10):
            p.step(0.005, 10)
            o.step(0.005, 10)
            xp, vp, fp = tinymd.full_state(product)
            xo, vo, fo = tinymd.full_state(oracle)
            np.testing.assert_array_equal(xp, xo, err_msg=f"positions after {10 * (chunk + 1)} steps")
            np.testing.assert_array_equal(vp, vo)
            np.testing.assert_array_equal(fp, fo)
        lp = tinymd.neighbor_lists(product, p.n)
        lo = tinymd.neighbor_lists(oracle, o.n)
        assert all(np.array_equal(a, b) for a, b in zip(lp, lo))
        return product.md_last_error()
    finally:
        p.close()
        o.close()


def test_list_capacity_growth(product, oracle):
    """List capacity 8 against ~78 neighbours: both grow and redo the build; 40 steps (2 rebuilds)
    stay bit-identical."""
    run_both(product, oracle, 40, cells=(6, 6, 6), nb_capacity=8)


def test_list_capacity_growth_at_a_rebuild(product, oracle):
    """List capacity 80: the lattice's 78 neighbours fit, the liquid's longest list at the first
    rebuild (step 20) does not.  The force kernel that the next step launches on those lists
    before their status is read returns without writing; the lists grow, are built again and the
    kernel runs again: 40 steps stay bit-identical."""
    run_both(product, oracle, 40, cells=(6, 6, 6), nb_capacity=80)


def test_ghost_capacity_growth(product, oracle):
    """2x2x2 unit cells: 32 atoms and 633 ghosts, far above the initial slot capacity; 40 steps
    bit-identical."""
    run_both(product, oracle, 40, cells=(2, 2, 2))


@pytest.mark.parametrize("bench,cells", [("body_collision", (6, 6, 6)), ("half", (10, 10, 10))])
def test_sparse_setups(product, oracle, bench, cells):
    """The md driver's sparse setups, 40 steps bit-identical: body_collision (two bodies in a
    world box extended by 20, mostly empty cells: initialize.h:297-362) and half (the lower half
    of the box in y filled)."""
    run_both(product, oracle, 40, benchmark=bench, cells=cells)


def test_atom_outside_the_grid(product, oracle):
    """One atom starts 5 length units beyond the upper x face (outside the box extended by one
    2.8 cell): it is in no cell and no list; its ghost image (shifted by -L) lies inside and is
    binned; the first rebuild wraps it back.  40 steps bit-identical, and the library latches
    the out-of-grid warning."""
    m, x, v, world, rank = tinymd.setup_particles("default", (6, 6, 6), lib=product)
    x = x.copy()
    x[0, 0] = world[1] + 5.0
    product.md_clear_error()
    code = run_both(product, oracle, 40, particles=(m, x, v, world, rank))
    assert code == 5
    product.md_clear_error()


def test_atom_outside_the_grid_at_a_later_build(product, oracle):
    """The atom outside the grid again, now at a list build inside the run: the lists are built
    without the periodic wrap (md_borders without md_enforce_pbc), so the atom stays outside; the
    fused force kernel that the next md_initial_integration launches on those lists before their
    status is read returns without writing, the outside atom's list is cleared and the kernel
    runs again.  The states stay bit-identical to the oracle's, and the warning is latched."""
    m, x, v, world, rank = tinymd.setup_particles("default", (6, 6, 6), lib=product)
    x = x.copy()
    x[0, 0] = world[1] + 5.0
    p = make_sim(product, setup_lib=product, particles=(m, x, v, world, rank))
    o = make_sim(oracle, setup_lib=product, particles=(m, x, v, world, rank))
    try:
        product.md_clear_error()
        for sim in (p, o):
            sim.step(0.005, 5)
        for sim, lib in ((p, product), (o, oracle)):
            sim.reneighbor(wrap=False)
            sim.force()
            lib.md_final_integration(0.005)
            lib.md_initial_integration(0.005)
            lib.md_synchronize_ghost_layer()
            sim.force()
            lib.md_final_integration(0.005)
        assert product.md_last_error() == 5
        product.md_clear_error()
        for sim in (p, o):
            sim.step(0.005, 10)
        xp, vp, fp = tinymd.full_state(product)
        xo, vo, fo = tinymd.full_state(oracle)
        np.testing.assert_array_equal(xp, xo)
        np.testing.assert_array_equal(vp, vo)
        np.testing.assert_array_equal(fp, fo)
    finally:
        p.close()
        o.close()
        product.md_clear_error()


@pytest.mark.parametrize("half,half_mode", [(False, 0), (True, 0), (True, 1)])
def test_dense_cells(product, oracle, half, half_mode):
    """A compressed lattice (a = 1.1: ~66 atoms per cell, ~280 neighbours each) makes the list
    build take a cell's homes in several batches of 32 lanes and grow the list capacity; the
    ghosts, the lists (full, the reference's half lists, half lists with boundary pairs) and the
    FP64 forces equal the oracle's."""
    product.md_set_half_mode(half_mode)
    oracle.oracle_set_half_mode(half_mode)
    p = make_sim(product, setup_lib=product, cells=(6, 6, 6), potmin=1.1, half=half)
    o = make_sim(oracle, setup_lib=product, cells=(6, 6, 6), potmin=1.1, half=half)
    try:
        assert product.md_get_number_of_ghost_particles() == oracle.md_get_number_of_ghost_particles()
        lp = tinymd.neighbor_lists(product, p.n, capacity=512)
        lo = tinymd.neighbor_lists(oracle, o.n, capacity=512)
        assert max(len(a) for a in lo) > 100  # beyond the initial capacity
        for a, b in zip(lp, lo):
            np.testing.assert_array_equal(a, b)
        _, _, fp = tinymd.full_state(product)
        _, _, fo = tinymd.full_state(oracle)
        if half:
            # reactions land by atomics, in another order: on the perfect lattice the net forces
            # cancel to ~1e-11 while single pair forces are ~1e3, so the order shows at ~1e-12
            # absolute; a missing or extra pair would show at ~1e3
            assert np.max(np.abs(fp - fo)) < 1e-9
        else:
            np.testing.assert_array_equal(fp, fo)
    finally:
        p.close()
        o.close()
        product.md_set_half_mode(0)
        oracle.oracle_set_half_mode(0)
