"""Tiled full lists and the staged mixed force kernel against the per-cell path.

The tiled builder must write exactly the lists the per-cell builder writes (same
entries, same order), and the staged mixed kernel must reproduce the plain-list
mixed kernel's forces to FP32 summation-order differences (same pair
arithmetic), deterministically.  Builds whose shared-memory need exceeds the
limit go back to the per-cell path.
"""
import numpy as np
import pytest

import tinymd
from helpers import make_sim, rel_err

pytestmark = pytest.mark.gpu


def lists_and_state(product, tile, precision=0, steps=0, capacity=256, expect_tiles=None, **kw):
    product.md_set_tile_mode(tile)
    product.md_set_precision(precision)
    try:
        sim = make_sim(product, setup_lib=product, **kw)
        try:
            if steps:
                sim.run(0.005, steps)
            info = np.zeros(6, dtype=np.int32)
            product.md_tile_info(tinymd.ptr(info))
            if expect_tiles is not None:
                assert product.md_tiles_active() == (1 if (tile and expect_tiles) else 0), info
            elif tile:
                print(f"{kw}: tiled lists {'active' if product.md_tiles_active() else 'not used'}")
            lists = tinymd.neighbor_lists(product, sim.n, capacity)
            x, v, f = tinymd.full_state(product)
            return lists, x, v, f, info
        finally:
            sim.close()
    finally:
        product.md_set_tile_mode(0)
        product.md_set_precision(0)


@pytest.mark.parametrize("cells", [(8, 8, 8), (12, 7, 6), (2, 2, 2), (5, 7, 6), (3, 3, 3)])
def test_tiled_lists_equal_per_cell_lists(product, cells):
    """Lists of the tiled builder equal the per-cell builder's entry for entry, on cubic,
    elongated, odd and tiny grids (rows of one to eleven cells with locals)."""
    tiles = True
    a = lists_and_state(product, 1, cells=cells, expect_tiles=tiles)
    b = lists_and_state(product, 0, cells=cells, expect_tiles=tiles)
    assert len(a[0]) == len(b[0])
    for i, (la, lb) in enumerate(zip(a[0], b[0])):
        np.testing.assert_array_equal(la, lb, err_msg=f"atom {i}")


def staged_and_plain_forces(product, cells, steps):
    """Mixed-form forces on the same positions from the staged kernel (tiled lists) and from
    the plain-list kernel, after `steps` steps on the tiled path."""
    product.md_set_precision(1)
    product.md_set_tile_mode(1)
    try:
        sim = make_sim(product, setup_lib=product, cells=cells)
        try:
            if steps:
                sim.run(0.005, steps)
            assert product.md_tiles_active() == 1
            x, v, f_tile = tinymd.full_state(product)
            product.md_set_tile_mode(0)  # the next force call reads the plain list
            sim.force()
            product.md_final_integration(0.0)
            x2, v2, f_plain = tinymd.full_state(product)
            assert product.md_tiles_active() == 0
            np.testing.assert_array_equal(x, x2)
            np.testing.assert_array_equal(v, v2)
            return x, f_tile, f_plain
        finally:
            sim.close()
    finally:
        product.md_set_tile_mode(0)
        product.md_set_precision(0)


@pytest.mark.parametrize("cells,steps", [((8, 8, 8), 60), ((16, 16, 16), 20), ((32, 32, 32), 40)])
def test_staged_mixed_forces_match_plain_list(product, cells, steps):
    """Same pair arithmetic, other summation order: in the liquid (after 1-3 rebuilds) the
    staged kernel's forces agree with the plain-list mixed kernel's to 2e-6 of the rms force
    (the mixed form itself is within 1e-5 of FP64).  At the initial lattice the net forces
    nearly cancel (rms ~1e-6), so a relative measure there only shows FP32 rounding."""
    x, f_tile, f_plain = staged_and_plain_forces(product, cells, steps)
    assert rel_err(f_tile, f_plain) <= 2e-6, rel_err(f_tile, f_plain)


def test_staged_mixed_is_deterministic(product):
    """Two runs of 100 mixed steps on the tiled path give bit-identical trajectories (fixed
    reduction order, no atomics)."""
    a = lists_and_state(product, 1, precision=1, steps=100, cells=(8, 8, 8), expect_tiles=True)
    b = lists_and_state(product, 1, precision=1, steps=100, cells=(8, 8, 8), expect_tiles=True)
    for k, name in ((1, "positions"), (2, "velocities"), (3, "forces")):
        np.testing.assert_array_equal(a[k], b[k], err_msg=name)


def test_long_lists_fall_back(product):
    """A 5.0 cutoff at 6^3 unit cells (864 atoms, 6,949 ghosts): lists of ~530 entries and halos
    of thousands of atoms need more shared memory than the tiled builder may use, so the build
    finishes on the per-cell path with the same lists."""
    kw = {"cells": (6, 6, 6), "cutoff": 5.0}
    a = lists_and_state(product, 1, capacity=2048, expect_tiles=False, **kw)
    b = lists_and_state(product, 0, capacity=2048, expect_tiles=False, **kw)
    assert all(np.array_equal(la, lb) for la, lb in zip(a[0], b[0]))
    np.testing.assert_array_equal(a[3], b[3])


def test_halo_capacity_grows_and_stays_tiled(product):
    """8^3 unit cells with a 4.5 cutoff (2,048 atoms, 7,793 ghosts) and list capacity 400: the
    first tiled build meets halos above its initial capacity (2,560 atoms), the build is redone
    with a capacity that fits, and its lists equal the per-cell ones."""
    kw = {"cells": (8, 8, 8), "cutoff": 4.5, "nb_capacity": 400}
    a = lists_and_state(product, 1, capacity=1024, expect_tiles=True, **kw)
    assert a[4][1] > 2560 and a[4][2] > 2560, a[4]  # capacity grew past the initial one
    b = lists_and_state(product, 0, capacity=1024, expect_tiles=True, **kw)
    assert all(np.array_equal(la, lb) for la, lb in zip(a[0], b[0]))
    np.testing.assert_array_equal(a[3], b[3])
