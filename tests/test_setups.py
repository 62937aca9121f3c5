"""The md driver's setups (product host code) against the reference's own generators.

Golden fixtures come from the reference's initialize.h compiled from its tree
(tests/golden/make_golden.py); when that build is present the comparison is
also run live on more sizes.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

import tinymd
from conftest import GOLDEN, ROOT

CASES = [("default", (4, 4, 4)), ("default", (5, 7, 6)), ("half", (6, 6, 6)), ("granular_gas", (6, 6, 6)),
         ("body_collision", (3, 3, 3))]


@pytest.mark.parametrize("bench,cells", CASES)
def test_setup_matches_reference_golden(product, bench, cells):
    g = np.load(os.path.join(GOLDEN, f"setup_{bench}_{'x'.join(map(str, cells))}.npz"))
    m, x, v, world, rank = tinymd.setup_particles(bench, cells, lib=product)
    np.testing.assert_array_equal(m, g["masses"])
    np.testing.assert_array_equal(x, g["positions"])
    np.testing.assert_array_equal(v, g["velocities"])
    np.testing.assert_array_equal(world, g["world"])
    np.testing.assert_array_equal(rank, g["rank"])


@pytest.mark.parametrize("bench,kind,cells", [("default", 0, (8, 8, 8)), ("default", 0, (32, 32, 32)),
                                              ("half", 0, (16, 16, 16)), ("granular_gas", 1, (20, 20, 20)),
                                              ("body_collision", 2, (6, 6, 6))])
def test_setup_matches_reference_live(product, refsetup, bench, kind, cells):
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import reference_setup
    d = reference_setup(refsetup, bench, kind, cells, 1.6796)
    m, x, v, world, rank = tinymd.setup_particles(bench, cells, lib=product)
    np.testing.assert_array_equal(x, d["positions"])
    np.testing.assert_array_equal(v, d["velocities"])
    np.testing.assert_array_equal(m, d["masses"])


def test_known_counts(product):
    assert len(tinymd.setup_particles("default", (8, 8, 8), lib=product)[0]) == 2048
    assert len(tinymd.setup_particles("default", (32, 32, 32), lib=product)[0]) == 131072
    # DEM diagonal split: FCC sites (i, j, k) on the half-spacing grid with i + j < 96: 48 * 96 * 97 / 2
    assert len(tinymd.setup_particles("granular_gas_fcc", (48, 48, 48), lib=product)[0]) == 223488


def test_velocity_stream_is_park_miller(product):
    """Velocities of site (i, j, k) are draws 6, 12, 18 of the Park-Miller stream seeded with the site index."""
    draws = np.load(os.path.join(GOLDEN, "park_miller_seed1.npy"))
    m, x, v, world, rank = tinymd.setup_particles("default", (4, 4, 4), lib=product)
    # site (0,0,0) has seed 1: its velocity components are draws 6, 12 and 18
    assert tuple(v[0]) == (draws[5], draws[11], draws[17])


def test_bench_cpu_lattice_is_the_reference_generator(product, refsetup):
    """bench.py's CPU arm takes its lattice from oracle/ref_lattice.py (the reference's own
    initialize.h, no product code): the same particles and boxes as the product's setup."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_lattice
    for bench, cells in (("default", (8, 8, 8)), ("half", (6, 6, 6))):
        got = ref_lattice.reference_lattice(cells, bench)
        want = tinymd.setup_particles(bench, cells, lib=product)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)
