"""Host-side copies that do not stall the stream, against the synchronous ones.

* md_copy_data_from_accelerator takes a snapshot (core/grid.impala:369-374): whatever runs
  afterwards, md_write_grid_data_to_arrays and md_write_grid_ghost_data_to_arrays return the
  state as it was at that call, also across a rebuild that grows the slot arrays.
* md_thermo_request / md_thermo_fetch return the same sums md_get_thermo gives at the same
  point of the run, fetched after later steps were enqueued.
"""
import numpy as np
import pytest

import tinymd
from helpers import make_sim

pytestmark = pytest.mark.gpu


def ghost_arrays(lib):
    g = lib.md_get_number_of_ghost_particles()
    m, x, v, f = np.zeros(g), np.zeros((g, 3)), np.zeros((g, 3)), np.zeros((g, 3))
    lib.md_write_grid_ghost_data_to_arrays(tinymd.ptr(m), tinymd.ptr(x), tinymd.ptr(v), tinymd.ptr(f))
    return m, x, v, f


@pytest.mark.parametrize("precision", [0, 1])
def test_copy_from_accelerator_is_a_snapshot(product, precision):
    product.md_set_precision(precision)
    try:
        sim = make_sim(product, cells=(6, 6, 6))
        sim.step(0.005, 7)
        x_ref, v_ref, f_ref = tinymd.full_state(product)
        n = sim.n
        product.md_copy_data_from_accelerator()
        g0 = product.md_get_number_of_ghost_particles()
        sim.step(0.005, 25)  # one rebuild in between; the state moves on
        m, x, v, f = np.empty(n), np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        assert product.md_write_grid_data_to_arrays(tinymd.ptr(m), tinymd.ptr(x), tinymd.ptr(v), tinymd.ptr(f)) == n
        np.testing.assert_array_equal(x, x_ref[:n])
        np.testing.assert_array_equal(v, v_ref)
        np.testing.assert_array_equal(f, f_ref)
        assert np.all(m == 1.0)
        x_now, _, _ = tinymd.full_state(product)
        assert not np.array_equal(x_now[:n], x_ref[:n])
        # a fresh snapshot's ghosts equal the ghost positions of the full state
        product.md_copy_data_from_accelerator()
        xg = tinymd.full_state(product)[0][n:]
        gm, gx, gv, gf = ghost_arrays(product)
        np.testing.assert_array_equal(gx, xg)
        assert len(gm) == product.md_get_number_of_ghost_particles() and g0 > 0
        sim.close()
    finally:
        product.md_set_precision(0)


def test_snapshot_survives_slot_growth(product):
    """2^3 unit cells: the first rebuild multiplies the ghosts and grows the slot arrays (whose
    allocation also holds the device copy of the snapshot)."""
    sim = make_sim(product, cells=(2, 2, 2))
    n = sim.n
    x_ref, v_ref, f_ref = tinymd.full_state(product)
    product.md_copy_data_from_accelerator()
    sim.step(0.005, 45)
    m, x, v, f = np.empty(n), np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
    product.md_write_grid_data_to_arrays(tinymd.ptr(m), tinymd.ptr(x), tinymd.ptr(v), tinymd.ptr(f))
    np.testing.assert_array_equal(x, x_ref[:n])
    np.testing.assert_array_equal(v, v_ref)
    np.testing.assert_array_equal(f, f_ref)
    sim.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_thermo_request_matches_synchronous_read(product, precision):
    product.md_set_precision(precision)
    product.md_set_thermo(1)
    try:
        sums = {}
        for mode in ("sync", "async"):
            sim = make_sim(product, cells=(6, 6, 6))
            tickets, got = [], []
            for chunk in range(4):
                sim.step(0.005, 10)
                if mode == "sync":
                    t = np.zeros(4)
                    assert product.md_get_thermo(tinymd.ptr(t)) == 0
                    got.append(t)
                else:
                    tickets.append(product.md_thermo_request())
            for tk in tickets:
                t = np.zeros(4)
                assert product.md_thermo_fetch(tk, tinymd.ptr(t)) == 0
                got.append(t)
            sums[mode] = np.array(got)
            sim.close()
        np.testing.assert_array_equal(sums["async"], sums["sync"])
        assert np.all(sums["sync"][:, 2] > 0)  # pairs inside the cutoff
        t = np.zeros(4)
        assert product.md_thermo_fetch(12345, tinymd.ptr(t)) == -1  # never issued
        product.md_clear_error()
    finally:
        product.md_set_thermo(0)
        product.md_set_precision(0)
