"""Parity at the benchmark's own sizes, beyond the small lattices of test_gpu_parity.py.

* the 'half' setup at 64x64x64 unit cells (524,288 atoms, lists of ~160 MB, larger than L2):
  FP64 lists equal the oracle's entry for entry after the first build, and positions,
  velocities and forces are bit-identical after 10 steps;
* DEM at 48x48x48 cells in both shapes (the FCC diagonal split, 223,488 atoms, and the
  reference's granular gas, 260,800 atoms) with the contact-fixed model: FP64 bit-identical to
  the oracle over 10 steps;
* the mixed form at the LJ workload's size (32x32x32 cells, 131,072 atoms): max |dF| / rms(F)
  <= 1e-5 and the potential energy per atom within 1e-6 relative of the FP64 form on the same
  positions, after 25 steps (one rebuild) of the liquid.

References: core/neighborlist.impala:18-78 (list order), core/runtime.impala:188-247 (LJ and
DEM closures), initialize.h:91-201 and 226-295 (the setups).
"""
import numpy as np
import pytest

import tinymd
from helpers import make_sim, rel_err

pytestmark = pytest.mark.gpu

DEM = (0.1, 0.1, 100.0, 0.5)  # damping_n, damping_t, stiffness, friction


def list_arrays(lib, n, capacity=128):
    """(sizes [n], lists [n, capacity]) in reference index space, entries past a size zeroed."""
    sizes = np.zeros(n, dtype=np.int32)
    lists = np.zeros((n, capacity), dtype=np.int32)
    if tinymd.is_oracle(lib):
        lib.oracle_neighbor_lists(tinymd.ptr(sizes), tinymd.ptr(lists), capacity)
    else:
        lib.md_get_neighbor_lists(tinymd.ptr(sizes), tinymd.ptr(lists), capacity)
        tinymd.check(lib)
    assert sizes.max() <= capacity
    lists[np.arange(capacity)[None, :] >= sizes[:, None]] = 0
    return sizes, lists


def assert_same_state(product, oracle, what):
    xp, vp, fp = tinymd.full_state(product)
    xo, vo, fo = tinymd.full_state(oracle)
    assert xp.shape == xo.shape, what
    np.testing.assert_array_equal(xp, xo, err_msg=f"positions, {what}")
    np.testing.assert_array_equal(vp, vo, err_msg=f"velocities, {what}")
    np.testing.assert_array_equal(fp, fo, err_msg=f"forces, {what}")
    return fp


def test_half_setup_64_cubed_lists_and_steps_bitwise(product, oracle):
    parts = tinymd.setup_particles("half", (64, 64, 64), lib=product)
    assert len(parts[0]) == 524288
    p = make_sim(product, particles=parts)
    o = make_sim(oracle, particles=parts)
    try:
        assert p.counts() == o.counts()
        sp, lp = list_arrays(product, p.n)
        so, lo = list_arrays(oracle, o.n)
        np.testing.assert_array_equal(sp, so)
        np.testing.assert_array_equal(lp, lo)
        assert_same_state(product, oracle, "initial")
        p.step(0.005, 10)
        o.step(0.005, 10)
        fp = assert_same_state(product, oracle, "after 10 steps")
        assert np.any(fp != 0.0)
    finally:
        p.close()
        o.close()


@pytest.mark.parametrize("setup,natoms", [("granular_gas_fcc", 223488), ("granular_gas", 260800)])
def test_dem_48_cubed_contact_model_bitwise(product, oracle, setup, natoms):
    product.md_set_dem_model(1, 0.6)
    oracle.oracle_set_dem_mode(1, 0.6)
    try:
        parts = tinymd.setup_particles(setup, (48, 48, 48), lib=product)
        assert len(parts[0]) == natoms
        kw = dict(force_field="dem", cutoff=1.2, skin=0.3, dem=DEM, temp=None, particles=parts)
        p, o = make_sim(product, **kw), make_sim(oracle, **kw)
        try:
            assert p.counts() == o.counts()
            p.step(0.001, 10)
            o.step(0.001, 10)
            fp = assert_same_state(product, oracle, "after 10 steps")
            if setup == "granular_gas_fcc":
                assert np.any(fp != 0.0)  # the lattice's nearest neighbours overlap at R = 0.6
        finally:
            p.close()
            o.close()
    finally:
        product.md_set_dem_model(0, 1.0)
        oracle.oracle_set_dem_mode(0, 1.0)


def test_mixed_force_and_energy_error_131k(product):
    """The error bound of the mixed form stated at the benchmark size (tolerance 1e-5 of the
    rms force; measured ~7.5e-6), on the liquid after one rebuild."""
    p = make_sim(product, cells=(32, 32, 32))
    try:
        product.md_set_precision(1)
        p.run(0.005, 25)
        product.md_set_thermo(1)
        th32, th64 = np.zeros(4), np.zeros(4)
        p.force()
        product.md_final_integration(0.0)
        assert product.md_get_thermo(tinymd.ptr(th32)) == 0
        _, _, f32 = tinymd.full_state(product)
        product.md_set_precision(0)
        p.force()
        product.md_final_integration(0.0)
        assert product.md_get_thermo(tinymd.ptr(th64)) == 0
        _, _, f64 = tinymd.full_state(product)
        err = rel_err(f32, f64)
        assert err <= 1e-5, err
        u32, u64 = th32[0] / p.n, th64[0] / p.n
        assert abs(u32 - u64) <= 1e-6 * abs(u64), (u32, u64)
    finally:
        product.md_set_thermo(0)
        product.md_set_precision(0)
        p.close()
