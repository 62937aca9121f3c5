"""The DEM force (core/runtime.impala:203-247) on the GPU against the oracle.

Two models: the reference closure, whose contact branch cannot run (the force is
zero everywhere), and the contact-fixed spring-dashpot model selected with
md_set_dem_model(1, R).  The workload is the granular-gas FCC setup with the
parameters of the DEM benchmark configuration: cutoff 1.2, skin 0.3, dt 0.001,
stiffness 100, normal and tangential damping 0.1, friction 0.5, initial
velocities zero.  With R = 0.6 nearest lattice neighbours (1.1877 apart)
overlap, so contacts push the lattice apart from the first step.
"""
import numpy as np
import pytest

import tinymd
from helpers import make_sim, rel_err

pytestmark = pytest.mark.gpu

DEM = (0.1, 0.1, 100.0, 0.5)  # damping_n, damping_t, stiffness, friction
DT = 0.001


def dem_sim(lib, cells=(12, 12, 12), half=False):
    return make_sim(lib, benchmark="granular_gas_fcc", cells=cells, force_field="dem", cutoff=1.2, skin=0.3,
                    dem=DEM, half=half)


def set_model(product, oracle, fixed, radius=0.6):
    product.md_set_dem_model(fixed, radius)
    if oracle is not None:
        oracle.oracle_set_dem_mode(fixed, radius)


@pytest.fixture
def reset_dem(product, oracle):
    yield
    product.md_set_dem_model(0, 1.0)
    oracle.oracle_set_dem_mode(0, 1.0)
    product.md_set_precision(0)
    product.md_set_half_mode(0)


@pytest.mark.parametrize("precision", [0, 1])
def test_reference_closure_force_is_zero(product, oracle, reset_dem, precision):
    """The reference's contact branch needs r - 2R > 0 inside r < 2R: never.  Forces are zero
    in both forms and the lattice (at rest) stays where it is, as in the oracle."""
    set_model(product, oracle, 0)
    product.md_set_precision(precision)
    p, o = dem_sim(product), dem_sim(oracle)
    try:
        p.step(DT, 25)
        o.step(DT, 25)
        xp, vp, fp = tinymd.full_state(product)
        xo, vo, fo = tinymd.full_state(oracle)
        assert np.all(fp == 0.0) and np.all(fo == 0.0)
        np.testing.assert_array_equal(xp, xo)
        np.testing.assert_array_equal(vp, vo)
    finally:
        p.close()
        o.close()


def test_contact_model_fp64_bitwise(product, oracle, reset_dem):
    """Contact-fixed model, FP64 form: 45 steps (two list rebuilds) bit-identical to the oracle."""
    set_model(product, oracle, 1, 0.6)
    p, o = dem_sim(product), dem_sim(oracle)
    try:
        for chunk in range(3):
            p.step(DT, 15)
            o.step(DT, 15)
            xp, vp, fp = tinymd.full_state(product)
            xo, vo, fo = tinymd.full_state(oracle)
            assert np.any(fp != 0.0)
            np.testing.assert_array_equal(xp, xo, err_msg=f"positions after {15 * (chunk + 1)} steps")
            np.testing.assert_array_equal(vp, vo)
            np.testing.assert_array_equal(fp, fo)
    finally:
        p.close()
        o.close()


@pytest.mark.parametrize("cells", [(12, 12, 12), (24, 24, 24)])
def test_contact_model_mixed_forces(product, reset_dem, cells):
    """Mixed form (FP32 pair arithmetic on rebased positions, FP64 at the contact and cutoff
    decisions): forces on the same state agree with the FP64 form's to 1e-4 of the rms force
    (measured 4.6e-5 and 5.4e-5; 7.5e-5 at 48^3).  The normal force is k (2R - r) with overlaps of ~0.012 here:
    r carries ~1e-7 from the FP32 pair arithmetic, so the overlap itself is only good to
    ~1e-5 relative -- a cancellation that the LJ form does not have."""
    set_model(product, None, 1, 0.6)
    sim = dem_sim(product, cells=cells)
    try:
        sim.step(DT, 30)
        product.md_set_precision(0)
        sim.force()
        product.md_final_integration(0.0)
        _, _, f64 = tinymd.full_state(product)
        product.md_set_precision(1)
        sim.force()
        product.md_final_integration(0.0)
        _, _, f32 = tinymd.full_state(product)
        assert np.sqrt(np.mean(f64 ** 2)) > 0.0
        assert rel_err(f32, f64) <= 1e-4, rel_err(f32, f64)
    finally:
        sim.close()


def test_contact_model_mixed_trajectory_close(product, oracle, reset_dem):
    """30 mixed steps (one rebuild) keep the locals within 1e-6 of the oracle's FP64 positions
    (minimum image: an atom at the box face may wrap in one run and not in the other)."""
    set_model(product, oracle, 1, 0.6)
    product.md_set_precision(1)
    p, o = dem_sim(product), dem_sim(oracle)
    try:
        p.step(DT, 30)
        o.step(DT, 30)
        n = p.n
        xp, _, _ = tinymd.full_state(product)
        xo, _, _ = tinymd.full_state(oracle)
        box = p.world[1::2] - p.world[0::2]
        d = xp[:n] - xo[:n]
        d -= box * np.round(d / box)
        assert np.max(np.abs(d)) <= 1e-6, np.max(np.abs(d))
    finally:
        p.close()
        o.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_contact_model_half_lists(product, reset_dem, precision):
    """Half lists that keep the periodic-boundary pairs (reactions to the roots) give the
    full-list forces: to 1e-12 in FP64, to the FP32 tolerance in the mixed form."""
    set_model(product, None, 1, 0.6)
    product.md_set_precision(precision)
    product.md_set_ghost_mode(1)
    try:
        full = dem_sim(product)
        try:
            full.step(DT, 10)
            xf, _, ff = tinymd.full_state(product)
        finally:
            full.close()
        product.md_set_half_mode(1)
        half = dem_sim(product, half=True)
        try:
            half.step(DT, 10)
            xh, _, fh = tinymd.full_state(product)
        finally:
            half.close()
        tol = 1e-12 if precision == 0 else 1e-5
        assert np.max(np.abs(xh - xf)) <= (1e-12 if precision == 0 else 1e-6)
        assert rel_err(fh, ff) <= tol, rel_err(fh, ff)
    finally:
        product.md_set_ghost_mode(0)
