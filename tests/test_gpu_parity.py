"""Parity of the CUDA path against the CPU oracle, through the md_* C ABI.

Both libraries run the same calls on the same seeded lattice.  The FP64 form
with full lists is expected to be bit-identical to the oracle (same list
order, same operand order, no FMA contraction); half lists sum in a
different order (atomics) and are compared at 1e-12 relative.
"""
import numpy as np
import pytest

import tinymd
from helpers import lists_as_sets, make_sim, rel_err

pytestmark = pytest.mark.gpu


def both(product, oracle, **kw):
    a = make_sim(product, setup_lib=product, **kw)
    b = make_sim(oracle, setup_lib=product, **kw)
    return a, b


def close_all(*sims):
    for s in sims:
        s.close()


def assert_same_ghosts(product, oracle):
    gp, go = tinymd.ghost_info(product), tinymd.ghost_info(oracle)
    assert product.md_get_number_of_ghost_particles() == oracle.md_get_number_of_ghost_particles()
    for a, b, name in zip(gp, go, ("src", "pbc", "root", "tshift")):
        np.testing.assert_array_equal(a, b, err_msg=name)


@pytest.mark.parametrize("cells", [(8, 8, 8), (5, 7, 6)])
def test_initial_ghosts_lists_forces_bitwise(product, oracle, cells):
    p, o = both(product, oracle, cells=cells)
    try:
        assert p.counts() == o.counts()
        assert_same_ghosts(product, oracle)
        lp = tinymd.neighbor_lists(product, p.n)
        lo = tinymd.neighbor_lists(oracle, o.n)
        for i, (a, b) in enumerate(zip(lp, lo)):
            np.testing.assert_array_equal(a, b, err_msg=f"list of atom {i}")
        xp, vp, fp = tinymd.full_state(product)
        xo, vo, fo = tinymd.full_state(oracle)
        np.testing.assert_array_equal(xp, xo)
        np.testing.assert_array_equal(vp, vo)
        np.testing.assert_array_equal(fp, fo)
    finally:
        close_all(p, o)


def test_trajectory_bitwise_fp64_full(product, oracle):
    """100 steps (5 reneighbourings, lagged ghosts): positions, velocities, forces bit-identical."""
    p, o = both(product, oracle, cells=(8, 8, 8))
    try:
        for chunk in range(10):
            p.step(0.005, 10)
            o.step(0.005, 10)
            xp, vp, fp = tinymd.full_state(product)
            xo, vo, fo = tinymd.full_state(oracle)
            assert xp.shape == xo.shape
            np.testing.assert_array_equal(xp, xo, err_msg=f"positions after {10 * (chunk + 1)} steps")
            np.testing.assert_array_equal(vp, vo)
            np.testing.assert_array_equal(fp, fo)
        assert_same_ghosts(product, oracle)
        # the host-mirror path of the reference interface agrees too
        mp, xp2, vp2, fp2 = p.arrays()
        mo, xo2, vo2, fo2 = o.arrays()
        np.testing.assert_array_equal(mp, mo)
        np.testing.assert_array_equal(xp2, xo2)
        np.testing.assert_array_equal(vp2, vo2)
        np.testing.assert_array_equal(fp2, fo2)
        gp, go = p.ghost_arrays(), o.ghost_arrays()
        np.testing.assert_array_equal(gp[1], go[1])
    finally:
        close_all(p, o)


@pytest.mark.parametrize("precision", [0, 1])
def test_thermo_sums_match_oracle(product, oracle, precision):
    """md_get_thermo = {U sum, virial sum, pairs inside the cutoff, v.v} against the oracle's
    energy, virial and temperature at step 0 and after 20 and 40 steps (driver loop and native
    loop).  The device reductions sum in another order, so FP64 agrees to 1e-12 relative; the
    mixed form's pair energies carry its FP32 force error."""
    product.md_set_precision(precision)
    product.md_set_thermo(1)
    p, o = both(product, oracle, cells=(8, 8, 8))
    tol = 1e-12 if precision == 0 else 1e-5
    try:
        n = p.n
        t, to = np.zeros(4), np.zeros(2)
        for stage in range(3):
            if stage == 0:
                p.force()
                product.md_final_integration(0.0)
            elif stage == 1:
                p.step(0.005, 20)
                o.step(0.005, 20)
            else:
                p.run(0.005, 20)
                o.step(0.005, 20)
            assert product.md_get_thermo(tinymd.ptr(t)) == 0
            oracle.oracle_last_thermo(tinymd.ptr(to))
            temp = oracle.oracle_temperature()
            assert t[0] == pytest.approx(to[0], rel=tol), stage
            assert t[1] == pytest.approx(to[1], rel=tol * 10), stage
            assert t[3] / (3.0 * n - 3.0) == pytest.approx(temp, rel=1e-12 if precision == 0 else 1e-6), stage
            assert t[2] == float(round(t[2])) and t[2] > 0
    finally:
        close_all(p, o)
        product.md_set_thermo(0)
        product.md_set_precision(0)


def test_trajectory_exact_ghosts(product, oracle):
    product.md_set_ghost_mode(1)
    oracle.oracle_set_ghost_mode(1)
    p, o = both(product, oracle, cells=(6, 6, 6))
    try:
        p.step(0.005, 45)
        o.step(0.005, 45)
        xp, vp, fp = tinymd.full_state(product)
        xo, vo, fo = tinymd.full_state(oracle)
        np.testing.assert_array_equal(xp, xo)
        np.testing.assert_array_equal(vp, vo)
    finally:
        close_all(p, o)
        product.md_set_ghost_mode(0)
        oracle.oracle_set_ghost_mode(0)


@pytest.mark.parametrize("mode", ["full", "exact_ghosts", "half"])
def test_native_loop_matches_oracle(product, oracle, mode):
    """md_run_timesteps, the loop the benchmark times (the force held back and joined with the next
    initial integration and the ghost images; for half lists the final kick joined with it),
    against the oracle's step-by-step calls over 60 steps (3 rebuilds): bit-identical with full
    lists, to 1e-10 with half lists (reactions by atomics, another summation order).  The half
    lists keep the periodic-boundary pairs: with the reference's half lists, which drop them, two
    atoms can overlap across the boundary unrepelled until a wrap makes them list neighbours, and
    the kick that follows throws one out of the grid (the oracle does the same)."""
    if mode == "exact_ghosts":
        product.md_set_ghost_mode(1)
        oracle.oracle_set_ghost_mode(1)
    half = mode == "half"
    if half:
        product.md_set_half_mode(1)
        oracle.oracle_set_half_mode(1)
    product.md_clear_error()
    p, o = both(product, oracle, cells=(6, 6, 6), half=half)
    try:
        for chunk in range(3):
            p.run(0.005, 20)
            o.step(0.005, 20)
            assert product.md_last_error() == 0, (chunk, product.md_last_error())
            xp, vp, fp = tinymd.full_state(product)
            xo, vo, fo = tinymd.full_state(oracle)
            if half:
                assert rel_err(xp, xo) < 1e-10 and rel_err(vp, vo) < 1e-10 and rel_err(fp, fo) < 1e-10
            else:
                np.testing.assert_array_equal(xp, xo, err_msg=f"positions after {20 * (chunk + 1)} steps")
                np.testing.assert_array_equal(vp, vo)
                np.testing.assert_array_equal(fp, fo)
    finally:
        close_all(p, o)
        product.md_set_ghost_mode(0)
        oracle.oracle_set_ghost_mode(0)
        product.md_set_half_mode(0)
        oracle.oracle_set_half_mode(0)
        product.md_clear_error()


def test_half_lists(product, oracle):
    p, o = both(product, oracle, cells=(8, 8, 8), half=True)
    try:
        lp = tinymd.neighbor_lists(product, p.n)
        lo = tinymd.neighbor_lists(oracle, o.n)
        for a, b in zip(lp, lo):
            np.testing.assert_array_equal(a, b)
            assert np.all(a < p.n)  # the reference's half lists hold no ghosts
        _, _, fp = tinymd.full_state(product)
        _, _, fo = tinymd.full_state(oracle)
        assert rel_err(fp, fo) < 1e-12
        p.step(0.005, 10)
        o.step(0.005, 10)
        xp, vp, fp = tinymd.full_state(product)
        xo, vo, fo = tinymd.full_state(oracle)
        assert rel_err(xp, xo) < 1e-10
        assert rel_err(fp, fo) < 1e-10
    finally:
        close_all(p, o)


def test_mixed_force_error(product, oracle):
    """Mixed form on the FP64 form's own positions: max |dF| / rms(F) <= 1e-5."""
    p = make_sim(product, setup_lib=product, cells=(8, 8, 8))
    try:
        p.step(0.005, 60)
        _, _, f64 = tinymd.full_state(product)
        product.md_set_precision(1)
        p.force()
        product.md_final_integration(0.0)
        _, _, f32 = tinymd.full_state(product)
        err = rel_err(f32, f64)
        assert err <= 1e-5, err
    finally:
        product.md_set_precision(0)
        p.close()


def test_mixed_force_error_dense(product, oracle):
    """Mixed form on a compressed lattice (a = 1.3: the 12 nearest neighbours at ~0.92 sigma all
    take the FP64 path, spread over more list quads than a thread queues, so the kernel redoes
    such atoms with the FP64 pairs in place): max |dF| / rms(F) <= 1e-5 against the FP64 forces
    on the same positions."""
    p = make_sim(product, setup_lib=product, cells=(6, 6, 6), potmin=1.3, nb_capacity=256)
    try:
        p.step(0.005, 10)
        x, _, f64 = tinymd.full_state(product)
        lists = tinymd.neighbor_lists(product, p.n, capacity=512)
        most = 0  # list quads holding a pair closer than 1.04 sigma, per atom
        for i, l in enumerate(lists):
            d = x[l] - x[i]
            close = np.nonzero(np.einsum("ij,ij->i", d, d) < 1.04 ** 2)[0]
            most = max(most, len(set((close // 4).tolist())))
        assert most > 8, most
        product.md_set_precision(1)
        p.force()
        product.md_final_integration(0.0)
        _, _, f32 = tinymd.full_state(product)
        err = rel_err(f32, f64)
        assert err <= 1e-5, err
    finally:
        product.md_set_precision(0)
        p.close()


@pytest.mark.parametrize("half_mode", [0, 1])
def test_mixed_half_list_force_error(product, oracle, half_mode):
    """Mixed form over half lists (the reference's, and those keeping boundary pairs): the forces,
    reactions included, within 1e-5 of rms of the FP64 half-list forces on the same positions
    (15 steps: before the first rebuild, after which the reference's half lists let atoms overlap
    across the boundary)."""
    product.md_set_half_mode(half_mode)
    p = make_sim(product, setup_lib=product, cells=(8, 8, 8), half=True)
    try:
        p.step(0.005, 15)
        _, _, f64 = tinymd.full_state(product)
        product.md_set_precision(1)
        p.force()
        product.md_final_integration(0.0)
        _, _, f32 = tinymd.full_state(product)
        err = rel_err(f32, f64)
        assert err <= 1e-5, err
    finally:
        product.md_set_precision(0)
        product.md_set_half_mode(0)
        p.close()


def test_half_lists_with_ghost_pairs(product, oracle):
    """Corrected half mode: lists equal the oracle's; forces equal the full-list forces."""
    product.md_set_half_mode(1)
    oracle.oracle_set_half_mode(1)
    try:
        p, o = both(product, oracle, cells=(8, 8, 8), half=True)
        try:
            lp = tinymd.neighbor_lists(product, p.n)
            lo = tinymd.neighbor_lists(oracle, o.n)
            for a, b in zip(lp, lo):
                np.testing.assert_array_equal(a, b)
            _, _, fp = tinymd.full_state(product)
            _, _, fo = tinymd.full_state(oracle)
            assert np.abs(fp - fo).max() < 1e-12  # perfect lattice: forces are rounding noise
            p.step(0.005, 45)
            o.step(0.005, 45)
            xp, _, fp = tinymd.full_state(product)
            xo, _, fo = tinymd.full_state(oracle)
            assert rel_err(xp, xo) < 1e-10 and rel_err(fp, fo) < 1e-9
        finally:
            close_all(p, o)
        # same physics as the full list (exact periodic ghosts keep pair forces symmetric)
        product.md_set_ghost_mode(1)
        f = make_sim(product, setup_lib=product, cells=(8, 8, 8))
        f.step(0.005, 25)
        _, _, ffull = tinymd.full_state(product)
        f.close()
        h = make_sim(product, setup_lib=product, cells=(8, 8, 8), half=True)
        h.step(0.005, 25)
        _, _, fhalf = tinymd.full_state(product)
        h.close()
        assert rel_err(fhalf, ffull) < 1e-10
    finally:
        product.md_set_half_mode(0)
        product.md_set_ghost_mode(0)
        oracle.oracle_set_half_mode(0)


@pytest.mark.parametrize("precision", [0, 1])
def test_131k_workload_stable_and_matches_oracle_lists(product, oracle, precision):
    """The benchmark workload: lists equal the oracle's after reneighbouring, and in the FP64 form
    positions, velocities and forces equal the oracle's bit for bit after 40 steps (two rebuilds);
    energy stays bounded over 420 steps."""
    product.md_set_precision(precision)
    try:
        p = make_sim(product, setup_lib=product, cells=(32, 32, 32))
        o = make_sim(oracle, setup_lib=product, cells=(32, 32, 32))
        p.step(0.005, 40)
        o.step(0.005, 40)
        lp = tinymd.neighbor_lists(product, p.n)
        lo = tinymd.neighbor_lists(oracle, o.n)
        if precision == 0:
            for a, b in zip(lp, lo):
                np.testing.assert_array_equal(a, b)
            xp, vp, fp = tinymd.full_state(product)
            xo, vo, fo = tinymd.full_state(oracle)
            np.testing.assert_array_equal(xp, xo)
            np.testing.assert_array_equal(vp, vo)
            np.testing.assert_array_equal(fp, fo)
        o.close()
        p.run(0.005, 380)
        _, v, _ = tinymd.full_state(product)
        t = float((v ** 2).sum() / (3 * p.n - 3))
        assert 0.5 < t < 1.2, t
        assert product.md_last_error() == 0
        p.close()
    finally:
        product.md_set_precision(0)
