"""Device timing controls on the GPU: phase times and sampled kernel profiling.

A CUDA event recorded between two kernels costs the stream a few microseconds, so
the library records phase boundaries only when md_set_phase_timing(1) asks for
them (the md driver does, for its time report), and md_profile_sample(n) times
one launch in n of each profiled kernel.
"""
import ctypes

import numpy as np
import pytest

from helpers import make_sim

pytestmark = pytest.mark.gpu


def phase_times(lib):
    out = np.zeros(6)
    lib.md_get_phase_times(out.ctypes.data_as(ctypes.c_void_p))
    return out


def test_phase_times_only_when_enabled(product):
    """40 steps (two rebuilds) through the md_* calls: no phase times by default; with phase
    timing on, force and neighbour-list time are positive and the buckets add up to the total."""
    sim = make_sim(product, cells=(8, 8, 8))
    try:
        sim.step(0.005, 40)
        product.md_synchronize()
        assert np.all(phase_times(product) == 0.0)
    finally:
        sim.close()
    product.md_set_phase_timing(1)
    try:
        sim = make_sim(product, cells=(8, 8, 8))
        try:
            sim.step(0.005, 40)
            product.md_synchronize()
            t = phase_times(product)
            assert t[1] > 0.0 and t[2] > 0.0  # force, neighbour lists
            assert t[0] == pytest.approx(t[1:].sum(), rel=1e-9)
        finally:
            sim.close()
    finally:
        product.md_set_phase_timing(0)


def test_profile_sampling_times_one_launch_in_n(product):
    """The same 40 native steps timed with every force launch, then with one in ten."""
    counts = []
    for every in (1, 10):
        sim = make_sim(product, cells=(8, 8, 8))
        try:
            product.md_profile_enable(1 << 0)
            product.md_profile_sample(every)
            product.md_profile_reset()
            sim.run(0.005, 40)
            launches, ms = ctypes.c_longlong(), ctypes.c_double()
            product.md_profile_get(0, ctypes.byref(launches), ctypes.byref(ms))
            counts.append(launches.value)
            assert ms.value > 0.0
        finally:
            product.md_profile_enable(0)
            product.md_profile_sample(1)
            sim.close()
    assert counts[0] >= 40
    assert counts[1] == (counts[0] + 9) // 10
