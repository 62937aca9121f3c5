"""Helpers shared by the tests: run the same setup on the product and the oracle."""
import numpy as np

import tinymd


def make_sim(lib, benchmark="default", cells=(8, 8, 8), potmin=1.6796, half=False, temp=1.44, force_field="lj",
             cutoff=2.5, skin=0.3, dem=(0.0, 0.0, 0.0, 0.0), nb_capacity=100, setup_lib=None, reneigh=20,
             particles=None):
    m, x, v, world, rank = particles if particles is not None else tinymd.setup_particles(
        benchmark, cells, potmin, lib=setup_lib)
    if benchmark not in ("default", "half"):
        temp = None
    return tinymd.Simulation(lib, m, x, v, world, rank, cutoff=cutoff, skin=skin, half=half, temp=temp,
                             force_field=force_field, dem=dem, nb_capacity=nb_capacity, reneigh=reneigh)


def lists_as_sets(lists):
    return [set(map(int, l)) for l in lists]


def rel_err(a, b):
    """max |a-b| / rms(b) over all components."""
    rms = np.sqrt(np.mean(np.asarray(b) ** 2))
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / (rms if rms > 0 else 1.0))
