"""Benchmark lattices from the reference's own generator (TEST INFRASTRUCTURE ONLY).

The CPU arm of bench.py needs the benchmark's initial state without touching the product
library.  This module calls the reference's setup code itself, compiled from its tree into
oracle/_ref/libtinymd_refsetup.so by `make -C oracle ref` (oracle/ref_harness.cpp wraps
initialize.h:91-201): the world box of a 'default' or 'half' run is [0, cells * a] per axis
(main.cpp:513-519), the rank box is the world box on one process, and the lattice comes from
init_rectangular_grid with the lattice spacing a / 2 and the cell spacing 2.8, as
main.cpp:664-674 calls it.  The velocity rescale to T = 1.44 is the oracle's own
md_create_velocity, so nothing here runs product code.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SETUP = os.path.join(HERE, "_ref", "libtinymd_refsetup.so")


def available():
    return os.path.exists(REF_SETUP)


def reference_lattice(cells, benchmark="default", potmin=1.6796, cell_spacing=2.8):
    """(masses [n], positions [n, 3], velocities [n, 3], world [6], rank [6]) of a 'default' or
    'half' benchmark lattice as the reference generates it."""
    if benchmark not in ("default", "half"):
        raise ValueError(benchmark)
    if not available():
        raise FileNotFoundError(REF_SETUP + " is not built (make -C oracle ref, needs the reference tree)")
    ref = ctypes.CDLL(REF_SETUP, mode=ctypes.RTLD_LOCAL)
    vp = ctypes.c_void_p
    ref.ref_generate.argtypes = [ctypes.c_int, vp, vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    ref.ref_generate.restype = ctypes.c_int
    ref.ref_captured.argtypes = [vp] * 5 + [ctypes.POINTER(ctypes.c_double), vp]
    ref.ref_captured.restype = ctypes.c_int
    world = np.zeros(6)
    for d in range(3):
        world[2 * d + 1] = cells[d] * potmin
    rank = world.copy()
    a1, a2 = np.zeros(6), np.zeros(6)

    def p(a):
        return a.ctypes.data_as(vp)

    n = ref.ref_generate(0, p(world), p(rank), p(a1), p(a2), 1 if benchmark == "half" else 0, potmin * 0.5,
                         cell_spacing)
    m, x, v = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3))
    aabb, rk, caps = np.zeros(6), np.zeros(6), np.zeros(2, dtype=np.int32)
    sp = ctypes.c_double()
    ref.ref_captured(p(m), p(x), p(v), p(aabb), p(rk), ctypes.byref(sp), p(caps))
    return m, x, v, aabb, rk
