"""Generates the golden fixtures of tests/golden from the reference's own code.

Needs oracle/_ref/libtinymd_refsetup.so, which `make -C oracle ref` compiles
from the reference tree (initialize.h and core/force_lj.cpp where they lie).
Run from the repository root:  python tests/golden/make_golden.py

Fixtures:
  setup_<benchmark>_<cells>.npz   masses / positions / velocities / boxes that
                                  the reference's generators hand to md_initialize_grid
  park_miller_seed1.npy           the reference generator's first 2000 draws from seed 1
  force_lj_4x4x4_step7.npz        positions (locals + ghosts) of the 256-atom lattice
                                  after 7 oracle steps and the forces the reference's
                                  compute_fullneigh (core/force_lj.cpp) gives on the
                                  oracle's neighbour lists
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "molecular-dynamics_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import tinymd  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "libtinymd_refsetup.so")
ORACLE = os.path.join(ROOT, "oracle", "_build", "libtinymd_oracle.so")

# (benchmark, kind for ref_generate, cells, potmin)
SETUPS = [("default", 0, (4, 4, 4), 1.6796), ("default", 0, (5, 7, 6), 1.6796), ("half", 0, (6, 6, 6), 1.6796),
          ("granular_gas", 1, (6, 6, 6), 1.6796), ("body_collision", 2, (3, 3, 3), 1.6796)]


def reference_setup(ref, benchmark, kind, cells, potmin):
    lib = tinymd.load()
    grid = np.array(cells, dtype=np.int32)
    world, a1, a2 = np.zeros(6), np.zeros(6), np.zeros(6)
    lib.tmd_setup_world(tinymd.BENCHMARKS[benchmark], tinymd.ptr(grid), potmin, tinymd.ptr(world), tinymd.ptr(a1),
                        tinymd.ptr(a2))
    rank = np.zeros(6)
    lib.tmd_setup_rank_box(tinymd.ptr(world), tinymd.ptr(rank))
    ref.ref_generate.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_double,
                                                                            ctypes.c_double]
    n = ref.ref_generate(kind, tinymd.ptr(world), tinymd.ptr(rank), tinymd.ptr(a1), tinymd.ptr(a2),
                         1 if benchmark == "half" else 0, potmin * 0.5, 2.8)
    m, x, v = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3))
    aabb, rk, caps = np.zeros(6), np.zeros(6), np.zeros(2, dtype=np.int32)
    sp = ctypes.c_double()
    ref.ref_captured.argtypes = [ctypes.c_void_p] * 5 + [ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    ref.ref_captured(tinymd.ptr(m), tinymd.ptr(x), tinymd.ptr(v), tinymd.ptr(aabb), tinymd.ptr(rk), ctypes.byref(sp),
                     tinymd.ptr(caps))
    return dict(masses=m, positions=x, velocities=v, world=aabb, rank=rk, cell_spacing=sp.value, capacities=caps)


def main():
    ref = ctypes.CDLL(REF)
    for bench, kind, cells, pot in SETUPS:
        d = reference_setup(ref, bench, kind, cells, pot)
        name = f"setup_{bench}_{'x'.join(map(str, cells))}.npz"
        np.savez_compressed(os.path.join(HERE, name), **d)
        print(name, len(d["masses"]))
    ref.ref_random.restype = ctypes.c_double
    ref.ref_random.argtypes = [ctypes.POINTER(ctypes.c_int)]
    st = ctypes.c_int(1)
    draws = np.array([ref.ref_random(ctypes.byref(st)) for _ in range(2000)])
    np.save(os.path.join(HERE, "park_miller_seed1.npy"), draws)

    from helpers import make_sim
    from test_oracle_pins import _reference_force
    ora = tinymd.open_library(ORACLE)
    ora.oracle_set_threads(1)
    sim = make_sim(ora, setup_lib=tinymd.load(), cells=(4, 4, 4))
    sim.step(0.005, 7)
    x, _, _ = tinymd.full_state(ora)
    lists = tinymd.neighbor_lists(ora, sim.n)
    f = _reference_force(ref, x, lists, sim.n)
    sim.close()
    np.savez_compressed(os.path.join(HERE, "force_lj_4x4x4_step7.npz"), positions=x, forces=f)
    print("force_lj_4x4x4_step7.npz", f.shape)


if __name__ == "__main__":
    main()
