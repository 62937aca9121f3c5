"""Python binding of the tinyMD B200 C ABI (include/tinymd_b200.h).

``load()`` opens the in-tree libtinymd_b200.so (building it first when it is
missing) and declares the argument types of every entry point.  The same
wrapper also opens any other library exporting the md_* interface, which is
how the tests drive the CPU oracle through identical calls.

``Simulation`` runs the md driver's sequence (main.cpp:664-776 of tinyMD) on
one library: setup, velocities, upload, borders, binning, lists, forces,
timesteps with reneighbouring.  ``tinymd.adjoint`` holds the differentiable
form (a torch.autograd.Function over the md_adjoint_* entry points).
"""
import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ROOT = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "lib", "libtinymd_b200.so")
MD_BINARY = os.path.join(PKG_DIR, "lib", "md")

BENCHMARKS = {"default": 0, "half": 1, "granular_gas": 2, "body_collision": 3, "granular_gas_fcc": 4}

_c_int, _c_double, _c_bool, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_bool, ctypes.c_void_p
_c_ll = ctypes.c_longlong

# name -> (restype, argtypes) of the reference interface (anydsl_includes.h:10-48)
_REFERENCE_API = {
    "md_initialize_grid": (_c_int, [_vp, _vp, _vp, _c_int, _vp, _vp, _c_double, _c_int, _c_int]),
    "md_rescale_grid": (None, [_vp]),
    "md_copy_data_from_accelerator": (None, []),
    "md_copy_data_to_accelerator": (None, []),
    "md_initial_integration": (None, [_c_double]),
    "md_final_integration": (None, [_c_double]),
    "md_enforce_pbc": (None, []),
    "md_write_grid_data_to_arrays": (_c_int, [_vp, _vp, _vp, _vp]),
    "md_write_grid_ghost_data_to_arrays": (_c_int, [_vp, _vp, _vp, _vp]),
    "md_write_grid_aabb_data_to_arrays": (_c_int, [_vp, _vp, _vp, _vp]),
    "md_distribute_particles": (None, []),
    "md_assemble_neighborlists": (None, [_c_bool, _c_double]),
    "md_deallocate_grid": (None, []),
    "md_create_velocity": (None, [_c_double]),
    "md_compute_lennard_jones": (None, [_c_bool, _c_double, _c_double, _c_double]),
    "md_compute_dem": (None, [_c_bool, _c_double, _c_double, _c_double, _c_double, _c_double]),
    "md_mpi_initialize": (None, []),
    "md_mpi_finalize": (None, []),
    "md_synchronize_ghost_layer": (None, []),
    "md_borders": (None, []),
    "md_exchange_particles": (None, []),
    "md_get_world_size": (_c_int, []),
    "md_get_world_rank": (_c_int, []),
    "md_get_number_of_particles": (_c_int, []),
    "md_get_number_of_ghost_particles": (_c_int, []),
    "md_get_node_bounding_box": (None, [_vp, _vp]),
    "md_report_iterations": (None, []),
    "md_report_particles": (None, []),
    "md_report_time": (None, [_c_double] * 6),
    "md_barrier": (None, []),
}

_EXTENSION_API = {
    "md_last_error": (_c_int, []),
    "md_last_error_string": (ctypes.c_char_p, []),
    "md_clear_error": (None, []),
    "md_set_precision": (None, [_c_int]),
    "md_set_ghost_mode": (None, [_c_int]),
    "md_set_half_mode": (None, [_c_int]),
    "md_set_dem_model": (None, [_c_int, _c_double]),
    "md_set_thermo": (None, [_c_int]),
    "md_get_thermo": (_c_int, [_vp]),
    "md_thermo_request": (_c_int, []),
    "md_thermo_fetch": (_c_int, [_c_int, _vp]),
    "md_synchronize": (None, []),
    "md_set_stream": (None, [_vp]),
    "md_get_phase_times": (None, [_vp]),
    "md_profile_enable": (None, [_c_int]),
    "md_profile_sample": (None, [_c_int]),
    "md_set_phase_timing": (None, [_c_int]),
    "md_profile_count": (_c_int, []),
    "md_profile_name": (ctypes.c_char_p, [_c_int]),
    "md_profile_get": (_c_int, [_c_int, ctypes.POINTER(_c_ll), ctypes.POINTER(_c_double)]),
    "md_profile_reset": (None, []),
    "md_kernel_launches": (_c_ll, []),
    "md_device_bytes": (_c_ll, []),
    "md_get_neighbor_lists": (_c_int, [_vp, _vp, _c_int]),
    "md_get_ghost_info": (_c_int, [_vp, _vp, _vp, _vp]),
    "md_get_state": (_c_int, [_vp, _vp, _vp]),
    "md_set_positions": (_c_int, [_vp]),
    "md_set_velocities": (_c_int, [_vp]),
    "md_get_cell_sizes": (_c_int, [_vp, _c_int]),
    "md_get_grid_info": (_c_int, [_vp]),
    "md_run_timesteps": (_c_int, [_c_int, _c_double, _c_int, _c_int, _c_double, _vp, _vp, _c_ll]),
    "md_lj_forces_noalloc": (_c_int, [_vp, _c_int, _vp, _vp, _c_int, _c_int, _c_double, _c_double, _c_double, _vp,
                                      _vp, _vp]),
    "tmd_setup_world": (_c_int, [_c_int, _vp, _c_double, _vp, _vp, _vp]),
    "tmd_setup_rank_box": (None, [_vp, _vp]),
    "tmd_setup_generate": (_c_int, [_c_int, _vp, _vp, _vp, _vp, _c_double]),
    "tmd_setup_fetch": (_c_int, [_vp, _vp, _vp]),
    "tmd_setup_initialize": (_c_int, [_vp, _vp, _c_double, _c_int, _c_int]),
    "tmd_node_config": (_c_int, [_c_int, _vp, _vp]),
    "tmd_topology": (_c_int, [_c_int, _vp, _vp, _vp, _vp]),
    "tmd_comm_transport": (ctypes.c_char_p, []),
    "tmd_halo_info": (_c_int, [_vp]),
    "tmd_comm_nccl_selftest": (_c_int, [_c_ll]),
    "tmd_comm_allreduce_sum": (_c_int, [_vp, _c_int]),
    "tmd_comm_sendrecv": (_c_int, [_c_int, _vp, _c_ll, _c_int, _vp, _c_ll]),
    "md_adjoint_configure": (_c_int, [_c_int, _c_int, _c_double, _c_double, _c_double, _c_int]),
    "md_adjoint_forward": (_c_int, [_vp, _c_double, _c_double, _vp]),
    "md_adjoint_backward": (_c_int, [_vp, _vp, _vp]),
    "md_adjoint_times": (_c_int, [_vp, _vp]),
    "md_adjoint_set_loss": (_c_int, [_c_int]),
}

_ORACLE_API = {
    "oracle_set_ghost_mode": (None, [_c_int]),
    "oracle_set_half_mode": (None, [_c_int]),
    "oracle_set_dem_mode": (None, [_c_int, _c_double]),
    "oracle_set_threads": (None, [_c_int]),
    "oracle_max_threads": (_c_int, []),
    "oracle_temperature": (_c_double, []),
    "oracle_grid_info": (None, [_vp]),
    "oracle_aabb": (None, [_vp]),
    "oracle_positions": (None, [_vp]),
    "oracle_velocities": (None, [_vp]),
    "oracle_forces": (None, [_vp]),
    "oracle_set_positions": (None, [_vp]),
    "oracle_set_velocities": (None, [_vp]),
    "oracle_neighbor_lists": (_c_int, [_vp, _vp, _c_int]),
    "oracle_ghosts": (None, [_vp, _vp, _vp, _vp]),
    "oracle_cells": (None, [_vp, _vp]),
    "oracle_last_thermo": (None, [_vp]),
    "oracle_iters": (None, [_vp]),
}


def ptr(a):
    """ctypes pointer to the data of a C-contiguous numpy array (or None)."""
    return None if a is None else a.ctypes.data_as(_vp)


def declare(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


def open_library(path):
    """Opens any library exporting the md_* interface and declares its types."""
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    declare(lib, _REFERENCE_API)
    declare(lib, _EXTENSION_API)
    declare(lib, _ORACLE_API)
    return lib


_product = None


def load(build_if_missing=True):
    """The product library (CUDA, sm_100a).  Raises if it cannot be built or opened."""
    global _product
    if _product is not None:
        return _product
    if not os.path.exists(LIB_PATH) and build_if_missing:
        import importlib.util
        spec = importlib.util.spec_from_file_location("_tmd_build", os.path.join(PKG_DIR, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libtinymd_b200.so is not built: run molecular-dynamics_b200/build.py")
    _product = open_library(LIB_PATH)
    return _product


class MDError(RuntimeError):
    pass


def check(lib):
    """Raises MDError when the product library latched an error."""
    fn = getattr(lib, "md_last_error", None)
    if fn is None:
        return
    code = fn()
    if code not in (0, 5):  # 5 = out-of-grid warning
        msg = lib.md_last_error_string().decode()
        lib.md_clear_error()
        raise MDError(f"tinymd_b200 error {code}: {msg}")


def setup_particles(benchmark="default", cells=(8, 8, 8), potmin=1.6796, lib=None):
    """Particles of a md benchmark setup (product host code; no GPU needed).

    Returns (masses [n], positions [n,3], velocities [n,3], world [6], rank [6]).
    """
    lib = lib or load()
    grid = np.array(cells, dtype=np.int32)
    world, a1, a2 = np.zeros(6), np.zeros(6), np.zeros(6)
    b = BENCHMARKS[benchmark]
    if lib.tmd_setup_world(b, ptr(grid), potmin, ptr(world), ptr(a1), ptr(a2)) != 0:
        raise ValueError(benchmark)
    rank = np.zeros(6)
    lib.tmd_setup_rank_box(ptr(world), ptr(rank))
    n = lib.tmd_setup_generate(b, ptr(world), ptr(rank), ptr(a1), ptr(a2), potmin)
    if n < 0:
        raise ValueError(f"setup {benchmark} failed")
    m, x, v = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3))
    lib.tmd_setup_fetch(ptr(m), ptr(x), ptr(v))
    return m, x, v, world, rank


class Simulation:
    """The md driver's sequence on one md_* library (product or oracle).

    Positions/velocities are AoS [n,3] float64 arrays in input order."""

    def __init__(self, lib, masses, pos, vel, world, rank, cutoff=2.5, skin=0.3, half=False, force_field="lj",
                 eps=1.0, sigma=1.0, dem=(0.0, 0.0, 0.0, 0.0), temp=None, reneigh=20, nb_capacity=100):
        self.lib = lib
        self.n = len(masses)
        self.cutoff, self.skin, self.half = cutoff, skin, half
        self.cell = cutoff + skin
        self.force_field, self.eps, self.sigma, self.dem = force_field, eps, sigma, dem
        self.reneigh = reneigh
        self.step_count = 0
        self.world, self.rank = np.ascontiguousarray(world, dtype=np.float64), np.ascontiguousarray(rank)
        self._keep = [np.ascontiguousarray(masses, dtype=np.float64), np.ascontiguousarray(pos, dtype=np.float64),
                      np.ascontiguousarray(vel, dtype=np.float64)]
        n = lib.md_initialize_grid(ptr(self._keep[0]), ptr(self._keep[1]), ptr(self._keep[2]), self.n,
                                   ptr(self.world), ptr(self.rank), self.cell, 60, nb_capacity)
        check(lib)
        if n != self.n:
            raise MDError(f"md_initialize_grid returned {n}")
        if temp is not None:
            lib.md_create_velocity(temp)
        lib.md_copy_data_to_accelerator()
        self.reneighbor(wrap=False)
        self.force()
        check(lib)

    def force(self):
        if self.force_field == "dem":
            self.lib.md_compute_dem(self.half, self.cutoff, *self.dem)
        else:
            self.lib.md_compute_lennard_jones(self.half, self.cutoff, self.eps, self.sigma)

    def reneighbor(self, wrap=True):
        lib = self.lib
        lib.md_exchange_particles()
        if wrap:
            lib.md_enforce_pbc()
        lib.md_borders()
        lib.md_distribute_particles()
        lib.md_assemble_neighborlists(self.half, self.cell)

    def run(self, dt, steps, step_ms=None, flush=None):
        """`steps` timesteps issued natively by md_run_timesteps (product library only).

        step_ms: float32 array receiving per-step device times; flush: (pointer, bytes)
        of a device buffer overwritten before each step (outside the timed interval)."""
        fp, fb = (flush if flush is not None else (None, 0))
        rc = self.lib.md_run_timesteps(steps, dt, self.reneigh, self.step_count, self.cell,
                                       ptr(step_ms), fp, fb)
        check(self.lib)
        if rc != 0:
            raise MDError("md_run_timesteps failed")
        self.step_count += steps

    def step(self, dt, steps=1):
        """`steps` timesteps of main.cpp:715-776."""
        lib = self.lib
        for _ in range(steps):
            lib.md_initial_integration(dt)
            if (self.step_count + 1) % self.reneigh == 0:
                self.reneighbor(wrap=True)
            else:
                lib.md_synchronize_ghost_layer()
            self.force()
            lib.md_final_integration(dt)
            self.step_count += 1
        check(lib)

    # ---- state access -------------------------------------------------------
    def counts(self):
        return self.lib.md_get_number_of_particles(), self.lib.md_get_number_of_ghost_particles()

    def arrays(self):
        """(masses, positions, velocities, forces) of the locals via md_copy_data_from_accelerator
        (several ranks: this rank's current locals, whose number changes as atoms migrate)."""
        self.lib.md_copy_data_from_accelerator()
        n = self.n = self.lib.md_get_number_of_particles()
        # every element is written by md_write_grid_data_to_arrays
        m, x, v, f = np.empty(n), np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        self.lib.md_write_grid_data_to_arrays(ptr(m), ptr(x), ptr(v), ptr(f))
        check(self.lib)
        return m, x, v, f

    def ghost_arrays(self):
        self.lib.md_copy_data_from_accelerator()
        g = self.lib.md_get_number_of_ghost_particles()
        m, x, v, f = np.zeros(g), np.zeros((g, 3)), np.zeros((g, 3)), np.zeros((g, 3))
        self.lib.md_write_grid_ghost_data_to_arrays(ptr(m), ptr(x), ptr(v), ptr(f))
        return m, x, v, f

    def close(self):
        self.lib.md_deallocate_grid()


def is_oracle(lib):
    return hasattr(lib, "oracle_positions") and not hasattr(lib, "md_get_state")


def neighbor_lists(lib, n, capacity=256):
    """Neighbour lists in reference index space: list of int arrays (one per local)."""
    sizes = np.zeros(n, dtype=np.int32)
    lists = np.zeros((n, capacity), dtype=np.int32)
    if is_oracle(lib):
        lib.oracle_neighbor_lists(ptr(sizes), ptr(lists), capacity)
    else:
        lib.md_get_neighbor_lists(ptr(sizes), ptr(lists), capacity)
        check(lib)
    return [lists[i, :sizes[i]].copy() for i in range(n)]


def ghost_info(lib):
    g = lib.md_get_number_of_ghost_particles()
    src, root = np.zeros(g, dtype=np.int32), np.zeros(g, dtype=np.int32)
    pbc, tsh = np.zeros((g, 3), dtype=np.int32), np.zeros((g, 3), dtype=np.int32)
    if is_oracle(lib):
        lib.oracle_ghosts(ptr(src), ptr(pbc), ptr(root), ptr(tsh))
    else:
        lib.md_get_ghost_info(ptr(src), ptr(pbc), ptr(root), ptr(tsh))
        check(lib)
    return src, pbc, root, tsh


def full_state(lib):
    """(positions [N+G,3], velocities [N,3], forces [N,3]) in reference order, without the host mirror."""
    n, g = lib.md_get_number_of_particles(), lib.md_get_number_of_ghost_particles()
    x, v, f = np.zeros((n + g, 3)), np.zeros((n, 3)), np.zeros((n, 3))
    if is_oracle(lib):
        lib.oracle_positions(ptr(x))
        lib.oracle_velocities(ptr(v))
        lib.oracle_forces(ptr(f))
    else:
        lib.md_get_state(ptr(x), ptr(v), ptr(f))
        check(lib)
    return x, v, f
