"""The C ABI surface (CPU only: loads the libraries, calls no kernels)."""
import ctypes
import os
import re

from conftest import ORACLE_LIB, ROOT

HEADER = os.path.join(ROOT, "include", "tinymd_b200.h")
REFERENCE_NAMES = [  # the extern "C" interface of anydsl_includes.h:10-48
    "md_initialize_grid", "md_rescale_grid", "md_copy_data_from_accelerator", "md_copy_data_to_accelerator",
    "md_initial_integration", "md_final_integration", "md_enforce_pbc", "md_write_grid_data_to_arrays",
    "md_write_grid_ghost_data_to_arrays", "md_write_grid_aabb_data_to_arrays", "md_distribute_particles",
    "md_assemble_neighborlists", "md_deallocate_grid", "md_print_grid", "md_print_ghost", "md_create_velocity",
    "md_compute_lennard_jones", "md_compute_dem", "md_mpi_initialize", "md_mpi_finalize",
    "md_synchronize_ghost_layer", "md_borders", "md_exchange_particles", "md_get_send_buffer_value",
    "md_set_recv_buffer_value", "md_resize_recv_buffer_capacity", "md_serialize_particles",
    "md_deserialize_particles", "md_get_world_size", "md_get_world_rank", "md_get_number_of_particles",
    "md_get_number_of_ghost_particles", "md_get_node_bounding_box", "md_compute_boundary_weights",
    "md_update_neighborhood", "md_report_iterations", "md_report_particles", "md_report_time", "md_barrier"]


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b((?:md|tmd)_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_covers_reference_interface():
    declared = set(declared_functions())
    missing = [n for n in REFERENCE_NAMES if n not in declared]
    assert not missing, missing


def test_product_exports_every_declared_symbol(product):
    missing = [n for n in declared_functions() if not hasattr(product, n)]
    assert not missing, missing


def test_product_reports_missing_device_without_crashing(product):
    import torch
    if torch.cuda.is_available():
        return
    import numpy as np
    import tinymd
    m, x, v, w, r = tinymd.setup_particles("default", (2, 2, 2), lib=product)
    n = product.md_initialize_grid(tinymd.ptr(m), tinymd.ptr(x), tinymd.ptr(v), len(m), tinymd.ptr(w),
                                   tinymd.ptr(r), 2.8, 60, 100)
    assert n == -1 and product.md_last_error() == 6
    product.md_clear_error()


def test_oracle_exports_reference_interface(oracle):
    lib = ctypes.CDLL(ORACLE_LIB)
    missing = [n for n in REFERENCE_NAMES
               if n not in ("md_print_grid", "md_print_ghost", "md_rescale_grid", "md_get_send_buffer_value",
                            "md_set_recv_buffer_value", "md_resize_recv_buffer_capacity", "md_serialize_particles",
                            "md_deserialize_particles", "md_compute_boundary_weights", "md_update_neighborhood")
               and not hasattr(lib, n)]
    assert not missing, missing
