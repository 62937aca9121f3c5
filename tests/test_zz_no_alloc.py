"""md_lj_forces_noalloc: the allocation-free variant of the FP64 LJ force kernel.

Callers that cannot call cudaMalloc (inside another framework's memory pool,
during someone else's graph capture, fixed memory budgets) use this entry
point; its scratch is a fixed device array inside the library.  The test runs
it through the C ABI on device buffers holding the same positions and lists
the regular path used, twice in a row, and compares with the regular path's
forces and energy / virial sums.  It sits in its own file named to be
collected last.
"""
import ctypes

import numpy as np
import pytest

import tinymd
from helpers import make_sim, rel_err

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_path_twice(product, cuda_device):
    import torch
    product.md_set_thermo(1)
    try:
        sim = make_sim(product, setup_lib=product, cells=(8, 8, 8))
        sim.step(0.005, 30)  # forces of the last step are at the current positions
        n, g = sim.counts()
        x, _, f_ref = tinymd.full_state(product)
        thermo = np.zeros(4)
        assert product.md_get_thermo(tinymd.ptr(thermo)) == 0
        lists = tinymd.neighbor_lists(product, n)
        sim.close()
    finally:
        product.md_set_thermo(0)
    stride = ((n + 31) // 32) * 32
    max_nb = max(len(l) for l in lists)
    plain = np.zeros((max_nb, stride), dtype=np.int32)
    sizes = np.zeros(n, dtype=np.int32)
    for i, l in enumerate(lists):
        plain[:len(l), i] = l
        sizes[i] = len(l)
    pos4 = np.zeros((n + g, 4))
    pos4[:, :3] = x
    d_pos = torch.from_numpy(pos4).to(cuda_device)
    d_sizes = torch.from_numpy(sizes).to(cuda_device)
    d_lists = torch.from_numpy(plain).to(cuda_device)
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda_device).cuda_stream)
    for call in range(2):
        d_f = torch.full((n, 4), float("nan"), dtype=torch.float64, device=cuda_device)
        d_sums = torch.full((4,), float("nan"), dtype=torch.float64, device=cuda_device)
        rc = product.md_lj_forces_noalloc(ctypes.c_void_p(d_pos.data_ptr()), n, ctypes.c_void_p(d_sizes.data_ptr()),
                                          ctypes.c_void_p(d_lists.data_ptr()), stride, max_nb, 2.5, 1.0, 1.0,
                                          ctypes.c_void_p(d_f.data_ptr()), ctypes.c_void_p(d_sums.data_ptr()), stream)
        assert rc == 0, product.md_last_error_string()
        torch.cuda.synchronize()
        f = d_f.cpu().numpy()[:, :3]
        sums = d_sums.cpu().numpy()
        assert rel_err(f, f_ref) <= 1e-12, f"call {call}"
        np.testing.assert_allclose(sums[:3], thermo[:3], rtol=1e-12)
        assert sums[3] == 0.0


def test_noalloc_rejects_too_many_atoms(product):
    rc = product.md_lj_forces_noalloc(ctypes.c_void_p(16), 1_048_577, ctypes.c_void_p(16), ctypes.c_void_p(16), 1_048_577,
                                      1, 2.5, 1.0, 1.0, ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == 3
    assert b"exceed the fixed scratch" in product.md_last_error_string()
    product.md_clear_error()
    rc = product.md_lj_forces_noalloc(ctypes.c_void_p(16), -1, ctypes.c_void_p(16), ctypes.c_void_p(16), 32, 1, 2.5,
                                      1.0, 1.0, ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == 3
    assert b"invalid arguments" in product.md_last_error_string()
    product.md_clear_error()
