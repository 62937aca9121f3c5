"""Shared fixtures of the tinyMD B200 test suite.

Markers: ``gpu`` -- needs a CUDA device (runs the product kernels);
everything else runs on the CPU (the oracle, host logic, ABI surface).
The oracle (oracle/, a CPU restatement of the reference) is only the
checker here; the product under test is molecular-dynamics_b200/.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "molecular-dynamics_b200")
if PKG not in sys.path:
    sys.path.insert(0, PKG)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "libtinymd_oracle.so")
ORACLE_MD = os.path.join(ROOT, "oracle", "_build", "md_cpu")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtinymd_refsetup.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _build_oracle():
    if not os.path.exists(ORACLE_LIB) or not os.path.exists(ORACLE_MD):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)


@pytest.fixture(scope="session")
def product():
    import tinymd
    return tinymd.load()


@pytest.fixture(scope="session")
def oracle():
    import tinymd
    _build_oracle()
    lib = tinymd.open_library(ORACLE_LIB)
    lib.oracle_set_threads(min(8, os.cpu_count() or 1))
    return lib


@pytest.fixture(scope="session")
def refsetup():
    """The reference's own initialize.h / force_lj.cpp compiled from the reference tree."""
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref not built here (needs the reference tree); golden fixtures cover it")
    import ctypes
    return ctypes.CDLL(REF_LIB, mode=ctypes.RTLD_LOCAL)


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return torch.device("cuda:0")
