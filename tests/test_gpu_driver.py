"""The md command-line driver on the GPU against the same driver on the CPU oracle.

Both binaries come from host/main.cpp (the reference driver's flags, setups,
run loop and report lines, main.cpp:333-796): `md` links the B200 library,
`md_cpu` the oracle.  The FP64 form's trajectory is bit-identical, so the
thermo lines (temperature, potential energy and pressure per atom, total
energy) and the particle report agree; the device's energy and virial sums
use another summation order, so the printed values are compared to 1e-9.
The timing line is the only one that differs.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

MD = os.path.join(ROOT, "molecular-dynamics_b200", "lib", "md")
MD_CPU = os.path.join(ROOT, "oracle", "_build", "md_cpu")


def run(binary, args):
    r = subprocess.run([binary] + args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout.splitlines()


def section(lines, header):
    """The line after a report header."""
    i = lines.index(header)
    return lines[i + 1].split()


@pytest.mark.parametrize("args", [
    ["-x", "8", "-y", "8", "-z", "8", "-s", "100", "--thermo", "20"],
    ["-x", "6", "-y", "7", "-z", "5", "-s", "60", "--thermo", "10", "--ghost", "exact"],
])
def test_md_driver_matches_cpu_driver(args):
    if not os.path.exists(MD_CPU):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    gpu, cpu = run(MD, args), run(MD_CPU, args)
    tg = np.array([[float(v) for v in l.split()[1:]] for l in gpu if l.startswith("thermo ")])
    tc = np.array([[float(v) for v in l.split()[1:]] for l in cpu if l.startswith("thermo ")])
    assert tg.shape == tc.shape and tg.shape[0] > 1
    np.testing.assert_array_equal(tg[:, 0], tc[:, 0])  # steps
    np.testing.assert_allclose(tg[:, 1:], tc[:, 1:], rtol=1e-9, atol=1e-12)
    # "# Local # Ghost Temp": same counts, same temperature
    pg, pc = section(gpu, "# Local # Ghost Temp"), section(cpu, "# Local # Ghost Temp")
    assert pg[:2] == pc[:2]
    assert float(pg[2]) == pytest.approx(float(pc[2]), rel=1e-6)
    # the banner matches apart from the backend line
    bg = [l for l in gpu if l.startswith("- ") and not l.startswith("- Backend")]
    bc = [l for l in cpu if l.startswith("- ") and not l.startswith("- Backend")]
    assert bg == bc
