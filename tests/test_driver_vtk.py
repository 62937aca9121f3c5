"""The md driver's VTK dump (-v, host/main.cpp) against the reference's own writer (vtk.h:6-91).

Both drivers run over the CPU oracle: the reference's unmodified main.cpp linked against it
(oracle/_ref/refmd_oracle, `make -C oracle refmd`) and this repository's driver linked against
it (oracle/_build/md_cpu).  Every file (locals, ghosts and the box after setup and after each
step, main.cpp:702-775) must be byte-identical, and so must the particle report line.
"""
import filecmp
import os
import subprocess

import pytest

from conftest import ORACLE_MD, ROOT, _build_oracle

REF_ORACLE = os.path.join(ROOT, "oracle", "_ref", "refmd_oracle")


def test_vtk_files_match_reference_writer(tmp_path):
    if not os.path.exists(REF_ORACLE):
        pytest.skip("oracle/_ref/refmd_oracle not built (make -C oracle refmd needs the reference tree)")
    _build_oracle()
    args = ["-x", "5", "-y", "6", "-z", "5", "-s", "12"]
    outs = {}
    for name, binary in (("reference", REF_ORACLE), ("driver", ORACLE_MD)):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([binary] + args + ["-v", str(d)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        lines = r.stdout.splitlines()
        outs[name] = lines[lines.index("# Local # Ghost Temp") + 1].split()
    names = sorted(os.listdir(tmp_path / "reference"))
    assert len(names) == 3 * 13
    assert sorted(os.listdir(tmp_path / "driver")) == names
    match, mismatch, errors = filecmp.cmpfiles(tmp_path / "reference", tmp_path / "driver", names, shallow=False)
    assert not mismatch and not errors, (mismatch[:5], errors[:5])
    assert outs["reference"] == outs["driver"]
