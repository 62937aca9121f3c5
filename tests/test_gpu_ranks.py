"""Several ranks on one GPU against the one-box oracle (comm/comm.impala's decomposition).

Each rank is its own process (tests/rank_worker.py md) and owns the atoms of its box of the
default FCC lattice (8^3 cells, 2,048 atoms); the ranks exchange halos and migrate atoms
through the library (host-socket transport: the processes share the device, so no kernel
of one waits for another's).  The oracle runs the same setup as one box with exact ghosts.

* At the first lists every atom has the oracle's neighbour count (integer-exact), and the
  union of the ranks' atoms is the oracle's lattice.
* After 100 steps with a rebuild (migration + borders) every 10, every atom's position,
  velocity and force matches the oracle's to 1e-9 (FP64: only the summation order differs,
  since a rank's lists hold its ghosts in another order), and the atom count is conserved.
* The contact-fixed DEM model on two ranks (the halo carries velocities) matches likewise.
* The mixed form on four ranks stays close to the same run (a sanity bound over 100 steps).
* The reference's own driver (main.cpp, unmodified, linked to the product) runs on two ranks.
* A rank that leaves between steps is detected by the others (MD_ERR_COMM, no hang); half
  lists on several ranks are refused.
"""
import os
import subprocess
import sys

import numpy as np
import pytest
from scipy.spatial import cKDTree

from conftest import ORACLE_LIB, ROOT
from helpers import run_ranks

sys.path.insert(0, os.path.join(ROOT, "molecular-dynamics_b200"))
import tinymd  # noqa: E402

pytestmark = pytest.mark.gpu

WORKER = os.path.join(ROOT, "tests", "rank_worker.py")
REF_B200 = os.path.join(ROOT, "oracle", "_ref", "refmd_b200")
OUR_MD = os.path.join(ROOT, "molecular-dynamics_b200", "lib", "md")
CELLS, STEPS, REBUILD, DT = 8, 100, 10, 0.005


@pytest.fixture(scope="module")
def one_box():
    lib = tinymd.load()
    olib = tinymd.open_library(ORACLE_LIB)
    olib.oracle_set_ghost_mode(1)
    m, x, v, world, rank = tinymd.setup_particles("default", (CELLS,) * 3, lib=lib)
    sim = tinymd.Simulation(olib, m, x, v, world, rank, temp=1.44, reneigh=REBUILD)
    nb0 = np.array([len(l) for l in tinymd.neighbor_lists(olib, sim.n)])
    sim.step(DT, STEPS)
    _, x1, v1, f1 = sim.arrays()
    sim.close()
    olib.oracle_set_ghost_mode(0)
    box = np.array([world[1] - world[0], world[3] - world[2], world[5] - world[4]])
    return dict(x0=x, nb0=nb0, x=x1, v=v1, f=f1, box=box, lo=np.array(world[0::2]))


def run(world, tmp_path, precision=0, steps=STEPS):
    outs = run_ranks(world, [sys.executable, WORKER, "md", str(tmp_path / "r{rank}.npz"), str(CELLS), str(steps),
                             str(precision), str(REBUILD)],
                     {"TINYMD_COMM": "socket", "TINYMD_DEVICE": "0"}, timeout=600)
    for rc, out in outs:
        assert rc == 0, out
    return [dict(np.load(tmp_path / f"r{r}.npz")) for r in range(world)]


def match(ref_x, x, box, lo):
    """Index of the nearest reference atom (periodic) for each row of x, and its distance."""
    tree = cKDTree(np.mod(ref_x - lo, box), boxsize=box)
    d, i = tree.query(np.mod(x - lo, box))
    return i, d


@pytest.mark.parametrize("world", [2, 4, 8])
def test_ranks_match_the_one_box_oracle(one_box, tmp_path, world):
    res = run(world, tmp_path)
    assert all(str(r["transport"]) == "socket" for r in res)
    # the first lists: the ranks' atoms are the lattice, each with the oracle's neighbour count
    x0 = np.concatenate([r["x0"] for r in res])
    nb0 = np.concatenate([r["nb0"] for r in res])
    assert len(x0) == len(one_box["x0"])
    key = {tuple(p): k for k, p in enumerate(one_box["x0"])}
    idx = np.array([key[tuple(p)] for p in x0])
    assert len(set(idx.tolist())) == len(idx)
    assert np.array_equal(nb0, one_box["nb0"][idx])
    # after the run
    n = sum(int(r["n"]) for r in res)
    assert n == len(one_box["x"])
    x = np.concatenate([r["x"] for r in res])
    v = np.concatenate([r["v"] for r in res])
    f = np.concatenate([r["f"] for r in res])
    i, d = match(one_box["x"], x, one_box["box"], one_box["lo"])
    assert len(set(i.tolist())) == n
    assert d.max() < 1e-9
    np.testing.assert_allclose(v, one_box["v"][i], rtol=0, atol=1e-9)
    np.testing.assert_allclose(f, one_box["f"][i], rtol=0, atol=1e-8)
    # atoms did migrate: some rank's final count differs from its initial one
    assert any(int(r["n"]) != len(r["x0"]) for r in res)


@pytest.mark.parametrize("bench,cells,world", [("default", 8, 3), ("default", 8, 6), ("half", 10, 4),
                                               ("body_collision", 6, 4)])
def test_other_layouts_and_sparse_setups(tmp_path, bench, cells, world):
    """Layouts whose rank boxes are not powers of two of the lattice (1x1x3, 1x2x3), the half
    setup on 1x2x2 (the upper ranks start without atoms and receive the ones that expand into
    them) and body_collision (two bodies in a mostly empty box), 100 steps against the one-box
    oracle."""
    from helpers import make_sim
    lib = tinymd.load()
    olib = tinymd.open_library(ORACLE_LIB)
    olib.oracle_set_ghost_mode(1)
    try:
        o = make_sim(olib, benchmark=bench, cells=(cells,) * 3, setup_lib=lib, reneigh=REBUILD)
        o.step(DT, STEPS)
        _, xo, vo, fo = o.arrays()
        o.close()
    finally:
        olib.oracle_set_ghost_mode(0)
    outs = run_ranks(world, [sys.executable, WORKER, "md", str(tmp_path / "r{rank}.npz"), str(cells), str(STEPS), "0",
                             str(REBUILD), bench], {"TINYMD_COMM": "socket", "TINYMD_DEVICE": "0"}, timeout=600)
    for rc, out in outs:
        assert rc == 0, out
    res = [dict(np.load(tmp_path / f"r{r}.npz")) for r in range(world)]
    if bench == "half":
        assert any(len(r["x0"]) == 0 for r in res) and all(int(r["n"]) > 0 for r in res)
    x = np.concatenate([r["x"] for r in res])
    v = np.concatenate([r["v"] for r in res])
    f = np.concatenate([r["f"] for r in res])
    _, _, _, wbox, _ = tinymd.setup_particles(bench, (cells,) * 3, lib=lib)
    box = np.array([wbox[1] - wbox[0], wbox[3] - wbox[2], wbox[5] - wbox[4]])
    i, d = match(xo, x, box, np.array(wbox[0::2]))
    assert len(x) == len(xo) and len(set(i.tolist())) == len(xo)
    assert d.max() < 1e-9
    np.testing.assert_allclose(v, vo[i], rtol=0, atol=1e-9)
    np.testing.assert_allclose(f, fo[i], rtol=0, atol=1e-8)


def test_contact_dem_on_two_ranks(tmp_path):
    """The contact-fixed DEM model (ghosts carry their root's velocity, so the halo does too) on
    the granular-gas FCC setup, two ranks against the one-box oracle."""
    from helpers import make_sim
    lib = tinymd.load()
    olib = tinymd.open_library(ORACLE_LIB)
    olib.oracle_set_ghost_mode(1)
    olib.oracle_set_dem_mode(1, 0.6)
    try:
        o = make_sim(olib, benchmark="granular_gas_fcc", cells=(12, 12, 12), force_field="dem", cutoff=1.2,
                     skin=0.3, dem=(0.1, 0.1, 100.0, 0.5), setup_lib=lib, reneigh=10)
        o.step(0.001, 60)
        _, xo, vo, fo = o.arrays()
        o.close()
    finally:
        olib.oracle_set_ghost_mode(0)
        olib.oracle_set_dem_mode(0, 1.0)
    outs = run_ranks(2, [sys.executable, WORKER, "md", str(tmp_path / "r{rank}.npz"), "12", "60", "0", "10",
                         "granular_gas_fcc"], {"TINYMD_COMM": "socket", "TINYMD_DEVICE": "0"}, timeout=600)
    for rc, out in outs:
        assert rc == 0, out
    res = [dict(np.load(tmp_path / f"r{r}.npz")) for r in range(2)]
    x = np.concatenate([r["x"] for r in res])
    v = np.concatenate([r["v"] for r in res])
    f = np.concatenate([r["f"] for r in res])
    m, _, _, world, _ = tinymd.setup_particles("granular_gas_fcc", (12, 12, 12), lib=lib)
    box = np.array([world[1] - world[0], world[3] - world[2], world[5] - world[4]])
    i, d = match(xo, x, box, np.array(world[0::2]))
    assert len(x) == len(xo) and len(set(i.tolist())) == len(xo)
    assert d.max() < 1e-9
    assert np.abs(f).max() > 1.0  # contacts act
    np.testing.assert_allclose(v, vo[i], rtol=0, atol=1e-9)
    np.testing.assert_allclose(f, fo[i], rtol=0, atol=1e-8)


def test_mixed_form_on_four_ranks(one_box, tmp_path):
    res = run(4, tmp_path, precision=1)
    x = np.concatenate([r["x"] for r in res])
    f = np.concatenate([r["f"] for r in res])
    i, d = match(one_box["x"], x, one_box["box"], one_box["lo"])
    assert len(set(i.tolist())) == len(one_box["x"])
    assert d.max() < 1e-3
    rms = np.sqrt(np.mean(one_box["f"] ** 2))
    assert np.max(np.abs(f - one_box["f"][i])) / rms < 1e-2


def test_a_rank_that_leaves_is_detected(tmp_path):
    """Failure detection without a GPU fault: after 5 steps the last of three ranks waits for
    its device work and exits between steps.  The other two find the closed connections at
    their next halo exchange: MD_ERR_COMM is latched, and they finish their remaining steps
    in far less than the exchange timeout instead of waiting for the missing rank."""
    import json
    outs = run_ranks(3, [sys.executable, WORKER, "leave", str(tmp_path / "r{rank}.json"), "8"],
                     {"TINYMD_COMM": "socket", "TINYMD_DEVICE": "0", "TINYMD_COMM_TIMEOUT": "30"}, timeout=300)
    for rc, out in outs:
        assert rc == 0, out
    for r in range(2):
        x = json.load(open(tmp_path / f"r{r}.json"))
        assert x["err"] == 7, x
        assert x["seconds"] < 25.0


def test_half_lists_on_several_ranks_are_refused(tmp_path):
    import json
    outs = run_ranks(2, [sys.executable, WORKER, "half", str(tmp_path / "r{rank}.json"), "8"],
                     {"TINYMD_COMM": "socket", "TINYMD_DEVICE": "0"}, timeout=300)
    for rc, out in outs:
        assert rc == 0, out
    for r in range(2):
        x = json.load(open(tmp_path / f"r{r}.json"))
        assert x["err"] == 4 and "half lists" in x["msg"]


def test_nccl_binding_on_one_gpu():
    """The NCCL transport's calls (libnccl opened at run time, a communicator, a send/receive
    group on a stream) carry a device buffer to the same rank: the binding works on this GPU.
    Two ranks over NCCL need two GPUs."""
    env = dict(os.environ, NCCL_SOCKET_IFNAME=os.environ.get("NCCL_SOCKET_IFNAME", "lo"))
    r = subprocess.run([sys.executable, WORKER, "nccl", str(3 << 20)], capture_output=True, text=True, timeout=300,
                       env=env)
    assert r.returncode == 0, r.stdout + r.stderr


def test_reference_driver_on_two_ranks(tmp_path):
    """The reference's main.cpp on two ranks reports what this repository's md driver reports on
    one rank with exact ghosts (several ranks run exact ghosts): the same atom count,
    temperature (six digits) and iteration counts."""
    if not os.path.exists(REF_B200):
        pytest.skip("oracle/_ref/refmd_b200 not built (make -C oracle refmd needs the reference tree)")
    args = ["-x", "8", "-y", "8", "-z", "8", "-s", "100"]
    one = subprocess.run([OUR_MD] + args + ["--ghost", "exact"], capture_output=True, text=True, cwd=tmp_path,
                         timeout=600)
    assert one.returncode == 0, one.stdout + one.stderr
    outs = run_ranks(2, [REF_B200] + args, {"TINYMD_COMM": "socket", "TINYMD_DEVICE": "0"}, timeout=600)
    for rc, out in outs:
        assert rc == 0, out

    def report(lines, head):
        for k, line in enumerate(lines):
            if line.startswith(head) and k + 1 < len(lines):
                return lines[k + 1].split()
        return None

    r1 = report(one.stdout.splitlines(), "# Local")
    r2 = report(outs[0][1].splitlines(), "# Local")  # rank 0 prints the sums over the ranks
    assert report(outs[1][1].splitlines(), "# Local") is None
    assert r1 is not None and r2 is not None
    assert r2[0] == r1[0] == "2048"
    assert abs(float(r2[2]) - float(r1[2])) <= 1e-5 * float(r1[2])
    it1 = report(one.stdout.splitlines(), "ForceIters")
    it2 = report(outs[0][1].splitlines(), "ForceIters")
    assert it1 == it2
