"""Several ranks on the CPU: the rank layout, the transport and the halo routing.

* The rank grid and the periodic cart against a restatement of comm/comm.impala:221-299 and
  of the MPI cart of comm/mpi.cpp:19-49 (row-major, periodic, no reordering).
* Three processes connect through md_mpi_initialize (host sockets; no GPU here) and run the
  transport's reductions, a ring of messages larger than a socket buffer, the rank boxes of
  md_get_node_bounding_box and md_barrier.
* Two and four gloo ranks route the images of their atoms with the library's region tables
  (tmd_topology: owner and periodic shift of each of the 26 regions) and compute LJ forces
  from locals + received ghosts; the forces equal the single-box minimum-image forces, so the
  tables give every rank exactly the halo it needs.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT
from helpers import free_port, run_ranks

sys.path.insert(0, os.path.join(ROOT, "molecular-dynamics_b200"))
import tinymd  # noqa: E402
from tinymd import ptr  # noqa: E402

WORKER = os.path.join(ROOT, "tests", "rank_worker.py")


@pytest.fixture(scope="module")
def lib():
    return tinymd.load()


# ---- restatements of the reference's layout ------------------------------------------------
def node_config(world, lx, ly, lz):
    """comm/comm.impala:221-257 (range(a, b) is [a, b))."""
    areax, areay, areaz = lx * ly, lx * lz, ly * lz
    best = 2.0 * (areax + areay + areaz)
    dims = (1, 1, 1)
    for i in range(1, world):
        if world % i:
            continue
        rem = world // i
        for j in range(1, rem):
            if rem % j:
                continue
            k = rem // j
            surf = areax / i / j + areay / i / k + areaz / j / k
            if surf < best:
                dims, best = (i, j, k), surf
    return dims


def cart_coords(rank, dims):
    return (rank // (dims[1] * dims[2]), (rank // dims[2]) % dims[1], rank % dims[2])


def cart_rank(c, dims):
    return (c[0] * dims[1] + c[1]) * dims[2] + c[2]


def rank_box(world, dims, coords):
    """comm/comm.impala:260-299."""
    box = []
    for d in range(3):
        ln = (world[2 * d + 1] - world[2 * d]) / dims[d]
        lo = world[2 * d] + ln * coords[d]
        box += [lo, lo + ln]
    return box


def region_offsets(t):
    tt = t + 1
    e = (tt % 3, (tt // 3) % 3, tt // 9)
    return tuple(1 if x == 1 else (-1 if x == 2 else 0) for x in e)


def opposite(t):
    tt = t + 1
    e = [tt % 3, (tt // 3) % 3, tt // 9]
    e = [0 if x == 0 else 3 - x for x in e]
    return e[2] * 9 + e[1] * 3 + e[0] - 1


def topology(lib, rank, dims):
    peer, shift = np.zeros(26, dtype=np.int32), np.zeros(78, dtype=np.int32)
    mask = np.zeros(1, dtype=np.uint32)
    d = np.array(dims, dtype=np.int32)
    assert lib.tmd_topology(rank, ptr(d), ptr(peer), ptr(shift), ptr(mask)) == 0
    return peer, shift.reshape(26, 3), int(mask[0])


# ---- layout --------------------------------------------------------------------------------------
@pytest.mark.parametrize("shape", [(10.0, 10.0, 10.0), (30.0, 10.0, 10.0), (10.0, 10.0, 40.0), (7.0, 13.0, 9.0)])
def test_node_config_matches_reference(lib, shape):
    length = np.array(shape)
    for world in range(1, 49):
        dims = np.zeros(3, dtype=np.int32)
        assert lib.tmd_node_config(world, ptr(length), ptr(dims)) == 0
        assert tuple(int(x) for x in dims) == node_config(world, *shape), world
        assert int(np.prod(dims)) == world


@pytest.mark.parametrize("dims", [(1, 1, 1), (1, 1, 2), (1, 2, 2), (2, 2, 2), (1, 1, 3), (2, 1, 3), (3, 4, 2)])
def test_topology_is_the_periodic_cart(lib, dims):
    world = int(np.prod(dims))
    for rank in range(world):
        peer, shift, mask = topology(lib, rank, dims)
        c = cart_coords(rank, dims)
        for t in range(26):
            off = region_offsets(t)
            cn = [c[d] + off[d] for d in range(3)]
            sh = [(-1 if cn[d] >= dims[d] else (1 if cn[d] < 0 else 0)) for d in range(3)]
            cn = [cn[d] % dims[d] for d in range(3)]
            assert peer[t] == cart_rank(cn, dims)
            assert list(shift[t]) == sh
            assert bool((mask >> t) & 1) == (peer[t] == rank)
            # the neighbour sees this rank through the opposite region, with the opposite shift
            p2, s2, _ = topology(lib, int(peer[t]), dims)
            assert p2[opposite(t)] == rank
            assert list(s2[opposite(t)]) == [-x for x in sh]


# ---- transport -----------------------------------------------------------------------------------
def test_three_ranks_connect_reduce_and_exchange(lib, tmp_path):
    world = 3
    outs = run_ranks(world, [sys.executable, WORKER, "comm", str(tmp_path / "r{rank}.json")], {"TINYMD_COMM": "socket"})
    for rc, out in outs:
        assert rc == 0, out
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    wbox = [0.0, 12.0, 0.0, 10.0, -1.0, 9.0]
    dims = node_config(world, 12.0, 10.0, 10.0)
    for r, x in enumerate(res):
        assert x["err"] == 0, x["msg"]
        assert (x["world"], x["rank"], x["transport"]) == (world, r, "socket")
        assert x["allreduce_rc"] == 0 and x["allreduce"] == [3.0, 4.5, -6.0]
        assert x["ring_rc"] == 0 and x["ring_ok"]
        assert x["box"] == rank_box(wbox, dims, cart_coords(r, dims))
        assert x["err_after"] == 0
    # the rank boxes tile the world box
    vol = sum(np.prod([b[2 * d + 1] - b[2 * d] for d in range(3)]) for b in (x["box"] for x in res))
    assert abs(vol - 12.0 * 10.0 * 10.0) < 1e-9


def test_a_missing_rank_is_an_error_not_a_hang(lib, tmp_path):
    """A world of two whose second rank never starts: rank 0 gives up after the timeout and
    latches MD_ERR_COMM."""
    port = free_port()
    env = dict(os.environ, TINYMD_WORLD_SIZE="2", TINYMD_RANK="0", TINYMD_PORT=str(port), TINYMD_COMM_TIMEOUT="2")
    r = subprocess.run([sys.executable, WORKER, "comm", str(tmp_path / "r0.json")], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    x = json.load(open(tmp_path / "r0.json"))
    assert x["err"] == 7 and "connect" in x["msg"]


# ---- halo routing with the library's tables (gloo ranks) ---------------------------------------
def lj_forces(xi, xj, rc, exclude_self):
    d = xi[:, None, :] - xj[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", d, d)
    if exclude_self:
        np.fill_diagonal(r2, np.inf)
    inside = r2 < rc * rc
    sr2 = np.where(inside, 1.0 / np.where(inside, r2, 1.0), 0.0)
    sr6 = sr2 ** 3
    f = np.where(inside, 48.0 * sr6 * (sr6 - 0.5) * sr2, 0.0)
    return np.einsum("ij,ijk->ik", f, d)


def minimum_image_forces(x, box, rc):
    d = x[:, None, :] - x[None, :, :]
    d -= box * np.round(d / box)
    r2 = np.einsum("ijk,ijk->ij", d, d)
    np.fill_diagonal(r2, np.inf)
    inside = r2 < rc * rc
    sr2 = np.where(inside, 1.0 / np.where(inside, r2, 1.0), 0.0)
    sr6 = sr2 ** 3
    f = np.where(inside, 48.0 * sr6 * (sr6 - 0.5) * sr2, 0.0)
    return np.einsum("ij,ijk->ik", f, d)


def _halo_rank(rank, world, port, dims, results):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lib = tinymd.load(build_if_missing=False)
    rng = np.random.default_rng(7)
    box = np.array([9.0, 9.5, 10.0])
    x = rng.uniform(0.0, 1.0, size=(700, 3)) * box  # the same atoms on every rank
    rc, spacing = 2.5, 2.8
    peer, shift, mask = topology(lib, rank, dims)
    c = cart_coords(rank, dims)
    lo = np.array([box[d] / dims[d] * c[d] for d in range(3)])
    hi = lo + box / np.array(dims)
    own = np.all((x >= lo) & (x < hi), axis=1)
    loc = x[own]
    ids = np.nonzero(own)[0]
    # the border test of comm/comm.impala:116-127 per axis, the 26 regions combined from it
    near_hi, near_lo = loc > hi - spacing, loc < lo + spacing
    outgoing = [[] for _ in range(world)]
    ghosts = []
    for t in range(26):
        off = region_offsets(t)
        sel = np.ones(len(loc), dtype=bool)
        for d in range(3):
            if off[d] == 1:
                sel &= near_hi[:, d]
            elif off[d] == -1:
                sel &= near_lo[:, d]
        img = loc[sel] + shift[t] * box
        if (mask >> t) & 1:
            ghosts.append(img)
        else:
            outgoing[peer[t]].append(img)
    # one message per peer (sizes first), as the library's exchange does
    send = [np.concatenate(o) if o else np.zeros((0, 3)) for o in outgoing]
    counts = torch.tensor([len(s) for s in send], dtype=torch.int64)
    incoming = torch.zeros(world, dtype=torch.int64)
    dist.all_to_all_single(incoming, counts)
    recv = [torch.zeros((int(incoming[p]), 3), dtype=torch.float64) for p in range(world)]
    ops = []
    for p in range(world):
        if p == rank:
            continue
        if len(send[p]):
            ops.append(dist.isend(torch.from_numpy(np.ascontiguousarray(send[p])), p))
        if int(incoming[p]):
            ops.append(dist.irecv(recv[p], p))
    for op in ops:
        op.wait()
    ghosts += [r.numpy() for r in recv]
    g = np.concatenate(ghosts) if ghosts else np.zeros((0, 3))
    f = lj_forces(loc, loc, rc, True) + (lj_forces(loc, g, rc, False) if len(g) else 0.0)
    results.put((rank, ids, f))
    dist.destroy_process_group()


@pytest.mark.parametrize("dims", [(1, 1, 2), (1, 2, 2), (2, 1, 2)])
def test_halo_routing_gives_minimum_image_forces(dims):
    world = int(np.prod(dims))
    port = free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_halo_rank, args=(r, world, port, dims, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(7)
    box = np.array([9.0, 9.5, 10.0])
    x = rng.uniform(0.0, 1.0, size=(700, 3)) * box
    ref = minimum_image_forces(x, box, 2.5)
    seen = np.zeros(len(x), dtype=int)
    for _, ids, f in got:
        seen[ids] += 1
        np.testing.assert_allclose(f, ref[ids], rtol=1e-10, atol=1e-9)
    assert np.all(seen == 1)
