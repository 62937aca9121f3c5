"""The multi-rank path of bench.py on CPU: two gloo ranks as separate processes.

Under torchrun every rank runs an independent replica of the workload (the
path does not shard); the whole-job rate is all ranks' atoms over the slowest
rank's time, and the reference arm does its work on rank 0 only.  These run
the same functions bench.py uses, over a real process group.
"""
import argparse
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, results):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.dist_init(world, "gloo")
    # every rank reports its own step time; both must see the slowest one
    rate, ms = bench.replica_rate(1000, world, 10, [5.0, 7.0][rank], dist)
    bench.barrier(dist)
    # the reference arm: ranks other than 0 leave at once without work
    ref_rc = bench.run_reference(argparse.Namespace(gpus=world, steps=1, warmup=3)) if rank == 1 else None
    dist.destroy_process_group()
    results.put((rank, rate, ms, ref_rc))


def test_two_rank_replica_rate_and_reference_arm():
    world = 2
    ctx = mp.get_context("spawn")
    results = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, results)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        rank, rate, ms, ref_rc = results.get(timeout=120)
        got[rank] = (rate, ms, ref_rc)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in range(world):
        rate, ms, _ = got[rank]
        assert ms == pytest.approx(7.0)  # the slowest rank's time
        assert rate == pytest.approx(1000 * world * 10 / 7e-3)
    assert got[1][2] == 0
