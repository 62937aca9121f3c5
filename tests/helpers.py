"""Helpers shared by the tests: run the same setup on the product and the oracle."""
import os
import socket
import subprocess
import sys

import numpy as np

import tinymd


def make_sim(lib, benchmark="default", cells=(8, 8, 8), potmin=1.6796, half=False, temp=1.44, force_field="lj",
             cutoff=2.5, skin=0.3, dem=(0.0, 0.0, 0.0, 0.0), nb_capacity=100, setup_lib=None, reneigh=20,
             particles=None):
    m, x, v, world, rank = particles if particles is not None else tinymd.setup_particles(
        benchmark, cells, potmin, lib=setup_lib)
    if benchmark not in ("default", "half"):
        temp = None
    return tinymd.Simulation(lib, m, x, v, world, rank, cutoff=cutoff, skin=skin, half=half, temp=temp,
                             force_field=force_field, dem=dem, nb_capacity=nb_capacity, reneigh=reneigh)


def lists_as_sets(lists):
    return [set(map(int, l)) for l in lists]


def rel_err(a, b):
    """max |a-b| / rms(b) over all components."""
    rms = np.sqrt(np.mean(np.asarray(b) ** 2))
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / (rms if rms > 0 else 1.0))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(world, argv, env_extra=None, timeout=120):
    """Starts `world` processes of argv (each argument formatted with rank=r) as the ranks of one
    run (TINYMD_WORLD_SIZE / TINYMD_RANK / TINYMD_PORT); returns [(returncode, output)]."""
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, TINYMD_WORLD_SIZE=str(world), TINYMD_RANK=str(r), TINYMD_PORT=str(port),
                   TINYMD_COMM_TIMEOUT="60")
        env.update(env_extra or {})
        procs.append(subprocess.Popen([a.format(rank=r) for a in argv], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        outs.append((p.returncode, out))
    return outs
