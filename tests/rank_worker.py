"""One rank of a multi-process run, started by the rank tests (not collected by pytest).

    python tests/rank_worker.py comm OUT.json
        md_mpi_initialize over the environment's ranks, then the transport's collectives,
        a ring of messages, md_get_node_bounding_box and md_barrier (no GPU needed).
    python tests/rank_worker.py md OUT.npz CELLS STEPS PRECISION [REBUILD] [BENCHMARK]
        the md driver's sequence (main.cpp:614-776 of tinyMD) on this rank's part of a setup
        (default: the FCC lattice with LJ forces; granular_gas_fcc: the contact-fixed DEM
        configuration): setup inside the rank box, velocities, borders, lists, forces, STEPS
        timesteps with reneighbouring every REBUILD steps; saves the locals and the neighbour
        counts of the first lists.
    python tests/rank_worker.py leave OUT.json CELLS
        the last rank leaves after 5 steps; the others record the error of their next steps.
    python tests/rank_worker.py half OUT.json CELLS
        half lists on several ranks: the error md_assemble_neighborlists latches.
    python tests/rank_worker.py nccl BYTES
        the NCCL binding on this process's GPU alone (tmd_comm_nccl_selftest).
    python tests/rank_worker.py perf OUT.json CELLS STEPS REBUILD PRECISION
        the LJ lattice timed over STEPS native timesteps (md_run_timesteps) after warm-up: host
        time per step, the device phase split and this rank's halo size.

The environment names the world size and rank (TINYMD_WORLD_SIZE / TINYMD_RANK) and the
rendezvous port (TINYMD_PORT).
"""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "molecular-dynamics_b200"))
import tinymd  # noqa: E402
from tinymd import ptr  # noqa: E402


def comm_mode(out):
    lib = tinymd.load(build_if_missing=False)
    lib.md_mpi_initialize()
    err = lib.md_last_error()
    res = {"err": err, "msg": lib.md_last_error_string().decode()}
    if err == 0:
        w, r = lib.md_get_world_size(), lib.md_get_world_rank()
        res.update(world=w, rank=r, transport=lib.tmd_comm_transport().decode())
        v = np.array([float(r), 1.5, -2.0 * r])
        res["allreduce_rc"] = lib.tmd_comm_allreduce_sum(ptr(v), 3)
        res["allreduce"] = v.tolist()
        # a ring of 1 MiB messages (larger than a socket buffer)
        n = 1 << 17
        send = np.arange(n, dtype=np.float64) + 1000.0 * r
        recv = np.zeros(n)
        res["ring_rc"] = lib.tmd_comm_sendrecv((r + 1) % w, ptr(send), send.nbytes, (r - 1) % w, ptr(recv),
                                               recv.nbytes)
        res["ring_ok"] = bool(np.array_equal(recv, np.arange(n, dtype=np.float64) + 1000.0 * ((r - 1) % w)))
        world = np.array([0.0, 12.0, 0.0, 10.0, -1.0, 9.0])
        box = np.zeros(6)
        lib.md_get_node_bounding_box(ptr(world), ptr(box))
        res["box"] = box.tolist()
        lib.md_barrier()
        res["err_after"] = lib.md_last_error()
        lib.md_mpi_finalize()
    with open(out, "w") as f:
        json.dump(res, f)


# the DEM benchmark configuration (contact-fixed model, radius 0.6): damping_n, damping_t,
# stiffness, friction
DEM = (0.1, 0.1, 100.0, 0.5)


def md_mode(out, cells, steps, precision, rebuild, benchmark="default"):
    lib = tinymd.load(build_if_missing=False)
    lib.md_mpi_initialize()
    tinymd.check(lib)
    rank = lib.md_get_world_rank()
    grid = np.array([cells] * 3, dtype=np.int32)
    potmin = 1.6796
    dem = benchmark == "granular_gas_fcc"
    dt = 0.001 if dem else 0.005
    world, a1, a2 = np.zeros(6), np.zeros(6), np.zeros(6)
    b = tinymd.BENCHMARKS[benchmark]
    assert lib.tmd_setup_world(b, ptr(grid), potmin, ptr(world), ptr(a1), ptr(a2)) == 0
    box = np.zeros(6)
    lib.md_get_node_bounding_box(ptr(world), ptr(box))
    n = lib.tmd_setup_generate(b, ptr(world), ptr(box), ptr(a1), ptr(a2), potmin)
    m, x, v = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3))
    lib.tmd_setup_fetch(ptr(m), ptr(x), ptr(v))
    lib.md_set_precision(precision)
    if dem:
        lib.md_set_dem_model(1, 0.6)
        sim = tinymd.Simulation(lib, m, x, v, world, box, cutoff=1.2, skin=0.3, force_field="dem", dem=DEM,
                                reneigh=rebuild)
    else:  # main.cpp:664-667: velocities are created for the lattice setups only
        temp = 1.44 if benchmark in ("default", "half") else None
        sim = tinymd.Simulation(lib, m, x, v, world, box, temp=temp, reneigh=rebuild)
    # the first lists' neighbour counts, in the locals' reference order (the setup's order)
    _, x0, _, _ = sim.arrays()
    sizes = np.array([len(l) for l in tinymd.neighbor_lists(lib, sim.n)], dtype=np.int32)
    sim.step(dt, steps)
    nloc, ngh = sim.counts()
    _, x1, v1, f1 = sim.arrays()
    tinymd.check(lib)
    np.savez(out, x0=x0, nb0=sizes, x=x1, v=v1, f=f1, n=nloc, g=ngh, rank=rank, box=box,
             transport=lib.tmd_comm_transport().decode())
    sim.close()
    lib.md_mpi_finalize()


def leave_mode(out, cells):
    """Failure detection without a GPU fault: every rank runs 5 steps of the 8^3-style lattice;
    then the last rank waits for its device work and leaves (the process ends, its connections
    close) while the others try 20 more steps.  Their next halo exchange fails on the host and
    latches MD_ERR_COMM; they return instead of waiting for the missing rank."""
    import time
    lib = tinymd.load(build_if_missing=False)
    lib.md_mpi_initialize()
    tinymd.check(lib)
    rank, world_size = lib.md_get_world_rank(), lib.md_get_world_size()
    grid = np.array([cells] * 3, dtype=np.int32)
    world, a1, a2 = np.zeros(6), np.zeros(6), np.zeros(6)
    assert lib.tmd_setup_world(0, ptr(grid), 1.6796, ptr(world), ptr(a1), ptr(a2)) == 0
    box = np.zeros(6)
    lib.md_get_node_bounding_box(ptr(world), ptr(box))
    n = lib.tmd_setup_generate(0, ptr(world), ptr(box), ptr(a1), ptr(a2), 1.6796)
    m, x, v = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3))
    lib.tmd_setup_fetch(ptr(m), ptr(x), ptr(v))
    sim = tinymd.Simulation(lib, m, x, v, world, box, temp=1.44, reneigh=10)
    sim.step(0.005, 5)
    lib.md_synchronize()  # nothing of this rank in flight on the GPU
    if rank == world_size - 1:
        os._exit(0)  # leaves between steps, without finalising
    t0 = time.perf_counter()
    for _ in range(20):
        lib.md_initial_integration(0.005)
        lib.md_synchronize_ghost_layer()
        lib.md_compute_lennard_jones(False, 2.5, 1.0, 1.0)
        lib.md_final_integration(0.005)
    lib.md_synchronize()
    res = {"rank": rank, "err": lib.md_last_error(), "msg": lib.md_last_error_string().decode(),
           "seconds": time.perf_counter() - t0}
    with open(out, "w") as f:
        json.dump(res, f)
    lib.md_deallocate_grid()


def half_mode(out, cells):
    """Half lists on several ranks: md_assemble_neighborlists(half) latches MD_ERR_UNSUPPORTED."""
    lib = tinymd.load(build_if_missing=False)
    lib.md_mpi_initialize()
    tinymd.check(lib)
    grid = np.array([cells] * 3, dtype=np.int32)
    world, a1, a2 = np.zeros(6), np.zeros(6), np.zeros(6)
    assert lib.tmd_setup_world(0, ptr(grid), 1.6796, ptr(world), ptr(a1), ptr(a2)) == 0
    box = np.zeros(6)
    lib.md_get_node_bounding_box(ptr(world), ptr(box))
    n = lib.tmd_setup_generate(0, ptr(world), ptr(box), ptr(a1), ptr(a2), 1.6796)
    m, x, v = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3))
    lib.tmd_setup_fetch(ptr(m), ptr(x), ptr(v))
    keep = [np.ascontiguousarray(a) for a in (m, x, v)]
    lib.md_initialize_grid(ptr(keep[0]), ptr(keep[1]), ptr(keep[2]), n, ptr(world), ptr(box), 2.8, 60, 100)
    lib.md_copy_data_to_accelerator()
    lib.md_exchange_particles()
    lib.md_borders()
    lib.md_distribute_particles()
    lib.md_assemble_neighborlists(True, 2.8)
    res = {"err": lib.md_last_error(), "msg": lib.md_last_error_string().decode()}
    with open(out, "w") as f:
        json.dump(res, f)
    lib.md_deallocate_grid()
    lib.md_mpi_finalize()


def perf_mode(out, cells, steps, rebuild, precision):
    """The LJ lattice split over the ranks, timed through md_run_timesteps (host clock, after
    warm-up), with the device phase split and this rank's halo size."""
    import time
    lib = tinymd.load(build_if_missing=False)
    lib.md_mpi_initialize()
    tinymd.check(lib)
    grid = np.array([cells] * 3, dtype=np.int32)
    potmin = 1.6796
    world, a1, a2 = np.zeros(6), np.zeros(6), np.zeros(6)
    assert lib.tmd_setup_world(0, ptr(grid), potmin, ptr(world), ptr(a1), ptr(a2)) == 0
    box = np.zeros(6)
    lib.md_get_node_bounding_box(ptr(world), ptr(box))
    n = lib.tmd_setup_generate(0, ptr(world), ptr(box), ptr(a1), ptr(a2), potmin)
    m, x, v = np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3))
    lib.tmd_setup_fetch(ptr(m), ptr(x), ptr(v))
    lib.md_set_precision(precision)
    sim = tinymd.Simulation(lib, m, x, v, world, box, temp=1.44, reneigh=rebuild)
    sim.run(0.005, 2 * rebuild)  # warm-up
    lib.md_barrier()
    lib.md_set_phase_timing(1)
    t0 = time.perf_counter()
    sim.run(0.005, steps)
    lib.md_barrier()
    t1 = time.perf_counter()
    ph = np.zeros(6)
    lib.md_get_phase_times(ptr(ph))
    halo = np.zeros(4, dtype=np.int32)
    lib.tmd_halo_info(ptr(halo))
    nloc, ngh = sim.counts()
    res = {"rank": lib.md_get_world_rank(), "world": lib.md_get_world_size(),
           "transport": lib.tmd_comm_transport().decode(), "n": nloc, "g": ngh, "gself": int(halo[0]),
           "nsend": int(halo[1]), "nrecv": int(halo[2]), "peers": int(halo[3]),
           "us_per_step": (t1 - t0) / steps * 1e6, "phase_ms": ph.tolist()}
    tinymd.check(lib)
    with open(out, "w") as f:
        json.dump(res, f)
    sim.close()
    lib.md_mpi_finalize()


if __name__ == "__main__":
    if sys.argv[1] == "comm":
        comm_mode(sys.argv[2])
    elif sys.argv[1] == "nccl":  # the NCCL binding on this GPU alone (one-rank communicator)
        rc = tinymd.load(build_if_missing=False).tmd_comm_nccl_selftest(int(sys.argv[2]))
        print("nccl selftest", rc)
        sys.exit(0 if rc == 0 else 1)
    elif sys.argv[1] == "leave":
        leave_mode(sys.argv[2], int(sys.argv[3]))
    elif sys.argv[1] == "half":
        half_mode(sys.argv[2], int(sys.argv[3]))
    elif sys.argv[1] == "perf":
        perf_mode(sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), int(sys.argv[5]), int(sys.argv[6]))
    else:
        md_mode(sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), int(sys.argv[5]),
                int(sys.argv[6]) if len(sys.argv) > 6 else 10, sys.argv[7] if len(sys.argv) > 7 else "default")
