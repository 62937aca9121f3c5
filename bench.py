"""Benchmark of the tinyMD B200 timestep: LJ atom-steps/s on one B200.

Workload (the configuration the metric is quoted on): LJ 'default' FCC
lattice of 32x32x32 unit cells (131,072 atoms, lattice constant 1.6796),
velocities from the per-site Park-Miller seeds rescaled to T = 1.44,
eps = sigma = 1, cutoff 2.5, skin 0.3, dt 0.005, reneighbour every 20 steps,
full neighbour lists.  A "step" is one MD timestep (main.cpp:715-776).

value   atom-steps/s of the mixed form (FP64 state / FP32 pair forces) over K
        device-timed steps (CUDA events around each step on the library's
        stream; the 131k working set fits in L2, so L2 is flushed before every
        timed step, outside the timed interval, by writing a 256 MiB buffer and
        reading it back: the step starts cold and without the flush's dirty
        lines to write back).
forms   the FP64 form's atom-steps/s on the same workload, the ratio, and the
        mixed form's max force error / rms force against FP64 positions.
e2e     the same metric through the C ABI with host buffers: md_initialize_grid
        from host arrays, upload, K steps, download and md_write_grid_data_to_arrays,
        timed on the host clock around the whole run.
roofline  the mixed force kernel: algorithmic bytes per launch / average
        launch time (CUDA events around each force launch) against the
        measured HBM bandwidth.
cpu_baseline  the CPU oracle (a restatement of the reference's cpu backend)
        timed on this host over a bounded sample of the same workload.
drift   total energy per atom over 1000 steps of the workload, sampled every
        50 steps, in both forms (max |E(t) - E(0)| / N and the ratio).
adjoint the differentiable form on 16x16x16 cells (16,384 atoms), 200 steps,
        checkpoints every 20 steps: device time of the backward pass over the
        forward pass.
workloads the 131k lattice with half lists; the 'half' setup at 64^3 (524,288
        atoms, lists larger than L2) with its force-kernel roofline; DEM at 48^3
        (FCC diagonal split and the reference's granular gas, reference closure
        and contact-fixed model), each in both forms.

--impl reference runs that CPU path alone (all host threads) on the same
workload and prints the same JSON line.  Under torchrun each rank runs an
independent replica (the path does not shard); value sums the replicas and
uses the max time over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "molecular-dynamics_b200")
sys.path.insert(0, PKG)

METRIC = "LJ atom-steps/s, 1 B200: mixed-FP32 vs FP64 at stated error; adjoint/fwd time"
UNIT = "atom-steps/s"
CELLS = (32, 32, 32)
DT = 0.005
L2_FLUSH_BYTES = 256 << 20
PROFILE_EVERY = 10  # force launches timed by events: one in ten, spread over the timed steps
DRIFT_STEPS = 1000
DRIFT_EVERY = 50


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_traffic():
    """Per-launch DRAM bytes of the mixed force kernel from the committed ncu summary, and its
    L2 / L1 / issue fractions of peak from the same capture (None where absent)."""
    p = os.path.join(ROOT, "profiles", "force_lj_mixed_131k.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch"), {
            "l2_sectors_per_launch": d.get("l2_sectors_per_launch"),
            "l2_throughput_frac": (d["l2_throughput_pct_of_peak"] / 100.0 if "l2_throughput_pct_of_peak" in d
                                   else None),
            "l1_throughput_frac": (d["l1tex_throughput_pct_of_peak"] / 100.0
                                   if "l1tex_throughput_pct_of_peak" in d else None),
            "issue_frac": (d["sm_inst_executed_pct_of_peak"] / 100.0 if "sm_inst_executed_pct_of_peak" in d
                           else None)}
    return None, None


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.file:
            return None
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:  # a timed region shorter than the sampling period: one sample right after it
            try:
                out = subprocess.run(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-i",
                                      str(self.index)], capture_output=True, text=True, timeout=10).stdout
                rows = [[p.strip() for p in line.split(",")] for line in out.splitlines() if line.count(",") >= 8]
            except (OSError, subprocess.TimeoutExpired):
                rows = []
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def dist_init(world, backend):
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist if world > 1 else None


def allreduce_max(x, dist, device=None):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def replica_rate(atoms_per_rank, world, steps, ms_local, dist, device=None):
    """Whole-job atom-steps/s of `world` independent replicas: all ranks' atoms over the
    slowest rank's time (every rank calls this with its own time, in the same order)."""
    ms = allreduce_max(ms_local, dist, device)
    return atoms_per_rank * world * steps / (ms * 1e-3), ms


# ---------------------------------------------------------------------------
def cpu_info():
    """CPU model, the AVX-512 feature flags and the host threads of this machine."""
    model, flags = None, []
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if model is None and line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                if not flags and line.startswith("flags"):
                    flags = sorted(x for x in line.split(":", 1)[1].split() if x.startswith("avx512"))
    except OSError:
        pass
    return {"model": model, "avx512_flags": flags, "threads": os.cpu_count()}


_native_oracle = None


def native_oracle():
    """The oracle compiled on this host with -march=native (make -C oracle native, always remade
    here so a copy built on another machine is never timed); falls back to the portable build."""
    global _native_oracle
    if _native_oracle is None:
        r = subprocess.run(["make", "-B", "-C", os.path.join(ROOT, "oracle"), "native"], capture_output=True)
        if r.returncode == 0:
            _native_oracle = (os.path.join(ROOT, "oracle", "_build_native", "libtinymd_oracle.so"), "-O3 -march=native")
        else:
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
            _native_oracle = (os.path.join(ROOT, "oracle", "_build", "libtinymd_oracle.so"),
                              "-O3 -march=x86-64-v3 (native build failed)")
    return _native_oracle


def cpu_lattice(cells=CELLS):
    """The workload's lattice from the reference's own generator (oracle/_ref), so the CPU arm
    loads no product code; the product's identical generator only where oracle/_ref is absent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_lattice
    if ref_lattice.available():
        return ref_lattice.reference_lattice(cells), "reference initialize.h (oracle/_ref)"
    import tinymd
    return tinymd.setup_particles("default", cells, lib=tinymd.load()), "product setups (oracle/_ref not built)"


def cpu_run(steps, threads, cells=CELLS, warmup=1):
    """The oracle's CPU path on `threads` host threads; returns (atom-steps/s, atoms, seconds, notes)."""
    import tinymd
    path, flags = native_oracle()
    ora = tinymd.open_library(path)
    ora.oracle_set_threads(threads)
    (m, x, v, world, rank), source = cpu_lattice(cells)
    sim = tinymd.Simulation(ora, m, x, v, world, rank, temp=1.44)
    sim.step(DT, warmup)
    t0 = time.perf_counter()
    sim.step(DT, steps)
    t = time.perf_counter() - t0
    sim.close()
    notes = {"build": flags, "lattice": source, "cpu": cpu_info()}
    return len(m) * steps / t, len(m), t, notes


def run_reference(args):
    rank, world, local = dist_info()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    steps = args.steps
    rate, natoms, secs, notes = cpu_run(steps, threads, warmup=min(args.warmup, 20))
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3 / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded FCC lattice, reference Park-Miller velocities)",
        "config": {"workload": "lj_default_fcc_32x32x32_131072_atoms_full_list", "atoms": natoms, "dt": DT,
                   "reneigh": 20, "cutoff": 2.5, "skin": 0.3},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{natoms} atoms x {steps} timesteps (full workload), OpenMP over atoms",
                         **notes},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def fused_kernel_bytes(mean_nb, ghosts_per_atom):
    """Algorithmic bytes per atom of the timed force kernel, which also finishes the step and
    starts the next one: the mixed full-list force (count, list entry and FP32 neighbour
    position per pair, own position, FP32 force: 4 + 16 n + 24) and the integration with the
    ghost update it took over (5 x 24 per atom, 4 + 3 + 24 + 24 per ghost)."""
    force = 4 + mean_nb * (4 + 12) + 12 + 12
    step = 5 * 24 + ghosts_per_atom * (4 + 3 + 24 + 24)
    return force, step


def timed_steps(lib, sim, steps, flush):
    """Device time of `steps` native timesteps, each bracketed by CUDA events on the
    library stream, with `flush` (a device buffer larger than L2) overwritten before
    each step outside the timed interval."""
    step_ms = np.zeros(steps, dtype=np.float32)
    launches0 = lib.md_kernel_launches()
    sim.run(DT, steps, step_ms=step_ms, flush=(ctypes.c_void_p(flush.data_ptr()), flush.numel() * 4))
    return float(step_ms.astype(np.float64).sum()), lib.md_kernel_launches() - launches0


def energy_drift(lib, tm, parts, precision):
    """Total energy per atom, (KE + U) / N with U from the full list, sampled every
    DRIFT_EVERY steps over DRIFT_STEPS steps of the benchmark workload in one form."""
    lib.md_set_precision(precision)
    lib.md_set_thermo(1)
    sim = tm.Simulation(lib, *parts, temp=1.44)
    n = len(parts[0])
    t = np.zeros(4)
    series = []
    for k in range(DRIFT_STEPS // DRIFT_EVERY + 1):
        if k:
            sim.run(DT, DRIFT_EVERY)
        else:  # step 0: forces and kinetic energy of the initial state
            sim.force()
            lib.md_final_integration(0.0)
        if lib.md_get_thermo(tm.ptr(t)) != 0:
            tm.check(lib)
        series.append((0.5 * t[3] + 0.5 * t[0]) / n)  # t = {U sum, virial, pairs, v.v}
    sim.close()
    lib.md_set_thermo(0)
    lib.md_set_precision(0)
    e = np.array(series)
    return {"e0_per_atom": float(e[0]), "max_abs_drift_per_atom": float(np.max(np.abs(e - e[0]))),
            "end_drift_per_atom": float(e[-1] - e[0])}


def measure(lib, tm, parts, precision, steps, warmup, flush, half=False, force_field="lj", dem=(0.0, 0.0, 0.0, 0.0),
            cutoff=2.5, dt=DT, temp=1.44, profile_force=False):
    """Device-timed steps of one workload in one form: (atom-steps/s, ms per step, None or, with
    profile_force, (force ms per launch, ghosts per atom, mean list length))."""
    lib.md_set_precision(precision)
    if half:
        lib.md_set_half_mode(1)  # half lists that keep the periodic-boundary pairs
    sim = tm.Simulation(lib, *parts, temp=temp, half=half, force_field=force_field, dem=dem, cutoff=cutoff)
    sim.run(dt, warmup)
    if profile_force:
        lib.md_profile_enable(1 << 0)
        lib.md_profile_sample(PROFILE_EVERY)
        lib.md_profile_reset()
    step_ms = np.zeros(steps, dtype=np.float32)
    sim.run(dt, steps, step_ms=step_ms, flush=(ctypes.c_void_p(flush.data_ptr()), flush.numel() * 4))
    fms = None
    if profile_force:
        nl, t = ctypes.c_longlong(), ctypes.c_double()
        lib.md_profile_get(0, ctypes.byref(nl), ctypes.byref(t))
        lib.md_profile_enable(0)
        lib.md_profile_sample(1)
        natoms = len(parts[0])
        sizes = np.zeros(natoms, dtype=np.int32)
        lists = np.zeros((natoms, 1), dtype=np.int32)
        lib.md_get_neighbor_lists(tm.ptr(sizes), tm.ptr(lists), 1)
        fms = (t.value / max(nl.value, 1), sim.counts()[1] / natoms, float(sizes.mean()))
    sim.close()
    lib.md_set_half_mode(0)
    lib.md_set_precision(0)
    ms = float(step_ms.astype(np.float64).sum())
    return len(parts[0]) * steps / (ms * 1e-3), ms / steps, fms


def kernel_table(lib, tm, parts, peak, steps=60):
    """Per kernel class of the mixed 131k workload: mean launch time from CUDA events around every
    launch (a separate, untimed run: events drain the stream) and the SURVEY 8(d) algorithmic bytes
    per launch, as GB/s and a fraction of the measured HBM copy bandwidth."""
    lib.md_set_precision(1)
    sim = tm.Simulation(lib, *parts, temp=1.44)
    sim.run(DT, 20)
    n, g = sim.counts()
    sizes = np.zeros(n, dtype=np.int32)
    lists = np.zeros((n, 1), dtype=np.int32)
    lib.md_get_neighbor_lists(tm.ptr(sizes), tm.ptr(lists), 1)
    nb = float(sizes.mean())
    lib.md_profile_enable(0xffff)
    lib.md_profile_sample(1)
    lib.md_profile_reset()
    sim.run(DT, steps)
    # bytes per launch: force (4 + 16n + 24 per atom, plus the fused integration 5 x 24 per atom and
    # 55 per ghost), list build (27 x 24 staged + 4n per atom), binning (~128 per slot reordered),
    # borders (~80 per local scanned, ~200 per ghost written)
    model = {"force_lj": n * (4 + 16 * nb + 24 + 120) + g * 55, "neighbor_list": n * (27 * 24 + 4 * nb),
             "binning": (n + g) * 128, "borders": n * 80 + g * 200}
    out = {}
    for k in range(lib.md_profile_count()):
        name = lib.md_profile_name(k).decode()
        if name not in model:
            continue
        nl, t = ctypes.c_longlong(), ctypes.c_double()
        lib.md_profile_get(k, ctypes.byref(nl), ctypes.byref(t))
        if nl.value == 0:
            continue
        us = t.value * 1e3 / nl.value
        gbs = model[name] / (us * 1e-6) / 1e9
        out[name] = {"launches": nl.value, "launch_us": us, "bytes_per_launch": model[name], "GB/s": gbs,
                     "frac_of_hbm": gbs / peak}
    lib.md_profile_enable(0)
    sim.close()
    lib.md_set_precision(0)
    return out


def workloads(lib, tm, flush, peak):
    """The other measured configurations (atom-steps/s in both forms)."""
    out = {}
    parts = tm.setup_particles("default", CELLS, lib=lib)
    row = {"atoms": len(parts[0]), "steps": 300, "lists": "half (periodic-boundary pairs kept, reactions to roots)"}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        row[name] = measure(lib, tm, parts, prec, 300, 20, flush, half=True)[0]
    row["mixed_over_fp64"] = row["mixed"] / row["fp64"]
    out["lj_default_fcc_32x32x32_131072_atoms_half_list"] = row
    # the 'half' setup at 64^3: lists (~160 MB) larger than L2
    parts = tm.setup_particles("half", (64, 64, 64), lib=lib)
    row = {"atoms": len(parts[0]), "steps": 500, "lists": "full"}
    fms = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        row[name], _, fms[name] = measure(lib, tm, parts, prec, 500, 20, flush, profile_force=True)
    row["mixed_over_fp64"] = row["mixed"] / row["fp64"]
    launch_ms, ghosts_per_atom, mean_nb = fms["mixed"]
    fb, sb = fused_kernel_bytes(mean_nb, ghosts_per_atom)
    b32 = fb + sb
    achieved = len(parts[0]) * b32 / (launch_ms * 1e-3) / 1e9
    row["roofline_mixed_force"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                   "frac": achieved / peak, "launch_ms": launch_ms, "bytes_per_atom": b32,
                                   "force_bytes_per_atom": fb, "integrate_ghost_bytes_per_atom": sb,
                                   "mean_list_length": mean_nb,
                                   # ncu at this size: 263 MB of DRAM traffic per launch in 116 us (2.3 TB/s,
                                   # 0.35 of the measured peak); the neighbour gathers are served by L2
                                   "traffic": 263.2e6, "traffic_source": "profiles/lj_mixed_full_524k_dram.md",
                                   "limiter": "instruction issue and latency (71 M warp instructions per launch)"}
    out["lj_half_fcc_64x64x64_524288_atoms_full_list"] = row
    # DEM at 48^3: the FCC diagonal split and the reference's granular gas, with the
    # reference closure (zero force) and the contact-fixed model (R = 0.6)
    dem = (0.1, 0.1, 100.0, 0.5)  # damping_n, damping_t, stiffness, friction
    for setup in ("granular_gas_fcc", "granular_gas"):
        parts = tm.setup_particles(setup, (48, 48, 48), lib=lib)
        for model, radius in (("reference_closure", 1.0), ("contact_fixed_R0.6", 0.6)):
            lib.md_set_dem_model(1 if model.startswith("contact") else 0, radius)
            row = {"atoms": len(parts[0]), "steps": 300, "cutoff": 1.2, "skin": 0.3, "dt": 0.001,
                   "stiffness": 100.0, "damping_n": 0.1, "damping_t": 0.1, "friction": 0.5}
            for name, prec in (("fp64", 0), ("mixed", 1)):
                row[name] = measure(lib, tm, parts, prec, 300, 20, flush, force_field="dem", dem=dem, cutoff=1.2,
                                    dt=0.001, temp=None)[0]
            row["mixed_over_fp64"] = row["mixed"] / row["fp64"]
            out[f"dem_{setup}_48x48x48_{model}"] = row
    lib.md_set_dem_model(0, 1.0)
    return out


def adjoint_times(lib, tm):
    """Differentiable form on its own workload: 16x16x16 cells (16,384 atoms), 200 steps of dt
    0.005, checkpoints every 20 steps, mixed forward; device ms of one forward and one backward
    pass (after one untimed pass of each)."""
    import torch
    from tinymd import adjoint
    parts = tm.setup_particles("default", (16, 16, 16), lib=lib)
    sim = tm.Simulation(lib, *parts, temp=1.44)
    v0 = adjoint.initial_velocities(lib, sim)
    adjoint.configure(lib, steps=200, reneigh=20, dt=DT, precision=1, shifted_energy=True)
    rows = []
    for _ in range(2):
        v = torch.tensor(v0, requires_grad=True)
        e = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
        s = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
        adjoint.TrajectoryLoss.apply(v, e, s, lib).backward()
        rows.append(adjoint.times(lib))
    sim.close()
    fwd, bwd = rows[-1]
    return {"workload": "lj_default_fcc_16x16x16_16384_atoms_200_steps_checkpoint_20", "forward_ms": fwd,
            "backward_ms": bwd, "backward_over_forward": bwd / fwd,
            "loss": "MSD + shifted U(x_T)/N; grads wrt eps, sigma, all initial velocities"}


def run_ours(args):
    import torch
    import tinymd as tm
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = dist_init(world, "nccl")
    lib = tm.load()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    parts = tm.setup_particles("default", CELLS, lib=lib)
    natoms = len(parts[0])
    K, W = args.steps, args.warmup
    result = {}

    # ---- FP64 form ---------------------------------------------------------------
    lib.md_set_precision(0)
    sim = tm.Simulation(lib, *parts, temp=1.44)
    sim.run(DT, W)
    barrier(dist)
    ms64, _ = timed_steps(lib, sim, K, flush)
    sim.close()
    value64, ms64 = replica_rate(natoms, world, K, ms64, dist, dev)

    # ---- mixed form (headline) ----------------------------------------------------
    lib.md_set_precision(1)
    sim = tm.Simulation(lib, *parts, temp=1.44)
    sim.run(DT, W)
    # events around one LJ force launch in PROFILE_EVERY (each pair of events costs the
    # stream a few microseconds, so timing every launch would slow the timed steps)
    lib.md_profile_enable(1 << 0)
    lib.md_profile_sample(PROFILE_EVERY)
    lib.md_profile_reset()
    barrier(dist)
    with ClockSampler(local) as clk:
        ms32, launches = timed_steps(lib, sim, K, flush)
    clocks = clk.summary()
    nl = ctypes.c_longlong()
    fms = ctypes.c_double()
    lib.md_profile_get(0, ctypes.byref(nl), ctypes.byref(fms))
    lib.md_profile_enable(0)
    lib.md_profile_sample(1)
    # mean list length of the current lists (full list, FP64 cutoff 2.8)
    sizes = np.zeros(natoms, dtype=np.int32)
    lists = np.zeros((natoms, 1), dtype=np.int32)
    lib.md_get_neighbor_lists(tm.ptr(sizes), tm.ptr(lists), 1)
    mean_nb = float(sizes.mean())
    ghosts_per_atom = sim.counts()[1] / natoms
    # force and potential-energy error of the mixed form on the same state: both forms'
    # forces (and thermo sums) on the positions the timed run ended with
    lib.md_set_thermo(1)
    th32, th64 = np.zeros(4), np.zeros(4)
    sim.force()
    lib.md_final_integration(0.0)
    lib.md_get_thermo(tm.ptr(th32))
    _, _, f32 = tm.full_state(lib)
    lib.md_set_precision(0)
    sim.force()
    lib.md_final_integration(0.0)
    lib.md_get_thermo(tm.ptr(th64))
    _, _, f64 = tm.full_state(lib)
    lib.md_set_thermo(0)
    ferr = float(np.max(np.abs(f32 - f64)) / np.sqrt(np.mean(f64 ** 2)))
    u32, u64 = 0.5 * th32[0] / natoms, 0.5 * th64[0] / natoms  # full lists count each pair twice
    eerr = {"fp64_u_per_atom": u64, "mixed_minus_fp64_u_per_atom": u32 - u64,
            "relative": abs(u32 - u64) / abs(u64)}
    sim.close()
    value, ms32 = replica_rate(natoms, world, K, ms32, dist, dev)

    drift = {"steps": DRIFT_STEPS, "every": DRIFT_EVERY}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        drift[name] = energy_drift(lib, tm, parts, prec)
    drift["mixed_over_fp64"] = drift["mixed"]["max_abs_drift_per_atom"] / max(
        drift["fp64"]["max_abs_drift_per_atom"], 1e-300)
    adj = adjoint_times(lib, tm)
    more = workloads(lib, tm, flush, peaks()[0])
    ktable = kernel_table(lib, tm, parts, peaks()[0])

    # ---- end to end through the C ABI with host buffers ---------------------------
    m, x, v, world_box, rank_box = parts

    def e2e_best(precision):
        """Best of three host-clock runs (the host clock also sees the box's other load):
        (total, set-up: grid, device allocation, upload, first lists and force; steps; copy back)."""
        lib.md_set_precision(precision)
        runs = []
        for rep in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s = tm.Simulation(lib, m, x, v, world_box, rank_box, temp=1.44)
            lib.md_synchronize()
            ta = time.perf_counter()
            s.run(DT, K)
            lib.md_synchronize()
            tb = time.perf_counter()
            s.arrays()  # md_copy_data_from_accelerator + md_write_grid_data_to_arrays
            t1 = time.perf_counter()
            s.close()
            runs.append((t1 - t0, ta - t0, tb - ta, t1 - tb))
        lib.md_set_precision(0)
        return min(runs)

    best = e2e_best(1)
    best64 = e2e_best(0)
    e2e_value, e2e_ms = replica_rate(natoms, world, K, best[0] * 1e3, dist, dev)
    e2e_value64, _ = replica_rate(natoms, world, K, best64[0] * 1e3, dist, dev)
    h2d = natoms * (8 + 24 + 24)  # masses, positions, velocities up
    d2h = natoms * (8 + 24 + 24 + 24)  # the locals' masses, positions, velocities, forces down

    peak, peak_kind = peaks()
    force_ms = fms.value / max(nl.value, 1)
    # algorithmic bytes per atom and force launch (payload only, padding excluded): the list
    # count, per neighbour a 4-byte index and a 12-byte FP32 position, own FP32 position, FP32 force
    force_bytes, step_bytes = fused_kernel_bytes(mean_nb, ghosts_per_atom)
    bytes_per_atom = force_bytes + step_bytes
    achieved = natoms * bytes_per_atom / (force_ms * 1e-3) / 1e9
    traffic, cache_fracs = measured_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms32 / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 state + f32 pair forces (mixed form)",
        "data": "synthetic (seeded FCC lattice, reference Park-Miller velocities)",
        "config": {"workload": "lj_default_fcc_32x32x32_131072_atoms_full_list", "atoms_per_gpu": natoms,
                   "dt": DT, "reneigh": 20, "cutoff": 2.5, "skin": 0.3,
                   "l2": "flushed before every timed step: a 256 MiB buffer written, then read back (the read "
                         "evicts the written lines), outside the timed interval",
                   "parallelism": f"replicas x{world}"},
        "forms": {"mixed": value, "fp64": value64, "mixed_over_fp64": value / value64,
                  "mixed_max_force_err_over_rms": ferr, "mixed_energy_err": eerr},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind, "kernel": "force_lj (mixed, full list)",
                     # what the ncu capture of this kernel shows limits it (profiles/lj_mixed_full_131k_ncu.md)
                     "limiter": "instruction issue and latency, not HBM: ncu issue active 59 %, DRAM 21 % of peak, "
                                "gathers served by L1 (74 % hit) and L2",
                     "traffic_frac": (traffic / (force_ms * 1e-3) / 1e9 / peak) if traffic else None,
                     "bytes_per_atom": bytes_per_atom, "force_bytes_per_atom": force_bytes,
                     "integrate_ghost_bytes_per_atom": step_bytes, "mean_list_length": mean_nb,
                     "launch_ms": force_ms, "launches_timed": nl.value, "timed_every": PROFILE_EVERY,
                     # list count and entries plus the atom's own FP64 position and force: what
                     # must come from HBM once per step whatever the gathers hit
                     "compulsory_bytes_per_atom": 4 + 4 * mean_nb + 48,
                     "compulsory_frac": natoms * (4 + 4 * mean_nb + 48) / (force_ms * 1e-3) / 1e9 / peak,
                     # from the ncu capture: the gathers hit L1/L2, and neither runs near its peak
                     "ncu_fracs": cache_fracs},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
                "d2h_bytes_per_step": d2h / K,
                "note": "md_initialize_grid from host arrays .. K steps .. md_write_grid_data_to_arrays, host clock",
                "setup_ms": best[1] * 1e3, "steps_ms": best[2] * 1e3, "copy_back_ms": best[3] * 1e3,
                "fp64": {"value": e2e_value64, "setup_ms": best64[1] * 1e3, "steps_ms": best64[2] * 1e3,
                         "copy_back_ms": best64[3] * 1e3}},
        "drift": drift,
        "adjoint": adj,
        "workloads": more,
        "kernels": ktable,
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        steps = 40
        rate, n_cpu, secs, notes = cpu_run(steps, threads)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{n_cpu} atoms x {steps} timesteps of the same workload", **notes}
        # one thread: what the reference's cpu backend does (its -t flag is only printed)
        rate1, _, _, _ = cpu_run(10, 1)
        line["cpu_baseline_1thread"] = {"value": rate1, "unit": UNIT, "cores": 1, "kind": "port",
                                        "sample": f"{n_cpu} atoms x 10 timesteps of the same workload"}
    if dist is not None:
        barrier(dist)
        import torch.distributed as td
        td.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


import ctypes  # noqa: E402


def profile_case(args):
    """One workload in one form for `args.steps` steps, untimed (an ncu target):
    mixed / fp64 [_half]   the 131k LJ workload (full lists, or half lists keeping boundary pairs)
    mixed_c2 / fp64_c2     the 'half' setup at 64^3 (524,288 atoms), full lists
    dem_mixed / dem_fp64   DEM at 48^3, FCC diagonal split, contact-fixed model (R = 0.6)
    adjoint                the differentiable form: 16^3 cells, one forward and one backward pass"""
    import tinymd as tm
    lib = tm.load()
    case = args.profile_case
    if case == "adjoint":
        import torch
        from tinymd import adjoint
        parts = tm.setup_particles("default", (16, 16, 16), lib=lib)
        sim = tm.Simulation(lib, *parts, temp=1.44)
        v0 = adjoint.initial_velocities(lib, sim)
        adjoint.configure(lib, steps=args.steps, reneigh=20, dt=DT, precision=1, shifted_energy=True)
        v = torch.tensor(v0, requires_grad=True)
        e = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
        sg = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
        adjoint.TrajectoryLoss.apply(v, e, sg, lib).backward()
        sim.close()
    else:
        lib.md_set_precision(1 if case.startswith("mixed") or case == "dem_mixed" else 0)
        half = case.endswith("_half")
        if half:
            lib.md_set_half_mode(1)
            lib.md_set_ghost_mode(1)
        if case.startswith("dem"):
            lib.md_set_dem_model(1, 0.6)
            parts = tm.setup_particles("granular_gas_fcc", (48, 48, 48), lib=lib)
            sim = tm.Simulation(lib, *parts, force_field="dem", dem=(0.1, 0.1, 100.0, 0.5), cutoff=1.2)
            sim.run(0.001, args.steps)
        else:
            cells, setup = ((64, 64, 64), "half") if case.endswith("_c2") else (CELLS, "default")
            sim = tm.Simulation(lib, *tm.setup_particles(setup, cells, lib=lib), temp=1.44, half=half)
            sim.run(DT, args.steps)
        sim.close()
    print(f"profile case {case}: {args.steps} steps, error code {lib.md_last_error()}")
    return 0 if lib.md_last_error() == 0 else 1


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-case", choices=["mixed", "fp64", "mixed_half", "fp64_half", "mixed_c2", "fp64_c2",
                                               "dem_mixed", "dem_fp64", "adjoint"],
                    help="run the workload for --steps steps in one form and exit (for ncu captures)")
    args = ap.parse_args()
    if args.profile_case:
        return profile_case(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
