"""Benchmark of the MD step hot path: 1,048,576-atom Lennard-Jones argon, NVE, float32.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one velocity-Verlet step of the whole system: the drift with the on-GPU reuse
check, the neighbor rebuild behind its device flag, and the forces with the second half kick.
Workload (synthetic, seeded): a 64^3-cell FCC lattice (4 sites per cell) in L = 36.77 nm
(rho = 21.1 per nm^3) with Gaussian jitter 0.02 nm, sigma 0.34 nm, epsilon 0.996 kJ/mol, mass
39.948 Da, cutoff 1.0 nm, skin 0.1 nm, dt 0.004 ps, Maxwell-Boltzmann velocities at 120 K.
The working set (positions, velocities, forces, neighbor list of about 0.4 GB) is larger than
the 126 MB L2, so no flush is needed between steps.

Prints one JSON line (rank 0). With N > 1 each rank runs its own replica (the path does not
shard: replicas only); ``value`` is the atom-steps of all ranks over the slowest rank's time.
``--impl reference`` times the oracle port of the reference's algorithm on the host cores.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

ATOMS_PER_SIDE_CELLS = 64
LENGTH = 36.77
SIGMA, EPSILON, MASS, CUTOFF, SKIN, TIMESTEP, TEMPERATURE = 0.34, 0.996, 39.948, 1.0, 0.1, 0.004, 120.0
WORKLOAD = "LJ argon NVE, 1,048,576 atoms (64^3-cell FCC, L=36.77 nm, rho=21.1/nm^3), fp32"
METRIC = "atom-steps/s, 1M-atom LJ fp32 NVE"
# DRAM bytes (read + write) of one launch of the step's force kernel on this workload, from
# ncu's dram__bytes_read.sum + dram__bytes_write.sum on a B200 (the pair-list kernel), and what
# its counters say bounds it.
FORCE_KERNEL_DRAM_BYTES = 275.7e6
FORCE_KERNEL_LIMITER = "issue and shared-memory gathers, not HBM (ncu: issue slots and LSU wavefronts)"

# Algorithmic traffic of the force kernel per atom and launch: read x (12 B) and v (12 B),
# write F (12 B) and v (12 B), and the neighbor indices a half list needs, 58.8 x 4 B.
FORCE_BYTES_PER_ATOM = 48 + 58.8 * 4
# The step's algorithmic cost per atom-step: 307 B (state 72 B + 235 B indices) and
# 44.2 in-cutoff half pairs x 26 flop.
STEP_BYTES_PER_ATOM = 307.0
STEP_FLOPS_PER_ATOM = 44.2 * 26


def load_peaks() -> dict:
    """HBM copy GB/s and dense BF16 TFLOP/s (burst and sustained) measured on this pool's
    B200s, else the earlier pool measurement (6.65 TB/s, 1.59 and 1.4 PFLOP/s)."""
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        peaks = json.loads(path.read_text())
        bf16 = float(peaks.get("bf16_tflops", 1590.0))
        return {"hbm_gbs": float(peaks["hbm_gbs"]), "bf16_tflops": bf16,
                "bf16_tflops_sustained": float(peaks.get("bf16_tflops_sustained", bf16)),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.process = None

    def __enter__(self):
        try:
            self.process = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL,
            )
        except OSError:
            self.process = None
        return self

    def __exit__(self, *exc):
        if self.process is not None:
            time.sleep(0.25)
            self.process.terminate()
            self.process.wait(timeout=10)

    def summary(self) -> dict:
        self.file.seek(0)
        rows = [line.split(",") for line in self.file.read().strip().splitlines() if line]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        clocks = [float(r[1]) for r in rows if len(r) > 2 and r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({name for r in rows for name, value in zip(names, r[5:9])
                          if "Active" in value and "Not" not in value})
        return {
            "sm_mhz": statistics.median(clocks) if clocks else None,
            "sm_max_mhz": float(rows[0][2]) if rows[0][2].strip().replace(".", "").isdigit() else None,
            "reasons": reasons,
            "samples": len(rows),
        }


def build_system(torch, device, seed: int):
    from nabladyn_b200 import lattice, md, potential

    positions, cell = lattice.fcc(ATOMS_PER_SIDE_CELLS, LENGTH, 0.02, seed)
    n = positions.shape[0]
    dtype = torch.float32
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=device),
        sigma=torch.tensor([SIGMA], dtype=dtype, device=device),
        epsilon=torch.tensor([EPSILON], dtype=dtype, device=device),
        cutoff=CUTOFF,
    )
    masses = torch.full((n,), MASS, dtype=dtype, device=device)
    velocities = md.maxwell_boltzmann(masses, TEMPERATURE, seed=seed)
    host = {
        "positions": torch.tensor(positions, dtype=dtype).pin_memory(),
        "velocities": velocities.cpu().pin_memory(),
    }
    x = host["positions"].to(device)
    box = torch.tensor(cell, dtype=dtype, device=device)
    simulation = md.nve(model, x, velocities, masses, box, timestep=TIMESTEP, skin=SKIN)
    return simulation, host, n


def frame_accuracy(simulation) -> dict:
    """The current frame's float32 forces, energy and virial against a float64 evaluation of
    the same coordinates (the engine's cell-order positions, unwrapped as the kernels used
    them): this package's float64 LJ kernels over a float64 neighbor list of all atoms, which
    the tests pin to the float64 oracle (to 1e-9, and on a 4,096-atom sample of this box)."""
    import torch

    from nabladyn_b200 import neighbors, potential, quantity, space

    panel = simulation.sample()  # forces and virial of the current frame, float32
    engine = simulation._engine
    device = engine.device
    x32 = engine.tensors["positions"][:, :3]
    f32 = engine.tensors["forces"].double()
    totals = engine.totals.tolist()
    w32 = torch.tensor([[totals[2], totals[5], totals[6]], [totals[5], totals[3], totals[7]],
                        [totals[6], totals[7], totals[4]]], dtype=torch.float64)
    n = x32.shape[0]
    cell64 = engine.cell.double()
    x64, _ = space.wrap(x32.double(), cell64)
    exact = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=device),
        sigma=torch.tensor([SIGMA], dtype=torch.float64, device=device),
        epsilon=torch.tensor([EPSILON], dtype=torch.float64, device=device), cutoff=CUTOFF)
    listing = neighbors.NeighborList(CUTOFF, skin=0.0)
    listing.allocate(x64, cell64)
    e64, f64, w64 = quantity.energy_force_virial(exact)(x64, cell64, listing.tensors())
    w64 = w64.cpu()
    out = {
        "force_error_vs_fp64": float((f32 - f64).norm() / f64.norm()),
        "energy_error_vs_fp64": abs(float(panel["potential_energy"]) - float(e64)) / abs(float(e64)),
        "virial_error_vs_fp64": float((w32 - w64).norm() / w64.norm()),
        "measure": "||x32 - x64|| / ||x64|| on the last timed frame, all atoms",
    }
    del listing, f64
    torch.cuda.empty_cache()
    return out


def cpu_port_rate(steps: int = 3, cells: int = 24, threads: int | None = None) -> dict:
    """The oracle port of the reference's step on the host: pairs by the C restatement of the
    neighbor operator (one thread), LJ and velocity Verlet in float64 numpy with the pairs
    split over ``threads`` host threads (all the host's by default; numpy releases the GIL).

    Sample: a cells^3-cell FCC block of the same density (4 cells^3 atoms), ``steps`` steps,
    the pairs rebuilt every step (the port keeps no list between steps).
    """
    from concurrent.futures import ThreadPoolExecutor

    from nabladyn_b200 import lattice
    from oracle import lj
    from oracle import neighbors as on

    threads = threads or os.cpu_count() or 1
    pool = ThreadPoolExecutor(threads)

    def forces_of(x, first, second):
        bounds = np.linspace(0, len(first), threads + 1).astype(np.int64)
        parts = pool.map(
            lambda k: lj.energy_force_virial(x, cell, first[bounds[k]:bounds[k + 1]],
                                             second[bounds[k]:bounds[k + 1]], [SIGMA],
                                             [EPSILON], CUTOFF)[1],
            range(threads))
        return sum(parts)

    length = LENGTH * cells / ATOMS_PER_SIDE_CELLS
    positions, cell = lattice.fcc(cells, length, 0.02, seed=1)
    n = positions.shape[0]
    rng = np.random.default_rng(1)
    velocities = rng.normal(0.0, math.sqrt(0.00831446261815324 * TEMPERATURE / MASS), (n, 3))
    x = on.wrap(positions, cell)
    first, second, _ = on.pairs(x, cell, CUTOFF)
    forces = forces_of(x, first, second)
    start = time.perf_counter()
    for _ in range(steps):
        velocities += 0.5 * TIMESTEP * forces / MASS
        x = on.wrap(x + TIMESTEP * velocities, cell)
        first, second, _ = on.pairs(x, cell, CUTOFF)
        forces = forces_of(x, first, second)
        velocities += 0.5 * TIMESTEP * forces / MASS
    elapsed = time.perf_counter() - start
    pool.shutdown()
    return {
        "value": n * steps / elapsed,
        "unit": "atom-steps/s",
        "cores": threads,
        "kind": "port",
        "sample": f"{steps} NVE steps of a {cells}^3-cell FCC block ({n} atoms, same density) "
                  f"by the oracle port (C neighbor restatement on 1 thread + float64 numpy "
                  f"LJ on {threads} threads / Verlet)",
        "seconds": elapsed,
    }


REFERENCE_TREE = ROOT / "baseline" / "_ref"


def reference_cpu_rate(steps: int = 3, cells: int = 24, threads: int | None = None) -> dict:
    """The reference's own CPU path (installed in baseline/_ref): per step its
    quantity.energy_force_virial of its LennardJones on CPU float32 tensors (torch.func, with
    ``threads`` host threads, all of them by default), the two half kicks and the drift with its
    space.wrap. The reference builds pairs only on CUDA, so the pairs come from the oracle's C
    restatement of its operator, once per sample at the list radius (untimed; the atoms move
    well under half the skin in these steps).

    Sample: a cells^3-cell FCC block of the workload's density (4 cells^3 atoms).
    """
    import torch

    if str(REFERENCE_TREE) not in sys.path:
        sys.path.insert(0, str(REFERENCE_TREE))
    from nabladyn import potential, quantity, space  # the reference package
    from nabladyn.neighbors import NeighborPairs

    from nabladyn_b200 import lattice
    from oracle import neighbors as on

    threads = threads or os.cpu_count() or 1
    previous = torch.get_num_threads()
    torch.set_num_threads(threads)
    length = LENGTH * cells / ATOMS_PER_SIDE_CELLS
    positions, cell = lattice.fcc(cells, length, 0.02, seed=1)
    n = positions.shape[0]
    box = torch.tensor(cell, dtype=torch.float32)
    x, _ = space.wrap(torch.tensor(positions, dtype=torch.float32), box)
    first, second, _ = on.pairs(x.numpy(), box.numpy(), CUTOFF + SKIN)
    pairs = NeighborPairs(torch.tensor(np.stack([first, second]), dtype=torch.int64), n, CUTOFF)
    model = potential.lennard_jones(atom_types=torch.zeros(n, dtype=torch.int64),
                                    sigma=torch.tensor([SIGMA]), epsilon=torch.tensor([EPSILON]),
                                    cutoff=CUTOFF)
    evaluate = quantity.energy_force_virial(model)
    generator = torch.Generator().manual_seed(1)
    v = torch.randn((n, 3), generator=generator) * math.sqrt(0.00831446261815324 * TEMPERATURE / MASS)
    _, f, _ = evaluate(x, box, pairs)
    start = time.perf_counter()
    for _ in range(steps):
        v = v + (0.5 * TIMESTEP / MASS) * f
        x, _ = space.wrap(x + TIMESTEP * v, box)
        _, f, _ = evaluate(x, box, pairs)
        v = v + (0.5 * TIMESTEP / MASS) * f
    elapsed = time.perf_counter() - start
    torch.set_num_threads(previous)
    return {
        "value": n * steps / elapsed,
        "unit": "atom-steps/s",
        "cores": threads,
        "kind": "reference",
        "sample": f"{steps} NVE steps of a {cells}^3-cell FCC block ({n} atoms, same density): "
                  f"the reference's quantity.energy_force_virial (torch.func, float32, "
                  f"{threads} threads) + velocity Verlet on CPU tensors; pairs from the oracle's "
                  f"C restatement of its operator, untimed",
        "seconds": elapsed,
    }


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = max(1, args.steps)
    # Each bench step is one CPU step of the sample; warm-up steps run untimed. The reference's
    # own torch CPU path when baseline/_ref holds it, else the oracle port.
    rate = reference_cpu_rate if (REFERENCE_TREE / "nabladyn").exists() else cpu_port_rate
    rate(steps=max(1, min(args.warmup, 3)), cells=12)
    baseline = rate(steps=min(steps, 5), cells=24)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": baseline["value"],
        "unit": "atom-steps/s",
        "n_gpus": args.gpus,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * baseline["seconds"] / min(steps, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if baseline["kind"] == "reference" else "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": baseline["sample"]},
        "cpu_baseline": baseline,
        "e2e": {"value": baseline["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def serve_requests(device, ranks, requests: int, rate: float | None, seed: int = 7,
                   stage_ahead: int = 32, budget_gb: float = 16.0) -> dict:
    """``requests`` independent argon NVT replicas (64-16,384 atoms, 500 steps each) through
    the replica server (a pool of ``budget_gb`` GiB), Poisson arrivals at ``rate`` per second
    (None: all at t = 0). With N ranks each serves its share (replicas.shard_requests by
    atom-steps) on its own GPU with no collective on the data path; the wall time is the
    slowest rank's, the latencies are gathered from every rank for p50/p99."""
    import torch

    from nabladyn_b200.replicas import shard_requests
    from nabladyn_b200.serving import ReplicaServer, serving_requests

    work = serving_requests(requests, seed=seed, rate=rate)
    mine = shard_requests([r.steps * r.positions.shape[0] for r in work], ranks.world)[ranks.rank]
    server = ReplicaServer(device=device, budget_bytes=int(budget_gb * (1 << 30)), max_slots=2048,
                           stage_ahead=stage_ahead)
    server.serve(serving_requests(8, seed=99, steps=20), realtime=False)  # warm-up
    torch.cuda.synchronize(device)
    ranks.barrier()
    start = time.perf_counter()
    results = server.serve([work[k] for k in mine], realtime=rate is not None)
    wall = ranks.max(time.perf_counter() - start)
    rows = ranks.gather([(r.latency, r.steps, r.steps * r.num_atoms, int(r.status != 0))
                         for r in results])
    latencies = np.array([row[0] for row in rows])
    replica_steps = sum(row[1] for row in rows)
    atom_steps = sum(row[2] for row in rows)
    peaks = load_peaks()
    achieved = atom_steps / wall * STEP_BYTES_PER_ATOM / 1e9
    return {
        "workload": f"{requests} LJ argon NVT replicas, N log-uniform 64-16384, 500 steps, fp32, "
                    f"arrivals {'Poisson ' + str(rate) + '/s' if rate else 'all at t=0'}, "
                    f"{ranks.world} GPU(s)",
        "replica_steps_per_s": replica_steps / wall,
        "atom_steps_per_s": atom_steps / wall,
        "wall_s": wall,
        "latency_p50_s": float(np.percentile(latencies, 50)),
        "latency_p99_s": float(np.percentile(latencies, 99)),
        "failed": sum(row[3] for row in rows),
        "stage_ahead": stage_ahead,
        # The step's algorithmic bytes per atom-step (as the headline's step roofline) at the
        # served atom-step rate, against the measured HBM copy bandwidth.
        "roofline": {"bound": "hbm", "bytes_per_atom_step": STEP_BYTES_PER_ATOM,
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"]},
    }


def plain_requests(device, requests: int, sample: int, seed: int = 7) -> dict:
    """The plain path for the serving workload: a seeded sample of the same requests one at a
    time through md.nvt; with setup (model, simulation, capture) and run only."""
    import torch

    from nabladyn_b200 import md, potential
    from nabladyn_b200.serving import serving_requests

    work = serving_requests(requests, seed=seed)
    picked = np.random.default_rng(1).choice(len(work), sample, replace=False)
    total = run = 0.0
    steps = 0
    for request in (work[k] for k in picked):
        t0 = time.perf_counter()
        n = request.positions.shape[0]
        model = potential.lennard_jones(
            atom_types=torch.zeros(n, dtype=torch.int64, device=device),
            sigma=torch.tensor([request.sigma], device=device),
            epsilon=torch.tensor([request.epsilon], device=device), cutoff=request.cutoff)
        simulation = md.nvt(
            model, torch.tensor(request.positions, dtype=torch.float32, device=device),
            torch.tensor(request.velocities, dtype=torch.float32, device=device),
            torch.tensor(request.masses, dtype=torch.float32, device=device),
            torch.tensor(request.cell, dtype=torch.float32, device=device),
            timestep=request.timestep, temperature=request.temperature,
            thermostat_timescale=request.thermostat_timescale, skin=request.skin)
        torch.cuda.synchronize(device)
        t1 = time.perf_counter()
        simulation.run(request.steps)
        simulation.state()
        torch.cuda.synchronize(device)
        t2 = time.perf_counter()
        total += t2 - t0
        run += t2 - t1
        steps += request.steps
    return {"sample": sample, "replica_steps_per_s_with_setup": steps / total,
            "replica_steps_per_s_run_only": steps / run}


def run_serving(device, ranks, requests: int, plain_sample: int,
                rates: tuple[float | None, ...], stage_ahead: int = 32,
                budget_gb: float = 16.0) -> dict:
    """The serving workload at each arrival rate, against the plain path (rank 0 only)."""
    legs = {f"rate_{rate if rate else 'all_at_t0'}": serve_requests(device, ranks, requests, rate,
                                                                    stage_ahead=stage_ahead,
                                                                    budget_gb=budget_gb)
            for rate in rates}
    out = {"legs": legs}
    if ranks.rank == 0 and plain_sample:
        plain = plain_requests(device, requests, plain_sample)
        out["plain"] = plain
        out["vs_plain"] = {
            name: {"with_setup": leg["replica_steps_per_s"] / plain["replica_steps_per_s_with_setup"],
                   "run_only": leg["replica_steps_per_s"] / plain["replica_steps_per_s_run_only"]}
            for name, leg in legs.items()}
    return out


def small_system(module, device, dtype):
    """The plain small workload: 512 argon atoms on an 8^3 simple-cubic lattice in L = 2.90 nm
    with 0.02 nm seeded jitter, 120 K Maxwell-Boltzmann velocities; built with ``module``
    (this package or the reference), returns its NVT simulation."""
    import torch

    from nabladyn_b200 import lattice

    positions, cell = lattice.simple_cubic(8, 2.90, 0.02, seed=512)
    n = positions.shape[0]
    model = module.potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=device),
        sigma=torch.tensor([SIGMA], dtype=dtype, device=device),
        epsilon=torch.tensor([EPSILON], dtype=dtype, device=device), cutoff=CUTOFF)
    masses = torch.full((n,), MASS, dtype=dtype, device=device)
    velocities = module.md.maxwell_boltzmann(masses, TEMPERATURE, seed=512)
    return module.md.nvt(model, torch.tensor(positions, dtype=dtype, device=device), velocities,
                         masses, torch.tensor(cell, dtype=dtype, device=device),
                         timestep=TIMESTEP, temperature=TEMPERATURE, thermostat_timescale=0.1)


def run_small(module, device, steps: int, label: str) -> dict:
    """2,500 NVT steps (fp32) of the 512-atom system, timed by CUDA events after warm-up."""
    import torch

    simulation = small_system(module, device, torch.float32)
    simulation.run(100)
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    simulation.run(steps)
    end.record()
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(end)
    return {"impl": label, "workload": "512-atom argon NVT, fp32, dt 4 fs, NHC(3) at 120 K",
            "steps": steps, "us_per_step": 1e3 * ms / steps, "steps_per_s": steps / (ms / 1e3),
            "ns_per_day": steps / (ms / 1e3) * 0.004 * 86400 / 1000}


BEAD_MASS = 32.04  # the bead workload's mass: methanol, Da


def schnet_system(module, device, dtype):
    """The SchNet bead workload: 32,768 coarse-grained beads on a 32^3 simple-cubic lattice at
    10 per nm^3 (L = 14.86 nm) with 0.02 nm seeded jitter; SchNet of 64 features, 3 blocks,
    50 Gaussians, cutoff 1.2 nm, seed 0, one bead type; 300 K Maxwell-Boltzmann velocities.
    Built with ``module`` (this package or the reference); returns its NVT simulation
    (dt 0.01 ps, tau 0.1 ps, skin 0.1 nm) and the model."""
    import torch

    from nabladyn_b200 import lattice

    n_side = 32
    n = n_side**3
    length = (n / 10.0) ** (1.0 / 3.0)
    positions, cell = lattice.simple_cubic(n_side, length, 0.02, seed=n)
    model = module.potential.schnet(atom_types=torch.zeros(n, dtype=torch.int64, device=device),
                                    num_types=1, cutoff=1.2, dtype=dtype)
    masses = torch.full((n,), BEAD_MASS, dtype=dtype, device=device)
    velocities = module.md.maxwell_boltzmann(masses, 300.0, seed=n)
    simulation = module.md.nvt(model, torch.tensor(positions % cell, dtype=dtype, device=device),
                               velocities, masses, torch.tensor(cell, dtype=dtype, device=device),
                               timestep=0.01, temperature=300.0, thermostat_timescale=0.1,
                               skin=SKIN)
    return simulation, model


SCHNET_WORKLOAD = ("SchNet beads NVT, 32,768 beads (32^3 lattice, 10/nm^3), F=64, 3 blocks, "
                   "K=50, r_c 1.2 nm, dt 0.01 ps, 300 K, fp32 (BF16 tensor-core filters)")
# Algorithmic tensor-core work per pair within the cutoff and step: per block the filter
# network forward (50x64 + 64x64) and its reverse for the forces (64x64 + 64x50), 2 flop per
# multiply-add: 3 * 2 * 2 * (50 * 64 + 64 * 64) = 87,552 flop.
SCHNET_FLOP_PER_PAIR = 3 * 2 * 2 * (50 * 64 + 64 * 64)


def run_schnet(module, device, steps: int, warmup: int, label: str) -> dict:
    """``steps`` NVT steps of the bead workload after ``warmup``, timed by CUDA events; then
    the force error of the last frame against a float64 evaluation of the same network."""
    import torch

    simulation, model = schnet_system(module, device, torch.float32)
    simulation.run(max(3, warmup))
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    simulation.run(steps)
    end.record()
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(end)
    n = model.num_atoms
    out = {"impl": label, "workload": SCHNET_WORKLOAD, "steps": steps,
           "ms_per_step": ms / steps, "steps_per_s": steps / (ms / 1e3),
           "atom_steps_per_s": n * steps / (ms / 1e3)}
    state = simulation.state()
    exact = module.potential.schnet(atom_types=model.atom_types, num_types=1, cutoff=1.2,
                                    dtype=torch.float64)
    listing = module.neighbors.NeighborList(1.2, skin=SKIN)
    x64, cell64 = state.positions.double(), state.cell.double()
    listing.allocate(x64, cell64)
    pairs = listing.tensors()
    if pairs.index.dtype != torch.int64 and module.__name__ == "nabladyn":
        pairs = pairs._replace(index=pairs.index.long())
    _, f64, _ = module.quantity.energy_force_virial(exact)(x64, cell64, pairs)
    ours = state.forces.double()
    out["force_error_vs_fp64"] = float((ours - f64).norm() / f64.norm())
    out["temperature_K"] = float(simulation.sample()["temperature"])
    if label == "ours":
        engine = simulation._engine
        pairs_in_cutoff = int(engine.tensors["model_status"][0])
        flop = SCHNET_FLOP_PER_PAIR * pairs_in_cutoff
        peaks = load_peaks()
        achieved = flop / (ms / steps / 1e3) / 1e12
        out["pairs_within_cutoff"] = pairs_in_cutoff
        out["roofline"] = {"bound": "tensor", "achieved": achieved,
                           "peak": peaks["bf16_tflops_sustained"], "unit": "TFLOP/s",
                           "frac": achieved / peaks["bf16_tflops_sustained"],
                           "flop_per_step": flop, "peak_source": peaks["source"]}
    return out


GRADIENT_WORKLOAD = ("LJ parameter gradient: 2-type mixture, 4,096 atoms (16^3 lattice, "
                     "21/nm^3), 64 frames, loss over E/F/W in fp32, dLoss/d(sigma, epsilon)")


def gradient_data(device):
    """The differentiation workload: 64 jittered frames of a 16^3 simple-cubic lattice at 21 per
    nm^3 (L = 5.80 nm), types 50/50 seeded, labels from sigma rows (0.34, 0.32, 0.30) and
    epsilon rows (0.996, 0.8, 0.6) in float64, start parameters off by a seeded +-10%."""
    import numpy as np
    import torch

    from nabladyn_b200 import lattice, potential, training

    n_side, frames = 16, 64
    n = n_side**3
    length = (n / 21.0) ** (1.0 / 3.0)
    rng = np.random.default_rng(n)
    types = torch.tensor(rng.permutation(np.arange(n) % 2), device=device)
    positions = np.stack([lattice.simple_cubic(n_side, length, 0.02, seed=100 + f)[0] % length
                          for f in range(frames)])
    x = torch.tensor(positions, device=device)
    cells = torch.full((frames, 3), length, dtype=torch.float64, device=device)
    stack = training.pair_stack(x, cells, CUTOFF)
    sigma = torch.tensor([0.34, 0.32, 0.30], dtype=torch.float64, device=device)
    epsilon = torch.tensor([0.996, 0.8, 0.6], dtype=torch.float64, device=device)
    target = potential.lennard_jones(atom_types=types, sigma=sigma, epsilon=epsilon,
                                     cutoff=CUTOFF)
    with torch.no_grad():
        labels = training.predict(target, {}, x, cells, (stack,), ("energy", "forces", "virial"))
    start = torch.tensor(rng.uniform(0.9, 1.1, 6), device=device)
    return {"types": types, "positions": x.float(), "cells": cells.float(), "stack": stack,
            "labels": {k: v.float() for k, v in labels.items()},
            "sigma": (sigma * start[:3]).float(), "epsilon": (epsilon * start[3:]).float()}


def run_gradient(module, device, steps: int, warmup: int, label: str) -> dict:
    """``steps`` evaluations of the loss and dLoss/d(sigma, epsilon) over all 64 frames, after
    ``warmup``, timed by CUDA events: this package's hand-written backward, or the
    reference's compiled gradient_program (torch.func double backward under Inductor)."""
    import torch

    data = gradient_data(device)
    channels = ("energy", "forces", "virial")
    model = module.potential.lennard_jones(
        atom_types=data["types"], sigma=data["sigma"], epsilon=data["epsilon"], cutoff=CUTOFF,
        trainable=("sigma", "epsilon"))
    from nabladyn_b200 import training

    scales = training.scales(**data["labels"])
    weights = {"energy": 1.0, "forces": 1.0, "virial": 1.0}
    if label == "ours":
        def evaluate():
            params = {"sigma": model.sigma.detach().clone().requires_grad_(True),
                      "epsilon": model.epsilon.detach().clone().requires_grad_(True)}
            predicted = module.training.predict(model, params, data["positions"], data["cells"],
                                                (data["stack"],), channels)
            value, _ = module.training.loss(predicted, data["labels"], weights, scales)
            value.backward()
            return value, params["sigma"].grad
    else:
        from nabladyn.training import _fit

        program = _fit.gradient_program(model, channels)
        tensor = lambda v: torch.tensor(v, dtype=torch.float32, device=device)  # noqa: E731
        t_weights = {k: tensor(v) for k, v in weights.items()}
        t_scales = {k: tensor(v) for k, v in scales.items()}

        def evaluate():
            params = {"sigma": model.sigma.detach(), "epsilon": model.epsilon.detach()}
            gradient, (value, _) = program(params, data["positions"], data["cells"],
                                           (data["stack"],), data["labels"], None, t_weights,
                                           t_scales)
            return value, gradient["sigma"]

    for _ in range(max(3, warmup)):
        value, grad = evaluate()
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        value, grad = evaluate()
    end.record()
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(end) / steps
    # The float64 gradient of the same loss, by this package's backward (which matches the
    # reference's float64 gradient to 1e-9), as the accuracy yardstick of both arms.
    exact = training_gradient64(data, channels, weights, scales)
    error = float((grad.double() - exact).norm() / exact.norm())
    return {"impl": label, "workload": GRADIENT_WORKLOAD, "evaluations": steps,
            "ms_per_gradient": ms, "frames_per_s": 64 / (ms / 1e3),
            "loss": float(value), "dloss_dsigma": grad.tolist(),
            "dloss_dsigma_error_vs_fp64": error,
            "pairs_columns": int(data["stack"].shape[2])}


def training_gradient64(data, channels, weights, scales):
    """dLoss/dsigma of the differentiation workload in float64."""
    import nabladyn_b200

    model = nabladyn_b200.potential.lennard_jones(
        atom_types=data["types"], sigma=data["sigma"].double(),
        epsilon=data["epsilon"].double(), cutoff=CUTOFF, trainable=("sigma", "epsilon"))
    params = {"sigma": model.sigma.detach().clone().requires_grad_(True),
              "epsilon": model.epsilon.detach().clone().requires_grad_(True)}
    predicted = nabladyn_b200.training.predict(model, params, data["positions"].double(),
                                               data["cells"].double(), (data["stack"],),
                                               channels)
    labels = {k: v.double() for k, v in data["labels"].items()}
    value, _ = nabladyn_b200.training.loss(predicted, labels, weights, scales)
    value.backward()
    return params["sigma"].grad


TRAIN_WORKLOAD = ("SchNet training step: 32 frames of the 32,768-bead system, loss over E/F/W "
                  "(labels from the seed-1 network), gradient in every parameter, fp32")


def run_schnet_training(module, device, steps: int, warmup: int, label: str) -> dict:
    """``steps`` training steps (loss and gradient over 32 frames) after ``warmup``. Here the
    fused kernels with the written-out second-order pass (tcgen05 tangent kernels for the pair
    terms), frame by frame; there the reference's algorithm (torch.func double backward through
    the model, vmapped over chunks of 2 frames) under its Inductor compile."""
    import numpy as np
    import torch

    import nabladyn_b200
    from nabladyn_b200 import lattice, training

    n_side, frames, chunk = 32, 32, 2
    n = n_side**3
    length = (n / 10.0) ** (1.0 / 3.0)
    positions = torch.tensor(np.stack([
        lattice.simple_cubic(n_side, length, 0.03, seed=500 + f)[0] % length
        for f in range(frames)]), dtype=torch.float32, device=device)
    cells = torch.full((frames, 3), length, dtype=torch.float32, device=device)
    stack = training.pair_stack(positions, cells, 1.2)
    types = torch.zeros(n, dtype=torch.int64, device=device)
    teacher = nabladyn_b200.potential.schnet(atom_types=types, num_types=1, cutoff=1.2, seed=1)
    labels = {"energy": [], "forces": [], "virial": []}
    for f in range(frames):
        pairs = nabladyn_b200.neighbors.NeighborPairs(stack[f], n, 1.2)
        e, force, w = nabladyn_b200.quantity.energy_force_virial(teacher)(positions[f], cells[f],
                                                                         pairs)
        labels["energy"].append(e)
        labels["forces"].append(force)
        labels["virial"].append(w)
    labels = {k: torch.stack(v) for k, v in labels.items()}
    scales = training.scales(**labels)
    weights = {"energy": 1.0, "forces": 1.0, "virial": 1.0}
    model = module.potential.schnet(atom_types=types, num_types=1, cutoff=1.2, trainable=True)
    params = {k: v.detach().clone() for k, v in model.named_parameters()}
    if label == "ours":
        def evaluate():
            return training.loss_and_gradient(model, params, positions, cells, (stack,), labels,
                                              weights, scales, chunk=chunk)
    else:
        from nabladyn.training import _fit

        program = _fit.gradient_program(model, ("energy", "forces", "virial"))
        as_tensor = lambda v: torch.tensor(v, dtype=torch.float32, device=device)  # noqa: E731
        t_weights = {k: as_tensor(v) for k, v in weights.items()}
        t_scales = {k: as_tensor(v) for k, v in scales.items()}
        long_stack = stack.long()

        def evaluate():
            total, gradient = 0.0, None
            for begin in range(0, frames, chunk):
                end = begin + chunk
                part = {k: v[begin:end] for k, v in labels.items()}
                coefficients = torch.full((end - begin,), 1.0 / frames, device=device)
                grads, (value, _) = program(params, positions[begin:end], cells[begin:end],
                                            (long_stack[begin:end],), part, coefficients,
                                            t_weights, t_scales)
                total = total + value
                gradient = grads if gradient is None else {
                    k: gradient[k] + grads[k] for k in grads}
            return total, gradient

    for _ in range(max(1, warmup)):
        value, gradient = evaluate()
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        value, gradient = evaluate()
    end.record()
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(end) / steps
    norm = float(torch.sqrt(sum(g.double().square().sum() for g in gradient.values())))
    return {"impl": label, "workload": TRAIN_WORKLOAD, "steps": steps,
            "ms_per_training_step": ms, "loss": float(value), "gradient_norm": norm,
            "peak_memory_gb": torch.cuda.max_memory_allocated(device) / 1e9}


def run_reference_cuda(args) -> None:
    """The reference's own GPU path on this B200: its md.nve (Inductor programs around its
    CUDA neighbor operator, one CUDA Graph per step), installed in baseline/_ref. Not a driver
    arm: it prints the reference's atom-steps/s for the same workload, for comparison."""
    import torch

    sys.path.insert(0, str(ROOT / "baseline" / "_ref"))
    from nabladyn import md, potential  # the reference package

    from nabladyn_b200 import lattice

    device = torch.device("cuda", 0)
    if args.workload == "neighbors":
        import nabladyn

        print(json.dumps(run_neighbors(nabladyn, device, args.steps, args.warmup,
                                       "reference-cuda")), flush=True)
        return
    if args.workload == "small":
        import nabladyn

        print(json.dumps(run_small(nabladyn, device, args.steps, "reference-cuda")), flush=True)
        return
    if args.workload == "schnet-train":
        import nabladyn

        try:
            result = run_schnet_training(nabladyn, device, args.steps, args.warmup,
                                         "reference-cuda")
        except Exception as error:  # the reference's own failure, reported as its line
            result = {"impl": "reference-cuda", "workload": TRAIN_WORKLOAD,
                      "unavailable": f"{type(error).__name__}: {str(error).splitlines()[0]}"}
        print(json.dumps(result), flush=True)
        return
    if args.workload == "gradient":
        import nabladyn

        try:
            result = run_gradient(nabladyn, device, args.steps, args.warmup, "reference-cuda")
        except Exception as error:  # the reference's own failure, reported as its line
            result = {"impl": "reference-cuda", "workload": GRADIENT_WORKLOAD,
                      "unavailable": f"{type(error).__name__}: {str(error).splitlines()[0]}"}
        print(json.dumps(result), flush=True)
        return
    if args.workload == "schnet":
        import nabladyn

        try:
            result = run_schnet(nabladyn, device, args.steps, args.warmup, "reference-cuda")
        except Exception as error:  # the reference's own failure, reported as its line
            result = {"impl": "reference-cuda", "workload": SCHNET_WORKLOAD,
                      "unavailable": f"{type(error).__name__}: {str(error).splitlines()[0]}"}
        print(json.dumps(result), flush=True)
        return
    positions, cell = lattice.fcc(ATOMS_PER_SIDE_CELLS, LENGTH, 0.02, 2024)
    n = positions.shape[0]
    dtype = torch.float32
    model = potential.lennard_jones(
        atom_types=torch.zeros(n, dtype=torch.int64, device=device),
        sigma=torch.tensor([SIGMA], dtype=dtype, device=device),
        epsilon=torch.tensor([EPSILON], dtype=dtype, device=device),
        cutoff=CUTOFF,
    )
    masses = torch.full((n,), MASS, dtype=dtype, device=device)
    velocities = md.maxwell_boltzmann(masses, TEMPERATURE, seed=2024)
    setup = time.perf_counter()
    simulation = md.nve(model, torch.tensor(positions, dtype=dtype, device=device), velocities,
                        masses, torch.tensor(cell, dtype=dtype, device=device),
                        timestep=TIMESTEP, skin=SKIN)
    setup = time.perf_counter() - setup
    simulation.run(max(3, args.warmup))
    torch.cuda.synchronize(device)
    rebuilds = simulation._neighbors._rebuild_count
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    simulation.run(args.steps)
    end.record()
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(end)
    print(json.dumps({
        "impl": "reference-cuda",
        "metric": METRIC,
        "value": n * args.steps / (ms / 1e3),
        "unit": "atom-steps/s",
        "ms_per_step": ms / args.steps,
        "steps": args.steps,
        "setup_s": setup,
        "rebuilds_in_timed_steps": simulation._neighbors._rebuild_count - rebuilds,
        "pair_capacity": simulation._neighbors.pair_capacity,
        "config": {"workload": WORKLOAD},
    }), flush=True)


NEIGHBOR_SYSTEMS = {
    "lj_1m": "1,048,576 LJ atoms (64^3-cell FCC, L=36.77 nm), cutoff 1.0 nm, skin 0.1 nm, fp32",
    "beads_32k": "32,768 beads (32^3 lattice, 10/nm^3, L=14.86 nm), cutoff 1.2 nm, skin 0.1 nm, fp32",
}


def neighbor_frames(name: str):
    """Positions (wrapped), cell, cutoff and skin of a neighbor-operator workload."""
    from nabladyn_b200 import lattice

    if name == "lj_1m":
        positions, cell = lattice.fcc(ATOMS_PER_SIDE_CELLS, LENGTH, 0.02, 2024)
        return positions % cell, cell, CUTOFF, SKIN
    n_side = 32
    length = (n_side**3 / 10.0) ** (1.0 / 3.0)
    positions, cell = lattice.simple_cubic(n_side, length, 0.02, seed=n_side**3)
    return positions % cell, cell, 1.2, SKIN


def run_neighbors(module, device, steps: int, warmup: int, label: str) -> dict:
    """The neighbor operator alone through ``module``'s NeighborList (this package's, or the
    reference's own from baseline/_ref): per system, the first build (allocate), then
    ``steps`` forced rebuilds of the same frame and ``steps`` updates that reuse the pairs,
    each timed by CUDA events after ``warmup``."""
    import torch

    out = {"impl": label, "workload": "neighbor operator: rebuild and reuse", "systems": {}}
    for name, description in NEIGHBOR_SYSTEMS.items():
        positions, cell, cutoff, skin = neighbor_frames(name)
        x = torch.tensor(positions, dtype=torch.float32, device=device)
        box = torch.tensor(cell, dtype=torch.float32, device=device)
        listing = module.neighbors.NeighborList(cutoff, skin=skin)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        listing.allocate(x, box)
        torch.cuda.synchronize(device)
        allocate_s = time.perf_counter() - t0
        events = []
        for mode in ("rebuild", "reuse"):
            step = listing._rebuild_wrapped if mode == "rebuild" else listing._update_wrapped
            for _ in range(max(1, warmup)):
                step(x, box)
            torch.cuda.synchronize(device)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            for _ in range(steps):
                step(x, box)
            end.record()
            torch.cuda.synchronize(device)
            events.append(start.elapsed_time(end) / steps)
        out["systems"][name] = {
            "system": description, "atoms": int(x.shape[0]), "pairs": listing.num_pairs,
            "rebuilds_counted": listing._rebuild_count, "allocate_s": allocate_s,
            "ms_per_rebuild": events[0], "ms_per_reuse_update": events[1],
        }
        del listing
        torch.cuda.empty_cache()
    return out


# Serving legs of the default line: arrivals over-subscribing the server (about three times
# what it completes) and a moderate rate, both Poisson.
SERVING_RATES = (2000.0, 400.0)


def spawn_reference_cuda(args) -> dict | None:
    """The reference's own CUDA path on this GPU for the same workload, seeds, steps and
    warm-up (bench.py --impl reference-cuda, in a process of its own: it registers the same
    operator namespace); None when baseline/_ref holds no reference build."""
    if not any((REFERENCE_TREE / "nabladyn" / "neighbors").glob("_C*.so")):
        return None
    command = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference-cuda",
               "--steps", str(args.steps), "--warmup", str(args.warmup)]
    try:
        done = subprocess.run(command, capture_output=True, text=True, timeout=900, check=True)
        return json.loads(done.stdout.strip().splitlines()[-1])
    except (subprocess.SubprocessError, ValueError, IndexError) as error:
        return {"unavailable": f"{type(error).__name__}: {str(error).splitlines()[0][:200]}"}


def run_ours(args) -> None:
    import torch

    from nabladyn_b200.replicas import Ranks

    local = int(os.environ.get("LOCAL_RANK", "0"))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    ranks = Ranks("nccl", device, timeout_s=300)
    world, rank = ranks.world, ranks.rank
    barrier, max_over_ranks = ranks.barrier, ranks.max

    simulation, host, n = build_system(torch, device, seed=2024 + rank)
    engine = simulation._engine
    stream = torch.cuda.current_stream(device)
    simulation.run(max(3, args.warmup))
    torch.cuda.synchronize(device)

    # value: K steps replayed from the captured graphs, timed by CUDA events.
    rebuilds_before = simulation._rebuild_count
    barrier()
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        simulation.run(args.steps)
        end.record(stream)
        torch.cuda.synchronize(device)
    barrier()
    elapsed_ms = max_over_ranks(start.elapsed_time(end))
    rebuilds = simulation._rebuild_count - rebuilds_before
    value = world * n * args.steps / (elapsed_ms / 1e3)
    accuracy = frame_accuracy(simulation)

    # Roofline of the dominant kernel: the same steps run eagerly, each phase between events.
    phases = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    for events in phases:
        events[0].record(stream)
        for phase in range(3):
            engine.step_phase(phase, False)
            events[phase + 1].record(stream)
    torch.cuda.synchronize(device)
    phase_ms = [sum(e[p].elapsed_time(e[p + 1]) for e in phases) / args.steps for p in range(3)]
    peaks = load_peaks()
    force_bytes = FORCE_BYTES_PER_ATOM * n
    achieved = force_bytes / (phase_ms[2] / 1e3) / 1e9
    step_roof_s = STEP_BYTES_PER_ATOM / (peaks["hbm_gbs"] * 1e9)
    # dram__bytes_read.sum + dram__bytes_write.sum of one launch of this force kernel (the
    # pair-list step kernel) at this workload, measured by ncu on a B200; see the constant.
    traffic = FORCE_KERNEL_DRAM_BYTES if n == 1_048_576 else None

    # e2e: the public API with host buffers: per call, the frame from pinned host memory,
    # set_frame, run(chunk), state(), and the frame back into pinned host memory.
    chunk = 100
    calls = max(1, args.steps // chunk)
    back = {name: torch.empty((n, 3), dtype=torch.float32).pin_memory()
            for name in ("positions", "velocities", "forces")}
    back_images = torch.empty((n, 3), dtype=torch.int64).pin_memory()
    staged = {name: torch.empty((n, 3), dtype=torch.float32, device=device)
              for name in ("positions", "velocities")}
    barrier()
    torch.cuda.synchronize(device)
    e2e_start, e2e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_start.record(stream)
    for _ in range(calls):
        staged["positions"].copy_(host["positions"], non_blocking=True)
        staged["velocities"].copy_(host["velocities"], non_blocking=True)
        simulation.set_frame(staged["positions"], staged["velocities"])
        simulation.run(chunk)
        state = simulation.state()
        back["positions"].copy_(state.positions, non_blocking=True)
        back["velocities"].copy_(state.velocities, non_blocking=True)
        back["forces"].copy_(state.forces, non_blocking=True)
        back_images.copy_(state.images, non_blocking=True)
    e2e_end.record(stream)
    torch.cuda.synchronize(device)
    e2e_ms = max_over_ranks(e2e_start.elapsed_time(e2e_end))
    e2e_value = world * n * chunk * calls / (e2e_ms / 1e3)
    h2d = 2 * n * 3 * 4 / chunk
    d2h = (3 * n * 3 * 4 + n * 3 * 8) / chunk

    cpu = port = reference_cuda = None
    if rank == 0 and world == 1:
        port = cpu_port_rate()
        cpu = reference_cpu_rate() if (REFERENCE_TREE / "nabladyn").exists() else port
        reference_cuda = spawn_reference_cuda(args) if args.reference_cuda == "auto" else None
    serving = None
    if args.serving:
        serving = run_serving(device, ranks, args.serving, plain_sample=16 if rank == 0 else 0,
                              rates=SERVING_RATES)
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "atom-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": WORKLOAD,
                "atoms_per_replica": n,
                "ensemble": "NVE",
                "timestep_ps": TIMESTEP,
                "skin_nm": SKIN,
                "parallelism": f"replicas x{world}",
                "l2": "working set > L2 (126 MB); no flush",
                "rebuilds_in_timed_steps": rebuilds,
            },
            "accuracy": accuracy,
            "roofline": {
                "kernel": "force_kernel (forces, second half kick, float64 tail)",
                "bound": "hbm",
                "limiter": FORCE_KERNEL_LIMITER,
                "achieved": achieved,
                "peak": peaks["hbm_gbs"],
                "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"],
                "peak_source": peaks["source"],
                "traffic": traffic,
                "algorithmic_bytes_per_launch": force_bytes,
                "avg_launch_ms": phase_ms[2],
            },
            "phases_ms": {"drift": phase_ms[0], "rebuild_gated": phase_ms[1],
                          "forces": phase_ms[2]},
            "step_roofline": {
                "bytes_per_atom_step": STEP_BYTES_PER_ATOM,
                "flops_per_atom_step": STEP_FLOPS_PER_ATOM,
                "t_roof_ps": step_roof_s * 1e12,
                "frac": (value / world) * step_roof_s,
            },
            "e2e": {"value": e2e_value, "unit": "atom-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps_per_call": chunk},
            # Per step the drift (which also sets the rebuild condition) and the forces; the
            # rebuild's kernels only in steps whose conditional node takes the rebuild.
            "gpu_launches": (2 * args.steps + rebuilds * (engine.step_launches - 2)
                             if not engine.small else engine.step_launches * args.steps),
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "cpu_port": port,
            "reference_cuda": reference_cuda,
            "vs_reference_cuda": (value / reference_cuda["value"]
                                  if reference_cuda and reference_cuda.get("value") else None),
            "e2e_vs_reference_cuda": (e2e_value / reference_cuda["value"]
                                      if reference_cuda and reference_cuda.get("value") else None),
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    ranks.close()


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=1000)
    parser.add_argument("--warmup", type=int, default=10)
    parser.add_argument("--impl", choices=("ours", "reference", "reference-cuda"), default="ours")
    parser.add_argument("--serving", type=int, default=4096,
                        help="requests of the serving workload (0 skips it)")
    parser.add_argument("--serving-rate", type=float, default=None,
                        help="with --workload serving: Poisson arrivals per second")
    parser.add_argument("--stage-ahead", type=int, default=32,
                        help="serving: arrived requests made ready on the host during a round")
    parser.add_argument("--serving-budget-gb", type=float, default=16.0,
                        help="serving: the replica pool's device memory, GiB")
    parser.add_argument("--reference-cuda", choices=("auto", "off"), default="auto",
                        help="auto: time the reference's CUDA path beside ours when installed")
    parser.add_argument("--workload",
                        choices=("large", "serving", "small", "schnet", "gradient",
                                 "schnet-train", "neighbors"),
                        default="large")
    args = parser.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "schnet-train" and args.impl == "ours":
        import torch

        import nabladyn_b200

        print(json.dumps(run_schnet_training(nabladyn_b200, torch.device("cuda", 0), args.steps,
                                             args.warmup, "ours")), flush=True)
        return
    if args.workload == "gradient" and args.impl == "ours":
        import torch

        import nabladyn_b200

        print(json.dumps(run_gradient(nabladyn_b200, torch.device("cuda", 0), args.steps,
                                      args.warmup, "ours")), flush=True)
        return
    if args.workload == "schnet" and args.impl == "ours":
        import torch

        import nabladyn_b200

        print(json.dumps(run_schnet(nabladyn_b200, torch.device("cuda", 0), args.steps,
                                    args.warmup, "ours")), flush=True)
        return
    if args.workload == "neighbors" and args.impl == "ours":
        import torch

        import nabladyn_b200

        result = run_neighbors(nabladyn_b200, torch.device("cuda", 0), args.steps, args.warmup,
                               "ours")
        if args.reference_cuda == "auto" and any(
                (REFERENCE_TREE / "nabladyn" / "neighbors").glob("_C*.so")):
            command = [sys.executable, str(ROOT / "bench.py"), "--workload", "neighbors",
                       "--impl", "reference-cuda", "--steps", str(args.steps), "--warmup",
                       str(args.warmup)]
            done = subprocess.run(command, capture_output=True, text=True, timeout=900)
            lines = [l for l in done.stdout.splitlines() if l.startswith("{")]
            reference = json.loads(lines[-1]) if lines else {"unavailable": done.stderr[-300:]}
            result["reference_cuda"] = reference
            if "systems" in reference:
                result["rebuild_speedup"] = {
                    name: reference["systems"][name]["ms_per_rebuild"] / mine["ms_per_rebuild"]
                    for name, mine in result["systems"].items()}
        print(json.dumps(result), flush=True)
        return
    if args.workload == "small" and args.impl == "ours":
        import torch

        import nabladyn_b200

        print(json.dumps(run_small(nabladyn_b200, torch.device("cuda", 0), args.steps, "ours")),
              flush=True)
        return
    if args.workload == "serving":
        import torch

        from nabladyn_b200.replicas import Ranks

        device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(device)
        ranks = Ranks("nccl", device, timeout_s=300)
        rates = (args.serving_rate,) if args.serving_rate else SERVING_RATES
        result = run_serving(device, ranks, args.serving, plain_sample=16 if ranks.rank == 0 else 0,
                             rates=rates, stage_ahead=args.stage_ahead,
                             budget_gb=args.serving_budget_gb)
        if ranks.rank == 0:
            print(json.dumps(result), flush=True)
        ranks.close()
        return
    if args.impl == "reference":
        run_reference(args)
    elif args.impl == "reference-cuda":
        run_reference_cuda(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
