#!/usr/bin/env python
"""Lennard-Jones particle-steps/s on B200.

Workload (default): 256,000 atoms on an fcc lattice (40^3 unit cells x 4) at
rho = 0.8442, force-shifted cutoff 2.5, Langevin T = 1.0, gamma = 1.0, seed 7,
dt = 0.005, Verlet list with skin 0.3 rebuilt on the skin/2 trigger (cell grid
rebuilt with it), f32 pair forces, i64 fixed-point energy and virial, f64
integration. Synthetic seeded input, no dataset.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One timed step is one MD step of the whole box. Between timed steps a
256 MiB buffer is written on the same stream to flush the 126 MB L2, so every
step starts cold; each step is bracketed by CUDA events on the simulation's
stream and the per-step device times are summed. Under torchrun every rank
runs its own independent box (weak scaling, no collective on the step path);
the time is the max over ranks.

`e2e`: the same metric through the public API with host buffers: per bench
step, the particles are written from pinned host memory (vlj_write_particles),
100 MD steps run (vlj_run), and the measurement and the particles are read
back into pinned host memory (vlj_measure_now, vlj_read_particles); wall
clock, max over ranks.

`--impl reference`: the reference has no CPU Lennard-Jones code and its GPU
path needs a graphics API, so the reference arm is the CPU oracle's f64
cell-list engine (same model, integrator and workload) on all host cores,
rank 0 only.
"""

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "virial-engine_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "LJ particle-steps/s on 1 B200, batched vs plain, at <=1e-6 rel PE/virial vs f64"
UNIT = "particle-steps/s"
WORK = dict(cells=40, density=0.8442, temperature=1.0, friction=1.0, seed=7, dt=0.005,
            cutoff=2.5, skin=0.3, shifted_force=True)
E2E_INNER = 100          # MD steps per end-to-end bench step
L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0
ALGO_BYTES = 96          # f64 x and v read + written per particle-step


BATCH = dict(replicas=512, seed=2024, sizes=(500, 20000), densities=(0.01, 0.90),
             temperatures=(0.7, 2.0), friction=1.0, dt=0.004, cutoff=2.5, skin=0.3,
             skins=(0.3, 0.4, 0.5, 0.6, 0.8), threads=(64, 128, 256))
PLAIN_SAMPLE_EVERY = 16  # plain-path comparison: every 16th replica as its own simulation
PLAIN_SAMPLE_STEPS = 50


def config(n, world):
    return {
        "workload": "lj-fcc40x4-256k-rho0.8442-shifted-force-langevin-grid-on-list-trigger",
        "particles_per_box": n, "boxes": world, "density": WORK["density"],
        "cutoff": WORK["cutoff"], "cutoff_style": "force-shifted", "skin": WORK["skin"],
        "thermostat": "langevin T=1.0 gamma=1.0 seed=7", "dt": WORK["dt"],
        "l2": "flushed between timed steps (256 MiB write on the stream)",
        "grid": "cell grid rebuilt with the Verlet list on the skin/2 trigger (the "
                "reference's schedule); grid_every_step times the grid rebuilt on every step",
        "parallelism": f"replicas x{world}",
    }


def flops_per_particle_step(density, per_pair=26.0, cutoff=None, skin=None):
    """Algorithmic f32 flops: 11 per list candidate, 26 per force-shifted
    (20 per truncated-shifted) pair inside the cutoff (FMA = 2)."""
    import math
    rc = WORK["cutoff"] if cutoff is None else cutoff
    sk = WORK["skin"] if skin is None else skin
    n_list = 4.0 / 3.0 * math.pi * (rc + sk) ** 3 * density
    n_rc = 4.0 / 3.0 * math.pi * rc ** 3 * density
    return 11.0 * n_list + per_pair * n_rc


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profile_traffic():
    """dram bytes per launch of the step kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "step_kernel_lj256k.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def roofline_line(hbm_achieved, hbm_peak, hbm_kind, fp32_achieved, fp32_peak, fpps, traffic,
                  avg_kernel_s, launches, kernel="step_kernel<true>"):
    """The step kernel against the roofline that binds it: the algorithmic
    bytes (96 B per particle-step) over the measured HBM copy bandwidth, or
    the algorithmic FP32 flops over the measured FMA throughput, whichever
    takes longer. At rho 0.8442 that is FP32 (about 24 flop/B against a
    machine balance of about 11)."""
    hbm = {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
           "frac": hbm_achieved / hbm_peak, "peak_source": hbm_kind,
           "algorithmic_bytes_per_particle_step": ALGO_BYTES}
    fp32 = {"achieved": fp32_achieved, "peak": fp32_peak, "unit": "TFLOP/s",
            "frac": fp32_achieved / fp32_peak if fp32_peak else None,
            "flops_per_particle_step": fpps,
            "peak_source": "measured live (FMA chains on every SM)"}
    fp32_binds = fp32["frac"] is not None and fp32["frac"] > hbm["frac"]
    top = fp32 if fp32_binds else hbm
    return {"bound": "fp32" if fp32_binds else "hbm", "achieved": top["achieved"],
            "peak": top["peak"], "unit": top["unit"], "frac": top["frac"], "traffic": traffic,
            "kernel": kernel, "avg_kernel_us": avg_kernel_s * 1e6,
            "kernel_launches_timed": launches, "hbm": hbm, "fp32": fp32}


class Clocks:
    """nvidia-smi samples every 100 ms while the timed regions run."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def nvtx(start, name="timed_steps"):
    """Opens or closes an NVTX range (a no-op without NVTX support)."""
    try:
        import torch
        if start:
            torch.cuda.nvtx.range_push(name)
        else:
            torch.cuda.nvtx.range_pop()
    except (RuntimeError, AttributeError):
        pass


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    gpu_index = local
    if world > 1:
        # one GPU per process; the CUDA library and torch both see it as device 0
        visible = os.environ.get("CUDA_VISIBLE_DEVICES")
        ids = visible.split(",") if visible else [str(i) for i in range(64)]
        gpu_index = int(ids[local]) if ids[local].isdigit() else local
        os.environ["CUDA_VISIBLE_DEVICES"] = ids[local]
    return world, rank, gpu_index


def reduce_max(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_port_rate(n_target_seconds, pos, vel, box, n_warm=2):
    """The f64 oracle engine on this workload: (particle-steps/s, steps, cores)."""
    import oracle as O
    md = O.MD(pos, vel, [box] * 3, cutoff=WORK["cutoff"], skin=WORK["skin"], dt=WORK["dt"],
              shifted_force=True, langevin=(WORK["temperature"], WORK["friction"], WORK["seed"]))
    md.run(n_warm)
    steps, t0 = 0, time.perf_counter()
    while True:
        md.run(1)
        steps += 1
        el = time.perf_counter() - t0
        if (el >= n_target_seconds and steps >= 3) or steps >= 2000:
            break
    md.close()
    return len(pos) * steps / el, steps, O.threads(), el


def run_reference(args, world, rank):
    if rank != 0:
        return
    import numpy as np
    import oracle as O
    pos, vel, box = O.lattice_fcc(WORK["cells"], WORK["density"], WORK["temperature"], WORK["seed"])
    n = len(pos)
    md = O.MD(pos, vel, [box] * 3, cutoff=WORK["cutoff"], skin=WORK["skin"], dt=WORK["dt"],
              shifted_force=True, langevin=(WORK["temperature"], WORK["friction"], WORK["seed"]))
    md.run(args.warmup)
    t0 = time.perf_counter()
    md.run(args.steps)
    el = time.perf_counter() - t0
    md.close()
    value = n * args.steps / el
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config(n, 1), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.threads(), "kind": "port",
                         "sample": f"{args.steps} MD steps of the {n}-particle box after "
                                   f"{args.warmup} warm-up steps (f64 OpenMP cell-list engine)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's LJ path runs only through wgpu (graphics API, unavailable on "
                "this box) and its CPU crate has no LJ code; this arm is the oracle's f64 port",
    }
    print(json.dumps(line), flush=True)


def run_batched(args, world, rank, stream, flush_l2, hbm_peak, fp32_peak):
    """512 replicas of uneven N, density and temperature in one arena: the
    batched form, timed like the plain box, then the same replicas (a
    sample) each run as a plain single-box simulation, back to back."""
    import torch
    import virial_lj as vl

    reps = vl.uneven_replicas(BATCH["replicas"], BATCH["seed"] + 7919 * rank, BATCH["sizes"],
                              BATCH["densities"], BATCH["temperatures"], BATCH["friction"])
    total = sum(len(r.particles) for r in reps)
    # the neighbour skin and the step kernel's block size for this set, chosen
    # by the autotuner on this GPU
    skin, threads, tuned = vl.tune_batch(reps, BATCH["skins"], BATCH["threads"],
                                         cutoff=BATCH["cutoff"], dt=BATCH["dt"], stream=stream)
    b = vl.Batch(reps, cutoff=BATCH["cutoff"], skin=skin, dt=BATCH["dt"],
                 stream=stream.cuda_stream)
    b.set_step_threads(threads)
    b.step(max(args.warmup, 3))
    stream.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    k0 = b.kernels_executed()
    barrier(world)
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush_l2()
        starts[k].record(stream)
        b.step(1)
        ends[k].record(stream)
    stream.synchronize()
    barrier(world)
    launches = b.kernels_executed() - k0
    total_ms = sum(x.elapsed_time(y) for x, y in zip(starts, ends))
    max_ms = reduce_max(world, total_ms)
    value = world * total * args.steps / (max_ms / 1e3)
    # step kernel alone
    b.kernel_timing(True)
    for k in range(args.steps):
        flush_l2()
        b.step(1)
    kern_ms, kern_n = b.kernel_time()
    b.kernel_timing(False)
    kern_s = kern_ms / 1e3 / max(kern_n, 1)
    ms = b.measure()
    b.close()
    # rooflines with each replica's own density (truncated-shifted pairs)
    dens = [len(r.particles) / (r.box_size[0] * r.box_size[1] * r.box_size[2]) for r in reps]
    flops = sum(len(r.particles) * flops_per_particle_step(d, 20.0, BATCH["cutoff"], skin)
                for r, d in zip(reps, dens))
    bytes_ = ALGO_BYTES * total
    bound_s = max(bytes_ / (hbm_peak * 1e9), flops / (fp32_peak * 1e12)) if fp32_peak else None

    # the plain path on the same replicas: every PLAIN_SAMPLE_EVERY-th replica
    # as its own simulation, one after another (as the reference would run them)
    plain_n, plain_s = 0, 0.0
    for r in reps[::PLAIN_SAMPLE_EVERY]:
        st = vl.Settings(r.box_size, cutoff=BATCH["cutoff"], dt=BATCH["dt"],
                         thermostat=r.thermostat, skin=BATCH["skin"])
        try:
            sim = vl.LennardJones(r.particles, st, stream=stream.cuda_stream)
        except vl.VljError:
            continue  # a box under three cells wide: the plain path refuses it
        sim.step(3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream.synchronize()
        e0.record(stream)
        sim.step(PLAIN_SAMPLE_STEPS)
        e1.record(stream)
        stream.synchronize()
        plain_s += e0.elapsed_time(e1) / 1e3
        plain_n += len(r.particles) * PLAIN_SAMPLE_STEPS
        sim.close()
    plain_value = plain_n / plain_s if plain_s else None
    # compressibility factor at the measured temperature: PV / NkT = 1 + W / (2 KE)
    pv = [1.0 + m.virial / (2.0 * m.kinetic) for m in ms]
    return {
        "workload": f"lj-batched-{BATCH['replicas']}-replicas-uneven",
        "value": value, "unit": UNIT, "ms_per_step": max_ms / args.steps, "steps": args.steps,
        "replicas": len(reps), "particles": total,
        "config": {"sizes": "N log-uniform in [500, 20000]", "densities": "uniform in [0.01, 0.90]",
                   "temperatures": "uniform in [0.7, 2.0], Langevin gamma=1.0",
                   "cutoff": BATCH["cutoff"], "cutoff_style": "truncated-shifted",
                   "skin": skin, "step_threads": threads,
                   "tuned_ms_per_step": {f"skin {k[0]} threads {k[1]}": v * 1e3
                                         for k, v in tuned.items()},
                   "plain_skin": BATCH["skin"], "dt": BATCH["dt"],
                   "seed": BATCH["seed"] + 7919 * rank,
                   "l2": "flushed between timed steps (256 MiB write on the stream)"},
        "gpu_launches": launches,
        "step_kernel_us": kern_s * 1e6,
        "roofline": {"hbm_achieved_gbs": bytes_ / kern_s / 1e9, "hbm_peak_gbs": hbm_peak,
                     "hbm_frac": bytes_ / kern_s / 1e9 / hbm_peak,
                     "fp32_achieved_tflops": flops / kern_s / 1e12, "fp32_peak_tflops": fp32_peak,
                     "fp32_frac": flops / kern_s / 1e12 / fp32_peak if fp32_peak else None,
                     "bound_us": bound_s * 1e6 if bound_s else None,
                     "frac": bound_s / kern_s if bound_s else None,
                     "kernel": "step_kernel<false>",
                     "flops_per_step": flops, "algorithmic_bytes_per_step": bytes_},
        "plain_same_replicas": {"value": plain_value, "unit": UNIT,
                                "sample": f"every {PLAIN_SAMPLE_EVERY}th replica as its own "
                                          f"simulation, {PLAIN_SAMPLE_STEPS} steps each, back "
                                          "to back (CUDA events)"},
        "batched_vs_plain": value / plain_value if plain_value else None,
        "pv_over_nkt": {"min": min(pv), "max": max(pv)},
    }


SLAB = dict(n=16000, lattice=(20.0, 20.0, 54.8), lift=47.6, box=(20.0, 20.0, 150.0),
            temperature=0.7, friction=0.5, dt=0.005, bins=300, every=20)
REFERENCE_PROFILE_SAMPLE_MS = 4.0  # 240 slabs, 15,600 molecules, M1 Air (published)


def run_slab(args, world, rank, stream, flush_l2):
    """The liquid-vapour slab with density and pressure-tensor profiles: 16,000
    atoms on the reference's lattice_box (20 x 20 x 54.8, lifted 47.6) in a
    20 x 20 x 150 box, Langevin T = 0.7, gamma = 0.5, force-shifted, dt 0.005,
    a 300-bin profile sample every 20 steps. Timed per cycle (20 steps and one
    sample, L2 flushed before each), and the sample alone."""
    import torch
    import virial_lj as vl

    p = vl.lattice_box(SLAB["n"], list(SLAB["lattice"]), SLAB["temperature"], 3 + rank)
    p["pos"][:, 2] += SLAB["lift"]
    sim = vl.LennardJones(p, vl.Settings(list(SLAB["box"]), cutoff=2.5, dt=SLAB["dt"], skin=0.3,
                                         shifted_force=True, profile_bins=SLAB["bins"],
                                         thermostat=vl.Langevin(SLAB["temperature"],
                                                                SLAB["friction"], 11 + rank)),
                          stream=stream.cuda_stream)
    sim.step(max(args.warmup, 3) * SLAB["every"])
    sim.clear_profile()
    cycles = max(args.steps // SLAB["every"], 5)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(cycles)]
    sample_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                 for _ in range(cycles)]
    stream.synchronize()
    barrier(world)
    for a, b in ev:
        flush_l2()
        a.record(stream)
        sim.step(SLAB["every"])
        sim.sample_profile()
        b.record(stream)
    for a, b in sample_ev:
        flush_l2()
        a.record(stream)
        sim.sample_profile()
        b.record(stream)
    stream.synchronize()
    cycle_ms = reduce_max(world, sum(a.elapsed_time(b) for a, b in ev))
    sample_ms = reduce_max(world, sum(a.elapsed_time(b) for a, b in sample_ev)) / cycles
    prof = sim.read_profile()
    m = sim.measure_now()
    sim.close()
    steps = cycles * SLAB["every"]
    return {"workload": "lj-slab-16k-20x20x150-fs-langevin0.7-profile300-every20",
            "value": world * SLAB["n"] * steps / (cycle_ms / 1e3), "unit": UNIT,
            "ms_per_step": cycle_ms / steps, "steps": steps, "profile_samples": cycles,
            "profile_sample_ms": sample_ms,
            "reference_profile_sample_ms": REFERENCE_PROFILE_SAMPLE_MS,
            "reference_note": "published: about 4 ms per 240-slab sample of 15,600 molecules "
                              "on an M1 Air (Metal), adding 25 % at one sample per 20 steps",
            "sampling_share": sample_ms * cycles / cycle_ms,
            "config": {"cutoff": 2.5, "cutoff_style": "force-shifted", "skin": 0.3,
                       "thermostat": "langevin T=0.7 gamma=0.5", "dt": SLAB["dt"],
                       "bins": SLAB["bins"], "sample_every": SLAB["every"],
                       "l2": "flushed before each cycle and each lone sample"},
            "check": {"interfaces": len(prof.interfaces(0.37)), "list_overflow": m.list_overflow,
                      "list_grows": m.list_grows}}


def run_small(args, world, rank, stream, flush_l2):
    """The small plain box in full: 1000 atoms on the reference's lattice()
    at rho 0.8442 (box 10.58; fcc 5^3 x 4 holds only 500, in a box under three
    cutoff + skin wide), truncated-shifted, Maxwell-Boltzmann at T = 0.72,
    constant energy, dt 0.005, 1000 steps, timed as one enqueue of the 1000
    steps (L2 flushed before it; the box's 100 KB stays in L2 for the run,
    as in any run of it), with PE, KE, virial, pressure and the drift of E
    per particle."""
    import torch
    import virial_lj as vl

    n = 1000
    box = (n / 0.8442) ** (1.0 / 3.0)
    p = vl.lattice(n, box, 0.72, 1 + rank)
    st = vl.Settings([box] * 3, cutoff=2.5, dt=0.005, skin=0.3)
    sim = vl.LennardJones(p, st, stream=stream.cuda_stream)
    sim.step(50)  # warm-up on a copy, to build the graphs
    sim.close()
    sim = vl.LennardJones(p, st, stream=stream.cuda_stream)
    sim.step(16)
    m0 = sim.measure_now()
    stream.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush_l2()
    e0.record(stream)
    sim.step(1000)
    e1.record(stream)
    stream.synchronize()
    ms = reduce_max(world, e0.elapsed_time(e1))
    m1 = sim.measure_now()
    sim.close()
    return {"workload": "lj-lattice-1000-rho0.8442-truncated-nve-T0.72-1000-steps",
            "value": world * n * 1000 / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / 1000,
            "ms_per_run": ms, "steps": 1000,
            "config": {"dt": 0.005, "cutoff": 2.5, "skin": 0.3, "thermostat": "none",
                       "launch": "one enqueue of 1000 steps (16-step graphs)",
                       "l2": "flushed before the run"},
            "readouts": {"potential_per_particle": m1.potential / n,
                         "kinetic_per_particle": m1.kinetic / n,
                         "virial_per_particle": m1.virial / n, "pressure": m1.pressure(),
                         "drift_per_particle": (m1.energy() - m0.energy()) / n,
                         "list_rebuilds": m1.list_rebuilds}}


def run_heat_flux(args, world, rank, stream):
    """The large constant-energy box with the heat current sampled every step:
    16,384,000 atoms (fcc 160^3 x 4, rho 0.8442), truncated-shifted, dt 0.004.
    Its working set (15 GB) dwarfs the L2, so steps run back to back."""
    import torch
    import virial_lj as vl

    p, box = vl.lattice_fcc(160, 0.8442, 0.722, 5 + rank)
    n = len(p)
    sim = vl.LennardJones(p, vl.Settings([box] * 3, cutoff=2.5, dt=0.004, skin=0.3),
                          stream=stream.cuda_stream)
    del p
    steps = max(args.steps // 4, 10)
    sim.record_heat_current(steps + 3)
    for _ in range(3):
        sim.step(1)
        sim.sample_heat_current()
    stream.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        sim.step(1)
        sim.sample_heat_current()
    e1.record(stream)
    stream.synchronize()
    ms = reduce_max(world, e0.elapsed_time(e1))
    j = sim.read_heat_current()
    m = sim.measure_now()
    sim.close()
    return {"workload": "lj-fcc160x4-16.4M-rho0.8442-truncated-nve-heat-current-every-step",
            "value": world * n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "particles_per_box": n,
            "config": {"dt": 0.004, "cutoff": 2.5, "skin": 0.3, "thermostat": "none",
                       "sample": "one heat-current sample (3 x i64 fixed point) per step",
                       "l2": "working set 15 GB, far above L2"},
            "heat_current_samples": len(j), "list_overflow": m.list_overflow}


def run_ours(args, world, rank, gpu_index):
    import numpy as np
    import torch
    import virial_lj as vl

    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    p, box = vl.lattice_fcc(WORK["cells"], WORK["density"], WORK["temperature"], WORK["seed"] + rank)
    n = len(p)
    settings = vl.Settings([box] * 3, cutoff=WORK["cutoff"], dt=WORK["dt"],
                           thermostat=vl.Langevin(WORK["temperature"], WORK["friction"],
                                                  WORK["seed"] + rank),
                           shifted_force=True, skin=WORK["skin"])
    # the step kernel's form (cell tiles' bricks per row, particles per
    # block), timed on a copy of the box; none of them changes the trajectory
    tune_stats = {}
    tile_cols, step_threads, form_times = vl.tune_box(p, settings, stream=stream, stats=tune_stats)
    sim = vl.LennardJones(p, settings, stream=stream.cuda_stream)
    sim.set_tile_cols(tile_cols)
    sim.set_step_threads(step_threads)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.fill_(1)

    # warm-up
    sim.step(max(args.warmup, 3))
    stream.synchronize()

    # ---- timed region: K steps, L2 flushed between them ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    reb0 = sim.measure_now().list_rebuilds
    k0 = sim.kernels_executed()
    barrier(world)
    torch.cuda.synchronize()
    clocks = Clocks(gpu_index)
    if rank == 0:
        clocks.start()
    # an NVTX range around the timed steps, so that a profiler can take
    # exactly their launches (ncu --nvtx --nvtx-include "timed_steps/")
    nvtx(True)
    for k in range(args.steps):
        flush_l2()
        starts[k].record(stream)
        sim.step(1)
        ends[k].record(stream)
    nvtx(False)
    stream.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    total_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    launches = sim.kernels_executed() - k0  # this library's kernels that ran in the region
    m = sim.measure_now()
    rebuilds = m.list_rebuilds - reb0
    max_ms = reduce_max(world, total_ms)
    value = world * n * args.steps / (max_ms / 1e3)

    # ---- the step kernel alone, for the roofline (CUDA events around each launch) ----
    sim.kernel_timing(True)
    for k in range(args.steps):
        flush_l2()
        sim.step(1)
    kern_ms, kern_n = sim.kernel_time()
    sim.kernel_timing(False)
    avg_kernel_s = kern_ms / 1e3 / max(kern_n, 1)
    peak, peak_kind = measured_peaks()
    achieved = ALGO_BYTES * n / avg_kernel_s / 1e9
    fp32_peak = vl.fp32_peak()
    fpps = flops_per_particle_step(WORK["density"])
    fp32_achieved = fpps * n / avg_kernel_s / 1e12
    traffic = profile_traffic()

    # ---- the same steps with the cell grid also rebuilt on every step (the
    # 256k workload's wording; the reference bins only with the lists) ----
    sim.set_grid_every_step(True)
    sim.step(max(args.warmup, 3))
    g_starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    g_ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush_l2()
        g_starts[k].record(stream)
        sim.step(1)
        g_ends[k].record(stream)
    stream.synchronize()
    barrier(world)
    grid_ms = reduce_max(world, sum(s.elapsed_time(e) for s, e in zip(g_starts, g_ends)))
    sim.set_grid_every_step(False)
    grid_every = {"value": world * n * args.steps / (grid_ms / 1e3), "unit": UNIT,
                  "ms_per_step": grid_ms / args.steps,
                  "note": "bin, scan, scatter and per-cell sort on every step, lists on the "
                          "skin/2 trigger; same trajectory to the bit; timed like value"}

    # ---- the batched form on 512 uneven replicas, and the plain path on them ----
    batched = run_batched(args, world, rank, stream, flush_l2, peak, fp32_peak)
    heat_flux = run_heat_flux(args, world, rank, stream)
    slab = run_slab(args, world, rank, stream, flush_l2)
    small = run_small(args, world, rank, stream, flush_l2)
    clk = clocks.stop() if rank == 0 else None

    # ---- end to end through the C ABI with host buffers (pinned) ----
    e2e_steps = max(3, min(args.steps, 10))
    start = vl.lattice_fcc(WORK["cells"], WORK["density"], WORK["temperature"], WORK["seed"] + rank)[0]
    pinned_in = torch.empty(start.nbytes, dtype=torch.uint8, pin_memory=True)
    pinned_out = torch.empty(start.nbytes, dtype=torch.uint8, pin_memory=True)
    host = pinned_in.numpy().view(vl.PARTICLE)
    back = pinned_out.numpy().view(vl.PARTICLE)
    host[:] = start
    sim.write_particles(host)
    sim.run(E2E_INNER)  # warm
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.write_particles(host)
        sim.run(E2E_INNER)
        meas = sim.measure_now()
        sim.read_particles(out=back)
    e2e_s = time.perf_counter() - t0
    e2e_max = reduce_max(world, e2e_s)
    e2e_value = world * n * E2E_INNER * e2e_steps / e2e_max
    # the particle array each way (48 B per particle), plus the measurement's
    # fixed-point sums and control words and the upload's status word
    h2d = 48 * n
    d2h = 48 * n + 8 * 8 + 32 + 48

    # ---- CPU baseline (rank 0, one GPU only) ----
    cpu = None
    if rank == 0 and world == 1:
        rate, steps, cores, el = cpu_port_rate(args.cpu_seconds, p["pos"], p["vel"], box)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{steps} MD steps of the same {n}-particle box ({el:.1f} s, f64 "
                         f"OpenMP cell-list engine, 2 warm-up steps)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "state_dtype": "f64",
            "data": "synthetic",
            "config": dict(config(n, world), step_form={
                "tile_cols": tile_cols, "step_threads": step_threads,
                "tuned_ms_per_step": {f"tiles {c} threads {t}": v * 1e3
                                      for (c, t), v in form_times.items()},
                "note": "virial_lj.tune_box on a copy of the box (L2 flushed per step); "
                        "every form gives the same trajectory to the bit"}),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "note": f"per bench step: write particles from pinned host memory, "
                            f"{E2E_INNER} MD steps, measure_now, read_particles into pinned "
                            "host memory; wall clock"},
            "roofline": roofline_line(achieved, peak, peak_kind, fp32_achieved, fp32_peak, fpps,
                                      traffic, avg_kernel_s, kern_n,
                                      "tile_step_kernel<true>" if tile_cols
                                      else f"step_kernel<true, false, {step_threads}>"),
            "cpu_baseline": cpu,
            "grid_every_step": grid_every,
            "batched": batched,
            "heat_flux": heat_flux,
            "slab": slab,
            "small_box": small,
            "clocks": clk,
            "gpu_launches": launches,
            # this library's kernels that ran before the timed steps (the
            # tuner's copy of the box, then the box's creation and warm-up),
            # counted on the device (graph nodes included)
            "kernels_before_timed": tune_stats.get("kernels", 0) + k0,
            "list_rebuilds_timed": rebuilds,
            "check": {"potential": meas.potential, "virial": meas.virial,
                      "temperature": 2 * meas.kinetic / (3 * n), "list_overflow": meas.list_overflow},
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    world, rank, gpu_index = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, gpu_index)


if __name__ == "__main__":
    main()
