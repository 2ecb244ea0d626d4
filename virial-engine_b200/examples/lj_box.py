"""Run one Lennard-Jones box through the library and print measurements.

The reference's `examples/gas` drives LennardJones the same way (new, step,
measure). Also the target of the committed ncu summaries in profiles/.

    python virial-engine_b200/examples/lj_box.py --cells 40 --steps 100
    python virial-engine_b200/examples/lj_box.py --cells 10 --steps 1000 --record run1
    python virial-engine_b200/examples/lj_box.py --lattice 1000 --temperature 0.72 --nve --truncated
"""

import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import virial_lj as vl  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=40, help="fcc unit cells per side (4 atoms each)")
    ap.add_argument("--lattice", type=int, default=0, metavar="N",
                    help="N atoms on the reference's lattice() in a cube of the density "
                         "instead of the fcc lattice")
    ap.add_argument("--density", type=float, default=0.8442)
    ap.add_argument("--temperature", type=float, default=1.0)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--dt", type=float, default=0.005)
    ap.add_argument("--truncated", action="store_true", help="truncated-shifted, not force-shifted")
    ap.add_argument("--nve", action="store_true", help="constant energy instead of Langevin")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--no-graphs", action="store_true",
                    help="enqueue steps as direct launches (profilers see each kernel)")
    ap.add_argument("--no-tiles", action="store_true",
                    help="step kernel with per-particle gathers instead of cell tiles")
    ap.add_argument("--threads", type=int, default=0, choices=(0, 64, 128, 256),
                    help="particles per block of the step kernel (0: the library's default)")
    ap.add_argument("--record", default=None, metavar="DIR",
                    help="write measurements.csv (a row every --every steps), positions.npy "
                         "and run.json into DIR, in the reference's formats")
    ap.add_argument("--every", type=int, default=10)
    args = ap.parse_args()
    if args.lattice:
        box = (args.lattice / args.density) ** (1.0 / 3.0)
        p = vl.lattice(args.lattice, box, args.temperature, args.seed)
    else:
        p, box = vl.lattice_fcc(args.cells, args.density, args.temperature, args.seed)
    thermostat = None if args.nve else vl.Langevin(args.temperature, 1.0, args.seed)
    sim = vl.LennardJones(p, vl.Settings([box] * 3, dt=args.dt, thermostat=thermostat,
                                         shifted_force=not args.truncated))
    if args.no_graphs:
        sim.set_graphs(False)
    if args.no_tiles:
        sim.set_tiles(False)
    if args.threads:
        sim.set_step_threads(args.threads)
    m = sim.measure_now()
    print(f"{len(p)} particles, box {box:.4f}: E {m.energy():.6f} P {m.pressure():.6f}")
    t0 = time.perf_counter()
    if args.record:
        record(sim, args, len(p), box)
    else:
        sim.run(args.steps)
    el = time.perf_counter() - t0
    m = sim.measure_now()
    print(f"after {args.steps} steps ({el * 1e6 / max(args.steps, 1):.1f} us/step wall): "
          f"E {m.energy():.6f} T {2 * m.kinetic / (3 * len(p)):.5f} P {m.pressure():.6f} "
          f"rebuilds {m.list_rebuilds} overflow {m.list_overflow}")


def gpu_name():
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:  # no torch, or no device name to be had
        return "unknown"


def record(sim, args, n, box):
    from virial_lj import data
    log = data.DataLog(args.record)
    dof = 3 * n if not args.nve else 3 * n - 3
    done = 0
    while True:
        m = sim.measure_now()
        log.row([("step", m.step), ("time", m.time), ("kinetic", m.kinetic),
                 ("potential", m.potential), ("energy", m.energy()), ("virial", m.virial),
                 ("temperature", m.temperature(dof)), ("pressure", m.pressure()),
                 ("list_rebuilds", m.list_rebuilds)])
        if done >= args.steps:
            break
        k = min(args.every, args.steps - done)
        sim.run(k)
        done += k
    q = sim.read_particles()
    log.snapshot("positions", q["pos"].shape, q["pos"])
    log.meta("particles", n)
    log.meta("box", data.exact(box))
    settings = [("dt", args.dt), ("density", args.density), ("temperature", args.temperature),
                ("thermostat", "none" if args.nve else "langevin"), ("seed", args.seed),
                ("cutoff_style", "truncated-shifted" if args.truncated else "force-shifted")]
    log.write(data.Manifest("lennard-jones box", gpu=gpu_name(), version="b200",
                            frames=done, settings=settings))


if __name__ == "__main__":
    main()
