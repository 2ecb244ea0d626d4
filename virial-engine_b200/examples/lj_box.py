"""Run one Lennard-Jones box through the library and print measurements.

The reference's `examples/gas` drives LennardJones the same way (new, step,
measure). Also the target of the committed ncu summaries in profiles/.

    python virial-engine_b200/examples/lj_box.py --cells 40 --steps 100
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
    ap.add_argument("--density", type=float, default=0.8442)
    ap.add_argument("--temperature", type=float, default=1.0)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--dt", type=float, default=0.005)
    ap.add_argument("--truncated", action="store_true", help="truncated-shifted, not force-shifted")
    ap.add_argument("--nve", action="store_true", help="constant energy instead of Langevin")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--no-graphs", action="store_true",
                    help="enqueue steps as direct launches (profilers see each kernel)")
    args = ap.parse_args()
    p, box = vl.lattice_fcc(args.cells, args.density, args.temperature, args.seed)
    thermostat = None if args.nve else vl.Langevin(args.temperature, 1.0, args.seed)
    sim = vl.LennardJones(p, vl.Settings([box] * 3, dt=args.dt, thermostat=thermostat,
                                         shifted_force=not args.truncated))
    if args.no_graphs:
        sim.set_graphs(False)
    m = sim.measure_now()
    print(f"{len(p)} particles, box {box:.4f}: E {m.energy():.6f} P {m.pressure():.6f}")
    t0 = time.perf_counter()
    sim.run(args.steps)
    el = time.perf_counter() - t0
    m = sim.measure_now()
    print(f"after {args.steps} steps ({el * 1e6 / max(args.steps, 1):.1f} us/step wall): "
          f"E {m.energy():.6f} T {2 * m.kinetic / (3 * len(p)):.5f} P {m.pressure():.6f} "
          f"rebuilds {m.list_rebuilds} overflow {m.list_overflow}")


if __name__ == "__main__":
    main()
