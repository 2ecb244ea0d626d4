"""A liquid-vapour slab with density and pressure-tensor profiles.

The reference's coexistence setup (crates/virial-particles/tests/
coexistence.rs:241-244): atoms on lattice_box in the middle of a long
periodic box, which melts into a liquid slab between two vapour regions; a
profile along z every few steps gives the densities, the normal and
tangential pressures and the surface tension (lennard_jones.rs:209-279).
Also the target of the profile kernel's ncu summary in profiles/.

    python virial-engine_b200/examples/lj_slab.py --steps 2000 --every 20
"""

import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import virial_lj as vl  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--atoms", type=int, default=16000)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=20, help="steps between profile samples")
    ap.add_argument("--bins", type=int, default=300)
    ap.add_argument("--temperature", type=float, default=0.7)
    ap.add_argument("--no-graphs", action="store_true",
                    help="enqueue steps as direct launches (profilers see each kernel)")
    args = ap.parse_args()
    p = vl.lattice_box(args.atoms, [20.0, 20.0, 54.8], args.temperature, 3)
    p["pos"][:, 2] += 47.6
    sim = vl.LennardJones(p, vl.Settings([20.0, 20.0, 150.0], cutoff=2.5, dt=0.005, skin=0.3,
                                         shifted_force=True, profile_bins=args.bins,
                                         thermostat=vl.Langevin(args.temperature, 0.5, 11)))
    if args.no_graphs:
        sim.set_graphs(False)
    t0 = time.perf_counter()
    for _ in range(max(args.steps // args.every, 1)):
        sim.step(args.every)
        sim.sample_profile()
    prof = sim.read_profile()
    el = time.perf_counter() - t0
    m = sim.measure_now()
    d = prof.density()
    print(f"{args.atoms} atoms, {prof.samples} samples in {el:.2f} s: densities "
          f"{max(d):.4f} / {min(d):.4f}, interfaces {len(prof.interfaces(0.37))}, "
          f"surface tension {prof.surface_tension():.4f}, T {2 * m.kinetic / (3 * args.atoms):.4f}, "
          f"list grows {m.list_grows}")


if __name__ == "__main__":
    main()
