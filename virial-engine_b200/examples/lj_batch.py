"""Step many uneven Lennard-Jones boxes together and print what they measure.

512 replicas by default: N log-uniform in [500, 20000], density uniform in
[0.01, 0.90], temperature uniform in [0.7, 2.0] under Langevin friction 1,
truncated-shifted cutoff 2.5, dt 0.004, all in one arena. Also the target of
the committed ncu summaries of the batched kernels in profiles/.

    python virial-engine_b200/examples/lj_batch.py --replicas 512 --steps 100
"""

import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import virial_lj as vl  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--replicas", type=int, default=512)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--dt", type=float, default=0.004)
    ap.add_argument("--no-graphs", action="store_true",
                    help="enqueue steps as direct launches (profilers see each kernel)")
    args = ap.parse_args()
    reps = vl.uneven_replicas(args.replicas, args.seed)
    total = sum(len(r.particles) for r in reps)
    b = vl.Batch(reps, cutoff=2.5, skin=0.3, dt=args.dt)
    if args.no_graphs:
        b.set_graphs(False)
    t0 = time.perf_counter()
    b.run(args.steps)
    el = time.perf_counter() - t0
    ms = b.measure()
    rebuilds = sum(m.list_rebuilds for m in ms)
    print(f"{len(reps)} replicas, {total} particles: {args.steps} steps in {el:.3f} s "
          f"({total * args.steps / el:.3e} particle-steps/s wall), {rebuilds} box rebuilds, "
          f"overflow {max(m.list_overflow for m in ms)}")
    for r in (0, len(reps) // 2, len(reps) - 1):
        m = ms[r]
        print(f"  replica {r}: N {m.count} rho {m.count / m.volume:.4f} "
              f"T {2 * m.kinetic / (3 * m.count):.4f} PV/NkT {1 + m.virial / (2 * m.kinetic):.4f}")


if __name__ == "__main__":
    main()
