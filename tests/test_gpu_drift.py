"""Energy drift of the CUDA path against the reference's double-float path.

The reference holds positions and velocities as double-floats and reports
its drift from its own time-step study (crates/virial-particles/tests/
lj_dt_study.rs; docs/VALIDATION.md: 4096 molecules at density 0.1 on its
lattice at T = 2 (seed 13), force-shifted cutoff 2.5, constant energy, dt
0.004, 40 time units: drift 5.0e-5 on its GPU). Its path is restated in the
oracle (oracle/dfpath.c: double-float state, f32 pair arithmetic on packed
positions, df64 sums). Here both paths, and the f64 engine beside them, run
the same starts side by side: the reference's drift configuration and the
small plain workload (1000 atoms at rho 0.8442, T 0.72, both cutoff styles,
1000 steps). The reference's lattice seeds its generator with seed | 1
(lennard_jones.rs:1409), so seeds 2 and 3 give the same start: the distinct
odd seeds 1, 3, ..., 11 stand in for "seeds 1, 2, 3". Each drift is the
relative change of total
energy over the run. Over these runs the trajectories decorrelate (the
dynamics is chaotic), so each path's drift is a sample: the CUDA path must
be no worse than the double-float path, within the double-float path's own
seed-to-seed spread. Run with -s for the table.
"""

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def drifts(gpu, O, n, density, temperature, seed, shifted_force, dt, steps):
    length = (n / density) ** (1.0 / 3.0)
    pos, vel = O.lattice(n, length, temperature, seed)
    box = np.array([float(np.float32(length))] * 3)
    sim = gpu.LennardJones(gpu.particles(pos, vel),
                           gpu.Settings([length] * 3, cutoff=2.5, dt=dt, skin=0.3,
                                        shifted_force=shifted_force))
    df = O.DoubleFloatMD(pos, vel, box, 2.5, dt, shifted_force)
    f64 = O.MD(pos, vel, box, cutoff=2.5, skin=0.3, dt=dt, shifted_force=shifted_force)
    e = [sim.measure_now().energy(), sum(df.measure()[:2])]
    m = f64.measure()
    e.append(m.kinetic + m.potential)
    sim.run(steps)
    df.run(steps)
    f64.run(steps)
    m = f64.measure()
    e1 = [sim.measure_now().energy(), sum(df.measure()[:2]), m.kinetic + m.potential]
    df.close()
    f64.close()
    sim.close()
    return [(b - a) / abs(a) for a, b in zip(e, e1)]


def check(rows, label):
    d = np.array(rows)  # seeds x (CUDA, double-float, f64)
    print(f"\n{label}")
    for r in d:
        print(f"  CUDA {r[0]:+.3e}   double-float {r[1]:+.3e}   f64 {r[2]:+.3e}")
    cuda, df = np.abs(d[:, 0]).mean(), np.abs(d[:, 1]).mean()
    spread = d[:, 1].std()
    print(f"  mean |drift|: CUDA {cuda:.3e}, double-float {df:.3e} (seed spread {spread:.1e})")
    assert cuda <= df + spread, (label, cuda, df, spread)


@pytest.mark.parametrize("shifted_force", [False, True])
def test_drift_small_plain_workload(gpu, O, shifted_force):
    rows = [drifts(gpu, O, 1000, 0.8442, 0.72, seed, shifted_force, 0.005, 1000)
            for seed in (1, 3, 5, 7, 9, 11)]
    check(rows, f"1000 atoms, rho 0.8442, T 0.72, dt 0.005, 1000 steps, "
                f"{'force' if shifted_force else 'truncated'}-shifted")


def test_drift_reference_study_configuration(gpu, O):
    # lj_dt_study.rs: 4096 molecules, density 0.1, T = 2, force-shifted,
    # dt 0.004, 40 time units; seed 13 is the reference's, 15 and 17 give the spread
    rows = [drifts(gpu, O, 4096, 0.1, 2.0, seed, True, 0.004, 10_000) for seed in (13, 15, 17)]
    check(rows, "4096 molecules, rho 0.1, T 2, force-shifted, dt 0.004, 40 time units "
                "(the reference measured +5.0e-5 with seed 13)")
    # the reference's own figure sets the scale: every path within 4x of it
    assert all(abs(r[0]) < 4 * 5.0e-5 for r in rows), rows
