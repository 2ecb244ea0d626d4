"""The error of every reported quantity against the f64 truth, for the CUDA
path and, beside it, for the reference's plain double-float path (restated in
the oracle, dfpath.c), on the small plain workload: 1000 atoms on the
reference's lattice at rho 0.8442 and T 0.72, truncated-shifted cutoff 2.5,
constant energy, dt 0.005, 1000 steps.

Each path's PE, KE, virial and pressure are compared with the f64 values of
the state that path holds (its own positions and velocities); energy drift
is each path's own relative change of total energy over the run, next to the
f64 engine's. Run with -s to see the table.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 1000


def truth(O, pos, vel, box):
    pe, w = O.all_pairs(np.mod(pos, box), box, 2.5, False)
    ke = 0.5 * float(np.sum(vel * vel))
    return ke, pe, float(w.sum())


def rel(a, b):
    return abs((a - b) / b)


def errors(O, box, ke, pe, w, pos, vel):
    ke64, pe64, w64 = truth(O, pos, vel, box)
    volume = float(np.prod(box))
    p, p64 = (2 * ke + w) / (3 * volume), (2 * ke64 + w64) / (3 * volume)
    return {"PE": rel(pe, pe64), "KE": rel(ke, ke64), "virial": rel(w, w64),
            "pressure": rel(p, p64)}


def test_error_table(gpu, O):
    length = (1000 / 0.8442) ** (1.0 / 3.0)
    pos, vel = O.lattice(1000, length, 0.72, 1)
    box = np.array([float(np.float32(length))] * 3)

    sim = gpu.LennardJones(gpu.particles(pos, vel),
                           gpu.Settings([length] * 3, cutoff=2.5, dt=0.005, skin=0.3))
    ref = O.DoubleFloatMD(pos, vel, box, 2.5, 0.005, False)
    f64 = O.MD(pos, vel, box, cutoff=2.5, skin=0.3, dt=0.005)

    def gpu_state():
        m = sim.measure_now()
        q = sim.read_particles()
        return m.kinetic, m.potential, m.virial, q["pos"], q["vel"]

    table = {}
    g0, r0 = gpu_state(), ref.measure()
    m0 = f64.measure()
    table["CUDA path, t = 0"] = errors(O, box, *g0)
    table["double-float path, t = 0"] = errors(O, box, *r0)
    sim.run(STEPS)
    ref.run(STEPS)
    f64.run(STEPS)
    g1, r1 = gpu_state(), ref.measure()
    m1 = f64.measure()
    table[f"CUDA path, t = {STEPS} steps"] = errors(O, box, *g1)
    table[f"double-float path, t = {STEPS} steps"] = errors(O, box, *r1)

    def drift(e0, e1):
        return (e1 - e0) / abs(e0)

    drifts = {"CUDA path": drift(g0[0] + g0[1], g1[0] + g1[1]),
              "double-float path": drift(r0[0] + r0[1], r1[0] + r1[1]),
              "f64 engine": drift(m0.kinetic + m0.potential, m1.kinetic + m1.potential)}
    print()
    print(f"{'':36s} {'PE':>9s} {'KE':>9s} {'virial':>9s} {'pressure':>9s}")
    for name, e in table.items():
        print(f"{name:36s} " + " ".join(f"{e[k]:9.1e}" for k in ("PE", "KE", "virial", "pressure")))
    for name, d in drifts.items():
        print(f"energy drift over {STEPS} steps, {name:18s} {d:+.3e}")

    for name, e in table.items():
        if name.startswith("CUDA"):
            assert e["PE"] < 1e-6 and e["virial"] < 1e-6 and e["pressure"] < 1e-6, (name, e)
            assert e["KE"] < 1e-9, (name, e)
        else:
            assert e["PE"] < 1e-5 and e["virial"] < 1e-5, (name, e)
    # no worse than f64: the change over the run is the integrator's
    assert abs(drifts["CUDA path"]) <= 2.0 * abs(drifts["f64 engine"]) + 1e-5, drifts
