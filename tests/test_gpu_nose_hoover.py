"""Nose-Hoover thermostat on the CUDA path (lennard_jones.wgsl:309-397).

Against the oracle's f64 restatement of the same splitting (oracle/md.c
nh_step): a short trajectory agrees particle by particle, the extended energy
KE + PE + Q xi^2 / 2 + g k T eta drifts no more than the f64 engine's, and the
temperature settles at the target.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs((a - b) / b)


def liquid(gpu, t0=0.72):
    L = (1000 / 0.8442) ** (1 / 3)
    return gpu.lattice(1000, L, t0, 1), L


def make(gpu, p, L, temperature=1.0, period=0.5, shifted_force=False, dt=0.005):
    s = gpu.Settings([L] * 3, dt=dt, shifted_force=shifted_force,
                     thermostat=gpu.NoseHoover(temperature, period))
    return gpu.LennardJones(p, s)


@pytest.mark.parametrize("shifted_force", [False, True])
def test_short_trajectory_matches_f64_oracle(gpu, O, shifted_force):
    p, L = liquid(gpu)
    sim = make(gpu, p, L, shifted_force=shifted_force)
    md = O.MD(p["pos"], p["vel"], sim.box_size(), dt=0.005, shifted_force=shifted_force,
              nose_hoover=(1.0, 0.5))
    m0 = sim.measure_now()
    assert m0.thermostat_energy == 0.0
    sim.run(20)
    md.run(20)
    q = sim.read_particles()
    pos, vel = md.read()
    box = np.array(sim.box_size())
    d = q["pos"] - pos
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-5
    assert np.abs(q["vel"] - vel).max() < 1e-4
    mg, mc = sim.measure_now(), md.measure()
    assert rel(mg.kinetic, mc.kinetic) < 1e-6
    assert rel(mg.potential, mc.potential) < 1e-6
    assert abs(mg.thermostat_energy - mc.thermostat_energy) < 1e-6 * abs(mc.kinetic)


def test_extended_energy_drift_no_worse_than_f64(gpu, O):
    p, L = liquid(gpu)
    sim = make(gpu, p, L, shifted_force=True)
    md = O.MD(p["pos"], p["vel"], sim.box_size(), dt=0.005, shifted_force=True,
              nose_hoover=(1.0, 0.5))
    e0g = sim.measure_now().extended_energy()
    m0 = md.measure()
    e0c = m0.kinetic + m0.potential + m0.thermostat_energy
    assert rel(e0g, e0c) < 1e-6
    sim.run(1000)
    md.run(1000)
    m1 = md.measure()
    dg = (sim.measure_now().extended_energy() - e0g) / abs(e0g)
    dc = (m1.kinetic + m1.potential + m1.thermostat_energy - e0c) / abs(e0c)
    assert abs(dg) <= 2.0 * abs(dc) + 2e-5, (dg, dc)


def test_temperature_settles_and_follows_set_temperature(gpu):
    p, L = liquid(gpu)
    sim = make(gpu, p, L, temperature=1.0, period=0.5)
    dof = 3 * 1000 - 3

    def mean_t(steps, every=20):
        ts = []
        for _ in range(steps // every):
            sim.run(every)
            ts.append(2.0 * sim.measure_now().kinetic / dof)
        return float(np.mean(ts))

    sim.run(1000)
    assert abs(mean_t(3000) - 1.0) < 0.03
    sim.set_temperature(1.4)
    assert sim.target_temperature() == 1.4
    sim.run(2000)
    assert abs(mean_t(3000) - 1.4) < 0.04


def test_graphs_and_direct_launches_agree(gpu):
    p, L = liquid(gpu)
    a = make(gpu, p, L)
    b = make(gpu, p, L)
    b.set_graphs(False)
    before = a.kernels_executed()
    a.run(48)
    executed = a.kernels_executed() - before
    b.run(48)
    ma, mb = a.measure_now(), b.measure_now()
    assert (ma.kinetic, ma.potential, ma.thermostat_energy) == \
        (mb.kinetic, mb.potential, mb.thermostat_energy)
    qa, qb = a.read_particles(), b.read_particles()
    assert np.array_equal(qa["pos"], qb["pos"]) and np.array_equal(qa["vel"], qb["vel"])
    # nh_begin, decide and nh_force every step, plus 6 per rebuild
    assert executed >= 3 * 48 and (executed - 3 * 48) % 6 == 0
