"""Heat exchange (eHEX/a) on the CUDA path (lennard_jones.wgsl:732-893).

Restates tests/heat.rs:159-214 (heat_exchange_moves_energy_and_keeps_momentum)
and checks a short trajectory with the exchange on against the oracle's f64
restatement (oracle/md.c hex_step).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 0.002


def liquid(gpu, size, t=1.0):
    count = int(round(0.8442 * size[0] * size[1] * size[2]))
    return gpu.lattice_box(count, size, t, 11)


def make(gpu, p, size, bins=0):
    s = gpu.Settings(size, cutoff=2.5, dt=DT, shifted_force=True, skin=0.3, profile_bins=bins)
    return gpu.LennardJones(p, s)


def test_short_trajectory_matches_f64_oracle(gpu, O):
    size = [9.0, 9.0, 24.0]
    p = liquid(gpu, size)
    sim = make(gpu, p, size)
    md = O.MD(p["pos"], p["vel"], sim.box_size(), dt=DT, shifted_force=True)
    sim.run(20)
    md.run(20)
    ex = gpu.HeatExchange(hot=(0.0, 3.0), cold=(12.0, 15.0), energy=0.05)
    sim.set_heat_exchange(ex)
    md.set_heat_exchange((0.0, 3.0), (12.0, 15.0), 0.05)
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
    assert abs((mg.kinetic - mc.kinetic) / mc.kinetic) < 1e-6
    # and back to constant energy without the exchange
    sim.set_heat_exchange(None)
    md.set_heat_exchange(None)
    assert sim.heat_flux() is None
    sim.run(20)
    md.run(20)
    q = sim.read_particles()
    pos, vel = md.read()
    d = q["pos"] - pos
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-5
    assert np.abs(q["vel"] - vel).max() < 1e-4


def drift(time, energy):
    t, e = np.asarray(time), np.asarray(energy)
    return np.polyfit(t, e, 1)[0]


def test_moves_energy_and_keeps_momentum(gpu):
    # tests/heat.rs:159-214
    size = [9.0, 9.0, 36.0]
    sim = make(gpu, liquid(gpu, size), size, bins=12)
    sim.run(2000)
    before = sim.measure_now()
    energy = 0.01
    sim.set_heat_exchange(gpu.HeatExchange(hot=(0.0, 3.0), cold=(18.0, 21.0), energy=energy))
    flux = sim.heat_flux()
    assert flux == pytest.approx(float(np.float32(energy)) / (2 * 81.0 * DT), rel=1e-12)
    time, total = [], []
    for _ in range(200):
        sim.run(100)
        sim.sample_profile_now()
        m = sim.measure_now()
        time.append(m.time)
        total.append(m.energy())
    after = sim.measure_now()
    rate = drift(time, total)
    duration = time[-1] - time[0]
    moved = energy / DT * duration
    assert abs(rate * duration) < 1e-3 * moved, (rate, moved)
    assert np.all(np.abs(np.array(after.momentum) - np.array(before.momentum))
                  < 1e-6 * after.count)
    t = sim.read_profile().temperature()
    assert t[0] > t[6] + 0.04, t


def test_kernel_count_and_graphs(gpu):
    size = [9.0, 9.0, 24.0]
    p = liquid(gpu, size)
    ex = gpu.HeatExchange(hot=(0.0, 3.0), cold=(12.0, 15.0), energy=0.05)
    a, b = make(gpu, p, size), make(gpu, p, size)
    b.set_graphs(False)
    a.set_heat_exchange(ex)
    b.set_heat_exchange(ex)
    before = a.kernels_executed()
    a.run(32)
    executed = a.kernels_executed() - before
    b.run(32)
    # begin, decide, force pass and apply pass every step, plus 6 per rebuild
    assert executed >= 4 * 32 and (executed - 4 * 32) % 6 == 0
    qa, qb = a.read_particles(), b.read_particles()
    assert np.array_equal(qa["pos"], qb["pos"]) and np.array_equal(qa["vel"], qb["vel"])


def test_exchange_needs_constant_energy(gpu):
    size = [9.0, 9.0, 24.0]
    p = liquid(gpu, size)
    s = gpu.Settings(size, dt=DT, thermostat=gpu.Langevin(1.0, 1.0, 3))
    sim = gpu.LennardJones(p, s)
    with pytest.raises(gpu.VljError, match="NOT_ENABLED"):
        sim.set_heat_exchange(gpu.HeatExchange(hot=(0.0, 3.0), cold=(12.0, 15.0), energy=0.05))
