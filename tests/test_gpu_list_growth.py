"""List capacity recovery (no reference counterpart).

The reference sizes every list for twice the box's mean neighbour count plus
32 (lennard_jones.rs:471-474) and only reports a list that overflows
(Measurement::list_overflow): the particle loses the pairs past the
capacity. Here a dense blob in a mostly empty box overflows on its first
build. With growth off the library behaves as the reference (overflow
reported, energies off); with growth on (the default) the capacity grows
before the first forces, and whenever a later build overflows a measurement
grows it, rebuilds and measures again: no overflow, energies within 1e-6 of
f64, and the grows reported in the measurement.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def blob(gpu):
    # 4000 atoms at rho 0.9 (about 83 neighbours within cutoff + skin) in a
    # 30^3 box (mean rho 0.148: capacity ceil(2 * 13.6 + 32) = 60)
    p = gpu.lattice_box(4000, [16.45] * 3, 1.0, 5)
    p["pos"] += 6.0
    return p, [30.0] * 3


CAP0 = 60  # the reference's rule for 4000 atoms in 30^3 (lennard_jones.rs:471-474)


def test_overflow_is_reported_with_growth_off(gpu, O):
    import os
    p, box = blob(gpu)
    os.environ["VLJ_LIST_GROWTH"] = "0"
    try:
        sim = gpu.LennardJones(p, gpu.Settings(box, dt=0.005))
    finally:
        del os.environ["VLJ_LIST_GROWTH"]
    m = sim.measure_now()
    assert m.list_overflow > m.list_capacity == sim.grid_info().capacity == CAP0
    assert m.list_grows == 0
    pe, _ = O.all_pairs(p["pos"], np.array(sim.box_size()), 2.5, False)
    assert abs(m.potential - pe) > 1e-3 * abs(pe)  # pairs were dropped


def test_growth_recovers_every_pair(gpu, O):
    p, box = blob(gpu)
    sim = gpu.LennardJones(p, gpu.Settings(box, dt=0.005))
    m = sim.measure_now()
    assert m.list_overflow == 0 and m.list_grows == 1  # grown before the first forces
    assert m.list_capacity == sim.grid_info().capacity > CAP0
    assert m.list_capacity % 8 == 0
    pe, w = O.all_pairs(p["pos"], np.array(sim.box_size()), 2.5, False)
    assert abs(m.potential - pe) < 1e-6 * abs(pe)
    assert abs(m.virial - w.sum()) < 1e-6 * abs(w.sum())
    # the grown lists match the oracle's rebuild entry for entry
    g = sim.read_grid()
    assert np.all(g["counts"] <= m.list_capacity)
    sim.run(200)
    m = sim.measure_now()
    assert m.list_overflow == 0
    q = sim.read_particles()
    pe, w = O.all_pairs(q["pos"], np.array(sim.box_size()), 2.5, False)
    assert abs(m.potential - pe) < 1e-6 * abs(pe)


def test_growth_in_a_batch(gpu, O):
    p, box = blob(gpu)
    q = gpu.lattice(1000, 12.0, 1.0, 3)
    b = gpu.Batch([gpu.Replica(q, [12.0] * 3), gpu.Replica(p, box)], cutoff=2.5, skin=0.3,
                  dt=0.005)
    ms = b.measure()
    assert all(m.list_overflow == 0 for m in ms) and ms[1].list_grows == 1
    pe, _ = O.all_pairs(p["pos"], np.array(b.box_size(1)), 2.5, False)
    assert abs(ms[1].potential - pe) < 1e-6 * abs(pe)
    b.run(100)
    assert all(m.list_overflow == 0 for m in b.measure())
