"""The large constant-energy box of the heat-flux workload on the CUDA path:
16,384,000 atoms (fcc 160^3 x 4 at rho 0.8442), truncated-shifted cutoff 2.5,
skin 0.3, dt 0.004, the microscopic heat current sampled every step.

At this size the checks are the size-independent ones: potential energy and
virial against the oracle's f64 cell-list sums (within 1e-6), energy kept at
constant energy, zero total momentum kept, a finite heat-current series of one
sample per step, no list overflow.
"""

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def test_sixteen_million_atoms_with_heat_current_every_step(gpu, O):
    p, L = gpu.lattice_fcc(160, 0.8442, 0.722, 5)
    assert len(p) == 16_384_000
    sim = gpu.LennardJones(p, gpu.Settings([L] * 3, cutoff=2.5, dt=0.004, skin=0.3))
    del p
    m0 = sim.measure_now()
    steps = 40
    sim.record_heat_current(steps)
    for _ in range(steps):
        sim.step(1)
        sim.sample_heat_current()
    j = sim.read_heat_current()
    m1 = sim.measure_now()
    assert j.shape == (steps, 3) and np.all(np.isfinite(j))
    assert m1.list_overflow == 0
    drift = (m1.energy() - m0.energy()) / abs(m0.energy())
    assert abs(drift) < 1e-5, drift
    assert np.all(np.abs(m1.momentum) < 1e-6 * m1.count)
    q = sim.read_particles()
    sim.close()
    box = np.array([float(np.float32(L))] * 3)
    pe, w = O.cell_pairs(np.mod(q["pos"], box), box, 2.5, False)
    assert abs((m1.potential - pe) / pe) < 1e-6, (m1.potential, pe)
    assert abs((m1.virial - w.sum()) / w.sum()) < 1e-6, (m1.virial, w.sum())
