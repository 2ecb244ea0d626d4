"""Edge cases on the CUDA path: a lone particle, a single pair, a box almost
all empty cells, lists that overflow their capacity (reported, as the
reference reports it in Measurement::list_overflow), and bad input."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs((a - b) / b)


def settings(gpu, L, **kw):
    return gpu.Settings([L] * 3, cutoff=2.5, dt=0.005, skin=0.3, **kw)


def test_one_particle_drifts_freely(gpu):
    p = gpu.particles([[1.0, 2.0, 3.0]], [[0.5, -0.25, 1.0]])
    sim = gpu.LennardJones(p, settings(gpu, 9.0))
    m = sim.measure_now()
    assert m.potential == 0.0 and m.virial == 0.0 and m.count == 1
    sim.run(400)  # 2 time units
    q = sim.read_particles()
    want = np.mod(np.array([1.0, 2.0, 3.0]) + 2.0 * np.array([0.5, -0.25, 1.0]),
                  float(np.float32(9.0)))
    assert np.allclose(q["pos"][0], want, atol=1e-12)
    assert np.array_equal(q["vel"][0], [0.5, -0.25, 1.0])


@pytest.mark.parametrize("shifted_force", [False, True])
def test_one_pair(gpu, O, shifted_force):
    p = gpu.particles([[4.0, 4.0, 4.0], [5.5, 4.0, 4.0]], [[0.0] * 3, [0.0] * 3])
    sim = gpu.LennardJones(p, settings(gpu, 9.0, shifted_force=shifted_force))
    m = sim.measure_now()
    pe, w = O.all_pairs(np.array([[4.0, 4.0, 4.0], [5.5, 4.0, 4.0]]), np.array([9.0] * 3), 2.5,
                        shifted_force)
    assert rel(m.potential, pe) < 1e-6 and rel(m.virial, w.sum()) < 1e-6
    sim.run(100)
    q = sim.read_particles()
    # equal and opposite: the pair's centre and momentum stay put
    assert np.allclose(q["pos"].mean(0), [4.75, 4.0, 4.0], atol=1e-9)
    assert np.allclose(q["vel"].sum(0), 0.0, atol=1e-9)


def test_mostly_empty_cells(gpu, O):
    # 100 particles in a box of 16 x 16 x 16 cells
    L = 46.0
    sim = gpu.LennardJones(gpu.lattice(100, L, 2.0, 4), settings(gpu, L))
    sim.run(2000)
    m = sim.measure_now()
    q = sim.read_particles()
    box = np.array(sim.box_size())
    pe, w = O.all_pairs(np.mod(q["pos"], box), box, 2.5, False)
    if pe != 0.0:
        assert rel(m.potential, pe) < 1e-6
    assert m.list_overflow == 0 and m.count == 100


def test_list_overflow_is_reported(gpu):
    # 216 particles packed 0.2 apart at a mean density of 0.125: far more
    # neighbours than the lists hold. With list growth off (the reference's
    # behaviour) the overflow is reported and nothing is written past the
    # lists; with it on (the default) the lists grow to hold all 215.
    import os
    g = np.arange(6) * 0.2 + 3.0
    pos = np.array([[x, y, z] for x in g for y in g for z in g])
    os.environ["VLJ_LIST_GROWTH"] = "0"
    try:
        sim = gpu.LennardJones(gpu.particles(pos), settings(gpu, 12.0))
    finally:
        del os.environ["VLJ_LIST_GROWTH"]
    cap = sim.grid_info().capacity
    m = sim.measure_now()
    assert m.list_overflow == 215 > cap and m.list_grows == 0
    sim = gpu.LennardJones(gpu.particles(pos), settings(gpu, 12.0))
    m = sim.measure_now()
    assert m.list_overflow == 0 and m.list_grows == 1
    assert m.list_capacity == sim.grid_info().capacity >= 215 > cap


def test_non_finite_input_is_refused(gpu):
    p = gpu.lattice(1000, 11.0, 1.0, 3)
    bad = p.copy()
    bad["vel"][17, 1] = np.nan
    with pytest.raises(gpu.VljError, match="INVALID_ARG"):
        gpu.LennardJones(bad, settings(gpu, 11.0))
    sim = gpu.LennardJones(p, settings(gpu, 11.0))
    bad["vel"][17, 1] = 0.0
    bad["pos"][3, 0] = np.inf
    with pytest.raises(gpu.VljError, match="INVALID_ARG"):
        sim.write_particles(bad)
    sim.write_particles(p)  # and a good write after a refused one
    m = sim.measure_now()
    assert m.count == 1000
    with pytest.raises(gpu.VljError, match="INVALID_ARG"):
        gpu.LennardJones(p[:0], settings(gpu, 11.0))
