"""Run-time choices of the step kernel's form on a single box: the cell
tiles' bricks per x-row (vlj_set_tile_cols), the particles per block and the
lanes per particle keep the trajectory to the bit, and virial_lj.tune_box
times them on a copy of the box and returns the fastest."""

import numpy as np
import pytest
from test_gpu_tiles import check_tile_lists

pytestmark = pytest.mark.gpu


def fcc_box(gpu, cells, seed):
    p, L = gpu.lattice_fcc(cells, 0.8442, 1.0, seed)
    st = gpu.Settings([L] * 3, dt=0.005, shifted_force=True,
                      thermostat=gpu.Langevin(1.0, 1.0, seed))
    return p, st


def test_tile_cols_at_run_time_keep_the_trajectory(gpu):
    p, st = fcc_box(gpu, 16, 3)
    ref = gpu.LennardJones(p, st)
    sim = gpu.LennardJones(p, st)
    assert sim.tile_info() == (0, 0, 0, 0)
    sim.set_tile_cols(3)
    cols, bricks, cap, threads = sim.tile_info()
    assert cols == 3 and bricks > 0 and cap > 0 and threads >= 64
    ref.run(60)
    sim.run(60)
    assert sim.measure_now().list_rebuilds >= 2
    assert sim.read_particles().tobytes() == ref.read_particles().tobytes()
    # the scheduled rebuilds since wrote the tile lists of these bricks
    check_tile_lists(sim)
    # another brick size mid-run, then back to the per-particle gathers
    sim.set_tile_cols(5)
    assert sim.tile_info()[0] == 5
    ref.run(40)
    sim.run(40)
    assert sim.read_particles().tobytes() == ref.read_particles().tobytes()
    check_tile_lists(sim)
    sim.set_tile_cols(0)
    assert sim.tile_info() == (0, 0, 0, 0)
    ref.run(40)
    sim.run(40)
    m, r = sim.measure_now(), ref.measure_now()
    assert sim.read_particles().tobytes() == ref.read_particles().tobytes()
    assert (m.potential, m.virial, m.list_rebuilds) == (r.potential, r.virial, r.list_rebuilds)
    ref.close()
    sim.close()


def test_tile_cols_refusals(gpu):
    p, st = fcc_box(gpu, 12, 2)
    sim = gpu.LennardJones(p, st)
    nx = sim.grid_info().cells[0]
    with pytest.raises(gpu.VljError):
        sim.set_tile_cols(nx + 1)
    sim.close()
    # a dilute box: under four particles per cell on average
    L = 30.0
    gas = gpu.LennardJones(gpu.lattice(1000, L, 1.0, 5), gpu.Settings([L] * 3, dt=0.005))
    with pytest.raises(gpu.VljError):
        gas.set_tile_cols(2)
    gas.set_tile_cols(0)
    gas.run(10)
    gas.close()


def test_tune_box_times_every_form(gpu):
    import torch

    p, st = fcc_box(gpu, 20, 4)
    cols, threads, times = gpu.tune_box(p, st, tile_cols=(0, 3, 4), threads=(64, 128),
                                        steps=5, warmup=3)
    assert set(times) == {(0, 64), (0, 128), (3, 128), (4, 128)}
    assert all(t > 0 for t in times.values())
    assert times[(cols, threads)] == min(times.values())
    torch.cuda.synchronize()
    # the choice applies to the box itself without changing its trajectory
    a = gpu.LennardJones(p, st)
    b = gpu.LennardJones(p, st)
    b.set_tile_cols(cols)
    b.set_step_threads(threads)
    a.run(30)
    b.run(30)
    assert a.read_particles().tobytes() == b.read_particles().tobytes()
    a.close()
    b.close()


def lanes_run(gpu, p, st, lanes, steps, heat_every=0):
    sim = gpu.LennardJones(p, st)
    sim.set_step_lanes(lanes)
    if heat_every:
        sim.record_heat_current(steps // heat_every + 1)
        for k in range(steps):
            sim.step(1)
            if k % heat_every == 0:
                sim.sample_heat_current()
    else:
        sim.run(steps)
    m = sim.measure_now()
    out = (sim.read_particles().tobytes(), m.potential, m.virial, m.kinetic, m.list_rebuilds,
           np.asarray(sim.read_heat_current()).tobytes() if heat_every else None)
    sim.close()
    return out


@pytest.mark.parametrize("case", ["lattice1000", "fcc20_langevin", "fcc40_langevin"])
def test_two_lanes_per_particle_keep_the_trajectory(gpu, case):
    # forces summed in two parts (even and odd list rows) in every kernel:
    # two lanes a particle and one give the same bits, on a small box (where
    # two lanes are the default), a mid-size and the 256k box
    if case == "lattice1000":
        L = (1000 / 0.8442) ** (1 / 3)
        p = gpu.lattice(1000, L, 0.72, 1)
        st = gpu.Settings([L] * 3, dt=0.005)
        steps = 300
    else:
        cells = 20 if case == "fcc20_langevin" else 40
        p, L = gpu.lattice_fcc(cells, 0.8442, 1.0, 5)
        st = gpu.Settings([L] * 3, dt=0.005, shifted_force=True,
                          thermostat=gpu.Langevin(1.0, 1.0, 5))
        steps = 100
    one = lanes_run(gpu, p, st, 1, steps)
    two = lanes_run(gpu, p, st, 2, steps)
    auto = lanes_run(gpu, p, st, 0, steps)
    assert one[4] >= 2  # rebuilds on the way
    assert one == two == auto


def test_two_lanes_beside_heat_current_samples(gpu):
    # steps that take a heat-current sample run the one-lane kernel, the
    # others two lanes: the same trajectory and series as one lane throughout
    p, L = gpu.lattice_fcc(12, 0.8442, 0.722, 5)
    st = gpu.Settings([L] * 3, dt=0.004)
    one = lanes_run(gpu, p, st, 1, 60, heat_every=3)
    two = lanes_run(gpu, p, st, 2, 60, heat_every=3)
    assert one == two
