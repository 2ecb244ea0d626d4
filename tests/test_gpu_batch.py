"""Batched replicas on the CUDA path.

The batch steps many boxes in one arena with one launch per kernel per step;
each replica must follow the single-box method exactly, so the checks are:
every replica's measurement and particles bit-for-bit equal to a single-box
simulation of it (which the other GPU tests tie to the oracle), energies of
every replica within 1e-6 of the oracle's f64 all-pairs sums, and boxes only
two cells wide (which the single-box path refuses, as the reference does)
against the same f64 sums.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs((a - b) / b)


def small_set(vl):
    """Six replicas from the uneven-replica generator, at small N (every side
    at least three cells, so each also runs as a single box)."""
    return vl.uneven_replicas(count=6, seed=80, sizes=(300, 3000))


def measure_fields(m):
    return np.array([m.kinetic, m.potential, m.virial, *m.momentum, m.condensed,
                     m.list_rebuilds, m.list_overflow, m.count, m.volume])


def test_replicas_match_single_boxes_bit_for_bit(gpu):
    reps = small_set(gpu)
    batch = gpu.Batch(reps, cutoff=2.5, skin=0.3, dt=0.004)
    batch.run(300)
    got = batch.measure()
    for r, rep in enumerate(reps):
        s = gpu.Settings(rep.box_size, cutoff=2.5, dt=0.004, thermostat=rep.thermostat, skin=0.3)
        single = gpu.LennardJones(rep.particles, s)
        single.run(300)
        want = single.measure_now()
        assert np.array_equal(measure_fields(got[r]), measure_fields(want)), r
        a, b = batch.read_particles(r), single.read_particles()
        assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"]), r
        assert batch.box_size(r) == single.box_size()


def test_replica_energies_match_f64(gpu, O):
    # on the starting lattices, and after they melted
    reps = small_set(gpu)
    batch = gpu.Batch(reps, cutoff=2.5, skin=0.3, dt=0.004)
    for steps in (0, 200):
        batch.run(steps)
        ms = batch.measure()
        for r, rep in enumerate(reps):
            box = np.array(batch.box_size(r))
            p = batch.read_particles(r) if steps else rep.particles
            pe, w = O.all_pairs(np.mod(p["pos"], box), box, 2.5, False)
            assert rel(ms[r].potential, pe) < 1e-6, (steps, r, ms[r].potential, pe)
            assert rel(ms[r].virial, w.sum()) < 1e-6, (steps, r, ms[r].virial, w.sum())
            ke = 0.5 * (p["vel"] ** 2).sum()
            assert rel(ms[r].kinetic, ke) < 1e-9
            assert ms[r].count == len(rep.particles) and ms[r].list_overflow == 0


@pytest.mark.parametrize("shifted_force", [False, True])
def test_two_cell_boxes_match_f64(gpu, O, shifted_force):
    # sides 6.0 and 7.5 give two cells of 2.8 on some axes: the list build
    # visits each distinct neighbour cell once
    reps = []
    for k, side in enumerate([[6.0, 6.0, 6.0], [7.5, 9.0, 6.5], [6.2, 12.0, 8.5]]):
        n = int(0.8 * side[0] * side[1] * side[2])
        p = gpu.lattice_box(n, side, 1.0, 5 + k)
        reps.append(gpu.Replica(p, side, gpu.Langevin(1.0, 1.0, 9 + k)))
    batch = gpu.Batch(reps, cutoff=2.5, skin=0.3, dt=0.004, shifted_force=shifted_force)
    for step in range(3):
        ms = batch.measure()
        for r in range(len(reps)):
            box = np.array(batch.box_size(r))
            p = batch.read_particles(r)
            pe, w = O.all_pairs(np.mod(p["pos"], box), box, 2.5, shifted_force)
            assert rel(ms[r].potential, pe) < 1e-6, (step, r, ms[r].potential, pe)
            assert rel(ms[r].virial, w.sum()) < 1e-6, (step, r)
            assert ms[r].list_overflow == 0
        batch.run(100)
    with pytest.raises(gpu.VljError, match="BOX_TOO_SMALL"):
        gpu.LennardJones(reps[0].particles, gpu.Settings(reps[0].box_size, cutoff=2.5, skin=0.3))


def test_batch_reruns_are_bit_identical(gpu):
    reps = small_set(gpu)

    def run():
        b = gpu.Batch(reps, cutoff=2.5, skin=0.3, dt=0.004)
        b.run(200)
        return [measure_fields(m) for m in b.measure()], b.read_particles(3)

    m1, p1 = run()
    m2, p2 = run()
    assert all(np.array_equal(a, b) for a, b in zip(m1, m2))
    assert np.array_equal(p1["pos"], p2["pos"]) and np.array_equal(p1["vel"], p2["vel"])


def test_batch_graphs_and_kernel_count(gpu):
    reps = small_set(gpu)
    b = gpu.Batch(reps, cutoff=2.5, skin=0.3, dt=0.004)
    b.run(64)
    before = b.kernels_executed()
    b.run(32)
    after = b.kernels_executed()
    rebuilds = sum(m.list_rebuilds for m in b.measure())
    # a step kernel every step, a decide per 16-step graph, plus 6 per step on
    # which some box rebuilt
    executed = after - before
    assert executed >= 32 + 2 and (executed - 32 - 2) % 6 == 0
    assert rebuilds > 0
    # direct launches give the same trajectory
    c = gpu.Batch(reps, cutoff=2.5, skin=0.3, dt=0.004)
    c.set_graphs(False)
    c.run(96)
    assert all(np.array_equal(measure_fields(x), measure_fields(y))
               for x, y in zip(b.measure(), c.measure()))


def test_batch_errors(gpu):
    p = gpu.lattice(100, 4.0, 1.0, 1)
    with pytest.raises(gpu.VljError, match="BOX_TOO_SMALL"):
        gpu.Batch([gpu.Replica(p, [4.0] * 3)])
    q = gpu.lattice(500, 9.0, 1.0, 1)
    with pytest.raises(gpu.VljError, match="NOT_ENABLED"):
        gpu.Batch([gpu.Replica(q, [9.0] * 3, gpu.NoseHoover(1.0, 0.5))])
    with pytest.raises(gpu.VljError, match="INVALID_ARG"):
        gpu.Batch([])


def test_step_block_size_keeps_the_trajectory(gpu):
    # the tuner's block-size knob changes how particles are grouped, not what
    # they compute: the same replicas step to the same bits with 64, 128 and
    # 256 particles per block (and a single box the same)
    reps = gpu.uneven_replicas(12, 77, (500, 4000), (0.05, 0.85), (0.8, 1.6), 1.0)
    out = []
    for threads in (64, 128, 256):
        b = gpu.Batch(reps, cutoff=2.5, skin=0.3, dt=0.004)
        b.set_step_threads(threads)
        b.run(60)
        ms = b.measure()
        out.append(([b.read_particles(r).tobytes() for r in range(len(reps))],
                     [(m.potential, m.virial, m.list_rebuilds) for m in ms]))
        b.close()
    assert out[0] == out[1] == out[2]
    p, L = gpu.lattice_fcc(8, 0.8442, 1.0, 3)
    st = gpu.Settings([L] * 3, dt=0.005, shifted_force=True, thermostat=gpu.Langevin(1.0, 1.0, 2))
    runs = []
    for threads in (64, 256):
        sim = gpu.LennardJones(p, st)
        sim.set_step_threads(threads)
        sim.run(50)
        runs.append(sim.read_particles().tobytes())
    assert runs[0] == runs[1]
