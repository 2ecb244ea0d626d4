"""CUDA path against the CPU oracle on the same seeded inputs.

Restates the reference's GPU tests (crates/virial-particles/tests/
thermodynamics.rs, coexistence.rs) with tighter tolerances: potential energy
and virial within 1e-6 relative of the f64 sums (the reference asks 1e-5);
binning, per-cell order and Verlet lists bit-for-bit equal to the oracle's
restatement of the reference's f32 arithmetic; fixed-point totals exactly the
sum of the per-particle terms; reruns bit-identical.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "lj_golden.npz"))
TOL = 1e-6  # relative PE / virial error against f64


def rel(a, b):
    return abs((a - b) / b)


def make(vl, pos, vel, box, shifted_force=False, dt=0.002, thermostat=None, bins=0):
    s = vl.Settings(box, cutoff=2.5, dt=dt, thermostat=thermostat, shifted_force=shifted_force,
                    skin=0.3, profile_bins=bins)
    return vl.LennardJones(vl.particles(pos, vel), s)


def wrapped(pos, box):
    b = np.array([float(np.float32(x)) for x in box])
    return np.mod(pos, b), b


def test_cell_grid_finds_every_pair(gpu, O):
    # tests/thermodynamics.rs:55-98
    pos, vel = GOLDEN["jittered_cube"], GOLDEN["lattice_vel"]
    sim = make(gpu, pos, vel, [11.0] * 3)
    m = sim.measure_now()
    wp, b = wrapped(pos, [11.0] * 3)
    pe, w = O.all_pairs(wp, b, 2.5, False)
    assert rel(m.potential, pe) < TOL, (m.potential, pe)
    assert rel(m.virial, w.sum()) < TOL, (m.virial, w.sum())
    assert m.list_overflow == 0 and m.count == 1000
    ke = 0.5 * (vel ** 2).sum()
    assert rel(m.kinetic, ke) < 1e-9


@pytest.mark.parametrize("shifted_force", [False, True])
def test_rectangular_box_matches_all_pairs(gpu, O, shifted_force):
    # tests/coexistence.rs:93-130
    size = [9.0, 10.5, 14.25]
    pos, vel = GOLDEN["jittered_box"], GOLDEN["box_vel"]
    sim = make(gpu, pos, vel, size, shifted_force=shifted_force)
    m = sim.measure_now()
    wp, b = wrapped(pos, size)
    pe, w = O.all_pairs(wp, b, 2.5, shifted_force)
    assert rel(m.potential, pe) < TOL
    assert rel(m.virial, w.sum()) < TOL


def compare_rebuild(sim, O, pre, reorder, vel_stored=None, grown=False):
    """The sim's current grid and lists against the oracle's rebuild of `pre`
    (with `grown`, at the capacity the sim's lists grew to, not the
    reference's starting capacity)."""
    g = sim.grid_info()
    s = O.setup(np.zeros((sim.count(), 3)), sim.box_size(), 2.5, 0.3, False)
    if grown:
        assert g.capacity >= s.capacity
        s.capacity = g.capacity
    assert list(g.cells) == list(s.cells) and g.capacity == s.capacity
    r = O.rebuild_ref(s, pre["x"], pre["v"], pre["ids"], reorder)
    now = sim.read_grid()
    assert np.array_equal(now["ids"], r["ids"])
    assert np.array_equal(now["x"], r["x"])
    assert np.array_equal(now["cell_of_slot"], r["cell_of_slot"])
    assert np.array_equal(now["cell_start"], r["cell_start"])
    assert np.array_equal(now["sorted"], r["sorted"])
    assert np.array_equal(now["counts"], r["counts"])
    used = np.arange(g.capacity)[None, :] < r["counts"][:, None]
    assert np.array_equal(np.where(used, now["lists"], 0), np.where(used, r["lists"], 0))


def test_first_lists_match_reference_bit_for_bit(gpu, O):
    pos, vel = GOLDEN["jittered_cube"], GOLDEN["lattice_vel"]
    sim = make(gpu, pos, vel, [11.0] * 3)
    wp, _ = wrapped(pos, [11.0] * 3)
    pre = dict(x=wp, v=vel, ids=np.arange(1000, dtype=np.uint32))
    compare_rebuild(sim, O, pre, reorder=True)  # the first rebuild reorders


def test_later_rebuilds_match_reference_bit_for_bit(gpu, O):
    # a warm liquid so lists rebuild and particles change cells; both the
    # rebuilds that reorder (every fourth) and those that do not
    p = gpu.lattice_box(2000, [12.0, 12.0, 16.0], 2.0, 5)
    sim = gpu.LennardJones(p, gpu.Settings([12.0, 12.0, 16.0], dt=0.005))
    seen = set()
    for _ in range(6):
        sim.run(37)
        pre = sim.read_grid()
        before = sim.grid_info().rebuilds
        sim.force_rebuild()
        reorder = before % 4 == 0
        seen.add(reorder)
        compare_rebuild(sim, O, dict(x=pre["x"], v=pre["v"], ids=pre["ids"]), reorder)
    assert seen == {True, False}


# name: (atoms, box, lift of the lattice along z, box the lattice fills,
# temperature, steps before each compared rebuild)
LIST_CASES = {
    "dilute_gas_rho0.04": (3000, [42.0, 42.0, 42.0], 0.0, None, 2.0, 120),
    "dense_liquid_rho0.95": (4000, [16.15] * 3, 0.0, None, 1.5, 60),
    "elongated_box": (3000, [10.0, 10.0, 40.0], 0.0, None, 1.2, 80),
    "three_cells_a_side": (500, [8.5] * 3, 0.0, None, 1.0, 80),
    "liquid_vapour_slab": (16000, [20.0, 20.0, 150.0], 47.6, [20.0, 20.0, 54.8], 0.7, 60),
}


@pytest.mark.parametrize("case", sorted(LIST_CASES))
def test_lists_bit_exact_across_densities_and_shapes(gpu, O, case):
    # binning, per-cell order and lists after the box has moved (two forced
    # rebuilds, reordering or not as the schedule has it), against the
    # oracle (at the slab's grown capacity if its liquid overflowed the
    # reference's)
    n, box, lift, fill, t, steps = LIST_CASES[case]
    p = gpu.lattice_box(n, fill or box, t, 9)
    p["pos"][:, 2] += lift
    sim = gpu.LennardJones(p, gpu.Settings(box, dt=0.005, shifted_force=True,
                                           thermostat=gpu.Langevin(t, 1.0, 9)))
    for _ in range(2):
        sim.run(steps)
        pre = sim.read_grid()
        before = sim.grid_info().rebuilds
        sim.force_rebuild()
        reorder = before % 4 == 0
        compare_rebuild(sim, O, dict(x=pre["x"], v=pre["v"], ids=pre["ids"]), reorder,
                        grown=case == "liquid_vapour_slab")
    sim.close()


def test_fixed_point_totals_are_exact(gpu, O):
    pos, vel = GOLDEN["jittered_cube"], GOLDEN["lattice_vel"]
    sim = make(gpu, pos, vel, [11.0] * 3)
    sim.measure_now()
    pe, w, raw = sim.read_partials()
    es = O.setup(vel, [11.0] * 3, 2.5, 0.3, False).energy_scale
    to_raw = lambda a: int(np.rint(a.astype(np.float64) * es * 2.0 ** 32).astype(np.int64).sum())
    assert raw[1] == to_raw(pe[:, 0]) + to_raw(pe[:, 1])
    assert raw[2] == to_raw(w[:, 0]) + to_raw(w[:, 1])


def test_thermostatted_reruns_are_bit_identical(gpu):
    # tests/thermodynamics.rs:295-326
    p = gpu.lattice(2000, 16.0, 1.5, 11)
    st = gpu.Settings([16.0] * 3, dt=0.004, thermostat=gpu.Langevin(1.5, 0.5, 3))

    def run():
        sim = gpu.LennardJones(p, st)
        sim.run(300)
        m = sim.measure_now()
        return sim.read_particles(), m.potential, m.virial

    a, b = run(), run()
    assert a[0].tobytes() == b[0].tobytes()
    assert (a[1], a[2]) == (b[1], b[2])


def test_measurements_after_steps_match_f64(gpu, O):
    p = gpu.lattice_box(3000, [14.0, 14.0, 16.0], 1.2, 8)
    sim = gpu.LennardJones(p, gpu.Settings([14.0, 14.0, 16.0], dt=0.005, shifted_force=True,
                                           thermostat=gpu.Langevin(1.2, 1.0, 9)))
    sim.run(250)
    m = sim.measure_now()
    q = sim.read_particles()
    pe, w = O.all_pairs(q["pos"], np.array(sim.box_size()), 2.5, True)
    assert rel(m.potential, pe) < TOL and rel(m.virial, w.sum()) < TOL
    assert rel(m.kinetic, 0.5 * (q["vel"] ** 2).sum()) < 1e-9
    assert np.allclose(m.momentum, q["vel"].sum(0), atol=1e-6)


def test_nve_short_trajectory_matches_f64_oracle(gpu, O):
    # 1000 particles on the reference's simple cubic lattice at rho 0.8442
    L = (1000 / 0.8442) ** (1 / 3)
    p = gpu.lattice(1000, L, 0.72, 1)
    sim = gpu.LennardJones(p, gpu.Settings([L] * 3, dt=0.005))
    md = O.MD(p["pos"], p["vel"], sim.box_size(), dt=0.005)
    sim.run(20)
    md.run(20)
    q = sim.read_particles()
    pos, vel = md.read()
    d = q["pos"] - pos
    d -= np.array(sim.box_size()) * np.round(d / np.array(sim.box_size()))
    assert np.abs(d).max() < 1e-5
    assert np.abs(q["vel"] - vel).max() < 1e-4


def test_nve_energy_drift_no_worse_than_f64(gpu, O):
    L = (1000 / 0.8442) ** (1 / 3)
    p = gpu.lattice(1000, L, 0.72, 1)
    sim = gpu.LennardJones(p, gpu.Settings([L] * 3, dt=0.005))
    md = O.MD(p["pos"], p["vel"], sim.box_size(), dt=0.005)
    e0g = sim.measure_now().energy()
    m0 = md.measure()
    e0c = m0.kinetic + m0.potential
    assert rel(e0g, e0c) < 1e-6
    sim.run(1000)
    md.run(1000)
    m1 = md.measure()
    dg = (sim.measure_now().energy() - e0g) / abs(e0g)
    dc = (m1.kinetic + m1.potential - e0c) / abs(e0c)
    # the truncated-shifted force jumps at the cutoff, so both drift alike
    assert abs(dg) <= 2.0 * abs(dc) + 2e-5, (dg, dc)


def test_measure_ring_and_poll(gpu):
    p = gpu.lattice(1000, 11.0, 1.0, 3)
    sim = gpu.LennardJones(p, gpu.Settings([11.0] * 3))
    ok = []
    for _ in range(4):
        sim.step(5)
        ok.append(sim.measure())
    assert ok == [True, True, True, False]
    import time
    got = []
    for _ in range(200):
        got += sim.poll()
        if len(got) == 3:
            break
        time.sleep(0.01)
    assert [m.step for m in got] == [5, 10, 15]
    assert sim.measure()


def test_write_then_read_particles(gpu):
    p = gpu.lattice(1000, 11.0, 1.0, 3)
    sim = gpu.LennardJones(p, gpu.Settings([11.0] * 3))
    sim.run(10)
    q = gpu.lattice(1000, 11.0, 2.0, 4)
    sim.write_particles(q)
    back = sim.read_particles()
    assert np.allclose(back["pos"], np.mod(q["pos"], 11.0), atol=1e-12)
    assert np.allclose(back["vel"], q["vel"], atol=1e-12)


def test_errors_match_reference_panics(gpu):
    p = gpu.lattice(100, 8.0, 1.0, 3)
    with pytest.raises(gpu.VljError) as e:
        gpu.LennardJones(p, gpu.Settings([8.0] * 3))  # below 3 (rc + skin)
    assert e.value.status == "BOX_TOO_SMALL"
    sim = gpu.LennardJones(gpu.lattice(1000, 11.0, 1.0, 3), gpu.Settings([11.0] * 3))
    with pytest.raises(gpu.VljError) as e:
        sim.set_temperature(1.0)  # lennard_jones.rs:907
    assert e.value.status == "NOT_ENABLED"


@pytest.mark.parametrize("thermostat", ["nve", "langevin"])
def test_large_box_lists_and_energies(gpu, O, thermostat):
    # the 256,000-particle fcc box (40^3 x 4 at rho 0.8442), force-shifted
    p, L = gpu.lattice_fcc(40, 0.8442, 1.0, 7)
    t = gpu.Langevin(1.0, 1.0, 7) if thermostat == "langevin" else None
    sim = gpu.LennardJones(p, gpu.Settings([L] * 3, dt=0.005, shifted_force=True, thermostat=t))
    sim.run(30)
    pre = sim.read_grid()
    before = sim.grid_info().rebuilds
    sim.force_rebuild()
    compare_rebuild(sim, O, dict(x=pre["x"], v=pre["v"], ids=pre["ids"]), before % 4 == 0)
    m = sim.measure_now()
    q = sim.read_particles()
    pe, w = O.cell_pairs(q["pos"], np.array(sim.box_size()), 2.5, True)
    assert rel(m.potential, pe) < TOL, (m.potential, pe)
    assert rel(m.virial, w.sum()) < TOL, (m.virial, w.sum())
    assert m.list_overflow == 0


def test_graph_and_direct_launches_agree_bit_for_bit(gpu):
    p, L = gpu.lattice_fcc(10, 0.8442, 1.0, 3)
    st = gpu.Settings([L] * 3, dt=0.005, shifted_force=True, thermostat=gpu.Langevin(1.0, 1.0, 2))
    out = []
    for graphs in (True, False):
        sim = gpu.LennardJones(p, st)
        sim.set_graphs(graphs)
        sim.run(137)  # chunks of 16 plus single steps
        m = sim.measure_now()
        out.append((sim.read_particles().tobytes(), m.potential, m.virial, m.list_rebuilds))
    assert out[0] == out[1]


def test_kernel_counter_counts_skipped_rebuilds_out(gpu):
    p, L = gpu.lattice_fcc(10, 0.8442, 0.5, 3)
    sim = gpu.LennardJones(p, gpu.Settings([L] * 3, dt=0.002))
    sim.run(5)
    r0, k0 = sim.measure_now().list_rebuilds, sim.kernels_executed()
    sim.run(64)
    k1 = sim.kernels_executed()
    r1 = sim.measure_now().list_rebuilds
    # a step kernel per step, a decide per 16-step graph (the step kernels take
    # the later steps' decisions), six per rebuild
    assert k1 - k0 == 64 + 64 // 16 + 6 * (r1 - r0)


def test_grid_every_step_keeps_the_trajectory(gpu):
    # the 256k workload's wording rebuilds the cell grid on every step; the
    # reference bins only with the lists. Both give the same lists and the
    # same trajectory to the bit; the grid kernels run on every step.
    p, L = gpu.lattice_fcc(10, 0.8442, 1.0, 7)
    settings = gpu.Settings([L] * 3, dt=0.005, shifted_force=True,
                            thermostat=gpu.Langevin(1.0, 1.0, 7))
    plain, every = gpu.LennardJones(p, settings), gpu.LennardJones(p, settings)
    every.set_grid_every_step(True)
    direct = gpu.LennardJones(p, settings)
    direct.set_grid_every_step(True)
    direct.set_graphs(False)
    r0 = plain.measure_now().list_rebuilds
    every.measure_now()
    k_plain, k_every = plain.kernels_executed(), every.kernels_executed()
    for sim in (plain, every, direct):
        sim.run(200)
    k_plain, k_every = plain.kernels_executed() - k_plain, every.kernels_executed() - k_every
    # a step kernel per step, a decide per 16-step graph launch (12), one for
    # the first of the 8 one-step graphs (each of them takes the next one's
    # decision), six more per rebuild
    rebuilds, rest = divmod(k_plain - 200 - 13, 6)
    assert rest == 0 and rebuilds > 0
    ms = [sim.measure_now() for sim in (plain, every, direct)]
    assert ms[0].list_rebuilds - r0 >= rebuilds
    assert ms[0].list_rebuilds == ms[1].list_rebuilds == ms[2].list_rebuilds
    assert (ms[0].potential, ms[0].virial, ms[0].kinetic) == (ms[1].potential, ms[1].virial, ms[1].kinetic)
    assert (ms[0].potential, ms[0].virial) == (ms[2].potential, ms[2].virial)
    q = [sim.read_particles() for sim in (plain, every, direct)]
    for other in q[1:]:
        assert np.array_equal(q[0]["pos"], other["pos"]) and np.array_equal(q[0]["vel"], other["vel"])
    g0, g1 = plain.read_grid(), every.read_grid()
    assert np.array_equal(g0["counts"], g1["counts"]) and np.array_equal(g0["lists"], g1["lists"])
    # bin, scan, scatter and sort also on every step without a rebuild
    assert k_every - k_plain == 4 * (200 - rebuilds)


def test_single_steps_carry_their_decisions(gpu):
    # one-step graphs take the next step's rebuild decision in their step
    # kernel and skip their decide kernel while it stands; measurements,
    # forced rebuilds and chunks in between must leave the trajectory as
    # direct launches (a decide kernel every step) make it
    p, L = gpu.lattice_fcc(10, 0.8442, 1.5, 5)
    st = gpu.Settings([L] * 3, dt=0.005, shifted_force=True, thermostat=gpu.Langevin(1.5, 1.0, 4))
    out = []
    for graphs in (True, False):
        sim = gpu.LennardJones(p, st)
        sim.set_graphs(graphs)
        k0 = sim.kernels_executed()
        for k in range(120):
            sim.step(1)
            if k % 37 == 5:
                sim.measure_now()
            if k == 70:
                sim.force_rebuild()
            if k == 90:
                sim.step(16)
        m = sim.measure_now()
        out.append((sim.read_particles().tobytes(), m.potential, m.virial, m.list_rebuilds,
                    sim.kernels_executed() - k0))
    assert out[0][:4] == out[1][:4]
    assert out[0][3] > 10  # rebuilds on the way
    assert out[0][4] < out[1][4]  # the graphs launched fewer decide kernels
