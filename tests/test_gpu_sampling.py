"""Profiles along z and the heat current on the CUDA path.

Restates the reference's GPU tests tests/coexistence.rs:93-189
(rectangular_box_matches_all_pairs, profiles_add_up_to_the_whole_box) and
tests/heat.rs:54-135 (heat_current_matches_cpu), and adds slab-by-slab checks
against the oracle's f64 Irving-Kirkwood profile (oracle/pairs.c vo_profile).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MASK = (1 << 64) - 1


def jitter(pos, seed=99):
    """tests/coexistence.rs:81-88: xorshift jitter of +-0.15 per axis."""
    s = seed
    out = pos.copy()
    for i in range(len(out)):
        for k in range(3):
            s ^= (s << 13) & MASK
            s ^= s >> 7
            s ^= (s << 17) & MASK
            out[i, k] += ((s >> 11) / float(1 << 53) - 0.5) * 0.3
    return out


def make(vl, pos, vel, box, shifted_force=True, dt=0.005, thermostat=None, bins=0):
    s = vl.Settings(box, cutoff=2.5, dt=dt, thermostat=thermostat, shifted_force=shifted_force,
                    skin=0.3, profile_bins=bins)
    return vl.LennardJones(vl.particles(pos, vel), s)


def canonical(sim):
    """Positions wrapped into the box and the canonical velocities."""
    p = sim.read_particles()
    box = np.array(sim.box_size())
    return np.mod(p["pos"], box), p["vel"].copy(), box


def rel(a, b):
    return abs((a - b) / b)


@pytest.mark.parametrize("shifted_force", [False, True])
def test_rectangular_box_virial_tensor(gpu, O, shifted_force):
    # tests/coexistence.rs:93-130: whole-box W_aa of the profile against f64 pairs
    size = [9.0, 10.5, 14.25]
    pos, vel = O.lattice_box(1000, size, 1.0, 3)
    sim = make(gpu, jitter(pos), vel, size, shifted_force=shifted_force, bins=57)
    m = sim.measure_now()
    sim.sample_profile_now()
    prof = sim.read_profile()
    wp, v, box = canonical(sim)
    pe, w = O.all_pairs(wp, box, 2.5, shifted_force)
    assert prof.samples == 1
    assert rel(m.potential, pe) < 1e-6
    for a in range(3):
        assert rel(prof.virial[a], w[a]) < 2e-6, (a, prof.virial, w)


def _profile_run(vl, pos, vel, size):
    sim = make(vl, pos, vel, size, thermostat=vl.Langevin(0.7, 1.0, 5), bins=120)
    sim.run(200)
    m = sim.measure_now()
    sim.sample_profile_now()
    return sim, m, sim.read_profile()


def _bits(p):
    vals = []
    for s in p.slabs:
        vals += [s.particles, s.potential] + list(s.kinetic) + list(s.virial)
    vals += list(p.virial)
    return np.array(vals, dtype=np.float64).view(np.uint64)


def test_profiles_add_up_to_the_whole_box(gpu, O):
    # tests/coexistence.rs:132-189
    size = [10.0, 10.0, 30.0]
    pos, vel = O.lattice_box(2400, size, 1.0, 3)
    pos = jitter(pos)
    sim, m, p = _profile_run(gpu, pos, vel, size)
    _, _, p2 = _profile_run(gpu, pos, vel, size)
    assert np.array_equal(_bits(p), _bits(p2)), "profiles differ between runs"
    count = sum(s.particles for s in p.slabs)
    kinetic = sum(sum(s.kinetic) for s in p.slabs)
    potential = sum(s.potential for s in p.slabs)
    slab_virial = [sum(s.virial[a] for s in p.slabs) for a in range(3)]
    assert count == m.count == 2400
    assert rel(kinetic, 2.0 * m.kinetic) < 1e-6
    assert rel(potential, m.potential) < 1e-5
    assert rel(sum(p.virial), m.virial) < 1e-5
    for a in range(3):
        assert rel(slab_virial[a], p.virial[a]) < 1e-6


def test_profile_slabs_match_f64_oracle(gpu, O):
    # every slab of one sample against the oracle's f64 Irving-Kirkwood profile
    size = [10.0, 10.0, 30.0]
    bins = 60
    pos, vel = O.lattice_box(2400, size, 1.0, 3)
    sim = make(gpu, jitter(pos), vel, size, thermostat=gpu.Langevin(0.7, 1.0, 5), bins=bins)
    sim.run(100)
    sim.sample_profile_now()
    p = sim.read_profile()
    wp, v, box = canonical(sim)
    ref = O.profile(wp, v, box, 2.5, True, bins).reshape(-1)
    got = np.array([[s.particles] + list(s.kinetic) + list(s.virial) + [s.potential]
                    for s in p.slabs]).reshape(-1)
    want = ref[: bins * 8].reshape(bins, 8)
    got = got.reshape(bins, 8)
    # counts are exact; the rest is f32 pair arithmetic against f64
    assert np.array_equal(got[:, 0], want[:, 0])
    scale = [1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
    for c in range(1, 8):
        scale[c] = np.abs(want[:, c]).max()
        err = np.abs(got[:, c] - want[:, c]).max() / scale[c]
        assert err < 1e-5, (c, err)
    assert np.allclose(p.virial, ref[bins * 8:], rtol=2e-6)
    # slab centres
    width = box[2] / bins
    assert np.allclose([s.z for s in p.slabs], (np.arange(bins) + 0.5) * width)


def test_profile_averages_over_samples_and_clears(gpu, O):
    size = [10.0, 10.0, 30.0]
    pos, vel = O.lattice_box(2400, size, 1.0, 3)
    sim = make(gpu, jitter(pos), vel, size, bins=30)
    sim.sample_profile_now()
    one = sim.read_profile()
    sim.sample_profile_now()  # same state: the average is unchanged
    two = sim.read_profile()
    assert two.samples == 2
    assert np.array_equal(_bits(one), _bits(two))
    sim.clear_profile()
    cleared = sim.read_profile()
    assert cleared.samples == 0
    assert all(s.particles == 0.0 and s.potential == 0.0 for s in cleared.slabs)


def test_heat_current_matches_f64(gpu, O):
    # tests/heat.rs:98-135 (Langevin-free, shifted force, dt 0.002)
    size = [9.0, 9.0, 12.0]
    count = int(round(0.8442 * 9 * 9 * 12))
    pos, vel = O.lattice_box(count, size, 1.0, 11)
    sim = make(gpu, pos, vel, size, dt=0.002)
    sim.run(500)
    sim.record_heat_current(2)
    sim.sample_heat_current()
    j = sim.read_heat_current()
    assert j.shape == (1, 3)
    wp, v, box = canonical(sim)
    ref = O.heat_current(wp, v, box, 2.5, True)
    # terms of order one per particle with both signs: compare against the size
    # of the sum of their magnitudes, as the reference does, but 10x tighter
    scale = np.sqrt(count) * 10.0
    err = np.abs(j[0] - ref).max()
    print("heat current", j[0], ref, "error", err, "of scale", scale)
    assert err < 1e-5 * scale, (j[0], ref)
    # a second sample of the same state adds the same current
    sim.sample_heat_current()
    j2 = sim.read_heat_current()
    assert j2.shape == (2, 3) and np.array_equal(j2[0], j2[1])
    with pytest.raises(gpu.VljError, match="full"):
        sim.sample_heat_current()
    sim.record_heat_current(4)
    assert sim.read_heat_current().shape == (0, 3)


@pytest.mark.parametrize("shifted_force", [False, True])
def test_heat_current_taken_by_the_next_step(gpu, O, shifted_force):
    # A sample requested between steps is taken by the next step's force pass
    # (the state it starts from); before anything else reads the series or
    # changes the state, by the sampling kernel. Both give the f64 current.
    size = [9.0, 9.0, 12.0]
    count = int(round(0.8442 * 9 * 9 * 12))
    pos, vel = O.lattice_box(count, size, 1.0, 11)
    fused = make(gpu, pos, vel, size, shifted_force=shifted_force, dt=0.002)
    alone = make(gpu, pos, vel, size, shifted_force=shifted_force, dt=0.002)
    direct = make(gpu, pos, vel, size, shifted_force=shifted_force, dt=0.002)
    direct.set_graphs(False)
    scale = np.sqrt(count) * 10.0
    refs = []
    for sim in (fused, alone, direct):
        sim.run(300)
        sim.record_heat_current(24)
    for k in range(24):
        if k % 8 == 0:
            wp, v, box = canonical(fused)
            refs.append((k, O.heat_current(wp, v, box, 2.5, shifted_force)))
        for sim in (fused, alone, direct):
            sim.sample_heat_current()
        alone.read_heat_current()  # takes its sample now, with the sampling kernel
        for sim in (fused, alone, direct):
            sim.step(1)
    jf, ja, jd = fused.read_heat_current(), alone.read_heat_current(), direct.read_heat_current()
    assert jf.shape == ja.shape == (24, 3)
    assert np.array_equal(jf, jd)  # captured and direct steps: the same kernel
    assert np.abs(jf - ja).max() < 1e-5 * scale, np.abs(jf - ja).max()
    for k, ref in refs:
        assert np.abs(jf[k] - ref).max() < 1e-5 * scale, (k, jf[k], ref)
    # taking the sample changes nothing in the trajectory
    qf, qa = fused.read_particles(), alone.read_particles()
    assert np.array_equal(qf["pos"], qa["pos"]) and np.array_equal(qf["vel"], qa["vel"])
    # a sample pending when the state is overwritten is taken first
    fused.record_heat_current(2)
    fused.sample_heat_current()
    wp, v, box = canonical(fused)
    ref = O.heat_current(wp, v, box, 2.5, shifted_force)
    fused.write_particles(fused.read_particles())
    j = fused.read_heat_current()
    assert j.shape == (1, 3) and np.abs(j[0] - ref).max() < 1e-5 * scale


def test_sampling_errors(gpu, O):
    pos, vel = O.lattice(1000, 11.0, 1.0, 3)
    sim = make(gpu, pos, vel, [11.0] * 3)
    with pytest.raises(gpu.VljError, match="profile_bins"):
        sim.sample_profile_now()
    with pytest.raises(gpu.VljError, match="record_heat_current"):
        sim.sample_heat_current()
    sim.clear_profile()  # nothing to clear: fine


@pytest.mark.parametrize("drawn", ["NEIGHBOURS", "TEMPERATURE"])
def test_drawn_values(gpu, O, drawn):
    # lennard_jones.wgsl:595-602: neighbours within 1.5 sigma, or the local
    # temperature over the particle and its neighbours within the cutoff
    pos, vel = O.lattice(1000, 11.0, 1.0, 3)
    sim = make(gpu, jitter(pos), vel, [11.0] * 3, shifted_force=False)
    sim.run(50)
    sim.set_drawn(getattr(gpu.Drawn, drawn))
    sim.measure_now()
    got = sim.read_vel4()
    wp, v, box = canonical(sim)
    d = wp[None, :, :] - wp[:, None, :]
    d -= box * np.round(d / box)
    r2 = (d ** 2).sum(-1)
    np.fill_diagonal(r2, np.inf)
    assert np.allclose(got[:, :3], v, rtol=1e-6, atol=1e-6)
    if drawn == "NEIGHBOURS":
        assert np.array_equal(got[:, 3], (r2 < 2.25).sum(1).astype(np.float32))
    else:
        near = r2 < 6.25
        v2 = (v ** 2).sum(1)
        want = (v2 + (near * v2[None, :]).sum(1)) / (3.0 * (near.sum(1) + 1))
        assert np.allclose(got[:, 3], want, rtol=2e-5)
