"""The Langevin branch of the CUDA step against the oracle.

The 256,000-atom workload runs the BAOAB Langevin step (lennard_jones.wgsl:
225-276: half drift, friction and noise, half drift) with noise from a
counter-based Philox-4x32-10 stream keyed by (seed, step, particle id). These
tests pin that stream on the device -- Random123's published known answers,
then the oracle's restatement (oracle/precision.c vo_langevin_noise) for many
(seed, step, id) -- and then whole trajectories against the oracle's f64
engine with the same integrator and noise (oracle/md.c advance), on the
1000-atom box and on the 256,000-atom box.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LJV1 = 0x4C4A5631  # the stream's second key word


def test_device_philox_matches_random123_known_answers(gpu):
    ctr = [[0, 0, 0, 0], [0xFFFFFFFF] * 4, [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344]]
    key = [[0, 0], [0xFFFFFFFF] * 2, [0xA4093822, 0x299F31D0]]
    out, _ = gpu.philox(ctr, key)
    assert [[int(v) for v in row] for row in out] == [
        [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8],
        [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD],
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1],
    ]


def test_device_noise_matches_the_oracle(gpu, O):
    rng = np.random.default_rng(11)
    n = 4000
    ids = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    ids[:100] = np.arange(100)
    steps = rng.integers(0, 2 ** 40, n, dtype=np.uint64)
    steps[100:200] = np.arange(100)
    seeds = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    ctr = np.stack([ids, (steps & 0xFFFFFFFF).astype(np.uint32),
                    (steps >> 32).astype(np.uint32), np.zeros(n, np.uint32)], axis=1)
    key = np.stack([seeds, np.full(n, LJV1, np.uint32)], axis=1)
    words, noise = gpu.philox(ctr, key)
    want_words = np.array([O.philox(ctr[k], key[k]) for k in range(n)])
    assert np.array_equal(words, want_words)
    want = np.array([O.langevin_noise(int(seeds[k]), int(steps[k]), int(ids[k]))
                     for k in range(n)])
    # the same 24-bit uniforms; Box-Muller through CUDA's logf / sinf / cosf
    # against the host's, each within an ulp or two
    assert np.allclose(noise, want, rtol=4e-6, atol=1e-6), np.abs(noise - want).max()
    assert np.mean(noise == want) > 0.5


def _compare(q, pos, vel, box):
    d = q["pos"] - pos
    d -= box * np.round(d / box)
    return np.abs(d).max(), np.abs(q["vel"] - vel).max()


@pytest.mark.parametrize("shifted_force", [True, False])
def test_langevin_trajectory_matches_the_oracle_1000(gpu, O, shifted_force):
    # the 1000-atom box at rho 0.8442, Langevin T = 1, gamma = 1, seed 7
    L = (1000 / 0.8442) ** (1 / 3)
    p = gpu.lattice(1000, L, 1.0, 7)
    sim = gpu.LennardJones(p, gpu.Settings([L] * 3, dt=0.005, shifted_force=shifted_force,
                                           thermostat=gpu.Langevin(1.0, 1.0, 7)))
    box = np.array(sim.box_size())
    md = O.MD(p["pos"], p["vel"], box, dt=0.005, shifted_force=shifted_force,
              langevin=(1.0, 1.0, 7))
    for steps in (1, 9, 40):  # 1, 10 and 50 steps in all
        sim.run(steps)
        md.run(steps)
        dx, dv = _compare(sim.read_particles(), *md.read(), box)
        assert dx < 1e-5 and dv < 1e-4, (sim.steps(), dx, dv)
    m = sim.measure_now()
    mo = md.measure()
    assert abs(m.potential - mo.potential) < 1e-6 * abs(mo.potential)
    assert abs(m.kinetic - mo.kinetic) < 1e-5 * abs(mo.kinetic)
    md.close()


def test_langevin_trajectory_matches_the_oracle_256k(gpu, O):
    # the 256,000-atom workload: fcc 40^3 x 4 at rho 0.8442, force-shifted,
    # Langevin T = 1, gamma = 1, seed 7, dt 0.005
    p, L = gpu.lattice_fcc(40, 0.8442, 1.0, 7)
    sim = gpu.LennardJones(p, gpu.Settings([L] * 3, dt=0.005, shifted_force=True,
                                           thermostat=gpu.Langevin(1.0, 1.0, 7)))
    box = np.array(sim.box_size())
    md = O.MD(p["pos"], p["vel"], box, dt=0.005, shifted_force=True, langevin=(1.0, 1.0, 7))
    sim.run(20)
    md.run(20)
    dx, dv = _compare(sim.read_particles(), *md.read(), box)
    assert dx < 1e-5 and dv < 1e-4, (dx, dv)
    m = sim.measure_now()
    mo = md.measure()
    assert abs(m.potential - mo.potential) < 1e-6 * abs(mo.potential)
    assert abs(m.virial - mo.virial) < 1e-6 * abs(mo.virial)
    md.close()
