"""The reference's own known-answer tests, run against the CPU oracle:
crates/virial-precision/src/fixed.rs:73-113, df64.rs:133-177, and the Philox
published test vectors (Salmon et al., Random123)."""

import math

import numpy as np
import pytest

ONE = 4294967296.0


def xorshift(seed):
    s = seed
    mask = (1 << 64) - 1
    while True:
        s ^= (s << 13) & mask
        s ^= s >> 7
        s ^= (s << 17) & mask
        yield s


def test_fixed_round_trips(O):
    # fixed.rs:73-80
    for x in [0.0, 1.0, -1.0, 0.5, -0.5, 1234.5678, -98765.43, 0.0625, -3.0e5]:
        assert O.fixed_to_raw(x) / ONE == float(np.float32(x))


def test_fixed_rounds_finer_bits_to_nearest_step(O):
    # fixed.rs:82-88
    for x in [1e-3, -1e-3, 1e-12, -7.25e-9, 3.3e-6]:
        assert abs(O.fixed_to_raw(x) / ONE - float(np.float32(x))) <= 0.5 / ONE


def test_fixed_exact_rounding_across_magnitudes(O):
    # fixed.rs:90-103: 200,000 xorshift values from 2^-34 to 2^30, seed 12345.
    # Also checks that RNE(x * 2^32) in f64 (the CUDA path's conversion)
    # equals the reference's integer split for every value.
    g = xorshift(12345)
    for _ in range(200_000):
        seed = next(g)
        magnitude = 2.0 ** ((seed >> 11) / float(1 << 53) * 64.0 - 34.0)
        x = float(np.float32(magnitude if seed & 1 == 0 else -magnitude))
        exact = round(x * ONE)  # Python's round is ties-to-even, exact for these
        assert O.fixed_to_raw(x) == exact
        assert O.fixed_raw_f64(x) == exact


def test_fixed_sums_exact_in_any_order(O):
    # fixed.rs:105-113
    values = [float(np.float32(((i * 7919) % 1000) * 0.37 - 150.0)) for i in range(1000)]
    fwd = sum(O.fixed_to_raw(x) for x in values)
    bwd = sum(O.fixed_to_raw(x) for x in reversed(values))
    assert fwd == bwd


def test_fixed_split_words(O):
    # two's complement words, high word signed (fixed.wgsl:50-54)
    assert O.fixed_split(1.0) == (0, 1)
    assert O.fixed_split(-1.0) == (0, 0xFFFFFFFF)
    assert O.fixed_split(0.5) == (0x80000000, 0)
    assert O.fixed_split(-0.5) == (0x80000000, 0xFFFFFFFF)
    assert O.fixed_split(1e-20) == (0, 0)


def test_df64_accurate_to_about_14_digits(O):
    # df64.rs:141-177: 20,000 pairs from xorshift seed 0x9e3779b9
    g = xorshift(0x9E3779B9)
    nxt = lambda: (next(g) >> 11) / float(1 << 53)
    worst = [0.0] * 4
    for _ in range(20_000):
        a = (nxt() - 0.5) * 10.0 ** (nxt() * 8.0 - 4.0)
        b = (nxt() - 0.5) * 10.0 ** (nxt() * 8.0 - 4.0)
        da, db = O.df(a), O.df(b)
        x, y = O.df_value(da), O.df_value(db)
        rel = lambda p, q: abs((p - q) / q)
        scale = max(abs(x), abs(y))
        worst[0] = max(worst[0], abs(O.df_value(O.df_op("add", da, db)) - (x + y)) / scale)
        worst[1] = max(worst[1], rel(O.df_value(O.df_op("mul", da, db)), x * y))
        worst[2] = max(worst[2], rel(O.df_value(O.df_op("div", da, db)), x / y))
        sq = rel(max(abs(O.df_value(O.df_op("sqrt", da))), 1e-300), math.sqrt(abs(x)))
        sq = min(sq, rel(O.df_value(O.df_op("sqrt", O.df(abs(x)))), math.sqrt(abs(x))))
        worst[3] = max(worst[3], sq)
    for name, err in zip(["add", "mul", "div", "sqrt"], worst):
        assert err < 1e-13, (name, err)


def test_philox_known_answers(O):
    # Random123's published Philox-4x32-10 known-answer vectors
    assert [int(v) for v in O.philox([0, 0, 0, 0], [0, 0])] == \
        [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert [int(v) for v in O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == \
        [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert [int(v) for v in O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                     [0xA4093822, 0x299F31D0])] == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_langevin_noise_is_gaussian(O):
    g = np.array([O.langevin_noise(7, s, i) for s in range(40) for i in range(500)]).ravel()
    assert abs(g.mean()) < 0.02 and abs(g.std() - 1.0) < 0.02
    # distinct per step, per particle and per seed
    assert not np.array_equal(O.langevin_noise(7, 0, 1), O.langevin_noise(7, 1, 1))
    assert not np.array_equal(O.langevin_noise(7, 0, 1), O.langevin_noise(7, 0, 2))
    assert not np.array_equal(O.langevin_noise(7, 0, 1), O.langevin_noise(8, 0, 1))


def test_pack_round_trip(O):
    # packed lo keeps ~9 bits below the hi part's last bit (lennard_jones.wgsl:128-152)
    rng = np.random.default_rng(3)
    for x in rng.uniform(0, 70, size=(200, 3)):
        hi = x.astype(np.float32)
        lo = (x - hi.astype(np.float64)).astype(np.float32)
        bits = O.pack_lo(hi, lo)
        back = O.unpack_lo(hi, bits)
        for k in range(3):
            assert abs(float(back[k]) - float(lo[k])) <= O.last_bit(float(hi[k])) / 510.0 * 0.51


def second_virial(t, cutoff):
    """tests/thermodynamics.rs:216-232: B2 of the cut-and-shifted potential."""
    def potential(r2, rc2):
        if r2 >= rc2:
            return 0.0
        lj = lambda q: 4.0 * ((1 / q ** 3) ** 2 - 1 / q ** 3)
        return lj(r2) - lj(rc2)
    steps = 200_000
    h = cutoff / steps
    r = np.arange(steps + 1) * h
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        s6 = np.where(r > 0, 1.0 / np.where(r > 0, r, 1.0) ** 6, 0.0)
        u = 4.0 * (s6 * s6 - s6) - 4.0 * (cutoff ** -12 - cutoff ** -6)
        f = np.where(r > 0, (np.exp(-u / t) - 1.0) * r * r, 0.0)
    f[-1] = (math.exp(-potential(cutoff * cutoff, cutoff * cutoff) / t) - 1.0) * cutoff ** 2
    w = np.where(np.arange(steps + 1) % 2 == 1, 4.0, 2.0)
    w[0] = w[-1] = 1.0
    return -2.0 * math.pi * float((f * w).sum()) * h / 3.0


def test_second_virial_coefficient():
    # the dilute-gas reference value: 1 + B2 rho = 0.99228 at rho 0.01, T 2
    # (docs/VALIDATION.md:45 quotes the reference's measurement against it)
    b2 = second_virial(2.0, 2.5)
    assert abs(1.0 + b2 * 0.01 - 0.99228) < 2e-5


def test_double_float_path_meets_the_reference_bound(O):
    # The reference's own arithmetic (dfpath.c) on the small plain workload:
    # PE and virial within the 1e-5 its tests allow against f64 pairs
    # (tests/thermodynamics.rs:93-97); over 100 constant-energy steps its
    # energy moves as the f64 engine's does (the change from the lattice start
    # is the integrator's, not the arithmetic's).
    L = (1000 / 0.8442) ** (1.0 / 3.0)
    pos, vel = O.lattice(1000, L, 0.72, 1)
    box = np.array([float(np.float32(L))] * 3)
    md = O.DoubleFloatMD(pos, vel, box, 2.5, 0.005, False)
    ke, pe, w, p, _ = md.measure()
    pe64, w64 = O.all_pairs(np.mod(p, box), box, 2.5, False)
    assert abs((pe - pe64) / pe64) < 1e-5 and abs((w - w64.sum()) / w64.sum()) < 1e-5
    md.run(100)
    ke1, pe1, _, _, _ = md.measure()
    f64 = O.MD(pos, vel, box, cutoff=2.5, skin=0.3, dt=0.005)
    m0 = f64.measure()
    f64.run(100)
    m1 = f64.measure()
    e0 = m0.kinetic + m0.potential
    change = ((ke1 + pe1) - (ke + pe)) / abs(ke + pe)
    change64 = ((m1.kinetic + m1.potential) - e0) / abs(e0)
    assert abs(change - change64) < 1e-5, (change, change64)
    with pytest.raises(ValueError):
        O.DoubleFloatMD(pos, vel, [7.0, 7.0, 7.0], 2.5, 0.005, False)


@pytest.mark.parametrize("shifted_force", [False, True])
def test_double_float_path_in_the_liquid(O, shifted_force):
    # after 200 steps from the lattice (a liquid): the reference's arithmetic
    # stays within its own 1e-5 of the f64 pair sums in both cutoff styles
    L = (1000 / 0.8442) ** (1.0 / 3.0)
    pos, vel = O.lattice(1000, L, 0.72, 1)
    box = np.array([float(np.float32(L))] * 3)
    md = O.DoubleFloatMD(pos, vel, box, 2.5, 0.005, shifted_force)
    md.run(200)
    ke, pe, w, p, v = md.measure()
    pe64, w64 = O.all_pairs(np.mod(p, box), box, 2.5, shifted_force)
    assert abs((pe - pe64) / pe64) < 1e-5 and abs((w - w64.sum()) / w64.sum()) < 1e-5
    assert abs(ke - 0.5 * np.sum(v * v)) < 1e-9 * ke


def test_grain_oracle_block_and_symmetry(O):
    # granular.rs:634-665: floor((hi - lo) / spacing) grains per axis, radii
    # within r (1 +- spread), none overlapping at spacing 2 r (1 + spread) 1.02
    pos, radius = O.grain_block([0.004, 0.004, 0.004], [0.03, 0.03, 0.02], 0.0015, 0.1, 7)
    spacing = 2 * 0.0015 * 1.1 * 1.02
    assert len(pos) == int(0.026 // spacing) ** 2 * int(0.016 // spacing)
    assert radius.min() >= 0.0015 * 0.9 and radius.max() <= 0.0015 * 1.1
    _, counts = O.grain_contacts(pos, radius, 0.05, 16, 16)
    assert counts.max() == 0
    # grown radii: the contact test is symmetric, so the partner relation is
    partners, counts = O.grain_contacts(pos, radius * 1.12, 0.05, 16, 16)
    assert counts.sum() > 0
    pairs = {(i, int(j)) for i in range(len(pos)) for j in partners[i, :counts[i]]}
    assert all((j, i) in pairs for i, j in pairs)
