"""The reference's output formats (crates/virial/src/data.rs, manifest.rs):
shortest exact numbers in measurements.csv, .npy snapshots, run.json."""

import json
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def data():
    from virial_lj import data
    return data


def test_numbers_round_trip_exactly(data):
    # data.rs:169-181
    for v in [0.1, -1.0 / 3.0, 6.02214076e23, 1e-300, -0.0, 12345.678901234567]:
        assert float(data.exact(v)).hex() == float(v).hex()
    rng = np.random.default_rng(12345)
    for v in np.concatenate([rng.standard_normal(2000) * 10.0 ** rng.integers(-320, 300, 2000),
                             rng.integers(-10**9, 10**9, 200).astype(float)]):
        assert float(data.exact(v)).hex() == float(v).hex()


def test_numbers_are_spelled_as_rust_debug_spells_them(data):
    # scientific below 1e-4 and from 1e16, no '+' and no leading zeros in
    # the exponent, no ".0" on a scientific mantissa; ".0" on whole decimals
    cases = [(0.1, "0.1"), (1.0, "1.0"), (-0.0, "-0.0"), (0.0, "0.0"), (1e-300, "1e-300"),
             (6.02214076e23, "6.02214076e23"), (1e-5, "1e-5"), (0.0001, "0.0001"),
             (9e-5, "9e-5"), (1e16, "1e16"), (1.5e16, "1.5e16"), (1e15, "1000000000000000.0"),
             (-2.5e-7, "-2.5e-7"), (12345.678901234567, "12345.678901234567"),
             (float("inf"), "inf"), (float("-inf"), "-inf"), (float("nan"), "NaN")]
    for v, text in cases:
        assert data.exact(v) == text, (v, data.exact(v))


def test_npy_header_is_aligned_and_sized(data, tmp_path):
    # data.rs:183-193
    b = data.npy([3, 2], [1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    assert b[:8] == b"\x93NUMPY\x01\x00"
    header_len = int.from_bytes(b[8:10], "little")
    assert (10 + header_len) % 64 == 0
    assert len(b) == 10 + header_len + 6 * 8
    header = b[10:10 + header_len].decode()
    assert "'shape': (3, 2)" in header and header.endswith("\n")
    assert "'shape': (4,)" in data.npy([4], [0.0] * 4)[10:80].decode()
    path = tmp_path / "a.npy"
    path.write_bytes(b)
    assert np.array_equal(np.load(path), np.arange(1.0, 7.0).reshape(3, 2))
    with pytest.raises(ValueError):
        data.npy([4], [1.0])


def test_fnv1a(data):
    # the published FNV-1a 64-bit test vectors
    assert data.fnv1a(b"") == 0xCBF29CE484222325
    assert data.fnv1a(b"a") == 0xAF63DC4C8601EC8C
    assert data.fnv1a(b"foobar") == 0x85944171F73967E8


def test_data_log_writes_csv_npy_and_run_json(data, tmp_path):
    log = data.DataLog(str(tmp_path / "run"))
    assert log.is_recording()
    log.row([("step", 0), ("potential", -1.0 / 3.0), ("pressure", 6.02214076e23)])
    log.row([("step", 10), ("potential", 0.1), ("pressure", -0.0)])
    with pytest.raises(ValueError):
        log.row([("potential", 1.0), ("step", 0)])
    log.meta("particles", 256000)
    log.meta("box", 67.18)
    log.meta("particles", 1000)  # the last value wins, first-seen order
    log.snapshot("positions", [2, 3], np.arange(6.0))
    m = data.Manifest("lj", gpu="B200", version="0.1.0", settings=[("dt", 0.005), ("cutoff", 2.5)],
                      seconds=1.23456)
    log.write(m)
    d = tmp_path / "run"
    assert (d / "measurements.csv").read_text() == (
        "step,potential,pressure\n0.0,-0.3333333333333333,6.02214076e23\n10.0,0.1,-0.0\n")
    assert np.array_equal(np.load(d / "positions.npy"), np.arange(6.0).reshape(2, 3))
    text = (d / "run.json").read_text()
    run = json.loads(text)
    assert run["scene"] == "lj" and run["git_commit"] is None and run["render_seconds"] == 1.235
    assert list(run["settings"]) == ["cutoff", "dt"]
    assert run["scene_meta"] == {"particles": "1000", "box": "67.18"}
    assert text.startswith('{\n  "scene": "lj",\n') and text.endswith("}\n")
    assert data.json_string('a"b\\c\nd\x01') == '"a\\"b\\\\c\\nd\\u0001"'
    # not recording: rows kept, nothing written
    preview = data.DataLog()
    preview.row([("x", 1.0)])
    preview.snapshot("s", [1], [1.0])
    preview.write()
    assert not preview.is_recording() and preview.csv() == "x\n1.0\n"


@pytest.mark.gpu
def test_measurements_recorded_exactly(gpu, tmp_path):
    from virial_lj import data
    p = gpu.lattice(1000, 11.0, 1.0, 3)
    sim = gpu.LennardJones(p, gpu.Settings([11.0] * 3, dt=0.002))
    log = data.DataLog(str(tmp_path))
    ms = []
    for _ in range(3):
        sim.run(10)
        m = sim.measure_now()
        ms.append(m)
        log.row([("step", m.step), ("kinetic", m.kinetic), ("potential", m.potential),
                 ("virial", m.virial), ("pressure", m.pressure())])
    q = sim.read_particles()
    log.snapshot("positions", q["pos"].shape, q["pos"])
    log.write()
    rows = np.loadtxt(tmp_path / "measurements.csv", delimiter=",", skiprows=1)
    for row, m in zip(rows, ms):
        assert list(row) == [m.step, m.kinetic, m.potential, m.virial, m.pressure()]
    assert np.array_equal(np.load(tmp_path / "positions.npy"), q["pos"])
