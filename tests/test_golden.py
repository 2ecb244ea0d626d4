"""The C oracle and the library's host helpers against the golden vectors of
tests/golden/make_golden.py (an independent numpy restatement of the
reference's lattices, random streams, packing, binning and list build)."""

import os

import numpy as np
import pytest

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "lj_golden.npz"))


def test_lattice_matches_golden(O):
    pos, vel = O.lattice(1000, 11.0, 1.0, 3)
    assert np.array_equal(pos, GOLDEN["lattice_pos"])
    assert np.array_equal(vel, GOLDEN["lattice_vel"])


def test_lattice_box_matches_golden(O):
    pos, vel = O.lattice_box(1000, [9.0, 10.5, 14.25], 1.0, 3)
    assert np.array_equal(pos, GOLDEN["box_pos"])
    assert np.array_equal(vel, GOLDEN["box_vel"])
    n = len(GOLDEN["liquid_pos"])
    pos, vel = O.lattice_box(n, [9.0, 9.0, 12.0], 1.0, 11)
    assert np.array_equal(pos, GOLDEN["liquid_pos"]) and np.array_equal(vel, GOLDEN["liquid_vel"])


def test_library_lattices_match_golden(vl):
    p = vl.lattice(1000, 11.0, 1.0, 3)
    assert np.array_equal(p["pos"], GOLDEN["lattice_pos"])
    assert np.array_equal(p["vel"], GOLDEN["lattice_vel"])
    p = vl.lattice_box(1000, [9.0, 10.5, 14.25], 1.0, 3)
    assert np.array_equal(p["pos"], GOLDEN["box_pos"])
    assert np.array_equal(p["vel"], GOLDEN["box_vel"])


def test_library_fcc_matches_oracle(vl, O):
    p, box = vl.lattice_fcc(5, 0.8442, 0.72, 1)
    pos, vel, obox = O.lattice_fcc(5, 0.8442, 0.72, 1)
    assert box == obox and len(p) == 500
    assert np.array_equal(p["pos"], pos) and np.array_equal(p["vel"], vel)
    assert abs(len(p) / box ** 3 - 0.8442) < 1e-12
    assert np.all(np.abs(vel.sum(0)) < 1e-12)


def test_pcg_matches_golden(O):
    seeds = [O.pcg_seed(s, i) for s in (1, 3, 7) for i in range(16)]
    assert seeds == list(map(int, GOLDEN["pcg_seed"]))
    seq = []
    for st in (1, 12345, 0xDEADBEEF):
        seq += O.pcg_sequence(st, 8)
    assert seq == list(map(int, GOLDEN["pcg_sequence"]))


def test_rebuild_matches_golden(O):
    pos = np.mod(GOLDEN["jittered_cube"], float(np.float32(11.0)))
    vel = GOLDEN["lattice_vel"]
    s = O.setup(vel, [11.0] * 3, 2.5, 0.3, False)
    assert s.capacity == int(GOLDEN["rebuild_capacity"][0])
    r = O.rebuild_ref(s, pos, vel, np.arange(len(pos)), reorder=True)
    assert np.array_equal(r["ids"], GOLDEN["rebuild_ids"])
    assert np.array_equal(r["cell_of_slot"], GOLDEN["rebuild_cell"])
    assert np.array_equal(r["cell_start"], GOLDEN["rebuild_start"])
    assert np.array_equal(r["counts"], GOLDEN["rebuild_counts"])
    flat = np.concatenate([r["lists"][i, :c] for i, c in enumerate(r["counts"])])
    assert np.array_equal(flat, GOLDEN["rebuild_lists"])
    assert r["overflow"] == 0
