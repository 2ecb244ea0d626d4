"""Granular contacts through the cell grid (the reference's granular solver
includes the same grid as the Lennard-Jones one, granular.rs:327-328).

The contact finder bins grains with the library's grid pipeline and walks
the 27 cells around each grain (not periodic) in the reference's order
(granular.wgsl:204-263); its partner tables must equal the oracle's
restatement entry for entry: a packed block of grains with radii grown
until neighbours overlap, loose random grains (some with more contacts than
the table holds, some past the walls, which bin into the edge cells), and
the grid it leaves against a stable sort of the cells.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(gpu, O, pos, radius, box, capacity):
    import torch
    cells = gpu.grain_cells(box, radius.max())
    d_pos = torch.tensor(pos, dtype=torch.float64, device="cuda")
    d_rad = torch.tensor(radius, dtype=torch.float64, device="cuda")
    got = gpu.grain_contacts(d_pos, d_rad, box, capacity=capacity, cells=cells)
    torch.cuda.synchronize()
    partners, counts, sorted_, start, cell_of = [t.cpu().numpy() for t in got]
    want_p, want_c = O.grain_contacts(pos, radius, box, cells, capacity)
    assert np.array_equal(counts, want_c)
    assert np.array_equal(partners.astype(np.int64), want_p)
    # the grid: cells of f32 positions over f32(box / cells), stable order
    size = np.float32(box / cells)
    c = np.clip(np.floor(pos.astype(np.float32) / size).astype(np.int64), 0, cells - 1)
    cell = (c[:, 2] * cells + c[:, 1]) * cells + c[:, 0]
    assert np.array_equal(cell_of, cell)
    assert np.array_equal(sorted_, np.argsort(cell, kind="stable"))
    assert np.array_equal(start, np.searchsorted(np.sort(cell), np.arange(cells ** 3 + 1)))
    return counts


def test_grain_cells_rule(gpu):
    # granular.rs:179-181: floor(box / (2 r_max)), within 1 .. 64
    assert gpu.grain_cells(0.1, 0.0015) == 33
    assert gpu.grain_cells(0.1, 0.08) == 1
    assert gpu.grain_cells(1.0, 0.001) == 64


def test_packed_block_contacts(gpu, O):
    # the reference's glass-bead block (tests/granular.rs:128-129), radii
    # grown 12 % so that neighbours overlap
    pos, radius = O.grain_block([0.004, 0.004, 0.004], [0.05, 0.05, 0.04], 0.0015, 0.1, 7)
    counts = run(gpu, O, pos, radius * 1.12, 0.1, 16)
    assert counts.max() > 0 and counts.mean() > 1.0


def test_loose_grains_with_crowded_contacts(gpu, O):
    rng = np.random.default_rng(5)
    n = 3000
    box = 0.05
    pos = rng.uniform(0.0, box, (n, 3))
    pos[:20] += 0.003  # a few past the far walls: the edge cells take them
    pos[20:40] -= 0.003
    radius = rng.uniform(0.0015, 0.0035, n)
    counts = run(gpu, O, pos, radius, box, 8)
    assert counts.max() > 8  # some grains have more contacts than the table holds
