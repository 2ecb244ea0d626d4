"""The step kernel over cell tiles against the per-particle gathers.

With cell tiles a block stages the encoded positions of its brick's
neighbour cells in shared memory and each home particle walks a 16-bit list
of indices into that tile, in the slot list's order, with the same pair
arithmetic. So the tile lists must name exactly the slot lists' particles,
entry for entry, and a trajectory must be the same to the bit with tiles on
and off -- on the 256,000-atom workload, the 1000-atom box, the liquid-vapour
slab (bricks of liquid and of vapour), with the heat current fused into the
step, and when a tile overflows its shared memory and the block falls back
to the slot list.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def tiles_on():
    # cell tiles are opt-in at creation (VLJ_TILES=1)
    before = os.environ.get("VLJ_TILES")
    os.environ["VLJ_TILES"] = "1"
    yield
    if before is None:
        del os.environ["VLJ_TILES"]
    else:
        os.environ["VLJ_TILES"] = before


def tile_of_brick(grid, cells, cols, index):
    """The slots a brick's tile holds, in tile order (nine x-rows dz, dy =
    -1..1 over the brick's cells and one more each side, or the whole row)."""
    nx, ny, nz = cells
    cs, order = grid["cell_start"], grid["sorted"]
    r, yz = index % cols, index // cols
    y, z = yz % ny, yz // ny
    q, rem = divmod(nx, cols)
    w = q + (1 if r < rem else 0)
    x0 = r * q + min(r, rem)
    full = cols == 1
    rx = nx if full else w + 2
    xs = 0 if full else (x0 - 1) % nx
    tile = []
    for rho in range(9):
        dz, dy = rho // 3 - 1, rho % 3 - 1
        row = (((z + dz) % nz) * ny + (y + dy) % ny) * nx
        for xp in range(rx):
            c = row + (xs + xp) % nx
            tile.extend(order[cs[c]:cs[c + 1]])
    homes = range(cs[(z * ny + y) * nx + x0], cs[(z * ny + y) * nx + x0 + w])
    return np.array(tile, np.uint32), homes


def check_tile_lists(sim):
    cols, bricks, cap, threads = sim.tile_info()
    assert bricks > 0 and threads >= 64
    g = sim.grid_info()
    grid = sim.read_grid()
    t16 = sim.read_tile_lists()
    seen = 0
    for b in range(bricks):
        tile, homes = tile_of_brick(grid, list(g.cells), cols, b)
        for p in homes:
            i = grid["sorted"][p]
            c = grid["counts"][i]
            assert np.array_equal(tile[t16[p, :c]], grid["lists"][i, :c]), (b, p)
            # the last row's padding is the particle itself
            pad = t16[p, c:(c + 7) // 8 * 8]
            assert np.all(tile[pad] == i)
            seen += 1
    assert seen == sim.count()


def same_run(make, steps, heat=False):
    out = []
    for tiles in (True, False):
        sim = make()
        sim.set_tiles(tiles)
        if heat:
            sim.record_heat_current(steps)
            for _ in range(steps):
                sim.step(1)
                sim.sample_heat_current()
        else:
            sim.run(steps)
        m = sim.measure_now()
        q = sim.read_particles()
        j = sim.read_heat_current() if heat else None
        out.append((q.tobytes(), m.potential, m.virial, m.kinetic, m.list_rebuilds,
                    None if j is None else np.asarray(j).tobytes()))
        sim.close()
    assert out[0] == out[1]
    return out[0]


def test_tile_lists_name_the_slot_lists_256k(gpu):
    p, L = gpu.lattice_fcc(40, 0.8442, 1.0, 7)
    sim = gpu.LennardJones(p, gpu.Settings([L] * 3, dt=0.005, shifted_force=True,
                                           thermostat=gpu.Langevin(1.0, 1.0, 7)))
    assert sim.tile_info()[0] > 1  # several bricks per row
    sim.run(40)
    sim.force_rebuild()
    check_tile_lists(sim)
    sim.close()


def test_tile_lists_small_box_and_slab(gpu):
    L = (1000 / 0.8442) ** (1 / 3)
    sim = gpu.LennardJones(gpu.lattice(1000, L, 1.0, 3), gpu.Settings([L] * 3, dt=0.005))
    assert sim.tile_info()[0] == 1  # three cells a row: the row is one brick
    sim.run(30)
    check_tile_lists(sim)
    sim.close()
    p = gpu.lattice_box(16000, [20.0, 20.0, 54.8], 0.7, 4)
    p["pos"][:, 2] += 47.6
    sim = gpu.LennardJones(p, gpu.Settings([20.0, 20.0, 150.0], dt=0.005, shifted_force=True,
                                           thermostat=gpu.Langevin(0.7, 0.5, 4)))
    sim.run(50)
    check_tile_lists(sim)
    sim.close()


def test_tiles_keep_the_trajectory_256k(gpu):
    p, L = gpu.lattice_fcc(40, 0.8442, 1.0, 7)
    st = gpu.Settings([L] * 3, dt=0.005, shifted_force=True, thermostat=gpu.Langevin(1.0, 1.0, 7))
    r = same_run(lambda: gpu.LennardJones(p, st), 60)
    assert r[4] >= 2  # rebuilds happened on the way


@pytest.mark.parametrize("shifted_force", [False, True])
def test_tiles_keep_the_trajectory_small_box(gpu, shifted_force):
    L = (1000 / 0.8442) ** (1 / 3)
    p = gpu.lattice(1000, L, 0.72, 1)
    st = gpu.Settings([L] * 3, dt=0.005, shifted_force=shifted_force)
    same_run(lambda: gpu.LennardJones(p, st), 300)


def test_tiles_keep_the_trajectory_slab(gpu):
    p = gpu.lattice_box(16000, [20.0, 20.0, 54.8], 0.7, 4)
    p["pos"][:, 2] += 47.6
    st = gpu.Settings([20.0, 20.0, 150.0], dt=0.005, shifted_force=True,
                      thermostat=gpu.Langevin(0.7, 0.5, 4))
    same_run(lambda: gpu.LennardJones(p, st), 200)


def test_tiles_keep_the_heat_current(gpu):
    p, L = gpu.lattice_fcc(12, 0.8442, 0.722, 5)
    st = gpu.Settings([L] * 3, dt=0.004)
    same_run(lambda: gpu.LennardJones(p, st), 40, heat=True)


def test_overfull_tiles_fall_back_to_the_slot_list(gpu):
    # a tile capacity far below the tiles' size: every block walks the slot
    # list with global gathers, and the trajectory is still the same
    p, L = gpu.lattice_fcc(16, 0.8442, 1.0, 2)
    st = gpu.Settings([L] * 3, dt=0.005, shifted_force=True, thermostat=gpu.Langevin(1.0, 1.0, 2))
    os.environ["VLJ_TILE_CAP"] = "64"
    try:
        small = gpu.LennardJones(p, st)
    finally:
        del os.environ["VLJ_TILE_CAP"]
    assert small.tile_info()[2] == 64
    small.run(50)
    ref = gpu.LennardJones(p, st)
    ref.set_tiles(False)
    ref.run(50)
    assert small.read_particles().tobytes() == ref.read_particles().tobytes()
