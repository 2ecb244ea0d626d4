"""vlj_bin_noalloc: the cell binning for callers that cannot let the library
allocate device memory (a framework that owns all device memory through its
own pool, or a latency-critical loop where cudaMalloc would synchronise the
device). Its scratch is a fixed device array shared by every call, so this
checks two calls in a row, each against the binning the simulation itself
performs (its first list rebuild) on the same positions, read through the
existing inspection entry point. Kept last in collection order: it is an
add-on to the library and must not stop the other tests from running."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bin_noalloc_matches_the_simulation_twice(gpu):
    import torch

    lib = C.CDLL(gpu.library_path())
    f = lib.vlj_bin_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.vlj_last_error.restype = C.c_char_p

    for size, n, seed in [([14.0, 14.0, 16.0], 3000, 8), ([9.0, 10.5, 14.25], 1000, 3)]:
        p = gpu.lattice_box(n, size, 1.2, seed)
        sim = gpu.LennardJones(p, gpu.Settings(size))
        g = sim.grid_info()
        ref = sim.read_grid()  # the first rebuild: bin, stable sort, reorder
        box = np.array(sim.box_size())
        pos = torch.tensor(np.mod(p["pos"], box), dtype=torch.float64, device="cuda")
        cells = (C.c_uint32 * 3)(*g.cells)
        for call in range(2):
            sorted_ = torch.full((n,), -1, dtype=torch.int32, device="cuda")
            start = torch.full((g.total_cells + 1,), -1, dtype=torch.int32, device="cuda")
            cell_of = torch.full((n,), -1, dtype=torch.int32, device="cuda")
            stream = torch.cuda.current_stream()
            rc = f(pos.data_ptr(), n, (C.c_double * 3)(*box), cells, sorted_.data_ptr(),
                   start.data_ptr(), cell_of.data_ptr(), stream.cuda_stream)
            assert rc == 0, lib.vlj_last_error()
            stream.synchronize()
            got_sorted = sorted_.cpu().numpy().view(np.uint32)
            got_start = start.cpu().numpy().view(np.uint32)
            got_cell = cell_of.cpu().numpy().view(np.uint32)
            # the simulation's slots after its first reorder hold the
            # particles in cell order: slot s holds particle ids[s]
            assert np.array_equal(got_sorted, ref["ids"]), call
            assert np.array_equal(got_start, ref["cell_start"]), call
            assert np.array_equal(got_cell[ref["ids"]], ref["cell_of_slot"]), call
        sim.close()


def test_bin_noalloc_rejects_grids_beyond_its_limit(gpu):
    import torch

    lib = C.CDLL(gpu.library_path())
    f = lib.vlj_bin_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    pos = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    out = torch.zeros(8, dtype=torch.int32, device="cuda")
    too_many = (C.c_uint32 * 3)(128, 128, 17)  # 278,528 > 262,144 cells
    rc = f(pos.data_ptr(), 4, (C.c_double * 3)(10.0, 10.0, 10.0), too_many, out.data_ptr(),
           out.data_ptr(), out.data_ptr(), None)
    assert rc == 1  # VLJ_INVALID_ARG, before touching the GPU


def _numpy_binning(pos, box, cells):
    """The binning in numpy: f32 positions over f32 cell sizes of the
    f32-rounded box, clamped, then a stable sort of the cell indices."""
    cells = np.asarray(cells)
    size = np.array([np.float32(float(np.float32(b)) / c) for b, c in zip(box, cells)],
                    dtype=np.float32)
    c = np.floor(pos.astype(np.float32) / size).astype(np.int64)
    c = np.clip(c, 0, cells - 1)
    cell = (c[:, 2] * cells[1] + c[:, 1]) * cells[0] + c[:, 0]
    order = np.argsort(cell, kind="stable")
    start = np.searchsorted(cell[order], np.arange(int(np.prod(cells)) + 1))
    return order.astype(np.uint32), start.astype(np.uint32), cell.astype(np.uint32)


@pytest.mark.parametrize("n, cells", [(1000, (2, 2, 2)), (20000, (1, 1, 1)), (5000, (3, 1, 2))])
def test_bin_noalloc_crowded_cells(gpu, n, cells):
    # cells far above 32 particles take the block-wide sort: in shared memory
    # (125 a cell), in place in global memory (20,000 in one cell), and mixed
    import torch

    lib = C.CDLL(gpu.library_path())
    f = lib.vlj_bin_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.vlj_last_error.restype = C.c_char_p
    box = [7.0, 9.0, 11.0]
    rng = np.random.default_rng(n)
    pos = rng.uniform(0.0, 1.0, (n, 3)) * np.array(box)
    want = _numpy_binning(pos, box, cells)
    d_pos = torch.tensor(pos, dtype=torch.float64, device="cuda")
    total = int(np.prod(cells))
    for call in range(2):
        sorted_ = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        start = torch.full((total + 1,), -1, dtype=torch.int32, device="cuda")
        cell_of = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream()
        rc = f(d_pos.data_ptr(), n, (C.c_double * 3)(*box), (C.c_uint32 * 3)(*cells),
               sorted_.data_ptr(), start.data_ptr(), cell_of.data_ptr(), stream.cuda_stream)
        assert rc == 0, lib.vlj_last_error()
        stream.synchronize()
        assert np.array_equal(sorted_.cpu().numpy().view(np.uint32), want[0]), call
        assert np.array_equal(start.cpu().numpy().view(np.uint32), want[1]), call
        assert np.array_equal(cell_of.cpu().numpy().view(np.uint32), want[2]), call
