"""ctypes wrapper of the CPU test oracle (liboracle.so, built by oracle/Makefile).

Test infrastructure only: the tests, the smoke check and the benchmark's CPU
baseline leg import this module to check or to time against. The CUDA library
and its Python mirror never import it.
"""

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build():
    """Compile liboracle.so with the recipe in oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "CC=gcc"], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    return C.CDLL(LIB_PATH)


_lib = _load()
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


class Setup(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("box", C.c_double * 3),
        ("box_f", C.c_float * 3),
        ("cells", C.c_uint32 * 3),
        ("total_cells", C.c_uint32),
        ("cell_size_f", C.c_float * 3),
        ("segment", C.c_uint32),
        ("capacity", C.c_uint32),
        ("cutoff", C.c_double),
        ("skin", C.c_double),
        ("rc2", C.c_float),
        ("list_r2", C.c_float),
        ("half_skin2", C.c_float),
        ("shift", C.c_float),
        ("force_shift", C.c_float),
        ("energy_scale", C.c_double),
        ("momentum_scale", C.c_double),
    ]


class MdMeasurement(C.Structure):
    _fields_ = [
        ("step", C.c_uint64),
        ("kinetic", C.c_double),
        ("potential", C.c_double),
        ("virial", C.c_double),
        ("momentum", C.c_double * 3),
        ("list_rebuilds", C.c_uint32),
        ("thermostat_energy", C.c_double),
    ]


def _sig(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args
    return f


_fixed_split = _sig("vo_fixed_split", None, [C.c_float, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)])
_fixed_to_raw = _sig("vo_fixed_to_raw", C.c_int64, [C.c_float])
_fixed_raw_f64 = _sig("vo_fixed_raw_f64", C.c_int64, [C.c_double])


class DF(C.Structure):
    _fields_ = [("hi", C.c_float), ("lo", C.c_float)]


for _name in ("vo_df_add", "vo_df_sub", "vo_df_mul", "vo_df_div"):
    _sig(_name, DF, [DF, DF])
_sig("vo_df_sqrt", DF, [DF])
_sig("vo_df_from_f64", DF, [C.c_double])
_sig("vo_df_to_f64", C.c_double, [DF])
_sig("vo_last_bit", C.c_float, [C.c_float])
_sig("vo_pack_lo", C.c_uint32, [_fp, _fp])
_sig("vo_unpack_lo", None, [_fp, C.c_uint32, _fp])
_sig("vo_pcg_seed", C.c_uint32, [C.c_uint32, C.c_uint32])
_sig("vo_pcg", C.c_uint32, [C.POINTER(C.c_uint32)])
_sig("vo_gaussian2", None, [C.POINTER(C.c_uint32), _fp])
_sig("vo_philox4x32_10", None, [_up, _up, _up])
_sig("vo_langevin_noise", None, [C.c_uint32, C.c_uint64, C.c_uint32, _fp])
_sig("vo_lattice", None, [C.c_size_t, C.c_double, C.c_double, C.c_uint64, _dp, _dp])
_sig("vo_lattice_box", None, [C.c_size_t, _dp, C.c_double, C.c_uint64, _dp, _dp])
_sig("vo_lattice_fcc", None, [C.c_uint32, C.c_double, C.c_double, C.c_uint64, _dp, _dp, C.POINTER(C.c_double)])
_sig("vo_setup_compute", C.c_int, [C.c_uint32, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_double, C.POINTER(Setup)])
_sig("vo_rebuild_ref", None, [C.POINTER(Setup), C.c_uint32, _dp, _dp, _up, C.c_int, _up, _up, _up, _up, _up, C.POINTER(C.c_uint32)])
_sig("vo_all_pairs", None, [_dp, C.c_uint32, _dp, C.c_double, C.c_int, C.POINTER(C.c_double), _dp])
_sig("vo_cell_pairs", None, [_dp, C.c_uint32, _dp, C.c_double, C.c_int, C.POINTER(C.c_double), _dp])
_sig("vo_heat_current", None, [_dp, _dp, C.c_uint32, _dp, C.c_double, C.c_int, _dp])
_sig("vo_profile", None, [_dp, _dp, C.c_uint32, _dp, C.c_double, C.c_int, C.c_uint32, _dp])
_sig("vo_md_create", C.c_void_p, [_dp, _dp, C.c_uint32, _dp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint32])
_sig("vo_md_destroy", None, [C.c_void_p])
_sig("vo_md_run", None, [C.c_void_p, C.c_uint64])
_sig("vo_md_measure", None, [C.c_void_p, C.POINTER(MdMeasurement)])
_sig("vo_md_read", None, [C.c_void_p, _dp, _dp])
_sig("vo_md_set_heat_exchange", None, [C.c_void_p, C.c_int, _dp, C.c_double])
_sig("vo_md_set_threads", None, [C.c_int])
_sig("vo_md_threads", C.c_int, [])
_sig("vo_dfmd_create", C.c_void_p, [_dp, _dp, C.c_uint32, _dp, C.c_double, C.c_int, C.c_double])
_sig("vo_dfmd_run", None, [C.c_void_p, C.c_uint64])
_sig("vo_dfmd_measure", None, [C.c_void_p, _dp, C.c_void_p, C.c_void_p])
_sig("vo_dfmd_destroy", None, [C.c_void_p])


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def fixed_split(x):
    lo, hi = C.c_uint32(), C.c_uint32()
    _fixed_split(C.c_float(x), C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def fixed_to_raw(x):
    return _fixed_to_raw(C.c_float(x))


def fixed_raw_f64(x):
    return _fixed_raw_f64(C.c_double(x))


def df(x):
    return _lib.vo_df_from_f64(C.c_double(x))


def df_op(name, a, b=None):
    f = getattr(_lib, "vo_df_" + name)
    return f(a) if b is None else f(a, b)


def df_value(a):
    return _lib.vo_df_to_f64(a)


def last_bit(h):
    return _lib.vo_last_bit(C.c_float(h))


def pack_lo(hi, lo):
    return _lib.vo_pack_lo(np.asarray(hi, np.float32), np.asarray(lo, np.float32))


def unpack_lo(hi, bits):
    out = np.zeros(3, np.float32)
    _lib.vo_unpack_lo(np.asarray(hi, np.float32), bits, out)
    return out


def pcg_seed(seed, index):
    return _lib.vo_pcg_seed(seed, index)


def pcg_sequence(state, count):
    s = C.c_uint32(state)
    return [_lib.vo_pcg(C.byref(s)) for _ in range(count)]


def gaussian2(state):
    s = C.c_uint32(state)
    out = np.zeros(2, np.float32)
    _lib.vo_gaussian2(C.byref(s), out)
    return out, s.value


def philox(ctr, key):
    out = np.zeros(4, np.uint32)
    _lib.vo_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
    return out


def langevin_noise(seed, step, pid):
    out = np.zeros(3, np.float32)
    _lib.vo_langevin_noise(seed, step, pid, out)
    return out


def lattice(count, box_size, temperature, seed):
    pos = np.zeros((count, 3))
    vel = np.zeros((count, 3))
    _lib.vo_lattice(count, box_size, temperature, seed, pos, vel)
    return pos, vel


def lattice_box(count, size, temperature, seed):
    pos = np.zeros((count, 3))
    vel = np.zeros((count, 3))
    _lib.vo_lattice_box(count, _f64(size), temperature, seed, pos, vel)
    return pos, vel


def lattice_fcc(cells, density, temperature, seed):
    n = 4 * cells ** 3
    pos = np.zeros((n, 3))
    vel = np.zeros((n, 3))
    box = C.c_double()
    _lib.vo_lattice_fcc(cells, density, temperature, seed, pos, vel, C.byref(box))
    return pos, vel, box.value


def setup(vel, box, cutoff, skin, shifted_force, thermostat_temperature=0.0):
    s = Setup()
    vel = _f64(vel)
    rc = _lib.vo_setup_compute(len(vel), vel, _f64(box), cutoff, skin, int(shifted_force),
                               thermostat_temperature, C.byref(s))
    if rc != 0:
        raise ValueError("the box must be at least three (cutoff + skin) wide on every axis")
    return s


def rebuild_ref(s, pos, vel, ids, reorder):
    """One list rebuild as the reference orders it. Returns a dict of the
    permuted state and the grid/list arrays (list as n x capacity rows)."""
    n = len(pos)
    x = _f64(pos).copy()
    v = _f64(vel).copy()
    ids = np.ascontiguousarray(ids, np.uint32).copy()
    cell_of_slot = np.zeros(n, np.uint32)
    cell_start = np.zeros(s.total_cells + 1, np.uint32)
    sorted_ = np.zeros(n, np.uint32)
    counts = np.zeros(n, np.uint32)
    lists = np.zeros(n * s.capacity, np.uint32)
    overflow = C.c_uint32()
    _lib.vo_rebuild_ref(C.byref(s), n, x, v, ids, int(reorder), cell_of_slot, cell_start,
                        sorted_, counts, lists, C.byref(overflow))
    return dict(x=x, v=v, ids=ids, cell_of_slot=cell_of_slot, cell_start=cell_start,
                sorted=sorted_, counts=counts, lists=lists.reshape(n, s.capacity),
                overflow=overflow.value)


def all_pairs(pos, box, cutoff, shifted_force):
    pe = C.c_double()
    w = np.zeros(3)
    _lib.vo_all_pairs(_f64(pos), len(pos), _f64(box), cutoff, int(shifted_force), C.byref(pe), w)
    return pe.value, w


def cell_pairs(pos, box, cutoff, shifted_force):
    pe = C.c_double()
    w = np.zeros(3)
    _lib.vo_cell_pairs(_f64(pos), len(pos), _f64(box), cutoff, int(shifted_force), C.byref(pe), w)
    return pe.value, w


def heat_current(pos, vel, box, cutoff, shifted_force):
    j = np.zeros(3)
    _lib.vo_heat_current(_f64(pos), _f64(vel), len(pos), _f64(box), cutoff, int(shifted_force), j)
    return j


def profile(pos, vel, box, cutoff, shifted_force, bins):
    out = np.zeros(bins * 8 + 3)
    _lib.vo_profile(_f64(pos), _f64(vel), len(pos), _f64(box), cutoff, int(shifted_force), bins, out)
    return out


def set_threads(threads):
    _lib.vo_md_set_threads(int(threads))


def threads():
    return _lib.vo_md_threads()


class MD:
    """f64 cell-list MD with the CUDA path's integrator (the CPU baseline)."""

    def __init__(self, pos, vel, box, cutoff=2.5, skin=0.3, dt=0.005, shifted_force=False,
                 langevin=None, nose_hoover=None):
        thermostat, t, gamma, seed = 0, 0.0, 0.0, 0
        if langevin is not None:
            thermostat = 1
            t, gamma, seed = langevin
        elif nose_hoover is not None:
            thermostat = 2
            t, gamma = nose_hoover  # temperature, period
        self._h = _lib.vo_md_create(_f64(pos), _f64(vel), len(pos), _f64(box), cutoff, skin, dt,
                                    int(shifted_force), thermostat, t, gamma, seed)
        self.n = len(pos)

    def run(self, steps):
        _lib.vo_md_run(self._h, steps)

    def measure(self):
        m = MdMeasurement()
        _lib.vo_md_measure(self._h, C.byref(m))
        return m

    def set_heat_exchange(self, hot=None, cold=None, energy=0.0):
        """hot and cold (lo, hi) slabs in z, energy per step; None stops."""
        on = hot is not None
        slabs = np.array(list(hot) + list(cold) if on else [0.0] * 4, dtype=np.float64)
        _lib.vo_md_set_heat_exchange(self._h, int(on), slabs, float(energy))

    def read(self):
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        _lib.vo_md_read(self._h, pos, vel)
        return pos, vel

    def close(self):
        if self._h:
            _lib.vo_md_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class DoubleFloatMD:
    """The reference's plain double-float path at constant energy
    (double-float state, f32 pair arithmetic on packed positions, df64 sums;
    dfpath.c), for the error table against the f64 truth."""

    def __init__(self, pos, vel, box, cutoff=2.5, dt=0.005, shifted_force=False):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        self._h = _lib.vo_dfmd_create(pos, vel, len(pos), _f64(box), cutoff, int(shifted_force), dt)
        if not self._h:
            raise ValueError("the box must be at least three cutoffs wide on every axis")
        self.n = len(pos)

    def run(self, steps):
        _lib.vo_dfmd_run(self._h, steps)

    def measure(self):
        """(kinetic, potential, virial, positions, velocities)"""
        out = np.zeros(3)
        pos = np.zeros((self.n, 3))
        vel = np.zeros((self.n, 3))
        _lib.vo_dfmd_measure(self._h, out, pos.ctypes.data_as(C.c_void_p),
                             vel.ctypes.data_as(C.c_void_p))
        return out[0], out[1], out[2], pos, vel

    def close(self):
        if self._h:
            _lib.vo_dfmd_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ---- granular contacts through the cell grid (test oracle) ----

def grain_block(lo, hi, radius, spread, seed):
    """Grains on a jittered cubic lattice filling [lo, hi] (granular.rs:634-665):
    spacing 2 r (1 + spread) 1.02, xorshift64 seeded with seed | 1, positions
    jittered by +-1 % of r, radii r (1 + spread (2 u - 1)). Returns (pos, radius)."""
    spacing = 2.0 * radius * (1.0 + spread) * 1.02
    counts = [max(int(np.floor((hi[k] - lo[k]) / spacing)), 1) for k in range(3)]
    mask = (1 << 64) - 1
    s = (seed | 1) & mask

    def random():
        nonlocal s
        s ^= (s << 13) & mask
        s ^= s >> 7
        s ^= (s << 17) & mask
        return (s >> 11) / float(1 << 53)

    pos, rad = [], []
    for z in range(counts[2]):
        for y in range(counts[1]):
            for x in range(counts[0]):
                jit = [(random() - 0.5) * 0.02 * radius for _ in range(3)]
                pos.append([lo[0] + (x + 0.5) * spacing + jit[0],
                            lo[1] + (y + 0.5) * spacing + jit[1],
                            lo[2] + (z + 0.5) * spacing + jit[2]])
                rad.append(radius * (1.0 + spread * (2.0 * random() - 1.0)))
    return np.array(pos), np.array(rad)


def grain_contacts(pos, radius, box_size, cells, capacity):
    """The granular solver's contact search (granular.wgsl:204-263) on its
    grid (grid.wgsl:11-148; cell side f32(box / cells), granular.rs:182):
    for each grain, the overlapping grains of the 27 cells around its own
    (skipping cells past the walls) in the order dz, dy, dx, each cell in
    grain order; double-float positions, f32 radii, IEEE f32 operations as
    written. Returns (partners n x capacity, -1 where empty; counts)."""
    f32 = np.float32
    n = len(pos)
    hi = pos.astype(f32)
    lo = (pos - hi.astype(np.float64)).astype(f32)
    rad = radius.astype(f32)
    size = f32(box_size / cells)
    c = np.floor(hi / size).astype(np.int64)
    c = np.clip(c, 0, cells - 1)
    cell = (c[:, 2] * cells + c[:, 1]) * cells + c[:, 0]
    order = np.argsort(cell, kind="stable")
    start = np.searchsorted(cell[order], np.arange(cells ** 3 + 1))
    partners = np.full((n, capacity), -1, np.int64)
    counts = np.zeros(n, np.int64)
    for i in range(n):
        cand = []
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    q = c[i] + np.array([dx, dy, dz])
                    if (q < 0).any() or (q >= cells).any():
                        continue
                    k = (q[2] * cells + q[1]) * cells + q[0]
                    cand.extend(order[start[k]:start[k + 1]])
        cand = np.array([j for j in cand if j != i], np.int64)
        if len(cand) == 0:
            continue
        d = (hi[i] - hi[cand]) + (lo[i] - lo[cand])
        dist2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        reach = rad[i] + rad[cand]
        dist = np.sqrt(dist2)
        hit = cand[((reach - dist) > f32(0)) & (dist2 > f32(0))]
        counts[i] = len(hit)
        partners[i, :min(len(hit), capacity)] = hit[:capacity]
    return partners, counts
