"""Python mirror of virial_particles::lennard_jones over the B200 CUDA library.

Same names and argument meanings as the reference's Rust API
(crates/virial-particles/src/lennard_jones.rs): `LennardJones(particles,
settings)`, `step`, `run`, `measure`/`poll`/`measure_now`, `read_particles`,
profiles along z, the heat current, setters, and the `lattice` helpers.
The reference panics on misuse; here every failure raises `VljError` carrying
the C ABI status. Particles are numpy arrays of dtype `PARTICLE`
(fields `pos` and `vel`, three f64 each), the layout of `vlj_particle`.

All work runs in the CUDA library (libvirial_lj.so); there is no CPU path:
importing this module without the built library raises ImportError.
"""

import ctypes as C
import enum
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Union

import numpy as np

from . import _ffi
from ._ffi import PARTICLE

_lib = _ffi.load()

__all__ = [
    "PARTICLE", "VljError", "Langevin", "NoseHoover", "Settings", "Measurement", "Slab", "Profile",
    "Phase", "Drawn", "HeatExchange", "LennardJones", "Batch", "Replica", "lattice", "lattice_box",
    "lattice_fcc", "particles", "device_count", "library_path", "launches", "uneven_replicas",
    "replica_cost", "shard_replicas", "tune_batch_skin", "tune_batch", "tune_box", "grain_cells",
    "grain_contacts",
]


class VljError(RuntimeError):
    """A C ABI call failed; `status` is the vlj_status name."""

    def __init__(self, status, message):
        self.status = _ffi.STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.status}: {message}")


def _check(status):
    if status != 0:
        raise VljError(status, _lib.vlj_last_error().decode(errors="replace"))


def library_path():
    return _lib._name


def device_count():
    n = C.c_int()
    _check(_lib.vlj_device_count(C.byref(n)))
    return n.value


def fp32_peak():
    """Measured FP32 FMA throughput of the current device, TFLOP/s."""
    t = C.c_double()
    _check(_lib.vlj_debug_fp32_peak(C.byref(t)))
    return t.value


def philox(ctr, key):
    """The device's noise stream for known-answer checks: Philox-4x32-10 of
    each counter (n x 4 uint32) and key (n x 2 uint32), and the three Gaussian
    numbers the step kernel draws for (id, step, seed) = (ctr[:, 0],
    ctr[:, 1] + 2^32 ctr[:, 2], key[:, 0]). Returns (words n x 4, noise n x 3)."""
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    key = np.ascontiguousarray(key, dtype=np.uint32).reshape(-1, 2)
    if len(ctr) != len(key):
        raise ValueError("one key per counter")
    out = np.zeros((len(ctr), 4), np.uint32)
    noise = np.zeros((len(ctr), 3), np.float32)
    _check(_lib.vlj_debug_philox(_ffi.ptr(ctr), _ffi.ptr(key), len(ctr), _ffi.ptr(out),
                                 _ffi.ptr(noise)))
    return out, noise


def grain_cells(box_size, max_radius):
    """Cells per axis of the granular solver's grid (granular.rs:179-181)."""
    c = C.c_uint32()
    _check(_lib.vlj_grain_cells(float(box_size), float(max_radius), C.byref(c)))
    return c.value


def grain_contacts(pos, radius, box_size, capacity=16, cells=None, stream=None):
    """Overlapping partners of every grain through the cell grid, in the
    reference's order (granular.wgsl:204-263). `pos` (n x 3) and `radius` (n)
    are torch tensors of float64 on the device (the entry point works on
    device memory and allocates nothing; the buffers here are torch's).
    Returns (partners n x capacity, counts n, sorted, cell_start, cell_of)
    as torch int32 tensors on the device."""
    import torch
    n = pos.shape[0]
    if cells is None:
        cells = grain_cells(box_size, float(radius.max()))
    dev = pos.device
    i32 = dict(dtype=torch.int32, device=dev)
    total = cells ** 3
    scratch = torch.zeros(total + 1, **i32)
    sorted_, cell_start = torch.zeros(n, **i32), torch.zeros(total + 1, **i32)
    cell_of, counts = torch.zeros(n, **i32), torch.zeros(n, **i32)
    partners = torch.full((n, max(capacity, 1)), -1, **i32)
    pos = pos.contiguous()
    radius = radius.contiguous()
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    _check(_lib.vlj_grain_contacts(pos.data_ptr(), radius.data_ptr(), n, float(box_size), cells,
                                   capacity, scratch.data_ptr(), sorted_.data_ptr(),
                                   cell_start.data_ptr(), cell_of.data_ptr(), partners.data_ptr(),
                                   counts.data_ptr(), s))
    return partners, counts, sorted_, cell_start, cell_of


def launches():
    """Kernel launches this library has made in this process."""
    n = C.c_uint64()
    _check(_lib.vlj_debug_launches(C.byref(n)))
    return n.value


def particles(pos, vel=None):
    """Particle array from n x 3 positions (and velocities)."""
    pos = np.asarray(pos, dtype=np.float64)
    out = np.zeros(len(pos), PARTICLE)
    out["pos"] = pos
    if vel is not None:
        out["vel"] = np.asarray(vel, dtype=np.float64)
    return out


# ---- settings (lennard_jones.rs:32-82) ----

@dataclass
class Langevin:
    temperature: float
    friction: float
    seed: int


@dataclass
class NoseHoover:
    temperature: float
    period: float


Thermostat = Optional[Union[Langevin, NoseHoover]]


@dataclass
class Settings:
    box_size: Sequence[float]
    cutoff: float = 2.5
    dt: float = 0.005
    thermostat: Thermostat = None
    shifted_force: bool = False
    skin: float = 0.3
    profile_bins: int = 0

    def _c(self):
        t = _ffi.Thermostat()
        if isinstance(self.thermostat, Langevin):
            t.kind, t.temperature, t.friction, t.seed = 1, self.thermostat.temperature, \
                self.thermostat.friction, self.thermostat.seed & 0xFFFFFFFF
        elif isinstance(self.thermostat, NoseHoover):
            t.kind, t.temperature, t.period = 2, self.thermostat.temperature, self.thermostat.period
        elif self.thermostat is not None:
            raise TypeError("thermostat must be None, Langevin or NoseHoover")
        s = _ffi.Settings()
        s.box_size[:] = [float(x) for x in self.box_size]
        s.cutoff, s.dt, s.thermostat = self.cutoff, self.dt, t
        s.shifted_force, s.skin, s.profile_bins = int(bool(self.shifted_force)), self.skin, \
            self.profile_bins
        return s


# ---- results (lennard_jones.rs:84-280) ----

@dataclass
class Measurement:
    step: int
    time: float
    kinetic: float
    potential: float
    virial: float
    momentum: List[float]
    count: int
    volume: float
    list_rebuilds: int
    list_overflow: int
    thermostat_energy: float
    condensed: int
    list_capacity: int = 0  # list entries per particle the measurement ran with
    list_grows: int = 0     # capacity grows since creation (set_list_growth)

    @staticmethod
    def _from(m):
        return Measurement(m.step, m.time, m.kinetic, m.potential, m.virial, list(m.momentum),
                           m.count, m.volume, m.list_rebuilds, m.list_overflow,
                           m.thermostat_energy, m.condensed, m.list_capacity, m.list_grows)

    def energy(self):
        return self.kinetic + self.potential

    def temperature(self, dof):
        """2 KE / dof: 3N with a thermostat, 3N - 3 at constant energy."""
        return 2.0 * self.kinetic / dof

    def pressure(self):
        """P = (2 KE + W) / (3 V), the virial theorem."""
        return (2.0 * self.kinetic + self.virial) / (3.0 * self.volume)

    def extended_energy(self):
        return self.energy() + self.thermostat_energy


@dataclass
class Slab:
    z: float
    particles: float
    kinetic: List[float]
    virial: List[float]
    potential: float


class Phase(enum.IntEnum):
    LIQUID = 0
    VAPOUR = 1
    INTERFACE = 2
    BETWEEN = 3


class Drawn(enum.IntEnum):
    NEIGHBOURS = 0
    TEMPERATURE = 1


@dataclass
class Profile:
    samples: int
    box_size: List[float]
    slabs: List[Slab]
    virial: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])

    def slab_volume(self):
        lx, ly, lz = self.box_size
        return lx * ly * lz / len(self.slabs)

    def density(self):
        v = self.slab_volume()
        return [s.particles / v for s in self.slabs]

    def temperature(self):
        return [sum(s.kinetic) / (3.0 * s.particles) if s.particles else math.nan
                for s in self.slabs]

    def pressure_tensor(self):
        v = self.slab_volume()
        return [[(s.kinetic[a] + s.virial[a]) / v for a in range(3)] for s in self.slabs]

    def total_pressure_tensor(self):
        volume = self.box_size[0] * self.box_size[1] * self.box_size[2]
        return [(sum(s.kinetic[a] for s in self.slabs) + self.virial[a]) / volume
                for a in range(3)]

    def interfaces(self, midpoint):
        d = np.ascontiguousarray(self.density(), np.float64)
        found = C.c_size_t()
        out = np.zeros(len(d), np.float64)
        _check(_lib.vlj_profile_interfaces(d.ctypes.data_as(C.POINTER(C.c_double)), len(d),
                                           float(self.box_size[2]), midpoint,
                                           out.ctypes.data_as(C.POINTER(C.c_double)), len(out),
                                           C.byref(found)))
        return list(out[:found.value])

    def phases(self, midpoint, margin):
        d = np.ascontiguousarray(self.density(), np.float64)
        out = np.zeros(len(d), np.int32)
        _check(_lib.vlj_profile_phases(d.ctypes.data_as(C.POINTER(C.c_double)), len(d),
                                       float(self.box_size[2]), midpoint, margin,
                                       out.ctypes.data_as(C.POINTER(C.c_int32))))
        return [Phase(int(p)) for p in out]

    def mean_in(self, values, phases, phase):
        chosen = [v for v, p in zip(values, phases) if p == phase]
        return sum(chosen) / len(chosen) if chosen else None

    def surface_tension(self):
        pxx, pyy, pzz = self.total_pressure_tensor()
        return 0.5 * self.box_size[2] * (pzz - 0.5 * (pxx + pyy))


@dataclass
class HeatExchange:
    hot: Sequence[float]
    cold: Sequence[float]
    energy: float


# ---- the simulation (lennard_jones.rs:334-1375) ----

class LennardJones:
    """Lennard-Jones particles in a periodic box on one GPU."""

    def __init__(self, particles, settings: Settings, stream=None):
        p = np.ascontiguousarray(particles, dtype=PARTICLE)
        self._settings = settings
        h = C.c_void_p()
        cs = settings._c()
        _check(_lib.vlj_create(_ffi.ptr(p), len(p), C.byref(cs), stream, C.byref(h)))
        self._h = h
        self._n = len(p)
        # kept on the object: a collection at interpreter exit may run after
        # the module's globals are gone
        self._destroy = _lib.vlj_destroy

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # accessors
    def count(self):
        return self._n

    def box_size(self):
        out = (C.c_double * 3)()
        _check(_lib.vlj_box_size(self._h, out))
        return list(out)

    def volume(self):
        v = C.c_double()
        _check(_lib.vlj_volume(self._h, C.byref(v)))
        return v.value

    def steps(self):
        v = C.c_uint64()
        _check(_lib.vlj_steps(self._h, C.byref(v)))
        return v.value

    def time(self):
        v = C.c_double()
        _check(_lib.vlj_time(self._h, C.byref(v)))
        return v.value

    def target_temperature(self):
        has, t = C.c_int(), C.c_double()
        _check(_lib.vlj_target_temperature(self._h, C.byref(has), C.byref(t)))
        return t.value if has.value else None

    def positions(self):
        """(device pointer, stride): three f64 arrays x, y, z of `stride` each."""
        p, stride = C.c_void_p(), C.c_size_t()
        _check(_lib.vlj_positions(self._h, C.byref(p), C.byref(stride)))
        return p.value, stride.value

    def velocities(self):
        """Device pointer to float4 (vx, vy, vz, drawn) per slot."""
        p = C.c_void_p()
        _check(_lib.vlj_velocities(self._h, C.byref(p)))
        return p.value

    # stepping
    def step(self, steps=1):
        _check(_lib.vlj_step(self._h, int(steps)))

    def run(self, steps):
        _check(_lib.vlj_run(self._h, int(steps)))

    # measurements
    def measure(self):
        ok = C.c_int()
        _check(_lib.vlj_measure(self._h, C.byref(ok)))
        return bool(ok.value)

    def after_submit(self):
        """Nothing to do: work goes to the stream when it is enqueued."""

    def poll(self):
        buf = (_ffi.Measurement * 8)()
        n = C.c_size_t()
        _check(_lib.vlj_poll(self._h, buf, 8, C.byref(n)))
        return [Measurement._from(buf[i]) for i in range(n.value)]

    def measure_now(self):
        m = _ffi.Measurement()
        _check(_lib.vlj_measure_now(self._h, C.byref(m)))
        return Measurement._from(m)

    # state
    def read_particles(self, out=None):
        """Positions and canonical velocities in input order; into `out` (a
        contiguous PARTICLE array of count() entries, e.g. over pinned host
        memory) when given."""
        if out is None:
            out = np.zeros(self._n, PARTICLE)
        elif out.dtype != PARTICLE or len(out) != self._n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous PARTICLE array of count() entries")
        _check(_lib.vlj_read_particles(self._h, _ffi.ptr(out)))
        return out

    def write_particles(self, particles):
        p = np.ascontiguousarray(particles, dtype=PARTICLE)
        _check(_lib.vlj_write_particles(self._h, _ffi.ptr(p), len(p)))

    # setters
    def set_drawn(self, drawn: Drawn):
        _check(_lib.vlj_set_drawn(self._h, int(drawn)))

    def set_condensed_neighbours(self, neighbours):
        _check(_lib.vlj_set_condensed_neighbours(self._h, int(neighbours)))

    def set_temperature(self, temperature):
        _check(_lib.vlj_set_temperature(self._h, float(temperature)))

    def set_heat_exchange(self, exchange: Optional[HeatExchange]):
        if exchange is None:
            _check(_lib.vlj_set_heat_exchange(self._h, None))
            return
        h = _ffi.HeatExchange()
        h.hot[:] = list(exchange.hot)
        h.cold[:] = list(exchange.cold)
        h.energy = exchange.energy
        _check(_lib.vlj_set_heat_exchange(self._h, C.byref(h)))

    def heat_flux(self):
        has, f = C.c_int(), C.c_double()
        _check(_lib.vlj_heat_flux(self._h, C.byref(has), C.byref(f)))
        return f.value if has.value else None

    def set_list_growth(self, on):
        """Grow the list capacity when a list overflows (on by default; off is
        the reference's report-only behaviour)."""
        _check(_lib.vlj_set_list_growth(self._h, int(bool(on))))

    def set_tile_cols(self, cols):
        """Cell tiles in the step kernel at run time: `cols` bricks per x-row
        (each block stages its brick's neighbour rows in shared memory), or 0
        for the per-particle gathers (the default). Same trajectory either
        way; the tiles take over at the next scheduled list rebuild."""
        _check(_lib.vlj_set_tile_cols(self._h, int(cols)))

    def set_grid_every_step(self, on):
        """Rebuild the cell grid on every step as well (the lists still on the
        skin / 2 trigger): the same trajectory, more work per step. Not in the
        reference, which bins only when the lists rebuild."""
        _check(_lib.vlj_set_grid_every_step(self._h, int(bool(on))))

    # profiles
    def sample_profile(self):
        _check(_lib.vlj_sample_profile(self._h))

    def sample_profile_now(self):
        self.sample_profile()

    def clear_profile(self):
        _check(_lib.vlj_clear_profile(self._h))

    def read_profile(self):
        bins = self._settings.profile_bins
        slabs = (_ffi.Slab * max(bins, 1))()
        virial = (C.c_double * 3)()
        samples = C.c_uint64()
        _check(_lib.vlj_read_profile(self._h, slabs, virial, C.byref(samples)))
        out = [Slab(s.z, s.particles, list(s.kinetic), list(s.virial), s.potential)
               for s in slabs[:bins]]
        return Profile(samples.value, self.box_size(), out, list(virial))

    # heat current
    def record_heat_current(self, capacity):
        self._series_capacity = int(capacity)
        _check(_lib.vlj_record_heat_current(self._h, int(capacity)))

    def sample_heat_current(self):
        _check(_lib.vlj_sample_heat_current(self._h))

    def read_heat_current(self):
        cap = getattr(self, "_series_capacity", 0)
        out = np.zeros((max(cap, 1), 3))
        n = C.c_size_t()
        _check(_lib.vlj_read_heat_current(self._h, out.ctypes.data_as(C.POINTER(C.c_double)),
                                          cap, C.byref(n)))
        return out[:n.value].copy()

    # inspection for tests
    def grid_info(self):
        g = _ffi.GridInfo()
        _check(_lib.vlj_debug_grid_info(self._h, C.byref(g)))
        return g

    def read_grid(self):
        g = self.grid_info()
        n = self._n
        out = dict(
            sorted=np.zeros(n, np.uint32), cell_start=np.zeros(g.total_cells + 1, np.uint32),
            cell_of_slot=np.zeros(n, np.uint32), ids=np.zeros(n, np.uint32),
            counts=np.zeros(n, np.uint32), lists=np.zeros((n, g.capacity), np.uint32),
            x=np.zeros((n, 3)), v=np.zeros((n, 3)))
        _check(_lib.vlj_debug_read_grid(
            self._h, *[_ffi.ptr(out[k]) for k in
                       ("sorted", "cell_start", "cell_of_slot", "ids", "counts", "lists", "x", "v")]))
        return out

    def set_graphs(self, on):
        _check(_lib.vlj_debug_set_graphs(self._h, int(bool(on))))

    def set_step_threads(self, threads):
        """Particles per block of the step kernel (64, 128 or 256)."""
        _check(_lib.vlj_debug_set_step_threads(self._h, int(threads)))

    def set_step_lanes(self, lanes):
        """Lanes per particle of the step kernel: 0 by grid size, 1 or 2 (same
        trajectory to the bit)."""
        _check(_lib.vlj_debug_set_step_lanes(self._h, int(lanes)))

    def set_tiles(self, on):
        """Cell tiles in the step kernel on or off (same trajectory either way)."""
        _check(_lib.vlj_debug_set_tiles(self._h, int(bool(on))))

    def tile_info(self):
        """(bricks per x-row, bricks, tile capacity, threads per block); zeros without tiles."""
        v = [C.c_uint32() for _ in range(4)]
        _check(_lib.vlj_debug_tile_info(self._h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def read_tile_lists(self):
        """The 16-bit tile lists by sorted position: (n, capacity rounded up to 8)."""
        g = self.grid_info()
        rows = (g.capacity + 7) // 8
        raw = np.zeros(rows * g.segment * 8, np.uint16)
        _check(_lib.vlj_debug_read_tile_lists(self._h, _ffi.ptr(raw)))
        return raw.reshape(rows, g.segment, 8)[:, :self._n, :].transpose(1, 0, 2).reshape(
            self._n, rows * 8)

    def kernel_timing(self, on):
        _check(_lib.vlj_debug_kernel_timing(self._h, int(bool(on))))

    def kernel_time(self):
        """(total ms, launches) of the step kernel since timing was switched on."""
        ms, n = C.c_double(), C.c_uint64()
        _check(_lib.vlj_debug_kernel_time(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def kernels_executed(self):
        n = C.c_uint64()
        _check(_lib.vlj_debug_kernels_executed(self._h, C.byref(n)))
        return n.value

    def read_vel4(self):
        """The last measurement's (vx, vy, vz, drawn value) per particle, input order."""
        out = np.zeros((self._n, 4), np.float32)
        _check(_lib.vlj_debug_read_vel4(self._h, _ffi.ptr(out)))
        return out

    def force_rebuild(self):
        _check(_lib.vlj_debug_force_rebuild(self._h))

    def read_partials(self):
        """(pe, w, raw): per-slot (hi, lo) halves of pair energy and virial."""
        pe = np.zeros((self._n, 2), np.float32)
        w = np.zeros((self._n, 2), np.float32)
        raw = np.zeros(8, np.int64)
        _check(_lib.vlj_debug_read_partials(self._h, _ffi.ptr(pe), _ffi.ptr(w), _ffi.ptr(raw)))
        return pe, w, raw


# ---- batched replicas (no reference counterpart) ----

@dataclass
class Replica:
    particles: np.ndarray
    box_size: Sequence[float]
    thermostat: Thermostat = None


class Batch:
    """Many independent periodic boxes stepped together in one launch per step."""

    def __init__(self, replicas: Sequence[Replica], cutoff=2.5, skin=0.3, dt=0.005,
                 shifted_force=False, stream=None):
        self._keep = [np.ascontiguousarray(r.particles, dtype=PARTICLE) for r in replicas]
        descs = (_ffi.ReplicaDesc * len(replicas))()
        for d, r, p in zip(descs, replicas, self._keep):
            d.particles = p.ctypes.data
            d.count = len(p)
            d.box_size[:] = [float(x) for x in r.box_size]
            d.thermostat = Settings(r.box_size, thermostat=r.thermostat)._c().thermostat
        h = C.c_void_p()
        _check(_lib.vlj_batch_create(descs, len(replicas), cutoff, skin, dt, int(shifted_force),
                                     stream, C.byref(h)))
        self._h = h
        self._counts = [len(p) for p in self._keep]
        self._keep = None
        self._destroy = _lib.vlj_batch_destroy

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def replicas(self):
        return len(self._counts)

    def total(self):
        return sum(self._counts)

    def step(self, steps=1):
        _check(_lib.vlj_batch_step(self._h, int(steps)))

    def measure(self):
        buf = (_ffi.Measurement * len(self._counts))()
        _check(_lib.vlj_batch_measure(self._h, buf))
        return [Measurement._from(m) for m in buf]

    def read_particles(self, replica):
        out = np.zeros(self._counts[replica], PARTICLE)
        _check(_lib.vlj_batch_read_particles(self._h, int(replica), _ffi.ptr(out)))
        return out

    def run(self, steps):
        """Step, then wait for the steps to finish."""
        _check(_lib.vlj_batch_run(self._h, int(steps)))

    def box_size(self, replica):
        out = (C.c_double * 3)()
        _check(_lib.vlj_batch_box_size(self._h, int(replica), out))
        return list(out)

    # inspection and timing, through the simulation that steps the arena
    def _sim(self):
        h = C.c_void_p()
        _check(_lib.vlj_debug_batch_sim(self._h, C.byref(h)))
        return h

    def set_step_threads(self, threads):
        """Particles per block of the step kernel (64, 128 or 256)."""
        _check(_lib.vlj_debug_set_step_threads(self._sim(), int(threads)))

    def set_graphs(self, on):
        _check(_lib.vlj_debug_set_graphs(self._sim(), int(bool(on))))

    def kernel_timing(self, on):
        _check(_lib.vlj_debug_kernel_timing(self._sim(), int(bool(on))))

    def kernel_time(self):
        ms, n = C.c_double(), C.c_uint64()
        _check(_lib.vlj_debug_kernel_time(self._sim(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def kernels_executed(self):
        n = C.c_uint64()
        _check(_lib.vlj_debug_kernels_executed(self._sim(), C.byref(n)))
        return n.value


# ---- host helpers (lennard_jones.rs:1377-1441) ----

def lattice(count, box_size, temperature, seed):
    out = np.zeros(int(count), PARTICLE)
    _check(_lib.vlj_lattice(int(count), float(box_size), float(temperature), int(seed),
                            _ffi.ptr(out)))
    return out


def lattice_box(count, size, temperature, seed):
    out = np.zeros(int(count), PARTICLE)
    sz = (C.c_double * 3)(*[float(s) for s in size])
    _check(_lib.vlj_lattice_box(int(count), sz, float(temperature), int(seed), _ffi.ptr(out)))
    return out


def lattice_fcc(cells, density, temperature, seed):
    """fcc lattice of cells^3 unit cells; returns (particles, box side)."""
    out = np.zeros(4 * int(cells) ** 3, PARTICLE)
    box = C.c_double()
    _check(_lib.vlj_lattice_fcc(int(cells), float(density), float(temperature), int(seed),
                                _ffi.ptr(out), C.byref(box)))
    return out, box.value


def uneven_replicas(count=512, seed=2024, sizes=(500, 20000), densities=(0.01, 0.90),
                    temperatures=(0.7, 2.0), friction=1.0):
    """Replicas of uneven size, density and temperature from one seed.

    Replica r draws, from a xorshift64 stream (the reference's generator,
    lennard_jones.rs:1410-1415), N log-uniform in `sizes`, density and
    temperature uniform in their ranges; its box is the cube of side
    (N / density)^(1/3) holding lattice(N, side, T, seed + r), under a
    Langevin thermostat at T (friction `friction`, noise seed seed + r).
    """
    mask = (1 << 64) - 1
    s = seed | 1

    def uniform():
        nonlocal s
        s ^= (s << 13) & mask
        s ^= s >> 7
        s ^= (s << 17) & mask
        return ((s >> 11) + 0.5) / float(1 << 53)

    out = []
    for r in range(int(count)):
        n = int(round(math.exp(math.log(sizes[0]) + uniform() *
                               (math.log(sizes[1]) - math.log(sizes[0])))))
        rho = densities[0] + uniform() * (densities[1] - densities[0])
        t = temperatures[0] + uniform() * (temperatures[1] - temperatures[0])
        side = (n / rho) ** (1.0 / 3.0)
        p = lattice(n, side, t, seed + r)
        out.append(Replica(p, [side] * 3, Langevin(t, friction, (seed + r) & 0xFFFFFFFF)))
    return out


def replica_cost(replica, cutoff=2.5, skin=0.3):
    """Relative cost of stepping a replica: its particles times (the 96 B of
    state each moves per step, plus its pair work at the machine balance of
    about 11 flop per byte): 11 flops per list candidate and 20 per pair
    inside the cutoff, at the replica's density."""
    n = len(replica.particles)
    volume = replica.box_size[0] * replica.box_size[1] * replica.box_size[2]
    rho = n / volume
    n_list = 4.0 / 3.0 * math.pi * (cutoff + skin) ** 3 * rho
    n_rc = 4.0 / 3.0 * math.pi * cutoff ** 3 * rho
    return n * (96.0 + (11.0 * n_list + 20.0 * n_rc) / 11.0)


def shard_replicas(replicas, world_size, cutoff=2.5, skin=0.3):
    """Whole replicas to ranks, balancing the summed cost (longest first, each
    to the rank with the least so far). Returns one list of replica indices
    per rank, each in ascending order; every rank computes the same answer."""
    world_size = int(world_size)
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    costs = [replica_cost(r, cutoff, skin) for r in replicas]
    order = sorted(range(len(replicas)), key=lambda i: (-costs[i], i))
    load = [0.0] * world_size
    shards = [[] for _ in range(world_size)]
    for i in order:
        rank = min(range(world_size), key=lambda k: (load[k], k))
        shards[rank].append(i)
        load[rank] += costs[i]
    return [sorted(s) for s in shards]


def tune_batch(replicas, skins=(0.3, 0.4, 0.5, 0.6, 0.8), threads=(64, 128, 256), cutoff=2.5,
               dt=0.005, shifted_force=False, steps=60, warmup=20, stream=None):
    """The neighbour skin and the step kernel's particles per block that step
    this replica set fastest on this GPU.

    The skin trades list length against rebuild frequency (tune_batch_skin);
    the block size trades the step kernel's tail (blocks that straddle two
    replicas, or hold a dense replica's long lists) against its scheduling
    granularity. Every (skin, threads) pair runs `warmup` then `steps` steps
    of the actual set, timed with CUDA events on `stream` (a torch stream);
    the trajectory does not depend on the block size and only the list length
    on the skin. Returns (skin, threads, {(skin, threads): seconds per step}).
    """
    import torch

    s = stream or torch.cuda.current_stream()
    times = {}
    for skin in skins:
        b = Batch(replicas, cutoff=cutoff, skin=skin, dt=dt, shifted_force=shifted_force,
                  stream=s.cuda_stream)
        b.step(warmup)
        for t in threads:
            b.set_step_threads(t)
            b.step(3)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            b.step(steps)
            e1.record(s)
            s.synchronize()
            times[(skin, t)] = e0.elapsed_time(e1) / 1e3 / steps
        b.close()
    skin, t = min(times, key=times.get)
    return skin, t, times


def tune_box(particles, settings: Settings, tile_cols=(0, 3, 4, 5, 6), threads=(64, 128, 256),
             steps=30, warmup=10, flush_bytes=256 << 20, stream=None, stats=None):
    """The step kernel's form that steps this box fastest on this GPU: the
    cell tiles' bricks per x-row (0: per-particle gathers, the default) and
    the particles per block of the per-particle kernel.

    Neither changes the trajectory, so the choice carries over to the box
    itself. A copy of the box (the same particles and settings) runs every
    candidate: `warmup` steps, then `steps` single steps timed with CUDA events
    on `stream` (a torch stream), each after a write of `flush_bytes` that
    clears the L2 (0: no flush). Tile sizes the box cannot take (too few
    particles per cell, more bricks than cells along x) are skipped. Returns
    (cols, threads, {(cols, threads): seconds per step}); apply them with
    set_tile_cols and set_step_threads. A dict given as `stats` receives the
    number of the library's kernels the copy ran ("kernels").
    """
    import torch

    s = stream or torch.cuda.current_stream()
    flush = torch.empty(max(int(flush_bytes), 1), dtype=torch.uint8, device="cuda")
    sim = LennardJones(particles, settings, stream=s.cuda_stream)
    times = {}
    try:
        sim.step(warmup)
        candidates = [(0, t) for t in threads] + [(c, 128) for c in tile_cols if c]
        for cols, t in candidates:
            try:
                sim.set_tile_cols(cols)
            except VljError:
                continue
            sim.set_step_threads(t)
            if cols:
                sim.force_rebuild()  # the copy's schedule does not matter: tiles from now on
            sim.step(3)
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(steps)]
            for a, b in ev:
                if flush_bytes:
                    with torch.cuda.stream(s):
                        flush.fill_(1)
                a.record(s)
                sim.step(1)
                b.record(s)
            s.synchronize()
            times[(cols, t)] = sum(a.elapsed_time(b) for a, b in ev) / 1e3 / steps
        if stats is not None:
            stats["kernels"] = sim.kernels_executed()
    finally:
        sim.close()
    cols, t = min(times, key=times.get)
    return cols, t, times


def tune_batch_skin(replicas, skins=(0.3, 0.4, 0.5, 0.6, 0.8), cutoff=2.5, dt=0.005,
                    shifted_force=False, steps=60, warmup=20, stream=None):
    """The neighbour skin that steps this replica set fastest on this GPU.

    A wider skin makes longer lists (more work every step) but rebuilds them
    less often; the best trade depends on the replicas' densities and
    temperatures, so each candidate runs `warmup` then `steps` steps of the
    actual set (timed with CUDA events through `torch.cuda`, on `stream`, a
    torch stream). Forces are exact within the cutoff at any skin, so the choice
    changes speed, not physics. Returns (best skin, {skin: seconds per step}).
    """
    import torch

    s = stream or torch.cuda.current_stream()
    times = {}
    for skin in skins:
        b = Batch(replicas, cutoff=cutoff, skin=skin, dt=dt, shifted_force=shifted_force,
                  stream=s.cuda_stream)
        b.step(warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        b.step(steps)
        e1.record(s)
        s.synchronize()
        times[skin] = e0.elapsed_time(e1) / 1e3 / steps
        b.close()
    best = min(times, key=times.get)
    return best, times
