/*
 * virial_lj.h -- C ABI of the B200 Lennard-Jones step.
 *
 * A drop-in replacement for the public API of virial_particles::lennard_jones
 * (crates/virial-particles/src/lennard_jones.rs in anshullaikar/virial-engine),
 * backed by CUDA kernels for sm_100a. Plain C types only: pointers, sizes and
 * the structs below. Every function returns a vlj_status and never throws or
 * aborts across the ABI; vlj_last_error() gives a message for the calling
 * thread's last failure.
 *
 * Threading: a simulation is owned by one thread at a time and bound to one
 * CUDA stream (given at creation; NULL means a stream the library creates).
 * Work is enqueued on that stream, which plays the role of the reference's
 * command encoder: vlj_step / vlj_measure / vlj_sample_profile return as soon
 * as the work is queued; vlj_run / vlj_measure_now / vlj_read_* wait for it.
 *
 * Units are the reference's reduced LJ units (sigma = epsilon = m = k_B = 1).
 */
#ifndef VIRIAL_LJ_H
#define VIRIAL_LJ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VLJ_API __attribute__((visibility("default")))

/* Replaces the reference's assert!/expect panics (lennard_jones.rs:458-461,
 * 907, 930-933, 987-991, 1176-1178, 1252-1255, 1269) by status codes. */
typedef enum {
    VLJ_OK = 0,
    VLJ_INVALID_ARG = 1,      /* null pointer, non-finite or out-of-range value */
    VLJ_BOX_TOO_SMALL = 2,    /* a side below three (cutoff + skin), lennard_jones.rs:458-461 */
    VLJ_LIST_OVERFLOW = 3,    /* reported through vlj_measurement.list_overflow, never returned */
    VLJ_CUDA_ERROR = 4,       /* a CUDA call failed; see vlj_last_error() */
    VLJ_TIMEOUT = 5,          /* a bounded device wait ran out */
    VLJ_BUSY = 6,             /* every measurement read-back slot is in flight */
    VLJ_NOT_ENABLED = 7,      /* profiles without profile_bins, heat current not recorded,
                                 set_temperature without a thermostat, heat exchange
                                 with one (lennard_jones.rs:907, 930-933, 990, 1178) */
    VLJ_FULL = 8,             /* heat-current series full (lennard_jones.rs:991) */
    VLJ_NO_DEVICE = 9         /* no CUDA device visible */
} vlj_status;

/* lennard_jones.rs:25-30 */
typedef struct {
    double pos[3];
    double vel[3];
} vlj_particle;

/* lennard_jones.rs:32-61 (Thermostat::None / Langevin / NoseHoover) */
typedef enum {
    VLJ_THERMOSTAT_NONE = 0,
    VLJ_THERMOSTAT_LANGEVIN = 1,
    VLJ_THERMOSTAT_NOSE_HOOVER = 2
} vlj_thermostat_kind;

typedef struct {
    int32_t kind;          /* vlj_thermostat_kind */
    double temperature;
    double friction;       /* Langevin */
    uint32_t seed;         /* Langevin: key of the counter-based noise stream */
    double period;         /* Nose-Hoover */
} vlj_thermostat;

/* lennard_jones.rs:63-82 */
typedef struct {
    double box_size[3];
    double cutoff;
    double dt;
    vlj_thermostat thermostat;
    int32_t shifted_force;
    double skin;
    uint32_t profile_bins;
} vlj_settings;

/* lennard_jones.rs:84-131 */
typedef struct {
    uint64_t step;
    double time;
    double kinetic;
    double potential;
    double virial;          /* sum over pairs of r . F */
    double momentum[3];
    uint32_t count;
    double volume;
    uint32_t list_rebuilds;
    uint32_t list_overflow; /* 0, or the largest neighbour count that did not fit */
    double thermostat_energy;
    uint32_t condensed;
    /* No reference counterpart: the list capacity (entries per particle) the
     * measurement ran with, and how many times it has grown since creation
     * (vlj_set_list_growth). */
    uint32_t list_capacity;
    uint32_t list_grows;
} vlj_measurement;

/* lennard_jones.rs:133-147: one slab's averages per sample */
typedef struct {
    double z;
    double particles;
    double kinetic[3];
    double virial[3];
    double potential;
} vlj_slab;

/* lennard_jones.rs:365-373 */
typedef enum { VLJ_DRAWN_NEIGHBOURS = 0, VLJ_DRAWN_TEMPERATURE = 1 } vlj_drawn;

/* lennard_jones.rs:149-156 */
typedef enum {
    VLJ_PHASE_LIQUID = 0,
    VLJ_PHASE_VAPOUR = 1,
    VLJ_PHASE_INTERFACE = 2,
    VLJ_PHASE_BETWEEN = 3
} vlj_phase;

/* lennard_jones.rs:375-387 */
typedef struct {
    double hot[2];
    double cold[2];
    double energy;
} vlj_heat_exchange;

typedef struct vlj_sim vlj_sim;

/* ---- errors and devices ---- */
VLJ_API const char *vlj_last_error(void);
VLJ_API const char *vlj_status_name(vlj_status s);
VLJ_API vlj_status vlj_device_count(int *count);

/* ---- construction: LennardJones::new (lennard_jones.rs:443-801) ----
 * `stream` is a cudaStream_t (or NULL). Sizes the grid and lists, rounds the
 * box to f32, uploads the particles and builds the first lists. */
VLJ_API vlj_status vlj_create(const vlj_particle *particles, size_t count,
                              const vlj_settings *settings, void *stream, vlj_sim **out);
VLJ_API vlj_status vlj_destroy(vlj_sim *sim);

/* ---- stepping: LennardJones::step (lennard_jones.rs:1092-1138), enqueue only */
VLJ_API vlj_status vlj_step(vlj_sim *sim, uint32_t steps);
/* LennardJones::run (lennard_jones.rs:1274-1284): step, then wait. */
VLJ_API vlj_status vlj_run(vlj_sim *sim, uint64_t steps);

/* ---- measurements: measure / after_submit / poll / measure_now
 * (lennard_jones.rs:1141-1163, 1194-1260). vlj_measure enqueues one
 * measurement and its read-back; *accepted is 0 when all read-back slots are
 * busy (the reference returns false). vlj_poll returns finished measurements,
 * oldest first. */
VLJ_API vlj_status vlj_measure(vlj_sim *sim, int *accepted);
VLJ_API vlj_status vlj_poll(vlj_sim *sim, vlj_measurement *out, size_t capacity, size_t *written);
VLJ_API vlj_status vlj_measure_now(vlj_sim *sim, vlj_measurement *out);

/* ---- state: read_particles (lennard_jones.rs:1354-1374), in input order */
VLJ_API vlj_status vlj_read_particles(vlj_sim *sim, vlj_particle *out);
/* Replaces every particle's position and velocity (a restart from a
 * snapshot); lists rebuild before the next force evaluation. No reference
 * counterpart beyond LennardJones::new on the same sizes. */
VLJ_API vlj_status vlj_write_particles(vlj_sim *sim, const vlj_particle *particles, size_t count);

/* ---- accessors (lennard_jones.rs:870-881, 1014-1030) ---- */
VLJ_API vlj_status vlj_count(const vlj_sim *sim, uint32_t *count);
VLJ_API vlj_status vlj_box_size(const vlj_sim *sim, double out[3]);
VLJ_API vlj_status vlj_volume(const vlj_sim *sim, double *volume);
VLJ_API vlj_status vlj_steps(const vlj_sim *sim, uint64_t *steps);
VLJ_API vlj_status vlj_time(const vlj_sim *sim, double *time);
/* *has = 0 without a thermostat (the reference returns None). */
VLJ_API vlj_status vlj_target_temperature(const vlj_sim *sim, int *has, double *temperature);
/* positions()/velocities() (lennard_jones.rs:1041-1051) hand a renderer GPU
 * buffers; with no graphics interop these are plain device pointers:
 * positions as three f64 arrays (x, y, z) of `stride` elements each, in slot
 * order; velocities as float4 (vx, vy, vz, drawn value) per slot, written by
 * each measurement. */
VLJ_API vlj_status vlj_positions(const vlj_sim *sim, const double **xyz, size_t *stride);
VLJ_API vlj_status vlj_velocities(const vlj_sim *sim, const float **vel4);

/* ---- setters (lennard_jones.rs:885-952) ---- */
VLJ_API vlj_status vlj_set_drawn(vlj_sim *sim, vlj_drawn drawn);
VLJ_API vlj_status vlj_set_condensed_neighbours(vlj_sim *sim, uint32_t neighbours);
VLJ_API vlj_status vlj_set_temperature(vlj_sim *sim, double temperature);
/* NULL stops the exchange. */
VLJ_API vlj_status vlj_set_heat_exchange(vlj_sim *sim, const vlj_heat_exchange *exchange);
/* *has = 0 when no exchange is set. */
VLJ_API vlj_status vlj_heat_flux(const vlj_sim *sim, int *has, double *flux);
/* List capacity recovery (no reference counterpart; on by default). The
 * capacity starts at the reference's rule (twice the mean neighbour count
 * within cutoff + skin, plus 32; lennard_jones.rs:471-474), which a dense
 * region of a mostly dilute box (a liquid slab) can exceed. The reference
 * only reports that through list_overflow, and the particles concerned lose
 * pairs until the next rebuild. With growth on, when a list overflows the
 * host raises that box's capacity to 1.25 x the largest count (rounded up to
 * a multiple of 8), reallocates the lists and rebuilds them: vlj_run checks
 * after its steps, vlj_measure_now grows and measures again (so the
 * measurement it returns has every pair), a measurement read by vlj_poll
 * schedules the grow for the next vlj_step. Each grow is counted in
 * vlj_measurement.list_grows; a build that overflows at creation grows the
 * lists before the first forces. 0 restores the reference's report-only
 * behaviour (from creation on when the environment sets
 * VLJ_LIST_GROWTH=0). */
VLJ_API vlj_status vlj_set_list_growth(vlj_sim *sim, int on);
/* No reference counterpart: the step kernel's cell tiles of a single box at
 * run time (a tuning knob, virial_lj.tune_box). cols >= 1: bricks of whole
 * cells along x, `cols` bricks per x-row (at most the cells along x), each
 * block staging its brick's neighbour rows in shared memory; 0: the
 * per-particle gathers from the slot list (the default). The trajectory is
 * the same to the bit either way. Waits for the stream; the tiles take over
 * at the next list rebuild the skin schedule brings (which builds their
 * 16-bit lists beside the slot lists: a rebuild out of turn would change
 * the trajectory's bits), the slot lists until then. VLJ_INVALID_ARG for a
 * batch's simulation, or cols >= 1 in a box of fewer than four particles per
 * cell on average. */
VLJ_API vlj_status vlj_set_tile_cols(vlj_sim *sim, uint32_t cols);
/* No reference counterpart (the reference bins only when the lists rebuild):
 * with on != 0, rebuild the cell grid (bin, scan, scatter, per-cell sort) on
 * every step, the Verlet lists still on the skin / 2 trigger. Same trajectory
 * to the bit, more work per step. A single box only (VLJ_NOT_ENABLED for a
 * batch's simulation). */
VLJ_API vlj_status vlj_set_grid_every_step(vlj_sim *sim, int on);

/* ---- profiles along z: sample_profile / clear_profile / read_profile
 * (lennard_jones.rs:1167-1191, 1286-1325). `slabs` holds profile_bins
 * entries; virial gets the whole-box W_aa. Values are averages per sample. */
VLJ_API vlj_status vlj_sample_profile(vlj_sim *sim);
VLJ_API vlj_status vlj_clear_profile(vlj_sim *sim);
VLJ_API vlj_status vlj_read_profile(vlj_sim *sim, vlj_slab *slabs, double virial[3],
                                    uint64_t *samples);

/* ---- heat current for Green-Kubo: record_heat_current / sample_heat_current
 * / read_heat_current (lennard_jones.rs:954-1012). `out` holds 3 doubles per
 * recorded sample. */
VLJ_API vlj_status vlj_record_heat_current(vlj_sim *sim, uint32_t capacity);
VLJ_API vlj_status vlj_sample_heat_current(vlj_sim *sim);
VLJ_API vlj_status vlj_read_heat_current(vlj_sim *sim, double *out, size_t capacity,
                                         size_t *samples);

/* ---- host-only helpers ---- */
/* lattice / lattice_box (lennard_jones.rs:1377-1441): `out` holds `count`. */
VLJ_API vlj_status vlj_lattice(size_t count, double box_size, double temperature, uint64_t seed,
                               vlj_particle *out);
VLJ_API vlj_status vlj_lattice_box(size_t count, const double size[3], double temperature,
                                   uint64_t seed, vlj_particle *out);
/* fcc lattice of cells^3 unit cells (4 * cells^3 particles) at `density`;
 * no reference counterpart (the reference has only simple cubic lattices). */
VLJ_API vlj_status vlj_lattice_fcc(uint32_t cells, double density, double temperature,
                                   uint64_t seed, vlj_particle *out, double *box_size);
/* Profile analysis (lennard_jones.rs:209-279): interfaces where the density
 * crosses `midpoint`, and each slab's phase. `density` has `bins` values of
 * slabs of width lz / bins centred at (b + 0.5) * width. */
VLJ_API vlj_status vlj_profile_interfaces(const double *density, size_t bins, double lz,
                                          double midpoint, double *out, size_t capacity,
                                          size_t *found);
VLJ_API vlj_status vlj_profile_phases(const double *density, size_t bins, double lz,
                                      double midpoint, double margin, int32_t *phases);

/* ---- batched replicas: many independent boxes in one step launch ----
 * No reference counterpart: the reference runs one box per LennardJones.
 * Each replica has its own particles, box, thermostat and lists; all share
 * cutoff, skin, dt and the cutoff style. */
typedef struct {
    const vlj_particle *particles;
    size_t count;
    double box_size[3];
    vlj_thermostat thermostat;
} vlj_replica_desc;

typedef struct vlj_batch vlj_batch;

VLJ_API vlj_status vlj_batch_create(const vlj_replica_desc *replicas, size_t count,
                                    double cutoff, double skin, double dt, int32_t shifted_force,
                                    void *stream, vlj_batch **out);
VLJ_API vlj_status vlj_batch_destroy(vlj_batch *batch);
VLJ_API vlj_status vlj_batch_step(vlj_batch *batch, uint32_t steps);
/* Step, then wait for the steps to finish. */
VLJ_API vlj_status vlj_batch_run(vlj_batch *batch, uint64_t steps);
/* One measurement per replica into out[replicas]; waits. */
VLJ_API vlj_status vlj_batch_measure(vlj_batch *batch, vlj_measurement *out);
/* Replica r's particles into out (its count), input order; waits. */
VLJ_API vlj_status vlj_batch_read_particles(vlj_batch *batch, size_t replica, vlj_particle *out);
VLJ_API vlj_status vlj_batch_count(const vlj_batch *batch, size_t *replicas, uint64_t *particles);
/* Replica r's box sides as the simulation uses them (rounded to f32). */
VLJ_API vlj_status vlj_batch_box_size(const vlj_batch *batch, size_t replica, double out[3]);

/* ---- cell binning that allocates no device memory ----
 * No counterpart in the reference. For callers that cannot let a library
 * allocate: an embedding framework that hands out all device memory from its
 * own pool, or a latency-critical loop where cudaMalloc / cudaFree would
 * synchronise the device and stall other streams. The caller passes every
 * buffer; this call allocates nothing.
 *
 * Bins `count` positions (device memory, count x 3 doubles, row-major, each
 * inside [0, box_size)) into cells[0] x cells[1] x cells[2] cells the way the
 * simulation bins them (the reference's grid.wgsl: clamp(floor(f32(x) /
 * cell size)), cell index (z * ny + y) * nx + x, a stable counting sort).
 * Outputs, all device memory the caller owns: sorted[count] (particle indices
 * in cell order, index order within a cell), cell_start[cells + 1],
 * cell_of[count]. Work is enqueued on `stream` (a cudaStream_t, or NULL).
 *
 * Limits and sharing: at most VLJ_BIN_NOALLOC_MAX_CELLS cells (larger grids
 * are rejected with VLJ_INVALID_ARG). Any number of particles per cell: cells
 * of more than 32 are ordered by a block-wide sorting network, O(m log^2 m)
 * for m particles, in shared memory up to 8192 and in place in `sorted`
 * beyond that (correct but slow: a million particles in one cell take a
 * sizeable fraction of a second). The per-cell counters live in one fixed
 * device array ((VLJ_BIN_NOALLOC_MAX_CELLS + 1) x 4 bytes) that every GPU
 * loading the library holds until exit and that every call shares: calls
 * whose work overlaps on the GPU race with each other, so serialise them (one
 * stream, or events). Each call looks up that array's address in the current
 * context (so a device reset between calls is safe); the first call on a
 * device also loads the library's device code and should come before any
 * stream capture. */
#define VLJ_BIN_NOALLOC_MAX_CELLS 262144u
VLJ_API vlj_status vlj_bin_noalloc(const double *pos, size_t count, const double box_size[3],
                                   const uint32_t cells[3], uint32_t *sorted,
                                   uint32_t *cell_start, uint32_t *cell_of, void *stream);

/* ---- granular contacts through the cell grid ----
 * The reference's granular solver includes the same grid (granular.rs:
 * 327-328 appends grid.wgsl): grains binned into cells at least one diameter
 * wide, each cell sorted by grain index, and every grain's contacts found in
 * the 27 cells around its own -- not periodic: cells past a wall are skipped
 * -- in the order dz, dy, dx = -1..1, each in its sorted order
 * (granular.wgsl:204-263). vlj_grain_cells gives the reference's cells per
 * axis, clamp(floor(box_size / (2 max_radius)), 1, 64) (granular.rs:
 * 179-181). vlj_grain_contacts bins `count` grains (pos: count x 3 doubles,
 * radius: count doubles; device memory) into cells^3 cubic cells of side
 * box_size / cells and writes, for grain i, its overlapping partners in that
 * order to partners[i * capacity ..] (the first `capacity` of them) and their
 * number to counts[i]; the reference's test is double-float positions, f32
 * radii, reach - sqrt(dot(d, d)) > 0. It also leaves the grid: sorted
 * (count), cell_start (cells^3 + 1), cell_of (count). Every buffer is the
 * caller's, device memory, including `scratch` (cells^3 + 1 words); nothing
 * is allocated. Enqueued on `stream`. */
VLJ_API vlj_status vlj_grain_cells(double box_size, double max_radius, uint32_t *cells);
VLJ_API vlj_status vlj_grain_contacts(const double *pos, const double *radius, size_t count,
                                      double box_size, uint32_t cells, uint32_t capacity,
                                      uint32_t *scratch, uint32_t *sorted, uint32_t *cell_start,
                                      uint32_t *cell_of, uint32_t *partners, uint32_t *counts,
                                      void *stream);

/* ---- inspection for tests (no reference counterpart) ----
 * Reads the grid and lists of the last rebuild: slot of each position in
 * cell order (`sorted`, n), cell starts (total_cells + 1), cell of each slot
 * (n), original id of each slot (n), list counts (n) and entries (n rows of
 * `capacity`, slot indices), plus slot-ordered positions and stored
 * velocities (n x 3 each). Any pointer may be NULL to skip it. */
typedef struct {
    uint32_t cells[3];
    uint32_t total_cells;
    uint32_t capacity;
    uint32_t segment;
    uint32_t rebuilds;
    uint32_t reorder_every;
    float cell_size[3];
    float list_r2;
} vlj_grid_info;

VLJ_API vlj_status vlj_debug_grid_info(vlj_sim *sim, vlj_grid_info *info);
VLJ_API vlj_status vlj_debug_read_grid(vlj_sim *sim, uint32_t *sorted, uint32_t *cell_start,
                                       uint32_t *cell_of_slot, uint32_t *ids,
                                       uint32_t *list_count, uint32_t *list, double *pos,
                                       double *vel_stored);
/* Forces a list rebuild now (the decision ignores the displacement). */
VLJ_API vlj_status vlj_debug_force_rebuild(vlj_sim *sim);
/* Per-slot halves of each particle's pair energy and virial from the last
 * measurement, as (hi, lo) f32 pairs whose exact sum is the value (2n each),
 * and the raw 64-bit fixed-point slots (8). */
VLJ_API vlj_status vlj_debug_read_partials(vlj_sim *sim, float *pe_half, float *w_half,
                                           int64_t *raw_slots);
/* Kernel launches this library enqueued from the host so far (all
 * simulations; a graph launch counts its always-run nodes). */
VLJ_API vlj_status vlj_debug_launches(uint64_t *launches);
/* Kernels of this simulation that ran on the device (waits). */
VLJ_API vlj_status vlj_debug_kernels_executed(vlj_sim *sim, uint64_t *kernels);
/* The last measurement's per-particle float4 (vx, vy, vz, drawn value), in
 * input order (n x 4 floats); waits. */
VLJ_API vlj_status vlj_debug_read_vel4(vlj_sim *sim, float *out);
/* 0: enqueue steps as direct launches instead of CUDA graphs. */
VLJ_API vlj_status vlj_debug_set_graphs(vlj_sim *sim, int on);
/* While on, steps are direct launches with CUDA events around every launch
 * of the step kernel; vlj_debug_kernel_time returns their summed device time
 * and count since timing was switched on or last read. */
VLJ_API vlj_status vlj_debug_kernel_timing(vlj_sim *sim, int on);
VLJ_API vlj_status vlj_debug_kernel_time(vlj_sim *sim, double *total_ms, uint64_t *launches);
/* FP32 FMA throughput of the current device in TFLOP/s (a calibration kernel
 * of independent FMA chains on every SM). */
VLJ_API vlj_status vlj_debug_fp32_peak(double *tflops);
/* Cell tiles of the step kernel: single boxes of four or more particles per
 * cell on average created with the environment variable VLJ_TILES=1 (off by
 * default: slower than the per-particle gathers on the workloads measured).
 * set_tiles(sim, 0) switches the step kernel back to per-particle gathers
 * from the slot list (same trajectory to the bit); tile_info gives the
 * bricks per x-row, the bricks in all, the tile capacity (particles a block
 * stages) and the threads per block (all 0 without tiles). read_tile_lists
 * copies the 16-bit tile lists of the last rebuild, as vlj_debug_read_grid
 * reads the slot lists (capacity rounded up to 8 rows of `segment` x 8
 * entries: entry k of sorted position p at [(k / 8) * segment * 8 + p * 8 +
 * k % 8]). */
VLJ_API vlj_status vlj_debug_set_tiles(vlj_sim *sim, int on);
/* Particles per block of the step kernel: 64, 128 (the default) or 256 (a
 * tuning knob: virial_lj.tune_batch times it per replica set; the same
 * trajectory to the bit). */
VLJ_API vlj_status vlj_debug_set_step_threads(vlj_sim *sim, uint32_t threads);
/* Lanes per particle of the step kernel: 0 (the default) chooses by grid
 * size (two lanes for grids of a few blocks per SM), 1 or 2 forces one form.
 * Every kernel sums a particle's force in two parts (the list's even and odd
 * rows) added once at the end, so the trajectory is the same to the bit
 * either way; the switch is for tests and timing. */
VLJ_API vlj_status vlj_debug_set_step_lanes(vlj_sim *sim, uint32_t lanes);
VLJ_API vlj_status vlj_debug_tile_info(vlj_sim *sim, uint32_t *brick_cols, uint32_t *bricks,
                                       uint32_t *tile_cap, uint32_t *threads);
VLJ_API vlj_status vlj_debug_read_tile_lists(vlj_sim *sim, uint16_t *out);
/* The Langevin noise stream as the device computes it (known-answer checks):
 * for k < n, out[4k..4k+3] = Philox-4x32-10 of counter ctr[4k..4k+3] and key
 * key[2k..2k+1], and noise[3k..3k+2] = the three Gaussian numbers the step
 * kernel draws for particle id ctr[4k] at step ctr[4k+1] + 2^32 ctr[4k+2]
 * with seed key[2k]. Host buffers; n at most 2^24; waits. */
VLJ_API vlj_status vlj_debug_philox(const uint32_t *ctr, const uint32_t *key, size_t n,
                                    uint32_t *out, float *noise);
/* The simulation that steps a batch's arena, for vlj_debug_set_graphs,
 * vlj_debug_kernel_timing / _time and vlj_debug_kernels_executed only (it
 * stays owned by the batch). */
VLJ_API vlj_status vlj_debug_batch_sim(vlj_batch *batch, vlj_sim **sim);

#ifdef __cplusplus
}
#endif
#endif
