/*
 * vlj_oracle.h -- CPU test oracle for the Lennard-Jones step of
 * virial_particles::lennard_jones (anshullaikar/virial-engine).
 *
 * TEST INFRASTRUCTURE ONLY. The CUDA library never links, loads or calls
 * anything here. Only the tests, the smoke check and the CPU baseline leg of
 * the benchmark use it, and only to check or to time against.
 *
 * What it restates (file:line in the reference project):
 *   - 32.32 fixed point: crates/virial-precision/src/fixed.wgsl:20-65,
 *     fixed.rs:9-67
 *   - double-float arithmetic: crates/virial-precision/src/df64.rs:15-131
 *     (the Rust mirror of df64.wgsl:17-116)
 *   - packed positions: crates/virial-particles/src/lennard_jones.wgsl:128-152
 *   - per-particle PCG stream: lennard_jones.wgsl:168-184, seeding
 *     lennard_jones.rs:584-592
 *   - lattices: lennard_jones.rs:1379-1441
 *   - box / grid / list set-up: lennard_jones.rs:443-560
 *   - cell binning and per-cell order: crates/virial-particles/src/grid.wgsl:11-148
 *   - reorder and Verlet-list build: lennard_jones.wgsl:281-307, 421-499
 *   - f64 pair sums used by the reference tests as their truth:
 *     crates/virial-particles/tests/thermodynamics.rs:21-53,
 *     tests/coexistence.rs:39-76, tests/heat.rs:40-91
 *
 * New here (no counterpart in the reference): the Philox-4x32-10 counter RNG
 * keyed by (seed, step, particle id) that the CUDA path uses for Langevin
 * noise, an fcc lattice, and an f64 cell-list molecular-dynamics engine with
 * the same integrator and rebuild rule as the CUDA path, parallelised with
 * OpenMP. That engine is the timed CPU baseline.
 *
 * Positions and velocities are n x 3 row-major doubles (x0 y0 z0 x1 ...).
 * Build: see oracle/Makefile (gcc, -ffp-contract=off so every f32 operation
 * is rounded exactly as written).
 */
#ifndef VLJ_ORACLE_H
#define VLJ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- 32.32 fixed point ---- */
void vo_fixed_split(float x, uint32_t *low, uint32_t *high);
int64_t vo_fixed_to_raw(float x);
int64_t vo_fixed_from_words(uint32_t low, uint32_t high);
double vo_fixed_to_f64(int64_t raw);
/* Round-to-nearest-even of x * 2^32 for an f64 value (|x| < 2^31). */
int64_t vo_fixed_raw_f64(double x);

/* ---- double-float (hi + lo) ---- */
typedef struct {
    float hi, lo;
} vo_df;
vo_df vo_df_from_f64(double x);
double vo_df_to_f64(vo_df a);
vo_df vo_df_add(vo_df a, vo_df b);
vo_df vo_df_sub(vo_df a, vo_df b);
vo_df vo_df_mul(vo_df a, vo_df b);
vo_df vo_df_div(vo_df a, vo_df b);
vo_df vo_df_sqrt(vo_df a);
vo_df vo_df_add_f(vo_df a, float b);
vo_df vo_df_mul_f(vo_df a, float b);

/* ---- packed positions (hi in xyz, lo as three 9-bit fractions) ---- */
float vo_last_bit(float h);
uint32_t vo_pack_lo(const float hi[3], const float lo[3]);
void vo_unpack_lo(const float hi[3], uint32_t bits, float lo[3]);

/* ---- random numbers ---- */
uint32_t vo_pcg(uint32_t *state);
float vo_uniform01(uint32_t *state);
void vo_gaussian2(uint32_t *state, float out[2]);
uint32_t vo_pcg_seed(uint32_t seed, uint32_t index);
void vo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* The three Langevin gaussians of particle `id` at MD step `step`. */
void vo_langevin_noise(uint32_t seed, uint64_t step, uint32_t id, float out[3]);

/* ---- lattices ---- */
void vo_lattice(size_t count, double box_size, double temperature, uint64_t seed,
                double *pos, double *vel);
void vo_lattice_box(size_t count, const double size[3], double temperature, uint64_t seed,
                    double *pos, double *vel);
/* fcc: cells^3 unit cells x 4 sites at number density `density`; writes the
 * cube side to *box_size. Velocities as in vo_lattice. */
void vo_lattice_fcc(uint32_t cells, double density, double temperature, uint64_t seed,
                    double *pos, double *vel, double *box_size);

/* ---- set-up: what LennardJones::new derives from the settings ---- */
typedef struct {
    uint32_t n;
    double box[3];        /* sides rounded to f32 */
    float box_f[3];
    uint32_t cells[3];
    uint32_t total_cells;
    float cell_size_f[3];
    uint32_t segment;
    uint32_t capacity;
    double cutoff, skin;
    float rc2, list_r2, half_skin2;
    float shift, force_shift;
    double energy_scale, momentum_scale;
} vo_setup;

/* thermostat_temperature <= 0 means constant energy (no thermostat). Returns
 * 0, or 1 when a side holds fewer than three (cutoff + skin) widths. */
int vo_setup_compute(uint32_t n, const double *vel, const double box[3], double cutoff,
                     double skin, int shifted_force, double thermostat_temperature,
                     vo_setup *out);

/* ---- one neighbour-list rebuild, exactly as the reference orders it ----
 * Slots hold particles; x, v, ids are in slot order and are permuted in place
 * when `reorder` is set (every fourth rebuild in the reference). Outputs:
 * cell_of_slot[n], cell_start[total_cells + 1], sorted[n], list_count[n],
 * list[n * capacity] (row i holds slot i's neighbours in build order), and the
 * largest neighbour count that did not fit (0 when none). */
void vo_rebuild_ref(const vo_setup *s, uint32_t n, double *x, double *v, uint32_t *ids,
                    int reorder, uint32_t *cell_of_slot, uint32_t *cell_start,
                    uint32_t *sorted, uint32_t *list_count, uint32_t *list,
                    uint32_t *overflow);

/* ---- f64 truth ---- */
/* Potential energy and virial tensor diagonal over all pairs within cutoff,
 * nearest image, O(n^2). */
void vo_all_pairs(const double *pos, uint32_t n, const double box[3], double cutoff,
                  int shifted_force, double *pe, double w[3]);
/* Same sums through a cell grid (any n; needs every side >= 2 * cutoff). */
void vo_cell_pairs(const double *pos, uint32_t n, const double box[3], double cutoff,
                   int shifted_force, double *pe, double w[3]);
/* Heat current J = sum_i e_i v_i + 1/2 sum_i sum_j (F_ij . v_i) r_ij, O(n^2). */
void vo_heat_current(const double *pos, const double *vel, uint32_t n, const double box[3],
                     double cutoff, int shifted_force, double j[3]);
/* Irving-Kirkwood profile sums in f64 over all pairs: per slab `bins` x 8
 * values (count, m v_a^2, W_aa, PE) and 3 whole-box W_aa, as one sample. */
void vo_profile(const double *pos, const double *vel, uint32_t n, const double box[3],
                double cutoff, int shifted_force, uint32_t bins, double *out);

/* ---- f64 cell-list molecular dynamics (the CPU baseline) ---- */
typedef struct vo_md vo_md;
typedef struct {
    uint64_t step;
    double kinetic, potential, virial, momentum[3];
    uint32_t list_rebuilds;
    double thermostat_energy; /* Nose-Hoover: Q xi^2 / 2 + g k T eta */
} vo_md_measurement;

/* thermostat: 0 constant energy, 1 Langevin (temperature, friction, seed),
 * 2 Nose-Hoover (temperature, `friction` read as the period). */
vo_md *vo_md_create(const double *pos, const double *vel, uint32_t n, const double box[3],
                    double cutoff, double skin, double dt, int shifted_force,
                    int thermostat, double temperature, double friction, uint32_t seed);
void vo_md_destroy(vo_md *md);
void vo_md_run(vo_md *md, uint64_t steps);
void vo_md_measure(vo_md *md, vo_md_measurement *out);
/* Canonical positions and velocities in input order. */
void vo_md_read(vo_md *md, double *pos, double *vel);
/* Heat exchange (eHEX/a) from the next step on: slabs = hot lo, hi, cold lo,
 * hi in z; energy moved per step; on = 0 stops it. Constant energy only. */
void vo_md_set_heat_exchange(vo_md *md, int on, const double slabs[4], double energy);
void vo_md_set_threads(int threads);
int vo_md_threads(void);


/* The reference's plain double-float path (dfpath.c), constant energy:
 * double-float state, f32 pair arithmetic on packed positions, df64 sums.
 * NULL when the box is under three cutoffs wide on some axis. measure gives
 * kinetic, potential and virial, and the state as f64 into pos / vel (either
 * may be NULL). */
typedef struct vo_dfmd vo_dfmd;
vo_dfmd *vo_dfmd_create(const double *pos, const double *vel, uint32_t n, const double box[3],
                        double cutoff, int shifted_force, double dt);
void vo_dfmd_run(vo_dfmd *m, uint64_t steps);
void vo_dfmd_measure(vo_dfmd *m, double out[3], double *pos, double *vel);
void vo_dfmd_destroy(vo_dfmd *m);

#ifdef __cplusplus
}
#endif
#endif
