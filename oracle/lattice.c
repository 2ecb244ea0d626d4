/*
 * Lattice generators: crates/virial-particles/src/lennard_jones.rs:1379-1441
 * (simple cubic and box-filling lattices with xorshift64 + Box-Muller
 * velocities and zero net momentum), plus an fcc lattice that uses the same
 * velocity stream. Test oracle only (see vlj_oracle.h).
 */
#include "vlj_oracle.h"

#include <math.h>

typedef struct {
    uint64_t s;
} xorshift;

/* lennard_jones.rs:1410-1415: uniform in (0, 1) from 53 bits */
static double xs_random(xorshift *r) {
    r->s ^= r->s << 13;
    r->s ^= r->s >> 7;
    r->s ^= r->s << 17;
    return ((double)(r->s >> 11) + 0.5) / 9007199254740992.0;
}

/* lennard_jones.rs:1416-1419: one Box-Muller gaussian per two uniforms */
static double xs_gaussian(xorshift *r) {
    double radius = sqrt(-2.0 * log(xs_random(r)));
    return radius * cos(6.283185307179586 * xs_random(r));
}

/* lennard_jones.rs:1433-1439: subtract the mean velocity */
static void zero_momentum(size_t count, double *vel) {
    double mean[3];
    for (int k = 0; k < 3; k++) {
        double sum = 0.0;
        for (size_t i = 0; i < count; i++) sum += vel[3 * i + k];
        mean[k] = sum / (double)count;
    }
    for (size_t i = 0; i < count; i++)
        for (int k = 0; k < 3; k++) vel[3 * i + k] -= mean[k];
}

/* lennard_jones.rs:1401-1441 */
static void lattice_sites(size_t count, const double size[3], const size_t sites[3],
                          double temperature, uint64_t seed, double *pos, double *vel) {
    double gap[3];
    for (int k = 0; k < 3; k++) gap[k] = size[k] / (double)sites[k];
    xorshift r = {seed | 1u};
    double root_t = sqrt(temperature);
    for (size_t i = 0; i < count; i++) {
        size_t c[3] = {i % sites[0], (i / sites[0]) % sites[1], i / (sites[0] * sites[1])};
        for (int k = 0; k < 3; k++) pos[3 * i + k] = ((double)c[k] + 0.5) * gap[k];
        for (int k = 0; k < 3; k++) vel[3 * i + k] = xs_gaussian(&r) * root_t;
    }
    zero_momentum(count, vel);
}

/* lennard_jones.rs:1379-1382 */
void vo_lattice(size_t count, double box_size, double temperature, uint64_t seed, double *pos,
                double *vel) {
    size_t per_side = (size_t)ceil(cbrt((double)count));
    double size[3] = {box_size, box_size, box_size};
    size_t sites[3] = {per_side, per_side, per_side};
    lattice_sites(count, size, sites, temperature, seed, pos, vel);
}

/* lennard_jones.rs:1388-1399. Rust's max_by returns the last of equal
 * maxima, so ties go to the later axis. */
void vo_lattice_box(size_t count, const double size[3], double temperature, uint64_t seed,
                    double *pos, double *vel) {
    double spacing = cbrt(size[0] * size[1] * size[2] / (double)count);
    size_t sites[3];
    for (int k = 0; k < 3; k++) {
        double s = round(size[k] / spacing);
        sites[k] = s < 1.0 ? 1 : (size_t)s;
    }
    while (sites[0] * sites[1] * sites[2] < count) {
        int widest = 0;
        for (int k = 1; k < 3; k++) {
            double a = size[widest] / (double)sites[widest];
            double b = size[k] / (double)sites[k];
            if (!(a > b)) widest = k;
        }
        sites[widest] += 1;
    }
    lattice_sites(count, size, sites, temperature, seed, pos, vel);
}

/* fcc: four sites per cubic cell, offset a quarter cell so no site sits on a
 * face. Particle 4 * ((cz * cells + cy) * cells + cx) + b. */
void vo_lattice_fcc(uint32_t cells, double density, double temperature, uint64_t seed,
                    double *pos, double *vel, double *box_size) {
    static const double basis[4][3] = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.5, 0.0, 0.5},
                                       {0.0, 0.5, 0.5}};
    double a = cbrt(4.0 / density);
    *box_size = (double)cells * a;
    xorshift r = {seed | 1u};
    double root_t = sqrt(temperature);
    size_t i = 0;
    for (uint32_t cz = 0; cz < cells; cz++)
        for (uint32_t cy = 0; cy < cells; cy++)
            for (uint32_t cx = 0; cx < cells; cx++)
                for (int b = 0; b < 4; b++, i++) {
                    double c[3] = {(double)cx, (double)cy, (double)cz};
                    for (int k = 0; k < 3; k++) pos[3 * i + k] = (c[k] + basis[b][k] + 0.25) * a;
                    for (int k = 0; k < 3; k++) vel[3 * i + k] = xs_gaussian(&r) * root_t;
                }
    zero_momentum(i, vel);
}
