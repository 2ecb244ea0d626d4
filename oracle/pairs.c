/*
 * f64 truth for the pair sums: the sums the reference's own tests compute on
 * the CPU and compare the GPU against.
 *   potential + virial tensor: crates/virial-particles/tests/coexistence.rs:38-76
 *   (and tests/thermodynamics.rs:20-53 for the truncated-shifted scalar form)
 *   heat current: tests/heat.rs:39-90
 *   Irving-Kirkwood profile: the semantics of lennard_jones.wgsl:644-730 in f64
 * Test oracle only (see vlj_oracle.h).
 */
#include "vlj_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* coexistence.rs:39-53: (potential, r . F), shifted as the GPU does */
static void pair_f64(double r2, double cutoff, int shifted_force, double *u_out, double *rf_out) {
    double s6 = 1.0 / (r2 * r2 * r2);
    double u = 4.0 * (s6 * s6 - s6);
    double rf = 24.0 * (2.0 * s6 * s6 - s6);
    double rc2 = cutoff * cutoff;
    double sc6 = 1.0 / (rc2 * rc2 * rc2);
    double uc = 4.0 * (sc6 * sc6 - sc6);
    double rfc = 24.0 * (2.0 * sc6 * sc6 - sc6);
    if (shifted_force) {
        double r = sqrt(r2);
        double fc = rfc / cutoff;
        *u_out = u - uc + (r - cutoff) * fc;
        *rf_out = rf - r * fc;
    } else {
        *u_out = u - uc;
        *rf_out = rf;
    }
}

static double nearest_f64(double x, double side) { return x - side * round(x / side); }

void vo_all_pairs(const double *pos, uint32_t n, const double box[3], double cutoff,
                  int shifted_force, double *pe, double w[3]) {
    double e = 0.0, t[3] = {0.0, 0.0, 0.0};
    double rc2 = cutoff * cutoff;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = i + 1; j < n; j++) {
            double d[3];
            for (int k = 0; k < 3; k++)
                d[k] = nearest_f64(pos[3 * (size_t)j + k] - pos[3 * (size_t)i + k], box[k]);
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (r2 < rc2) {
                double u, rf;
                pair_f64(r2, cutoff, shifted_force, &u, &rf);
                e += u;
                for (int k = 0; k < 3; k++) t[k] += d[k] * d[k] * rf / r2;
            }
        }
    *pe = e;
    for (int k = 0; k < 3; k++) w[k] = t[k];
}

typedef struct {
    uint32_t cells[3], total;
    uint32_t *start, *order;
} f64_grid;

/* A cell grid with cells at least `radius` wide; returns 0 when some side has
 * fewer than three cells (callers then fall back to all pairs). */
static int grid_build(const double *pos, uint32_t n, const double box[3], double radius,
                      f64_grid *g) {
    for (int k = 0; k < 3; k++) {
        double c = floor(box[k] / radius);
        g->cells[k] = c < 0.0 ? 0u : (uint32_t)c;
        if (g->cells[k] < 3) return 0;
    }
    g->total = g->cells[0] * g->cells[1] * g->cells[2];
    g->start = calloc((size_t)g->total + 1, sizeof(uint32_t));
    g->order = malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    uint32_t *cell = malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    for (uint32_t i = 0; i < n; i++) {
        uint32_t c[3];
        for (int k = 0; k < 3; k++) {
            double f = floor(pos[3 * (size_t)i + k] / (box[k] / (double)g->cells[k]));
            int64_t v = (int64_t)f;
            if (v < 0) v = 0;
            if (v > (int64_t)g->cells[k] - 1) v = (int64_t)g->cells[k] - 1;
            c[k] = (uint32_t)v;
        }
        cell[i] = (c[2] * g->cells[1] + c[1]) * g->cells[0] + c[0];
        g->start[cell[i] + 1] += 1;
    }
    for (uint32_t c = 0; c < g->total; c++) g->start[c + 1] += g->start[c];
    uint32_t *fill = calloc(g->total, sizeof(uint32_t));
    for (uint32_t i = 0; i < n; i++) g->order[g->start[cell[i]] + fill[cell[i]]++] = i;
    free(fill);
    free(cell);
    return 1;
}

static void grid_free(f64_grid *g) {
    free(g->start);
    free(g->order);
}

void vo_cell_pairs(const double *pos, uint32_t n, const double box[3], double cutoff,
                   int shifted_force, double *pe, double w[3]) {
    f64_grid g;
    if (!grid_build(pos, n, box, cutoff, &g)) {
        vo_all_pairs(pos, n, box, cutoff, shifted_force, pe, w);
        return;
    }
    double rc2 = cutoff * cutoff;
    double e = 0.0, t[3] = {0.0, 0.0, 0.0};
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : e, t[:3])
    for (uint32_t c = 0; c < g.total; c++) {
        int32_t cx = (int32_t)(c % g.cells[0]), cy = (int32_t)((c / g.cells[0]) % g.cells[1]),
                cz = (int32_t)(c / (g.cells[0] * g.cells[1]));
        for (uint32_t a = g.start[c]; a < g.start[c + 1]; a++) {
            uint32_t i = g.order[a];
            for (int dz = -1; dz <= 1; dz++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dx = -1; dx <= 1; dx++) {
                        uint32_t nxc = (uint32_t)((cx + dx + (int32_t)g.cells[0]) % (int32_t)g.cells[0]);
                        uint32_t nyc = (uint32_t)((cy + dy + (int32_t)g.cells[1]) % (int32_t)g.cells[1]);
                        uint32_t nzc = (uint32_t)((cz + dz + (int32_t)g.cells[2]) % (int32_t)g.cells[2]);
                        uint32_t nc = (nzc * g.cells[1] + nyc) * g.cells[0] + nxc;
                        for (uint32_t b = g.start[nc]; b < g.start[nc + 1]; b++) {
                            uint32_t j = g.order[b];
                            if (j <= i) continue;
                            double d[3];
                            for (int k = 0; k < 3; k++)
                                d[k] = nearest_f64(pos[3 * (size_t)j + k] - pos[3 * (size_t)i + k],
                                                   box[k]);
                            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                            if (r2 < rc2) {
                                double u, rf;
                                pair_f64(r2, cutoff, shifted_force, &u, &rf);
                                e += u;
                                for (int k = 0; k < 3; k++) t[k] += d[k] * d[k] * rf / r2;
                            }
                        }
                    }
        }
    }
    grid_free(&g);
    *pe = e;
    for (int k = 0; k < 3; k++) w[k] = t[k];
}

/* tests/heat.rs:54-90 */
void vo_heat_current(const double *pos, const double *vel, uint32_t n, const double box[3],
                     double cutoff, int shifted_force, double j_out[3]) {
    double *energy = malloc(sizeof(double) * (size_t)(n ? n : 1));
    double *pairs = calloc(3 * (size_t)(n ? n : 1), sizeof(double));
    double rc2 = cutoff * cutoff;
    for (uint32_t i = 0; i < n; i++) {
        double v2 = 0.0;
        for (int k = 0; k < 3; k++) v2 += vel[3 * (size_t)i + k] * vel[3 * (size_t)i + k];
        energy[i] = 0.5 * v2;
    }
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = i + 1; j < n; j++) {
            double d[3];
            for (int k = 0; k < 3; k++)
                d[k] = nearest_f64(pos[3 * (size_t)j + k] - pos[3 * (size_t)i + k], box[k]);
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (r2 >= rc2) continue;
            double u, rf;
            pair_f64(r2, cutoff, shifted_force, &u, &rf);
            energy[i] += 0.5 * u;
            energy[j] += 0.5 * u;
            double dvi = 0.0, dvj = 0.0;
            for (int k = 0; k < 3; k++) {
                dvi += d[k] * vel[3 * (size_t)i + k];
                dvj += d[k] * vel[3 * (size_t)j + k];
            }
            for (int k = 0; k < 3; k++) {
                pairs[3 * (size_t)i + k] += d[k] * dvi * rf / r2;
                pairs[3 * (size_t)j + k] += d[k] * dvj * rf / r2;
            }
        }
    for (int k = 0; k < 3; k++) {
        double s = 0.0;
        for (uint32_t i = 0; i < n; i++)
            s += energy[i] * vel[3 * (size_t)i + k] + 0.5 * pairs[3 * (size_t)i + k];
        j_out[k] = s;
    }
    free(energy);
    free(pairs);
}

/* Irving-Kirkwood slab profile, lennard_jones.wgsl:644-730 in f64 over all
 * ordered pairs: each particle books its count, m v_a^2 and half of each pair
 * energy into its own slab, and half of each pair's virial tensor along the
 * line to the partner, split over the slabs the line crosses in proportion to
 * the length inside each (the last slab takes what is left). */
void vo_profile(const double *pos, const double *vel, uint32_t n, const double box[3],
                double cutoff, int shifted_force, uint32_t bins, double *out) {
    const int slots = 8;
    memset(out, 0, sizeof(double) * ((size_t)bins * slots + 3));
    double width = box[2] / (double)bins;
    double rc2 = cutoff * cutoff;
    for (uint32_t i = 0; i < n; i++) {
        double z = pos[3 * (size_t)i + 2];
        int64_t h = (int64_t)floor(z / width);
        if (h < 0) h = 0;
        if (h > (int64_t)bins - 1) h = (int64_t)bins - 1;
        double *home = out + (size_t)h * slots;
        home[0] += 1.0;
        for (int k = 0; k < 3; k++) home[1 + k] += vel[3 * (size_t)i + k] * vel[3 * (size_t)i + k];
        double pe = 0.0;
        for (uint32_t j = 0; j < n; j++) {
            if (j == i) continue;
            double d[3];
            for (int k = 0; k < 3; k++)
                d[k] = nearest_f64(pos[3 * (size_t)j + k] - pos[3 * (size_t)i + k], box[k]);
            double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (r2 >= rc2) continue;
            double u, rf;
            pair_f64(r2, cutoff, shifted_force, &u, &rf);
            pe += 0.5 * u;
            double wk[3];
            for (int k = 0; k < 3; k++) {
                wk[k] = 0.5 * d[k] * d[k] * (rf / r2);
                out[(size_t)bins * slots + k] += wk[k];
            }
            double lo = z + (d[2] < 0.0 ? d[2] : 0.0);
            double hi = z + (d[2] > 0.0 ? d[2] : 0.0);
            double length = hi - lo;
            if (length < 1e-6 * width) {
                for (int k = 0; k < 3; k++) home[4 + k] += wk[k];
                continue;
            }
            int64_t b = (int64_t)floor(lo / width);
            double left = 1.0;
            for (;;) {
                int last = (double)(b + 1) * width >= hi;
                double start = lo > (double)b * width ? lo : (double)b * width;
                double end = hi < (double)(b + 1) * width ? hi : (double)(b + 1) * width;
                double share = last ? left : (end - start) / length;
                if (share < 0.0) share = 0.0;
                left -= share;
                int64_t slab = ((b % (int64_t)bins) + (int64_t)bins) % (int64_t)bins;
                for (int k = 0; k < 3; k++) out[(size_t)slab * slots + 4 + k] += wk[k] * share;
                if (last) break;
                b += 1;
            }
        }
        home[7] += pe;
    }
}
