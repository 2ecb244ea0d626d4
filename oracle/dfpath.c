/* The reference's plain double-float path, restated for the error table:
 * how far its own arithmetic lands from the f64 truth, next to the CUDA
 * path's. Test oracle only.
 *
 * State as the reference keeps it: positions and velocities as double-floats
 * (an f32 hi and an f32 lo each, Df64::from_f64 at set-up,
 * lennard_jones.rs:476-489), the acceleration in f32. Constant energy:
 *   half kick   v = df_add_f(v, a * dt/2)            (lennard_jones.wgsl:252)
 *   drift       x = df_add(x, df_mul_f(v, dt)); wrap  (lennard_jones.wgsl:260-262)
 *   forces      a = -sum d * (rf / r2) over pairs in f32, the separation
 *               d = nearest((pj.hi - xh) + (unpack(pj) - xl)) from the packed
 *               position of the neighbour (9-bit lo) and the full lo of the
 *               particle itself, pair(r2) as written (lennard_jones.wgsl:503-545)
 *   half kick   v = df_add_f(v, a * dt/2)            (lennard_jones.wgsl:567-574)
 * and the measurement: per particle pe += u/2 and w += rf/2 as df_add_f
 * (lennard_jones.wgsl:518-519), kinetic energy from the double-float
 * velocity. Every f32 operation is rounded as written (-ffp-contract=off).
 *
 * Pairs: the reference walks a Verlet list built on the same separation; a
 * pair inside the cutoff is in it for as long as the list is valid, so the
 * pairs here are those of the 27-cell stencil of a grid rebuilt before every
 * force pass (cells at least cutoff wide), walked cell by cell in the
 * reference's stencil order and by slot within a cell. The order of the f32
 * sums can differ from a list built some steps earlier, by rounding only.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "vlj_oracle.h"

struct vo_dfmd {
    uint32_t n;
    float box[3];
    float rc2, shift, force_shift, rc, dt, half_dt;
    int shifted_force;
    uint32_t cells[3];
    float cell_size[3];
    vo_df *x, *v;  /* 3 per particle */
    float *a;      /* 3 per particle */
    /* grid scratch */
    uint32_t *cell_of, *start, *sorted;
};

static float nearest1(float d, float side) {
    float r = rintf(d / side);
    float m = side * r;
    return d - m;
}

/* r . F and u of a pair at r2 < rc2 (lennard_jones.wgsl:531-545) */
static void pair(const vo_dfmd *m, float r2, float *rf, float *u) {
    float inv2 = 1.0f / r2;
    float s6 = inv2 * inv2 * inv2;
    float s12 = s6 * s6;
    float f = 24.0f * (2.0f * s12 - s6);
    float e = 4.0f * (s12 - s6) - m->shift;
    if (m->shifted_force) {
        float r = sqrtf(r2);
        f = f - r * m->force_shift;
        e = e + (r - m->rc) * m->force_shift;
    }
    *rf = f;
    *u = e;
}

static void bin(vo_dfmd *m) {
    const uint32_t total = m->cells[0] * m->cells[1] * m->cells[2];
    memset(m->start, 0, sizeof(uint32_t) * (total + 1));
    for (uint32_t i = 0; i < m->n; i++) {
        uint32_t c[3];
        for (int k = 0; k < 3; k++) {
            int32_t q = (int32_t)floorf(m->x[3 * i + k].hi / m->cell_size[k]);
            int32_t top = (int32_t)m->cells[k] - 1;
            c[k] = (uint32_t)(q < 0 ? 0 : (q > top ? top : q));
        }
        m->cell_of[i] = (c[2] * m->cells[1] + c[1]) * m->cells[0] + c[0];
        m->start[m->cell_of[i] + 1] += 1u;
    }
    for (uint32_t c = 0; c < total; c++) m->start[c + 1] += m->start[c];
    uint32_t *cursor = malloc(sizeof(uint32_t) * total);
    memcpy(cursor, m->start, sizeof(uint32_t) * total);
    for (uint32_t i = 0; i < m->n; i++) m->sorted[cursor[m->cell_of[i]]++] = i;
    free(cursor);
}

/* Forces (and, with pe / w, the per-particle halves summed as double-floats,
 * then in f64 over particles) from the current positions. */
static void forces(vo_dfmd *m, double *pe, double *w) {
    bin(m);
    const int32_t nx = (int32_t)m->cells[0], ny = (int32_t)m->cells[1], nz = (int32_t)m->cells[2];
    double pe_sum = 0.0, w_sum = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pe_sum, w_sum)
    for (uint32_t i = 0; i < m->n; i++) {
        float xh[3], xl[3];
        for (int k = 0; k < 3; k++) {
            xh[k] = m->x[3 * i + k].hi;
            xl[k] = m->x[3 * i + k].lo;
        }
        const int32_t ci = (int32_t)m->cell_of[i];
        const int32_t cc[3] = {ci % nx, (ci / nx) % ny, ci / (nx * ny)};
        float acc[3] = {0.0f, 0.0f, 0.0f};
        vo_df pei = {0.0f, 0.0f}, wi = {0.0f, 0.0f};
        for (int32_t dz = -1; dz <= 1; dz++)
            for (int32_t dy = -1; dy <= 1; dy++)
                for (int32_t dx = -1; dx <= 1; dx++) {
                    const uint32_t ncx = (uint32_t)((cc[0] + dx + nx) % nx);
                    const uint32_t ncy = (uint32_t)((cc[1] + dy + ny) % ny);
                    const uint32_t ncz = (uint32_t)((cc[2] + dz + nz) % nz);
                    const uint32_t cell = (ncz * (uint32_t)ny + ncy) * (uint32_t)nx + ncx;
                    for (uint32_t t = m->start[cell]; t < m->start[cell + 1]; t++) {
                        const uint32_t j = m->sorted[t];
                        if (j == i) continue;
                        float ph[3], pl[3], ulo[3];
                        for (int k = 0; k < 3; k++) {
                            ph[k] = m->x[3 * j + k].hi;
                            pl[k] = m->x[3 * j + k].lo;
                        }
                        vo_unpack_lo(ph, vo_pack_lo(ph, pl), ulo);
                        float d[3];
                        for (int k = 0; k < 3; k++) {
                            float a = ph[k] - xh[k];
                            float b = ulo[k] - xl[k];
                            d[k] = nearest1(a + b, m->box[k]);
                        }
                        float r2 = d[0] * d[0];
                        r2 = r2 + d[1] * d[1];
                        r2 = r2 + d[2] * d[2];
                        if (!(r2 < m->rc2)) continue;
                        float rf, u;
                        pair(m, r2, &rf, &u);
                        const float q = rf / r2;
                        for (int k = 0; k < 3; k++) acc[k] = acc[k] - d[k] * q;
                        if (pe) {
                            pei = vo_df_add_f(pei, 0.5f * u);
                            wi = vo_df_add_f(wi, 0.5f * rf);
                        }
                    }
                }
        for (int k = 0; k < 3; k++) m->a[3 * i + k] = acc[k];
        if (pe) {
            pe_sum += vo_df_to_f64(pei);
            w_sum += vo_df_to_f64(wi);
        }
    }
    if (pe) {
        *pe = pe_sum;
        *w = w_sum;
    }
}

static vo_df wrap(vo_df x, float side) {
    if (x.hi >= side) return vo_df_add_f(x, -side);
    if (x.hi < 0.0f) return vo_df_add_f(x, side);
    return x;
}

vo_dfmd *vo_dfmd_create(const double *pos, const double *vel, uint32_t n, const double box[3],
                        double cutoff, int shifted_force, double dt) {
    vo_dfmd *m = calloc(1, sizeof(vo_dfmd));
    m->n = n;
    for (int k = 0; k < 3; k++) {
        m->box[k] = (float)box[k];
        /* cells at least the cutoff wide, three or more per axis so the
         * stencil visits 27 distinct cells */
        const uint32_t c = (uint32_t)floor((double)m->box[k] / cutoff);
        if (c < 3u) {
            free(m);
            return NULL;
        }
        m->cells[k] = c;
        m->cell_size[k] = m->box[k] / (float)m->cells[k];
    }
    /* set-up constants in f64 rounded to f32, as lennard_jones.rs:507-515 */
    const double rc2 = cutoff * cutoff;
    const double s6 = 1.0 / (rc2 * rc2 * rc2);
    m->rc = (float)cutoff;
    m->rc2 = (float)rc2;
    m->shifted_force = shifted_force;
    m->force_shift = shifted_force ? (float)(24.0 * (2.0 * s6 * s6 - s6) / cutoff) : 0.0f;
    m->shift = (float)(4.0 * (s6 * s6 - s6));
    m->dt = (float)dt;
    m->half_dt = (float)(0.5 * dt);
    m->x = malloc(sizeof(vo_df) * 3 * (size_t)n);
    m->v = malloc(sizeof(vo_df) * 3 * (size_t)n);
    m->a = malloc(sizeof(float) * 3 * (size_t)n);
    m->cell_of = malloc(sizeof(uint32_t) * n);
    m->sorted = malloc(sizeof(uint32_t) * n);
    m->start = malloc(sizeof(uint32_t) * (m->cells[0] * m->cells[1] * m->cells[2] + 1));
    for (size_t q = 0; q < 3 * (size_t)n; q++) {
        const int k = (int)(q % 3);
        double x = fmod(pos[q], (double)m->box[k]);
        if (x < 0.0) x += (double)m->box[k];
        m->x[q] = vo_df_from_f64(x);
        m->v[q] = vo_df_from_f64(vel[q]);
    }
    forces(m, NULL, NULL);  /* a(0) for the first half kick (lennard_jones.rs:1080-1089) */
    return m;
}

void vo_dfmd_run(vo_dfmd *m, uint64_t steps) {
    for (uint64_t s = 0; s < steps; s++) {
        for (size_t q = 0; q < 3 * (size_t)m->n; q++) {
            const int k = (int)(q % 3);
            m->v[q] = vo_df_add_f(m->v[q], m->a[q] * m->half_dt);
            m->x[q] = wrap(vo_df_add(m->x[q], vo_df_mul_f(m->v[q], m->dt)), m->box[k]);
        }
        forces(m, NULL, NULL);
        for (size_t q = 0; q < 3 * (size_t)m->n; q++)
            m->v[q] = vo_df_add_f(m->v[q], m->a[q] * m->half_dt);
    }
}

/* kinetic, potential, virial of the current state; positions (wrapped) and
 * velocities as f64 into pos / vel when given */
void vo_dfmd_measure(vo_dfmd *m, double out[3], double *pos, double *vel) {
    double pe = 0.0, w = 0.0, ke = 0.0;
    forces(m, &pe, &w);
    for (size_t q = 0; q < 3 * (size_t)m->n; q++) {
        const double v = vo_df_to_f64(m->v[q]);
        ke += 0.5 * v * v;
        if (pos) pos[q] = vo_df_to_f64(m->x[q]);
        if (vel) vel[q] = v;
    }
    out[0] = ke;
    out[1] = pe;
    out[2] = w;
}

void vo_dfmd_destroy(vo_dfmd *m) {
    if (!m) return;
    free(m->x);
    free(m->v);
    free(m->a);
    free(m->cell_of);
    free(m->sorted);
    free(m->start);
    free(m);
}
