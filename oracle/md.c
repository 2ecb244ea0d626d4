/*
 * f64 cell-list molecular dynamics: the CPU baseline and the long-run oracle.
 *
 * Same model and control flow as the CUDA path: Verlet lists of everything
 * within cutoff + skin built from a cell grid, rebuilt when any particle has
 * moved more than skin / 2 since the last build (lennard_jones.wgsl:281-307),
 * velocity Verlet or BAOAB Langevin (lennard_jones.wgsl:225-276, 556-574)
 * with velocities stored half a kick behind so one force pass serves the
 * closing half kick of one step and the opening half kick of the next, and
 * Langevin noise from the Philox stream keyed by (seed, step, particle id);
 * or Nose-Hoover (lennard_jones.wgsl:309-397) on canonical velocities.
 * Everything is f64; particles are kept in cell order (reordered at every
 * rebuild) and the loops run under OpenMP. Test oracle only.
 */
#include "vlj_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct vo_md {
    uint32_t n;
    double box[3];
    double cutoff, rc2, skin, list_r2, half_skin2;
    double dt;
    int shifted_force;
    int thermostat;
    double c1, c2;
    /* Nose-Hoover: g k T, Q, and the thermostat's xi and eta */
    double nh_gkt, nh_q, xi, eta;
    /* heat exchange: on, slab bounds (hot lo, hi, cold lo, hi; f32 values),
     * energy per step (its f32 value) */
    int hex;
    float hex_slabs[4];
    double hex_energy;
    uint32_t seed;
    double uc, fc; /* U(rc) and F(rc) for the shifts */
    /* slot-ordered state: positions, velocities half a kick behind, ids */
    double *x, *vm, *xb, *a;
    uint32_t *ids;
    double *pe_i, *w_i;
    /* grid and lists */
    int use_grid;
    uint32_t cells[3], total;
    uint32_t *start, *cell, *order, *fill;
    uint32_t cap;
    uint32_t *nl, *nc;
    double *tmp;
    uint32_t *tmp_ids;
    uint64_t step;
    uint32_t rebuilds;
    int built;
};

static double nearest(double x, double side) { return x - side * round(x / side); }

static void pair(const vo_md *m, double r2, double *u, double *rf) {
    double s6 = 1.0 / (r2 * r2 * r2);
    *u = 4.0 * (s6 * s6 - s6) - m->uc;
    *rf = 24.0 * (2.0 * s6 * s6 - s6);
    if (m->shifted_force) {
        double r = sqrt(r2);
        *u += (r - m->cutoff) * m->fc;
        *rf -= r * m->fc;
    }
}

static void rebuild(vo_md *m) {
    uint32_t n = m->n;
    if (m->use_grid) {
        memset(m->fill, 0, sizeof(uint32_t) * m->total);
        memset(m->start, 0, sizeof(uint32_t) * ((size_t)m->total + 1));
        for (uint32_t i = 0; i < n; i++) {
            uint32_t c[3];
            for (int k = 0; k < 3; k++) {
                int64_t v = (int64_t)floor(m->x[3 * (size_t)i + k] / (m->box[k] / (double)m->cells[k]));
                if (v < 0) v = 0;
                if (v > (int64_t)m->cells[k] - 1) v = (int64_t)m->cells[k] - 1;
                c[k] = (uint32_t)v;
            }
            m->cell[i] = (c[2] * m->cells[1] + c[1]) * m->cells[0] + c[0];
            m->start[m->cell[i] + 1] += 1;
        }
        for (uint32_t c = 0; c < m->total; c++) m->start[c + 1] += m->start[c];
        for (uint32_t i = 0; i < n; i++)
            m->order[m->start[m->cell[i]] + m->fill[m->cell[i]]++] = i;
        /* move particles into cell order: neighbours then sit close in memory */
        double *arrays[2] = {m->x, m->vm};
        for (int a = 0; a < 2; a++) {
            for (uint32_t t = 0; t < n; t++)
                for (int k = 0; k < 3; k++)
                    m->tmp[3 * (size_t)t + k] = arrays[a][3 * (size_t)m->order[t] + k];
            memcpy(arrays[a], m->tmp, sizeof(double) * 3 * (size_t)n);
        }
        for (uint32_t t = 0; t < n; t++) m->tmp_ids[t] = m->ids[m->order[t]];
        memcpy(m->ids, m->tmp_ids, sizeof(uint32_t) * n);
        for (uint32_t t = 0; t < n; t++) m->tmp_ids[t] = m->cell[m->order[t]];
        memcpy(m->cell, m->tmp_ids, sizeof(uint32_t) * n);
    }
    for (;;) {
        uint32_t worst = 0;
#pragma omp parallel for schedule(static) reduction(max : worst)
        for (uint32_t i = 0; i < n; i++) {
            uint32_t found = 0;
            uint32_t *row = m->nl + (size_t)i * m->cap;
            const double *xi = m->x + 3 * (size_t)i;
            if (m->use_grid) {
                uint32_t c = m->cell[i];
                int32_t cx = (int32_t)(c % m->cells[0]), cy = (int32_t)((c / m->cells[0]) % m->cells[1]),
                        cz = (int32_t)(c / (m->cells[0] * m->cells[1]));
                for (int dz = -1; dz <= 1; dz++)
                    for (int dy = -1; dy <= 1; dy++)
                        for (int dx = -1; dx <= 1; dx++) {
                            uint32_t ax = (uint32_t)((cx + dx + (int32_t)m->cells[0]) % (int32_t)m->cells[0]);
                            uint32_t ay = (uint32_t)((cy + dy + (int32_t)m->cells[1]) % (int32_t)m->cells[1]);
                            uint32_t az = (uint32_t)((cz + dz + (int32_t)m->cells[2]) % (int32_t)m->cells[2]);
                            uint32_t nc = (az * m->cells[1] + ay) * m->cells[0] + ax;
                            for (uint32_t j = m->start[nc]; j < m->start[nc + 1]; j++) {
                                if (j == i) continue;
                                double d0 = nearest(m->x[3 * (size_t)j] - xi[0], m->box[0]);
                                double d1 = nearest(m->x[3 * (size_t)j + 1] - xi[1], m->box[1]);
                                double d2 = nearest(m->x[3 * (size_t)j + 2] - xi[2], m->box[2]);
                                if (d0 * d0 + d1 * d1 + d2 * d2 < m->list_r2) {
                                    if (found < m->cap) row[found] = j;
                                    found++;
                                }
                            }
                        }
            } else {
                for (uint32_t j = 0; j < n; j++) {
                    if (j == i) continue;
                    double d0 = nearest(m->x[3 * (size_t)j] - xi[0], m->box[0]);
                    double d1 = nearest(m->x[3 * (size_t)j + 1] - xi[1], m->box[1]);
                    double d2 = nearest(m->x[3 * (size_t)j + 2] - xi[2], m->box[2]);
                    if (d0 * d0 + d1 * d1 + d2 * d2 < m->list_r2) {
                        if (found < m->cap) row[found] = j;
                        found++;
                    }
                }
            }
            m->nc[i] = found;
            if (found > worst) worst = found;
        }
        if (worst <= m->cap) break;
        m->cap = worst + 16;
        free(m->nl);
        m->nl = malloc(sizeof(uint32_t) * (size_t)n * m->cap);
    }
    memcpy(m->xb, m->x, sizeof(double) * 3 * (size_t)n);
    m->built = 1;
    m->rebuilds += 1;
}

static int needs_rebuild(const vo_md *m) {
    if (!m->built) return 1;
    double worst = 0.0;
#pragma omp parallel for schedule(static) reduction(max : worst)
    for (uint32_t i = 0; i < m->n; i++) {
        double s = 0.0;
        for (int k = 0; k < 3; k++) {
            double d = nearest(m->x[3 * (size_t)i + k] - m->xb[3 * (size_t)i + k], m->box[k]);
            s += d * d;
        }
        if (s > worst) worst = s;
    }
    return worst > m->half_skin2;
}

/* Accelerations (mass 1) into m->a; with energies, each particle's half of
 * its pair energies and virials into pe_i / w_i. */
static void forces(vo_md *m, int energies) {
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < m->n; i++) {
        const double *xi = m->x + 3 * (size_t)i;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, pe = 0.0, w = 0.0;
        const uint32_t *row = m->nl + (size_t)i * m->cap;
        for (uint32_t k = 0; k < m->nc[i]; k++) {
            uint32_t j = row[k];
            double d0 = nearest(m->x[3 * (size_t)j] - xi[0], m->box[0]);
            double d1 = nearest(m->x[3 * (size_t)j + 1] - xi[1], m->box[1]);
            double d2 = nearest(m->x[3 * (size_t)j + 2] - xi[2], m->box[2]);
            double r2 = d0 * d0 + d1 * d1 + d2 * d2;
            if (r2 < m->rc2) {
                double u, rf;
                pair(m, r2, &u, &rf);
                double f = rf / r2;
                a0 -= d0 * f;
                a1 -= d1 * f;
                a2 -= d2 * f;
                pe += 0.5 * u;
                w += 0.5 * rf;
            }
        }
        m->a[3 * (size_t)i] = a0;
        m->a[3 * (size_t)i + 1] = a1;
        m->a[3 * (size_t)i + 2] = a2;
        if (energies) {
            m->pe_i[i] = pe;
            m->w_i[i] = w;
        }
    }
}

static double wrap(double x, double side) {
    if (x >= side) x -= side;
    if (x < 0.0) x += side;
    if (x >= side) x -= side;
    return x;
}

/* One Nose-Hoover half step (lennard_jones.wgsl:309-397, Tuckerman's
 * time-reversible splitting): xi a quarter step with the kinetic energy,
 * eta a half step, the velocity scale s = exp(-xi dt / 2), xi another quarter
 * step with the kinetic energy after scaling, then v <- s v. The velocities
 * here are the canonical ones. */
static void nh_half(vo_md *m) {
    double ke = 0.0;
#pragma omp parallel for reduction(+ : ke) schedule(static)
    for (size_t q = 0; q < 3 * (size_t)m->n; q++) ke += 0.5 * m->vm[q] * m->vm[q];
    double quarter = 0.25 * m->dt, half = 0.5 * m->dt;
    m->xi += (2.0 * ke - m->nh_gkt) / m->nh_q * quarter;
    double s = exp(-m->xi * half);
    m->eta += m->xi * half;
    double ke2 = ke * s * s;
    m->xi += (2.0 * ke2 - m->nh_gkt) / m->nh_q * quarter;
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < 3 * (size_t)m->n; q++) m->vm[q] *= s;
}

/* A Nose-Hoover step (lennard_jones.rs:1108-1127): thermostat half step,
 * half kick, drift, lists, forces, half kick, thermostat half step. */
static void nh_step(vo_md *m) {
    nh_half(m);
    double dt = m->dt, half = 0.5 * m->dt;
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < m->n; i++)
        for (int k = 0; k < 3; k++) {
            size_t q = 3 * (size_t)i + k;
            m->vm[q] += m->a[q] * half;
            m->x[q] = wrap(m->x[q] + m->vm[q] * dt, m->box[k]);
        }
    m->step += 1;
    if (needs_rebuild(m)) rebuild(m);
    forces(m, 0);
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < 3 * (size_t)m->n; q++) m->vm[q] += m->a[q] * half;
    nh_half(m);
}

/* ---- heat exchange, eHEX/a (lennard_jones.wgsl:732-893; Wirnsberger,
 * Frenkel and Dellago 2015, eq. 20) on canonical velocities ---- */
static int hex_slab(const vo_md *m, double z) {
    float zf = (float)z;
    if (zf >= m->hex_slabs[0] && zf < m->hex_slabs[1]) return 0;
    if (zf >= m->hex_slabs[2] && zf < m->hex_slabs[3]) return 1;
    return 2;
}

static void hex_apply(vo_md *m) {
    double dt = m->dt, dt3 = dt * dt * dt;
    double cnt[2] = {0, 0}, p[2][3] = {{0}}, f[2][3] = {{0}}, v2[2] = {0, 0}, fv[2] = {0, 0};
    for (uint32_t i = 0; i < m->n; i++) {
        int sl = hex_slab(m, m->x[3 * (size_t)i + 2]);
        if (sl == 2) continue;
        const double *v = m->vm + 3 * (size_t)i, *a = m->a + 3 * (size_t)i;
        cnt[sl] += 1.0;
        for (int k = 0; k < 3; k++) {
            p[sl][k] += v[k];
            f[sl][k] += a[k];
        }
        v2[sl] += v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        fv[sl] += a[0] * v[0] + a[1] * v[1] + a[2] * v[2];
    }
    double com[2][3] = {{0}}, mf[2][3] = {{0}}, sm1[2] = {0, 0}, cv[2] = {0, 0}, cf[2] = {0, 0};
    for (int sl = 0; sl < 2; sl++) {
        double mm = cnt[sl];
        if (!(mm > 0.0)) continue;
        for (int k = 0; k < 3; k++) {
            com[sl][k] = p[sl][k] / mm;
            mf[sl][k] = f[sl][k] / mm;
        }
        double pp = p[sl][0] * p[sl][0] + p[sl][1] * p[sl][1] + p[sl][2] * p[sl][2];
        double kinetic = 0.5 * v2[sl] - 0.5 * pp / mm;
        double energy = (sl == 0 ? 1.0 : -1.0) * m->hex_energy;
        double flux = energy / dt;
        double x = energy / kinetic;
        sm1[sl] = x / (1.0 + sqrt(1.0 + x));
        double power = fv[sl] - (f[sl][0] * com[sl][0] + f[sl][1] * com[sl][1] + f[sl][2] * com[sl][2]);
        cv[sl] = dt3 * flux / (2.0 * kinetic * kinetic) * (flux / 48.0 + power / 6.0);
        cf[sl] = dt3 * flux / (12.0 * kinetic);
    }
    for (uint32_t i = 0; i < m->n; i++) {
        int sl = hex_slab(m, m->x[3 * (size_t)i + 2]);
        if (sl == 2) continue;
        for (int k = 0; k < 3; k++) {
            size_t q = 3 * (size_t)i + k;
            double rel = m->vm[q] - com[sl][k];
            double shift = cv[sl] * rel - cf[sl] * (m->a[q] - mf[sl][k]);
            m->x[q] = wrap(m->x[q] - shift, m->box[k]);
            m->vm[q] += sm1[sl] * rel;
        }
    }
}

/* A constant-energy step with the exchange: half kick, drift, lists,
 * forces, half kick, exchange (lennard_jones.rs:1108-1138). */
static void hex_step(vo_md *m) {
    double dt = m->dt, half = 0.5 * m->dt;
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < m->n; i++)
        for (int k = 0; k < 3; k++) {
            size_t q = 3 * (size_t)i + k;
            m->vm[q] += m->a[q] * half;
            m->x[q] = wrap(m->x[q] + m->vm[q] * dt, m->box[k]);
        }
    m->step += 1;
    if (needs_rebuild(m)) rebuild(m);
    forces(m, 0);
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < 3 * (size_t)m->n; q++) m->vm[q] += m->a[q] * half;
    hex_apply(m);
}

/* Starts (energy and slabs) or, with on = 0, stops the exchange at the
 * current step boundary: velocities switch between half a kick behind and
 * canonical with the forces at the current positions. */
void vo_md_set_heat_exchange(vo_md *m, int on, const double slabs[4], double energy) {
    if (on && !m->hex) {
        if (needs_rebuild(m)) rebuild(m);
        forces(m, 0);
        for (size_t q = 0; q < 3 * (size_t)m->n; q++) m->vm[q] += m->a[q] * 0.5 * m->dt;
    } else if (!on && m->hex) {
        for (size_t q = 0; q < 3 * (size_t)m->n; q++) m->vm[q] -= m->a[q] * 0.5 * m->dt;
    }
    m->hex = on;
    if (on) {
        for (int k = 0; k < 4; k++) m->hex_slabs[k] = (float)slabs[k];
        m->hex_energy = (double)(float)energy;
    }
}

/* Closing half kick of the previous step + opening half kick of this one,
 * then the drift (with friction and noise for Langevin). */
static void advance(vo_md *m) {
    double dt = m->dt, half = 0.5 * m->dt;
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < m->n; i++) {
        float g[3] = {0.0f, 0.0f, 0.0f};
        if (m->thermostat == 1) vo_langevin_noise(m->seed, m->step, m->ids[i], g);
        for (int k = 0; k < 3; k++) {
            size_t q = 3 * (size_t)i + k;
            double v = m->vm[q] + m->a[q] * dt;
            double x = m->x[q];
            if (m->thermostat == 1) {
                x += v * half;
                v = m->c1 * v + m->c2 * (double)g[k];
                x += v * half;
            } else {
                x += v * dt;
            }
            m->x[q] = wrap(x, m->box[k]);
            m->vm[q] = v;
        }
    }
    m->step += 1;
}

vo_md *vo_md_create(const double *pos, const double *vel, uint32_t n, const double box[3],
                    double cutoff, double skin, double dt, int shifted_force, int thermostat,
                    double temperature, double friction, uint32_t seed) {
    vo_md *m = calloc(1, sizeof(vo_md));
    m->n = n;
    for (int k = 0; k < 3; k++) m->box[k] = (double)(float)box[k];
    m->cutoff = cutoff;
    m->rc2 = cutoff * cutoff;
    m->skin = skin;
    m->list_r2 = (cutoff + skin) * (cutoff + skin);
    m->half_skin2 = 0.25 * skin * skin;
    m->dt = dt;
    m->shifted_force = shifted_force;
    m->thermostat = thermostat;
    m->c1 = 1.0;
    m->c2 = 0.0;
    if (thermostat == 1) {
        m->c1 = exp(-friction * dt);
        m->c2 = sqrt((1.0 - m->c1 * m->c1) * temperature);
    }
    if (thermostat == 2) {
        /* lennard_jones.rs:516-528: g = 3N - 3 (zero total momentum),
         * Q = g T period^2 / (4 pi^2); `friction` carries the period */
        double dof = 3.0 * (double)n - 3.0;
        m->nh_gkt = dof * temperature;
        m->nh_q = dof * temperature * friction * friction / (4.0 * 3.141592653589793 * 3.141592653589793);
    }
    m->seed = seed;
    double sc6 = 1.0 / (m->rc2 * m->rc2 * m->rc2);
    m->uc = 4.0 * (sc6 * sc6 - sc6);
    m->fc = shifted_force ? 24.0 * (2.0 * sc6 * sc6 - sc6) / cutoff : 0.0;
    size_t n3 = 3 * (size_t)(n ? n : 1);
    m->x = malloc(sizeof(double) * n3);
    m->vm = malloc(sizeof(double) * n3);
    m->xb = malloc(sizeof(double) * n3);
    m->a = calloc(n3, sizeof(double));
    m->tmp = malloc(sizeof(double) * n3);
    m->ids = malloc(sizeof(uint32_t) * (n ? n : 1));
    m->tmp_ids = malloc(sizeof(uint32_t) * (n ? n : 1));
    m->cell = malloc(sizeof(uint32_t) * (n ? n : 1));
    m->order = malloc(sizeof(uint32_t) * (n ? n : 1));
    m->pe_i = calloc(n ? n : 1, sizeof(double));
    m->w_i = calloc(n ? n : 1, sizeof(double));
    m->nc = calloc(n ? n : 1, sizeof(uint32_t));
    for (uint32_t i = 0; i < n; i++) {
        m->ids[i] = i;
        for (int k = 0; k < 3; k++) {
            double x = fmod(pos[3 * (size_t)i + k], m->box[k]);
            if (x < 0.0) x += m->box[k];
            m->x[3 * (size_t)i + k] = wrap(x, m->box[k]);
        }
    }
    double radius = cutoff + skin;
    m->use_grid = 1;
    for (int k = 0; k < 3; k++) {
        double c = floor(m->box[k] / radius);
        m->cells[k] = c < 0.0 ? 0u : (uint32_t)c;
        if (m->cells[k] < 3) m->use_grid = 0;
    }
    if (m->use_grid) {
        m->total = m->cells[0] * m->cells[1] * m->cells[2];
        m->start = calloc((size_t)m->total + 1, sizeof(uint32_t));
        m->fill = calloc(m->total, sizeof(uint32_t));
    }
    double volume = m->box[0] * m->box[1] * m->box[2];
    double expected = 4.0 / 3.0 * 3.141592653589793 * radius * radius * radius * (double)n / volume;
    m->cap = (uint32_t)ceil(2.0 * expected + 32.0);
    m->nl = malloc(sizeof(uint32_t) * (size_t)(n ? n : 1) * m->cap);
    /* velocities enter in input order; rebuild() moves them with the slots */
    for (uint32_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) m->vm[3 * (size_t)i + k] = vel[3 * (size_t)i + k];
    rebuild(m);
    forces(m, 0);
    if (thermostat != 2)
        for (size_t q = 0; q < 3 * (size_t)n; q++) m->vm[q] -= m->a[q] * 0.5 * dt;
    return m;
}

void vo_md_destroy(vo_md *m) {
    if (!m) return;
    free(m->x);
    free(m->vm);
    free(m->xb);
    free(m->a);
    free(m->tmp);
    free(m->ids);
    free(m->tmp_ids);
    free(m->cell);
    free(m->order);
    free(m->pe_i);
    free(m->w_i);
    free(m->nc);
    free(m->nl);
    free(m->start);
    free(m->fill);
    free(m);
}

void vo_md_run(vo_md *m, uint64_t steps) {
    if (m->thermostat == 2) {
        for (uint64_t s = 0; s < steps; s++) nh_step(m);
        return;
    }
    if (m->hex) {
        for (uint64_t s = 0; s < steps; s++) hex_step(m);
        return;
    }
    for (uint64_t s = 0; s < steps; s++) {
        if (needs_rebuild(m)) rebuild(m);
        forces(m, 0);
        advance(m);
    }
}

void vo_md_measure(vo_md *m, vo_md_measurement *out) {
    if (needs_rebuild(m)) rebuild(m);
    forces(m, 1);
    double ke = 0.0, pe = 0.0, w = 0.0, p0 = 0.0, p1 = 0.0, p2 = 0.0;
    /* Nose-Hoover and the exchange keep canonical velocities; otherwise half
     * a kick behind */
    double half = (m->thermostat == 2 || m->hex) ? 0.0 : 0.5 * m->dt;
    for (uint32_t i = 0; i < m->n; i++) {
        double v[3];
        for (int k = 0; k < 3; k++) v[k] = m->vm[3 * (size_t)i + k] + m->a[3 * (size_t)i + k] * half;
        ke += 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        p0 += v[0];
        p1 += v[1];
        p2 += v[2];
        pe += m->pe_i[i];
        w += m->w_i[i];
    }
    out->step = m->step;
    out->kinetic = ke;
    out->potential = pe;
    out->virial = w;
    out->momentum[0] = p0;
    out->momentum[1] = p1;
    out->momentum[2] = p2;
    out->list_rebuilds = m->rebuilds;
    out->thermostat_energy =
        m->thermostat == 2 ? 0.5 * m->nh_q * m->xi * m->xi + m->nh_gkt * m->eta : 0.0;
}

void vo_md_read(vo_md *m, double *pos, double *vel) {
    if (needs_rebuild(m)) rebuild(m);
    forces(m, 0);
    double half = (m->thermostat == 2 || m->hex) ? 0.0 : 0.5 * m->dt;
    for (uint32_t i = 0; i < m->n; i++) {
        uint32_t id = m->ids[i];
        for (int k = 0; k < 3; k++) {
            pos[3 * (size_t)id + k] = m->x[3 * (size_t)i + k];
            vel[3 * (size_t)id + k] = m->vm[3 * (size_t)i + k] + m->a[3 * (size_t)i + k] * half;
        }
    }
}

void vo_md_set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

int vo_md_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
