/*
 * Set-up, cell binning, per-cell order, reorder and Verlet-list build, as the
 * reference does them in f32. Test oracle only (see vlj_oracle.h).
 */
#include "vlj_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* lennard_jones.rs:435-440 */
static double scale_for(double magnitude) {
    if (magnitude <= 0.0 || !isfinite(magnitude)) return 1.0;
    return pow(2.0, floor(20.0 - log2(magnitude)));
}

/* lennard_jones.rs:443-560 (the parts that feed the step). Rust's max_by_key
 * returns the last of equal maxima. */
int vo_setup_compute(uint32_t n, const double *vel, const double box[3], double cutoff,
                     double skin, int shifted_force, double thermostat_temperature,
                     vo_setup *s) {
    memset(s, 0, sizeof(*s));
    s->n = n;
    double list_radius = cutoff + skin;
    for (int k = 0; k < 3; k++) {
        s->box_f[k] = (float)box[k];
        s->box[k] = (double)s->box_f[k];
        double c = floor(s->box[k] / list_radius);
        s->cells[k] = c < 0.0 ? 0u : (uint32_t)c;
    }
    if (s->cells[0] < 3 || s->cells[1] < 3 || s->cells[2] < 3) return 1;
    while ((uint64_t)s->cells[0] * s->cells[1] * s->cells[2] > (1u << 20)) {
        int longest = 0;
        for (int k = 1; k < 3; k++)
            if (s->cells[k] >= s->cells[longest]) longest = k;
        s->cells[longest] -= 1;
    }
    s->total_cells = s->cells[0] * s->cells[1] * s->cells[2];
    for (int k = 0; k < 3; k++) s->cell_size_f[k] = (float)(s->box[k] / (double)s->cells[k]);
    double volume = s->box[0] * s->box[1] * s->box[2];
    s->segment = (n + 15u) / 16u * 16u;
    double density = (double)n / volume;
    double expected = 4.0 / 3.0 * 3.141592653589793 * (list_radius * list_radius * list_radius) *
                      density;
    s->capacity = (uint32_t)ceil(2.0 * expected + 32.0);

    double kinetic = 0.0, speed = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        double v2 = 0.0;
        for (int k = 0; k < 3; k++) v2 += vel[3 * i + k] * vel[3 * i + k];
        kinetic += 0.5 * v2;
        speed += sqrt(v2);
    }
    double thermal = thermostat_temperature > 0.0 ? 1.5 * thermostat_temperature * (double)n : 0.0;
    double m = kinetic > thermal ? kinetic : thermal;
    if ((double)n > m) m = (double)n;
    s->energy_scale = scale_for(m);
    s->momentum_scale = scale_for(speed > (double)n ? speed : (double)n);

    s->cutoff = cutoff;
    s->skin = skin;
    double rc2 = cutoff * cutoff;
    double inv6 = 1.0 / (rc2 * rc2 * rc2);
    s->shift = (float)(4.0 * (inv6 * inv6 - inv6));
    s->force_shift = shifted_force ? (float)(24.0 * (2.0 * inv6 * inv6 - inv6) / cutoff) : 0.0f;
    s->rc2 = (float)rc2;
    s->list_r2 = (float)(list_radius * list_radius);
    s->half_skin2 = (float)(0.25 * skin * skin);
    return 0;
}

/* grid.wgsl:11-20: clamp(floor(x / cell), 0, n - 1) per axis */
static uint32_t cell_of(const vo_setup *s, const float hi[3]) {
    int32_t c[3];
    for (int k = 0; k < 3; k++) {
        int32_t v = (int32_t)floorf(hi[k] / s->cell_size_f[k]);
        int32_t m = (int32_t)s->cells[k] - 1;
        c[k] = v < 0 ? 0 : (v > m ? m : v);
    }
    return ((uint32_t)c[2] * s->cells[1] + (uint32_t)c[1]) * s->cells[0] + (uint32_t)c[0];
}

/* lennard_jones.wgsl:199-202: d - side * round(d / side), round to even */
static float nearest1(float d, float side) {
    float r = rintf(d / side);
    float m = side * r;
    return d - m;
}

void vo_rebuild_ref(const vo_setup *s, uint32_t n, double *x, double *v, uint32_t *ids,
                    int reorder, uint32_t *cell_of_slot, uint32_t *cell_start, uint32_t *sorted,
                    uint32_t *list_count, uint32_t *list, uint32_t *overflow) {
    float *hi = malloc(sizeof(float) * 3 * (size_t)n);
    float *lo = malloc(sizeof(float) * 3 * (size_t)n);
    uint32_t *count = calloc(s->total_cells, sizeof(uint32_t));
    /* Df64::from_f64 of each coordinate (lennard_jones.rs:476-489) */
    for (size_t i = 0; i < 3 * (size_t)n; i++) {
        vo_df d = vo_df_from_f64(x[i]);
        hi[i] = d.hi;
        lo[i] = d.lo;
    }
    /* bin, scan, scatter (grid.wgsl:29-127); the per-cell sort by slot
     * (grid.wgsl:131-148) makes the order the same as a stable scatter */
    for (uint32_t i = 0; i < n; i++) {
        cell_of_slot[i] = cell_of(s, &hi[3 * (size_t)i]);
        count[cell_of_slot[i]] += 1;
    }
    uint32_t run = 0;
    for (uint32_t c = 0; c < s->total_cells; c++) {
        cell_start[c] = run;
        run += count[c];
        count[c] = 0;
    }
    cell_start[s->total_cells] = n;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t c = cell_of_slot[i];
        sorted[cell_start[c] + count[c]++] = i;
    }
    /* reorder_gather / reorder_scatter (lennard_jones.wgsl:421-452) */
    if (reorder) {
        double *x2 = malloc(sizeof(double) * 3 * (size_t)n);
        double *v2 = malloc(sizeof(double) * 3 * (size_t)n);
        float *h2 = malloc(sizeof(float) * 3 * (size_t)n);
        float *l2 = malloc(sizeof(float) * 3 * (size_t)n);
        uint32_t *id2 = malloc(sizeof(uint32_t) * (size_t)n);
        uint32_t *c2 = malloc(sizeof(uint32_t) * (size_t)n);
        for (uint32_t t = 0; t < n; t++) {
            uint32_t i = sorted[t];
            for (int k = 0; k < 3; k++) {
                x2[3 * (size_t)t + k] = x[3 * (size_t)i + k];
                v2[3 * (size_t)t + k] = v[3 * (size_t)i + k];
                h2[3 * (size_t)t + k] = hi[3 * (size_t)i + k];
                l2[3 * (size_t)t + k] = lo[3 * (size_t)i + k];
            }
            id2[t] = ids[i];
            c2[t] = cell_of_slot[i];
        }
        memcpy(x, x2, sizeof(double) * 3 * (size_t)n);
        memcpy(v, v2, sizeof(double) * 3 * (size_t)n);
        memcpy(hi, h2, sizeof(float) * 3 * (size_t)n);
        memcpy(lo, l2, sizeof(float) * 3 * (size_t)n);
        memcpy(ids, id2, sizeof(uint32_t) * (size_t)n);
        memcpy(cell_of_slot, c2, sizeof(uint32_t) * (size_t)n);
        for (uint32_t t = 0; t < n; t++) sorted[t] = t;
        free(x2);
        free(v2);
        free(h2);
        free(l2);
        free(id2);
        free(c2);
    }
    /* packed positions (lennard_jones.wgsl:154-156) */
    uint32_t *packed = malloc(sizeof(uint32_t) * (size_t)n);
    for (uint32_t i = 0; i < n; i++) packed[i] = vo_pack_lo(&hi[3 * (size_t)i], &lo[3 * (size_t)i]);
    /* build_list (lennard_jones.wgsl:456-499) */
    uint32_t worst = 0;
    const int32_t nx = (int32_t)s->cells[0], ny = (int32_t)s->cells[1], nz = (int32_t)s->cells[2];
    for (uint32_t i = 0; i < n; i++) {
        const float *xh = &hi[3 * (size_t)i];
        const float *xl = &lo[3 * (size_t)i];
        int32_t ci = (int32_t)cell_of_slot[i];
        int32_t cc[3] = {ci % nx, (ci / nx) % ny, ci / (nx * ny)};
        uint32_t found = 0;
        for (int32_t dz = -1; dz <= 1; dz++)
            for (int32_t dy = -1; dy <= 1; dy++)
                for (int32_t dx = -1; dx <= 1; dx++) {
                    uint32_t ncx = (uint32_t)((cc[0] + dx + nx) % nx);
                    uint32_t ncy = (uint32_t)((cc[1] + dy + ny) % ny);
                    uint32_t ncz = (uint32_t)((cc[2] + dz + nz) % nz);
                    uint32_t cell = (ncz * (uint32_t)ny + ncy) * (uint32_t)nx + ncx;
                    for (uint32_t t = cell_start[cell]; t < cell_start[cell + 1]; t++) {
                        uint32_t j = sorted[t];
                        if (j == i) continue;
                        const float *pj = &hi[3 * (size_t)j];
                        float ulo[3];
                        vo_unpack_lo(pj, packed[j], ulo);
                        float d[3];
                        for (int k = 0; k < 3; k++) {
                            float a = pj[k] - xh[k];
                            float b = ulo[k] - xl[k];
                            d[k] = nearest1(a + b, s->box_f[k]);
                        }
                        float r2 = d[0] * d[0];
                        r2 = r2 + d[1] * d[1];
                        r2 = r2 + d[2] * d[2];
                        if (r2 < s->list_r2) {
                            if (found < s->capacity) list[(size_t)i * s->capacity + found] = j;
                            found += 1;
                        }
                    }
                }
        list_count[i] = found < s->capacity ? found : s->capacity;
        if (found > s->capacity && found > worst) worst = found;
    }
    *overflow = worst;
    free(packed);
    free(hi);
    free(lo);
    free(count);
}
