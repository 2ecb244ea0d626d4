/*
 * Arithmetic primitives of the reference path, restated on the CPU:
 * 32.32 fixed point, double-float, packed positions and the two random
 * number generators. Test oracle only (see vlj_oracle.h).
 */
#include "vlj_oracle.h"

#include <math.h>
#include <string.h>

static uint32_t f32_bits(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    return b;
}

static float bits_f32(uint32_t b) {
    float x;
    memcpy(&x, &b, 4);
    return x;
}

/* ---- fixed point ---- */

/* fixed_split, crates/virial-precision/src/fixed.wgsl:20-55 (== fixed.rs:9-41):
 * (low, high) words of x rounded to the nearest 2^-32, ties to even, in
 * integer arithmetic on the float's bits. Valid for |x| < 2^31. WGSL masks
 * shift amounts to 5 bits; the masks below do the same. */
void vo_fixed_split(float x, uint32_t *low_out, uint32_t *high_out) {
    uint32_t bits = f32_bits(x);
    int32_t exponent = (int32_t)((bits >> 23) & 0xffu) - 127;
    if (exponent < -34) {
        *low_out = 0;
        *high_out = 0;
        return;
    }
    uint32_t mantissa = (bits & 0x7fffffu) | 0x800000u;
    int32_t shift = exponent + 9;
    uint32_t low = 0, high = 0;
    if (shift >= 32) {
        high = mantissa << ((uint32_t)(shift - 32) & 31u);
    } else if (shift > 0) {
        low = mantissa << (uint32_t)shift;
        high = mantissa >> (uint32_t)(32 - shift);
    } else if (shift == 0) {
        low = mantissa;
    } else {
        uint32_t r = (uint32_t)(-shift);
        low = mantissa >> r;
        uint32_t rest = mantissa & ((1u << r) - 1u);
        uint32_t half = 1u << (r - 1u);
        if (rest > half || (rest == half && (low & 1u) == 1u)) low += 1u;
    }
    if ((bits & 0x80000000u) == 0u) {
        *low_out = low;
        *high_out = high;
    } else {
        *low_out = ~low + 1u;
        *high_out = ~high + (low == 0u ? 1u : 0u);
    }
}

/* fixed.rs:44-52 */
int64_t vo_fixed_from_words(uint32_t low, uint32_t high) {
    return (int64_t)(((uint64_t)high << 32) | (uint64_t)low);
}

int64_t vo_fixed_to_raw(float x) {
    uint32_t lo, hi;
    vo_fixed_split(x, &lo, &hi);
    return vo_fixed_from_words(lo, hi);
}

/* fixed.rs:55-57 */
double vo_fixed_to_f64(int64_t raw) { return (double)raw / 4294967296.0; }

int64_t vo_fixed_raw_f64(double x) { return (int64_t)llrint(x * 4294967296.0); }

/* ---- double-float: crates/virial-precision/src/df64.rs:15-131 ---- */

static vo_df two_sum(float a, float b) {
    float s = a + b;
    float bb = s - a;
    vo_df r = {s, (a - (s - bb)) + (b - bb)};
    return r;
}

static vo_df quick_two_sum(float a, float b) {
    float s = a + b;
    vo_df r = {s, b - (s - a)};
    return r;
}

static void dekker_split(float a, float *hi, float *lo) {
    float c = 4097.0f * a;
    float h = c - (c - a);
    *hi = h;
    *lo = a - h;
}

static vo_df two_prod(float a, float b) {
    float p = a * b;
    float ah, al, bh, bl;
    dekker_split(a, &ah, &al);
    dekker_split(b, &bh, &bl);
    vo_df r = {p, ((ah * bh - p) + ah * bl + al * bh) + al * bl};
    return r;
}

vo_df vo_df_from_f64(double x) {
    float hi = (float)x;
    vo_df r = {hi, (float)(x - (double)hi)};
    return r;
}

double vo_df_to_f64(vo_df a) { return (double)a.hi + (double)a.lo; }

vo_df vo_df_add_f(vo_df a, float b) {
    vo_df s = two_sum(a.hi, b);
    return quick_two_sum(s.hi, s.lo + a.lo);
}

vo_df vo_df_mul_f(vo_df a, float b) {
    vo_df p = two_prod(a.hi, b);
    return quick_two_sum(p.hi, p.lo + a.lo * b);
}

vo_df vo_df_add(vo_df a, vo_df b) {
    vo_df s = two_sum(a.hi, b.hi);
    vo_df t = two_sum(a.lo, b.lo);
    vo_df u = quick_two_sum(s.hi, s.lo + t.hi);
    return quick_two_sum(u.hi, u.lo + t.lo);
}

vo_df vo_df_sub(vo_df a, vo_df b) {
    vo_df nb = {-b.hi, -b.lo};
    return vo_df_add(a, nb);
}

vo_df vo_df_mul(vo_df a, vo_df b) {
    vo_df p = two_prod(a.hi, b.hi);
    return quick_two_sum(p.hi, p.lo + (a.hi * b.lo + a.lo * b.hi));
}

vo_df vo_df_div(vo_df a, vo_df b) {
    float q1 = a.hi / b.hi;
    vo_df r = vo_df_sub(a, vo_df_mul_f(b, q1));
    float q2 = r.hi / b.hi;
    r = vo_df_sub(r, vo_df_mul_f(b, q2));
    float q3 = r.hi / b.hi;
    return vo_df_add_f(quick_two_sum(q1, q2), q3);
}

vo_df vo_df_sqrt(vo_df a) {
    if (a.hi <= 0.0f) {
        vo_df z = {0.0f, 0.0f};
        return z;
    }
    float s = sqrtf(a.hi);
    vo_df e = vo_df_sub(a, two_prod(s, s));
    vo_df f = {s, 0.0f};
    return vo_df_add_f(f, (e.hi + e.lo) / (2.0f * s));
}

/* ---- packed positions: crates/virial-particles/src/lennard_jones.wgsl:128-152 ---- */

float vo_last_bit(float h) {
    uint32_t e = (f32_bits(h) >> 23) & 0xffu;
    if (e < 24u) e = 24u;
    return bits_f32((e - 23u) << 23);
}

uint32_t vo_pack_lo(const float hi[3], const float lo[3]) {
    uint32_t bits = 0x20000000u;
    for (int k = 0; k < 3; k++) {
        float t = lo[k] / vo_last_bit(hi[k]);
        t = fminf(fmaxf(t, -0.5f), 0.5f);
        int32_t q = (int32_t)rintf(t * 510.0f);
        bits |= (uint32_t)(q + 256) << (9u * (uint32_t)k);
    }
    return bits;
}

void vo_unpack_lo(const float hi[3], uint32_t bits, float lo[3]) {
    for (int k = 0; k < 3; k++) {
        float q = (float)((int32_t)((bits >> (9u * (uint32_t)k)) & 511u) - 256);
        lo[k] = q / 510.0f * vo_last_bit(hi[k]);
    }
}

/* ---- reference random numbers: lennard_jones.wgsl:168-184 ---- */

uint32_t vo_pcg(uint32_t *state) {
    uint32_t s = *state * 747796405u + 2891336453u;
    *state = s;
    uint32_t word = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (word >> 22u) ^ word;
}

float vo_uniform01(uint32_t *state) {
    return ((float)(vo_pcg(state) >> 8u) + 1.0f) / 16777216.0f;
}

void vo_gaussian2(uint32_t *state, float out[2]) {
    float r = sqrtf(-2.0f * logf(vo_uniform01(state)));
    float a = 6.283185307179586f * vo_uniform01(state);
    out[0] = r * cosf(a);
    out[1] = r * sinf(a);
}

/* lennard_jones.rs:584-592: splitmix-style hash of (seed << 32 | index). */
uint32_t vo_pcg_seed(uint32_t seed, uint32_t index) {
    uint64_t z = ((uint64_t)seed << 32) | (uint64_t)index;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return (uint32_t)(z ^ (z >> 31));
}

/* ---- Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ----
 * Ten rounds of two 32x32->64 multiplies; the key is bumped by the Weyl
 * constants between rounds. */
void vo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; round++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0;
        c1 = n1;
        c2 = n2;
        c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* Langevin noise of the CUDA path: one Philox block per (particle, step),
 * counter (id, step low, step high, 0), key (seed, "LJV1"). Uniforms in
 * (0, 1] from 24 bits as the reference's uniform01; Box-Muller in f32. */
void vo_langevin_noise(uint32_t seed, uint64_t step, uint32_t id, float out[3]) {
    uint32_t ctr[4] = {id, (uint32_t)step, (uint32_t)(step >> 32), 0u};
    uint32_t key[2] = {seed, 0x4C4A5631u};
    uint32_t r[4];
    vo_philox4x32_10(ctr, key, r);
    float u0 = ((float)(r[0] >> 8) + 1.0f) / 16777216.0f;
    float u1 = ((float)(r[1] >> 8) + 1.0f) / 16777216.0f;
    float u2 = ((float)(r[2] >> 8) + 1.0f) / 16777216.0f;
    float u3 = ((float)(r[3] >> 8) + 1.0f) / 16777216.0f;
    float ra = sqrtf(-2.0f * logf(u0));
    float aa = 6.283185307179586f * u1;
    float rb = sqrtf(-2.0f * logf(u2));
    float ab = 6.283185307179586f * u3;
    out[0] = ra * cosf(aa);
    out[1] = ra * sinf(aa);
    out[2] = rb * cosf(ab);
}
