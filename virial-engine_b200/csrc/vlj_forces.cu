// CUDA kernels of the pair forces, the integrator and the measurements,
// sm_100a.
//
// One thread per particle, 128 per block. Each thread reads its Verlet-list
// rows (a row is four entries of a particle, 16 B; a warp's rows are 512
// contiguous bytes) one ahead with loads that do not allocate in L1, issues
// the four neighbour gathers of a row through L1 together, then does the four
// pairs' arithmetic. The force kernels use almost no shared memory and ask for
// the largest L1 carve-out, so the L1 holds the neighbourhood the gathers
// reuse. (The alternative, VLJ_LIST_STREAM=0, stages the rows in shared memory
// as TMA tiles of kTileRows rows x 128 particles on an mbarrier ring; the
// tuner measured it 16-45 % slower on the 256k-atom box, because the tiles
// take the shared memory the L1 needs.) Reference kernels are cited at each
// kernel.
#include <cuda.h>
#include <cuda_runtime.h>

#include "vlj_device.cuh"
#include "vlj_internal.cuh"

namespace vlj {

constexpr uint32_t kTileBytes = kTileRows * kForceThreads * 16u;
// Resident blocks per SM the step kernel's register budget is sized for.
#ifndef VLJ_STEP_MIN_BLOCKS
#define VLJ_STEP_MIN_BLOCKS 1
#endif
constexpr int kStepMinBlocks = VLJ_STEP_MIN_BLOCKS;
// Grids of at most this many blocks (of one particle a thread) per SM step
// with two lanes per particle (step_kernel_split).
#ifndef VLJ_SPLIT_BLOCKS_PER_SM
#define VLJ_SPLIT_BLOCKS_PER_SM 4
#endif
constexpr int kSplitBlocksPerSM = VLJ_SPLIT_BLOCKS_PER_SM;
constexpr unsigned long long kWaitLimitNs = 500000000ull;  // 0.5 s per TMA tile

struct PairSums {
    float ax, ay, az;
    float pe, pe_lo;  // this particle's half of its pair energies, hi + lo
    float w, w_lo;    // and of its pair virials r . F
    uint32_t near;    // neighbours within 1.5 sigma
    // heat current: half of the pair energies, and T = sum_j d d^T |F| / r
    // (xx yy zz xy xz yz)
    float e_half, t[6];
    // The force is summed in two parts, the entries of the list's even rows
    // (ax, ay, az) and of its odd rows (these), added once at the end
    // (combine_parts): one thread walking all rows and two lanes walking
    // half of them each then give the same bits.
    float ax1, ay1, az1;
};

__device__ __forceinline__ void combine_parts(PairSums& s) {
    s.ax = __fadd_rn(s.ax, s.ax1);
    s.ay = __fadd_rn(s.ay, s.ay1);
    s.az = __fadd_rn(s.az, s.az1);
    s.ax1 = s.ay1 = s.az1 = 0.0f;
}

// the force part of the list's row parity PART
template <int PART>
__device__ __forceinline__ void add_force(PairSums& s, float dx, float dy, float dz, float f) {
    if (PART == 0) {
        s.ax = __fmaf_rn(-dx, f, s.ax);
        s.ay = __fmaf_rn(-dy, f, s.ay);
        s.az = __fmaf_rn(-dz, f, s.az);
    } else {
        s.ax1 = __fmaf_rn(-dx, f, s.ax1);
        s.ay1 = __fmaf_rn(-dy, f, s.ay1);
        s.az1 = __fmaf_rn(-dz, f, s.az1);
    }
}

// Shared memory of a force-kernel block: the tile ring and its barriers
// (none when the rows stream straight from global memory).
#if VLJ_LIST_STREAM
struct Stage {
    unsigned long long unused;
};
#else
struct Stage {
    uint4 rows[kTileSlots][kTileRows][kForceThreads];
    unsigned long long bar[kTileSlots];
};
#endif

// A list row (four entries of one slot, 16 B) read once: no L1 allocation,
// so the L1 keeps the neighbour positions the gathers reuse.
__device__ __forceinline__ uint4 load_row_streaming(const uint4* p) {
    uint4 r;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w) : "l"(p));
    return r;
}

// ---- TMA and mbarrier primitives (PTX, sm_90+) ----
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One tile: rows [y, y + kTileRows) of the block's particles (x = first
// particle * 2 u64 elements). Rows and particles past the list's end arrive
// as zeros. No multicast.
__device__ __forceinline__ void tile_load(const CUtensorMap* map, void* dst, unsigned long long* bar,
                                          int x, int y) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_addr(bar)), "r"(kTileBytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_addr(dst)), "l"((unsigned long long)map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool bar_try_wait(unsigned long long* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return done != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for a tile with a time limit; false when it did not arrive.
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, uint32_t parity) {
    if (bar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!bar_try_wait(bar, parity))
        if (global_ns() - t0 > kWaitLimitNs) return false;
    return true;
}

// ---- forces from the list (lennard_jones.wgsl:503-545) ----
// One list entry's terms into the particle's sums: the separation from the
// 32-bit box fractions (the wrapped integer difference is the nearest
// image), the force factor (the same expression in every pass, so the step,
// the first forces and the measurement agree to the bit), and with ENERGIES
// the halves of the pair energy and virial as unevaluated f32 pairs (as the
// reference sums them in double-float, lennard_jones.wgsl:518-519). A zero
// separation (the padding of a list's last row) adds nothing.
template <bool SHIFTED_FORCE, bool ENERGIES, bool HEAT, int PART = 0>
__device__ __forceinline__ void pair_terms(PairSums& s, const uint4 own, const uint4 pj,
                                           const Box& bx, float dec0, float dec1, float dec2,
                                           uint32_t rc2_bits_m1, float fshift) {
    const float dx = decode_diff(pj.x, own.x, dec0);
    const float dy = decode_diff(pj.y, own.y, dec1);
    const float dz = decode_diff(pj.z, own.z, dec2);
    const float r2 = sep_r2(dx, dy, dz);
    const bool in = __float_as_uint(r2) - 1u < rc2_bits_m1;
    // branch-free: most list entries are inside the cutoff; the select
    // drops whatever the pair math gives for entries that are not
    const float f = in ? lj_force_over_r2<SHIFTED_FORCE>(r2, fshift) : 0.0f;
    add_force<PART>(s, dx, dy, dz, f);
    if (HEAT) {
        s.e_half += in ? 0.5f * lj_energy_fast<SHIFTED_FORCE>(r2, bx) : 0.0f;
        const float fx = dx * f, fy = dy * f, fz = dz * f;
        s.t[0] += dx * fx;
        s.t[1] += dy * fy;
        s.t[2] += dz * fz;
        s.t[3] += dx * fy;
        s.t[4] += dx * fz;
        s.t[5] += dy * fz;
    }
    if (ENERGIES && in) {
        // The sums take r^2 rounded once from the exact separation (the
        // integer differences times the box step are exact in f64): on a
        // lattice, where every pair at one distance rounds alike, the f32
        // components' three roundings would bias the virial coherently.
        const double ex = (double)(int32_t)(pj.x - own.x) * (double)dec0;
        const double ey = (double)(int32_t)(pj.y - own.y) * (double)dec1;
        const double ez = (double)(int32_t)(pj.z - own.z) * (double)dec2;
        float rf, u, t, e;
        lj_pair<SHIFTED_FORCE>((float)(ex * ex + ey * ey + ez * ez), bx, rf, u);
        two_sum(s.pe, 0.5f * u, t, e);
        s.pe = t;
        s.pe_lo += e;
        two_sum(s.w, 0.5f * rf, t, e);
        s.w = t;
        s.w_lo += e;
        s.near += r2 < 2.25f ? 1u : 0u;
    }
}

// pair_terms on positions given as f32 offsets from a common origin near
// both (the cell tiles' f32 form): the separation is their plain difference.
template <bool SHIFTED_FORCE, bool HEAT, int PART = 0>
__device__ __forceinline__ void pair_terms_rel(PairSums& s, const float4 own, const float4 pj,
                                               const Box& bx, uint32_t rc2_bits_m1, float fshift) {
    const float dx = __fsub_rn(pj.x, own.x);
    const float dy = __fsub_rn(pj.y, own.y);
    const float dz = __fsub_rn(pj.z, own.z);
    const float r2 = sep_r2(dx, dy, dz);
    const bool in = __float_as_uint(r2) - 1u < rc2_bits_m1;
    const float f = in ? lj_force_over_r2<SHIFTED_FORCE>(r2, fshift) : 0.0f;
    add_force<PART>(s, dx, dy, dz, f);
    if (HEAT) {
        s.e_half += in ? 0.5f * lj_energy_fast<SHIFTED_FORCE>(r2, bx) : 0.0f;
        const float fx = dx * f, fy = dy * f, fz = dz * f;
        s.t[0] += dx * fx;
        s.t[1] += dy * fy;
        s.t[2] += dz * fz;
        s.t[3] += dx * fy;
        s.t[4] += dx * fz;
        s.t[5] += dy * fz;
    }
}

// The particle's pair sums over its list. Every thread of the block must
// call this: it synchronises the block between tiles.
template <bool SHIFTED_FORCE, bool ENERGIES, bool HEAT = false>
__device__ __forceinline__ PairSums block_pair_sums(Stage& st, const CUtensorMap* map,
                                                    const Arena& a, const Box& bx, uint32_t i,
                                                    bool valid, const uint4* __restrict__ cur) {
    PairSums s = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u,
                  0.0f, {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}};
#if !VLJ_LIST_STREAM
    const uint32_t first = blockIdx.x * kForceThreads;
    const uint32_t rows = a.block_rows[blockIdx.x];
    const uint32_t tiles = (rows + kTileRows - 1u) / kTileRows;
    if (threadIdx.x == 0) {
        for (int k = 0; k < kTileSlots; k++) bar_init(&st.bar[k]);
        init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (uint32_t t = 0; t < tiles && t < (uint32_t)kTileSlots; t++)
            tile_load(map, &st.rows[t][0][0], &st.bar[t], (int)(first * 2u), (int)(t * kTileRows));
#else
    (void)st;
    (void)map;
#endif

    uint4 own = make_uint4(0u, 0u, 0u, 0u);
    uint32_t cnt = 0;
    if (valid) {
        own = __ldg(cur + i);
        cnt = __ldg(a.list_count + i);
    }
    const uint32_t my_rows = (cnt + 3u) / 4u;
    const float dec0 = bx.dec[0], dec1 = bx.dec[1], dec2 = bx.dec[2], rc2 = bx.rc2;
    const float fshift = bx.force_shift;
    // 0 < r2 < rc2 as one unsigned comparison of the bit patterns (r2 >= +0)
    const uint32_t rc2_bits_m1 = __float_as_uint(rc2) - 1u;
    // The list's last row is padded with the particle itself, whose zero
    // separation drops out with the entries beyond the cutoff.
    auto acc0 = [&](const uint4 pj) {
        pair_terms<SHIFTED_FORCE, ENERGIES, HEAT, 0>(s, own, pj, bx, dec0, dec1, dec2,
                                                     rc2_bits_m1, fshift);
    };
    auto acc1 = [&](const uint4 pj) {
        pair_terms<SHIFTED_FORCE, ENERGIES, HEAT, 1>(s, own, pj, bx, dec0, dec1, dec2,
                                                     rc2_bits_m1, fshift);
    };
    // the four entries of list row `row`, into the force part of its parity
    auto row_terms = [&](uint32_t row, const uint4 p0, const uint4 p1, const uint4 p2,
                         const uint4 p3) {
        if (row & 1u) {
            acc1(p0);
            acc1(p1);
            acc1(p2);
            acc1(p3);
        } else {
            acc0(p0);
            acc0(p1);
            acc0(p2);
            acc0(p3);
        }
    };

#if VLJ_LIST_STREAM
    const uint4* rowp = reinterpret_cast<const uint4*>(a.list) + i;
#if VLJ_GATHER_AHEAD
    // gathers one row ahead: row r + 1's neighbours are in flight while row
    // r's pairs are computed (its list row two ahead)
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
    uint4 e_next = my_rows > 1u ? load_row_streaming(rowp + a.seg) : zero;
    uint4 q0 = own, q1 = own, q2 = own, q3 = own;
    if (my_rows) {
        const uint4 e = load_row_streaming(rowp);
        q0 = __ldg(cur + e.x);
        q1 = __ldg(cur + e.y);
        q2 = __ldg(cur + e.z);
        q3 = __ldg(cur + e.w);
    }
    for (uint32_t row = 0; row < my_rows; row++) {
        const uint4 p0 = q0, p1 = q1, p2 = q2, p3 = q3;
        if (row + 1u < my_rows) {
            const uint4 e = e_next;
            if (row + 2u < my_rows) e_next = load_row_streaming(rowp + (size_t)(row + 2u) * a.seg);
            q0 = __ldg(cur + e.x);
            q1 = __ldg(cur + e.y);
            q2 = __ldg(cur + e.z);
            q3 = __ldg(cur + e.w);
        }
        row_terms(row, p0, p1, p2, p3);
    }
#else
    // each thread its own rows, the next one in flight while it works on
    // this; two rows an iteration, the even one's force part then the odd's
    uint4 next = my_rows ? load_row_streaming(rowp) : make_uint4(0u, 0u, 0u, 0u);
    for (uint32_t row = 0; row < my_rows; row += 2u) {
        {
            const uint4 e = next;
            if (row + 1u < my_rows) next = load_row_streaming(rowp + (size_t)(row + 1u) * a.seg);
            const uint4 p0 = __ldg(cur + e.x);
            const uint4 p1 = __ldg(cur + e.y);
            const uint4 p2 = __ldg(cur + e.z);
            const uint4 p3 = __ldg(cur + e.w);
            acc0(p0);
            acc0(p1);
            acc0(p2);
            acc0(p3);
        }
        if (row + 1u < my_rows) {
            const uint4 e = next;
            if (row + 2u < my_rows) next = load_row_streaming(rowp + (size_t)(row + 2u) * a.seg);
            const uint4 p0 = __ldg(cur + e.x);
            const uint4 p1 = __ldg(cur + e.y);
            const uint4 p2 = __ldg(cur + e.z);
            const uint4 p3 = __ldg(cur + e.w);
            acc1(p0);
            acc1(p1);
            acc1(p2);
            acc1(p3);
        }
    }
#endif
    combine_parts(s);
    return s;
#else
    bool lost = false;
    for (uint32_t t = 0; t < tiles; t++) {
        const uint32_t slot = t % kTileSlots;
        const bool ok = bar_wait(&st.bar[slot], (t / kTileSlots) & 1u);
        if (__syncthreads_or(!ok)) {
            lost = true;
            break;
        }
#pragma unroll
        for (int r = 0; r < kTileRows; r++) {
            const uint32_t row = t * kTileRows + (uint32_t)r;
            if (row < my_rows) {
                // one row: four entries, the last ones live only up to cnt
                const uint4 e = st.rows[slot][r][threadIdx.x];
                const uint4 p0 = __ldg(cur + e.x);
                const uint4 p1 = __ldg(cur + e.y);
                const uint4 p2 = __ldg(cur + e.z);
                const uint4 p3 = __ldg(cur + e.w);
                row_terms(row, p0, p1, p2, p3);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && t + kTileSlots < tiles) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tile_load(map, &st.rows[slot][0][0], &st.bar[slot], (int)(first * 2u),
                      (int)((t + kTileSlots) * kTileRows));
        }
    }
    if (lost) {
        // record the fault, then let the tiles still in flight land before
        // the block's shared memory goes away
        if (threadIdx.x == 0) {
            atomicCAS(&a.glob->fault, 0u, kFaultTmaTimeout);
            for (uint32_t t = 0; t < tiles && t < (uint32_t)kTileSlots; t++)
                bar_wait(&st.bar[t], 0u);
        }
        __syncthreads();
    }
    combine_parts(s);
    return s;
#endif
}

// Sum of one heat-current sample's three components over the block into
// series slot 1 + 3 * sample: one atomic each (integer sums, any order).
__device__ __forceinline__ void block_sum_series(const Arena& a, const long long (&raw)[3],
                                                 uint32_t sample) {
    __shared__ long long s_sum[kBlock / 32][3];  // blocks of up to kBlock threads
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        long long x = raw[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) s_sum[warp][c] = x;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        long long x = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) x += s_sum[w][threadIdx.x];
        if (x) atomicAdd(&a.series[1 + 3 * (size_t)sample + threadIdx.x], (unsigned long long)x);
    }
}

// Langevin noise of a particle at a step: Philox-4x32-10 (Salmon et al.,
// SC'11) with counter (id, step lo, step hi, 0) and key (seed, "LJV1");
// uniforms in (0, 1] from 24 bits as the reference's uniform01
// (lennard_jones.wgsl:175-178); Box-Muller in f32: x and y from the first
// pair of uniforms (cosine and sine), z from the second (cosine).
__device__ __forceinline__ void langevin_noise(uint32_t id, unsigned long long step,
                                               uint32_t seed, float xi[3]) {
    const uint4 r = philox(id, step, seed);
    // (q + 1) / 2^24 for a 24-bit q: the sum is exact and so is scaling by a
    // power of two, so the product is the IEEE quotient
    const float scale = 5.9604644775390625e-08f;  // 2^-24
    const float u0 = ((float)(r.x >> 8) + 1.0f) * scale;
    const float u1 = ((float)(r.y >> 8) + 1.0f) * scale;
    const float u2 = ((float)(r.z >> 8) + 1.0f) * scale;
    const float u3 = ((float)(r.w >> 8) + 1.0f) * scale;
    const float ra = sqrtf(-2.0f * logf(u0));
    const float aa = 6.283185307179586f * u1;
    const float rb = sqrtf(-2.0f * logf(u2));
    const float ab = 6.283185307179586f * u3;
    xi[0] = ra * cosf(aa);
    xi[1] = ra * sinf(aa);
    xi[2] = rb * cosf(ab);
}

// The heat current of slot i in the state a step starts from, as the
// sampling kernel takes it: J_i = e_i v_i + T_i v_i / 2 with the canonical
// velocity v_i = v + a dt / 2 (one box, velocities half a kick behind), each
// component to 32.32 fixed point, added into raw.
__device__ __forceinline__ void heat_terms(const Arena& a, const Box& bx, uint32_t i,
                                           const PairSums& s, long long (&raw)[3]) {
    const float acc3[3] = {s.ax, s.ay, s.az};
    double v[3];
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = canonical_velocity(a, bx, 0, i, c, acc3[c]);
    const double e = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + (double)s.e_half;
    const double tv[3] = {s.t[0] * v[0] + s.t[3] * v[1] + s.t[4] * v[2],
                          s.t[3] * v[0] + s.t[1] * v[1] + s.t[5] * v[2],
                          s.t[4] * v[0] + s.t[5] * v[1] + s.t[2] * v[2]};
#pragma unroll
    for (int c = 0; c < 3; c++) raw[c] += fixed_raw_f64(e * v[c] + 0.5 * tv[c]);
}

// begin + force_kick of the reference for slot i (lennard_jones.wgsl:204-276,
// 556-574), with its forces in s: the stored velocity is half a kick behind,
// so the two half kicks go on together, then the drift: x += v dt (constant
// energy), or the Langevin A-O-A: x += v dt/2; v = c1 v + c2 xi; x += v dt/2.
// State in f64; the new position goes to the other cache copy (neighbours
// still read this step's). Returns the squared displacement since the last
// list build.
__device__ __forceinline__ float advance_slot(const Arena& a, const Box& bx, uint32_t i,
                                              uint32_t phase, const PairSums& s) {
    const float acc[3] = {s.ax, s.ay, s.az};
    float xi[3] = {0.0f, 0.0f, 0.0f};
    const bool langevin = bx.thermostat == 1;
    if (langevin) langevin_noise(a.id[i], a.glob->step, bx.seed, xi);
    const uint4 snap = a.snap[i];
    const uint32_t sw[3] = {snap.x, snap.y, snap.z};
    uint32_t enc[3];
    float disp2 = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const size_t q = (size_t)k * a.seg + i;
        double x = a.x[q];
        double v = a.v[q] + (double)acc[k] * bx.dt;
        if (langevin) {
            x += v * bx.half_dt;
            v = bx.c1 * v + bx.c2 * (double)xi[k];
            x += v * bx.half_dt;
        } else {
            x += v * bx.dt;
        }
        x = wrap(x, bx.box[k]);
        a.x[q] = x;
        a.v[q] = v;
        enc[k] = encode(x, bx.enc[k]);
        const float d = decode_diff(enc[k], sw[k], bx.dec[k]);
        disp2 += d * d;
    }
    a.cache[phase ^ 1u][i] = make_uint4(enc[0], enc[1], enc[2], 0u);
    return disp2;
}

// ---- prime (lennard_jones.wgsl:547-553): first forces; the stored velocity
// becomes half a kick behind the given one ----
template <bool SHIFTED_FORCE>
__global__ void __launch_bounds__(kForceThreads) prime_kernel(Arena a,
                                                              const __grid_constant__ CUtensorMap map) {
    count_kernel(a);
    __shared__ __align__(128) Stage st;
    const uint32_t i = blockIdx.x * kForceThreads + threadIdx.x;
    const bool valid = i < a.nslots;
    const Box& bx = a.boxes[valid ? box_of_slot(a, i) : 0u];
    const PairSums s =
        block_pair_sums<SHIFTED_FORCE, false>(st, &map, a, bx, i, valid, a.cache[a.glob->phase]);
    if (!valid) return;
    a.v[i] -= (double)s.ax * bx.half_dt;
    a.v[a.seg + i] -= (double)s.ay * bx.half_dt;
    a.v[2 * (size_t)a.seg + i] -= (double)s.az * bx.half_dt;
}

// ---- one step: begin + force_kick of the reference fused
// (lennard_jones.wgsl:204-276, 556-574) ----
// The stored velocity is half a kick behind, so this kernel's force pass
// applies the previous step's closing half kick and this step's opening half
// kick together, then drifts: x += v dt (constant energy), or the Langevin
// A-O-A: x += v dt/2; v = c1 v + c2 xi; x += v dt/2. State updates in f64.
// The new position goes to the other cache copy (neighbours still read this
// step's), and the largest squared displacement since the last list build
// feeds the next step's rebuild decision.
// The block's run of particles when the blocks that share an SM in the
// first wave take neighbouring runs (VLJ_STEP_REMAP): the hardware hands out
// blocks g, g + sms, g + 2 sms, ... to one SM in that wave, so within each
// group of sms x per_sm blocks the order is transposed; blocks past the last
// whole group keep their own run. A bijection on [0, n).
__device__ __forceinline__ uint32_t resident_neighbours(uint32_t b, uint32_t n, uint32_t sms,
                                                       uint32_t per_sm) {
    const uint32_t w = sms * per_sm;
    if (w == 0u || b >= n / w * w) return b;
    const uint32_t t = b % w;
    return b - t + (t % sms) * per_sm + t / sms;
}

// THREADS particles per block (Arena::step_threads, tuned per replica set
// by virial_lj.tune_batch; the TMA tile ring needs kForceThreads).
template <bool SHIFTED_FORCE, bool HEAT, int THREADS>
__global__ void __launch_bounds__(THREADS, kStepMinBlocks) step_kernel(Arena a,
                                                             const __grid_constant__ CUtensorMap map,
                                                             cudaGraphConditionalHandle next) {
    static_assert(VLJ_LIST_STREAM || THREADS == kForceThreads, "TMA tiles need kForceThreads");
    count_kernel(a);
    consume_decision(a);
    __shared__ __align__(128) Stage st;
#if VLJ_STEP_REMAP
    const uint32_t vb = resident_neighbours(blockIdx.x, gridDim.x, a.remap_sms, a.remap_per_sm);
#else
    const uint32_t vb = blockIdx.x;
#endif
    const uint32_t i = vb * THREADS + threadIdx.x;
    const bool valid = i < a.nslots;
    const uint32_t phase = a.glob->phase;
    const uint32_t b = valid ? box_of_slot(a, i) : 0u;
    const Box& bx = a.boxes[b];
    const PairSums s =
        block_pair_sums<SHIFTED_FORCE, false, HEAT>(st, &map, a, bx, i, valid, a.cache[phase]);
    if (HEAT) {
        const uint32_t sample = a.glob->heat_next;
        long long raw[3] = {0, 0, 0};
        if (valid) heat_terms(a, bx, i, s, raw);
        block_sum_series(a, raw, sample);
    }
    float disp2 = 0.0f;
    if (valid) disp2 = advance_slot(a, bx, i, phase, s);
    block_max_per_box(a, valid, b, vb * THREADS, disp2);
    if (i == 0) a.glob->pending = 1u;
    if (!next && !HEAT) return;
    // the last block to finish takes the next step's rebuild decision and
    // moves the heat-current series on
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&a.glob->blocks_done, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        a.glob->blocks_done = 0u;
        if (HEAT) a.glob->heat_next += 1u;
    }
    if (next) decide_block(a, next, true, true);
}

// ---- one step with two lanes per particle, for grids of a few blocks per
// SM (small boxes), whose lone warps cannot hide their latency behind each
// other's: lane h of a pair walks the particle's list rows h, h + 2, ...
// into one force part, the pair adds the two parts as combine_parts does
// (even rows' first), and lane 0 integrates. The same step as step_kernel
// to the bit (no heat-current sample). ----
template <bool SHIFTED_FORCE, int THREADS>
__global__ void __launch_bounds__(THREADS) step_kernel_split(Arena a, cudaGraphConditionalHandle next) {
    count_kernel(a);
    consume_decision(a);
    constexpr uint32_t kPer = THREADS / 2;  // particles per block
    const uint32_t h = threadIdx.x & 1u;
    const uint32_t i = blockIdx.x * kPer + (threadIdx.x >> 1);
    const bool valid = i < a.nslots;
    const uint32_t phase = a.glob->phase;
    const uint32_t b = valid ? box_of_slot(a, i) : 0u;
    const Box& bx = a.boxes[b];
    const uint4* __restrict__ cur = a.cache[phase];
    PairSums s = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u,
                  0.0f, {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}};
    if (valid) {
        const uint4 own = __ldg(cur + i);
        const uint32_t rows = (__ldg(a.list_count + i) + 3u) / 4u;
        const float dec0 = bx.dec[0], dec1 = bx.dec[1], dec2 = bx.dec[2];
        const float fshift = bx.force_shift;
        const uint32_t rc2_bits_m1 = __float_as_uint(bx.rc2) - 1u;
        const uint4* rowp = reinterpret_cast<const uint4*>(a.list) + i;
        uint4 nxt = h < rows ? load_row_streaming(rowp + (size_t)h * a.seg) : make_uint4(0u, 0u, 0u, 0u);
        for (uint32_t row = h; row < rows; row += 2u) {
            const uint4 e = nxt;
            if (row + 2u < rows) nxt = load_row_streaming(rowp + (size_t)(row + 2u) * a.seg);
            const uint4 p0 = __ldg(cur + e.x);
            const uint4 p1 = __ldg(cur + e.y);
            const uint4 p2 = __ldg(cur + e.z);
            const uint4 p3 = __ldg(cur + e.w);
            pair_terms<SHIFTED_FORCE, false, false, 0>(s, own, p0, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
            pair_terms<SHIFTED_FORCE, false, false, 0>(s, own, p1, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
            pair_terms<SHIFTED_FORCE, false, false, 0>(s, own, p2, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
            pair_terms<SHIFTED_FORCE, false, false, 0>(s, own, p3, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
        }
    }
    // lane 0 holds the even rows' part, lane 1 the odd rows'
    const float ox = __shfl_xor_sync(0xffffffffu, s.ax, 1);
    const float oy = __shfl_xor_sync(0xffffffffu, s.ay, 1);
    const float oz = __shfl_xor_sync(0xffffffffu, s.az, 1);
    s.ax = __fadd_rn(s.ax, ox);
    s.ay = __fadd_rn(s.ay, oy);
    s.az = __fadd_rn(s.az, oz);
    const bool mine = valid && h == 0u;
    float disp2 = 0.0f;
    if (mine) disp2 = advance_slot(a, bx, i, phase, s);
    block_max_per_box(a, mine, b, blockIdx.x * kPer, disp2);
    if (i == 0 && h == 0u) a.glob->pending = 1u;
    if (!next) return;
    // the last block to finish takes the next step's rebuild decision
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&a.glob->blocks_done, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) a.glob->blocks_done = 0u;
    decide_block(a, next, true, true);
}

// ---- one step over cell tiles: the same step as step_kernel, with the
// neighbour positions staged in shared memory ----
// A block takes one brick (a run of cells along x in one row of the box; the
// bricks tile the box) and stages its tile -- the encoded positions of every
// particle in the nine neighbour rows of those cells, each row one or two
// runs of the sorted order -- in shared memory, 16 B a particle. Its threads
// take the brick's home particles in sorted order; each walks its list as
// 16-bit tile indices (eight to a 16-byte row, streamed past L1), so every
// neighbour read is a shared-memory load instead of a scattered global
// gather. The list order and the pair arithmetic are step_kernel's, so the
// step is the same to the bit. A brick whose tile would not fit in
// a.tile_cap entries walks the slot list with global gathers instead.
template <bool SHIFTED_FORCE, bool HEAT>
__global__ void __launch_bounds__(kBlock) tile_step_kernel(Arena a, cudaGraphConditionalHandle next) {
    count_kernel(a);
    consume_decision(a);
    extern __shared__ __align__(16) uint4 s_tile[];
    __shared__ uint32_t s_run[9][3];  // per tile row: first run's sorted start, its length, second run's start
    __shared__ uint32_t s_base[10];   // tile index of each row's first particle; [9]: the tile's size
    __shared__ uint32_t s_home[3];    // the brick's home particles' sorted range; [2]: first one's tile index
    const uint32_t phase = a.glob->phase;
    const uint4* __restrict__ cur = a.cache[phase];
    const Box& bx = a.boxes[0];
    const Brick k = brick_at(bx, blockIdx.x - bx.brick_base);
    const uint32_t* __restrict__ cs = a.cell_start;
    if (threadIdx.x < 9u) {
        const uint32_t row = tile_row_cell(bx, k, threadIdx.x);
        const uint32_t nx = bx.cells[0], end = k.x_start + k.rx;
        const uint32_t first = cs[row + k.x_start];
        const uint32_t len1 = cs[row + min(end, nx)] - first;
        const uint32_t len2 = end > nx ? cs[row + end - nx] - cs[row] : 0u;
        s_run[threadIdx.x][0] = first;
        s_run[threadIdx.x][1] = len1;
        s_run[threadIdx.x][2] = cs[row];
        s_base[threadIdx.x + 1] = len1 + len2;
    } else if (threadIdx.x == 32u) {
        const uint32_t row = tile_row_cell(bx, k, 4u);
        s_home[0] = cs[row + k.x0];
        s_home[1] = cs[row + k.x0 + k.w];
        s_home[2] = tile_row_prefix(cs, bx, k, row, tile_col(bx, k, k.x0, 0));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s_base[0] = 0u;
        for (int r = 0; r < 9; r++) s_base[r + 1] += s_base[r];
    }
    __syncthreads();
    const uint32_t tile_size = s_base[9];
    // until a build has written the tile lists for these bricks (tiles just
    // switched on or resized), every block takes the slot list
    const bool staged = tile_size <= a.tile_cap && a.glob->tiles_ready != 0u;
#if VLJ_TILE_F32
    // the tile as f32 offsets from the brick's centre (encoded)
    const uint32_t org[3] = {
        encode(((double)k.x0 + 0.5 * (double)k.w) * (double)bx.cell_size_f[0], bx.enc[0]),
        encode(((double)k.y + 0.5) * (double)bx.cell_size_f[1], bx.enc[1]),
        encode(((double)k.z + 0.5) * (double)bx.cell_size_f[2], bx.enc[2])};
    float4* s_tilef = reinterpret_cast<float4*>(s_tile);
#endif
    if (staged) {
        for (uint32_t t = threadIdx.x; t < tile_size; t += blockDim.x) {
            uint32_t rho = 0;
            while (t >= s_base[rho + 1]) rho++;
            const uint32_t q = t - s_base[rho];
            const uint32_t p = q < s_run[rho][1] ? s_run[rho][0] + q : s_run[rho][2] + (q - s_run[rho][1]);
#if VLJ_TILE_F32
            const uint4 w = cur[a.sorted[p]];
            s_tilef[t] = make_float4(decode_diff(w.x, org[0], bx.dec[0]), decode_diff(w.y, org[1], bx.dec[1]),
                                     decode_diff(w.z, org[2], bx.dec[2]), 0.0f);
#else
            s_tile[t] = cur[a.sorted[p]];
#endif
        }
    }
    __syncthreads();
    const uint32_t h0 = s_home[0], h1 = s_home[1];
    const uint32_t own0 = s_base[4] + s_home[2] - h0;  // tile index of home p: own0 + p
    const float dec0 = bx.dec[0], dec1 = bx.dec[1], dec2 = bx.dec[2];
    const float fshift = bx.force_shift;
    const uint32_t rc2_bits_m1 = __float_as_uint(bx.rc2) - 1u;
    float disp2 = 0.0f;
    long long raw[3] = {0, 0, 0};
    const uint32_t sample = HEAT ? a.glob->heat_next : 0u;
    for (uint32_t p = h0 + threadIdx.x; p < h1; p += blockDim.x) {
        const uint32_t i = a.sorted[p];
        const uint32_t cnt = a.list_count[i];
        PairSums s = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0u,
                      0.0f, {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}};
        if (staged) {
#if VLJ_TILE_F32
            const float4 own = s_tilef[own0 + p];
            // a 16-bit row's first four entries are a slot-list row of even
            // index (add0), its last four one of odd index (add1)
            auto add0 = [&](const float4 pj) {
                pair_terms_rel<SHIFTED_FORCE, HEAT, 0>(s, own, pj, bx, rc2_bits_m1, fshift);
            };
            auto add1 = [&](const float4 pj) {
                pair_terms_rel<SHIFTED_FORCE, HEAT, 1>(s, own, pj, bx, rc2_bits_m1, fshift);
            };
            auto fetch = [&](uint32_t t) { return s_tilef[t]; };
            using Pos = float4;
#else
            const uint4 own = s_tile[own0 + p];
            auto add0 = [&](const uint4 pj) {
                pair_terms<SHIFTED_FORCE, false, HEAT, 0>(s, own, pj, bx, dec0, dec1, dec2,
                                                          rc2_bits_m1, fshift);
            };
            auto add1 = [&](const uint4 pj) {
                pair_terms<SHIFTED_FORCE, false, HEAT, 1>(s, own, pj, bx, dec0, dec1, dec2,
                                                          rc2_bits_m1, fshift);
            };
            auto fetch = [&](uint32_t t) { return s_tile[t]; };
            using Pos = uint4;
#endif
            const uint4* rowp = reinterpret_cast<const uint4*>(a.list16) + p;
            const uint32_t rows = (cnt + 7u) / 8u;
            uint4 nxt = rows ? load_row_streaming(rowp) : make_uint4(0u, 0u, 0u, 0u);
#if VLJ_TILE_PIPE
            // the next row's eight neighbours are read while this row's pairs
            // are computed
            Pos q[8];
            if (rows) {
                const uint4 e = nxt;
                if (rows > 1u) nxt = load_row_streaming(rowp + a.seg);
                q[0] = fetch(e.x & 0xffffu); q[1] = fetch(e.x >> 16);
                q[2] = fetch(e.y & 0xffffu); q[3] = fetch(e.y >> 16);
                q[4] = fetch(e.z & 0xffffu); q[5] = fetch(e.z >> 16);
                q[6] = fetch(e.w & 0xffffu); q[7] = fetch(e.w >> 16);
            }
            for (uint32_t row = 0; row < rows; row++) {
                Pos c[8];
#pragma unroll
                for (int m = 0; m < 8; m++) c[m] = q[m];
                if (row + 1u < rows) {
                    const uint4 e = nxt;
                    if (row + 2u < rows) nxt = load_row_streaming(rowp + (size_t)(row + 2u) * a.seg);
                    q[0] = fetch(e.x & 0xffffu); q[1] = fetch(e.x >> 16);
                    q[2] = fetch(e.y & 0xffffu); q[3] = fetch(e.y >> 16);
                    q[4] = fetch(e.z & 0xffffu); q[5] = fetch(e.z >> 16);
                    q[6] = fetch(e.w & 0xffffu); q[7] = fetch(e.w >> 16);
                }
#pragma unroll
                for (int m = 0; m < 4; m++) add0(c[m]);
#pragma unroll
                for (int m = 4; m < 8; m++) add1(c[m]);
            }
#else
            for (uint32_t row = 0; row < rows; row++) {
                const uint4 e = nxt;
                if (row + 1u < rows) nxt = load_row_streaming(rowp + (size_t)(row + 1u) * a.seg);
                add0(fetch(e.x & 0xffffu));
                add0(fetch(e.x >> 16));
                add0(fetch(e.y & 0xffffu));
                add0(fetch(e.y >> 16));
                add1(fetch(e.z & 0xffffu));
                add1(fetch(e.z >> 16));
                add1(fetch(e.w & 0xffffu));
                add1(fetch(e.w >> 16));
            }
#endif
        } else {
            const uint4 own = cur[i];
            const uint4* rowp = reinterpret_cast<const uint4*>(a.list) + i;
            const uint32_t rows = (cnt + 3u) / 4u;
            for (uint32_t row = 0; row < rows; row++) {
                const uint4 e = load_row_streaming(rowp + (size_t)row * a.seg);
                const uint4 p0 = __ldg(cur + e.x), p1 = __ldg(cur + e.y);
                const uint4 p2 = __ldg(cur + e.z), p3 = __ldg(cur + e.w);
                if (row & 1u) {
                    pair_terms<SHIFTED_FORCE, false, HEAT, 1>(s, own, p0, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
                    pair_terms<SHIFTED_FORCE, false, HEAT, 1>(s, own, p1, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
                    pair_terms<SHIFTED_FORCE, false, HEAT, 1>(s, own, p2, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
                    pair_terms<SHIFTED_FORCE, false, HEAT, 1>(s, own, p3, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
                } else {
                    pair_terms<SHIFTED_FORCE, false, HEAT, 0>(s, own, p0, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
                    pair_terms<SHIFTED_FORCE, false, HEAT, 0>(s, own, p1, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
                    pair_terms<SHIFTED_FORCE, false, HEAT, 0>(s, own, p2, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
                    pair_terms<SHIFTED_FORCE, false, HEAT, 0>(s, own, p3, bx, dec0, dec1, dec2, rc2_bits_m1, fshift);
                }
            }
        }
        combine_parts(s);
        if (HEAT) heat_terms(a, bx, i, s, raw);
        disp2 = fmaxf(disp2, advance_slot(a, bx, i, phase, s));
    }
    if (HEAT) block_sum_series(a, raw, sample);
    block_max_per_box(a, true, 0u, 0u, disp2);
    if (blockIdx.x == 0 && threadIdx.x == 0) a.glob->pending = 1u;
    if (!next && !HEAT) return;
    // the last block to finish takes the next step's rebuild decision and
    // moves the heat-current series on
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&a.glob->blocks_done, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        a.glob->blocks_done = 0u;
        if (HEAT) a.glob->heat_next += 1u;
    }
    if (next) decide_block(a, next, true, true);
}

// ---- measure (lennard_jones.wgsl:576-626) ----
// Per particle: half of each pair energy and virial, neighbours within
// 1.5 sigma, the velocity at the step (stored velocity plus the closing half
// kick), kinetic energy and momentum in f64. Each value goes to 32.32 fixed
// point scaled like the reference and is summed exactly.
template <bool SHIFTED_FORCE>
__global__ void __launch_bounds__(kForceThreads) measure_kernel(Arena a,
                                                                const __grid_constant__ CUtensorMap map,
                                                                int canonical) {
    count_kernel(a);
    __shared__ __align__(128) Stage st;
    const uint32_t i = blockIdx.x * kForceThreads + threadIdx.x;
    const bool valid = i < a.nslots;
    const uint32_t b = valid ? box_of_slot(a, i) : 0u;
    const Box& bx = a.boxes[b];
    const PairSums s =
        block_pair_sums<SHIFTED_FORCE, true>(st, &map, a, bx, i, valid, a.cache[a.glob->phase]);
    long long v[kSlots] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (valid) {
        const float acc[3] = {s.ax, s.ay, s.az};
        double vel[3], ke = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            vel[k] = canonical_velocity(a, bx, b, i, k, acc[k]);
            ke += vel[k] * vel[k];
            if (canonical) a.vcanon[(size_t)k * a.seg + i] = vel[k];
        }
        ke *= 0.5;
        const double es = (double)bx.energy_scale, ms = (double)bx.momentum_scale;
        v[0] = fixed_raw_f64(ke * es);
        v[1] = fixed_raw_f32(s.pe * bx.energy_scale) + fixed_raw_f32(s.pe_lo * bx.energy_scale);
        v[2] = fixed_raw_f32(s.w * bx.energy_scale) + fixed_raw_f32(s.w_lo * bx.energy_scale);
#pragma unroll
        for (int k = 0; k < 3; k++) v[3 + k] = fixed_raw_f64(vel[k] * ms);
        v[6] = s.near >= bx.near_count ? (1ll << 32) : 0ll;
        a.pe_half[2 * i] = s.pe;
        a.pe_half[2 * i + 1] = s.pe_lo;
        a.w_half[2 * i] = s.w;
        a.w_half[2 * i + 1] = s.w_lo;
        a.vel4[i] = make_float4((float)vel[0], (float)vel[1], (float)vel[2], (float)s.near);
    }
    block_sum_slots(a, valid, b, blockIdx.x * kForceThreads, v);
}

// ---- steps on canonical velocities: Nose-Hoover (lennard_jones.wgsl:309-397)
// and the heat exchange (lennard_jones.wgsl:732-893); host order
// lennard_jones.rs:1108-1138 ----
// One box. A step runs begin (Nose-Hoover's pending end-half scale s2 of the
// last step and this step's start-half scale s1, the half kick, the drift),
// the decision and rebuild, then canon_force (forces, the closing half kick,
// and the end-of-step sums: the kinetic energy for Nose-Hoover, the slab sums
// for the exchange; the block that finishes last turns them into the
// thermostat update or the exchange coefficients), then for the exchange
// hex_apply. The stored velocity is canonical (before Nose-Hoover's s2).

// begin: every thread takes the start half step from the same state, so all
// of them compute the same s1; the box's first thread stores the result.
__global__ void __launch_bounds__(kBlock) begin_kernel(Arena a) {
    count_kernel(a);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < a.nslots;
    const uint32_t phase = a.glob->phase;
    const uint32_t b = valid ? box_of_slot(a, i) : 0u;
    const Box& bx = a.boxes[b];
    float disp2 = 0.0f;
    if (valid) {
        double s2 = 1.0, s1 = 1.0;  // exact no-ops without Nose-Hoover
        if (bx.thermostat == 2) {
            const Thermo& t = a.nh[b];
            double xi = t.xi_m, eta = t.eta_m, ke = t.ke_m;
            s2 = t.scale;
            s1 = nh_half(bx, xi, eta, ke);
            if (i == bx.first) {
                a.nh[b].xi_s = xi;
                a.nh[b].eta_s = eta;
            }
        }
        const float4 f = a.acc[i];
        const float acc[3] = {f.x, f.y, f.z};
        const uint4 snap = a.snap[i];
        const uint32_t sw[3] = {snap.x, snap.y, snap.z};
        uint32_t enc[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const size_t q = (size_t)k * a.seg + i;
            // the two half steps' scalings in turn, then the half kick
            const double v = a.v[q] * s2 * s1 + (double)acc[k] * bx.half_dt;
            const double x = wrap(a.x[q] + v * bx.dt, bx.box[k]);
            a.x[q] = x;
            a.v[q] = v;
            enc[k] = encode(x, bx.enc[k]);
            const float d = decode_diff(enc[k], sw[k], bx.dec[k]);
            disp2 += d * d;
        }
        a.cache[phase ^ 1u][i] = make_uint4(enc[0], enc[1], enc[2], 0u);
    }
    block_max_per_box(a, valid, b, blockIdx.x * blockDim.x, disp2);
    if (i == 0) a.glob->pending = 1u;
}

// The exchange slab of height z (f32, as the reference): 0 hot, 1 cold, 2 neither.
__device__ __forceinline__ int hex_slab(const Box& bx, double z) {
    const float zf = (float)z;
    if (zf >= bx.hex_slabs[0] && zf < bx.hex_slabs[1]) return 0;
    if (zf >= bx.hex_slabs[2] && zf < bx.hex_slabs[3]) return 1;
    return 2;
}

// The exchange's per-slab scale and eHEX/a correction coefficients from the
// slab sums (lennard_jones.wgsl:804-856), in f64; clears the sums.
__device__ void hex_coefficients(const Box& bx, Exchange* h) {
    const double one = 4294967296.0;
    const double es = (double)bx.energy_scale, ms = (double)bx.momentum_scale;
    const double dt = bx.dt, dt3 = dt * dt * dt;
    for (int sl = 0; sl < 2; sl++) {
        long long raw[9];
        for (int k = 0; k < 9; k++) {
            raw[k] = (long long)h->sums[sl][k];
            h->sums[sl][k] = 0ull;
        }
        const double m = (double)raw[0] / one;
        double p[3], f[3];
        for (int k = 0; k < 3; k++) {
            p[k] = (double)raw[1 + k] / one / ms;
            f[k] = (double)raw[6 + k] / one / ms;
        }
        const double v2 = (double)raw[4] / one / es, fv = (double)raw[5] / one / es;
        double com[3] = {0.0, 0.0, 0.0}, mf[3] = {0.0, 0.0, 0.0};
        double sm1 = 0.0, cv = 0.0, cf = 0.0;
        if (m > 0.0) {
            for (int k = 0; k < 3; k++) {
                com[k] = p[k] / m;
                mf[k] = f[k] / m;
            }
            // kinetic energy about the centre of mass
            const double kinetic = 0.5 * v2 - 0.5 * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) / m;
            const double energy = (sl == 0 ? 1.0 : -1.0) * bx.hex_energy;
            const double flux = energy / dt;
            const double x = energy / kinetic;
            sm1 = x / (1.0 + sqrt(1.0 + x));  // sqrt(1 + x) - 1
            const double power = fv - (f[0] * com[0] + f[1] * com[1] + f[2] * com[2]);
            cv = dt3 * flux / (2.0 * kinetic * kinetic) * (flux / 48.0 + power / 6.0);
            cf = dt3 * flux / (12.0 * kinetic);
        }
        for (int k = 0; k < 3; k++) {
            h->com[sl][k] = com[k];
            h->mean_f[sl][k] = mf[k];
        }
        h->s_minus_1[sl] = sm1;
        h->c_v[sl] = cv;
        h->c_f[sl] = cf;
    }
}

// canon_force: forces from the list, stored; the closing half kick (not for
// kPrime); the end-of-step sums in 32.32 fixed point, added per block, and in
// the last block to finish the Nose-Hoover update or the exchange
// coefficients.
template <bool SHIFTED_FORCE, int PASS>
__global__ void __launch_bounds__(kForceThreads) canon_force_kernel(Arena a,
                                                                    const __grid_constant__ CUtensorMap map) {
    count_kernel(a);
    __shared__ __align__(128) Stage st;
    __shared__ unsigned long long s_sum[2][9];
    __shared__ int s_last;
    const uint32_t i = blockIdx.x * kForceThreads + threadIdx.x;
    const bool valid = i < a.nslots;
    const Box& bx = a.boxes[0];
    if (threadIdx.x < 18) s_sum[threadIdx.x / 9][threadIdx.x % 9] = 0ull;
    const PairSums s =
        block_pair_sums<SHIFTED_FORCE, false>(st, &map, a, bx, i, valid, a.cache[a.glob->phase]);
    if (valid) {
        const float acc[3] = {s.ax, s.ay, s.az};
        a.acc[i] = make_float4(s.ax, s.ay, s.az, 0.0f);
        double v[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const size_t q = (size_t)k * a.seg + i;
            v[k] = a.v[q];
            if (PASS != kPrime) {
                v[k] += (double)acc[k] * bx.half_dt;
                a.v[q] = v[k];
            }
        }
        const double es = (double)bx.energy_scale, ms = (double)bx.momentum_scale;
        if (PASS == kPrime || PASS == kNoseHoover) {
            const long long raw = fixed_raw_f64(0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * es);
            if (raw) atomicAdd(&s_sum[0][0], (unsigned long long)raw);
        }
        if (PASS == kExchange) {
            const int sl = hex_slab(bx, a.x[2 * (size_t)a.seg + i]);
            if (sl < 2) {
                unsigned long long* t = s_sum[sl];
                atomicAdd(&t[0], 1ull << 32);
                for (int k = 0; k < 3; k++) {
                    atomicAdd(&t[1 + k], (unsigned long long)fixed_raw_f64(v[k] * ms));
                    atomicAdd(&t[6 + k], (unsigned long long)fixed_raw_f64((double)acc[k] * ms));
                }
                atomicAdd(&t[4], (unsigned long long)fixed_raw_f64(
                                     (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * es));
                atomicAdd(&t[5], (unsigned long long)fixed_raw_f64(
                                     ((double)acc[0] * v[0] + (double)acc[1] * v[1] +
                                      (double)acc[2] * v[2]) * es));
            }
        }
    }
    if (PASS == kKick) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t* done;
        if (PASS == kExchange) {
            for (int sl = 0; sl < 2; sl++)
                for (int k = 0; k < 9; k++)
                    if (s_sum[sl][k]) atomicAdd(&a.hex->sums[sl][k], s_sum[sl][k]);
            done = &a.hex->blocks_done;
        } else {
            if (s_sum[0][0]) atomicAdd(&a.nh->ke_raw, s_sum[0][0]);
            done = &a.nh->blocks_done;
        }
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    // every other block's sums are in
    __threadfence();
    if (PASS == kExchange) {
        a.hex->blocks_done = 0u;
        hex_coefficients(bx, a.hex);
        return;
    }
    Thermo* t = a.nh;
    const long long total = (long long)atomicExch(&t->ke_raw, 0ull);
    t->blocks_done = 0u;
    double ke = (double)total / 4294967296.0 / (double)bx.energy_scale;
    if (PASS == kPrime) {
        t->ke_m = ke;
        t->scale = 1.0;
        return;
    }
    double xi = t->xi_s, eta = t->eta_s;
    const double s2 = nh_half(bx, xi, eta, ke);
    t->xi_m = xi;
    t->eta_m = eta;
    t->ke_m = ke;
    t->scale = s2;
}

// hex_apply (lennard_jones.wgsl:858-893): in each slab, the position
// correction -dt^3 E_i from the velocity before scaling, then
// v <- v + (s - 1)(v - v_com); the moved positions go back into the current
// position copy.
__global__ void __launch_bounds__(kBlock) hex_apply_kernel(Arena a) {
    count_kernel(a);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nslots) return;
    const Box& bx = a.boxes[0];
    const int sl = hex_slab(bx, a.x[2 * (size_t)a.seg + i]);
    if (sl == 2) return;
    const Exchange& h = *a.hex;
    const float4 f = a.acc[i];
    const float acc[3] = {f.x, f.y, f.z};
    uint32_t enc[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const size_t q = (size_t)k * a.seg + i;
        const double v = a.v[q];
        const double rel = v - h.com[sl][k];
        const double shift = h.c_v[sl] * rel - h.c_f[sl] * ((double)acc[k] - h.mean_f[sl][k]);
        const double x = wrap(a.x[q] - shift, bx.box[k]);
        a.x[q] = x;
        a.v[q] = v + h.s_minus_1[sl] * rel;
        enc[k] = encode(x, bx.enc[k]);
    }
    a.cache[a.glob->phase][i] = make_uint4(enc[0], enc[1], enc[2], 0u);
}

// Canonical velocities back to half a kick behind, with the stored forces.
__global__ void __launch_bounds__(kBlock) half_kick_back_kernel(Arena a) {
    count_kernel(a);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nslots) return;
    const Box& bx = a.boxes[0];
    const float4 f = a.acc[i];
    a.v[i] -= (double)f.x * bx.half_dt;
    a.v[a.seg + i] -= (double)f.y * bx.half_dt;
    a.v[2 * (size_t)a.seg + i] -= (double)f.z * bx.half_dt;
}

// ---- FP32 calibration: eight independent FMA chains per thread, so the
// FMA pipes stay full; 2 flops per FMA ----
__global__ void __launch_bounds__(kBlock) fp32_peak_kernel(float* out, int iters) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = (float)(threadIdx.x + k) * 1e-3f;
    const float m = 0.999999f, c = 1e-6f;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fmaf(x[k], m, c);
    }
    float t = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) t += x[k];
    if (t == 12345.678f) out[blockIdx.x] = t;  // keeps the chains live
}

// ---- the noise stream as the step kernel draws it, for known-answer checks:
// Philox-4x32-10 of each (counter, key), and the Langevin noise of
// (id = ctr.x, step = ctr.y + 2^32 ctr.z, seed = key.x) ----
__global__ void __launch_bounds__(kBlock) philox_check_kernel(const uint4* __restrict__ ctr,
                                                              const uint2* __restrict__ key,
                                                              uint32_t n, uint4* __restrict__ out,
                                                              float4* __restrict__ noise) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint4 c = ctr[k];
    const uint2 q = key[k];
    out[k] = philox4x32_10(c, q);
    float xi[3];
    langevin_noise(c.x, (unsigned long long)c.y | ((unsigned long long)c.z << 32), q.x, xi);
    noise[k] = make_float4(xi[0], xi[1], xi[2], 0.0f);
}

cudaError_t launch_philox_check(const uint4* ctr, const uint2* key, uint32_t n, uint4* out,
                                float4* noise, cudaStream_t s) {
    philox_check_kernel<<<blocks_for(n), kBlock, 0, s>>>(ctr, key, n, out, noise);
    return after_launch();
}

// ---- launchers ----
static unsigned particle_blocks(const Arena& a) {
    return blocks_for(a.nslots, kForceThreads);
}

// With the list streamed from global memory the force kernels use no shared
// memory to speak of; ask for the largest L1 (it caches the gathers).
#ifndef VLJ_L1_CARVEOUT
#define VLJ_L1_CARVEOUT 4  // shared-memory carve-out hint, percent of the maximum (tuned)
#endif
template <class K>
static void prefer_l1(K kernel) {
#if VLJ_LIST_STREAM
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, VLJ_L1_CARVEOUT);
#else
    (void)kernel;
#endif
}

static void prefer_l1_once() {
    static bool done = false;
    if (done) return;
    done = true;
    prefer_l1(measure_kernel<true>);
    prefer_l1(measure_kernel<false>);
    prefer_l1(prime_kernel<true>);
    prefer_l1(prime_kernel<false>);
    prefer_l1(canon_force_kernel<true, kPrime>);
    prefer_l1(canon_force_kernel<false, kPrime>);
    prefer_l1(canon_force_kernel<true, kNoseHoover>);
    prefer_l1(canon_force_kernel<false, kNoseHoover>);
    prefer_l1(canon_force_kernel<true, kExchange>);
    prefer_l1(canon_force_kernel<false, kExchange>);
    prefer_l1(canon_force_kernel<true, kKick>);
    prefer_l1(canon_force_kernel<false, kKick>);
}

cudaError_t launch_prime(const Arena& a, const CUtensorMap& map, bool shifted_force,
                         cudaStream_t s) {
    prefer_l1_once();
    if (shifted_force)
        prime_kernel<true><<<particle_blocks(a), kForceThreads, 0, s>>>(a, map);
    else
        prime_kernel<false><<<particle_blocks(a), kForceThreads, 0, s>>>(a, map);
    return after_launch();
}

template <int THREADS>
static cudaError_t launch_step_kernel(const Arena& a, const CUtensorMap& map, bool shifted_force,
                                      cudaStream_t s, cudaGraphConditionalHandle next, bool heat) {
    static bool carved = false;
    if (!carved) {
        carved = true;
        prefer_l1(step_kernel<true, false, THREADS>);
        prefer_l1(step_kernel<false, false, THREADS>);
        prefer_l1(step_kernel<true, true, THREADS>);
        prefer_l1(step_kernel<false, true, THREADS>);
    }
    const unsigned blocks = blocks_for(a.nslots, THREADS);
#if VLJ_LIST_STREAM
    const bool split = a.step_lanes == 2u ||
                       (a.step_lanes == 0u && blocks <= (unsigned)sm_count() * kSplitBlocksPerSM);
    if (!heat && split) {
        // a grid of a few blocks per SM: two lanes per particle
        static bool split_carved = false;
        if (!split_carved) {
            split_carved = true;
            prefer_l1(step_kernel_split<true, THREADS>);
            prefer_l1(step_kernel_split<false, THREADS>);
        }
        const unsigned split_blocks = blocks_for(a.nslots, THREADS / 2);
        if (shifted_force) step_kernel_split<true, THREADS><<<split_blocks, THREADS, 0, s>>>(a, next);
        else step_kernel_split<false, THREADS><<<split_blocks, THREADS, 0, s>>>(a, next);
        return after_launch();
    }
#endif
    Arena r = a;
#if VLJ_STEP_REMAP
    static int per_sm = 0;
    if (!per_sm &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_kernel<true, false, THREADS>,
                                                      THREADS, 0) != cudaSuccess)
        per_sm = 0;
    r.remap_sms = (uint32_t)sm_count();
    r.remap_per_sm = (uint32_t)per_sm;
#endif
    if (shifted_force) {
        if (heat) step_kernel<true, true, THREADS><<<blocks, THREADS, 0, s>>>(r, map, next);
        else step_kernel<true, false, THREADS><<<blocks, THREADS, 0, s>>>(r, map, next);
    } else {
        if (heat) step_kernel<false, true, THREADS><<<blocks, THREADS, 0, s>>>(r, map, next);
        else step_kernel<false, false, THREADS><<<blocks, THREADS, 0, s>>>(r, map, next);
    }
    return after_launch();
}

template <bool SF, bool HEAT>
static cudaError_t launch_tile_step(const Arena& a, cudaStream_t s, cudaGraphConditionalHandle next) {
    const size_t smem = (size_t)a.tile_cap * sizeof(uint4);
    static size_t allowed = 0;  // dynamic shared memory the kernel was opened up to
    if (smem > allowed) {
        cudaError_t e = cudaFuncSetAttribute(tile_step_kernel<SF, HEAT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        cudaFuncSetAttribute(tile_step_kernel<SF, HEAT>,
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        allowed = smem;
    }
    tile_step_kernel<SF, HEAT><<<a.bricks, a.tile_threads, smem, s>>>(a, next);
    return after_launch();
}

cudaError_t launch_step(const Arena& a, const CUtensorMap& map, bool shifted_force,
                        cudaStream_t s, unsigned long long next_decision, bool heat) {
    prefer_l1_once();
    const cudaGraphConditionalHandle next = (cudaGraphConditionalHandle)next_decision;
    if (a.list16 && a.tile_threads) {
        if (shifted_force)
            return heat ? launch_tile_step<true, true>(a, s, next)
                        : launch_tile_step<true, false>(a, s, next);
        return heat ? launch_tile_step<false, true>(a, s, next)
                    : launch_tile_step<false, false>(a, s, next);
    }
#if VLJ_LIST_STREAM
    switch (a.step_threads) {
        case 64: return launch_step_kernel<64>(a, map, shifted_force, s, next, heat);
        case 256: return launch_step_kernel<256>(a, map, shifted_force, s, next, heat);
        default: return launch_step_kernel<kForceThreads>(a, map, shifted_force, s, next, heat);
    }
#else
    return launch_step_kernel<kForceThreads>(a, map, shifted_force, s, next, heat);
#endif
}

cudaError_t launch_measure(const Arena& a, const CUtensorMap& map, bool shifted_force,
                           bool canonical, cudaStream_t s) {
    prefer_l1_once();
    if (shifted_force)
        measure_kernel<true><<<particle_blocks(a), kForceThreads, 0, s>>>(a, map, canonical ? 1 : 0);
    else
        measure_kernel<false><<<particle_blocks(a), kForceThreads, 0, s>>>(a, map, canonical ? 1 : 0);
    return after_launch();
}

cudaError_t launch_begin(const Arena& a, cudaStream_t s) {
    begin_kernel<<<blocks_for(a.nslots), kBlock, 0, s>>>(a);
    return after_launch();
}

template <bool SF>
static void canon_force(const Arena& a, const CUtensorMap& map, CanonPass pass, cudaStream_t s) {
    const unsigned blocks = particle_blocks(a);
    switch (pass) {
        case kPrime: canon_force_kernel<SF, kPrime><<<blocks, kForceThreads, 0, s>>>(a, map); break;
        case kNoseHoover:
            canon_force_kernel<SF, kNoseHoover><<<blocks, kForceThreads, 0, s>>>(a, map);
            break;
        case kExchange:
            canon_force_kernel<SF, kExchange><<<blocks, kForceThreads, 0, s>>>(a, map);
            break;
        case kKick: canon_force_kernel<SF, kKick><<<blocks, kForceThreads, 0, s>>>(a, map); break;
    }
}

cudaError_t launch_canon_force(const Arena& a, const CUtensorMap& map, bool shifted_force,
                               CanonPass pass, cudaStream_t s) {
    prefer_l1_once();
    if (shifted_force)
        canon_force<true>(a, map, pass, s);
    else
        canon_force<false>(a, map, pass, s);
    return after_launch();
}

cudaError_t launch_hex_apply(const Arena& a, cudaStream_t s) {
    hex_apply_kernel<<<blocks_for(a.nslots), kBlock, 0, s>>>(a);
    return after_launch();
}

cudaError_t launch_half_kick_back(const Arena& a, cudaStream_t s) {
    half_kick_back_kernel<<<blocks_for(a.nslots), kBlock, 0, s>>>(a);
    return after_launch();
}

cudaError_t launch_fp32_peak(float* out, int blocks, int iters, cudaStream_t s) {
    fp32_peak_kernel<<<blocks, kBlock, 0, s>>>(out, iters);
    return after_launch();
}

}  // namespace vlj
