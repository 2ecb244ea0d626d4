// Sampling kernels, sm_100a: profiles along z (Irving-Kirkwood) and the
// microscopic heat current. Both walk each particle's Verlet list with the
// force kernels' pair arithmetic (the force factor, and the energy as the
// heat current's fused pass takes it) and add 32.32 fixed-point sums without
// a scale factor, as the reference does. The heat current walks each list in
// one thread, in list order, so the canonical velocity v + a dt/2 it needs is
// the measurement's bit for bit; the profile splits each list over several
// threads.
#include <cuda_runtime.h>

#include "vlj_device.cuh"
#include "vlj_internal.cuh"

namespace vlj {

constexpr int kSampleThreads = 128;
constexpr int kProfileSlots = 8;  // count, m v_a^2 (3), W_aa (3), PE

// Walks particle i's list in list order; for every pair inside the cutoff
// calls pair(dx, dy, dz, r2, rf, u) and accumulates the force as the force
// kernels do.
template <bool SHIFTED_FORCE, class Pair>
__device__ __forceinline__ void walk_pairs(const Arena& a, const Box& bx, uint32_t i,
                                           const uint4* __restrict__ cur, float& ax, float& ay,
                                           float& az, Pair pair) {
    const uint4 own = cur[i];
    const uint32_t cnt = a.list_count[i];
    ax = ay = az = 0.0f;
    for (uint32_t k = 0; k < cnt; k++) {
        const uint32_t j = a.list[((size_t)(k >> 2) * a.seg + i) * 4u + (k & 3u)];
        const uint4 pj = cur[j];
        const float dx = decode_diff(pj.x, own.x, bx.dec[0]);
        const float dy = decode_diff(pj.y, own.y, bx.dec[1]);
        const float dz = decode_diff(pj.z, own.z, bx.dec[2]);
        const float r2 = sep_r2(dx, dy, dz);
        if (!(r2 < bx.rc2)) continue;
        const float f = lj_force_over_r2<SHIFTED_FORCE>(r2, bx.force_shift);
        ax = __fmaf_rn(-dx, f, ax);
        ay = __fmaf_rn(-dy, f, ay);
        az = __fmaf_rn(-dz, f, az);
        float rf, u;
        lj_pair<SHIFTED_FORCE>(r2, bx, rf, u);
        pair(dx, dy, dz, r2, rf, u);
    }
}

// ---- profiles along z (lennard_jones.wgsl:644-730) ----
// Each particle books its count, m v_a^2 and half of each pair energy into its
// own slab, and half of each pair's virial tensor diagonal along the line to
// its partner, split over the slabs the line crosses in proportion to the
// length inside each (the last slab takes what is left, so the shares add up
// to one). After the slabs come three whole-box W_aa. The per-block sums
// collect in shared memory when they fit, then flush with one atomic per
// touched slot.
//
// kProfileLanes consecutive threads share a particle: each walks every
// kProfileLanes-th row of its list (four entries a row) and spreads those
// pairs; the force for the canonical velocity is their partial sums added
// in a fixed order (shuffles), so it is the same on every run. Samples of
// small boxes (the 16,000-atom slab) would otherwise give the GPU too few
// threads to hide a list walk's latency.
constexpr int kProfileLanes = 8;

template <bool SHIFTED_FORCE>
__global__ void __launch_bounds__(kSampleThreads) profile_kernel(Arena a, int in_shared) {
    count_kernel(a);
    extern __shared__ unsigned long long s_prof[];
    const Box& bx = a.boxes[0];
    const uint32_t bins = bx.profile_bins;
    const uint32_t words = bins * kProfileSlots + 3u;
    if (in_shared) {
        for (uint32_t t = threadIdx.x; t < words; t += blockDim.x) s_prof[t] = 0ull;
        __syncthreads();
    }
    unsigned long long* acc = in_shared ? s_prof : a.profile;
    auto add = [&](uint32_t slot, long long raw) {
        if (raw) atomicAdd(acc + slot, (unsigned long long)raw);
    };
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t / (uint32_t)kProfileLanes, sub = t % (uint32_t)kProfileLanes;
    const bool valid = i < a.nslots;
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    int32_t home = 0;
    if (valid) {
        const uint4* __restrict__ cur = a.cache[a.glob->phase];
        const float width = bx.bin_width, inv_width = 1.0f / width;
        const int32_t nb = (int32_t)bins;
        const float z = (float)a.x[2 * (size_t)a.seg + i];
        home = (int32_t)floorf(z / width);
        home = home < 0 ? 0 : (home > nb - 1 ? nb - 1 : home);
        float pe = 0.0f, tot[3] = {0.0f, 0.0f, 0.0f};
        const uint4 own = cur[i];
        const uint32_t cnt = a.list_count[i];
        const uint32_t rows = (cnt + 3u) / 4u;
        const uint4* rowp = reinterpret_cast<const uint4*>(a.list) + i;
        for (uint32_t r = sub; r < rows; r += (uint32_t)kProfileLanes) {
            const uint4 e = rowp[(size_t)r * a.seg];
            const uint32_t js[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
            for (int q4 = 0; q4 < 4; q4++) {
                const uint4 pj = cur[js[q4]];
                const float dx = decode_diff(pj.x, own.x, bx.dec[0]);
                const float dy = decode_diff(pj.y, own.y, bx.dec[1]);
                const float dz = decode_diff(pj.z, own.z, bx.dec[2]);
                const float r2 = sep_r2(dx, dy, dz);
                // the last row's padding (the particle itself) and the
                // entries past the cutoff drop out here
                if (!(r2 < bx.rc2) || r2 == 0.0f) continue;
                const float f = lj_force_over_r2<SHIFTED_FORCE>(r2, bx.force_shift);
                ax = __fmaf_rn(-dx, f, ax);
                ay = __fmaf_rn(-dy, f, ay);
                az = __fmaf_rn(-dz, f, az);
                pe += 0.5f * lj_energy_fast<SHIFTED_FORCE>(r2, bx);
                // f = |F| / r, so r_a F_a = d_a^2 f
                const float w[3] = {0.5f * dx * dx * f, 0.5f * dy * dy * f, 0.5f * dz * dz * f};
#pragma unroll
                for (int c = 0; c < 3; c++) tot[c] += w[c];
                const float lo = z + fminf(dz, 0.0f);
                const float hi = z + fmaxf(dz, 0.0f);
                const float length = hi - lo;
                if (length < 1e-6f * width) {
#pragma unroll
                    for (int c = 0; c < 3; c++) add(home * kProfileSlots + 4 + c, fixed_raw_f32(w[c]));
                    continue;
                }
                const float inv_length = 1.0f / length;
                int32_t b = (int32_t)floorf(lo * inv_width);
                float left = 1.0f;
                for (;;) {
                    const bool last = (float)(b + 1) * width >= hi;
                    const float start = fmaxf(lo, (float)b * width);
                    const float end = fminf(hi, (float)(b + 1) * width);
                    float share = last ? left : (end - start) * inv_length;
                    share = fmaxf(share, 0.0f);
                    left -= share;
                    // b lies within one box length of the home slab
                    const int32_t slab = b < 0 ? b + nb : (b >= nb ? b - nb : b);
#pragma unroll
                    for (int c = 0; c < 3; c++)
                        add((uint32_t)slab * kProfileSlots + 4 + c, fixed_raw_f32(w[c] * share));
                    if (last) break;
                    b += 1;
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) add(bins * kProfileSlots + c, fixed_raw_f32(tot[c]));
        add((uint32_t)home * kProfileSlots + 7, fixed_raw_f32(pe));
    }
    // the particle's force: its lanes' partial sums, added pairwise
#pragma unroll
    for (int o = 1; o < kProfileLanes; o <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    if (valid && sub == 0u) {
        const float acc3[3] = {ax, ay, az};
        add((uint32_t)home * kProfileSlots, 1ll << 32);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double v = canonical_velocity(a, bx, 0, i, c, acc3[c]);
            add((uint32_t)home * kProfileSlots + 1 + c, fixed_raw_f64(v * v));
        }
    }
    if (in_shared) {
        __syncthreads();
        for (uint32_t t2 = threadIdx.x; t2 < words; t2 += blockDim.x)
            if (s_prof[t2]) atomicAdd(&a.profile[t2], s_prof[t2]);
    }
}

// ---- heat current (lennard_jones.wgsl:895-947) ----
// J = sum_i e_i v_i + 1/2 sum_i sum_j (F_ij . v_i) r_ij, e_i the particle's
// kinetic energy plus half of each of its pair energies. With r_ij = -d and
// F_ij = -d rf / r^2 the pair term is T v_i for T = sum_j d d^T rf / r^2,
// which one list pass collects together with the force that the canonical
// velocity needs. Adds one sample into series slot 1 + 3 * sample.
template <bool SHIFTED_FORCE>
__global__ void __launch_bounds__(kSampleThreads) heat_current_kernel(Arena a, uint32_t sample) {
    count_kernel(a);
    // the series' count of written samples moves on (no other block reads it)
    if (blockIdx.x == 0 && threadIdx.x == 0) a.glob->heat_next = sample + 1u;
    const Box& bx = a.boxes[0];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < a.nslots;
    long long raw[3] = {0, 0, 0};
    if (valid) {
        float epair = 0.0f;
        float t[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};  // xx yy zz xy xz yz
        float ax, ay, az;
        walk_pairs<SHIFTED_FORCE>(a, bx, i, a.cache[a.glob->phase], ax, ay, az,
            [&](float dx, float dy, float dz, float r2, float rf, float u) {
                epair += 0.5f * u;
                const float q = rf / r2;
                t[0] += dx * dx * q;
                t[1] += dy * dy * q;
                t[2] += dz * dz * q;
                t[3] += dx * dy * q;
                t[4] += dx * dz * q;
                t[5] += dy * dz * q;
            });
        const float acc3[3] = {ax, ay, az};
        double v[3];
#pragma unroll
        for (int c = 0; c < 3; c++) v[c] = canonical_velocity(a, bx, 0, i, c, acc3[c]);
        const double e = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) + (double)epair;
        const double tv[3] = {t[0] * v[0] + t[3] * v[1] + t[4] * v[2],
                              t[3] * v[0] + t[1] * v[1] + t[5] * v[2],
                              t[4] * v[0] + t[5] * v[1] + t[2] * v[2]};
#pragma unroll
        for (int c = 0; c < 3; c++) raw[c] = fixed_raw_f64(e * v[c] + 0.5 * tv[c]);
    }
    // block sum of the three components, then one atomic each
    __shared__ long long s_sum[kSampleThreads / 32][3];
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
        for (int w = 0; w < kSampleThreads / 32; w++) x += s_sum[w][threadIdx.x];
        if (x) atomicAdd(&a.series[1 + 3 * (size_t)sample + threadIdx.x], (unsigned long long)x);
    }
}

// ---- drawn local temperature (lennard_jones.wgsl:595-602) ----
// Runs after the measure kernel, which left each particle's canonical
// velocity in vel4.xyz: (v_i^2 + sum over neighbours within the cutoff of
// v_j^2) / (3 (neighbours + 1)), into vel4.w.
__global__ void __launch_bounds__(kSampleThreads) drawn_temperature_kernel(Arena a) {
    count_kernel(a);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nslots) return;
    const Box& bx = a.boxes[box_of_slot(a, i)];
    const uint4* __restrict__ cur = a.cache[a.glob->phase];
    const uint4 own = cur[i];
    const uint32_t cnt = a.list_count[i];
    float v2 = 0.0f;
    uint32_t within = 0;
    for (uint32_t k = 0; k < cnt; k++) {
        const uint32_t j = a.list[((size_t)(k >> 2) * a.seg + i) * 4u + (k & 3u)];
        if (encoded_r2(cur[j], own, bx.dec) < bx.rc2) {
            const float4 vj = a.vel4[j];
            v2 += vj.x * vj.x + vj.y * vj.y + vj.z * vj.z;
            within += 1u;
        }
    }
    float4 vi = a.vel4[i];
    vi.w = (vi.x * vi.x + vi.y * vi.y + vi.z * vi.z + v2) / (3.0f * (float)(within + 1u));
    a.vel4[i] = vi;
}

cudaError_t launch_drawn_temperature(const Arena& a, cudaStream_t s) {
    drawn_temperature_kernel<<<blocks_for(a.nslots, kSampleThreads), kSampleThreads, 0, s>>>(a);
    return after_launch();
}

cudaError_t launch_profile(const Arena& a, uint32_t bins, bool shifted_force, cudaStream_t s) {
    const size_t words = (size_t)bins * kProfileSlots + 3;
    const size_t bytes = words * sizeof(unsigned long long);
    const int in_shared = bytes <= 48 * 1024 ? 1 : 0;
    const unsigned blocks = blocks_for((uint64_t)a.nslots * kProfileLanes, kSampleThreads);
    const size_t smem = in_shared ? bytes : 0;
    if (shifted_force)
        profile_kernel<true><<<blocks, kSampleThreads, smem, s>>>(a, in_shared);
    else
        profile_kernel<false><<<blocks, kSampleThreads, smem, s>>>(a, in_shared);
    return after_launch();
}

cudaError_t launch_heat_current(const Arena& a, bool shifted_force, uint32_t sample,
                                cudaStream_t s) {
    const unsigned blocks = blocks_for(a.nslots, kSampleThreads);
    if (shifted_force)
        heat_current_kernel<true><<<blocks, kSampleThreads, 0, s>>>(a, sample);
    else
        heat_current_kernel<false><<<blocks, kSampleThreads, 0, s>>>(a, sample);
    return after_launch();
}

}  // namespace vlj
