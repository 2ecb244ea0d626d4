// Verlet list build for sm_100a (lennard_jones.wgsl:454-499).
//
// Each particle's list holds everything within cutoff + skin, in the
// reference's order: the 27 cells dz, dy, dx = -1..1 (periodic wrap), each in
// its sorted order, skipping the particle itself. Acceptance is the
// reference's f32 test on packed positions, operation for operation, so the
// lists are the reference's entry for entry.
//
// A warp serves one home cell at a time: up to 32 home particles, one per
// lane. The grid is resident at once (kBuildBlocksPerSM blocks per SM) and
// its warps take the non-empty cells of the rebuilding boxes from the step's
// work list, so boxes that do not rebuild and empty cells cost nothing. The
// warp reads the 27 neighbour cells' ranges at once (a lane each), which makes
// the cells' candidates one stream in stencil order; it fetches the stream
// kRound candidates at a time (slot, then encoded position, all loads of a
// round in flight together) and copies those within reach of the home cell
// into shared memory (a dense cell's all of them). The test then takes 32
// staged candidates at a time, a lane each, against every home particle in
// turn, so every lane is busy whatever the cell's occupancy; the lanes that
// accept write their candidates into that home particle's list at once (its
// count so far plus their rank in the ballot, so stream order). The inner
// loops read only shared memory, and a dense home cell costs a few rounds of
// two dependent loads.
//
// A test on the 32-bit encoded positions settles every candidate farther than
// sqrt(prefilter_r2) (out) or nearer than sqrt(accept_r2) (in); the two radii
// bracket list_r2 by more than the reference's f32 separations and the encoded
// ones can differ, so only candidates in the thin shell between them need the
// reference's own arithmetic.
#include <cuda_runtime.h>

#include "vlj_device.cuh"
#include "vlj_internal.cuh"

namespace vlj {

// Tuning knobs of the list build (tune.py --kernel build sweeps them): the
// candidates a warp fetches per round, the staged candidates it holds (a
// dense cell's all), and the resident blocks per SM its registers are sized for.
#ifndef VLJ_BUILD_ROUND
#define VLJ_BUILD_ROUND 128
#endif
#ifndef VLJ_BUILD_STAGE
#define VLJ_BUILD_STAGE 512
#endif
#ifndef VLJ_BUILD_BLOCKS_PER_SM
#define VLJ_BUILD_BLOCKS_PER_SM 6
#endif
// 0: the test walks the staged candidates' groups outermost, each against
// every home particle; 1: the home particles outermost, each over all staged
// candidates (more instructions: 147 M against 142 M for the 256k box's full
// build)
#ifndef VLJ_BUILD_ORDER
#define VLJ_BUILD_ORDER 0
#endif
constexpr int kBuildWarps = 4;  // warps per block, each building one home cell at a time
constexpr int kRound = VLJ_BUILD_ROUND;
constexpr int kStage = VLJ_BUILD_STAGE;
// with the cell tiles' 16-bit lists the staged candidates also carry their
// tile indices, so fewer fit beside them
constexpr int kStageTiles = kStage - 64;
constexpr int kBuildBlocksPerSM = VLJ_BUILD_BLOCKS_PER_SM;
static_assert(kRound % 32 == 0 && kStage % 32 == 0 && kRound <= kStage, "build stage shape");

// The reference's packed position of slot s: the f32 hi part of each f64
// coordinate and the f32 lo part of the rest (Df64::from_f64,
// lennard_jones.rs:476-489, lennard_jones.wgsl:154-164).
__device__ __forceinline__ void ref_parts(const Arena& a, uint32_t s, float h[3], float l[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double x = a.x[(size_t)k * a.seg + s];
        h[k] = (float)x;
        l[k] = (float)(x - (double)h[k]);
    }
}

// The reference's predicate for slots i and j: nearest((pj.hi - xh) +
// (unpack(pj) - xl)), squared length < list_r2, in f32 as written
// (lennard_jones.wgsl:482-484), where unpack(pj) is pj's lo part as the
// reference packs it (nine bits of its hi part's last bit). Derives its
// operands from the f64 positions itself: it runs only for candidates in the
// thin shell around the list radius.
__device__ __noinline__ bool ref_test(const Arena& a, const Box& bx, uint32_t i, uint32_t j,
                                      const float* q510) {
    float xh[3], xl[3], ph[3], pl[3];
    ref_parts(a, i, xh, xl);
    ref_parts(a, j, ph, pl);
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float lo = packed_lo(ph[k], pl[k], q510);
        const float e = __fadd_rn(__fsub_rn(ph[k], xh[k]), __fsub_rn(lo, xl[k]));
        d[k] = nearest_ref_fast(e, bx.box_f[k], bx.inv_box_f[k]);
    }
    const float r2 =
        __fadd_rn(__fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1])), __fmul_rn(d[2], d[2]));
    return r2 < bx.list_r2;
}

// A store the predicate guards, without a branch around it.
__device__ __forceinline__ void store_if(bool p, uint32_t* ptr, uint32_t v) {
    asm volatile("{\n .reg .pred q;\n setp.ne.u32 q, %2, 0;\n @q st.global.u32 [%0], %1;\n}"
                 ::"l"(ptr), "r"(v), "r"((uint32_t)p) : "memory");
}

__device__ __forceinline__ void store16_if(bool p, uint16_t* ptr, uint32_t v) {
    asm volatile("{\n .reg .pred q;\n setp.ne.u32 q, %2, 0;\n @q st.global.u16 [%0], %1;\n}"
                 ::"l"(ptr), "h"((unsigned short)v), "r"((uint32_t)p) : "memory");
}

// Whether stencil offset d (-1, 0, 1) along an axis of n cells reaches a cell
// an earlier offset already did: with two cells -1 and +1 are the same
// neighbour, with one cell every offset is the home cell. Boxes of three or
// more cells (all the reference allows) visit all 27 cells.
__device__ __forceinline__ bool repeats(int32_t d, int32_t n) {
    return (n == 2 && d == 1) || (n == 1 && d != 0);
}

// TILES: also write the 16-bit tile lists of the cell-tile step kernel (a
// box with bricks; the instantiation without it carries none of their work).
template <bool TILES>
__global__ void __launch_bounds__(kBuildWarps * 32, kBuildBlocksPerSM) build_list_kernel(Arena a) {
    constexpr int kStage = TILES ? kStageTiles : vlj::kStage;
    count_kernel(a);
    if (!a.glob->any) return;
    // the tile step kernel reads the 16-bit lists from the next step on
    if (TILES && blockIdx.x == 0 && threadIdx.x == 0) a.glob->tiles_ready = 1u;
    __shared__ float s_q510[512];  // q / 510 for q = -256..255, IEEE quotients
    // staged candidates: (x, y, z) as f32 offsets from the home cell's centre
    // (wide boxes) or as encoded words (narrow ones), the slot in w
    __shared__ uint4 s_cand[kBuildWarps][kStage];
    // with cell tiles: each staged candidate's index in the brick's tile
    __shared__ uint16_t s_tix[kBuildWarps][TILES ? kStage : 1];
    __shared__ uint4 s_home[kBuildWarps][32];
    for (int t = threadIdx.x; t < 512; t += blockDim.x)
        s_q510[t] = __fdiv_rn((float)(t - 256), 510.0f);
    __syncthreads();
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    // Warps take home cells (or, in narrow boxes, parts of their home
    // particles) from the step's work list (the non-empty cells of the boxes
    // that rebuild) until it runs out.
    const uint32_t cells = work_total(a), front = a.glob->work_front;
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&a.glob->next_build, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= cells) break;
        const uint32_t entry = work_item(a, front, t);
        const uint32_t cell = entry >> 3, part = entry & 7u;
        const uint32_t b = box_of_cell(a, cell);
        const Box& bx = a.boxes[b];
        // this entry's home particles: the whole cell, or part `part` of it
        // (kPartHomes each, the last part the rest)
        const uint32_t cs0 = a.cell_start[cell], cs1 = a.cell_start[cell + 1];
        const uint32_t parts = cell_parts(cs1 - cs0, narrow_box(bx));
        const uint32_t hbeg = parts > 1u ? cs0 + part * kPartHomes : cs0;
        const uint32_t hend = parts > 1u && part + 1u < parts ? hbeg + kPartHomes : cs1;
        const uint4* __restrict__ cur = a.cache[a.glob->phase];
        const float dec[3] = {bx.dec[0], bx.dec[1], bx.dec[2]};
        const int32_t n[3] = {(int32_t)bx.cells[0], (int32_t)bx.cells[1], (int32_t)bx.cells[2]};
        const int32_t ci = (int32_t)(cell - bx.cell_base);
        const int32_t c[3] = {ci % n[0], (ci / n[0]) % n[1], ci / (n[0] * n[1])};
        const uint32_t cap = bx.capacity;
        const float pre_r2 = bx.prefilter_r2, acc_r2 = bx.accept_r2;

        // Lane s < 27 takes stencil cell s = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1),
        // so lane order is the reference's order; its candidates are
        // sorted[cs, cs + cnt), at offset off in the stream of all of them.
        uint32_t cs = 0, cnt = 0;
        if (lane < 27u) {
            const int32_t d[3] = {(int32_t)(lane % 3u) - 1, (int32_t)((lane / 3u) % 3u) - 1,
                                  (int32_t)(lane / 9u) - 1};
            if (!repeats(d[0], n[0]) && !repeats(d[1], n[1]) && !repeats(d[2], n[2])) {
                int32_t u[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    u[k] = c[k] + d[k];
                    u[k] = u[k] < 0 ? u[k] + n[k] : (u[k] >= n[k] ? u[k] - n[k] : u[k]);
                }
                const uint32_t nc = bx.cell_base +
                    ((uint32_t)u[2] * (uint32_t)n[1] + (uint32_t)u[1]) * (uint32_t)n[0] + (uint32_t)u[0];
                cs = a.cell_start[nc];
                cnt = a.cell_start[nc + 1] - cs;
            }
        }
        uint32_t off = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, off, o);
            if (lane >= (uint32_t)o) off += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, off, 31);
        off -= cnt;  // exclusive; lanes 27..31 sit at `total`

        // With cell tiles: lane s's stencil cell's first particle's index in
        // the tile of the home cell's brick (tile_step_kernel stages the same
        // tile), and the home cell's own (stencil lane 13).
        const bool tiles = TILES && bx.brick_cols != 0u;
        uint32_t tbase = 0;
        if (tiles) {
            const Brick k = make_brick(bx, brick_col_of(bx, (uint32_t)c[0]), (uint32_t)c[1],
                                       (uint32_t)c[2]);
            uint32_t rowc = lane < 9u ? tile_row_prefix(a.cell_start, bx, k,
                                                        tile_row_cell(bx, k, lane), k.rx)
                                      : 0u;
            uint32_t incl = rowc;
#pragma unroll
            for (int o = 1; o < 16; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += t;
            }
            // lane s = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1) lies in tile row s / 3
            const uint32_t row_base = __shfl_sync(0xffffffffu, incl - rowc, min(lane / 3u, 8u));
            if (lane < 27u) {
                const uint32_t rho = lane / 3u;
                tbase = row_base + tile_row_prefix(a.cell_start, bx, k, tile_row_cell(bx, k, rho),
                                                   tile_col(bx, k, (uint32_t)c[0],
                                                            (int32_t)(lane % 3u) - 1));
            }
        }
        const uint32_t home_tix0 = __shfl_sync(0xffffffffu, tbase, 13) - cs0;
        const uint32_t row16_stride = a.seg * 8u;  // entries between a position's rows

        // The home cell as an interval of encoded coordinates per axis, for the
        // staging filter: a candidate farther than reach_r2 from the whole home
        // cell cannot be in any home particle's list.
        uint32_t home_lo[3], home_w[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            home_lo[k] = (uint32_t)(unsigned long long)__double2ll_rn((double)c[k] * (double)bx.cell_size_f[k] * bx.enc[k]);
            home_w[k] = (uint32_t)(unsigned long long)__double2ll_rn((double)bx.cell_size_f[k] * bx.enc[k]);
        }
        const float reach_r2 = bx.reach_r2;
        // In a box at least five cells wide on every axis, a home particle and
        // a candidate within reach lie less than 0.3 of a side from the home
        // cell's centre, so the plain difference of their f32 offsets from it
        // is the nearest image, within 1e-6 of the exact separation -- far
        // inside the accept / prefilter margins. Narrower boxes (batched
        // replicas) test on the encoded words, which wrap to the nearest image.
        const bool wide = n[0] >= 5 && n[1] >= 5 && n[2] >= 5;
        uint32_t mid[3];
#pragma unroll
        for (int k = 0; k < 3; k++) mid[k] = home_lo[k] + home_w[k] / 2u;
        const uint32_t row_stride = a.seg * 4u;  // entries between a slot's rows
        const unsigned below = (1u << lane) - 1u;
        for (uint32_t h0 = hbeg; h0 < hend; h0 += 32) {
            const bool home = h0 + lane < hend;
            const uint32_t i = home ? a.sorted[h0 + lane] : 0u;
            const uint4 own_enc = home ? cur[i] : make_uint4(0u, 0u, 0u, 0u);
            // offsets from the home cell's centre (wide boxes); a lane with no
            // home particle sits far away and accepts nothing
            float own_rel[3] = {3.0e18f, 3.0e18f, 3.0e18f};
            if (home) {
                own_rel[0] = (float)(int32_t)(own_enc.x - mid[0]) * dec[0];
                own_rel[1] = (float)(int32_t)(own_enc.y - mid[1]) * dec[1];
                own_rel[2] = (float)(int32_t)(own_enc.z - mid[2]) * dec[2];
            }
            // this lane's home particle's list length so far (every accepted
            // candidate, also those past the capacity)
            uint32_t found = 0;
            const uint32_t homes = min(hend - h0, 32u);
            uint32_t staged = 0;
            // the home particles, for broadcast reads: f32 offsets from the
            // cell's centre (wide boxes) or encoded words, slot in w
            s_home[warp][lane] = wide ? make_uint4(__float_as_uint(own_rel[0]),
                                                   __float_as_uint(own_rel[1]),
                                                   __float_as_uint(own_rel[2]), i)
                                      : make_uint4(own_enc.x, own_enc.y, own_enc.z, i);
            __syncwarp();
            for (uint32_t base = 0; base < total; base += kRound) {
                // Fetch the next kRound candidates of the stream (kRound / 32 per
                // lane, loads in flight together), keep those within reach of the
                // home cell, and stage them in stream order.
                uint32_t j[kRound / 32], tix[kRound / 32];
#pragma unroll
                for (int r = 0; r < kRound / 32; r++) {
                    const uint32_t t = base + (uint32_t)r * 32u + lane;
                    // the last stencil lane whose stream offset is <= t (all
                    // lanes search, past-the-end ones for the last candidate)
                    const uint32_t tt = t < total ? t : total - 1u;
                    uint32_t lo = 0, hi = 32;
#pragma unroll
                    for (int q = 0; q < 5; q++) {
                        const uint32_t m = (lo + hi) >> 1;
                        if (__shfl_sync(0xffffffffu, off, m) <= tt) lo = m; else hi = m;
                    }
                    const uint32_t from = __shfl_sync(0xffffffffu, cs, lo);
                    const uint32_t at = __shfl_sync(0xffffffffu, off, lo);
                    j[r] = t < total ? a.sorted[from + t - at] : 0xffffffffu;
                    // (tiles is the same for the whole warp)
                    if (tiles) tix[r] = __shfl_sync(0xffffffffu, tbase, lo) + t - at;
                }
                uint4 pe[kRound / 32];
#pragma unroll
                for (int r = 0; r < kRound / 32; r++)
                    pe[r] = j[r] != 0xffffffffu ? __ldg(cur + j[r]) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                for (int r = 0; r < kRound / 32; r++) {
                    bool keep = false;
                    if (j[r] != 0xffffffffu) {
                        float g2 = 0.0f;
#pragma unroll
                        for (int k = 0; k < 3; k++) {
                            // periodic gap between the candidate and the interval
                            // [lo, lo + w): above it, or below it around the box,
                            // whichever is shorter
                            const uint32_t w = k == 0 ? pe[r].x : (k == 1 ? pe[r].y : pe[r].z);
                            const uint32_t o = w - home_lo[k];
                            const uint32_t gap = o < home_w[k] ? 0u : min(o - home_w[k], 0u - o);
                            const float g = (float)gap * dec[k];
                            g2 += g * g;
                        }
                        keep = g2 < reach_r2;
                    }
                    const unsigned kept_mask = __ballot_sync(0xffffffffu, keep);
                    if (keep) {
                        const uint32_t to = staged + (uint32_t)__popc(kept_mask & below);
                        if (wide)
                            s_cand[warp][to] = make_uint4(
                                __float_as_uint((float)(int32_t)(pe[r].x - mid[0]) * dec[0]),
                                __float_as_uint((float)(int32_t)(pe[r].y - mid[1]) * dec[1]),
                                __float_as_uint((float)(int32_t)(pe[r].z - mid[2]) * dec[2]), j[r]);
                        else
                            s_cand[warp][to] = make_uint4(pe[r].x, pe[r].y, pe[r].z, j[r]);
                        if (tiles) s_tix[warp][to] = (uint16_t)tix[r];
                    }
                    staged += (uint32_t)__popc(kept_mask);
                }
                // test once the stream is done or the stage has no room for
                // another round
                if (base + kRound < total && staged + kRound <= (uint32_t)kStage) continue;
                __syncwarp();
                // Test: every home particle in turn against the staged
                // candidates, 32 at a time, a lane each. The lanes that
                // accept write their candidates into that home particle's
                // list themselves, in stream order (its count so far plus
                // their rank in the ballot), so every lane is busy whatever
                // the cell's occupancy and however unevenly the homes
                // accept. Candidates in the thin shell between the two radii
                // take the reference's test.
#if VLJ_BUILD_ORDER == 0
                // The candidates' group is the outer loop, the homes' counts
                // in their lanes; one loop for each form of the separation.
                auto test_groups = [&](auto r2_of) {
                    for (uint32_t c0 = 0; c0 < staged; c0 += 32) {
                        const uint32_t q = c0 + lane;
                        const bool valid = q < staged;
                        const uint4 e = s_cand[warp][valid ? q : 0u];
                        const uint32_t e_tix = tiles ? s_tix[warp][valid ? q : 0u] : 0u;
                        for (uint32_t h = 0; h < homes; h++) {
                            const uint4 hp = s_home[warp][h];
                            const float r2e = r2_of(e, hp);
                            const bool near = valid && r2e < pre_r2 && e.w != hp.w;
                            bool take = near && r2e < acc_r2;
                            if (near && !take) take = ref_test(a, bx, hp.w, e.w, s_q510);
                            const unsigned m = __ballot_sync(0xffffffffu, take);
                            if (m == 0u) continue;
                            // entry k of the home particle's list: row k / 4, place k % 4
                            const uint32_t k = __shfl_sync(0xffffffffu, found, h) +
                                               (uint32_t)__popc(m & below);
                            store_if(take && k < cap,
                                     a.list + ((unsigned long long)(k >> 2) * row_stride +
                                               (hp.w * 4u + (k & 3u))),
                                     e.w);
                            // entry k of the 16-bit list of the home's sorted
                            // position h0 + h: row k / 8, place k % 8
                            if (tiles)
                                store16_if(take && k < cap,
                                           a.list16 + ((unsigned long long)(k >> 3) * row16_stride +
                                                       ((h0 + h) * 8u + (k & 7u))),
                                           e_tix);
                            if (lane == h) found += (uint32_t)__popc(m);
                        }
                    }
                };
                if (wide)
                    test_groups([](const uint4& e, const uint4& hp) {
                        const float dx = __uint_as_float(e.x) - __uint_as_float(hp.x);
                        const float dy = __uint_as_float(e.y) - __uint_as_float(hp.y);
                        const float dz = __uint_as_float(e.z) - __uint_as_float(hp.z);
                        return dx * dx + dy * dy + dz * dz;
                    });
                else
                    test_groups([&](const uint4& e, const uint4& hp) { return encoded_r2(e, hp, dec); });
#else
                // The home is the outer loop: its position and its count so
                // far sit in warp-uniform registers for all its groups.
                auto test_homes = [&](auto r2_of) {
                    for (uint32_t h = 0; h < homes; h++) {
                        const uint4 hp = s_home[warp][h];
                        uint32_t fh = __shfl_sync(0xffffffffu, found, h);
                        uint32_t* const row0 = a.list + (size_t)hp.w * 4u;
                        uint16_t* const row16 = tiles ? a.list16 + (size_t)(h0 + h) * 8u : nullptr;
                        for (uint32_t c0 = 0; c0 < staged; c0 += 32) {
                            const uint32_t q = c0 + lane;
                            const bool valid = q < staged;
                            const uint4 e = s_cand[warp][valid ? q : 0u];
                            const float r2e = r2_of(e, hp);
                            const bool near = valid && r2e < pre_r2 && e.w != hp.w;
                            bool take = near && r2e < acc_r2;
                            if (near && !take) take = ref_test(a, bx, hp.w, e.w, s_q510);
                            const unsigned m = __ballot_sync(0xffffffffu, take);
                            // (most groups of a home on the far side of the
                            // stencil take nothing)
                            if (m == 0u) continue;
                            // entry k of the home particle's list: row k / 4, place k % 4
                            const uint32_t k = fh + (uint32_t)__popc(m & below);
                            store_if(take && k < cap, row0 + ((size_t)(k >> 2) * row_stride + (k & 3u)),
                                     e.w);
                            // entry k of the 16-bit list of the home's sorted
                            // position h0 + h: row k / 8, place k % 8
                            if (tiles)
                                store16_if(take && k < cap,
                                           row16 + ((size_t)(k >> 3) * row16_stride + (k & 7u)),
                                           s_tix[warp][valid ? q : 0u]);
                            fh += (uint32_t)__popc(m);
                        }
                        if (lane == h) found = fh;
                    }
                };
                if (wide)
                    test_homes([&](const uint4& e, const uint4& hp) {
                        const float dx = __uint_as_float(e.x) - __uint_as_float(hp.x);
                        const float dy = __uint_as_float(e.y) - __uint_as_float(hp.y);
                        const float dz = __uint_as_float(e.z) - __uint_as_float(hp.z);
                        return dx * dx + dy * dy + dz * dz;
                    });
                else
                    test_homes([&](const uint4& e, const uint4& hp) { return encoded_r2(e, hp, dec); });
#endif
                __syncwarp();
                staged = 0;
            }
            const uint32_t kept = found < cap ? found : cap;
            if (home) {
                // the last row's unused places hold the particle itself: a zero
                // separation, which the force kernels skip, so they read whole
                // rows without a per-entry count test
                uint32_t* row_of_i = a.list + (size_t)i * 4u;
                for (uint32_t k = kept; k & 3u; k++)
                    row_of_i[(size_t)(k >> 2) * row_stride + (k & 3u)] = i;
                if (tiles) {
                    // the home's own tile index: a zero separation, skipped
                    uint16_t* row16 = a.list16 + (size_t)(h0 + lane) * 8u;
                    const uint16_t own_tix = (uint16_t)(home_tix0 + h0 + lane);
                    for (uint32_t k = kept; k & 7u; k++)
                        row16[(size_t)(k >> 3) * row16_stride + (k & 7u)] = own_tix;
                }
                a.list_count[i] = kept;
                if (found > cap) atomicMax(&a.ctrl[b].overflow, found);
                a.snap[i] = own_enc;
            }
#if !VLJ_LIST_STREAM
            // rows each force block stages in its TMA tiles: one atomic per
            // block these lanes touch (a cell's slots are mostly in one block
            // after a reorder)
            const uint32_t blk = home ? i / (uint32_t)kForceThreads : 0xffffffffu;
            const unsigned peers = __match_any_sync(0xffffffffu, blk);
            const uint32_t rows = __reduce_max_sync(peers, home ? (kept + 3u) / 4u : 0u);
            if (home && lane == (uint32_t)(__ffs(peers) - 1)) atomicMax(&a.block_rows[blk], rows);
#endif
        }
    }
}

cudaError_t launch_build_list(const Arena& a, cudaStream_t s) {
    const unsigned blocks = (unsigned)sm_count() * kBuildBlocksPerSM;
    if (a.list16)
        build_list_kernel<true><<<blocks, kBuildWarps * 32, 0, s>>>(a);
    else
        build_list_kernel<false><<<blocks, kBuildWarps * 32, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace vlj
