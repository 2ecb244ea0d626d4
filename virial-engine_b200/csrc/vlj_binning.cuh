// The cell grid as a stand-alone pipeline on caller-owned buffers: the
// reference's binning and stable per-cell order (grid.wgsl:11-148) for any
// particle kind. Used by the binning that allocates nothing
// (vlj_noalloc.cu) and by the granular contact finder (vlj_grains.cu); each
// includes its own copy of these kernels.
//
// Positions are count x 3 doubles (row-major); a particle's cell is
// clamp(floor(f32(x) / cell size), 0, cells - 1) per axis, index
// (z * ny + y) * nx + x; `counts` is total + 1 words of scratch (per-cell
// counters, then the list of cells over 32 particles and, in its last word,
// their number).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vlj {
namespace {

constexpr uint32_t kSharedSort = 8192;  // a crowded cell sorted in shared memory up to this size
constexpr int kSortThreads = 1024;
constexpr unsigned kLargeBlocks = 296;  // blocks that take the crowded cells in turn

struct BinGrid {
    float cell_size[3];
    uint32_t cells[3];
    uint32_t total;
    uint32_t n;
};

__global__ void nb_bin(const double* __restrict__ pos, BinGrid g, uint32_t* __restrict__ cell_of,
                       uint32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    int32_t c[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float hi = (float)pos[3 * (size_t)i + k];
        const int32_t v = (int32_t)floorf(__fdiv_rn(hi, g.cell_size[k]));
        const int32_t m = (int32_t)g.cells[k] - 1;
        c[k] = v < 0 ? 0 : (v > m ? m : v);
    }
    const uint32_t cell = ((uint32_t)c[2] * g.cells[1] + (uint32_t)c[1]) * g.cells[0] + (uint32_t)c[0];
    cell_of[i] = cell;
    atomicAdd(&counts[cell], 1u);
}

// One block: exclusive prefix sum of the counts into cell_start; the counts
// become zeroed fill cursors.
__global__ void __launch_bounds__(1024) nb_scan(BinGrid g, uint32_t* __restrict__ counts,
                                                uint32_t* __restrict__ cell_start) {
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < g.total; base += 1024u) {
        const uint32_t c = base + threadIdx.x;
        const uint32_t v = c < g.total ? counts[c] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = s_warp[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += t;
            }
            s_warp[lane] = w;
        }
        __syncthreads();
        if (c < g.total) {
            cell_start[c] = s_carry + (warp ? s_warp[warp - 1] : 0u) + incl - v;
            counts[c] = 0u;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry += s_warp[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        cell_start[g.total] = g.n;
        counts[g.total] = 0u;  // no crowded cell listed yet
    }
}

__global__ void nb_scatter(BinGrid g, const uint32_t* __restrict__ cell_of,
                           const uint32_t* __restrict__ cell_start, uint32_t* __restrict__ counts,
                           uint32_t* __restrict__ sorted) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const uint32_t c = cell_of[i];
    sorted[cell_start[c] + atomicAdd(&counts[c], 1u)] = i;
}

// One warp per cell: each index's rank is the number of smaller indices in
// the cell, which undoes whatever order the scatter's atomics produced.
// Cells of more than 32 particles are listed (in the scratch words the
// counts no longer need) for nb_order_large.
__global__ void nb_order(BinGrid g, const uint32_t* __restrict__ cell_start,
                         uint32_t* __restrict__ sorted, uint32_t* __restrict__ large, uint32_t large_at) {
    const uint32_t cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (cell >= g.total) return;
    const uint32_t start = cell_start[cell], end = cell_start[cell + 1];
    const uint32_t m = end - start;
    if (m <= 32u) {
        const uint32_t key = lane < m ? sorted[start + lane] : 0xffffffffu;
        uint32_t rank = 0;
        for (uint32_t src = 0; src < m; src++)
            rank += __shfl_sync(0xffffffffu, key, (int)src) < key ? 1u : 0u;
        __syncwarp();
        if (lane < m) sorted[start + rank] = key;
    } else if (lane == 0) {
        large[atomicAdd(&large[large_at], 1u)] = cell;
    }
}

// Bitonic sorting network on a[0, m) as the first m of 2^p places, the rest
// read as +infinity: every comparator puts the smaller value first (the
// first stage of each merge compares mirror images, i with i ^ (k - 1)), so
// the padding never moves and comparators that reach it are skipped.
// O(m log^2 m) work over the block's threads; the values are distinct.
__device__ void block_bitonic(uint32_t* a, uint32_t m) {
    uint64_t size = 1;  // up to 2^31: 64-bit, so the doubling below ends
    while (size < m) size <<= 1;
    for (uint64_t k = 2; k <= size; k <<= 1) {
        for (uint64_t j = k >> 1; j > 0; j >>= 1) {
            for (uint64_t i = threadIdx.x; i < size; i += blockDim.x) {
                const uint64_t l = j == (k >> 1) ? (i ^ (k - 1u)) : (i ^ j);
                if (l > i && l < m) {
                    const uint32_t x = a[i], y = a[l];
                    if (y < x) {
                        a[i] = y;
                        a[l] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// The listed cells of more than 32 particles, one block each at a time:
// sorted in shared memory up to kSharedSort particles, in place in global
// memory beyond that.
__global__ void __launch_bounds__(kSortThreads) nb_order_large(const uint32_t* __restrict__ cell_start,
                                                               uint32_t* __restrict__ sorted,
                                                               const uint32_t* __restrict__ large, uint32_t large_at) {
    __shared__ uint32_t s_keys[kSharedSort];
    const uint32_t listed = large[large_at];
    for (uint32_t t = blockIdx.x; t < listed; t += gridDim.x) {
        const uint32_t cell = large[t];
        const uint32_t start = cell_start[cell], m = cell_start[cell + 1] - start;
        if (m <= kSharedSort) {
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) s_keys[i] = sorted[start + i];
            __syncthreads();
            block_bitonic(s_keys, m);
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) sorted[start + i] = s_keys[i];
        } else {
            block_bitonic(sorted + start, m);
        }
        __syncthreads();
    }
}

// Enqueues the whole pipeline; `counts` needs g.total + 1 words.
inline cudaError_t enqueue_binning(const double* pos, const BinGrid& g, uint32_t* counts,
                                   uint32_t* sorted, uint32_t* cell_start, uint32_t* cell_of,
                                   cudaStream_t s) {
    // the scratch keeps the previous call's cursors: counts start at zero
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(uint32_t) * g.total, s);
    if (e != cudaSuccess) return e;
    const unsigned blocks = (g.n + 255u) / 256u;
    nb_bin<<<blocks, 256, 0, s>>>(pos, g, cell_of, counts);
    nb_scan<<<1, 1024, 0, s>>>(g, counts, cell_start);
    nb_scatter<<<blocks, 256, 0, s>>>(g, cell_of, cell_start, counts, sorted);
    nb_order<<<(unsigned)(((uint64_t)g.total * 32u + 255u) / 256u), 256, 0, s>>>(
        g, cell_start, sorted, counts, g.total);
    nb_order_large<<<kLargeBlocks, kSortThreads, 0, s>>>(cell_start, sorted, counts, g.total);
    return cudaGetLastError();
}

}  // namespace
}  // namespace vlj
