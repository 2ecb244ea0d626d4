// Cell binning that allocates no device memory: vlj_bin_noalloc.
//
// Some programs that would like this library's binning cannot let it
// allocate: an embedding framework that owns all device memory through its
// own pool and forbids libraries from calling cudaMalloc behind its back, or
// a latency-critical loop in which cudaMalloc / cudaFree would synchronise the
// whole device and stall every other stream. This entry point serves them.
// The caller passes the inputs and every output buffer; the only scratch --
// one counter per cell -- lives in the fixed device array below, which every
// GPU that loads the library holds until the process exits.
//
// The binning is the reference's (grid.wgsl:11-148): cell = clamp(floor(f32(x)
// / cell size), 0, cells - 1) per axis, cell index (z * ny + y) * nx + x, then
// a stable counting sort, so each cell lists its particles in index order.
#include <cuda_runtime.h>

#include <mutex>

#include "virial_lj.h"
#include "vlj_common.h"

namespace vlj {
namespace {

// Per-cell counts, then fill cursors, shared by every call on a device.
__device__ __align__(256) uint32_t g_bin_scratch[VLJ_BIN_NOALLOC_MAX_CELLS];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
uint32_t* g_scratch[kMaxDevices] = {};

struct BinGrid {
    float cell_size[3];
    uint32_t cells[3];
    uint32_t total;
    uint32_t n;
};

// The device address of the scratch array on the current device, looked up
// once per device (in host code the array's name is not a device address).
vlj_status scratch_address(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(VLJ_CUDA_ERROR, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(VLJ_INVALID_ARG, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_bin_scratch);
        if (e != cudaSuccess)
            return fail(VLJ_CUDA_ERROR, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_scratch[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch[dev];
    return VLJ_OK;
}

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
    if (threadIdx.x == 0) cell_start[g.total] = g.n;
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
__global__ void nb_order(BinGrid g, const uint32_t* __restrict__ cell_start,
                         uint32_t* __restrict__ sorted) {
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
        for (uint32_t s = start + 1; s < end; s++) {
            const uint32_t key = sorted[s];
            uint32_t t = s;
            while (t > start && sorted[t - 1] > key) {
                sorted[t] = sorted[t - 1];
                t -= 1;
            }
            sorted[t] = key;
        }
    }
}

}  // namespace
}  // namespace vlj

using vlj::fail;

extern "C" vlj_status vlj_bin_noalloc(const double* pos, size_t count, const double box_size[3],
                                      const uint32_t cells[3], uint32_t* sorted,
                                      uint32_t* cell_start, uint32_t* cell_of, void* stream) {
    if (!pos || !box_size || !cells || !sorted || !cell_start || !cell_of)
        return fail(VLJ_INVALID_ARG, "bin_noalloc: null argument");
    if (count == 0 || count >= (1ull << 31))
        return fail(VLJ_INVALID_ARG, "bin_noalloc: count must be in 1 .. 2^31 - 1");
    vlj::BinGrid g;
    uint64_t total = 1;
    for (int k = 0; k < 3; k++) {
        if (!(box_size[k] > 0.0) || !(box_size[k] < 1e30))
            return fail(VLJ_INVALID_ARG, "bin_noalloc: box side %d must be positive and finite", k);
        if (cells[k] == 0) return fail(VLJ_INVALID_ARG, "bin_noalloc: cells[%d] is zero", k);
        g.cells[k] = cells[k];
        // box rounded to f32 first, as LennardJones::new does (lennard_jones.rs:450)
        g.cell_size[k] = (float)((double)(float)box_size[k] / (double)cells[k]);
        total *= cells[k];
    }
    if (total > VLJ_BIN_NOALLOC_MAX_CELLS)
        return fail(VLJ_INVALID_ARG, "bin_noalloc: %llu cells exceed the maximum of %u",
                    (unsigned long long)total, (unsigned)VLJ_BIN_NOALLOC_MAX_CELLS);
    g.total = (uint32_t)total;
    g.n = (uint32_t)count;
    uint32_t* counts = nullptr;
    vlj_status st = vlj::scratch_address(&counts);
    if (st != VLJ_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the scratch keeps the previous call's cursors: counts start at zero
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(uint32_t) * g.total, s);
    if (e == cudaSuccess) {
        const unsigned blocks = (g.n + 255u) / 256u;
        vlj::nb_bin<<<blocks, 256, 0, s>>>(pos, g, cell_of, counts);
        vlj::nb_scan<<<1, 1024, 0, s>>>(g, counts, cell_start);
        vlj::nb_scatter<<<blocks, 256, 0, s>>>(g, cell_of, cell_start, counts, sorted);
        vlj::nb_order<<<(unsigned)(((uint64_t)g.total * 32u + 255u) / 256u), 256, 0, s>>>(
            g, cell_start, sorted);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return fail(VLJ_CUDA_ERROR, "bin_noalloc: %s", cudaGetErrorString(e));
    return VLJ_OK;
}
