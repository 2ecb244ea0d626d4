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

#include "virial_lj.h"
#include "vlj_binning.cuh"
#include "vlj_common.h"

namespace vlj {
namespace {

// Per-cell counts, then fill cursors, shared by every call on a device; once
// the particles are scattered, the same words list the cells of more than 32
// particles for the block-wide sort, and the word after the last cell counts
// them.
__device__ __align__(256) uint32_t g_bin_scratch[VLJ_BIN_NOALLOC_MAX_CELLS + 1];

// The device address of the scratch array in the current device's context.
// In host code the array's name is only a stand-in for it. Looked up on every
// call, so an address never outlives the context it belongs to (a device
// reset creates a new one).
vlj_status scratch_address(uint32_t** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_bin_scratch);
    if (e != cudaSuccess) return fail(VLJ_CUDA_ERROR, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    *out = static_cast<uint32_t*>(p);
    return VLJ_OK;
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
    cudaError_t e = vlj::enqueue_binning(pos, g, counts, sorted, cell_start, cell_of,
                                         static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(VLJ_CUDA_ERROR, "bin_noalloc: %s", cudaGetErrorString(e));
    return VLJ_OK;
}
