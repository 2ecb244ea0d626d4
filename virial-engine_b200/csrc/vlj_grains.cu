// Contacts of granular spheres found through the cell grid:
// vlj_grain_cells, vlj_grain_contacts.
//
// The reference's granular solver includes the same grid as the
// Lennard-Jones one (granular.rs:327-328 appends grid.wgsl to granular.wgsl):
// it bins the grains into cells of at least one diameter, sorts each cell by
// grain index, and every grain visits the 27 cells around its own (not
// periodic: cells past a wall are skipped) in the order dz, dy, dx = -1..1,
// each in its sorted order, keeping the grains whose spheres overlap its own
// (granular.wgsl:204-263). Here that search runs on the library's grid
// pipeline (vlj_binning.cuh) and writes each grain's partners in that order,
// the table the reference's contact springs are indexed by.
//
// Arithmetic as the reference's: positions as double-float (hi = f32(x), lo
// = f32(x - hi)), d = (x_i.hi - x_j.hi) + (x_i.lo - x_j.lo) per axis in f32,
// dist2 = dot(d, d), reach = r_i + r_j (f32 radii), dist = sqrt(dist2), and a
// contact when reach - dist > 0 and dist2 > 0, each operation rounded as
// written (no contraction).
#include <cuda_runtime.h>

#include <cmath>

#include "virial_lj.h"
#include "vlj_binning.cuh"
#include "vlj_common.h"

namespace vlj {
namespace {

struct GrainGrid {
    uint32_t n;        // grains
    uint32_t cells;    // cells per axis
    uint32_t capacity; // partners kept per grain
};

__device__ __forceinline__ void df_parts(const double* pos, uint32_t i, float h[3], float l[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double x = pos[3 * (size_t)i + k];
        h[k] = (float)x;
        l[k] = (float)(x - (double)h[k]);
    }
}

// One grain per thread: the 27 cells around its own (dz, dy, dx), each in
// sorted order, partners in that order; counts[i] is the number of
// contacts (also those past the capacity, which are not written).
__global__ void grain_contacts_kernel(const double* __restrict__ pos,
                                      const double* __restrict__ radius, GrainGrid g,
                                      const uint32_t* __restrict__ sorted,
                                      const uint32_t* __restrict__ cell_start,
                                      const uint32_t* __restrict__ cell_of,
                                      uint32_t* __restrict__ partners,
                                      uint32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    float xh[3], xl[3];
    df_parts(pos, i, xh, xl);
    const float r = (float)radius[i];
    const int32_t n = (int32_t)g.cells;
    const uint32_t c = cell_of[i];
    const int32_t cc[3] = {(int32_t)(c % g.cells), (int32_t)((c / g.cells) % g.cells),
                           (int32_t)(c / (g.cells * g.cells))};
    uint32_t found = 0;
    for (int32_t dz = -1; dz <= 1; dz++)
        for (int32_t dy = -1; dy <= 1; dy++)
            for (int32_t dx = -1; dx <= 1; dx++) {
                const int32_t nc[3] = {cc[0] + dx, cc[1] + dy, cc[2] + dz};
                if (nc[0] < 0 || nc[1] < 0 || nc[2] < 0 || nc[0] >= n || nc[1] >= n || nc[2] >= n)
                    continue;
                const uint32_t cell = ((uint32_t)nc[2] * g.cells + (uint32_t)nc[1]) * g.cells +
                                      (uint32_t)nc[0];
                for (uint32_t t = cell_start[cell]; t < cell_start[cell + 1]; t++) {
                    const uint32_t j = sorted[t];
                    if (j == i) continue;
                    float ph[3], pl[3];
                    df_parts(pos, j, ph, pl);
                    float d[3];
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        d[k] = __fadd_rn(__fsub_rn(xh[k], ph[k]), __fsub_rn(xl[k], pl[k]));
                    const float dist2 = __fadd_rn(__fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1])),
                                                  __fmul_rn(d[2], d[2]));
                    const float reach = __fadd_rn(r, (float)radius[j]);
                    const float dist = __fsqrt_rn(dist2);
                    if (__fsub_rn(reach, dist) > 0.0f && dist2 > 0.0f) {
                        if (found < g.capacity) partners[(size_t)i * g.capacity + found] = j;
                        found += 1u;
                    }
                }
            }
    counts[i] = found;
}

}  // namespace
}  // namespace vlj

using vlj::fail;

extern "C" {

vlj_status vlj_grain_cells(double box_size, double max_radius, uint32_t* cells) {
    if (!cells) return fail(VLJ_INVALID_ARG, "grain_cells: null argument");
    if (!(box_size > 0.0) || !(box_size < 1e30) || !(max_radius > 0.0) || !(max_radius < 1e30))
        return fail(VLJ_INVALID_ARG, "grain_cells: box size and radius must be positive and finite");
    // granular.rs:179-181
    const double c = std::floor(box_size / (2.0 * max_radius));
    *cells = c < 1.0 ? 1u : (c > 64.0 ? 64u : (uint32_t)c);
    return VLJ_OK;
}

vlj_status vlj_grain_contacts(const double* pos, const double* radius, size_t count,
                              double box_size, uint32_t cells, uint32_t capacity,
                              uint32_t* scratch, uint32_t* sorted, uint32_t* cell_start,
                              uint32_t* cell_of, uint32_t* partners, uint32_t* counts,
                              void* stream) {
    if (!pos || !radius || !scratch || !sorted || !cell_start || !cell_of || !counts ||
        (!partners && capacity))
        return fail(VLJ_INVALID_ARG, "grain_contacts: null argument");
    if (count == 0 || count >= (1ull << 31))
        return fail(VLJ_INVALID_ARG, "grain_contacts: count must be in 1 .. 2^31 - 1");
    if (!(box_size > 0.0) || !(box_size < 1e30))
        return fail(VLJ_INVALID_ARG, "grain_contacts: box size must be positive and finite");
    if (cells == 0 || cells > 64)
        return fail(VLJ_INVALID_ARG, "grain_contacts: cells per axis must be in 1 .. 64");
    if ((uint64_t)count * capacity >= (1ull << 40))
        return fail(VLJ_INVALID_ARG, "grain_contacts: partner table too large");
    vlj::BinGrid g;
    for (int k = 0; k < 3; k++) {
        g.cells[k] = cells;
        // granular.rs:182: the cell side in f64, then f32 as the shader gets it
        g.cell_size[k] = (float)(box_size / (double)cells);
    }
    g.total = cells * cells * cells;
    g.n = (uint32_t)count;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = vlj::enqueue_binning(pos, g, scratch, sorted, cell_start, cell_of, s);
    if (e == cudaSuccess) {
        const vlj::GrainGrid gg{g.n, cells, capacity};
        vlj::grain_contacts_kernel<<<(g.n + 127u) / 128u, 128, 0, s>>>(
            pos, radius, gg, sorted, cell_start, cell_of, partners, counts);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return fail(VLJ_CUDA_ERROR, "grain_contacts: %s", cudaGetErrorString(e));
    return VLJ_OK;
}

}  // extern "C"
