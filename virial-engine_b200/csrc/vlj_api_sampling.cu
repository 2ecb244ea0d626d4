// C ABI of the profiles along z and the heat-current series
// (crates/virial-particles/src/lennard_jones.rs:954-1012, 1165-1191, 1286-1325).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "virial_lj.h"
#include "vlj_common.h"
#include "vlj_internal.cuh"
#include "vlj_sim.h"

using namespace vlj;

#define CUDA_TRY(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(VLJ_CUDA_ERROR, "%s: %s", #call, cudaGetErrorString(e_));        \
    } while (0)

#define TRY(expr)                    \
    do {                             \
        vlj_status s_ = (expr);      \
        if (s_ != VLJ_OK) return s_; \
    } while (0)

namespace {

constexpr double kOne = 4294967296.0;  // one unit of 32.32 fixed point

vlj_status need_profile(const vlj_sim* s) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (!s->box.profile_bins || !s->arena.profile)
        return fail(VLJ_NOT_ENABLED, "profiles need Settings::profile_bins above zero");
    return VLJ_OK;
}

}  // namespace

extern "C" {

// lennard_jones.rs:1165-1183: one sample added to the running sums
vlj_status vlj_sample_profile(vlj_sim* s) {
    TRY(need_profile(s));
    TRY(sim_lists_now(s));
    CUDA_TRY(launch_profile(s->arena, s->box.profile_bins, s->shifted_force, s->stream));
    s->profile_samples += 1;
    return VLJ_OK;
}

// lennard_jones.rs:1185-1191 (no profiles: nothing to clear)
vlj_status vlj_clear_profile(vlj_sim* s) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (!s->arena.profile) return VLJ_OK;
    const size_t words = (size_t)s->box.profile_bins * 8 + 3;
    CUDA_TRY(cudaMemsetAsync(s->arena.profile, 0, words * sizeof(unsigned long long), s->stream));
    s->profile_samples = 0;
    return VLJ_OK;
}

// lennard_jones.rs:1294-1325: averages per sample
vlj_status vlj_read_profile(vlj_sim* s, vlj_slab* slabs, double virial[3], uint64_t* samples) {
    TRY(need_profile(s));
    if (!slabs || !virial || !samples) return fail(VLJ_INVALID_ARG, "null argument");
    const uint32_t bins = s->box.profile_bins;
    std::vector<long long> raw((size_t)bins * 8 + 3);
    CUDA_TRY(cudaMemcpyAsync(raw.data(), s->arena.profile, raw.size() * sizeof(long long),
                             cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    TRY(check_fault(s));
    const double n = (double)s->profile_samples;
    const double width = s->box.box[2] / (double)bins;
    auto q = [&](size_t w) { return n > 0.0 ? (double)raw[w] / kOne / n : 0.0; };
    for (uint32_t b = 0; b < bins; b++) {
        const size_t o = (size_t)b * 8;
        slabs[b].z = ((double)b + 0.5) * width;
        slabs[b].particles = q(o);
        for (int k = 0; k < 3; k++) {
            slabs[b].kinetic[k] = q(o + 1 + k);
            slabs[b].virial[k] = q(o + 4 + k);
        }
        slabs[b].potential = q(o + 7);
    }
    for (int k = 0; k < 3; k++) virial[k] = q((size_t)bins * 8 + k);
    *samples = s->profile_samples;
    return VLJ_OK;
}

// lennard_jones.rs:954-974: room for `capacity` samples, earlier ones dropped
vlj_status vlj_record_heat_current(vlj_sim* s, uint32_t capacity) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    s->heat_pending = false;  // a sample of the series being dropped
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (s->series) {
        cudaFree(s->series);
        s->series = nullptr;
    }
    const size_t words = 1 + 3 * (size_t)capacity;
    void* p = nullptr;
    CUDA_TRY(cudaMalloc(&p, words * sizeof(unsigned long long)));
    s->series = static_cast<unsigned long long*>(p);
    CUDA_TRY(cudaMemset(s->series, 0, words * sizeof(unsigned long long)));
    s->arena.series = s->series;
    s->arena.series_capacity = capacity;
    s->series_capacity = capacity;
    s->series_samples = 0;
    CUDA_TRY(cudaMemsetAsync(&s->arena.glob->heat_next, 0, sizeof(uint32_t), s->stream));
    // the captured steps hold the old series' address
    sim_drop_step_graphs(s);
    return VLJ_OK;
}

// lennard_jones.rs:976-998
vlj_status vlj_sample_heat_current(vlj_sim* s) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (!s->series) return fail(VLJ_NOT_ENABLED, "record_heat_current first");
    if (s->series_samples >= s->series_capacity)
        return fail(VLJ_FULL, "heat current series full");
    TRY(sim_flush_heat(s));
    if (s->canonical()) {
        TRY(sim_lists_now(s));
        CUDA_TRY(launch_heat_current(s->arena, s->shifted_force, s->series_samples, s->stream));
    } else {
        // taken by the next step's force pass, which sees this same state
        s->heat_pending = true;
    }
    s->series_samples += 1;
    return VLJ_OK;
}

// lennard_jones.rs:1000-1012: (x, y, z) per sample, oldest first
vlj_status vlj_read_heat_current(vlj_sim* s, double* out, size_t capacity, size_t* samples) {
    if (!s || !samples) return fail(VLJ_INVALID_ARG, "null argument");
    if (!s->series) return fail(VLJ_NOT_ENABLED, "record_heat_current first");
    TRY(sim_flush_heat(s));
    const size_t n = s->series_samples;
    std::vector<long long> raw(1 + 3 * n);
    CUDA_TRY(cudaMemcpyAsync(raw.data(), s->series, raw.size() * sizeof(long long),
                             cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    TRY(check_fault(s));
    const size_t m = std::min(n, capacity);
    for (size_t k = 0; k < m && out; k++)
        for (int c = 0; c < 3; c++) out[3 * k + c] = (double)raw[1 + 3 * k + c] / kOne;
    *samples = n;
    return VLJ_OK;
}

}  // extern "C"
