// The simulation object behind the opaque vlj_sim handle.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <vector>

#include "virial_lj.h"
#include "vlj_internal.cuh"

namespace vlj {

constexpr int kRing = 3;  // measurement read-back slots (lennard_jones.rs:320)
constexpr uint32_t kGraphChunk = 16;  // steps per graph launch

// One measurement's words as read back into pinned host memory.
struct Readback {
    long long slots[kSlots];
    Control ctrl;
    Thermo nh;
};

double scale_for(double magnitude);
vlj_status check_settings(const vlj_settings* st);
vlj_status make_box(const vlj_particle* p, size_t count, const double box_size[3], double cutoff,
                    double skin, double dt, bool shifted_force, const vlj_thermostat& t,
                    uint32_t profile_bins, Box& b, uint32_t min_cells);

}  // namespace vlj

struct vlj_sim {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    vlj_settings settings{};
    uint32_t n = 0;
    bool shifted_force = false;
    bool nose_hoover = false;  // steps on canonical velocities with the thermostat
    bool exchange = false;     // heat exchange on (constant energy, canonical velocities)
    vlj_heat_exchange exchange_settings{};
    bool canonical() const { return nose_hoover || exchange; }
    bool grid_every_step = false;  // bin, scan, scatter, sort every step; lists on the trigger
    bool tiles_on = true;  // the step kernel stages cell tiles (when the box has them)
    bool list_growth = true;   // grow the list capacity when a list overflows
    bool grow_pending = false; // a polled measurement showed an overflow
    uint32_t list_grows = 0;   // capacity grows so far
    vlj::Box box{};
    // batched: one Box per replica, in slot order (empty for a single box)
    std::vector<vlj::Box> replicas;
    vlj::Arena arena{};
    CUtensorMap list_map;  // list rows for the force kernels' TMA tiles
    std::vector<void*> allocations;
    uint64_t steps = 0;
    // measurement read-back ring
    vlj::Readback* ring = nullptr;
    cudaEvent_t ring_event[vlj::kRing] = {};
    bool ring_busy[vlj::kRing] = {};
    uint64_t ring_step[vlj::kRing] = {};
    // profiles
    uint64_t profile_samples = 0;
    // heat current series
    uint32_t series_samples = 0;
    // the last requested sample is not taken yet: the next step's force pass
    // takes it (or, before anything that would change the state or read the
    // series, the sampling kernel)
    bool heat_pending = false;
    uint32_t series_capacity = 0;
    unsigned long long* series = nullptr;  // owned here (reallocated by record)
    // pinned staging for particle uploads and read-backs (x, v: 3 * seg; id: seg)
    double* pin_x = nullptr;
    double* pin_v = nullptr;
    uint32_t* pin_id = nullptr;
    // captured steps: a graph of kGraphChunk steps and one of a single step,
    // each step's rebuild chain under a conditional node
    bool use_graphs = true;
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t graph_chunk = nullptr;
    cudaGraphExec_t graph_one = nullptr;
    // graph_one's template (kept for node updates) and its decide node: while
    // the last step enqueued was graph_one's, whose step kernel took this
    // step's decision and set graph_one's condition, the node is disabled
    cudaGraph_t graph_one_tmpl = nullptr;
    cudaGraphNode_t one_decide = nullptr;
    bool one_decide_on = true;
    bool one_ready = false;
    cudaGraphExec_t graph_one_heat = nullptr;  // one step that also takes the pending sample
    cudaGraphExec_t graph_lists = nullptr;  // decide -> IF(rebuild){rebuild chain}
    // per-launch timing of the step kernel (direct launches while on)
    bool timing = false;
    std::vector<cudaEvent_t> ev_start, ev_end;
    size_t ev_used = 0;

    ~vlj_sim();
};

namespace vlj {
vlj_status sim_allocate(vlj_sim* s, void* stream);
vlj_status make_list_map(const Arena& a, uint32_t rows, CUtensorMap* out);
// Decide and, when due, rebuild the lists now (positions are about to be read).
vlj_status sim_lists_now(vlj_sim* s);
vlj_status check_fault(vlj_sim* s);
vlj_status sim_enqueue_steps(vlj_sim* s, uint32_t steps);
// Takes a pending heat-current sample now, with the sampling kernel.
vlj_status sim_flush_heat(vlj_sim* s);
// With list growth on and a list overflowed since the last build: raise the
// capacity of every box that overflowed, reallocate the lists, drop the
// captured graphs and force a rebuild (waits). *grew says whether it did.
vlj_status sim_grow_lists(vlj_sim* s, bool* grew);
// List growth at creation: on, unless the environment sets VLJ_LIST_GROWTH=0
// (the reference's report-only behaviour from the first build on).
bool list_growth_default();
// Drops the captured step graphs (their shape changed).
void sim_drop_step_graphs(vlj_sim* s);
// The decision and, when due, the rebuild as one graph launch.
vlj_status sim_launch_lists_graph(vlj_sim* s);
}  // namespace vlj
