// C ABI of batched replicas: many independent periodic boxes of uneven size,
// density and temperature stepped together. No reference counterpart (the
// reference runs one box per LennardJones); each replica follows exactly the
// single-box method, so a replica's trajectory is bit for bit the one a
// single-box simulation of it takes.
//
// All replicas share one arena: box r owns slots [first, first + n) and cells
// [cell_base, cell_base + cells), and every kernel of a step covers all boxes
// in one launch (one thread per slot, or one warp per cell), looking up its
// box through box_of_slot / box_of_cell. The per-box words (rebuild trigger,
// measurement sums) sit side by side, so a box rebuilds only when its own
// particles crossed its skin / 2, and a whole step -- decide, the rebuild
// chain under a conditional node, the fused force + integration kernel -- is
// the same captured CUDA graph as a single box's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
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

struct vlj_batch {
    vlj_sim* sim = nullptr;
    long long* accum = nullptr;  // pinned: kSlots per replica
    Control* ctrl = nullptr;     // pinned: one per replica
    ~vlj_batch() {
        if (sim) {
            if (sim->stream) cudaStreamSynchronize(sim->stream);
            delete sim;
        }
        if (accum) cudaFreeHost(accum);
        if (ctrl) cudaFreeHost(ctrl);
    }
};

namespace {

double rem_euclid(double x, double side) {
    double r = std::fmod(x, side);
    return r < 0.0 ? r + side : r;
}

// Every replica's particles into its slots (positions wrapped into its box),
// ids the input order within the replica.
vlj_status upload(vlj_sim* s, const vlj_replica_desc* r) {
    const size_t seg = s->arena.seg;
    for (size_t b = 0; b < s->replicas.size(); b++) {
        const Box& bx = s->replicas[b];
        const vlj_particle* p = r[b].particles;
        for (uint32_t i = 0; i < bx.n; i++) {
            const size_t slot = (size_t)bx.first + i;
            for (int k = 0; k < 3; k++) {
                if (!std::isfinite(p[i].pos[k]) || !std::isfinite(p[i].vel[k]))
                    return fail(VLJ_INVALID_ARG, "replica %zu particle %u has a non-finite coordinate",
                                b, i);
                s->pin_x[k * seg + slot] = rem_euclid(p[i].pos[k], bx.box[k]);
                s->pin_v[k * seg + slot] = p[i].vel[k];
            }
            s->pin_id[slot] = i;
        }
    }
    CUDA_TRY(cudaMemcpyAsync(s->arena.x, s->pin_x, sizeof(double) * 3 * seg,
                             cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->arena.v, s->pin_v, sizeof(double) * 3 * seg,
                             cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->arena.id, s->pin_id, sizeof(uint32_t) * seg,
                             cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return VLJ_OK;
}

// One replica's measurement from its fixed-point sums (lennard_jones.rs:1209-1246).
vlj_measurement decode(const vlj_sim* s, const Box& bx, const long long* slots,
                       const Control& c) {
    vlj_measurement m;
    std::memset(&m, 0, sizeof m);
    auto value = [](long long raw) { return (double)raw / 4294967296.0; };
    const double es = (double)bx.energy_scale, ms = (double)bx.momentum_scale;
    m.step = s->steps;
    m.time = (double)s->steps * bx.dt;
    m.kinetic = value(slots[0]) / es;
    m.potential = value(slots[1]) / es;
    m.virial = value(slots[2]) / es;
    for (int k = 0; k < 3; k++) m.momentum[k] = value(slots[3 + k]) / ms;
    m.count = bx.n;
    m.volume = bx.box[0] * bx.box[1] * bx.box[2];
    m.list_rebuilds = c.rebuilds;
    m.list_overflow = c.overflow;
    m.condensed = (uint32_t)std::llround(value(slots[6]));
    m.list_capacity = bx.capacity;
    m.list_grows = s->list_grows;
    return m;
}

// Forces, energies and canonical velocities of every box now (the lists
// brought up to date first); the sums land in a.accum.
vlj_status measure_all(vlj_batch* bt, bool canonical) {
    vlj_sim* s = bt->sim;
    const size_t boxes = s->replicas.size();
    CUDA_TRY(cudaMemsetAsync(s->arena.accum, 0, sizeof(unsigned long long) * kSlots * boxes,
                             s->stream));
    TRY(sim_lists_now(s));
    CUDA_TRY(launch_measure(s->arena, s->list_map, s->shifted_force, canonical, s->stream));
    return VLJ_OK;
}

}  // namespace

extern "C" {

vlj_status vlj_batch_create(const vlj_replica_desc* replicas, size_t count, double cutoff,
                            double skin, double dt, int32_t shifted_force, void* stream,
                            vlj_batch** out) {
    clear_error();
    if (!out) return fail(VLJ_INVALID_ARG, "out is null");
    *out = nullptr;
    if (!replicas || count == 0) return fail(VLJ_INVALID_ARG, "no replicas");
    if (count > (1u << 20)) return fail(VLJ_INVALID_ARG, "at most 2^20 replicas");
    uint64_t total = 0;
    for (size_t r = 0; r < count; r++) {
        if (!replicas[r].particles || replicas[r].count == 0)
            return fail(VLJ_INVALID_ARG, "replica %zu has no particles", r);
        vlj_settings st;
        std::memset(&st, 0, sizeof st);
        for (int k = 0; k < 3; k++) st.box_size[k] = replicas[r].box_size[k];
        st.cutoff = cutoff;
        st.skin = skin;
        st.dt = dt;
        st.thermostat = replicas[r].thermostat;
        st.shifted_force = shifted_force;
        TRY(check_settings(&st));
        if (st.thermostat.kind == VLJ_THERMOSTAT_NOSE_HOOVER)
            return fail(VLJ_NOT_ENABLED, "replicas take Langevin or no thermostat");
        total += replicas[r].count;
    }
    if (total >= (1ull << 30)) return fail(VLJ_INVALID_ARG, "at most 2^30 - 1 particles in all");
    int devices = 0;
    vlj_device_count(&devices);
    if (devices == 0) return fail(VLJ_NO_DEVICE, "no CUDA device is visible");

    vlj_batch* bt = new vlj_batch();
    vlj_sim* s = new vlj_sim();
    s->list_growth = list_growth_default();
    bt->sim = s;
    std::memset(&s->settings, 0, sizeof s->settings);
    s->settings.cutoff = cutoff;
    s->settings.skin = skin;
    s->settings.dt = dt;
    s->settings.shifted_force = shifted_force;
    s->shifted_force = shifted_force != 0;
    s->replicas.resize(count);
    vlj_status st = VLJ_OK;
    for (size_t r = 0; r < count && st == VLJ_OK; r++) {
        st = make_box(replicas[r].particles, replicas[r].count, replicas[r].box_size, cutoff, skin,
                      dt, s->shifted_force, replicas[r].thermostat, 0, s->replicas[r], 2);
        if (st != VLJ_OK) {
            const std::string why = vlj_last_error();
            fail(st, "replica %zu: %s", r, why.c_str());
        }
    }
    if (st == VLJ_OK) st = sim_allocate(s, stream);
    if (st == VLJ_OK && (cudaMallocHost(&bt->accum, sizeof(long long) * kSlots * count) != cudaSuccess ||
                         cudaMallocHost(&bt->ctrl, sizeof(Control) * count) != cudaSuccess))
        st = fail(VLJ_CUDA_ERROR, "pinned read-back buffers");
    if (st == VLJ_OK) st = upload(s, replicas);
    if (st == VLJ_OK) {
        // never built: every box rebuilds at the first decision
        cudaError_t e = launch_decide(s->arena, s->stream, 0);
        if (e == cudaSuccess) e = launch_encode(s->arena, s->stream);
        if (e == cudaSuccess) e = launch_rebuild(s->arena, s->stream);
        // lists that overflowed on the first build grow before the first forces
        bool grew = false;
        if (e == cudaSuccess) st = sim_grow_lists(s, &grew);
        if (st != VLJ_OK) e = cudaErrorUnknown;
        if (e == cudaSuccess) e = launch_prime(s->arena, s->list_map, s->shifted_force, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess && st == VLJ_OK)
            st = fail(VLJ_CUDA_ERROR, "first lists: %s", cudaGetErrorString(e));
    }
    if (st == VLJ_OK) st = check_fault(s);
    if (st != VLJ_OK) {
        delete bt;
        return st;
    }
    *out = bt;
    return VLJ_OK;
}

vlj_status vlj_batch_destroy(vlj_batch* batch) {
    delete batch;
    return VLJ_OK;
}

vlj_status vlj_batch_step(vlj_batch* bt, uint32_t steps) {
    if (!bt) return fail(VLJ_INVALID_ARG, "batch is null");
    if (bt->sim->grow_pending) {
        bool grew = false;
        TRY(sim_grow_lists(bt->sim, &grew));
    }
    TRY(sim_enqueue_steps(bt->sim, steps));
    bt->sim->steps += steps;
    return VLJ_OK;
}

vlj_status vlj_batch_run(vlj_batch* bt, uint64_t steps) {
    if (!bt) return fail(VLJ_INVALID_ARG, "batch is null");
    while (steps > 0) {
        const uint32_t chunk = (uint32_t)std::min<uint64_t>(steps, 200);
        TRY(vlj_batch_step(bt, chunk));
        steps -= chunk;
    }
    CUDA_TRY(cudaStreamSynchronize(bt->sim->stream));
    TRY(check_fault(bt->sim));
    bool grew = false;
    return sim_grow_lists(bt->sim, &grew);
}

vlj_status vlj_batch_measure(vlj_batch* bt, vlj_measurement* out) {
    if (!bt || !out) return fail(VLJ_INVALID_ARG, "null argument");
    vlj_sim* s = bt->sim;
    const size_t boxes = s->replicas.size();
    TRY(measure_all(bt, false));
    CUDA_TRY(cudaMemcpyAsync(bt->accum, s->arena.accum, sizeof(long long) * kSlots * boxes,
                             cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaMemcpyAsync(bt->ctrl, s->arena.ctrl, sizeof(Control) * boxes,
                             cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    TRY(check_fault(s));
    bool overflow = false;
    for (size_t r = 0; r < boxes; r++) overflow = overflow || bt->ctrl[r].overflow != 0u;
    if (overflow && s->list_growth) {
        // lists that dropped pairs: grow them, rebuild, measure again
        bool grew = false;
        TRY(sim_grow_lists(s, &grew));
        if (grew) return vlj_batch_measure(bt, out);
    }
    for (size_t r = 0; r < boxes; r++)
        out[r] = decode(s, s->replicas[r], bt->accum + kSlots * r, bt->ctrl[r]);
    return VLJ_OK;
}

vlj_status vlj_batch_read_particles(vlj_batch* bt, size_t replica, vlj_particle* out) {
    if (!bt || !out) return fail(VLJ_INVALID_ARG, "null argument");
    vlj_sim* s = bt->sim;
    if (replica >= s->replicas.size())
        return fail(VLJ_INVALID_ARG, "replica %zu of %zu", replica, s->replicas.size());
    const Box& bx = s->replicas[replica];
    const size_t seg = s->arena.seg, first = bx.first, n = bx.n;
    TRY(measure_all(bt, true));
    for (int k = 0; k < 3; k++) {
        CUDA_TRY(cudaMemcpyAsync(s->pin_x + k * seg + first, s->arena.x + k * seg + first,
                                 sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(s->pin_v + k * seg + first, s->arena.vcanon + k * seg + first,
                                 sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    }
    CUDA_TRY(cudaMemcpyAsync(s->pin_id + first, s->arena.id + first, sizeof(uint32_t) * n,
                             cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    TRY(check_fault(s));
    for (size_t slot = first; slot < first + n; slot++) {
        const uint32_t i = s->pin_id[slot];
        if (i >= n) return fail(VLJ_CUDA_ERROR, "corrupt particle id %u in slot %zu", i, slot);
        for (int k = 0; k < 3; k++) {
            out[i].pos[k] = s->pin_x[k * seg + slot];
            out[i].vel[k] = s->pin_v[k * seg + slot];
        }
    }
    return VLJ_OK;
}

vlj_status vlj_batch_count(const vlj_batch* bt, size_t* replicas, uint64_t* particles) {
    if (!bt || !replicas || !particles) return fail(VLJ_INVALID_ARG, "null argument");
    *replicas = bt->sim->replicas.size();
    *particles = bt->sim->n;
    return VLJ_OK;
}

vlj_status vlj_batch_box_size(const vlj_batch* bt, size_t replica, double out[3]) {
    if (!bt || !out) return fail(VLJ_INVALID_ARG, "null argument");
    if (replica >= bt->sim->replicas.size())
        return fail(VLJ_INVALID_ARG, "replica %zu of %zu", replica, bt->sim->replicas.size());
    for (int k = 0; k < 3; k++) out[k] = bt->sim->replicas[replica].box[k];
    return VLJ_OK;
}

vlj_status vlj_debug_batch_sim(vlj_batch* bt, vlj_sim** sim) {
    if (!bt || !sim) return fail(VLJ_INVALID_ARG, "null argument");
    *sim = bt->sim;
    return VLJ_OK;
}

}  // extern "C"
