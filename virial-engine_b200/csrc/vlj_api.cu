// C ABI of the single-box simulation (include/virial_lj.h): the B200 stand-in
// for virial_particles::lennard_jones::LennardJones
// (crates/virial-particles/src/lennard_jones.rs:334-1375).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "virial_lj.h"
#include "vlj_common.h"
#include "vlj_internal.cuh"
#include "vlj_sim.h"

using namespace vlj;

namespace vlj {

// lennard_jones.rs:435-440
double scale_for(double magnitude) {
    if (magnitude <= 0.0 || !std::isfinite(magnitude)) return 1.0;
    return std::pow(2.0, std::floor(20.0 - std::log2(magnitude)));
}

vlj_status check_settings(const vlj_settings* st) {
    if (!st) return fail(VLJ_INVALID_ARG, "settings is null");
    for (int k = 0; k < 3; k++)
        if (!(st->box_size[k] > 0.0) || !std::isfinite(st->box_size[k]))
            return fail(VLJ_INVALID_ARG, "box side %d is not a positive finite number", k);
    if (!(st->cutoff > 0.0) || !std::isfinite(st->cutoff))
        return fail(VLJ_INVALID_ARG, "cutoff must be positive");
    if (!(st->skin >= 0.0) || !std::isfinite(st->skin))
        return fail(VLJ_INVALID_ARG, "skin must be non-negative");
    if (!(st->dt > 0.0) || !std::isfinite(st->dt)) return fail(VLJ_INVALID_ARG, "dt must be positive");
    const vlj_thermostat& t = st->thermostat;
    switch (t.kind) {
        case VLJ_THERMOSTAT_NONE: break;
        case VLJ_THERMOSTAT_LANGEVIN:
            if (!(t.temperature >= 0.0) || !(t.friction >= 0.0) || !std::isfinite(t.temperature) ||
                !std::isfinite(t.friction))
                return fail(VLJ_INVALID_ARG, "Langevin needs temperature >= 0 and friction >= 0");
            break;
        case VLJ_THERMOSTAT_NOSE_HOOVER:
            if (!(t.temperature > 0.0) || !(t.period > 0.0))
                return fail(VLJ_INVALID_ARG, "Nose-Hoover needs temperature > 0 and period > 0");
            break;
        default: return fail(VLJ_INVALID_ARG, "unknown thermostat kind %d", (int)t.kind);
    }
    return VLJ_OK;
}

// What LennardJones::new derives from the settings (lennard_jones.rs:450-560).
// min_cells is 3 for the reference's 27-cell search (lennard_jones.rs:457-461);
// batched replicas accept 2, where the list build visits each distinct
// neighbour cell once.
vlj_status make_box(const vlj_particle* p, size_t count, const double box_size[3], double cutoff,
                    double skin, double dt, bool shifted_force, const vlj_thermostat& t,
                    uint32_t profile_bins, Box& b, uint32_t min_cells) {
    std::memset(&b, 0, sizeof b);
    const double list_radius = cutoff + skin;
    uint32_t cells[3];
    for (int k = 0; k < 3; k++) {
        b.box_f[k] = (float)box_size[k];
        b.box[k] = (double)b.box_f[k];
        double c = std::floor(b.box[k] / list_radius);
        cells[k] = c < 0.0 ? 0u : (c > 4.0e9 ? 4000000000u : (uint32_t)c);
    }
    if (cells[0] < min_cells || cells[1] < min_cells || cells[2] < min_cells)
        return fail(VLJ_BOX_TOO_SMALL,
                    "the box must be at least %s (cutoff + skin) wide on every axis",
                    min_cells >= 3 ? "three" : "two");
    while ((uint64_t)cells[0] * cells[1] * cells[2] > (1u << 20)) {
        int longest = 0;
        for (int k = 1; k < 3; k++)
            if (cells[k] >= cells[longest]) longest = k;
        cells[longest] -= 1;
    }
    for (int k = 0; k < 3; k++) {
        b.cells[k] = cells[k];
        b.cell_size_f[k] = (float)(b.box[k] / (double)cells[k]);
        b.enc[k] = 4294967296.0 / b.box[k];
        b.dec[k] = (float)(b.box[k] / 4294967296.0);
    }
    b.total_cells = cells[0] * cells[1] * cells[2];
    const double volume = b.box[0] * b.box[1] * b.box[2];
    const double density = (double)count / volume;
    const double expected =
        4.0 / 3.0 * 3.141592653589793 * (list_radius * list_radius * list_radius) * density;
    b.capacity = (uint32_t)std::ceil(2.0 * expected + 32.0);
    b.n = (uint32_t)count;

    double kinetic = 0.0, speed = 0.0;
    for (size_t i = 0; i < count; i++) {
        double v2 = 0.0;
        for (int k = 0; k < 3; k++) v2 += p[i].vel[k] * p[i].vel[k];
        kinetic += 0.5 * v2;
        speed += std::sqrt(v2);
    }
    double thermal = 0.0;
    if (t.kind != VLJ_THERMOSTAT_NONE) thermal = 1.5 * t.temperature * (double)count;
    double m = std::max(std::max(kinetic, thermal), (double)count);
    b.energy_scale = (float)scale_for(m);
    b.momentum_scale = (float)scale_for(std::max(speed, (double)count));

    const double rc2 = cutoff * cutoff;
    const double inv6 = 1.0 / (rc2 * rc2 * rc2);
    b.shift = (float)(4.0 * (inv6 * inv6 - inv6));
    b.force_shift = shifted_force ? (float)(24.0 * (2.0 * inv6 * inv6 - inv6) / cutoff) : 0.0f;
    b.rc = (float)std::sqrt((double)(float)rc2);
    b.rc2 = (float)rc2;
    b.list_r2 = (float)(list_radius * list_radius);
    b.half_skin2 = (float)(0.25 * skin * skin);
    // The reference's f32 separations can be off by a few units in the last
    // place of the box side (pairs across the boundary); the encoded ones by
    // far less. Bracket the list radius by more than both.
    double side_max = std::max(b.box[0], std::max(b.box[1], b.box[2]));
    double margin = 8.0 * std::ldexp(1.0, std::ilogb(side_max) - 23) + 1e-4;
    double list_r = std::sqrt((double)b.list_r2);
    b.prefilter_r2 = (float)((list_r + margin) * (list_r + margin));
    b.accept_r2 = (float)((list_r - margin) * (list_r - margin));
    // a particle binned into a cell lies within 1e-3 of the cell's box
    b.reach_r2 = (float)((list_r + margin + 1e-3) * (list_r + margin + 1e-3));
    for (int k = 0; k < 3; k++) b.inv_box_f[k] = 1.0f / b.box_f[k];
    b.dt = dt;
    b.half_dt = 0.5 * dt;
    b.c1 = 1.0;
    b.c2 = 0.0;
    b.thermostat = t.kind;
    if (t.kind == VLJ_THERMOSTAT_LANGEVIN) {
        b.c1 = std::exp(-t.friction * dt);
        b.c2 = std::sqrt((1.0 - b.c1 * b.c1) * t.temperature);
        b.seed = t.seed;
    }
    b.nh_q = 1.0;
    b.canonical = t.kind == VLJ_THERMOSTAT_NOSE_HOOVER ? 1u : 0u;
    if (t.kind == VLJ_THERMOSTAT_NOSE_HOOVER) {
        // lennard_jones.rs:516-528: g = 3N - 3 (zero total momentum),
        // Q = g T period^2 / (4 pi^2)
        const double dof = 3.0 * (double)count - 3.0;
        b.nh_gkt = dof * t.temperature;
        b.nh_q = dof * t.temperature * t.period * t.period / (4.0 * M_PI * M_PI);
    }
    b.near_count = 4;
    b.drawn = VLJ_DRAWN_NEIGHBOURS;
    b.reorder_every = 4;
    b.profile_bins = profile_bins;
    b.bin_width = (float)(b.box[2] / (double)std::max(profile_bins, 1u));
    return VLJ_OK;
}

}  // namespace vlj

#define CUDA_TRY(call)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(VLJ_CUDA_ERROR, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                        __FILE__, __LINE__);                                                \
    } while (0)

#define TRY(expr)                          \
    do {                                   \
        vlj_status s_ = (expr);            \
        if (s_ != VLJ_OK) return s_;       \
    } while (0)

namespace {

template <class T>
vlj_status dalloc(vlj_sim* s, T** p, size_t count) {
    void* q = nullptr;
    size_t bytes = sizeof(T) * (count ? count : 1);
    CUDA_TRY(cudaMalloc(&q, bytes));
    s->allocations.push_back(q);
    CUDA_TRY(cudaMemset(q, 0, bytes));
    *p = static_cast<T*>(q);
    return VLJ_OK;
}

// The particles as given (one copy of the caller's array), then on the
// device: positions wrapped into the box, structure of arrays, ids the input
// order. A non-finite coordinate is reported once the copy has landed.
vlj_status upload_particles(vlj_sim* s, const vlj_particle* p, size_t count) {
    CUDA_TRY(cudaMemsetAsync(&s->arena.glob->fault, 0, sizeof(uint32_t), s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->arena.aos, p, sizeof(vlj_particle) * count, cudaMemcpyHostToDevice,
                             s->stream));
    CUDA_TRY(launch_load_particles(s->arena, s->stream));
    Global g;
    CUDA_TRY(cudaMemcpyAsync(&g, s->arena.glob, sizeof g, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (g.fault == kFaultNonFinite) {
        cudaMemsetAsync(&s->arena.glob->fault, 0, sizeof(uint32_t), s->stream);
        return fail(VLJ_INVALID_ARG, "a particle has a non-finite coordinate");
    }
    return VLJ_OK;
}

vlj_status lists_now(vlj_sim* s) {
    s->one_ready = false;
    if (s->use_graphs && !s->timing) return sim_launch_lists_graph(s);
    CUDA_TRY(launch_decide(s->arena, s->stream, 0));
    CUDA_TRY(launch_rebuild(s->arena, s->stream));
    return VLJ_OK;
}

// Fresh state from `p`: forced rebuild, then the first forces turn the given
// velocities into ones half a kick behind (lennard_jones.rs:1080-1089).
vlj_status restart(vlj_sim* s, const vlj_particle* p, size_t count) {
    s->one_ready = false;
    TRY(upload_particles(s, p, count));
    uint32_t one = 1u;
    CUDA_TRY(cudaMemcpyAsync(&s->arena.ctrl[0].forced, &one, sizeof one, cudaMemcpyHostToDevice,
                             s->stream));
    CUDA_TRY(launch_decide(s->arena, s->stream, 0));
    CUDA_TRY(launch_encode(s->arena, s->stream));
    CUDA_TRY(launch_rebuild(s->arena, s->stream));
    // lists that overflowed on the first build grow before the first forces
    bool grew = false;
    TRY(sim_grow_lists(s, &grew));
    if (s->canonical()) {
        // the thermostat starts at rest (xi = eta = 0) from the given
        // velocities; the first forces are recorded for the first half kick
        CUDA_TRY(cudaMemsetAsync(s->arena.nh, 0, sizeof(Thermo), s->stream));
        CUDA_TRY(cudaMemsetAsync(s->arena.hex, 0, sizeof(Exchange), s->stream));
        CUDA_TRY(launch_canon_force(s->arena, s->list_map, s->shifted_force, kPrime, s->stream));
    } else {
        CUDA_TRY(launch_prime(s->arena, s->list_map, s->shifted_force, s->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return VLJ_OK;
}

vlj_status push_box(vlj_sim* s) {
    CUDA_TRY(cudaMemcpyAsync(const_cast<Box*>(s->arena.boxes), &s->box, sizeof(Box),
                             cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return VLJ_OK;
}

vlj_measurement decode(const vlj_sim* s, const Readback& r, uint64_t step) {
    vlj_measurement m;
    std::memset(&m, 0, sizeof m);
    auto value = [](long long raw) { return (double)raw / 4294967296.0; };
    const double es = (double)s->box.energy_scale, ms = (double)s->box.momentum_scale;
    m.step = step;
    m.time = (double)step * s->settings.dt;
    m.kinetic = value(r.slots[0]) / es;
    m.potential = value(r.slots[1]) / es;
    m.virial = value(r.slots[2]) / es;
    for (int k = 0; k < 3; k++) m.momentum[k] = value(r.slots[3 + k]) / ms;
    m.count = s->n;
    m.volume = s->box.box[0] * s->box.box[1] * s->box.box[2];
    m.list_rebuilds = r.ctrl.rebuilds;
    m.list_overflow = r.ctrl.overflow;
    m.condensed = (uint32_t)std::llround(value(r.slots[6]));
    m.list_capacity = s->box.capacity;
    m.list_grows = s->list_grows;
    // lennard_jones.rs:1235-1241: Q xi^2 / 2 + g k T eta
    m.thermostat_energy = s->nose_hoover
        ? 0.5 * s->box.nh_q * r.nh.xi_m * r.nh.xi_m + s->box.nh_gkt * r.nh.eta_m : 0.0;
    return m;
}

vlj_status enqueue_measure(vlj_sim* s, bool canonical, int slot) {
    CUDA_TRY(cudaMemsetAsync(s->arena.accum, 0, sizeof(unsigned long long) * kSlots, s->stream));
    TRY(lists_now(s));
    CUDA_TRY(launch_measure(s->arena, s->list_map, s->shifted_force, canonical, s->stream));
    if (s->box.drawn == VLJ_DRAWN_TEMPERATURE) CUDA_TRY(launch_drawn_temperature(s->arena, s->stream));
    if (slot >= 0) {
        Readback* r = &s->ring[slot];
        CUDA_TRY(cudaMemcpyAsync(r->slots, s->arena.accum, sizeof(r->slots), cudaMemcpyDeviceToHost,
                                 s->stream));
        CUDA_TRY(cudaMemcpyAsync(&r->ctrl, s->arena.ctrl, sizeof(Control), cudaMemcpyDeviceToHost,
                                 s->stream));
        if (s->nose_hoover)
            CUDA_TRY(cudaMemcpyAsync(&r->nh, s->arena.nh, sizeof(Thermo), cudaMemcpyDeviceToHost,
                                     s->stream));
        CUDA_TRY(cudaEventRecord(s->ring_event[slot], s->stream));
        s->ring_busy[slot] = true;
        s->ring_step[slot] = s->steps;
    }
    return VLJ_OK;
}

}  // namespace

vlj_sim::~vlj_sim() {
    if (graph_chunk) cudaGraphExecDestroy(graph_chunk);
    if (graph_one) cudaGraphExecDestroy(graph_one);
    if (graph_one_tmpl) cudaGraphDestroy(graph_one_tmpl);
    if (graph_one_heat) cudaGraphExecDestroy(graph_one_heat);
    if (graph_lists) cudaGraphExecDestroy(graph_lists);
    if (capture_stream) cudaStreamDestroy(capture_stream);
    for (cudaEvent_t e : ev_start) cudaEventDestroy(e);
    for (cudaEvent_t e : ev_end) cudaEventDestroy(e);
    if (pin_x) cudaFreeHost(pin_x);
    if (pin_v) cudaFreeHost(pin_v);
    if (pin_id) cudaFreeHost(pin_id);
    if (series) cudaFree(series);
    for (int k = 0; k < kRing; k++)
        if (ring_event[k]) cudaEventDestroy(ring_event[k]);
    if (ring) cudaFreeHost(ring);
    for (void* p : allocations) cudaFree(p);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

namespace vlj {
static bool plan_tiles(Box& b, Arena& a, uint32_t want_cols);  // below
static vlj_status free_device(vlj_sim* s, void* p);
}  // namespace vlj

extern "C" {

vlj_status vlj_device_count(int* count) {
    if (!count) return fail(VLJ_INVALID_ARG, "count is null");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return VLJ_OK;
}

vlj_status vlj_create(const vlj_particle* particles, size_t count, const vlj_settings* settings,
                      void* stream, vlj_sim** out) {
    clear_error();
    if (!out) return fail(VLJ_INVALID_ARG, "out is null");
    *out = nullptr;
    if (!particles || count == 0) return fail(VLJ_INVALID_ARG, "no particles");
    // list offsets are 32-bit (a slot's four entries per row, rows 4 * seg
    // apart); 2^30 particles' lists would be far beyond one GPU's memory anyway
    if (count >= (1ull << 30)) return fail(VLJ_INVALID_ARG, "at most 2^30 - 1 particles");
    TRY(check_settings(settings));
    int devices = 0;
    vlj_device_count(&devices);
    if (devices == 0) return fail(VLJ_NO_DEVICE, "no CUDA device is visible");
    if (settings->thermostat.kind == VLJ_THERMOSTAT_NOSE_HOOVER && count < 2)
        return fail(VLJ_INVALID_ARG, "Nose-Hoover needs at least two particles");

    vlj_sim* s = new vlj_sim();
    s->list_growth = list_growth_default();
    s->settings = *settings;
    s->n = (uint32_t)count;
    s->shifted_force = settings->shifted_force != 0;
    s->nose_hoover = settings->thermostat.kind == VLJ_THERMOSTAT_NOSE_HOOVER;
    vlj_status st = make_box(particles, count, settings->box_size, settings->cutoff,
                             settings->skin, settings->dt, s->shifted_force, settings->thermostat,
                             settings->profile_bins, s->box, 3);
    if (st != VLJ_OK) {
        delete s;
        return st;
    }
    st = sim_allocate(s, stream);
    if (st == VLJ_OK) st = restart(s, particles, count);
    if (st != VLJ_OK) {
        delete s;
        return st;
    }
    *out = s;
    return VLJ_OK;
}

vlj_status vlj_destroy(vlj_sim* sim) {
    if (!sim) return VLJ_OK;
    if (sim->stream) cudaStreamSynchronize(sim->stream);
    delete sim;
    return VLJ_OK;
}

vlj_status vlj_step(vlj_sim* s, uint32_t steps) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (s->grow_pending) {
        bool grew = false;
        TRY(sim_grow_lists(s, &grew));
    }
    TRY(sim_enqueue_steps(s, steps));
    s->steps += steps;
    return VLJ_OK;
}

vlj_status vlj_run(vlj_sim* s, uint64_t steps) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    while (steps > 0) {
        uint32_t batch = (uint32_t)std::min<uint64_t>(steps, 200);
        TRY(vlj_step(s, batch));
        steps -= batch;
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    TRY(check_fault(s));
    bool grew = false;
    return sim_grow_lists(s, &grew);
}

vlj_status vlj_measure(vlj_sim* s, int* accepted) {
    if (!s || !accepted) return fail(VLJ_INVALID_ARG, "null argument");
    *accepted = 0;
    int slot = -1;
    for (int k = 0; k < kRing; k++)
        if (!s->ring_busy[k]) {
            slot = k;
            break;
        }
    if (slot < 0) return VLJ_OK;
    TRY(enqueue_measure(s, false, slot));
    *accepted = 1;
    return VLJ_OK;
}

vlj_status vlj_poll(vlj_sim* s, vlj_measurement* out, size_t capacity, size_t* written) {
    if (!s || !written) return fail(VLJ_INVALID_ARG, "null argument");
    *written = 0;
    std::vector<std::pair<uint64_t, int>> ready;
    for (int k = 0; k < kRing; k++) {
        if (!s->ring_busy[k]) continue;
        cudaError_t e = cudaEventQuery(s->ring_event[k]);
        if (e == cudaSuccess)
            ready.push_back({s->ring_step[k], k});
        else if (e != cudaErrorNotReady)
            return fail(VLJ_CUDA_ERROR, "measurement read-back: %s", cudaGetErrorString(e));
    }
    std::sort(ready.begin(), ready.end());
    size_t n = 0;
    for (auto& r : ready) {
        if (n >= capacity || !out) break;
        out[n] = decode(s, s->ring[r.second], r.first);
        if (out[n].list_overflow && s->list_growth) s->grow_pending = true;
        n++;
        s->ring_busy[r.second] = false;
    }
    *written = n;
    return VLJ_OK;
}

vlj_status vlj_measure_now(vlj_sim* s, vlj_measurement* out) {
    if (!s || !out) return fail(VLJ_INVALID_ARG, "null argument");
    int accepted = 0;
    TRY(vlj_measure(s, &accepted));
    if (!accepted) return fail(VLJ_BUSY, "a measurement is already in flight");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    vlj_measurement buf[kRing];
    size_t n = 0;
    TRY(vlj_poll(s, buf, kRing, &n));
    if (n == 0) return fail(VLJ_CUDA_ERROR, "the measurement did not finish");
    *out = buf[n - 1];
    TRY(check_fault(s));
    if (out->list_overflow && s->list_growth) {
        // lists that dropped pairs: grow them, rebuild, measure again
        bool grew = false;
        TRY(sim_grow_lists(s, &grew));
        if (grew) return vlj_measure_now(s, out);
    }
    return VLJ_OK;
}

vlj_status vlj_read_particles(vlj_sim* s, vlj_particle* out) {
    if (!s || !out) return fail(VLJ_INVALID_ARG, "null argument");
    TRY(enqueue_measure(s, true, -1));
    CUDA_TRY(launch_store_particles(s->arena, s->stream));
    CUDA_TRY(cudaMemcpyAsync(out, s->arena.aos, sizeof(vlj_particle) * s->n, cudaMemcpyDeviceToHost,
                             s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return check_fault(s);
}

vlj_status vlj_write_particles(vlj_sim* s, const vlj_particle* p, size_t count) {
    if (!s || !p) return fail(VLJ_INVALID_ARG, "null argument");
    if (count != s->n) return fail(VLJ_INVALID_ARG, "expected %u particles, got %zu", s->n, count);
    TRY(sim_flush_heat(s));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return restart(s, p, count);
}

vlj_status vlj_count(const vlj_sim* s, uint32_t* count) {
    if (!s || !count) return fail(VLJ_INVALID_ARG, "null argument");
    *count = s->n;
    return VLJ_OK;
}

vlj_status vlj_box_size(const vlj_sim* s, double out[3]) {
    if (!s || !out) return fail(VLJ_INVALID_ARG, "null argument");
    for (int k = 0; k < 3; k++) out[k] = s->box.box[k];
    return VLJ_OK;
}

vlj_status vlj_volume(const vlj_sim* s, double* volume) {
    if (!s || !volume) return fail(VLJ_INVALID_ARG, "null argument");
    *volume = s->box.box[0] * s->box.box[1] * s->box.box[2];
    return VLJ_OK;
}

vlj_status vlj_steps(const vlj_sim* s, uint64_t* steps) {
    if (!s || !steps) return fail(VLJ_INVALID_ARG, "null argument");
    *steps = s->steps;
    return VLJ_OK;
}

vlj_status vlj_time(const vlj_sim* s, double* time) {
    if (!s || !time) return fail(VLJ_INVALID_ARG, "null argument");
    *time = (double)s->steps * s->settings.dt;
    return VLJ_OK;
}

vlj_status vlj_target_temperature(const vlj_sim* s, int* has, double* temperature) {
    if (!s || !has || !temperature) return fail(VLJ_INVALID_ARG, "null argument");
    *has = s->settings.thermostat.kind != VLJ_THERMOSTAT_NONE;
    *temperature = *has ? s->settings.thermostat.temperature : 0.0;
    return VLJ_OK;
}

vlj_status vlj_positions(const vlj_sim* s, const double** xyz, size_t* stride) {
    if (!s || !xyz || !stride) return fail(VLJ_INVALID_ARG, "null argument");
    *xyz = s->arena.x;
    *stride = s->arena.seg;
    return VLJ_OK;
}

vlj_status vlj_velocities(const vlj_sim* s, const float** vel4) {
    if (!s || !vel4) return fail(VLJ_INVALID_ARG, "null argument");
    *vel4 = reinterpret_cast<const float*>(s->arena.vel4);
    return VLJ_OK;
}

vlj_status vlj_set_drawn(vlj_sim* s, vlj_drawn drawn) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (drawn != VLJ_DRAWN_NEIGHBOURS && drawn != VLJ_DRAWN_TEMPERATURE)
        return fail(VLJ_INVALID_ARG, "unknown drawn value %d", (int)drawn);
    s->box.drawn = (uint32_t)drawn;
    return push_box(s);
}

vlj_status vlj_set_condensed_neighbours(vlj_sim* s, uint32_t neighbours) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    s->box.near_count = neighbours;
    return push_box(s);
}

// lennard_jones.rs:905-925
vlj_status vlj_set_temperature(vlj_sim* s, double temperature) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (!(temperature >= 0.0) || !std::isfinite(temperature))
        return fail(VLJ_INVALID_ARG, "temperature must be a non-negative number");
    vlj_thermostat& t = s->settings.thermostat;
    if (t.kind == VLJ_THERMOSTAT_NONE)
        return fail(VLJ_NOT_ENABLED, "set_temperature needs a thermostat");
    t.temperature = temperature;
    if (t.kind == VLJ_THERMOSTAT_LANGEVIN) {
        double c1 = std::exp(-t.friction * s->settings.dt);
        s->box.c2 = std::sqrt((1.0 - c1 * c1) * temperature);
    } else {
        if (!(temperature > 0.0))
            return fail(VLJ_INVALID_ARG, "Nose-Hoover needs a temperature above zero");
        const double dof = 3.0 * (double)s->n - 3.0;
        s->box.nh_gkt = dof * temperature;
        s->box.nh_q = dof * temperature * t.period * t.period / (4.0 * M_PI * M_PI);
    }
    return push_box(s);
}

// lennard_jones.rs:927-946. Switching the exchange on moves the velocities
// from half a kick behind to canonical (forces at the current positions);
// switching it off moves them back. Either way the captured steps change.
vlj_status vlj_set_heat_exchange(vlj_sim* s, const vlj_heat_exchange* exchange) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (s->settings.thermostat.kind != VLJ_THERMOSTAT_NONE)
        return fail(VLJ_NOT_ENABLED, "heat exchange runs at constant energy, without a thermostat");
    if (exchange) {
        for (int k = 0; k < 2; k++)
            if (!std::isfinite(exchange->hot[k]) || !std::isfinite(exchange->cold[k]))
                return fail(VLJ_INVALID_ARG, "slab bounds must be finite");
        if (!std::isfinite(exchange->energy))
            return fail(VLJ_INVALID_ARG, "energy must be finite");
    }
    const bool on = exchange != nullptr;
    TRY(sim_flush_heat(s));
    if (on != s->exchange) {
        CUDA_TRY(cudaStreamSynchronize(s->stream));
        sim_drop_step_graphs(s);
    }
    if (on) {
        s->box.hex_slabs[0] = (float)exchange->hot[0];
        s->box.hex_slabs[1] = (float)exchange->hot[1];
        s->box.hex_slabs[2] = (float)exchange->cold[0];
        s->box.hex_slabs[3] = (float)exchange->cold[1];
        s->box.hex_energy = (double)(float)exchange->energy;
        s->exchange_settings = *exchange;
    }
    if (on && !s->exchange) {
        // to canonical velocities: forces now, then the closing half kick
        TRY(lists_now(s));
        CUDA_TRY(cudaMemsetAsync(s->arena.hex, 0, sizeof(Exchange), s->stream));
        CUDA_TRY(launch_canon_force(s->arena, s->list_map, s->shifted_force, kKick, s->stream));
        s->box.canonical = 1u;
    } else if (!on && s->exchange) {
        CUDA_TRY(launch_half_kick_back(s->arena, s->stream));
        s->box.canonical = 0u;
        for (int k = 0; k < 4; k++) s->box.hex_slabs[k] = 0.0f;
        s->box.hex_energy = 0.0;
    }
    s->exchange = on;
    return push_box(s);
}

// lennard_jones.rs:948-952: the energy moved per step (its f32 value) over 2 A dt.
// Not in the reference, which bins only when the lists rebuild: rebuild the
// cell grid (bin, scan, scatter, per-cell sort) on every step as well, the
// lists still on the skin / 2 trigger. The trajectory is the same to the bit;
// only the work per step changes. A single box only.
vlj_status vlj_set_grid_every_step(vlj_sim* s, int on) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (!s->replicas.empty()) return fail(VLJ_NOT_ENABLED, "grid every step is for a single box");
    const bool want = on != 0;
    if (want == s->grid_every_step) return VLJ_OK;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    sim_drop_step_graphs(s);
    const uint32_t flag = want ? 1u : 0u;
    CUDA_TRY(cudaMemcpyAsync(&s->arena.glob->grid_every_step, &flag, sizeof flag,
                             cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->grid_every_step = want;
    return VLJ_OK;
}

vlj_status vlj_set_list_growth(vlj_sim* s, int on) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    s->list_growth = on != 0;
    if (!s->list_growth) s->grow_pending = false;
    return VLJ_OK;
}

vlj_status vlj_heat_flux(const vlj_sim* s, int* has, double* flux) {
    if (!s || !has || !flux) return fail(VLJ_INVALID_ARG, "null argument");
    *has = s->exchange ? 1 : 0;
    *flux = s->exchange ? s->box.hex_energy / (2.0 * s->box.box[0] * s->box.box[1] * s->settings.dt)
                        : 0.0;
    return VLJ_OK;
}

vlj_status vlj_debug_grid_info(vlj_sim* s, vlj_grid_info* info) {
    if (!s || !info) return fail(VLJ_INVALID_ARG, "null argument");
    Control c;
    CUDA_TRY(cudaMemcpyAsync(&c, s->arena.ctrl, sizeof c, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < 3; k++) {
        info->cells[k] = s->box.cells[k];
        info->cell_size[k] = s->box.cell_size_f[k];
    }
    info->total_cells = s->box.total_cells;
    info->capacity = s->box.capacity;
    info->segment = s->arena.seg;
    info->rebuilds = c.rebuilds;
    info->reorder_every = s->box.reorder_every;
    info->list_r2 = s->box.list_r2;
    return VLJ_OK;
}

vlj_status vlj_debug_read_grid(vlj_sim* s, uint32_t* sorted, uint32_t* cell_start,
                               uint32_t* cell_of_slot, uint32_t* ids, uint32_t* list_count,
                               uint32_t* list, double* pos, double* vel_stored) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    const size_t n = s->n, seg = s->arena.seg, cap = s->box.capacity;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    auto get = [&](void* dst, const void* src, size_t bytes) -> vlj_status {
        if (!dst) return VLJ_OK;
        CUDA_TRY(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
        return VLJ_OK;
    };
    TRY(get(sorted, s->arena.sorted, sizeof(uint32_t) * n));
    TRY(get(cell_start, s->arena.cell_start, sizeof(uint32_t) * (s->box.total_cells + 1)));
    TRY(get(cell_of_slot, s->arena.cell_of_slot, sizeof(uint32_t) * n));
    TRY(get(ids, s->arena.id, sizeof(uint32_t) * n));
    TRY(get(list_count, s->arena.list_count, sizeof(uint32_t) * n));
    if (list) {
        const size_t rows = (cap + 3) / 4;
        std::vector<uint32_t> t(seg * rows * 4);
        TRY(get(t.data(), s->arena.list, sizeof(uint32_t) * t.size()));
        for (size_t i = 0; i < n; i++)
            for (size_t k = 0; k < cap; k++) list[i * cap + k] = t[((k / 4) * seg + i) * 4 + k % 4];
    }
    if (pos || vel_stored) {
        std::vector<double> x(3 * seg), v(3 * seg);
        TRY(get(x.data(), s->arena.x, sizeof(double) * 3 * seg));
        TRY(get(v.data(), s->arena.v, sizeof(double) * 3 * seg));
        for (size_t i = 0; i < n; i++)
            for (int k = 0; k < 3; k++) {
                if (pos) pos[3 * i + k] = x[k * seg + i];
                if (vel_stored) vel_stored[3 * i + k] = v[k * seg + i];
            }
    }
    return VLJ_OK;
}

vlj_status vlj_debug_force_rebuild(vlj_sim* s) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    uint32_t one = 1u;
    CUDA_TRY(cudaMemcpyAsync(&s->arena.ctrl[0].forced, &one, sizeof one, cudaMemcpyHostToDevice,
                             s->stream));
    TRY(lists_now(s));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return VLJ_OK;
}

vlj_status vlj_debug_read_partials(vlj_sim* s, float* pe_half, float* w_half, int64_t* raw) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (pe_half)
        CUDA_TRY(cudaMemcpy(pe_half, s->arena.pe_half, sizeof(float) * 2 * s->n,
                            cudaMemcpyDeviceToHost));
    if (w_half)
        CUDA_TRY(cudaMemcpy(w_half, s->arena.w_half, sizeof(float) * 2 * s->n,
                            cudaMemcpyDeviceToHost));
    if (raw)
        CUDA_TRY(cudaMemcpy(raw, s->arena.accum, sizeof(int64_t) * kSlots, cudaMemcpyDeviceToHost));
    return VLJ_OK;
}

vlj_status vlj_debug_read_vel4(vlj_sim* s, float* out) {
    if (!s || !out) return fail(VLJ_INVALID_ARG, "null argument");
    const size_t n = s->n;
    std::vector<float4> v(n);
    std::vector<uint32_t> id(n);
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    CUDA_TRY(cudaMemcpy(v.data(), s->arena.vel4, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(id.data(), s->arena.id, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
    for (size_t slot = 0; slot < n; slot++) {
        if (id[slot] >= n) return fail(VLJ_CUDA_ERROR, "corrupt particle id %u", id[slot]);
        float* o = out + 4 * (size_t)id[slot];
        o[0] = v[slot].x;
        o[1] = v[slot].y;
        o[2] = v[slot].z;
        o[3] = v[slot].w;
    }
    return VLJ_OK;
}

vlj_status vlj_debug_set_graphs(vlj_sim* s, int on) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    s->use_graphs = on != 0;
    return VLJ_OK;
}

vlj_status vlj_debug_kernel_timing(vlj_sim* s, int on) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->timing = on != 0;
    s->ev_used = 0;
    return VLJ_OK;
}

vlj_status vlj_debug_kernel_time(vlj_sim* s, double* total_ms, uint64_t* launches_out) {
    if (!s || !total_ms || !launches_out) return fail(VLJ_INVALID_ARG, "null argument");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    double total = 0.0;
    for (size_t k = 0; k < s->ev_used; k++) {
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, s->ev_start[k], s->ev_end[k]));
        total += ms;
    }
    *total_ms = total;
    *launches_out = s->ev_used;
    s->ev_used = 0;
    return VLJ_OK;
}

vlj_status vlj_debug_kernels_executed(vlj_sim* s, uint64_t* n) {
    if (!s || !n) return fail(VLJ_INVALID_ARG, "null argument");
    Global g;
    CUDA_TRY(cudaMemcpyAsync(&g, s->arena.glob, sizeof g, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    *n = g.kernels;
    return VLJ_OK;
}

vlj_status vlj_debug_fp32_peak(double* tflops) {
    if (!tflops) return fail(VLJ_INVALID_ARG, "null argument");
    int dev = 0, sms = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t st;
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    float* out = nullptr;
    const int blocks = sms * 8, iters = 8192;
    CUDA_TRY(cudaMalloc(&out, sizeof(float) * blocks));
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    double best = 0.0;
    for (int rep = 0; rep < 6; rep++) {
        CUDA_TRY(cudaEventRecord(a, st));
        CUDA_TRY(launch_fp32_peak(out, blocks, iters, st));
        CUDA_TRY(cudaEventRecord(b, st));
        CUDA_TRY(cudaEventSynchronize(b));
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
        double flops = 2.0 * 8.0 * (double)iters * (double)blocks * (double)kBlock;
        if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    cudaStreamDestroy(st);
    *tflops = best;
    return VLJ_OK;
}

vlj_status vlj_debug_set_tiles(vlj_sim* s, int on) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    const bool want = on != 0;
    if (want == s->tiles_on) return VLJ_OK;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    sim_drop_step_graphs(s);
    s->tiles_on = want;
    return VLJ_OK;
}

vlj_status vlj_set_tile_cols(vlj_sim* s, uint32_t cols) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (!s->replicas.empty()) return fail(VLJ_INVALID_ARG, "cell tiles are for a single box");
    if (cols > s->box.cells[0])
        return fail(VLJ_INVALID_ARG, "at most %u bricks per x-row (cells along x)", s->box.cells[0]);
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    Arena& a = s->arena;
    Box b = s->box;
    Arena plan = a;
    if (cols == 0u) {
        // per-particle gathers again; the 16-bit lists are no longer built
        b.brick_cols = b.brick_base = 0u;
        plan.bricks = plan.tile_cap = plan.tile_threads = 0u;
        if (a.list16) TRY(free_device(s, a.list16));
        a.list16 = nullptr;
    } else {
        if (!plan_tiles(b, plan, cols))
            return fail(VLJ_INVALID_ARG, "cell tiles need four or more particles per cell on average");
        if (!a.list16)
            TRY(dalloc(s, &a.list16, (size_t)a.seg * 8 * ((b.capacity + 7) / 8)));
    }
    a.bricks = plan.bricks;
    a.tile_cap = plan.tile_cap;
    a.tile_threads = plan.tile_threads;
    s->box = b;
    CUDA_TRY(cudaMemcpy(const_cast<Box*>(a.boxes), &b, sizeof(Box), cudaMemcpyHostToDevice));
    s->tiles_on = cols != 0u;
    // No rebuild here: one out of turn would move the reorder schedule and
    // with it the slot order, the list order and the trajectory's bits. The
    // tile step kernel walks the slot lists until the next scheduled build
    // writes the tiles' 16-bit lists for these bricks.
    const uint32_t zero = 0u;
    CUDA_TRY(cudaMemcpy(&a.glob->tiles_ready, &zero, sizeof zero, cudaMemcpyHostToDevice));
    // the captured graphs hold the old arena
    sim_drop_step_graphs(s);
    if (s->graph_lists) cudaGraphExecDestroy(s->graph_lists);
    s->graph_lists = nullptr;
    return VLJ_OK;
}

vlj_status vlj_debug_set_step_lanes(vlj_sim* s, uint32_t lanes) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (lanes > 2u) return fail(VLJ_INVALID_ARG, "step lanes must be 0 (by grid size), 1 or 2");
    if (lanes == s->arena.step_lanes) return VLJ_OK;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    sim_drop_step_graphs(s);
    s->arena.step_lanes = lanes;
    return VLJ_OK;
}

vlj_status vlj_debug_set_step_threads(vlj_sim* s, uint32_t threads) {
    if (!s) return fail(VLJ_INVALID_ARG, "sim is null");
    if (threads != 64 && threads != 128 && threads != 256)
        return fail(VLJ_INVALID_ARG, "step threads must be 64, 128 or 256");
    if (threads == s->arena.step_threads) return VLJ_OK;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    sim_drop_step_graphs(s);
    s->arena.step_threads = threads;
    return VLJ_OK;
}

vlj_status vlj_debug_tile_info(vlj_sim* s, uint32_t* brick_cols, uint32_t* bricks,
                               uint32_t* tile_cap, uint32_t* threads) {
    if (!s || !brick_cols || !bricks || !tile_cap || !threads)
        return fail(VLJ_INVALID_ARG, "null argument");
    const bool tiles = s->replicas.empty() && s->arena.list16;
    *brick_cols = tiles ? s->box.brick_cols : 0u;
    *bricks = tiles ? s->arena.bricks : 0u;
    *tile_cap = tiles ? s->arena.tile_cap : 0u;
    *threads = tiles ? s->arena.tile_threads : 0u;
    return VLJ_OK;
}

vlj_status vlj_debug_read_tile_lists(vlj_sim* s, uint16_t* out) {
    if (!s || !out) return fail(VLJ_INVALID_ARG, "null argument");
    if (!s->arena.list16) return fail(VLJ_NOT_ENABLED, "this simulation has no cell tiles");
    const size_t rows = (s->box.capacity + 7) / 8;
    CUDA_TRY(cudaMemcpyAsync(out, s->arena.list16, sizeof(uint16_t) * 8 * (size_t)s->arena.seg * rows,
                             cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return VLJ_OK;
}

vlj_status vlj_debug_philox(const uint32_t* ctr, const uint32_t* key, size_t n, uint32_t* out,
                            float* noise) {
    if (!ctr || !key || !out || !noise) return fail(VLJ_INVALID_ARG, "null argument");
    if (n == 0 || n > (1u << 24)) return fail(VLJ_INVALID_ARG, "n must be in 1 .. 2^24");
    cudaStream_t st;
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    uint4 *d_ctr = nullptr, *d_out = nullptr;
    uint2* d_key = nullptr;
    float4* d_noise = nullptr;
    cudaError_t e = cudaMalloc(&d_ctr, sizeof(uint4) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_key, sizeof(uint2) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(uint4) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_noise, sizeof(float4) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ctr, ctr, sizeof(uint4) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_key, key, sizeof(uint2) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_philox_check(d_ctr, d_key, (uint32_t)n, d_out, d_noise, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, sizeof(uint4) * n, cudaMemcpyDeviceToHost, st);
    std::vector<float4> nz(e == cudaSuccess ? n : 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(nz.data(), d_noise, sizeof(float4) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_ctr);
    cudaFree(d_key);
    cudaFree(d_out);
    cudaFree(d_noise);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return fail(VLJ_CUDA_ERROR, "debug_philox: %s", cudaGetErrorString(e));
    for (size_t k = 0; k < n; k++) {
        noise[3 * k] = nz[k].x;
        noise[3 * k + 1] = nz[k].y;
        noise[3 * k + 2] = nz[k].z;
    }
    return VLJ_OK;
}

vlj_status vlj_debug_launches(uint64_t* n) {
    if (!n) return fail(VLJ_INVALID_ARG, "null argument");
    *n = launches();
    return VLJ_OK;
}

}  // extern "C"

// ---- allocation and step enqueue (shared with the graph path) ----
namespace vlj {

// The 2D tensor map the force kernels stage list rows through: the list seen
// as u64 pairs of entries, inner dimension 2 * seg (a row holds four entries
// of every slot), outer one row per four list entries; box kTileRows rows of
// kForceThreads slots (2 * kForceThreads <= 256 elements, TMA's box limit).
// Row stride 16 * seg bytes (seg is a multiple of 16, so 16-byte aligned as
// TMA needs).
vlj_status make_list_map(const Arena& a, uint32_t rows, CUtensorMap* out) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn)
            return fail(VLJ_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)a.seg * 2u, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)a.seg * 16u};
    const cuuint32_t box[2] = {(cuuint32_t)kForceThreads * 2u, (cuuint32_t)kTileRows};
    const cuuint32_t estrides[2] = {1u, 1u};
    CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, a.list, dims, strides, box, estrides,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VLJ_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return VLJ_OK;
}

// VLJ_TIMEOUT when a kernel recorded a fault (a TMA tile that never arrived).
vlj_status check_fault(vlj_sim* s) {
    Global g;
    CUDA_TRY(cudaMemcpyAsync(&g, s->arena.glob, sizeof g, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (g.fault == kFaultTmaTimeout)
        return fail(VLJ_TIMEOUT, "a list tile did not arrive within the wait limit");
    if (g.fault) return fail(VLJ_CUDA_ERROR, "kernel fault code %u", g.fault);
    return VLJ_OK;
}

vlj_status sim_lists_now(vlj_sim* s) { return lists_now(s); }

// Cell tiles for the step kernel of a single box (tile_step_kernel), when
// VLJ_TILES=1 at creation: bricks of whole cells along x sized for about 112
// home particles at the box's occupancy (its mean, or 0.9 particles per unit
// volume if that is more: a liquid region in a box that is mostly vapour),
// one block each; a tile holds nine rows of the brick's cells and one more on
// each side, with 30 % room for density fluctuations (bricks beyond it take
// the slot list). Never in dilute boxes (under four particles per cell on
// average), where each particle's few neighbours cost little to gather. Off
// by default: on the 256,000-atom box the tiles' shared-memory gathers (about
// 11 bank wavefronts per warp-wide 16-byte load) and their staging measured
// 75-88 us a step against 51 us for the per-particle gathers through L1.
// want_cols: the bricks per x-row, or 0 for the size above (VLJ_TILE_COLS
// at creation, vlj_set_tile_cols at run time).
static bool plan_tiles(Box& b, Arena& a, uint32_t want_cols) {
    b.brick_cols = 0u;
    b.brick_base = 0u;
    a.bricks = a.tile_cap = a.tile_threads = 0u;
    const double cells = (double)b.total_cells;
    const double mean = (double)b.n / cells;
    if (mean < 4.0) return false;
    const double occupancy = std::max(mean, 0.9 * b.box[0] * b.box[1] * b.box[2] / cells);
    const uint32_t nx = b.cells[0];
    const double width = std::max(1.0, std::round(112.0 / occupancy));
    uint32_t cols = (uint32_t)std::ceil((double)nx / width);
    if (want_cols >= 1u) cols = want_cols;
    cols = std::max(1u, std::min(cols, nx));
    // each tile row holds distinct cells: w + 2 <= nx, or one brick per row
    while (cols > 1u && (nx + cols - 1u) / cols + 2u > nx) cols++;
    const uint32_t wmax = (nx + cols - 1u) / cols;
    const uint32_t rx = cols == 1u ? nx : wmax + 2u;
    const double homes = wmax * occupancy;
    uint32_t threads = 32u * (uint32_t)std::ceil(homes / 32.0);
    threads = std::max(64u, std::min(threads, (uint32_t)kBlock));
    uint32_t cap = 32u * (uint32_t)std::ceil(1.3 * 9.0 * rx * occupancy / 32.0);
    cap = std::min(cap, 4096u);  // 64 KB of shared memory at most
    // VLJ_TILE_CAP overrides the capacity (a tuning and testing knob: a small
    // one sends blocks to the slot-list fallback)
    if (const char* c = std::getenv("VLJ_TILE_CAP")) {
        const long v = std::strtol(c, nullptr, 10);
        if (v >= 16 && v <= 4096) cap = (uint32_t)v;
    }
    b.brick_cols = cols;
    a.bricks = cols * b.cells[1] * b.cells[2];
    a.tile_cap = cap;
    a.tile_threads = threads;
    return true;
}

vlj_status sim_allocate(vlj_sim* s, void* stream) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    s->device = dev;
    if (stream) {
        s->stream = static_cast<cudaStream_t>(stream);
        s->own_stream = false;
    } else {
        CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->own_stream = true;
    }
    Arena& a = s->arena;
    std::memset(&a, 0, sizeof a);
    // boxes own consecutive runs of slots and cells
    const bool batched = !s->replicas.empty();
    std::vector<Box> boxes = batched ? s->replicas : std::vector<Box>{s->box};
    uint64_t slots = 0, cells = 0;
    uint32_t cap = 0;
    for (Box& b : boxes) {
        b.first = (uint32_t)slots;
        b.cell_base = (uint32_t)cells;
        slots += b.n;
        cells += b.total_cells;
        cap = std::max(cap, b.capacity);
    }
    if (slots >= (1ull << 30)) return fail(VLJ_INVALID_ARG, "at most 2^30 - 1 particles in all");
    // work-list entries are cell * 8 + part
    if (cells >= (1ull << 29)) return fail(VLJ_INVALID_ARG, "too many cells in all boxes");
    if (batched)
        s->replicas = boxes;
    else
        s->box = boxes[0];
    const uint32_t n = (uint32_t)slots;
    const uint32_t seg = (n + 15u) / 16u * 16u;  // lennard_jones.rs:470
    s->n = n;
    a.nboxes = (uint32_t)boxes.size();
    a.nslots = n;
    a.seg = seg;
    a.step_threads = kForceThreads;
    a.ncells = (uint32_t)cells;
    Box* d_box = nullptr;
    TRY(dalloc(s, &d_box, boxes.size()));
    a.boxes = d_box;
    TRY(dalloc(s, &a.ctrl, boxes.size()));
    TRY(dalloc(s, &a.glob, 1));
    if (batched) {
        std::vector<uint32_t> of_slot(seg, 0u), of_cell(a.ncells);
        for (uint32_t b = 0; b < a.nboxes; b++) {
            std::fill(of_slot.begin() + boxes[b].first, of_slot.begin() + boxes[b].first + boxes[b].n, b);
            std::fill(of_cell.begin() + boxes[b].cell_base,
                      of_cell.begin() + boxes[b].cell_base + boxes[b].total_cells, b);
        }
        uint32_t *d_slot = nullptr, *d_cell = nullptr;
        TRY(dalloc(s, &d_slot, seg));
        TRY(dalloc(s, &d_cell, a.ncells));
        CUDA_TRY(cudaMemcpy(d_slot, of_slot.data(), sizeof(uint32_t) * seg, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(d_cell, of_cell.data(), sizeof(uint32_t) * a.ncells,
                            cudaMemcpyHostToDevice));
        a.box_of_slot = d_slot;
        a.box_of_cell = d_cell;
    }
    TRY(dalloc(s, &a.x, 3 * (size_t)seg));
    TRY(dalloc(s, &a.v, 3 * (size_t)seg));
    TRY(dalloc(s, &a.id, seg));
    TRY(dalloc(s, &a.cache[0], seg));
    TRY(dalloc(s, &a.cache[1], seg));
    TRY(dalloc(s, &a.snap, seg));
    TRY(dalloc(s, &a.cell_of_slot, seg));
    TRY(dalloc(s, &a.sorted, seg));
    TRY(dalloc(s, &a.cell_start, (size_t)a.ncells + 1));
    TRY(dalloc(s, &a.count, a.ncells));
    {
        // room for every part of every cell: kMaxParts per cell of a narrow box
        size_t cap = 0;
        for (const Box& b : boxes) {
            const bool narrow = b.cells[0] < 5u || b.cells[1] < 5u || b.cells[2] < 5u;
            cap += (size_t)b.total_cells * (narrow ? kMaxParts : 1u);
        }
        if (cap >= (1ull << 32)) return fail(VLJ_INVALID_ARG, "too many cells in all boxes");
        a.work_cap = (uint32_t)cap;
        TRY(dalloc(s, &a.work, cap));
    }
    TRY(dalloc(s, &a.rb_box, boxes.size()));
    TRY(dalloc(s, &a.rb_first, boxes.size() + 1));
    TRY(dalloc(s, &a.list_count, seg));
    TRY(dalloc(s, &a.list, (size_t)seg * 4 * ((cap + 3) / 4)));
    // VLJ_TILES=1: cell tiles from creation on, VLJ_TILE_COLS bricks per x-row
    const char* tiles_env = std::getenv("VLJ_TILES");
    uint32_t env_cols = 0u;
    if (const char* c = std::getenv("VLJ_TILE_COLS")) {
        const long v = std::strtol(c, nullptr, 10);
        if (v >= 1 && v <= 4096) env_cols = (uint32_t)v;
    }
    if (!batched && tiles_env && tiles_env[0] == '1' && plan_tiles(s->box, a, env_cols)) {
        TRY(dalloc(s, &a.list16, (size_t)seg * 8 * ((cap + 7) / 8)));
        boxes[0] = s->box;
    }
    TRY(dalloc(s, &a.block_rows, ((size_t)seg + kForceThreads - 1) / kForceThreads));
    TRY(make_list_map(a, (cap + 3) / 4, &s->list_map));
    TRY(dalloc(s, &a.aos, 6 * (size_t)seg));
    TRY(dalloc(s, &a.sx, 3 * (size_t)seg));
    TRY(dalloc(s, &a.sv, 3 * (size_t)seg));
    TRY(dalloc(s, &a.sid, seg));
    TRY(dalloc(s, &a.scell, seg));
    TRY(dalloc(s, &a.accum, (size_t)kSlots * boxes.size()));
    TRY(dalloc(s, &a.nh, boxes.size()));
    TRY(dalloc(s, &a.hex, 1));
    TRY(dalloc(s, &a.acc, seg));
    TRY(dalloc(s, &a.pe_half, 2 * (size_t)seg));
    TRY(dalloc(s, &a.w_half, 2 * (size_t)seg));
    TRY(dalloc(s, &a.vel4, seg));
    TRY(dalloc(s, &a.vcanon, 3 * (size_t)seg));
    if (!batched && s->box.profile_bins)
        TRY(dalloc(s, &a.profile, (size_t)s->box.profile_bins * 8 + 3));
    // the last cell of the last box ends at the last slot
    CUDA_TRY(cudaMemcpy(a.cell_start + a.ncells, &n, sizeof n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_box, boxes.data(), sizeof(Box) * boxes.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMallocHost(&s->ring, sizeof(Readback) * kRing));
    CUDA_TRY(cudaMallocHost(&s->pin_x, sizeof(double) * 3 * (size_t)seg));
    CUDA_TRY(cudaMallocHost(&s->pin_v, sizeof(double) * 3 * (size_t)seg));
    CUDA_TRY(cudaMallocHost(&s->pin_id, sizeof(uint32_t) * (size_t)seg));
    std::memset(s->pin_x, 0, sizeof(double) * 3 * (size_t)seg);
    std::memset(s->pin_v, 0, sizeof(double) * 3 * (size_t)seg);
    std::memset(s->pin_id, 0, sizeof(uint32_t) * (size_t)seg);
    CUDA_TRY(cudaStreamCreateWithFlags(&s->capture_stream, cudaStreamNonBlocking));
    for (int k = 0; k < kRing; k++) {
        CUDA_TRY(cudaEventCreateWithFlags(&s->ring_event[k], cudaEventDisableTiming));
        s->ring_busy[k] = false;
    }
    return VLJ_OK;
}

// Ends a capture on `cs`, returning the last captured node in *last.
static vlj_status end_capture(cudaStream_t cs, cudaError_t launched, cudaGraphNode_t* last) {
    cudaStreamCaptureStatus st;
    const cudaGraphNode_t* deps = nullptr;
    size_t n = 0;
    cudaError_t info = cudaStreamGetCaptureInfo(cs, &st, nullptr, nullptr, &deps, &n);
    if (last) *last = (info == cudaSuccess && n == 1) ? deps[0] : nullptr;
    cudaGraph_t out = nullptr;
    cudaError_t end = cudaStreamEndCapture(cs, &out);
    CUDA_TRY(launched);
    CUDA_TRY(info);
    CUDA_TRY(end);
    if (last && !*last) return fail(VLJ_CUDA_ERROR, "graph capture ended with %zu open nodes", n);
    return VLJ_OK;
}

// The arena as the step kernel sees it: without cell tiles while they are
// switched off, or while the cell grid is rebuilt on every step (the tiles
// follow the grid of the last list build, which that mode overwrites).
static Arena step_arena(const vlj_sim* s) {
    Arena a = s->arena;
    if (!s->tiles_on || s->grid_every_step) a.tile_threads = 0;
    return a;
}

// What follows the rebuild in a step: the fused step kernel, or on canonical
// velocities the force pass (and the exchange's apply pass).
static cudaError_t launch_step_tail(vlj_sim* s, cudaStream_t cs) {
    if (!s->canonical()) return launch_step(step_arena(s), s->list_map, s->shifted_force, cs);
    cudaError_t e = launch_canon_force(s->arena, s->list_map, s->shifted_force,
                                       s->nose_hoover ? kNoseHoover : kExchange, cs);
    if (e == cudaSuccess && s->exchange) e = launch_hex_apply(s->arena, cs);
    return e;
}

// A graph of `count` steps: decide -> IF(some box rebuilds){rebuild chain} ->
// step kernel, chained (canonical velocities: begin -> decide -> IF{...} ->
// canon_force [-> hex_apply]). The decide kernel sets the condition on the device, so a step
// with no rebuild launches no rebuild kernel at all.
// With `keep`, a graph of one step whose step kernel takes the next step's
// decision and sets this graph's own condition for its next launch: the
// template graph and the decide node come back through *keep and
// *decide_node (the caller disables the node while that decision stands).
static vlj_status build_graph(vlj_sim* s, uint32_t count, cudaGraphExec_t* out,
                              bool heat = false, cudaGraph_t* keep = nullptr,
                              cudaGraphNode_t* decide_node = nullptr) {
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaGraphCreate(&g, 0));
    struct Guard {
        cudaGraph_t g;
        ~Guard() {
            if (g) cudaGraphDestroy(g);
        }
    } guard{g};
    const bool self_fold = keep && count == 1 && !s->canonical();
    cudaStream_t cs = s->capture_stream;
    const auto mode = cudaStreamCaptureModeThreadLocal;
    // one conditional per step; with the fused step kernel, step k's kernel
    // takes step k + 1's decision, so only the first step launches decide
    const bool fold = !s->canonical();
    std::vector<cudaGraphConditionalHandle> h(count);
    // a condition that a step kernel sets for the graph's next launch keeps
    // its value between launches
    for (uint32_t k = 0; k < count; k++)
        CUDA_TRY(cudaGraphConditionalHandleCreate(&h[k], g, 0,
                                                  self_fold ? 0u : cudaGraphCondAssignDefault));
    cudaGraphNode_t prev = nullptr;
    for (uint32_t k = 0; k < count; k++) {
        cudaGraphNode_t n_decide = nullptr, n_cond = nullptr;
        if (k == 0 || !fold) {
            CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, g, prev ? &prev : nullptr, nullptr,
                                                   prev ? 1 : 0, mode));
            cudaError_t e = cudaSuccess;
            if (s->canonical()) e = launch_begin(s->arena, cs);
            if (e == cudaSuccess) e = launch_decide(s->arena, cs, h[k]);
            TRY(end_capture(cs, e, &n_decide));
            if (self_fold && decide_node) *decide_node = n_decide;
        } else {
            n_decide = prev;  // the previous step kernel decided
        }
        if (s->grid_every_step) {
            // the cell grid on every step, ahead of the conditional lists
            CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, g, &n_decide, nullptr, 1, mode));
            TRY(end_capture(cs, launch_grid(s->arena, cs), &n_decide));
        }
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h[k];
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        CUDA_TRY(cudaGraphAddNode(&n_cond, g, &n_decide, 1, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, mode));
        TRY(end_capture(cs, s->grid_every_step ? launch_lists(s->arena, cs)
                                               : launch_rebuild(s->arena, cs),
                        nullptr));
        CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, g, &n_cond, nullptr, 1, mode));
        cudaError_t e;
        if (fold)
            e = launch_step(step_arena(s), s->list_map, s->shifted_force, cs,
                            k + 1 < count ? (unsigned long long)h[k + 1]
                                          : (self_fold ? (unsigned long long)h[k] : 0ull),
                            heat && k == 0);
        else
            e = launch_step_tail(s, cs);
        TRY(end_capture(cs, e, &prev));
    }
    CUDA_TRY(cudaGraphInstantiate(out, g, 0));
    if (self_fold) {
        *keep = g;
        guard.g = nullptr;
    }
    return VLJ_OK;
}

vlj_status sim_launch_lists_graph(vlj_sim* s) {
    if (!s->graph_lists) {
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaGraphCreate(&g, 0));
        struct Guard {
            cudaGraph_t g;
            ~Guard() { cudaGraphDestroy(g); }
        } guard{g};
        cudaStream_t cs = s->capture_stream;
        const auto mode = cudaStreamCaptureModeThreadLocal;
        cudaGraphConditionalHandle h;
        CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
        cudaGraphNode_t n_decide = nullptr, n_cond = nullptr;
        CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, mode));
        TRY(end_capture(cs, launch_decide(s->arena, cs, h), &n_decide));
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        CUDA_TRY(cudaGraphAddNode(&n_cond, g, &n_decide, 1, &cp));
        CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, cp.conditional.phGraph_out[0], nullptr, nullptr,
                                               0, mode));
        TRY(end_capture(cs, launch_rebuild(s->arena, cs), nullptr));
        CUDA_TRY(cudaGraphInstantiate(&s->graph_lists, g, 0));
    }
    CUDA_TRY(cudaGraphLaunch(s->graph_lists, s->stream));
    return VLJ_OK;
}

static vlj_status step_direct(vlj_sim* s, bool heat = false) {
    s->one_ready = false;
    if (s->canonical()) {
        CUDA_TRY(launch_begin(s->arena, s->stream));
        CUDA_TRY(launch_decide(s->arena, s->stream, 0));
        CUDA_TRY(launch_rebuild(s->arena, s->stream));
        CUDA_TRY(launch_step_tail(s, s->stream));
        return VLJ_OK;
    }
    CUDA_TRY(launch_decide(s->arena, s->stream, 0));
    CUDA_TRY(launch_rebuild(s->arena, s->stream));
    if (s->timing) {
        if (s->ev_used == s->ev_start.size()) {
            cudaEvent_t a, b;
            CUDA_TRY(cudaEventCreate(&a));
            CUDA_TRY(cudaEventCreate(&b));
            s->ev_start.push_back(a);
            s->ev_end.push_back(b);
        }
        CUDA_TRY(cudaEventRecord(s->ev_start[s->ev_used], s->stream));
        CUDA_TRY(launch_step(step_arena(s), s->list_map, s->shifted_force, s->stream, 0, heat));
        CUDA_TRY(cudaEventRecord(s->ev_end[s->ev_used], s->stream));
        s->ev_used++;
    } else {
        CUDA_TRY(launch_step(step_arena(s), s->list_map, s->shifted_force, s->stream, 0, heat));
    }
    return VLJ_OK;
}

vlj_status sim_enqueue_steps(vlj_sim* s, uint32_t steps) {
    if (steps > 0 && s->heat_pending) {
        // the first step's force pass takes the requested heat-current sample
        if (s->timing || !s->use_graphs) {
            TRY(step_direct(s, true));
        } else {
            if (!s->graph_one_heat) TRY(build_graph(s, 1, &s->graph_one_heat, true));
            CUDA_TRY(cudaGraphLaunch(s->graph_one_heat, s->stream));
            s->one_ready = false;
        }
        s->heat_pending = false;
        steps -= 1;
    }
    if (s->timing || !s->use_graphs) {
        for (uint32_t k = 0; k < steps; k++) TRY(step_direct(s));
        return VLJ_OK;
    }
    if (!s->graph_chunk) TRY(build_graph(s, kGraphChunk, &s->graph_chunk));
    if (!s->graph_one) {
        s->one_decide = nullptr;
        TRY(build_graph(s, 1, &s->graph_one, false, &s->graph_one_tmpl, &s->one_decide));
        s->one_decide_on = true;
        s->one_ready = false;
    }
    for (; steps >= kGraphChunk; steps -= kGraphChunk) {
        CUDA_TRY(cudaGraphLaunch(s->graph_chunk, s->stream));
        s->one_ready = false;  // the chunk's last step leaves the decision open
    }
    for (; steps > 0; steps--) {
        if (s->one_decide) {
            // the previous step (graph_one's) decided this one already
            const bool need = !s->one_ready;
            if (need != s->one_decide_on) {
                CUDA_TRY(cudaGraphNodeSetEnabled(s->graph_one, s->one_decide, need ? 1u : 0u));
                s->one_decide_on = need;
            }
        }
        CUDA_TRY(cudaGraphLaunch(s->graph_one, s->stream));
        s->one_ready = s->one_decide != nullptr;
    }
    return VLJ_OK;
}

vlj_status sim_flush_heat(vlj_sim* s) {
    if (!s->heat_pending) return VLJ_OK;
    s->heat_pending = false;
    TRY(lists_now(s));
    CUDA_TRY(launch_heat_current(s->arena, s->shifted_force, s->series_samples - 1u, s->stream));
    return VLJ_OK;
}

// Frees device allocation `p` (one of s->allocations).
static vlj_status free_device(vlj_sim* s, void* p) {
    for (size_t k = 0; k < s->allocations.size(); k++)
        if (s->allocations[k] == p) {
            s->allocations.erase(s->allocations.begin() + (long)k);
            CUDA_TRY(cudaFree(p));
            return VLJ_OK;
        }
    return fail(VLJ_INVALID_ARG, "not an allocation of this sim");
}

// Replaces device allocation `old` (one of s->allocations) by a new one of
// `bytes` bytes.
static vlj_status realloc_device(vlj_sim* s, void** ptr, size_t bytes) {
    void* q = nullptr;
    CUDA_TRY(cudaMalloc(&q, bytes));
    CUDA_TRY(cudaMemset(q, 0, bytes));
    for (void*& p : s->allocations)
        if (p == *ptr) {
            cudaFree(p);
            p = q;
            *ptr = q;
            return VLJ_OK;
        }
    cudaFree(q);
    return fail(VLJ_CUDA_ERROR, "list allocation not found");
}

bool list_growth_default() {
    const char* env = std::getenv("VLJ_LIST_GROWTH");
    return !(env && env[0] == '0');
}

vlj_status sim_grow_lists(vlj_sim* s, bool* grew) {
    *grew = false;
    s->grow_pending = false;
    if (!s->list_growth) return VLJ_OK;
    Arena& a = s->arena;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    std::vector<Control> c(a.nboxes);
    CUDA_TRY(cudaMemcpy(c.data(), a.ctrl, sizeof(Control) * c.size(), cudaMemcpyDeviceToHost));
    const bool batched = !s->replicas.empty();
    std::vector<Box> single;
    if (!batched) single.push_back(s->box);
    std::vector<Box>& boxes = batched ? s->replicas : single;
    uint32_t old_max = 0, new_max = 0;
    bool any = false;
    for (size_t b = 0; b < boxes.size(); b++) {
        old_max = std::max(old_max, boxes[b].capacity);
        if (c[b].overflow > boxes[b].capacity) {
            const uint32_t want = (uint32_t)std::ceil(1.25 * (double)c[b].overflow);
            boxes[b].capacity = (want + 7u) / 8u * 8u;
            c[b].overflow = 0u;
            c[b].forced = 1u;
            any = true;
        }
        new_max = std::max(new_max, boxes[b].capacity);
    }
    if (!any) return VLJ_OK;
    const size_t seg = a.seg;
    if ((new_max + 3u) / 4u > (old_max + 3u) / 4u) {
        TRY(realloc_device(s, reinterpret_cast<void**>(&a.list),
                           sizeof(uint32_t) * seg * 4 * ((new_max + 3) / 4)));
        TRY(make_list_map(a, (new_max + 3) / 4, &s->list_map));
    }
    if (a.list16 && (new_max + 7u) / 8u > (old_max + 7u) / 8u)
        TRY(realloc_device(s, reinterpret_cast<void**>(&a.list16),
                           sizeof(uint16_t) * seg * 8 * ((new_max + 7) / 8)));
    if (!batched) s->box = boxes[0];
    CUDA_TRY(cudaMemcpy(const_cast<Box*>(a.boxes), boxes.data(), sizeof(Box) * boxes.size(),
                        cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(a.ctrl, c.data(), sizeof(Control) * c.size(), cudaMemcpyHostToDevice));
    // the captured graphs hold the old arena
    sim_drop_step_graphs(s);
    if (s->graph_lists) cudaGraphExecDestroy(s->graph_lists);
    s->graph_lists = nullptr;
    s->list_grows += 1;
    *grew = true;
    // the forced rebuild now, so what follows reads full lists
    return lists_now(s);
}

void sim_drop_step_graphs(vlj_sim* s) {
    if (s->graph_chunk) cudaGraphExecDestroy(s->graph_chunk);
    if (s->graph_one) cudaGraphExecDestroy(s->graph_one);
    if (s->graph_one_tmpl) cudaGraphDestroy(s->graph_one_tmpl);
    s->graph_one_tmpl = nullptr;
    s->one_decide = nullptr;
    s->one_ready = false;
    if (s->graph_one_heat) cudaGraphExecDestroy(s->graph_one_heat);
    s->graph_chunk = s->graph_one = s->graph_one_heat = nullptr;
}

}  // namespace vlj
