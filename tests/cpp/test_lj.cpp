// The reference's own LennardJones tests restated in C++ against the C++
// mirror in include/virial_lj.hpp, so that they read as the Rust ones do.
//
//   test_lj host   host-only entry points and error behaviour (no GPU needed)
//   test_lj gpu    the GPU tests as well
//
// Each test names the reference test it restates (crates/virial-particles/
// tests/*.rs, src/lennard_jones.rs). Prints one line per test; exits non-zero
// on the first failure.

#include "virial_lj.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <tuple>

using namespace virial_lj;

namespace {

int failures = 0;

#define EXPECT(cond, ...)                                                         \
    do {                                                                          \
        if (!(cond)) {                                                            \
            std::fprintf(stderr, "%s:%d: expectation failed: %s: ", __FILE__,     \
                         __LINE__, #cond);                                        \
            std::fprintf(stderr, __VA_ARGS__);                                    \
            std::fprintf(stderr, "\n");                                           \
            throw std::logic_error("expectation failed");                         \
        }                                                                         \
    } while (0)

template <class F>
vlj_status status_of(F&& f) {
    try {
        f();
    } catch (const Error& e) {
        return e.status;
    }
    return VLJ_OK;
}

void run(const char* name, const std::function<void()>& test) {
    try {
        test();
        std::printf("ok   %s\n", name);
    } catch (const std::exception& e) {
        std::printf("FAIL %s (%s)\n", name, e.what());
        failures++;
    }
    std::fflush(stdout);
}

double rel(double a, double b) { return std::fabs((a - b) / b); }

// The jitter of the reference tests (thermodynamics.rs:60-68,
// coexistence.rs:79-91): xorshift64 (13, 7, 17) from 99, uniform in
// [-0.15, 0.15) per coordinate.
void jitter(std::vector<Particle>& particles) {
    uint64_t s = 99;
    for (Particle& p : particles)
        for (int k = 0; k < 3; k++) {
            s ^= s << 13;
            s ^= s >> 7;
            s ^= s << 17;
            p.pos[k] += ((double)(s >> 11) / (double)(1ull << 53) - 0.5) * 0.3;
        }
}

// Pair potential and r . F in f64, shifted as the step shifts it
// (coexistence.rs:39-55).
std::pair<double, double> pair_terms(double r2, double cutoff, bool shifted_force) {
    auto lj = [](double q) {
        const double s6 = 1.0 / (q * q * q);
        return std::make_pair(4.0 * (s6 * s6 - s6), 24.0 * (2.0 * s6 * s6 - s6));
    };
    const auto [u, rf] = lj(r2);
    const auto [uc, rfc] = lj(cutoff * cutoff);
    if (!shifted_force) return {u - uc, rf};
    const double r = std::sqrt(r2), fc = rfc / cutoff;
    return {u - uc + (r - cutoff) * fc, rf - r * fc};
}

// Potential energy and virial tensor diagonal over all pairs, nearest image
// in a rectangular box, f64 (coexistence.rs:57-77). Positions are wrapped
// into the box first, as the reference tests wrap them (rem_euclid).
std::pair<double, std::array<double, 3>> all_pairs(const std::vector<Particle>& particles,
                                                   const std::array<double, 3>& size,
                                                   double cutoff, bool shifted_force) {
    std::vector<std::array<double, 3>> x(particles.size());
    for (size_t i = 0; i < particles.size(); i++)
        for (int k = 0; k < 3; k++) {
            double w = std::fmod(particles[i].pos[k], size[k]);
            x[i][k] = w < 0.0 ? w + size[k] : w;
        }
    double pe = 0.0;
    std::array<double, 3> w{};
    for (size_t i = 0; i < x.size(); i++)
        for (size_t j = i + 1; j < x.size(); j++) {
            double d[3], r2 = 0.0;
            for (int k = 0; k < 3; k++) {
                const double t = x[j][k] - x[i][k];
                d[k] = t - size[k] * std::nearbyint(t / size[k]);
                r2 += d[k] * d[k];
            }
            if (r2 < cutoff * cutoff) {
                const auto [u, rf] = pair_terms(r2, cutoff, shifted_force);
                pe += u;
                for (int k = 0; k < 3; k++) w[k] += d[k] * d[k] * rf / r2;
            }
        }
    return {pe, w};
}

Settings coexistence_settings(const std::array<double, 3>& size, bool shifted_force,
                              uint32_t bins) {
    Settings s;
    s.box_size = size;
    s.cutoff = 2.5;
    s.dt = 0.005;
    s.thermostat = NoseHoover{0.7, 0.5};
    s.shifted_force = shifted_force;
    s.skin = 0.3;
    s.profile_bins = bins;
    return s;
}

std::vector<uint64_t> bits(const std::vector<Particle>& particles) {
    std::vector<uint64_t> out(particles.size() * 6);
    std::memcpy(out.data(), particles.data(), out.size() * 8);
    return out;
}

uint64_t bits(double x) {
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return b;
}

// ---------------------------------------------------------------- host ----

void lattice_fills_the_box() {
    // lennard_jones.rs:1377-1441: count particles inside the box, zero
    // total momentum
    for (size_t n : {1u, 27u, 1000u, 1001u}) {
        const auto p = lattice(n, 11.0, 1.3, 5);
        EXPECT(p.size() == n, "%zu", p.size());
        double mom[3] = {0, 0, 0};
        for (const Particle& q : p)
            for (int k = 0; k < 3; k++) {
                EXPECT(q.pos[k] >= 0.0 && q.pos[k] < 11.0, "%g", q.pos[k]);
                mom[k] += q.vel[k];
            }
        if (n > 1)
            for (int k = 0; k < 3; k++) EXPECT(std::fabs(mom[k]) < 1e-9 * n, "%g", mom[k]);
    }
    const auto q = lattice_box(2400, {10.0, 10.0, 30.0}, 1.0, 3);
    for (const Particle& p : q) EXPECT(p.pos[2] >= 0.0 && p.pos[2] < 30.0, "%g", p.pos[2]);
}

void bad_arguments_throw() {
    EXPECT(status_of([] { lattice(0, 1.0, 1.0, 1); }) == VLJ_INVALID_ARG, "lattice(0)");
    EXPECT(status_of([] { lattice_box(10, {1.0, -1.0, 1.0}, 1.0, 1); }) == VLJ_INVALID_ARG,
           "negative side");
    try {
        lattice(0, 1.0, 1.0, 1);
    } catch (const Error& e) {
        // the status's name, then the library's message for this failure
        EXPECT(std::string(e.what()).rfind(vlj_status_name(VLJ_INVALID_ARG), 0) == 0 &&
                   std::string(e.what()).find("lattice") != std::string::npos,
               "%s", e.what());
    }
}

void phases_of_two_slabs_across_the_boundary() {
    // lennard_jones.rs:1468-1497: liquid in [0, 10), [25, 40), [50, 60) of a
    // 60-slab profile, vapour elsewhere; interfaces at 10, 25, 40, 50
    Profile p;
    p.samples = 1;
    p.box_size = {1.0, 1.0, 60.0};
    for (int b = 0; b < 60; b++) {
        const bool liquid = b < 10 || (b >= 25 && b < 40) || b >= 50;
        p.slabs.push_back({b + 0.5, liquid ? 0.7 : 0.02, {}, {}, 0.0});
    }
    auto found = p.interfaces(0.36);
    std::sort(found.begin(), found.end());
    EXPECT(found == std::vector<double>({10.0, 25.0, 40.0, 50.0}), "%zu interfaces",
           found.size());
    const auto phases = p.phases(0.36, 4.0);
    auto count = [&](Phase q) { return std::count(phases.begin(), phases.end(), q); };
    EXPECT(count(Phase::Liquid) == 6 + 6 + 7, "%ld", (long)count(Phase::Liquid));
    EXPECT(count(Phase::Interface) == 16, "%ld", (long)count(Phase::Interface));
    const auto density = p.density();
    EXPECT(std::fabs(*p.mean_in(density, phases, Phase::Liquid) - 0.7) < 1e-12, "liquid mean");
    EXPECT(std::fabs(*p.mean_in(density, phases, Phase::Vapour) - 0.02) < 1e-12, "vapour mean");
    Profile flat;
    flat.box_size = {1.0, 1.0, 8.0};
    for (int b = 0; b < 8; b++) flat.slabs.push_back({b + 0.5, 0.3, {}, {}, 0.0});
    const auto flat_phases = flat.phases(0.36, 4.0);
    for (Phase q : flat_phases) EXPECT(q == Phase::Between, "flat profile");
    EXPECT(!flat.mean_in(flat.density(), flat_phases, Phase::Liquid), "no liquid slab");
}

void no_device_is_an_error() {
    int devices = 0;
    check(vlj_device_count(&devices));
    if (devices > 0) return;
    const auto p = lattice(1000, 11.0, 1.0, 3);
    Settings s;
    s.box_size = {11.0, 11.0, 11.0};
    EXPECT(status_of([&] { LennardJones sim(p, s); }) == VLJ_NO_DEVICE, "without a device");
}

// ----------------------------------------------------------------- gpu ----

void cell_grid_finds_every_pair() {
    // thermodynamics.rs:55-100 (1e-5 there; 1e-6 here)
    auto particles = lattice(1000, 11.0, 1.0, 3);
    jitter(particles);
    Settings s;
    s.box_size = {11.0, 11.0, 11.0};
    s.dt = 0.002;
    LennardJones sim(particles, s);
    const Measurement m = sim.measure_now();
    const auto [pe, w] = all_pairs(particles, sim.box_size(), 2.5, false);
    const double wsum = w[0] + w[1] + w[2];
    EXPECT(rel(m.potential, pe) < 1e-6, "potential %.10f vs %.10f", m.potential, pe);
    EXPECT(rel(m.virial, wsum) < 1e-6, "virial %.10f vs %.10f", m.virial, wsum);
}

void rectangular_box_matches_all_pairs() {
    // coexistence.rs:93-130 (1e-5 there; 1e-6 here)
    const std::array<double, 3> size = {9.0, 10.5, 14.25};
    auto particles = lattice_box(1000, size, 1.0, 3);
    jitter(particles);
    for (bool shifted_force : {false, true}) {
        LennardJones sim(particles, coexistence_settings(size, shifted_force, 57));
        const Measurement m = sim.measure_now();
        sim.sample_profile_now();
        const Profile profile = sim.read_profile();
        const auto [pe, w] = all_pairs(particles, sim.box_size(), 2.5, shifted_force);
        EXPECT(rel(m.potential, pe) < 1e-6, "potential %.10f vs %.10f", m.potential, pe);
        EXPECT(rel(m.virial, w[0] + w[1] + w[2]) < 1e-6, "virial %.10f", m.virial);
        for (int k = 0; k < 3; k++)
            EXPECT(rel(profile.virial[k], w[k]) < 1e-6, "W_%d %.10f vs %.10f", k,
                   profile.virial[k], w[k]);
    }
}

void profiles_add_up_to_the_whole_box() {
    // coexistence.rs:132-191
    const std::array<double, 3> size = {10.0, 10.0, 30.0};
    auto particles = lattice_box(2400, size, 1.0, 3);
    jitter(particles);
    auto once = [&] {
        LennardJones sim(particles, coexistence_settings(size, true, 120));
        sim.run(200);
        const Measurement m = sim.measure_now();
        sim.sample_profile_now();
        return std::make_pair(m, sim.read_profile());
    };
    const auto [m, p] = once();
    const Profile again = once().second;
    auto words = [](const Profile& q) {
        std::vector<uint64_t> out;
        for (const Slab& s : q.slabs) {
            out.push_back(bits(s.particles));
            out.push_back(bits(s.potential));
            for (int k = 0; k < 3; k++) out.push_back(bits(s.kinetic[k]));
            for (int k = 0; k < 3; k++) out.push_back(bits(s.virial[k]));
        }
        for (int k = 0; k < 3; k++) out.push_back(bits(q.virial[k]));
        return out;
    };
    EXPECT(words(p) == words(again), "profiles differ between runs");
    double count = 0, kinetic = 0, potential = 0;
    std::array<double, 3> slab_virial{};
    for (const Slab& s : p.slabs) {
        count += s.particles;
        potential += s.potential;
        for (int k = 0; k < 3; k++) {
            kinetic += s.kinetic[k];
            slab_virial[k] += s.virial[k];
        }
    }
    EXPECT(count == m.count, "%g of %u particles", count, m.count);
    EXPECT(rel(kinetic, 2.0 * m.kinetic) < 1e-6, "2 KE %.8f vs %.8f", kinetic, 2.0 * m.kinetic);
    EXPECT(rel(potential, m.potential) < 1e-5, "potential %.8f vs %.8f", potential, m.potential);
    EXPECT(rel(p.virial[0] + p.virial[1] + p.virial[2], m.virial) < 1e-5, "virial");
    for (int k = 0; k < 3; k++)
        EXPECT(rel(slab_virial[k], p.virial[k]) < 1e-6, "slab W_%d %.8f vs %.8f", k,
               slab_virial[k], p.virial[k]);
}

void thermostatted_reruns_are_bit_identical() {
    // thermodynamics.rs:295-327
    const auto particles = lattice(2000, 16.0, 1.5, 11);
    Settings s;
    s.box_size = {16.0, 16.0, 16.0};
    s.dt = 0.004;
    s.thermostat = Langevin{1.5, 0.5, 3};
    auto once = [&] {
        LennardJones sim(particles, s);
        sim.run(300);
        const Measurement m = sim.measure_now();
        return std::make_tuple(bits(sim.read_particles()), bits(m.potential), bits(m.virial));
    };
    EXPECT(once() == once(), "states or measurements differ between runs");
}

// Least-squares rate of energy against time and its standard error
// (tests/heat.rs:141-157).
std::pair<double, double> drift(const std::vector<double>& t, const std::vector<double>& e) {
    const double n = (double)t.size();
    double mt = 0.0, me = 0.0;
    for (size_t k = 0; k < t.size(); k++) {
        mt += t[k] / n;
        me += e[k] / n;
    }
    double sxx = 0.0, sxy = 0.0;
    for (size_t k = 0; k < t.size(); k++) {
        sxx += (t[k] - mt) * (t[k] - mt);
        sxy += (t[k] - mt) * (e[k] - me);
    }
    const double rate = sxy / sxx;
    double residual = 0.0;
    for (size_t k = 0; k < t.size(); k++) {
        const double r = e[k] - me - rate * (t[k] - mt);
        residual += r * r;
    }
    return {rate, std::sqrt(residual / (n - 2.0) / sxx)};
}

void heat_exchange_moves_energy_and_keeps_momentum() {
    // tests/heat.rs:159-214
    const std::array<double, 3> size = {9.0, 9.0, 36.0};
    const double dt = 0.002;
    const size_t count = (size_t)std::lround(0.8442 * size[0] * size[1] * size[2]);
    Settings s;
    s.box_size = size;
    s.dt = dt;
    s.shifted_force = true;
    s.profile_bins = 12;
    LennardJones sim(lattice_box(count, size, 1.0, 11), s);
    sim.run(2000);
    const Measurement before = sim.measure_now();
    const double energy = 0.01;
    sim.set_heat_exchange(HeatExchange{{0.0, 3.0}, {18.0, 21.0}, energy});
    std::vector<double> time, total;
    for (int k = 0; k < 200; k++) {
        sim.run(100);
        sim.sample_profile_now();
        const Measurement m = sim.measure_now();
        time.push_back(m.time);
        total.push_back(m.energy());
    }
    const Measurement after = sim.measure_now();
    const auto [rate, error] = drift(time, total);
    const double duration = time.back() - time.front();
    const double moved = energy / dt * duration;
    const auto t = sim.read_profile().temperature();
    EXPECT(std::fabs(rate * duration) < 1e-3 * moved, "energy not conserved: %g +/- %g", rate,
           error);
    for (int k = 0; k < 3; k++)
        EXPECT(std::fabs(after.momentum[k] - before.momentum[k]) < 1e-6 * after.count,
               "momentum changed: %g", after.momentum[k] - before.momentum[k]);
    EXPECT(t[0] > t[6] + 0.04, "hot slab %.4f not hotter than cold slab %.4f", t[0], t[6]);
}

void measurements_arrive_in_order() {
    // lennard_jones.rs:1141-1163, 1194-1260: measure enqueues, poll returns
    // finished measurements oldest first; measure_now equals a polled one
    const auto particles = lattice(1000, 11.0, 1.0, 3);
    Settings s;
    s.box_size = {11.0, 11.0, 11.0};
    LennardJones sim(particles, s);
    std::vector<uint64_t> steps;
    for (int i = 0; i < 3; i++) {
        EXPECT(sim.measure(), "a read-back slot is free");
        sim.step(10);
        sim.after_submit();
    }
    EXPECT(!sim.measure(), "every read-back slot is in flight");
    std::vector<Measurement> got;
    const auto until = std::chrono::steady_clock::now() + std::chrono::seconds(30);
    while (got.size() < 3 && std::chrono::steady_clock::now() < until)
        for (const Measurement& m : sim.poll()) got.push_back(m);
    EXPECT(got.size() == 3, "%zu measurements", got.size());
    for (int i = 0; i < 3; i++) EXPECT(got[i].step == 10u * i, "step %llu", (unsigned long long)got[i].step);
    EXPECT(sim.steps() == 30, "%llu", (unsigned long long)sim.steps());
    EXPECT(std::fabs(sim.time() - 30 * s.dt) < 1e-12, "%g", sim.time());
    const Measurement now = sim.measure_now();
    EXPECT(now.step == 30 && now.count == 1000, "step %llu", (unsigned long long)now.step);
    EXPECT(rel(now.pressure(), (2.0 * now.kinetic + now.virial) / (3.0 * sim.volume())) < 1e-15,
           "pressure");
}

void panics_become_errors() {
    // lennard_jones.rs:458-461 (box below three cells), 907 (drawn
    // temperature needs no setup), 930-933 (set_temperature without a
    // thermostat), 990-991 (heat current not recorded / full), 1178
    // (profiles without bins)
    const auto particles = lattice(1000, 11.0, 1.0, 3);
    Settings s;
    s.box_size = {11.0, 11.0, 11.0};
    {
        Settings small = s;
        small.box_size = {11.0, 11.0, 8.0};
        EXPECT(status_of([&] { LennardJones sim(particles, small); }) == VLJ_BOX_TOO_SMALL,
               "box below three cells");
    }
    LennardJones sim(particles, s);
    EXPECT(!sim.target_temperature(), "no thermostat");
    EXPECT(status_of([&] { sim.set_temperature(1.0); }) == VLJ_NOT_ENABLED, "set_temperature");
    EXPECT(status_of([&] { sim.sample_profile(); }) == VLJ_NOT_ENABLED, "profile bins");
    EXPECT(status_of([&] { sim.sample_heat_current(); }) == VLJ_NOT_ENABLED, "not recorded");
    sim.record_heat_current(2);
    sim.sample_heat_current();
    sim.step(1);
    sim.sample_heat_current();
    EXPECT(status_of([&] { sim.sample_heat_current(); }) == VLJ_FULL, "series full");
    EXPECT(sim.read_heat_current().size() == 2, "two samples");
    sim.set_heat_exchange(HeatExchange{{0.0, 1.0}, {5.0, 6.0}, 1e-3});
    EXPECT(sim.heat_flux().has_value(), "flux with an exchange");
    sim.set_heat_exchange(std::nullopt);
    EXPECT(!sim.heat_flux().has_value(), "no flux without one");
    Settings lv = s;
    lv.thermostat = Langevin{1.0, 1.0, 7};
    LennardJones thermostatted(particles, lv);
    EXPECT(thermostatted.target_temperature() == 1.0, "target");
    thermostatted.set_temperature(0.8);
    EXPECT(thermostatted.target_temperature() == 0.8, "new target");
    EXPECT(status_of([&] {
               thermostatted.set_heat_exchange(HeatExchange{{0.0, 1.0}, {5.0, 6.0}, 1e-3});
           }) == VLJ_NOT_ENABLED,
           "exchange with a thermostat");
    LennardJones moved = std::move(thermostatted);
    moved.run(5);
    EXPECT(moved.steps() == 5, "moved simulation steps");
}

}  // namespace

int main(int argc, char** argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
    run("lattice_fills_the_box", lattice_fills_the_box);
    run("bad_arguments_throw", bad_arguments_throw);
    run("phases_of_two_slabs_across_the_boundary", phases_of_two_slabs_across_the_boundary);
    if (!gpu) {
        run("no_device_is_an_error", no_device_is_an_error);
    } else {
        run("cell_grid_finds_every_pair", cell_grid_finds_every_pair);
        run("rectangular_box_matches_all_pairs", rectangular_box_matches_all_pairs);
        run("profiles_add_up_to_the_whole_box", profiles_add_up_to_the_whole_box);
        run("thermostatted_reruns_are_bit_identical", thermostatted_reruns_are_bit_identical);
        run("heat_exchange_moves_energy_and_keeps_momentum",
            heat_exchange_moves_energy_and_keeps_momentum);
        run("measurements_arrive_in_order", measurements_arrive_in_order);
        run("panics_become_errors", panics_become_errors);
    }
    std::printf("%d failed\n", failures);
    return failures ? 1 : 0;
}
