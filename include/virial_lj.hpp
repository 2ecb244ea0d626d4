/* C++ mirror of virial_particles::lennard_jones (crates/virial-particles/src/
 * lennard_jones.rs) over the C ABI in virial_lj.h: the same types, method
 * names and argument meanings as the reference's Rust API, so a C++ caller
 * (or a test restated from the reference's) reads like the original. Where
 * the reference panics (assert!/expect), this throws virial_lj::Error carrying
 * the vlj_status and the message. Header-only, C++17; link libvirial_lj.so.
 *
 * Differences forced by the boundary: the wgpu device, queue and command
 * encoder become a CUDA stream (or none: the simulation makes its own), so
 * step / measure / sample_profile / sample_heat_current enqueue on that
 * stream and after_submit has nothing to do; positions() and velocities()
 * are device pointers rather than renderer bindings. */
#ifndef VIRIAL_LJ_HPP
#define VIRIAL_LJ_HPP

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <variant>
#include <vector>

#include "virial_lj.h"

namespace virial_lj {

class Error : public std::runtime_error {
public:
    Error(vlj_status status, const std::string& what) : std::runtime_error(what), status(status) {}
    vlj_status status;
};

inline void check(vlj_status s) {
    if (s != VLJ_OK)
        throw Error(s, std::string(vlj_status_name(s)) + ": " + vlj_last_error());
}

/* lennard_jones.rs:25-30: mass 1 */
struct Particle {
    std::array<double, 3> pos;
    std::array<double, 3> vel;
};
static_assert(sizeof(Particle) == sizeof(vlj_particle), "Particle mirrors vlj_particle");

/* lennard_jones.rs:32-61 */
struct Langevin {
    double temperature;
    double friction;
    uint32_t seed;
};
struct NoseHoover {
    double temperature;
    double period;
};
using Thermostat = std::variant<std::monostate, Langevin, NoseHoover>;

/* lennard_jones.rs:63-82 */
struct Settings {
    std::array<double, 3> box_size;
    double cutoff = 2.5;
    double dt = 0.005;
    Thermostat thermostat = std::monostate{};
    bool shifted_force = false;
    double skin = 0.3;
    uint32_t profile_bins = 0;

    vlj_settings c() const {
        vlj_settings s;
        std::memset(&s, 0, sizeof s);
        for (int k = 0; k < 3; k++) s.box_size[k] = box_size[k];
        s.cutoff = cutoff;
        s.dt = dt;
        s.shifted_force = shifted_force ? 1 : 0;
        s.skin = skin;
        s.profile_bins = profile_bins;
        if (auto* l = std::get_if<Langevin>(&thermostat)) {
            s.thermostat.kind = VLJ_THERMOSTAT_LANGEVIN;
            s.thermostat.temperature = l->temperature;
            s.thermostat.friction = l->friction;
            s.thermostat.seed = l->seed;
        } else if (auto* nh = std::get_if<NoseHoover>(&thermostat)) {
            s.thermostat.kind = VLJ_THERMOSTAT_NOSE_HOOVER;
            s.thermostat.temperature = nh->temperature;
            s.thermostat.period = nh->period;
        }
        return s;
    }
};

/* lennard_jones.rs:84-131 */
struct Measurement : vlj_measurement {
    Measurement() { std::memset(static_cast<vlj_measurement*>(this), 0, sizeof(vlj_measurement)); }
    explicit Measurement(const vlj_measurement& m) : vlj_measurement(m) {}
    double energy() const { return kinetic + potential; }
    double extended_energy() const { return energy() + thermostat_energy; }
    /* 2 KE / dof: 3N with a thermostat, 3N - 3 at constant energy */
    double temperature(double dof) const { return 2.0 * kinetic / dof; }
    /* P = (2 KE + W) / (3 V) */
    double pressure() const { return (2.0 * kinetic + virial) / (3.0 * volume); }
};

/* lennard_jones.rs:133-147 */
struct Slab {
    double z, particles;
    std::array<double, 3> kinetic, virial;
    double potential;
};

enum class Phase { Liquid = VLJ_PHASE_LIQUID, Vapour = VLJ_PHASE_VAPOUR,
                   Interface = VLJ_PHASE_INTERFACE, Between = VLJ_PHASE_BETWEEN };

/* lennard_jones.rs:149-280 */
struct Profile {
    uint64_t samples = 0;
    std::array<double, 3> box_size{};
    std::vector<Slab> slabs;
    std::array<double, 3> virial{};

    double slab_volume() const { return box_size[0] * box_size[1] * box_size[2] / slabs.size(); }
    std::vector<double> density() const {
        std::vector<double> d;
        for (const Slab& s : slabs) d.push_back(s.particles / slab_volume());
        return d;
    }
    std::vector<double> temperature() const {
        std::vector<double> t;
        for (const Slab& s : slabs)
            t.push_back(s.particles > 0 ? (s.kinetic[0] + s.kinetic[1] + s.kinetic[2]) /
                                              (3.0 * s.particles)
                                        : std::nan(""));
        return t;
    }
    std::vector<std::array<double, 3>> pressure_tensor() const {
        std::vector<std::array<double, 3>> p;
        for (const Slab& s : slabs)
            p.push_back({(s.kinetic[0] + s.virial[0]) / slab_volume(),
                         (s.kinetic[1] + s.virial[1]) / slab_volume(),
                         (s.kinetic[2] + s.virial[2]) / slab_volume()});
        return p;
    }
    std::array<double, 3> total_pressure_tensor() const {
        const double v = box_size[0] * box_size[1] * box_size[2];
        std::array<double, 3> out{};
        for (int a = 0; a < 3; a++) {
            double k = 0.0;
            for (const Slab& s : slabs) k += s.kinetic[a];
            out[a] = (k + virial[a]) / v;
        }
        return out;
    }
    // Mean of a per-slab quantity over the slabs in `phase` (lennard_jones.rs:262-271);
    // empty when there are none.
    std::optional<double> mean_in(const std::vector<double>& values,
                                  const std::vector<Phase>& phases, Phase phase) const {
        double sum = 0.0, n = 0.0;
        for (size_t k = 0; k < values.size() && k < phases.size(); k++)
            if (phases[k] == phase) {
                sum += values[k];
                n += 1.0;
            }
        return n > 0.0 ? std::optional<double>(sum / n) : std::nullopt;
    }
    double surface_tension() const {
        const auto p = total_pressure_tensor();
        return 0.5 * box_size[2] * (p[2] - 0.5 * (p[0] + p[1]));
    }
    std::vector<double> interfaces(double midpoint) const {
        const auto d = density();
        std::vector<double> out(d.size());
        size_t found = 0;
        check(vlj_profile_interfaces(d.data(), d.size(), box_size[2], midpoint, out.data(),
                                     out.size(), &found));
        out.resize(found);
        return out;
    }
    std::vector<Phase> phases(double midpoint, double margin) const {
        const auto d = density();
        std::vector<int32_t> p(d.size());
        check(vlj_profile_phases(d.data(), d.size(), box_size[2], midpoint, margin, p.data()));
        std::vector<Phase> out;
        for (int32_t x : p) out.push_back(static_cast<Phase>(x));
        return out;
    }
};

/* lennard_jones.rs:375-387 */
struct HeatExchange {
    std::pair<double, double> hot, cold;
    double energy;
};

enum class Drawn { Neighbours = VLJ_DRAWN_NEIGHBOURS, Temperature = VLJ_DRAWN_TEMPERATURE };

/* lennard_jones.rs:334-1375 */
class LennardJones {
public:
    LennardJones(const std::vector<Particle>& particles, const Settings& settings,
                 void* stream = nullptr)
        : bins_(settings.profile_bins), count_((uint32_t)particles.size()) {
        const vlj_settings s = settings.c();
        check(vlj_create(reinterpret_cast<const vlj_particle*>(particles.data()), particles.size(),
                         &s, stream, &sim_));
    }
    ~LennardJones() {
        if (sim_) vlj_destroy(sim_);
    }
    LennardJones(const LennardJones&) = delete;
    LennardJones& operator=(const LennardJones&) = delete;
    LennardJones(LennardJones&& o) noexcept
        : sim_(std::exchange(o.sim_, nullptr)), bins_(o.bins_), count_(o.count_),
          series_(o.series_) {}

    void step(uint32_t steps) { check(vlj_step(sim_, steps)); }
    void run(uint64_t steps) { check(vlj_run(sim_, steps)); }
    bool measure() {
        int accepted = 0;
        check(vlj_measure(sim_, &accepted));
        return accepted != 0;
    }
    void after_submit() {}
    std::vector<Measurement> poll() {
        vlj_measurement buf[8];
        size_t n = 0;
        check(vlj_poll(sim_, buf, 8, &n));
        return std::vector<Measurement>(buf, buf + n);
    }
    Measurement measure_now() {
        vlj_measurement m;
        check(vlj_measure_now(sim_, &m));
        return Measurement(m);
    }
    std::vector<Particle> read_particles() {
        std::vector<Particle> out(count_);
        check(vlj_read_particles(sim_, reinterpret_cast<vlj_particle*>(out.data())));
        return out;
    }

    void sample_profile() { check(vlj_sample_profile(sim_)); }
    void sample_profile_now() { sample_profile(); }
    void clear_profile() { check(vlj_clear_profile(sim_)); }
    Profile read_profile() {
        Profile p;
        std::vector<vlj_slab> slabs(bins_);
        check(vlj_read_profile(sim_, slabs.data(), p.virial.data(), &p.samples));
        p.box_size = box_size();
        for (const vlj_slab& s : slabs)
            p.slabs.push_back({s.z, s.particles, {s.kinetic[0], s.kinetic[1], s.kinetic[2]},
                               {s.virial[0], s.virial[1], s.virial[2]}, s.potential});
        return p;
    }

    void record_heat_current(uint32_t capacity) {
        check(vlj_record_heat_current(sim_, capacity));
        series_ = capacity;
    }
    void sample_heat_current() { check(vlj_sample_heat_current(sim_)); }
    std::vector<std::array<double, 3>> read_heat_current() {
        std::vector<std::array<double, 3>> out(series_);
        size_t n = 0;
        check(vlj_read_heat_current(sim_, out.empty() ? nullptr : out[0].data(), series_, &n));
        out.resize(n);
        return out;
    }

    void set_drawn(Drawn d) { check(vlj_set_drawn(sim_, static_cast<vlj_drawn>(d))); }
    void set_condensed_neighbours(uint32_t n) { check(vlj_set_condensed_neighbours(sim_, n)); }
    void set_temperature(double t) { check(vlj_set_temperature(sim_, t)); }
    void set_heat_exchange(const std::optional<HeatExchange>& e) {
        if (!e) {
            check(vlj_set_heat_exchange(sim_, nullptr));
            return;
        }
        vlj_heat_exchange h = {{e->hot.first, e->hot.second}, {e->cold.first, e->cold.second},
                               e->energy};
        check(vlj_set_heat_exchange(sim_, &h));
    }
    void set_grid_every_step(bool on) { check(vlj_set_grid_every_step(sim_, on ? 1 : 0)); }
    std::optional<double> heat_flux() const {
        int has = 0;
        double f = 0.0;
        check(vlj_heat_flux(sim_, &has, &f));
        return has ? std::optional<double>(f) : std::nullopt;
    }

    uint32_t count() const { return count_; }
    std::array<double, 3> box_size() const {
        std::array<double, 3> b{};
        check(vlj_box_size(sim_, b.data()));
        return b;
    }
    double volume() const {
        double v = 0.0;
        check(vlj_volume(sim_, &v));
        return v;
    }
    uint64_t steps() const {
        uint64_t s = 0;
        check(vlj_steps(sim_, &s));
        return s;
    }
    double time() const {
        double t = 0.0;
        check(vlj_time(sim_, &t));
        return t;
    }
    std::optional<double> target_temperature() const {
        int has = 0;
        double t = 0.0;
        check(vlj_target_temperature(sim_, &has, &t));
        return has ? std::optional<double>(t) : std::nullopt;
    }
    vlj_sim* raw() { return sim_; }

private:
    vlj_sim* sim_ = nullptr;
    uint32_t bins_ = 0;
    uint32_t count_ = 0;
    uint32_t series_ = 0;
};

/* lennard_jones.rs:1377-1441 */
inline std::vector<Particle> lattice(size_t count, double box_size, double temperature,
                                     uint64_t seed) {
    std::vector<Particle> out(count);
    check(vlj_lattice(count, box_size, temperature, seed,
                      reinterpret_cast<vlj_particle*>(out.data())));
    return out;
}

inline std::vector<Particle> lattice_box(size_t count, const std::array<double, 3>& size,
                                         double temperature, uint64_t seed) {
    std::vector<Particle> out(count);
    check(vlj_lattice_box(count, size.data(), temperature, seed,
                          reinterpret_cast<vlj_particle*>(out.data())));
    return out;
}

}  // namespace virial_lj

#endif
