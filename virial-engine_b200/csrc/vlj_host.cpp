// Host-only parts of the C ABI: error strings, lattices and profile analysis.
// Restates the reference's free functions and Profile methods
// (crates/virial-particles/src/lennard_jones.rs:209-279, 1377-1441).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "virial_lj.h"
#include "vlj_common.h"

namespace vlj {

static thread_local std::string t_error;

vlj_status fail(vlj_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_error = buf;
    return s;
}

void clear_error() { t_error.clear(); }

namespace {

struct Xorshift {
    uint64_t s;
    // lennard_jones.rs:1410-1415
    double random() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return ((double)(s >> 11) + 0.5) / 9007199254740992.0;
    }
    // lennard_jones.rs:1416-1419
    double gaussian() {
        double r = std::sqrt(-2.0 * std::log(random()));
        return r * std::cos(6.283185307179586 * random());
    }
};

void zero_momentum(size_t count, vlj_particle* out) {
    double mean[3];
    for (int k = 0; k < 3; k++) {
        double sum = 0.0;
        for (size_t i = 0; i < count; i++) sum += out[i].vel[k];
        mean[k] = sum / (double)count;
    }
    for (size_t i = 0; i < count; i++)
        for (int k = 0; k < 3; k++) out[i].vel[k] -= mean[k];
}

// lennard_jones.rs:1401-1441
void lattice_sites(size_t count, const double size[3], const size_t sites[3], double temperature,
                   uint64_t seed, vlj_particle* out) {
    double gap[3];
    for (int k = 0; k < 3; k++) gap[k] = size[k] / (double)sites[k];
    Xorshift r{seed | 1u};
    const double root_t = std::sqrt(temperature);
    for (size_t i = 0; i < count; i++) {
        size_t c[3] = {i % sites[0], (i / sites[0]) % sites[1], i / (sites[0] * sites[1])};
        for (int k = 0; k < 3; k++) out[i].pos[k] = ((double)c[k] + 0.5) * gap[k];
        for (int k = 0; k < 3; k++) out[i].vel[k] = r.gaussian() * root_t;
    }
    zero_momentum(count, out);
}

}  // namespace
}  // namespace vlj

using vlj::fail;

extern "C" {

const char* vlj_last_error(void) { return vlj::t_error.c_str(); }

const char* vlj_status_name(vlj_status s) {
    switch (s) {
        case VLJ_OK: return "ok";
        case VLJ_INVALID_ARG: return "invalid argument";
        case VLJ_BOX_TOO_SMALL: return "box too small";
        case VLJ_LIST_OVERFLOW: return "neighbour list overflow";
        case VLJ_CUDA_ERROR: return "CUDA error";
        case VLJ_TIMEOUT: return "timeout";
        case VLJ_BUSY: return "busy";
        case VLJ_NOT_ENABLED: return "not enabled";
        case VLJ_FULL: return "full";
        case VLJ_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

vlj_status vlj_lattice(size_t count, double box_size, double temperature, uint64_t seed,
                       vlj_particle* out) {
    if (!out || count == 0) return fail(VLJ_INVALID_ARG, "lattice: empty or null output");
    if (!(box_size > 0.0) || !std::isfinite(box_size) || !(temperature >= 0.0))
        return fail(VLJ_INVALID_ARG, "lattice: bad box size or temperature");
    // lennard_jones.rs:1379-1382
    size_t per_side = (size_t)std::ceil(std::cbrt((double)count));
    double size[3] = {box_size, box_size, box_size};
    size_t sites[3] = {per_side, per_side, per_side};
    vlj::lattice_sites(count, size, sites, temperature, seed, out);
    return VLJ_OK;
}

vlj_status vlj_lattice_box(size_t count, const double size[3], double temperature, uint64_t seed,
                           vlj_particle* out) {
    if (!out || !size || count == 0) return fail(VLJ_INVALID_ARG, "lattice_box: empty or null");
    for (int k = 0; k < 3; k++)
        if (!(size[k] > 0.0) || !std::isfinite(size[k]))
            return fail(VLJ_INVALID_ARG, "lattice_box: bad size");
    // lennard_jones.rs:1388-1399; ties between axes go to the later one, as
    // Rust's max_by does
    double spacing = std::cbrt(size[0] * size[1] * size[2] / (double)count);
    size_t sites[3];
    for (int k = 0; k < 3; k++) {
        double s = std::round(size[k] / spacing);
        sites[k] = s < 1.0 ? 1 : (size_t)s;
    }
    while (sites[0] * sites[1] * sites[2] < count) {
        int widest = 0;
        for (int k = 1; k < 3; k++)
            if (!(size[widest] / (double)sites[widest] > size[k] / (double)sites[k])) widest = k;
        sites[widest] += 1;
    }
    vlj::lattice_sites(count, size, sites, temperature, seed, out);
    return VLJ_OK;
}

vlj_status vlj_lattice_fcc(uint32_t cells, double density, double temperature, uint64_t seed,
                           vlj_particle* out, double* box_size) {
    if (!out || !box_size || cells == 0) return fail(VLJ_INVALID_ARG, "lattice_fcc: null or empty");
    if (!(density > 0.0) || !(temperature >= 0.0))
        return fail(VLJ_INVALID_ARG, "lattice_fcc: bad density or temperature");
    static const double basis[4][3] = {
        {0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.5, 0.0, 0.5}, {0.0, 0.5, 0.5}};
    const double a = std::cbrt(4.0 / density);
    *box_size = (double)cells * a;
    vlj::Xorshift r{seed | 1u};
    const double root_t = std::sqrt(temperature);
    size_t i = 0;
    for (uint32_t cz = 0; cz < cells; cz++)
        for (uint32_t cy = 0; cy < cells; cy++)
            for (uint32_t cx = 0; cx < cells; cx++)
                for (int b = 0; b < 4; b++, i++) {
                    const double c[3] = {(double)cx, (double)cy, (double)cz};
                    for (int k = 0; k < 3; k++) out[i].pos[k] = (c[k] + basis[b][k] + 0.25) * a;
                    for (int k = 0; k < 3; k++) out[i].vel[k] = r.gaussian() * root_t;
                }
    vlj::zero_momentum(i, out);
    return VLJ_OK;
}

// lennard_jones.rs:209-225
vlj_status vlj_profile_interfaces(const double* density, size_t bins, double lz, double midpoint,
                                  double* out, size_t capacity, size_t* found) {
    if (!density || !found || bins == 0 || !(lz > 0.0))
        return fail(VLJ_INVALID_ARG, "profile_interfaces: bad arguments");
    const double width = lz / (double)bins;
    size_t count = 0;
    for (size_t b = 0; b < bins; b++) {
        double a = density[b] - midpoint, c = density[(b + 1) % bins] - midpoint;
        if ((a < 0.0) != (c < 0.0)) {
            double z = ((double)b + 0.5) * width + width * a / (a - c);
            // rem_euclid
            double r = std::fmod(z, lz);
            if (r < 0.0) r += lz;
            if (out && count < capacity) out[count] = r;
            count++;
        }
    }
    *found = count;
    return VLJ_OK;
}

// lennard_jones.rs:231-260
vlj_status vlj_profile_phases(const double* density, size_t bins, double lz, double midpoint,
                              double margin, int32_t* phases) {
    if (!density || !phases || bins == 0 || !(lz > 0.0))
        return fail(VLJ_INVALID_ARG, "profile_phases: bad arguments");
    size_t n = 0;
    vlj_status s = vlj_profile_interfaces(density, bins, lz, midpoint, nullptr, 0, &n);
    if (s != VLJ_OK) return s;
    std::vector<double> interfaces(n);
    vlj_profile_interfaces(density, bins, lz, midpoint, interfaces.data(), n, &n);
    const double width = lz / (double)bins;
    for (size_t b = 0; b < bins; b++) {
        double z = ((double)b + 0.5) * width;
        double distance = INFINITY;
        for (double zi : interfaces) {
            double d = z - zi;
            // f64::round: half away from zero
            double e = std::fabs(d - lz * std::round(d / lz));
            distance = std::fmin(distance, e);
        }
        int32_t p;
        if (std::isinf(distance))
            p = VLJ_PHASE_BETWEEN;
        else if (distance >= margin)
            p = density[b] > midpoint ? VLJ_PHASE_LIQUID : VLJ_PHASE_VAPOUR;
        else if (distance <= margin / 2.0)
            p = VLJ_PHASE_INTERFACE;
        else
            p = VLJ_PHASE_BETWEEN;
        phases[b] = p;
    }
    return VLJ_OK;
}

}  // extern "C"
