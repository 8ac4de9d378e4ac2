// Oracle for the dense3D accepted-state frame: a CPU restatement of
// write_dense3d_frame (src/dense3d_sequence.rs:412-564). Test infrastructure
// only: the library's device encoder is checked against it byte for byte.
//
// Rust's LowerExp with a precision (`{:.9e}`, `{:.17e}`) prints the exact
// binary value rounded to precision+1 significant digits, ties to even, as
// [-]d.ddd...e<exponent> with the exponent in plain decimal ("e0", "e-3",
// "e21"); -0.0 keeps its sign. The C library's "%.*e" performs the same exact
// rounding; only its exponent spelling ("e+00", "e-03") differs and is
// rewritten here.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "oracle.h"

namespace {

void put_number(std::string& s, double v, int precision) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", precision, v);
    const char* e = std::strchr(buf, 'e');
    s.append(buf, size_t(e - buf));
    s += 'e';
    s += std::to_string(std::atoi(e + 1));
}

void put_u64(std::string& s, uint64_t v) { s += std::to_string(v); }

template <class T>
void put_array(std::string& s, const char* name, const T* values, size_t n, int precision) {
    s += '"';
    s += name;
    s += "\":[";
    for (size_t i = 0; i < n; ++i) {
        if (i) s += ',';
        put_number(s, values ? double(values[i]) : 0.0, precision);
    }
    s += ']';
}

}  // namespace

extern "C" int orc_dense3d_frame_text(const orc_grid* g, const orc_dense3d_frame* f, const float* u, const float* v,
                                      const float* w, const float* tracer, const double* fraction,
                                      const double* pressure, char* out, size_t capacity, size_t* length) {
    if (!g || !f || !u || !v || !w || !pressure || !length) return 10;
    const size_t nx = g->counts[0], ny = g->counts[1], nz = g->counts[2];
    const size_t cells = nx * ny * nz;
    const size_t faces[3] = {(nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)};
    const float* vel[3] = {u, v, w};
    // preflight (src/dense3d_sequence.rs:431-494): finite native fields,
    // fraction within [0, 1], clocks and report continuity
    for (int a = 0; a < 3; ++a)
        for (size_t i = 0; i < faces[a]; ++i)
            if (!std::isfinite(vel[a][i])) return 23;
    for (size_t i = 0; i < cells; ++i) {
        if (tracer && !std::isfinite(tracer[i])) return 23;
        if (!std::isfinite(pressure[i])) return 23;
        if (fraction && !(std::isfinite(fraction[i]) && fraction[i] >= 0.0 && fraction[i] <= 1.0)) return 23;
    }
    if (!std::isfinite(f->time_s)) return 23;
    const double diag[11] = {f->pressure_residual_m3_s2, f->carrier_divergence_s_inv, f->liquid_divergence_s_inv,
                             f->volume_before_m3,        f->volume_after_m3,          f->mass_after_kg,
                             f->inward_m3,               f->outward_m3,               f->source_m3,
                             f->balance_m3,              f->rounding_budget_m3};
    if (f->has_diagnostics) {
        if (!(std::isfinite(f->dt_s) && f->dt_s > 0.0)) return 23;
        for (double d : diag)
            if (!std::isfinite(d)) return 23;
    } else if (!(f->frame == 0 && f->time_s == 0.0 && f->carrier_stamp_version == 0)) {
        return 23;
    }
    std::string s;
    s += "{\"frame\":";
    put_u64(s, f->frame);
    s += ",\"time_s\":";
    put_number(s, f->time_s, 17);
    s += ",\"dt_s\":";
    put_number(s, f->has_diagnostics ? f->dt_s : 0.0, 17);
    s += ",\"carrier_stamp\":{\"id\":\"";
    put_u64(s, f->carrier_stamp_id);
    s += "\",\"version\":\"";
    put_u64(s, f->carrier_stamp_version);
    s += "\"},\"liquid_stamp\":{\"id\":\"";
    put_u64(s, f->liquid_stamp_id);
    s += "\",\"version\":\"";
    put_u64(s, f->liquid_stamp_version);
    s += "\"},\"fields\":{";
    put_array(s, "velocity_x", u, faces[0], 9);
    s += ',';
    put_array(s, "velocity_y", v, faces[1], 9);
    s += ',';
    put_array(s, "velocity_z", w, faces[2], 9);
    s += ',';
    put_array(s, "tracer", tracer, cells, 9);
    s += ',';
    put_array(s, "fraction", fraction, cells, 17);
    s += ',';
    put_array(s, "pressure", pressure, cells, 17);
    s += "},\"diagnostics\":";
    if (f->has_diagnostics) {
        static const char* names[11] = {"pressure_residual_m3_s2", "carrier_divergence_s_inv",
                                        "liquid_divergence_s_inv", "volume_before_m3",
                                        "volume_after_m3",         "mass_after_kg",
                                        "inward_m3",               "outward_m3",
                                        "source_m3",               "balance_m3",
                                        "rounding_budget_m3"};
        s += "{\"pressure_iterations\":";
        put_u64(s, f->pressure_iterations);
        for (int q = 0; q < 11; ++q) {
            s += ",\"";
            s += names[q];
            s += "\":";
            put_number(s, diag[q], 17);
        }
        s += '}';
    } else {
        s += "null";
    }
    s += "}\n";
    *length = s.size();
    if (!out || capacity < s.size()) return 24;
    std::memcpy(out, s.data(), s.size());
    return 0;
}
