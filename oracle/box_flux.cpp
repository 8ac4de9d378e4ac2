// Oracle for the box-flux projection: a serial CPU restatement of
// BoxFluxWorkspace::project (src/box_flux.rs:213-397) on the oracle's own
// pressure solve. Test infrastructure only: the library's device projection
// is checked against it.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "oracle.h"

namespace {

// compensated (src/box_flux.rs:444-459): Neumaier.
double compensated(const double* v, int n) {
    double sum = 0.0, correction = 0.0;
    for (int i = 0; i < n; ++i) {
        const double next = sum + v[i];
        correction += std::fabs(sum) >= std::fabs(v[i]) ? (sum - next) + v[i] : (v[i] - next) + sum;
        sum = next;
    }
    return sum + correction;
}

// PrescribedBoxFlux::component (src/box_flux.rs:36-45): the face value of a
// side (+ speed on an upper side, - speed on a lower one, +0 for a zero speed).
float component(const float outward[6], int d, bool upper) {
    const float speed = outward[2 * d + (upper ? 1 : 0)];
    if (speed == 0.0f) return 0.0f;
    return upper ? speed : -speed;
}

}  // namespace

extern "C" int orc_box_flux_project(const orc_grid* gi, double density, int method, const float* u, const float* v,
                                    const float* w, double dt, const float outward[6], const orc_settings* settings,
                                    double actual_divergence_limit, float* out_u, float* out_v, float* out_w,
                                    double* pressure_out, orc_box_flux_report* rep) {
    std::memset(rep, 0, sizeof(*rep));
    const uint64_t n[3] = {gi->counts[0], gi->counts[1], gi->counts[2]};
    const double h[3] = {gi->spacing[0], gi->spacing[1], gi->spacing[2]};
    const float* old[3] = {u, v, w};
    float* out[3] = {out_u, out_v, out_w};
    auto fc = [&](int a, int d) { return n[d] + (a == d ? 1 : 0); };
    auto face = [&](int a, const uint64_t p[3]) { return p[0] + fc(a, 0) * (p[1] + fc(a, 1) * p[2]); };
    auto cell = [&](const uint64_t p[3]) { return p[0] + n[0] * (p[1] + n[1] * p[2]); };
    const uint64_t cells = n[0] * n[1] * n[2];
    // BoxFluxWorkspace::new (:132-186)
    const double area[3] = {h[1] * h[2], h[0] * h[2], h[0] * h[1]};
    double side_area[3], factor[3];
    for (int d = 0; d < 3; ++d) {
        side_area[d] = area[d] * double(n[(d + 1) % 3]) * double(n[(d + 2) % 3]);
        factor[d] = 1.0 / (density * h[d]);
    }
    const double volume = h[0] * h[1] * h[2];
    const double mass = density * volume;
    if (!std::isfinite(mass) || mass <= 0.0) return 10;
    // project (:213-262)
    if (!std::isfinite(dt) || dt <= 0.0) return 10;
    if (!std::isfinite(actual_divergence_limit) || actual_divergence_limit < 0.0) return 10;
    for (int d = 0; d < 3; ++d) {
        uint64_t len = fc(d, 0) * fc(d, 1) * fc(d, 2);
        for (uint64_t f = 0; f < len; ++f)
            if (!std::isfinite(old[d][f])) return 12;
    }
    double terms[6], absolute_terms[6];
    for (int i = 0; i < 6; ++i) {
        terms[i] = side_area[i / 2] * double(outward[i]);
        if (terms[i] == 0.0 && outward[i] != 0.0f) return 14;
        absolute_terms[i] = std::fabs(terms[i]);
    }
    const double net = compensated(terms, 6), absolute = compensated(absolute_terms, 6);
    const double budget = 64.0 * std::numeric_limits<double>::epsilon() * absolute;
    rep->net_outward_flux = net;
    rep->flux_rounding_budget = budget;
    if (!std::isfinite(net) || !std::isfinite(absolute)) return 14;
    if (std::fabs(net) > budget) return 28;
    // RHS of the imposed field (:263-290)
    std::vector<double> rhs(cells);
    uint64_t p[3];
    for (p[2] = 0; p[2] < n[2]; ++p[2])
        for (p[1] = 0; p[1] < n[1]; ++p[1])
            for (p[0] = 0; p[0] < n[0]; ++p[0]) {
                double flux = 0.0;
                for (int d = 0; d < 3; ++d) {
                    uint64_t hi[3] = {p[0], p[1], p[2]};
                    hi[d] += 1;
                    const float lower = p[d] == 0 ? component(outward, d, false) : old[d][face(d, p)];
                    const float upper = hi[d] == n[d] ? component(outward, d, true) : old[d][face(d, hi)];
                    flux += area[d] * (double(lower) - double(upper));
                }
                const double r = flux / dt;
                if (!std::isfinite(r)) return 14;
                rhs[cell(p)] = r;
            }
    const int st = orc_solve_rhs(gi, density, method, rhs.data(), dt, settings, pressure_out, &rep->pressure,
                                 nullptr, 0, 1);
    rep->pressure_status = st;
    if (st) return st;
    // correction and the interior energy terms (:291-328)
    double kinetic_before = 0.0, kinetic_after = 0.0, correction_energy = 0.0, correction_residual = 0.0;
    for (int d = 0; d < 3; ++d)
        for (p[2] = 0; p[2] < fc(d, 2); ++p[2])
            for (p[1] = 0; p[1] < fc(d, 1); ++p[1])
                for (p[0] = 0; p[0] < fc(d, 0); ++p[0]) {
                    const uint64_t index = face(d, p);
                    if (p[d] == 0 || p[d] == n[d]) {
                        out[d][index] = component(outward, d, p[d] != 0);
                        continue;
                    }
                    uint64_t left[3] = {p[0], p[1], p[2]};
                    left[d] -= 1;
                    const double difference = pressure_out[cell(p)] - pressure_out[cell(left)];
                    const double uo = double(old[d][index]);
                    const double value = uo - dt * factor[d] * difference;
                    if (!std::isfinite(value) || std::fabs(value) > double(std::numeric_limits<float>::max()))
                        return 14;
                    const float stored = float(value);
                    out[d][index] = stored;
                    const double vv = double(stored);
                    const double delta = vv - uo;
                    kinetic_before += 0.5 * mass * uo * uo;
                    kinetic_after += 0.5 * mass * vv * vv;
                    correction_energy += 0.5 * mass * delta * delta;
                    correction_residual += (mass * delta + dt * area[d] * difference) * vv;
                }
    // divergence of the stored result (:329-337, :419-443)
    std::vector<double> div(cells);
    double actual = 0.0;
    for (p[2] = 0; p[2] < n[2]; ++p[2])
        for (p[1] = 0; p[1] < n[1]; ++p[1])
            for (p[0] = 0; p[0] < n[0]; ++p[0]) {
                double value = 0.0;
                for (int d = 0; d < 3; ++d) {
                    uint64_t hi[3] = {p[0], p[1], p[2]};
                    hi[d] += 1;
                    value += (double(out[d][face(d, hi)]) - double(out[d][face(d, p)])) / h[d];
                }
                if (!std::isfinite(value)) return 14;
                div[cell(p)] = value;
                actual = std::fmax(actual, std::fabs(value));
            }
    rep->actual_divergence_max = actual;
    if (actual > actual_divergence_limit) return 15;
    // boundary and residual work (:338-362)
    double boundary_work = 0.0, residual_work = 0.0;
    for (p[2] = 0; p[2] < n[2]; ++p[2])
        for (p[1] = 0; p[1] < n[1]; ++p[1])
            for (p[0] = 0; p[0] < n[0]; ++p[0]) {
                const uint64_t c = cell(p);
                double q = 0.0;
                for (int d = 0; d < 3; ++d) {
                    if (p[d] == 0) q += area[d] * double(outward[2 * d]);
                    if (p[d] + 1 == n[d]) q += area[d] * double(outward[2 * d + 1]);
                }
                boundary_work -= dt * pressure_out[c] * q;
                residual_work += dt * pressure_out[c] * volume * div[c];
            }
    const double budget_error = kinetic_after - kinetic_before + correction_energy -
                                (boundary_work + residual_work + correction_residual);
    rep->kinetic_before = kinetic_before;
    rep->kinetic_after = kinetic_after;
    rep->correction_energy = correction_energy;
    rep->boundary_pressure_work = boundary_work;
    rep->divergence_residual_work = residual_work;
    rep->correction_residual_work = correction_residual;
    rep->budget_error = budget_error;
    for (double x : {kinetic_before, kinetic_after, correction_energy, boundary_work, residual_work,
                     correction_residual, budget_error})
        if (!std::isfinite(x)) return 14;
    return 0;
}
