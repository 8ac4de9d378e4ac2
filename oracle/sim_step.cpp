// Oracle for the step owner with its forcing and boundary domains: a serial
// CPU restatement of Simulation::prepare_impl (src/simulation.rs:812-1403)
// for the sealed box and the box-flux boundary, with the smoke source
// (validate_source, apply_force, apply_source :1430-1496) and the caller's
// body forces (src/forces.rs:63-212), on the oracle's own primitives. Test
// infrastructure only: the library's forced carrier step is checked against it.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "oracle.h"

namespace {

struct G {
    uint64_t n[3];
    double h[3], o[3], up[3];
    uint64_t fc[3][3];
    uint64_t flen[3];
    uint64_t cells;
    double volume;
};

G geometry(const orc_grid* in) {
    G g{};
    for (int d = 0; d < 3; ++d) {
        g.n[d] = in->counts[d];
        g.h[d] = in->spacing[d];
        g.o[d] = in->origin[d];
        g.up[d] = g.o[d] + double(g.n[d]) * g.h[d];  // GridGeometry::new (src/geometry.rs:152-154)
    }
    for (int a = 0; a < 3; ++a) {
        g.flen[a] = 1;
        for (int d = 0; d < 3; ++d) {
            g.fc[a][d] = g.n[d] + (a == d ? 1 : 0);
            g.flen[a] *= g.fc[a][d];
        }
    }
    g.cells = g.n[0] * g.n[1] * g.n[2];
    g.volume = g.h[0] * g.h[1] * g.h[2];
    return g;
}

// face_position / cell_position (src/geometry.rs:235-248)
void face_position(const G& g, int axis, const uint64_t p[3], double out[3]) {
    for (int d = 0; d < 3; ++d) out[d] = g.o[d] + (double(p[d]) + (d == axis ? 0.0 : 0.5)) * g.h[d];
}
void cell_position(const G& g, const uint64_t p[3], double out[3]) {
    for (int d = 0; d < 3; ++d) out[d] = g.o[d] + (double(p[d]) + 0.5) * g.h[d];
}

bool inside_box(const double p[3], const double lower[3], const double upper[3]) {
    for (int d = 0; d < 3; ++d)
        if (!(p[d] >= lower[d] && p[d] < upper[d])) return false;
    return true;
}

// validate_source (src/simulation.rs:1430-1445)
bool source_valid(const G& g, const orc_smoke_source& s) {
    if (!std::isfinite(s.tracer_rate) || s.tracer_rate < 0.0 || !std::isfinite(s.vertical_acceleration))
        return false;
    for (int d = 0; d < 3; ++d)
        if (!std::isfinite(s.lower[d]) || !std::isfinite(s.upper[d]) || s.lower[d] >= s.upper[d] ||
            s.lower[d] < g.o[d] || s.upper[d] > g.up[d])
            return false;
    return true;
}

// BodyForce::acceleration (src/forces.rs:34-39)
void force_acceleration(const orc_body_force& f, double density, double a[3]) {
    for (int d = 0; d < 3; ++d) a[d] = f.units == 1 ? f.value[d] / density : f.value[d];
}

// forces::validate (src/forces.rs:63-94): 0, 31 InvalidForce or 14.
int forces_validate(const G& g, double density, const orc_body_force* forces, size_t n, double* rate_out) {
    double rate = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const orc_body_force& f = forces[i];
        for (double v : f.value)
            if (!std::isfinite(v)) return 31;
        if (f.has_region)
            for (int d = 0; d < 3; ++d)
                if (!std::isfinite(f.lower[d]) || !std::isfinite(f.upper[d]) || f.lower[d] >= f.upper[d] ||
                    f.lower[d] < g.o[d] || f.upper[d] > g.up[d])
                    return 31;
        double a[3];
        force_acceleration(f, density, a);
        for (int d = 0; d < 3; ++d) rate += std::fabs(a[d]) / g.h[d];
    }
    if (!std::isfinite(rate)) return ORC_ARITHMETIC_FAILURE;
    *rate_out = rate;
    return 0;
}

// interior_energy (src/box_flux_step.rs:118-149): serial sum of interior squares.
int interior_energy(const G& g, double density, float* const vel[3], double* out) {
    double sum = 0.0;
    for (int a = 0; a < 3; ++a) {
        uint64_t p[3];
        for (p[2] = 0; p[2] < g.fc[a][2]; ++p[2])
            for (p[1] = 0; p[1] < g.fc[a][1]; ++p[1])
                for (p[0] = 0; p[0] < g.fc[a][0]; ++p[0])
                    if (p[a] > 0 && p[a] < g.n[a]) {
                        const double v = double(vel[a][p[0] + g.fc[a][0] * (p[1] + g.fc[a][1] * p[2])]);
                        sum += v * v;
                    }
    }
    const double energy = 0.5 * density * g.volume * sum;
    if (!std::isfinite(energy)) return ORC_ARITHMETIC_FAILURE;
    *out = energy;
    return 0;
}

// all-face energy sum: fields.iter().flat_map(..).map(v^2).sum() (src/forces.rs:153-161)
double face_square_sum(const G& g, float* const vel[3]) {
    double sum = 0.0;
    for (int a = 0; a < 3; ++a)
        for (uint64_t f = 0; f < g.flen[a]; ++f) {
            const double v = double(vel[a][f]);
            sum += v * v;
        }
    return sum;
}

double tracer_sum(const G& g, const float* t) {
    double sum = 0.0;
    for (uint64_t c = 0; c < g.cells; ++c) sum += double(t[c]);
    return sum;
}

// velocity_rate (src/simulation.rs:1415-1429)
int velocity_rate(const G& g, float* const vel[3], double* rate) {
    double r = 0.0;
    for (int d = 0; d < 3; ++d) {
        double m = 0.0;
        for (uint64_t f = 0; f < g.flen[d]; ++f) m = std::fmax(m, std::fabs(double(vel[d][f])));
        r += m / g.h[d];
    }
    if (!std::isfinite(r)) return ORC_ARITHMETIC_FAILURE;
    *rate = r;
    return 0;
}

// apply_force (src/simulation.rs:1449-1472): interior Y faces inside the source.
int smoke_force(const G& g, float* y, const orc_smoke_source& s, double dt) {
    uint64_t p[3];
    for (p[2] = 0; p[2] < g.n[2]; ++p[2])
        for (p[1] = 1; p[1] < g.n[1]; ++p[1])
            for (p[0] = 0; p[0] < g.n[0]; ++p[0]) {
                double pos[3];
                face_position(g, 1, p, pos);
                if (!inside_box(pos, s.lower, s.upper)) continue;
                const uint64_t f = p[0] + g.fc[1][0] * (p[1] + g.fc[1][1] * p[2]);
                const double v = double(y[f]) + dt * s.vertical_acceleration;
                if (!std::isfinite(v) || std::fabs(v) > double(std::numeric_limits<float>::max()))
                    return ORC_ARITHMETIC_FAILURE;
                y[f] = float(v);
            }
    return 0;
}

// apply_source (src/simulation.rs:1473-1496)
int smoke_tracer(const G& g, float* tracer, const orc_smoke_source& s, double dt) {
    const double amount = dt * s.tracer_rate;
    if (!std::isfinite(amount)) return ORC_ARITHMETIC_FAILURE;
    uint64_t p[3];
    for (p[2] = 0; p[2] < g.n[2]; ++p[2])
        for (p[1] = 0; p[1] < g.n[1]; ++p[1])
            for (p[0] = 0; p[0] < g.n[0]; ++p[0]) {
                double pos[3];
                cell_position(g, p, pos);
                if (!inside_box(pos, s.lower, s.upper)) continue;
                const uint64_t c = p[0] + g.n[0] * (p[1] + g.n[1] * p[2]);
                tracer[c] = float(std::fmin(double(tracer[c]) + amount, 1.0));
            }
    return 0;
}

// forces::apply_evaluated (src/forces.rs:144-212) for constant vectors.
int apply_forces(const G& g, double density, const orc_body_force* forces, size_t n, double dt, float* const vel[3],
                 double* before, double* after, double* work_out) {
    const double mass = density * g.volume;
    const double b = 0.5 * mass * face_square_sum(g, vel);
    double work = 0.0;
    for (int a = 0; a < 3; ++a) {
        uint64_t p[3];
        for (p[2] = 0; p[2] < g.fc[a][2]; ++p[2])
            for (p[1] = 0; p[1] < g.fc[a][1]; ++p[1])
                for (p[0] = 0; p[0] < g.fc[a][0]; ++p[0]) {
                    if (p[a] == 0 || p[a] == g.n[a]) continue;
                    double pos[3];
                    face_position(g, a, p, pos);
                    double sum[3] = {0.0, 0.0, 0.0};
                    for (size_t i = 0; i < n; ++i) {
                        if (forces[i].has_region && !inside_box(pos, forces[i].lower, forces[i].upper)) continue;
                        double acc[3];
                        force_acceleration(forces[i], density, acc);
                        for (int d = 0; d < 3; ++d) sum[d] += acc[d];
                    }
                    const uint64_t f = p[0] + g.fc[a][0] * (p[1] + g.fc[a][1] * p[2]);
                    const double old = double(vel[a][f]);
                    const double updated = old + dt * sum[a];
                    if (!std::isfinite(updated) || std::fabs(updated) > double(std::numeric_limits<float>::max()))
                        return ORC_ARITHMETIC_FAILURE;
                    const float stored = float(updated);
                    const double delta = double(stored) - old;
                    work += mass * delta * (old + 0.5 * delta);
                    vel[a][f] = stored;
                }
    }
    const double e = 0.5 * mass * face_square_sum(g, vel);
    if (!std::isfinite(b) || !std::isfinite(e) || !std::isfinite(work)) return ORC_ARITHMETIC_FAILURE;
    *before = b;
    *after = e;
    *work_out = work;
    return 0;
}

}  // namespace

extern "C" int orc_sim_step(const orc_grid* gi, const orc_sim_config* c, orc_sim_state* state, double requested_dt,
                            const orc_smoke_source* source, const orc_body_force* forces, size_t force_count,
                            const float* outward, orc_sim_report* rep) {
    std::memset(rep, 0, sizeof(*rep));
    const G g = geometry(gi);
    const bool boundary = outward != nullptr;
    float* acc[3] = {state->u, state->v, state->w};
    // prepare_impl (src/simulation.rs:812-1403)
    if (!std::isfinite(requested_dt) || requested_dt <= 0.0) return ORC_INVALID_ARGUMENT;
    if (source && !source_valid(g, *source)) return rep->error = 1, 29;
    double external_rate = 0.0;
    int st = forces_validate(g, c->density, forces, force_count, &external_rate);
    if (st == 31) return rep->error = 2, 29;
    if (st) return st;
    if (boundary) {
        if ((st = interior_energy(g, c->density, acc, &rep->kinetic_old))) return st;
        rep->tracer_old_integral = tracer_sum(g, state->tracer) * g.volume;
    }
    double rate = 0.0;
    if (boundary) {
        for (int d = 0; d < 3; ++d) {
            double old = 0.0;
            for (uint64_t f = 0; f < g.flen[d]; ++f) old = std::fmax(old, std::fabs(double(acc[d][f])));
            rate += std::fmax(std::fmax(old, std::fabs(double(outward[2 * d]))), std::fabs(double(outward[2 * d + 1]))) /
                    g.h[d];
        }
        if (!std::isfinite(rate)) return ORC_ARITHMETIC_FAILURE;
    } else if ((st = velocity_rate(g, acc, &rate))) {
        return st;
    }
    const double acceleration =
        (source ? std::fabs(source->vertical_acceleration) / g.h[1] : 0.0) + external_rate;
    if (!std::isfinite(acceleration)) return ORC_ARITHMETIC_FAILURE;
    double dt = requested_dt;
    if (rate > 0.0) dt = std::fmin(dt, 0.5 * c->max_courant / rate);
    if (acceleration > 0.0) dt = std::fmin(dt, std::sqrt(0.5 * c->max_courant / acceleration));
    const double next_time = state->time + dt;
    if (dt <= 0.0 || !std::isfinite(next_time) || next_time <= state->time) return rep->error = 3, 29;
    rep->dt = dt;
    // advection into the candidate
    std::vector<float> cand[3], tracer(g.cells);
    for (int a = 0; a < 3; ++a) cand[a].resize(g.flen[a]);
    float* cv[3] = {cand[0].data(), cand[1].data(), cand[2].data()};
    if ((st = orc_advect_velocity_f32(gi, acc[0], acc[1], acc[2], dt, cv[0], cv[1], cv[2], 1))) return st;
    if (boundary) {
        if ((st = interior_energy(g, c->density, cv, &rep->kinetic_after_advection))) return st;
        rep->advection_change = rep->kinetic_after_advection - rep->kinetic_old;
    }
    if (source && (st = smoke_force(g, cv[1], *source, dt))) return st;
    if (boundary) {
        if ((st = interior_energy(g, c->density, cv, &rep->kinetic_after_smoke_force))) return st;
        rep->smoke_force_work = rep->kinetic_after_smoke_force - rep->kinetic_after_advection;
    }
    if (force_count) {
        rep->has_forces = 1;
        if ((st = apply_forces(g, c->density, forces, force_count, dt, cv, &rep->force_kinetic_before,
                               &rep->force_kinetic_after, &rep->force_applied_work)))
            return st;
    }
    // projection
    std::vector<double> pressure(g.cells);
    if (boundary) {
        std::vector<float> out[3];
        for (int a = 0; a < 3; ++a) out[a].resize(g.flen[a]);
        st = orc_box_flux_project(gi, c->density, c->method, cv[0], cv[1], cv[2], dt, outward, &c->pressure,
                                  c->actual_divergence_limit, out[0].data(), out[1].data(), out[2].data(),
                                  pressure.data(), &rep->projection);
        rep->pressure = rep->projection.pressure;
        if (st == ORC_DIVERGENCE_LIMIT) {
            rep->error_actual = rep->projection.actual_divergence_max;
            rep->error_limit = c->actual_divergence_limit;
        }
        if (st) return st;
        for (int a = 0; a < 3; ++a) cand[a] = out[a];
        for (int a = 0; a < 3; ++a) cv[a] = cand[a].data();
        rep->actual_divergence_max = rep->projection.actual_divergence_max;
        const orc_box_flux_report& p = rep->projection;
        rep->kinetic_before_projection = p.kinetic_before;
        rep->kinetic_accepted = p.kinetic_after;
        rep->external_force_work = rep->has_forces ? rep->force_applied_work : 0.0;
        rep->boundary_volume_imbalance = dt * p.net_outward_flux;
        rep->budget_error = rep->kinetic_accepted - rep->kinetic_old + p.correction_energy -
                            (rep->advection_change + rep->smoke_force_work + rep->external_force_work +
                             p.boundary_pressure_work + p.divergence_residual_work + p.correction_residual_work);
    } else {
        std::vector<double> rhs(g.cells), div(g.cells);
        if ((st = orc_build_rhs_f32(gi, c->density, cv[0], cv[1], cv[2], dt, rhs.data()))) return st;
        st = orc_solve_rhs(gi, c->density, c->method, rhs.data(), dt, &c->pressure, pressure.data(), &rep->pressure,
                           nullptr, 0, 1);
        if (st) return st;
        if ((st = orc_correct_f32(gi, c->density, pressure.data(), dt, cv[0], cv[1], cv[2]))) return st;
        if ((st = orc_divergence_f32(gi, cv[0], cv[1], cv[2], div.data()))) return st;
        double actual = 0.0;
        for (double x : div) actual = std::fmax(actual, std::fabs(x));
        rep->actual_divergence_max = actual;
        if (actual > c->actual_divergence_limit) {
            rep->error_actual = actual;
            rep->error_limit = c->actual_divergence_limit;
            return ORC_DIVERGENCE_LIMIT;
        }
    }
    double candidate_rate = 0.0;
    if ((st = velocity_rate(g, cv, &candidate_rate))) return st;
    const double courant = dt * candidate_rate;
    rep->courant = courant;
    if (!std::isfinite(courant)) return ORC_ARITHMETIC_FAILURE;
    if (courant > c->max_courant) {
        rep->error_actual = courant;
        rep->error_limit = c->max_courant;
        return ORC_COURANT_LIMIT;
    }
    // tracer
    if ((st = orc_advect_tracer_f32(gi, state->tracer, cv[0], cv[1], cv[2], dt, tracer.data(), 1))) return st;
    const double transported = boundary ? tracer_sum(g, tracer.data()) * g.volume : 0.0;
    if (source && (st = smoke_tracer(g, tracer.data(), *source, dt))) return st;
    double tsum = 0.0;
    for (uint64_t i = 0; i < g.cells; ++i) {
        const float t = tracer[i];
        if (!std::isfinite(t) || !(t >= 0.0f && t <= 1.0f)) return ORC_ARITHMETIC_FAILURE;
        tsum += double(t);
    }
    const double energy_sum = face_square_sum(g, cv);
    const double tracer_integral = tsum * g.volume;
    const double kinetic = boundary ? rep->kinetic_accepted : 0.5 * c->density * g.volume * energy_sum;
    if (boundary) {
        rep->tracer_transport_change = transported - rep->tracer_old_integral;
        rep->tracer_source_change = tracer_integral - transported;
        for (double x : {rep->budget_error, rep->boundary_volume_imbalance, rep->tracer_old_integral,
                         rep->tracer_transport_change, rep->tracer_source_change})
            if (!std::isfinite(x)) return ORC_ARITHMETIC_FAILURE;
    }
    if (!std::isfinite(tracer_integral) || !std::isfinite(kinetic)) return ORC_ARITHMETIC_FAILURE;
    // commit (src/simulation.rs:805-811)
    rep->tracer_integral = tracer_integral;
    rep->kinetic_energy = kinetic;
    rep->time = next_time;
    rep->generation = state->generation + 1;
    for (int a = 0; a < 3; ++a) std::memcpy(acc[a], cv[a], g.flen[a] * sizeof(float));
    std::memcpy(state->tracer, tracer.data(), g.cells * sizeof(float));
    state->time = next_time;
    state->generation += 1;
    return 0;
}
