// Oracle for the liquid-volume transport: a serial CPU restatement of
// LiquidVolumeState::prepare_with_boundary for an inlet boundary, the
// all-cells divergence domain and no reconstructed columns
// (src/liquid_volume.rs:520-776), with its flow, inlet and source validations.
// Test infrastructure only: the library's device transport is checked
// against it.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "oracle.h"

namespace {

// rb200_liquid_error codes (include/rheon_b200.h)
enum {
    OK = 0,
    INVALID_DENSITY = 1,
    INVALID_FRACTION = 2,
    INVALID_INLET = 3,
    INVALID_SOURCE = 4,
    INVALID_SETTINGS = 5,
    INVALID_TIME_STEP = 6,
    TIME_RESOLUTION = 7,
    TIME_MISMATCH = 8,
    LENGTH_MISMATCH = 9,
    NONFINITE_VELOCITY = 10,
    VERSION_OVERFLOW = 11,
    COURANT_LIMIT = 13,
    DIVERGENCE_LIMIT = 14,
    FRACTION_BOUNDS = 15,
    BALANCE_LIMIT = 16,
    ARITHMETIC_FAILURE = 17,
    PERIODIC_VELOCITY_MISMATCH = 20,
};

struct Fail {
    int code;
};

// product / quotient (src/liquid_volume.rs:879-896): overflow, subnormal
// results and underflow to zero are failures.
double product(double a, double b) {
    const double v = a * b;
    if (!std::isfinite(v) || (v != 0.0 && !std::isnormal(v)) || (v == 0.0 && a != 0.0 && b != 0.0))
        throw Fail{ARITHMETIC_FAILURE};
    return v;
}
double quotient(double a, double b) {
    const double v = a / b;
    if (!std::isfinite(v) || (v != 0.0 && !std::isnormal(v)) || (v == 0.0 && a != 0.0)) throw Fail{ARITHMETIC_FAILURE};
    return v;
}

// Accumulator (src/liquid_volume.rs:907-929): Neumaier.
struct Acc {
    double sum = 0.0, correction = 0.0;
    void add(double value) {
        const double next = sum + value;
        correction += std::fabs(sum) >= std::fabs(value) ? (sum - next) + value : (value - next) + sum;
        sum = next;
    }
    double total() const { return sum + correction; }
};

struct G {
    uint64_t n[3];
    double h[3];
    uint64_t cell(const uint64_t p[3]) const { return p[0] + n[0] * (p[1] + n[1] * p[2]); }
    uint64_t fc(int a, int d) const { return n[d] + (a == d ? 1 : 0); }
    uint64_t face(int a, const uint64_t p[3]) const { return p[0] + fc(a, 0) * (p[1] + fc(a, 1) * p[2]); }
    uint64_t face_len(int a) const { return fc(a, 0) * fc(a, 1) * fc(a, 2); }
    uint64_t cells() const { return n[0] * n[1] * n[2]; }
};

}  // namespace

extern "C" int orc_liquid_validate_state(const orc_grid* gi, double density, const double* fraction, uint64_t* cell) {
    // LiquidVolumeState::new (src/liquid_volume.rs:276-305)
    if (!std::isfinite(density) || density <= 0.0) return INVALID_DENSITY;
    G g{{gi->counts[0], gi->counts[1], gi->counts[2]}, {gi->spacing[0], gi->spacing[1], gi->spacing[2]}};
    const double volume = g.h[0] * g.h[1] * g.h[2];
    try {
        for (uint64_t c = 0; c < g.cells(); ++c) {
            if (!std::isfinite(fraction[c]) || !(fraction[c] >= 0.0 && fraction[c] <= 1.0)) {
                if (cell) *cell = c;
                return INVALID_FRACTION;
            }
            product(volume, fraction[c]);
        }
        Acc a;
        for (uint64_t c = 0; c < g.cells(); ++c) a.add(volume * fraction[c]);
        const double initial = a.total();
        if (!std::isfinite(initial) || !std::isfinite(product(density, initial))) return ARITHMETIC_FAILURE;
    } catch (Fail f) {
        return f.code;
    }
    return OK;
}

extern "C" int orc_liquid_advance(const orc_grid* gi, double density, double state_time, uint64_t state_version,
                                  const double* accepted, double* candidate, const float* u, const float* v,
                                  const float* w, double start, double dt, const double inlet[6],
                                  const double* source_rate, double max_outward_courant,
                                  double actual_divergence_limit, int periodic, orc_liquid_report* rep) {
    std::memset(rep, 0, sizeof(*rep));
    G g{{gi->counts[0], gi->counts[1], gi->counts[2]}, {gi->spacing[0], gi->spacing[1], gi->spacing[2]}};
    const float* vel[3] = {u, v, w};
    // LiquidFlowInterval::new (:123-150)
    if (!std::isfinite(start) || start < 0.0 || !std::isfinite(dt) || dt <= 0.0) return INVALID_TIME_STEP;
    const double end = start + dt;
    if (!std::isfinite(end) || end <= start) return TIME_RESOLUTION;
    for (int a = 0; a < 3; ++a)
        for (uint64_t f = 0; f < g.face_len(a); ++f)
            if (!std::isfinite(vel[a][f])) return NONFINITE_VELOCITY;
    // LiquidInlet::new (:84-96), LiquidVolumeSource::new (:185-190); a
    // periodic boundary has no inlet
    if (!periodic)
        for (int q = 0; q < 6; ++q)
            if (!std::isfinite(inlet[q]) || !(inlet[q] >= 0.0 && inlet[q] <= 1.0)) return INVALID_INLET;
    if (source_rate)
        for (uint64_t c = 0; c < g.cells(); ++c)
            if (!std::isfinite(source_rate[c])) return INVALID_SOURCE;
    // prepare_with_boundary (:520-529) and validate_advance (:485-506)
    uint64_t tb, sb;
    std::memcpy(&tb, &start, 8);
    std::memcpy(&sb, &state_time, 8);
    if (tb != sb) return TIME_MISMATCH;
    if (!std::isfinite(max_outward_courant) || max_outward_courant <= 0.0 || max_outward_courant > 1.0 ||
        !std::isfinite(actual_divergence_limit) || actual_divergence_limit < 0.0)
        return INVALID_SETTINGS;
    if (state_version == std::numeric_limits<uint64_t>::max()) return VERSION_OVERFLOW;
    // periodic seams (:530-554): the two faces of a seam carry the same velocity
    if (periodic)
        for (int d = 0; d < 3; ++d) {
            uint64_t q[3];
            for (q[2] = 0; q[2] < g.fc(d, 2); ++q[2])
                for (q[1] = 0; q[1] < g.fc(d, 1); ++q[1])
                    for (q[0] = 0; q[0] < g.fc(d, 0); ++q[0]) {
                        if (q[d] != 0) continue;
                        uint64_t hi[3] = {q[0], q[1], q[2]};
                        hi[d] = g.n[d];
                        const uint64_t low = g.face(d, q), high = g.face(d, hi);
                        if (vel[d][low] != vel[d][high]) {
                            rep->error_cell = low;
                            rep->error_actual = double(d);
                            return PERIODIC_VELOCITY_MISMATCH;
                        }
                    }
        }
    const double volume = g.h[0] * g.h[1] * g.h[2];
    std::vector<double> transfer[3];
    try {
        const double area[3] = {product(g.h[1], g.h[2]), product(g.h[0], g.h[2]), product(g.h[0], g.h[1])};
        // face transfers (:556-641): the upwind donor fraction, the inlet on inflow
        for (int d = 0; d < 3; ++d) {
            transfer[d].assign(g.face_len(d), 0.0);
            uint64_t p[3];
            for (p[2] = 0; p[2] < g.fc(d, 2); ++p[2])
                for (p[1] = 0; p[1] < g.fc(d, 1); ++p[1])
                    for (p[0] = 0; p[0] < g.fc(d, 0); ++p[0]) {
                        const uint64_t face = g.face(d, p);
                        if (periodic && p[d] == g.n[d]) {  // the seam's upper face repeats its lower one
                            uint64_t lo[3] = {p[0], p[1], p[2]};
                            lo[d] = 0;
                            transfer[d][face] = transfer[d][g.face(d, lo)];
                            continue;
                        }
                        const double velocity = double(vel[d][face]);
                        double donor = 0.0;
                        if (velocity > 0.0) {
                            if (p[d] == 0 && periodic) {
                                uint64_t lo[3] = {p[0], p[1], p[2]};
                                lo[d] = g.n[d] - 1;
                                donor = accepted[g.cell(lo)];
                            } else if (p[d] == 0) {
                                donor = inlet[2 * d];
                            } else {
                                uint64_t lo[3] = {p[0], p[1], p[2]};
                                lo[d] -= 1;
                                donor = accepted[g.cell(lo)];
                            }
                        } else if (velocity < 0.0) {
                            donor = p[d] == g.n[d] ? inlet[2 * d + 1] : accepted[g.cell(p)];
                        }
                        transfer[d][face] = product(product(product(dt, area[d]), velocity), donor);
                    }
        }
        // cell update (:642-699)
        double max_courant = 0.0, max_div = 0.0;
        uint64_t p[3];
        for (p[2] = 0; p[2] < g.n[2]; ++p[2])
            for (p[1] = 0; p[1] < g.n[1]; ++p[1])
                for (p[0] = 0; p[0] < g.n[0]; ++p[0]) {
                    const uint64_t cell = g.cell(p);
                    double amount = product(volume, accepted[cell]);
                    double courant = 0.0, div = 0.0;
                    for (int d = 0; d < 3; ++d) {
                        uint64_t hi[3] = {p[0], p[1], p[2]};
                        hi[d] += 1;
                        const uint64_t low = g.face(d, p), high = g.face(d, hi);
                        amount += transfer[d][low] - transfer[d][high];
                        const double a = double(vel[d][low]), b = double(vel[d][high]);
                        courant += quotient(product(dt, std::fmax(b, 0.0) - std::fmin(a, 0.0)), g.h[d]);
                        div += quotient(b - a, g.h[d]);
                    }
                    if (!std::isfinite(courant) || !std::isfinite(div)) throw Fail{ARITHMETIC_FAILURE};
                    if (courant > max_outward_courant) {
                        rep->error_cell = cell;
                        rep->error_actual = courant;
                        rep->error_limit = max_outward_courant;
                        return COURANT_LIMIT;
                    }
                    max_courant = std::fmax(max_courant, courant);
                    max_div = std::fmax(max_div, std::fabs(div));
                    if (source_rate) amount += product(dt, source_rate[cell]);
                    const double fraction = quotient(amount, volume);
                    if (!(fraction >= 0.0 && fraction <= 1.0)) {
                        rep->error_cell = cell;
                        rep->error_actual = fraction;
                        return FRACTION_BOUNDS;
                    }
                    product(volume, fraction);
                    candidate[cell] = fraction;
                }
        if (max_div > actual_divergence_limit) {
            rep->error_actual = max_div;
            rep->error_limit = actual_divergence_limit;
            return DIVERGENCE_LIMIT;
        }
        // volume ledger (:735-776)
        Acc before_a, after_a, inward_a, outward_a, src_a, src_abs_a;
        for (uint64_t c = 0; c < g.cells(); ++c) before_a.add(volume * accepted[c]);
        for (uint64_t c = 0; c < g.cells(); ++c) after_a.add(volume * candidate[c]);
        for (int d = 0; d < 3; ++d) {
            uint64_t q[3];
            for (q[2] = 0; q[2] < g.fc(d, 2); ++q[2])
                for (q[1] = 0; q[1] < g.fc(d, 1); ++q[1])
                    for (q[0] = 0; q[0] < g.fc(d, 0); ++q[0]) {
                        if (periodic || (q[d] != 0 && q[d] != g.n[d])) continue;
                        const double value = transfer[d][g.face(d, q)] * (q[d] == 0 ? -1.0 : 1.0);
                        if (value < 0.0)
                            inward_a.add(-value);
                        else
                            outward_a.add(value);
                    }
        }
        if (source_rate)
            for (uint64_t c = 0; c < g.cells(); ++c) {
                const double s = product(dt, source_rate[c]);
                src_a.add(s);
                src_abs_a.add(std::fabs(s));
            }
        const double before = before_a.total(), after = after_a.total();
        const double inward = inward_a.total(), outward = outward_a.total(), source_total = src_a.total();
        const double balance = after - before + outward - inward - source_total;
        const double budget = (64.0 * std::numeric_limits<double>::epsilon()) *
                              (std::fabs(before) + std::fabs(after) + outward + inward + src_abs_a.total());
        const double mass_before = product(density, before);
        const double mass_after = product(density, after);
        for (double x : {before, after, inward, outward, source_total, balance, budget, mass_before, mass_after})
            if (!std::isfinite(x)) throw Fail{ARITHMETIC_FAILURE};
        if (std::fabs(balance) > budget) {
            rep->error_actual = balance;
            rep->error_limit = budget;
            return BALANCE_LIMIT;
        }
        double mn = 1.0, mx = 0.0;
        uint64_t dry = 0, full = 0;
        for (uint64_t c = 0; c < g.cells(); ++c) {
            mn = std::fmin(mn, candidate[c]);
            mx = std::fmax(mx, candidate[c]);
            dry += candidate[c] == 0.0;
            full += candidate[c] == 1.0;
        }
        rep->dt = dt;
        rep->time = end;
        rep->liquid_volume_before = before;
        rep->liquid_volume_after = after;
        rep->inward_boundary_volume = inward;
        rep->outward_boundary_volume = outward;
        rep->source_volume = source_total;
        rep->volume_balance_error = balance;
        rep->volume_rounding_budget = budget;
        rep->liquid_mass_before = mass_before;
        rep->liquid_mass_after = mass_after;
        rep->max_outward_courant = max_courant;
        rep->actual_divergence_max = max_div;
        rep->fraction_min = mn;
        rep->fraction_max = mx;
        rep->dry_cells = dry;
        rep->full_cells = full;
        rep->mixed_cells = g.cells() - dry - full;
    } catch (Fail f) {
        return f.code;
    }
    return OK;
}
