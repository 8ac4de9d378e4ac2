// Oracle: CPU restatement of Rheon's fixed-box carrier arithmetic.
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the
// product library never links it. See oracle.h for the reference map.
// Build with -ffp-contract=off: every a*b+c below must round twice, as Rust does.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include <atomic>
#include <thread>

namespace {

constexpr double kEps = std::numeric_limits<double>::epsilon();
constexpr double kF32Max = 3.4028234663852886e38;

// Plane-parallel loop for the stencil/gather loops only; every output element
// is written by exactly one thread, so results do not depend on the thread
// count. Reductions stay serial, as in the reference (src/parallel.rs:1-3).
template <class F>
void parallel_for(int64_t n, int threads, F&& f) {
    if (threads <= 1 || n < 2) {
        for (int64_t i = 0; i < n; ++i) f(i);
        return;
    }
    int t = int(std::min<int64_t>(threads, n));
    std::vector<std::thread> pool;
    pool.reserve(t);
    for (int w = 0; w < t; ++w) {
        int64_t lo = n * w / t, hi = n * (w + 1) / t;
        pool.emplace_back([lo, hi, &f] {
            for (int64_t i = lo; i < hi; ++i) f(i);
        });
    }
    for (auto& th : pool) th.join();
}

inline void record(std::atomic<int>& status, int st) {
    int expected = ORC_OK;
    status.compare_exchange_strong(expected, st);
}

struct Grid {
    int64_t n[3];
    double h[3];
    double o[3];
    double up[3];
    int64_t fc[3][3];
    int64_t flen[3];
    int64_t cells;
    double volume;
};

// GridGeometry::new (src/geometry.rs:114-191), restricted to what the path needs.
int make_grid(const orc_grid* in, Grid* g) {
    if (!in) return ORC_INVALID_ARGUMENT;
    for (int d = 0; d < 3; ++d) {
        if (in->counts[d] == 0) return ORC_INVALID_GEOMETRY;
        if (!std::isfinite(in->spacing[d]) || in->spacing[d] <= 0.0) return ORC_INVALID_GEOMETRY;
        if (!std::isfinite(in->origin[d])) return ORC_INVALID_GEOMETRY;
        if (in->counts[d] > (uint64_t(1) << 40)) return ORC_INVALID_GEOMETRY;
        g->n[d] = int64_t(in->counts[d]);
        g->h[d] = in->spacing[d];
        g->o[d] = in->origin[d];
    }
    g->cells = g->n[0] * g->n[1] * g->n[2];
    for (int a = 0; a < 3; ++a) {
        for (int d = 0; d < 3; ++d) g->fc[a][d] = g->n[d] + (a == d ? 1 : 0);
        g->flen[a] = g->fc[a][0] * g->fc[a][1] * g->fc[a][2];
    }
    g->volume = g->h[0] * g->h[1] * g->h[2];
    if (!std::isfinite(g->volume) || g->volume <= 0.0) return ORC_INVALID_GEOMETRY;
    for (int d = 0; d < 3; ++d) {
        double n = double(g->n[d]);
        double extent = n * g->h[d];
        g->up[d] = g->o[d] + extent;
        double scale = std::max(std::max(std::fabs(g->o[d]), std::fabs(g->up[d])), extent);
        if (!std::isfinite(extent) || !std::isfinite(scale) || !std::isnormal(0.5 * g->h[d]) ||
            g->h[d] / scale < 32.0 * kEps)
            return ORC_INVALID_GEOMETRY;
        double first = g->o[d] + 0.5 * g->h[d];
        double last = g->o[d] + (n - 0.5) * g->h[d];
        if (!std::isfinite(g->up[d]) || g->up[d] <= g->o[d] || first <= g->o[d] || last >= g->up[d])
            return ORC_INVALID_GEOMETRY;
    }
    return ORC_OK;
}

inline int64_t cell_index(const Grid& g, int64_t i, int64_t j, int64_t k) {
    return i + g.n[0] * (j + g.n[1] * k);
}
inline int64_t face_index(const Grid& g, int a, int64_t i, int64_t j, int64_t k) {
    return i + g.fc[a][0] * (j + g.fc[a][1] * k);
}

inline double clampd(double x, double lo, double hi) {
    // f64::clamp: if x < min { min } then if x > max { max }.
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

// Rust f64::min / f64::max on finite operands.
inline double fmin_r(double a, double b) { return std::fmin(a, b); }
inline double fmax_r(double a, double b) { return std::fmax(a, b); }

// compensated_sum (src/pressure.rs:135-148): serial Neumaier.
struct Neumaier {
    double sum = 0.0, correction = 0.0;
    void add(double value) {
        double next = sum + value;
        if (std::fabs(sum) >= std::fabs(value))
            correction += (sum - next) + value;
        else
            correction += (value - next) + sum;
        sum = next;
    }
    double result() const { return sum + correction; }
};

// ----------------------------------------------------------------- sampling
template <class T>
struct Sampler {
    const Grid* g;
    const T* values;
    int64_t dims[3];
    double off[3];
};

template <class T>
Sampler<T> face_sampler(const Grid& g, int axis, const T* values) {
    Sampler<T> s;
    s.g = &g;
    s.values = values;
    for (int d = 0; d < 3; ++d) {
        s.dims[d] = g.fc[axis][d];
        s.off[d] = (d == axis) ? 0.0 : 0.5;
    }
    return s;
}
template <class T>
Sampler<T> cell_sampler(const Grid& g, const T* values) {
    Sampler<T> s;
    s.g = &g;
    s.values = values;
    for (int d = 0; d < 3; ++d) {
        s.dims[d] = g.n[d];
        s.off[d] = 0.5;
    }
    return s;
}

// ScalarSampler::sample (src/sampling.rs:74-122).
template <class T>
int sample(const Sampler<T>& s, const double pos[3], double* out) {
    const Grid& g = *s.g;
    for (int d = 0; d < 3; ++d)
        if (!std::isfinite(pos[d])) return ORC_NONFINITE_POSITION;
    int64_t lo[3], hi[3];
    double t[3];
    for (int d = 0; d < 3; ++d) {
        double x = clampd(pos[d], g.o[d], g.up[d]);
        double q = clampd((x - g.o[d]) / g.h[d] - s.off[d], 0.0, double(s.dims[d] - 1));
        if (!std::isfinite(q)) return ORC_ARITHMETIC_FAILURE;
        lo[d] = int64_t(std::floor(q));
        hi[d] = std::min(lo[d] + 1, s.dims[d] - 1);
        t[d] = q - double(lo[d]);
    }
    double result = 0.0;
    double minimum = std::numeric_limits<double>::infinity();
    double maximum = -std::numeric_limits<double>::infinity();
    for (int z = 0; z < 2; ++z)
        for (int y = 0; y < 2; ++y)
            for (int x = 0; x < 2; ++x) {
                int bits[3] = {x, y, z};
                int64_t p[3];
                double weight = 1.0;
                for (int d = 0; d < 3; ++d) {
                    p[d] = bits[d] ? hi[d] : lo[d];
                    weight = weight * (bits[d] ? t[d] : 1.0 - t[d]);
                }
                double value = double(s.values[p[0] + s.dims[0] * (p[1] + s.dims[1] * p[2])]);
                minimum = fmin_r(minimum, value);
                maximum = fmax_r(maximum, value);
                result += weight * value;
            }
    if (!std::isfinite(result)) return ORC_ARITHMETIC_FAILURE;
    *out = clampd(result, minimum, maximum);
    return ORC_OK;
}

template <class T>
struct VelocitySampler {
    Sampler<T> c[3];
};

template <class T>
int vsample(const VelocitySampler<T>& v, const double pos[3], double out[3]) {
    for (int d = 0; d < 3; ++d) {
        int st = sample(v.c[d], pos, &out[d]);
        if (st) return st;
    }
    return ORC_OK;
}

// VelocitySampler::departure (src/sampling.rs:160-175).
inline int departure(const Grid& g, const double pos[3], const double vel[3], double dt,
                     double out[3]) {
    for (int d = 0; d < 3; ++d) {
        double value = pos[d] - dt * vel[d];
        if (!std::isfinite(value)) return ORC_ARITHMETIC_FAILURE;
        out[d] = clampd(value, g.o[d], g.up[d]);
    }
    return ORC_OK;
}

// VelocitySampler::backtrace (src/sampling.rs:151-159): midpoint RK2.
template <class T>
int backtrace(const Grid& g, const VelocitySampler<T>& v, const double pos[3], double dt,
              double out[3]) {
    if (!std::isfinite(dt) || dt <= 0.0) return ORC_INVALID_TIME_STEP;
    double initial[3], mid[3], vel[3];
    int st = vsample(v, pos, initial);
    if (st) return st;
    st = departure(g, pos, initial, 0.5 * dt, mid);
    if (st) return st;
    st = vsample(v, mid, vel);
    if (st) return st;
    return departure(g, pos, vel, dt, out);
}

template <class T>
bool all_finite(const T* v, int64_t n) {
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(double(v[i]))) return false;
    return true;
}

template <class T>
VelocitySampler<T> velocity_sampler(const Grid& g, const T* u, const T* v, const T* w) {
    VelocitySampler<T> s;
    s.c[0] = face_sampler(g, 0, u);
    s.c[1] = face_sampler(g, 1, v);
    s.c[2] = face_sampler(g, 2, w);
    return s;
}

// GridGeometry::face_position (src/geometry.rs:242-248).
inline void face_position(const Grid& g, int axis, const int64_t p[3], double out[3]) {
    for (int d = 0; d < 3; ++d) {
        double offset = (d == axis) ? 0.0 : 0.5;
        out[d] = g.o[d] + (double(p[d]) + offset) * g.h[d];
    }
}
inline void cell_position(const Grid& g, const int64_t p[3], double out[3]) {
    for (int d = 0; d < 3; ++d) out[d] = g.o[d] + (double(p[d]) + 0.5) * g.h[d];
}

// advect_velocity (src/advection.rs:28-68); TOut is the stored face type.
template <class T>
int advect_velocity(const Grid& g, const T* const in[3], double dt, T* const out[3], int threads) {
    if (!std::isfinite(dt) || dt <= 0.0) return ORC_INVALID_TIME_STEP;
    for (int a = 0; a < 3; ++a)
        if (!all_finite(in[a], g.flen[a])) return ORC_NONFINITE_INPUT;
    VelocitySampler<T> vs = velocity_sampler(g, in[0], in[1], in[2]);
    std::atomic<int> status{ORC_OK};
    for (int a = 0; a < 3; ++a) {
        Sampler<T> comp = face_sampler(g, a, in[a]);
        const int64_t* dims = g.fc[a];
        int64_t planes = dims[2];
        parallel_for(planes, threads, [&](int64_t k) {
            for (int64_t j = 0; j < dims[1]; ++j)
                for (int64_t i = 0; i < dims[0]; ++i) {
                    int64_t p[3] = {i, j, k};
                    T* dst = &out[a][face_index(g, a, i, j, k)];
                    if (p[a] == 0 || p[a] + 1 == dims[a]) {
                        *dst = T(0);
                        continue;
                    }
                    double pos[3], dep[3], value;
                    face_position(g, a, p, pos);
                    int st = backtrace(g, vs, pos, dt, dep);
                    if (!st) st = sample(comp, dep, &value);
                    if (st) {
                        record(status, st);
                        continue;
                    }
                    *dst = T(value);
                }
        });
        if (status.load()) return status.load();
    }
    return ORC_OK;
}

// advect_tracer (src/advection.rs:72-102), evaluated densely: the reference's
// zero-support skip is bit-identical to the dense computation (its own test
// advection_contract.rs:7-41 asserts that).
template <class V>
int advect_tracer(const Grid& g, const float* old, const V* const vel[3], double dt, float* out,
                  int threads) {
    if (!std::isfinite(dt) || dt <= 0.0) return ORC_INVALID_TIME_STEP;
    if (!all_finite(old, g.cells)) return ORC_NONFINITE_INPUT;
    for (int a = 0; a < 3; ++a)
        if (!all_finite(vel[a], g.flen[a])) return ORC_NONFINITE_INPUT;
    Sampler<float> scalar = cell_sampler(g, old);
    VelocitySampler<V> vs = velocity_sampler(g, vel[0], vel[1], vel[2]);
    std::atomic<int> status{ORC_OK};
    parallel_for(g.n[2], threads, [&](int64_t k) {
        for (int64_t j = 0; j < g.n[1]; ++j)
            for (int64_t i = 0; i < g.n[0]; ++i) {
                int64_t p[3] = {i, j, k};
                double pos[3], dep[3], value;
                cell_position(g, p, pos);
                int st = backtrace(g, vs, pos, dt, dep);
                if (!st) st = sample(scalar, dep, &value);
                if (st) {
                    record(status, st);
                    continue;
                }
                out[cell_index(g, i, j, k)] = float(value);
            }
    });
    return status.load();
}

// ----------------------------------------------------------------- operator
struct Operator {
    double area[3];
    double accel[3];
    double weight[3];
    double box_diagonals[64];
};

// PressureOperator::new (src/operator.rs:58-97).
int make_operator(const Grid& g, double density, Operator* op) {
    if (!std::isfinite(density) || density <= 0.0) return ORC_INVALID_ARGUMENT;
    const double* h = g.h;
    op->area[0] = h[1] * h[2];
    op->area[1] = h[0] * h[2];
    op->area[2] = h[0] * h[1];
    for (int d = 0; d < 3; ++d) {
        op->accel[d] = 1.0 / (density * h[d]);
        op->weight[d] = op->area[d] * op->accel[d];
        if (!std::isfinite(op->area[d]) || op->area[d] <= 0.0 || !std::isfinite(op->accel[d]) ||
            op->accel[d] <= 0.0 || !std::isfinite(op->weight[d]) || op->weight[d] <= 0.0)
            return ORC_INVALID_ARGUMENT;
    }
    for (int mask = 0; mask < 64; ++mask) {
        double value = 0.0;
        for (int side = 0; side < 6; ++side)
            if (mask & (1 << side)) value += op->weight[side / 2];
        op->box_diagonals[mask] = value;
    }
    return ORC_OK;
}

// PressureOperator::diagonal (src/operator.rs:813-822).
inline double diagonal(const Grid& g, const Operator& op, const int64_t c[3]) {
    int mask = 0;
    for (int d = 0; d < 3; ++d) {
        mask |= int(c[d] > 0) << (2 * d);
        mask |= int(c[d] + 1 < g.n[d]) << (2 * d + 1);
    }
    return op.box_diagonals[mask];
}

int validate_cells(const Grid& g, const double* v) {
    return all_finite(v, g.cells) ? ORC_OK : ORC_NONFINITE_INPUT;
}

// PressureOperator::validate_velocity (src/operator.rs:850-875).
template <class T>
int validate_velocity(const Grid& g, const T* const vel[3]) {
    for (int a = 0; a < 3; ++a) {
        if (!all_finite(vel[a], g.flen[a])) return ORC_NONFINITE_INPUT;
        const int64_t* dims = g.fc[a];
        for (int64_t k = 0; k < dims[2]; ++k)
            for (int64_t j = 0; j < dims[1]; ++j)
                for (int64_t i = 0; i < dims[0]; ++i) {
                    int64_t p[3] = {i, j, k};
                    if (p[a] == 0 || p[a] == g.n[a])
                        if (vel[a][face_index(g, a, i, j, k)] != T(0))
                            return ORC_NONZERO_WALL_VELOCITY;
                }
    }
    return ORC_OK;
}

// apply_full, sealed-box fast path (src/operator.rs:378-456).
int apply_full(const Grid& g, const Operator& op, const double* p, double* out, int threads) {
    const int64_t s[3] = {1, g.n[0], g.n[0] * g.n[1]};
    std::atomic<int> status{ORC_OK};
    parallel_for(g.n[2], threads, [&](int64_t k) {
        for (int64_t j = 0; j < g.n[1]; ++j)
            for (int64_t i = 0; i < g.n[0]; ++i) {
                int64_t c[3] = {i, j, k};
                int64_t row = cell_index(g, i, j, k);
                double value = 0.0;
                for (int d = 0; d < 3; ++d) {
                    if (c[d] > 0) value += op.weight[d] * (p[row] - p[row - s[d]]);
                    if (c[d] + 1 < g.n[d]) value += op.weight[d] * (p[row] - p[row + s[d]]);
                }
                if (!std::isfinite(value)) record(status, ORC_ARITHMETIC_FAILURE);
                out[row] = value;
            }
    });
    return status.load();
}

// build_rhs (src/operator.rs:460-509) and build_rhs_f64 (:672-708).
template <class T>
int build_rhs(const Grid& g, const Operator& op, const T* const vel[3], double dt, double* out) {
    if (!std::isfinite(dt) || dt <= 0.0) return ORC_INVALID_TIME_STEP;
    int st = validate_velocity(g, vel);
    if (st) return st;
    for (int64_t k = 0; k < g.n[2]; ++k)
        for (int64_t j = 0; j < g.n[1]; ++j)
            for (int64_t i = 0; i < g.n[0]; ++i) {
                int64_t p[3] = {i, j, k};
                double flux = 0.0;
                for (int a = 0; a < 3; ++a) {
                    int64_t up[3] = {i, j, k};
                    up[a] += 1;
                    int64_t lo = face_index(g, a, p[0], p[1], p[2]);
                    int64_t hi = face_index(g, a, up[0], up[1], up[2]);
                    flux += op.area[a] * (double(vel[a][lo]) - double(vel[a][hi]));
                }
                double value = flux / dt;
                if (!std::isfinite(value)) return ORC_ARITHMETIC_FAILURE;
                out[cell_index(g, i, j, k)] = value;
            }
    return ORC_OK;
}

// divergence (src/operator.rs:543-567): ((dx/h0 + dy/h1) + dz/h2).
int divergence_f32(const Grid& g, const float* const vel[3], double* out) {
    int st = validate_velocity(g, vel);
    if (st) return st;
    for (int64_t k = 0; k < g.n[2]; ++k)
        for (int64_t j = 0; j < g.n[1]; ++j)
            for (int64_t i = 0; i < g.n[0]; ++i) {
                double value =
                    (double(vel[0][face_index(g, 0, i + 1, j, k)]) -
                     double(vel[0][face_index(g, 0, i, j, k)])) / g.h[0] +
                    (double(vel[1][face_index(g, 1, i, j + 1, k)]) -
                     double(vel[1][face_index(g, 1, i, j, k)])) / g.h[1] +
                    (double(vel[2][face_index(g, 2, i, j, k + 1)]) -
                     double(vel[2][face_index(g, 2, i, j, k)])) / g.h[2];
                if (!std::isfinite(value)) return ORC_ARITHMETIC_FAILURE;
                out[cell_index(g, i, j, k)] = value;
            }
    return ORC_OK;
}

// divergence_f64 (src/operator.rs:711-742): value = 0; value += diff/h per axis.
int divergence_f64(const Grid& g, const double* const vel[3], double* out) {
    int st = validate_velocity(g, vel);
    if (st) return st;
    for (int64_t k = 0; k < g.n[2]; ++k)
        for (int64_t j = 0; j < g.n[1]; ++j)
            for (int64_t i = 0; i < g.n[0]; ++i) {
                int64_t p[3] = {i, j, k};
                double value = 0.0;
                for (int a = 0; a < 3; ++a) {
                    int64_t up[3] = {i, j, k};
                    up[a] += 1;
                    value += (vel[a][face_index(g, a, up[0], up[1], up[2])] -
                              vel[a][face_index(g, a, p[0], p[1], p[2])]) / g.h[a];
                }
                if (!std::isfinite(value)) return ORC_ARITHMETIC_FAILURE;
                out[cell_index(g, i, j, k)] = value;
            }
    return ORC_OK;
}

// correct_candidate_in_place (src/operator.rs:627-668):
//   u <- f32( f64(u) - (dt*accel)*(p_c - p_l) )
int correct_f32(const Grid& g, const Operator& op, const double* p, double dt, float* const vel[3]) {
    if (!std::isfinite(dt) || dt <= 0.0) return ORC_INVALID_TIME_STEP;
    const float* cv[3] = {vel[0], vel[1], vel[2]};
    int st = validate_velocity(g, cv);
    if (st) return st;
    if ((st = validate_cells(g, p))) return st;
    const int64_t s[3] = {1, g.n[0], g.n[0] * g.n[1]};
    for (int a = 0; a < 3; ++a) {
        const int64_t* dims = g.fc[a];
        for (int64_t k = 0; k < dims[2]; ++k)
            for (int64_t j = 0; j < dims[1]; ++j)
                for (int64_t i = 0; i < dims[0]; ++i) {
                    int64_t q[3] = {i, j, k};
                    if (q[a] == 0 || q[a] == g.n[a]) continue;
                    int64_t idx = face_index(g, a, i, j, k);
                    int64_t c = cell_index(g, i, j, k);
                    double difference = p[c] - p[c - s[a]];
                    double value = double(vel[a][idx]) - dt * op.accel[a] * difference;
                    if (!std::isfinite(value) || std::fabs(value) > kF32Max)
                        return ORC_ARITHMETIC_FAILURE;
                    vel[a][idx] = float(value);
                }
    }
    return ORC_OK;
}

// correct_candidate_f64 (src/operator.rs:746-781):
//   u <- u - dt*(accel*(p_c - p_l))
int correct_f64(const Grid& g, const Operator& op, const double* p, double dt, double* const vel[3]) {
    if (!std::isfinite(dt) || dt <= 0.0) return ORC_INVALID_TIME_STEP;
    const double* cv[3] = {vel[0], vel[1], vel[2]};
    int st = validate_velocity(g, cv);
    if (st) return st;
    if ((st = validate_cells(g, p))) return st;
    const int64_t s[3] = {1, g.n[0], g.n[0] * g.n[1]};
    for (int a = 0; a < 3; ++a) {
        const int64_t* dims = g.fc[a];
        for (int64_t k = 0; k < dims[2]; ++k)
            for (int64_t j = 0; j < dims[1]; ++j)
                for (int64_t i = 0; i < dims[0]; ++i) {
                    int64_t q[3] = {i, j, k};
                    if (q[a] == 0 || q[a] == g.n[a]) continue;
                    int64_t idx = face_index(g, a, i, j, k);
                    int64_t c = cell_index(g, i, j, k);
                    double gradient = op.accel[a] * (p[c] - p[c - s[a]]);
                    double value = vel[a][idx] - dt * gradient;
                    if (!std::isfinite(value)) return ORC_ARITHMETIC_FAILURE;
                    vel[a][idx] = value;
                }
    }
    return ORC_OK;
}

double dot(const double* a, const double* b, int64_t n) {
    Neumaier acc;
    for (int64_t i = 0; i < n; ++i) acc.add(a[i] * b[i]);
    return acc.result();
}

// precondition_jacobi (src/pressure.rs:534-575).
int precondition_jacobi(const Grid& g, const Operator& op, double* r, double* z, double* rz,
                        int threads) {
    r[0] = 0.0;
    z[0] = 0.0;
    std::atomic<int> status{ORC_OK};
    parallel_for(g.n[2], threads, [&](int64_t k) {
        for (int64_t j = 0; j < g.n[1]; ++j)
            for (int64_t i = 0; i < g.n[0]; ++i) {
                int64_t row = cell_index(g, i, j, k);
                if (row == 0) continue;
                int64_t c[3] = {i, j, k};
                double diag = diagonal(g, op, c);
                if (!std::isfinite(diag) || diag <= 0.0) record(status, ORC_BREAKDOWN);
                z[row] = r[row] / diag;
            }
    });
    if (status.load()) return status.load();
    *rz = dot(r, z, g.cells);
    return ORC_OK;
}

// precondition_sgs serial lexicographic (src/pressure.rs:467-532):
// M = (D+L) D^-1 (D+L)^T on the gauge-eliminated system.
int precondition_sgs(const Grid& g, const Operator& op, double* r, double* z, double* rz) {
    r[0] = 0.0;
    z[0] = 0.0;
    const int64_t nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int64_t s[3] = {1, nx, nx * ny};
    const int64_t n = g.cells;
    for (int64_t row = 1; row < n; ++row) {
        int64_t p[3] = {row % nx, (row / nx) % ny, row / (nx * ny)};
        double diag = diagonal(g, op, p);
        double value = r[row];
        for (int d = 0; d < 3; ++d)
            if (p[d] > 0) value += op.weight[d] * z[row - s[d]];
        z[row] = value / diag;
        if (!std::isfinite(z[row]) || diag <= 0.0 || !std::isfinite(diag)) return ORC_BREAKDOWN;
    }
    const int64_t counts[3] = {nx, ny, nz};
    for (int64_t row = n - 1; row >= 1; --row) {
        int64_t p[3] = {row % nx, (row / nx) % ny, row / (nx * ny)};
        double diag = diagonal(g, op, p);
        double correction = 0.0;
        for (int d = 0; d < 3; ++d)
            if (p[d] + 1 < counts[d]) correction += op.weight[d] * z[row + s[d]];
        z[row] = z[row] + correction / diag;
        if (!std::isfinite(z[row])) return ORC_BREAKDOWN;
    }
    *rz = dot(r, z, n);
    return ORC_OK;
}

int precondition(const Grid& g, const Operator& op, int method, double* r, double* z, double* rz,
                 int threads) {
    if (method == ORC_SGS_PCG_V1) return precondition_sgs(g, op, r, z, rz);
    return precondition_jacobi(g, op, r, z, rz, threads);
}

struct Workspace {
    std::vector<double> rhs, residual, direction, product, pre;
};

// true_report (src/pressure.rs:432-456).
int true_report(const Grid& g, const Operator& op, const double* pressure, Workspace& w, double dt,
                uint64_t iterations, orc_report* rep, int threads) {
    int st = apply_full(g, op, pressure, w.product.data(), threads);
    if (st) return st;
    for (int64_t i = 0; i < g.cells; ++i) w.product[i] = w.rhs[i] - w.product[i];
    double squared = dot(w.product.data(), w.product.data(), g.cells);
    double maximum = 0.0;
    for (int64_t i = 0; i < g.cells; ++i) maximum = fmax_r(maximum, std::fabs(w.product[i]));
    double divergence = maximum * dt / g.volume;
    if (!std::isfinite(squared) || !std::isfinite(divergence)) {
        rep->breakdown_iteration = iterations;
        return ORC_BREAKDOWN;
    }
    rep->iterations = iterations;
    rep->true_residual_l2 = std::sqrt(squared);
    rep->true_residual_max = maximum;
    rep->predicted_divergence_max = divergence;
    return ORC_OK;
}

// solve_loaded (src/pressure.rs:577-740) with a cold start (p = 0).
// `initial`, when not null, is the caller's initial pressure
// (solve_*_with_initial_pressure, feature "accepted-pressure-warm-start",
// src/pressure.rs:395-430 and :615-624, :697-704).
int solve_loaded(const Grid& g, const Operator& op, int method, Workspace& w, double* pressure,
                 double dt, const orc_settings& s, orc_report* rep, orc_trace* trace, size_t cap,
                 int threads, const double* initial) {
    const int64_t n = g.cells;
    if (!std::isfinite(dt) || dt <= 0.0) return ORC_INVALID_ARGUMENT;
    const double vals[3] = {s.relative_residual, s.absolute_residual, s.divergence_limit};
    for (double v : vals)
        if (!std::isfinite(v) || v < 0.0) return ORC_INVALID_ARGUMENT;
    Neumaier sum, sum_abs;
    for (int64_t i = 0; i < n; ++i) sum.add(w.rhs[i]);
    for (int64_t i = 0; i < n; ++i) sum_abs.add(std::fabs(w.rhs[i]));
    double total = sum.result(), total_abs = sum_abs.result();
    double budget = (64.0 * kEps) * total_abs;
    if (!std::isfinite(total) || !std::isfinite(total_abs)) {
        rep->breakdown_iteration = 0;
        return ORC_BREAKDOWN;
    }
    if (std::fabs(total) > budget) {
        rep->incompatible_sum = total;
        rep->incompatible_budget = budget;
        return ORC_INCOMPATIBLE_RHS;
    }
    if (initial) {
        // operator.validate_cells(initial), then the sealed gauge p[0] == 0.
        for (int64_t i = 0; i < n; ++i)
            if (!std::isfinite(initial[i])) return ORC_NONFINITE_INPUT;
        if (initial[0] != 0.0) return ORC_INVALID_INITIAL_PRESSURE;
        std::copy(initial, initial + n, pressure);
    } else {
        std::fill(pressure, pressure + n, 0.0);
    }
    double rhs_l2 = std::sqrt(dot(w.rhs.data(), w.rhs.data(), n));
    double threshold = fmax_r(s.absolute_residual, s.relative_residual * rhs_l2);
    if (!std::isfinite(rhs_l2) || !std::isfinite(threshold)) {
        rep->breakdown_iteration = 0;
        return ORC_BREAKDOWN;
    }
    auto accepted = [&](const orc_report& r) {
        return r.true_residual_l2 <= threshold && r.predicted_divergence_max <= s.divergence_limit;
    };
    int st = true_report(g, op, pressure, w, dt, 0, rep, threads);
    if (st) return st;
    if (accepted(*rep)) return ORC_OK;
    if (s.max_iterations == 0) return ORC_ITERATION_LIMIT;
    std::copy(w.product.begin(), w.product.end(), w.residual.begin());
    double rz = 0.0;
    if ((st = precondition(g, op, method, w.residual.data(), w.pre.data(), &rz, threads))) {
        rep->breakdown_iteration = 0;
        return st;
    }
    std::copy(w.pre.begin(), w.pre.end(), w.direction.begin());
    for (uint64_t it = 1; it <= s.max_iterations; ++it) {
        orc_trace* tr = (trace && it - 1 < cap) ? &trace[it - 1] : nullptr;
        if ((st = apply_full(g, op, w.direction.data(), w.product.data(), threads))) return st;
        w.product[0] = 0.0;
        double curvature = dot(w.direction.data(), w.product.data(), n);
        if (tr) tr->curvature = curvature;
        if (!std::isfinite(curvature) || curvature <= 0.0 || !std::isfinite(rz) || rz <= 0.0) {
            rep->breakdown_iteration = it;
            return ORC_BREAKDOWN;
        }
        double alpha = rz / curvature;
        if (tr) tr->alpha = alpha;
        if (!std::isfinite(alpha)) {
            rep->breakdown_iteration = it;
            return ORC_BREAKDOWN;
        }
        for (int64_t i = 1; i < n; ++i) {
            pressure[i] += alpha * w.direction[i];
            w.residual[i] -= alpha * w.product[i];
        }
        double recursive_l2 = std::sqrt(dot(w.residual.data(), w.residual.data(), n));
        if (tr) {
            tr->recursive_l2 = recursive_l2;
            tr->replaced = 0;
            tr->checked = 0;
        }
        bool candidate = recursive_l2 <= threshold;
        bool replaced = false;
        if (candidate || it == s.max_iterations) {
            if ((st = true_report(g, op, pressure, w, dt, it, rep, threads))) return st;
            if (tr) tr->checked = 1;
            if (accepted(*rep)) return ORC_OK;
            // A seeded solve judges the restart without the gauge row
            // (src/pressure.rs:697-704).
            double replacement_l2 = rep->true_residual_l2;
            if (initial) replacement_l2 = std::sqrt(dot(w.product.data() + 1, w.product.data() + 1, n - 1));
            if (replacement_l2 > threshold) {
                std::copy(w.product.begin(), w.product.end(), w.residual.begin());
                replaced = true;
            }
        }
        if (it == s.max_iterations) return ORC_ITERATION_LIMIT;
        double next_rz = 0.0;
        if ((st = precondition(g, op, method, w.residual.data(), w.pre.data(), &next_rz, threads))) {
            rep->breakdown_iteration = 0;
            return st;
        }
        if (tr) {
            tr->rz = next_rz;
            tr->replaced = replaced ? 1 : 0;
        }
        if (!std::isfinite(next_rz) || next_rz <= 0.0) {
            rep->breakdown_iteration = it;
            return ORC_BREAKDOWN;
        }
        if (replaced) {
            std::copy(w.pre.begin(), w.pre.end(), w.direction.begin());
            if (tr) tr->beta = 0.0;
        } else {
            double beta = next_rz / rz;
            if (tr) tr->beta = beta;
            for (int64_t i = 1; i < n; ++i) w.direction[i] = w.pre[i] + beta * w.direction[i];
        }
        rz = next_rz;
    }
    return ORC_ITERATION_LIMIT;
}

template <class T>
int velocity_rate(const Grid& g, const T* const vel[3], double* rate) {
    double total = 0.0;
    for (int a = 0; a < 3; ++a) {
        double m = 0.0;
        for (int64_t i = 0; i < g.flen[a]; ++i) m = fmax_r(m, std::fabs(double(vel[a][i])));
        total += m / g.h[a];
    }
    if (!std::isfinite(total)) return ORC_ARITHMETIC_FAILURE;
    *rate = total;
    return ORC_OK;
}

// Buoyancy forcing hook on interior Y faces: v += dt * g_b * 0.5*(c_below + c_above).
// New (the reference has no buoyancy model); it plugs in where apply_force
// (src/simulation.rs:1449-1472) acts: after advection, before the pressure stage.
template <class T>
int apply_buoyancy(const Grid& g, T* v, const float* tracer, double gb, double dt) {
    for (int64_t k = 0; k < g.n[2]; ++k)
        for (int64_t j = 1; j < g.n[1]; ++j)
            for (int64_t i = 0; i < g.n[0]; ++i) {
                double c = 0.5 * (double(tracer[cell_index(g, i, j - 1, k)]) +
                                  double(tracer[cell_index(g, i, j, k)]));
                int64_t f = face_index(g, 1, i, j, k);
                double value = double(v[f]) + dt * (gb * c);
                if (!std::isfinite(value)) return ORC_ARITHMETIC_FAILURE;
                v[f] = T(value);
            }
    return ORC_OK;
}

template <class T>
int carrier_step(const Grid& g, const orc_step_params* prm, T* u, T* v, T* w, float* tracer,
                 orc_step_report* rep, const double* initial, double* pressure_out) {
    std::memset(rep, 0, sizeof(*rep));
    Operator op;
    int st = make_operator(g, prm->density, &op);
    if (st) return st;
    const T* old[3] = {u, v, w};
    std::vector<T> nu(g.flen[0]), nv(g.flen[1]), nw(g.flen[2]);
    T* out[3] = {nu.data(), nv.data(), nw.data()};
    if ((st = velocity_rate(g, old, &rep->rate_before))) return st;
    if ((st = advect_velocity<T>(g, old, prm->dt, out, prm->threads))) return st;
    if (tracer && prm->buoyancy != 0.0)
        if ((st = apply_buoyancy(g, nv.data(), tracer, prm->buoyancy, prm->dt))) return st;
    Workspace ws;
    ws.rhs.assign(g.cells, 0.0);
    ws.residual.assign(g.cells, 0.0);
    ws.direction.assign(g.cells, 0.0);
    ws.product.assign(g.cells, 0.0);
    ws.pre.assign(g.cells, 0.0);
    const T* cand[3] = {nu.data(), nv.data(), nw.data()};
    if ((st = build_rhs<T>(g, op, cand, prm->dt, ws.rhs.data()))) return st;
    std::vector<double> pressure(g.cells, 0.0);
    st = solve_loaded(g, op, prm->method, ws, pressure.data(), prm->dt, prm->settings,
                      &rep->pressure, nullptr, 0, prm->threads, initial);
    rep->pressure_status = st;
    if (pressure_out) std::copy(pressure.begin(), pressure.end(), pressure_out);
    if (st && !(st == ORC_ITERATION_LIMIT && prm->iteration_limit_ok)) {
        std::copy(nu.begin(), nu.end(), u);
        std::copy(nv.begin(), nv.end(), v);
        std::copy(nw.begin(), nw.end(), w);
        return st;
    }
    T* corr[3] = {nu.data(), nv.data(), nw.data()};
    if constexpr (sizeof(T) == 4)
        st = correct_f32(g, op, pressure.data(), prm->dt, corr);
    else
        st = correct_f64(g, op, pressure.data(), prm->dt, corr);
    if (st) return st;
    std::vector<double> div(g.cells);
    if constexpr (sizeof(T) == 4)
        st = divergence_f32(g, cand, div.data());
    else
        st = divergence_f64(g, cand, div.data());
    if (st) return st;
    double mx = 0.0;
    for (double x : div) mx = fmax_r(mx, std::fabs(x));
    rep->actual_divergence_max = mx;
    double rate = 0.0;
    if ((st = velocity_rate(g, cand, &rate))) return st;
    rep->courant = prm->dt * rate;
    if (tracer) {
        std::vector<float> nt(g.cells);
        if ((st = advect_tracer<T>(g, tracer, cand, prm->dt, nt.data(), prm->threads))) return st;
        std::copy(nt.begin(), nt.end(), tracer);
    }
    std::copy(nu.begin(), nu.end(), u);
    std::copy(nv.begin(), nv.end(), v);
    std::copy(nw.begin(), nw.end(), w);
    return ORC_OK;
}

}  // namespace

extern "C" {

int orc_grid_validate(const orc_grid* in) {
    Grid g;
    return make_grid(in, &g);
}

int orc_sample(const orc_grid* in, int axis, const float* values, const double position[3],
               double* out) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    if (axis < 0 || axis > 3) return ORC_INVALID_ARGUMENT;
    Sampler<float> s = axis == 3 ? cell_sampler(g, values) : face_sampler(g, axis, values);
    int64_t len = axis == 3 ? g.cells : g.flen[axis];
    if (!all_finite(values, len)) return ORC_NONFINITE_INPUT;
    return sample(s, position, out);
}

int orc_backtrace(const orc_grid* in, const float* u, const float* v, const float* w,
                  const double position[3], double dt, double out[3]) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    VelocitySampler<float> vs = velocity_sampler(g, u, v, w);
    return backtrace(g, vs, position, dt, out);
}

int orc_advect_velocity_f32(const orc_grid* in, const float* u, const float* v, const float* w,
                            double dt, float* ou, float* ov, float* ow, int threads) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    const float* i3[3] = {u, v, w};
    float* o3[3] = {ou, ov, ow};
    return advect_velocity<float>(g, i3, dt, o3, threads);
}

int orc_advect_velocity_f64(const orc_grid* in, const double* u, const double* v, const double* w,
                            double dt, double* ou, double* ov, double* ow, int threads) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    const double* i3[3] = {u, v, w};
    double* o3[3] = {ou, ov, ow};
    return advect_velocity<double>(g, i3, dt, o3, threads);
}

int orc_advect_tracer_f32(const orc_grid* in, const float* old, const float* u, const float* v,
                          const float* w, double dt, float* out, int threads) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    const float* vel[3] = {u, v, w};
    return advect_tracer<float>(g, old, vel, dt, out, threads);
}

int orc_apply_full(const orc_grid* in, double density, const double* p, double* out, int threads) {
    Grid g;
    Operator op;
    int st = make_grid(in, &g);
    if (st || (st = make_operator(g, density, &op))) return st;
    if ((st = validate_cells(g, p))) return st;
    return apply_full(g, op, p, out, threads);
}

int orc_build_rhs_f32(const orc_grid* in, double density, const float* u, const float* v,
                      const float* w, double dt, double* out) {
    Grid g;
    Operator op;
    int st = make_grid(in, &g);
    if (st || (st = make_operator(g, density, &op))) return st;
    const float* vel[3] = {u, v, w};
    return build_rhs<float>(g, op, vel, dt, out);
}

int orc_build_rhs_f64(const orc_grid* in, double density, const double* u, const double* v,
                      const double* w, double dt, double* out) {
    Grid g;
    Operator op;
    int st = make_grid(in, &g);
    if (st || (st = make_operator(g, density, &op))) return st;
    const double* vel[3] = {u, v, w};
    return build_rhs<double>(g, op, vel, dt, out);
}

int orc_divergence_f32(const orc_grid* in, const float* u, const float* v, const float* w,
                       double* out) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    const float* vel[3] = {u, v, w};
    return divergence_f32(g, vel, out);
}

int orc_divergence_f64(const orc_grid* in, const double* u, const double* v, const double* w,
                       double* out) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    const double* vel[3] = {u, v, w};
    return divergence_f64(g, vel, out);
}

int orc_correct_f32(const orc_grid* in, double density, const double* p, double dt, float* u,
                    float* v, float* w) {
    Grid g;
    Operator op;
    int st = make_grid(in, &g);
    if (st || (st = make_operator(g, density, &op))) return st;
    float* vel[3] = {u, v, w};
    return correct_f32(g, op, p, dt, vel);
}

int orc_correct_f64(const orc_grid* in, double density, const double* p, double dt, double* u,
                    double* v, double* w) {
    Grid g;
    Operator op;
    int st = make_grid(in, &g);
    if (st || (st = make_operator(g, density, &op))) return st;
    double* vel[3] = {u, v, w};
    return correct_f64(g, op, p, dt, vel);
}

double orc_diagonal(const orc_grid* in, double density, const uint64_t coordinate[3]) {
    Grid g;
    Operator op;
    if (make_grid(in, &g) || make_operator(g, density, &op)) return NAN;
    int64_t c[3] = {int64_t(coordinate[0]), int64_t(coordinate[1]), int64_t(coordinate[2])};
    return diagonal(g, op, c);
}

double orc_compensated_sum(const double* values, size_t n) {
    Neumaier acc;
    for (size_t i = 0; i < n; ++i) acc.add(values[i]);
    return acc.result();
}

double orc_dot(const double* a, const double* b, size_t n) { return dot(a, b, int64_t(n)); }

int orc_precondition(const orc_grid* in, double density, int method, double* r, double* z,
                     double* rz) {
    Grid g;
    Operator op;
    int st = make_grid(in, &g);
    if (st || (st = make_operator(g, density, &op))) return st;
    return precondition(g, op, method, r, z, rz, 1);
}

int orc_solve_rhs(const orc_grid* in, double density, int method, const double* rhs, double dt,
                  const orc_settings* s, double* pressure_out, orc_report* report,
                  orc_trace* trace, size_t trace_capacity, int threads) {
    return orc_solve_rhs_initial(in, density, method, rhs, nullptr, dt, s, pressure_out, report, trace,
                                 trace_capacity, threads);
}

// PressureWorkspace::solve_rhs_with_initial_pressure (src/pressure.rs:415-430);
// initial == NULL is solve_rhs.
int orc_solve_rhs_initial(const orc_grid* in, double density, int method, const double* rhs,
                          const double* initial, double dt, const orc_settings* s, double* pressure_out,
                          orc_report* report, orc_trace* trace, size_t trace_capacity, int threads) {
    std::memset(report, 0, sizeof(*report));
    Grid g;
    Operator op;
    int st = make_grid(in, &g);
    if (st || (st = make_operator(g, density, &op))) return st;
    if ((st = validate_cells(g, rhs))) return st;
    Workspace w;
    w.rhs.assign(rhs, rhs + g.cells);
    w.residual.assign(g.cells, 0.0);
    w.direction.assign(g.cells, 0.0);
    w.product.assign(g.cells, 0.0);
    w.pre.assign(g.cells, 0.0);
    return solve_loaded(g, op, method, w, pressure_out, dt, *s, report, trace, trace_capacity,
                        threads < 1 ? 1 : threads, initial);
}

// ProviderWorkspace::solve_observed qualification (src/solver_provider.rs:239-270).
int orc_qualify_pressure(const orc_grid* in, double density, const double* rhs, double dt,
                         const orc_settings* s, const double* pressure, orc_report* report) {
    std::memset(report, 0, sizeof(*report));
    Grid g;
    Operator op;
    int st = make_grid(in, &g);
    if (st || (st = make_operator(g, density, &op))) return st;
    Neumaier sq;
    for (int64_t i = 0; i < g.cells; ++i) sq.add(rhs[i] * rhs[i]);
    double norm = std::sqrt(sq.result());
    double threshold = fmax_r(s->absolute_residual, s->relative_residual * norm);
    if (!all_finite(pressure, g.cells)) return ORC_NONFINITE_OUTPUT;
    if (pressure[0] != 0.0) return ORC_NONZERO_GAUGE;
    std::vector<double> product(g.cells);
    if (apply_full(g, op, pressure, product.data(), 1)) return ORC_NONFINITE_OUTPUT;
    for (int64_t i = 0; i < g.cells; ++i) product[i] = rhs[i] - product[i];
    Neumaier l2;
    for (int64_t i = 0; i < g.cells; ++i) l2.add(product[i] * product[i]);
    double l2v = std::sqrt(l2.result());
    double mx = 0.0;
    for (int64_t i = 0; i < g.cells; ++i) mx = fmax_r(mx, std::fabs(product[i]));
    double divergence = mx * dt / g.volume;
    report->true_residual_l2 = l2v;
    report->true_residual_max = mx;
    report->predicted_divergence_max = divergence;
    if (!std::isfinite(l2v) || !std::isfinite(divergence) || l2v > threshold ||
        divergence > s->divergence_limit)
        return ORC_QUALITY_GATE;
    return ORC_OK;
}

int orc_velocity_rate_f32(const orc_grid* in, const float* u, const float* v, const float* w,
                          double* rate) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    const float* vel[3] = {u, v, w};
    return velocity_rate(g, vel, rate);
}

int orc_velocity_rate_f64(const orc_grid* in, const double* u, const double* v, const double* w,
                          double* rate) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    const double* vel[3] = {u, v, w};
    return velocity_rate(g, vel, rate);
}

double orc_max_abs(const double* values, size_t n) {
    double m = 0.0;
    for (size_t i = 0; i < n; ++i) m = fmax_r(m, std::fabs(values[i]));
    return m;
}

int orc_carrier_step_f32(const orc_grid* in, const orc_step_params* prm, float* u, float* v,
                         float* w, float* tracer, orc_step_report* rep) {
    return orc_carrier_step_seeded_f32(in, prm, u, v, w, tracer, nullptr, nullptr, rep);
}

int orc_carrier_step_f64(const orc_grid* in, const orc_step_params* prm, double* u, double* v,
                         double* w, float* tracer, orc_step_report* rep) {
    return orc_carrier_step_seeded_f64(in, prm, u, v, w, tracer, nullptr, nullptr, rep);
}

int orc_carrier_step_seeded_f32(const orc_grid* in, const orc_step_params* prm, float* u, float* v,
                                float* w, float* tracer, const double* initial, double* pressure_out,
                                orc_step_report* rep) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    return carrier_step<float>(g, prm, u, v, w, tracer, rep, initial, pressure_out);
}

int orc_carrier_step_seeded_f64(const orc_grid* in, const orc_step_params* prm, double* u, double* v,
                                double* w, float* tracer, const double* initial, double* pressure_out,
                                orc_step_report* rep) {
    Grid g;
    int st = make_grid(in, &g);
    if (st) return st;
    return carrier_step<double>(g, prm, u, v, w, tracer, rep, initial, pressure_out);
}

}  // extern "C"
