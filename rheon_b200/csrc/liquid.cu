// Liquid-volume transport on the device: LiquidVolumeState::advance with an
// inlet boundary and the all-cells divergence domain
// (src/liquid_volume.rs:520-776), first-order shared-face donor transfer of
// the represented liquid fraction through the carrier's face velocities, with
// the reference's checked arithmetic, error precedence and volume ledger.
//
// One kernel does the face transfers, the cell update and every reduction:
// each cell computes the transfers of its six faces (a face shared by two
// cells is computed twice, with the same operations, so both see the same
// value), its Courant number and divergence, and its new fraction into the
// candidate array; the ledger sums (volume before and after, inward and
// outward boundary volume, source volume), maxima and occupancy counts are
// reduced in double-double per block and folded by the last block, which
// also decides the outcome. Errors follow the reference's order: a failed
// face transfer (ArithmeticFailure) before any cell error; among cells, the
// first failing cell in x-fastest order with its own first failure
// (ArithmeticFailure, CourantLimit, FractionBounds); then the divergence
// limit, the ledger's finiteness and the balance limit. The accepted array is
// only replaced by the host after success.
#include <cfloat>

#include "liquid.hpp"

namespace rb200 {
namespace {

constexpr int LQ_THREADS = kLiquidThreads;
constexpr int LQ_K = 8;  // dd sums: before, after, inward, outward, source, |source|, dry, full
constexpr int LQ_M = 4;  // maxima: courant, |div|, -fraction (min), fraction
constexpr int LQ_STRIDE = 2 * LQ_K + LQ_M;

// rb200_liquid_error codes used on the device
enum : int { LQ_ARITH = RB200_LIQUID_ARITHMETIC_FAILURE, LQ_COURANT = RB200_LIQUID_COURANT_LIMIT,
             LQ_BOUNDS = RB200_LIQUID_FRACTION_BOUNDS };

struct LqArgs {
    GridDev g;
    LiquidDev* L;
    const LiquidFlowDev* flow;
    LiquidScratch sc;
    rb200_liquid_report* out;
};

// The per-thread view of one interval: the inputs read once from device memory.
struct LqView {
    const double* acc;
    double* cand;
    const float* vel[3];
    const double* src;
    double dt, volume;
    double dta[3];            // dt * area_d (its checks are part of the decision)
    double rh[3], rvol;       // RN(1/h_d), RN(1/volume) for correctly rounded division (0: divide)
    double inlet[6];
    double max_courant;
    int periodic;
};

// product / quotient (src/liquid_volume.rs:879-896): overflow, a subnormal
// result or underflow to zero fails. A result passes when it is normal (its
// biased exponent is 1..2046), or an exact zero with a zero factor (product)
// or a zero dividend (quotient); the exponent test is integer work.
// Biased exponent field of v.
__device__ __forceinline__ unsigned exp_field(double v) { return (unsigned(__double2hiint(v)) >> 20) & 0x7ffu; }
// A product a * b fails when it is infinite or NaN (exponent 2047), or has
// exponent 0 (zero or subnormal) while neither factor is zero: a subnormal
// product has nonzero factors, and a zero one with nonzero factors underflowed.
__device__ __forceinline__ double prod_chk(double a, double b, bool& bad) {
    const double v = a * b;
    const unsigned e = exp_field(v);
    if (e == 0x7ffu || (e == 0u && a != 0.0 && b != 0.0)) bad = true;
    return v;
}
// A quotient fails when infinite or NaN, or with exponent 0 and a nonzero dividend.
__device__ __forceinline__ double quot_chk(double a, double b, bool& bad) {
    const double v = a / b;
    const unsigned e = exp_field(v);
    if (e == 0x7ffu || (e == 0u && a != 0.0)) bad = true;
    return v;
}
// The same quotient by a positive divisor b with yb = RN(1/b): div_diag
// gives the correctly rounded a / b (three operations in range, a division
// otherwise).
__device__ __forceinline__ double quot_chk_r(double a, double b, double yb, bool& bad) {
    const double v = div_diag(a, b, yb);
    const unsigned e = exp_field(v);
    if (e == 0x7ffu || (e == 0u && a != 0.0)) bad = true;
    return v;
}

struct CellOut {
    double fraction, courant, div;
    double inward, outward, source;
    int code;
    bool face_bad, vel_bad, src_bad;
};

// Cell update (src/liquid_volume.rs:642-699) of cell (i, j, k), with the
// transfers of its six faces (src/liquid_volume.rs:587-639): the upwind donor
// fraction (the inlet's outside fraction on inflow through the box) times
// dt * area and the velocity. Donors are chosen by selects from the cell's
// and its neighbours' fractions (indices clamped at the box), so that lanes
// of a warp do not diverge on the velocity signs.
__device__ __forceinline__ CellOut liquid_cell(const GridDev& g, const LqView& a, int i, int j, int k) {
    CellOut o{};
    const int nx = g.n[0], ny = g.n[1];
    const int c = i + nx * (j + ny * k);
    const int p[3] = {i, j, k};
    const int stride[3] = {1, nx, nx * ny};
    // the lower face of the cell on each axis; the upper one is stride[d] further
    const int low[3] = {i + (nx + 1) * (j + ny * k), i + nx * (j + (ny + 1) * k), c};
    o.src_bad = a.src && !isfinite(a.src[c]);
    const double fc = a.acc[c];
    bool bad = false;
    double amount = prod_chk(a.volume, fc, bad);
    double courant = 0.0, div = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float fa = a.vel[d][low[d]];
        const float fb = a.vel[d][low[d] + stride[d]];
        o.vel_bad |= !isfinite(fa) || !isfinite(fb);
        const double va = double(fa), vb = double(fb);
        const bool first = p[d] == 0, last = p[d] + 1 == g.n[d];
        // periodic: the cell across the seam, and the seam's lower face (whose
        // transfer the upper one repeats, src/liquid_volume.rs:570-577)
        const int wrap = (g.n[d] - 1) * stride[d];
        const double fm = a.acc[first ? (a.periodic ? c + wrap : c) : c - stride[d]];
        const double fp = a.acc[last ? (a.periodic ? c - wrap : c) : c + stride[d]];
        const double dl = va > 0.0 ? (first && !a.periodic ? a.inlet[2 * d] : fm) : (va < 0.0 ? fc : 0.0);
        const double tl = prod_chk(prod_chk(a.dta[d], va, o.face_bad), dl, o.face_bad);
        double th;
        if (last && a.periodic) {
            const int fstride = d == 0 ? 1 : (d == 1 ? nx : nx * ny);
            const double vs = double(a.vel[d][low[d] + stride[d] - g.n[d] * fstride]);
            const double ds = vs > 0.0 ? fc : (vs < 0.0 ? fp : 0.0);
            th = prod_chk(prod_chk(a.dta[d], vs, o.face_bad), ds, o.face_bad);
        } else {
            const double dh = vb > 0.0 ? fc : (vb < 0.0 ? (last ? a.inlet[2 * d + 1] : fp) : 0.0);
            th = prod_chk(prod_chk(a.dta[d], vb, o.face_bad), dh, o.face_bad);
        }
        amount += tl - th;
        // boundary faces owned by this cell: inward / outward volume
        // (:739-757); a periodic box has none
        if (first && !a.periodic) {
            const double value = -tl;
            if (value < 0.0)
                o.inward += -value;
            else
                o.outward += value;
        }
        if (last && !a.periodic) {
            if (th < 0.0)
                o.inward += -th;
            else
                o.outward += th;
        }
        courant += quot_chk_r(prod_chk(a.dt, fmax(vb, 0.0) - fmin(va, 0.0), bad), g.h[d], a.rh[d], bad);
        div += quot_chk_r(vb - va, g.h[d], a.rh[d], bad);
    }
    o.courant = courant;
    o.div = div;
    if (bad || !isfinite(courant) || !isfinite(div)) {
        o.code = LQ_ARITH;
        return o;
    }
    if (courant > a.max_courant) {
        o.code = LQ_COURANT;
        return o;
    }
    bool bad2 = false;
    if (a.src) {
        o.source = prod_chk(a.dt, a.src[c], bad2);
        amount += o.source;
    }
    const double fraction = quot_chk_r(amount, a.volume, a.rvol, bad2);
    o.fraction = fraction;
    if (bad2) {
        o.code = LQ_ARITH;
        return o;
    }
    if (!(fraction >= 0.0 && fraction <= 1.0)) {
        o.code = LQ_BOUNDS;
        return o;
    }
    prod_chk(a.volume, fraction, bad2);
    if (bad2) o.code = LQ_ARITH;
    return o;
}

__device__ __forceinline__ bool dev_product(double a, double b, double& v) {
    bool bad = false;
    v = prod_chk(a, b, bad);
    return !bad;
}

__device__ __forceinline__ void lq_error(rb200_liquid_report& r, int code, unsigned long long cell = 0,
                                         double actual = 0.0, double limit = 0.0) {
    r.error = code;
    r.error_cell = cell;
    r.error_actual = actual;
    r.error_limit = limit;
}

// The outcome of one interval, in the reference's order: the checks of
// LiquidFlowInterval::new (:123-150), LiquidInlet::new (:84-96) and
// LiquidVolumeSource::new (:185-190) as a caller constructing them meets
// them, then prepare_with_boundary (:520-529, validate_advance :485-506), the
// face transfers, the first failing cell, the divergence limit and the ledger
// (:700-776). Thread 0 of the last block.
__device__ void liquid_decide(const GridDev& g, const LiquidDev& L, const LiquidFlowDev& f, const LqView& v,
                              const dd (&sums)[LQ_K], const double (&maxs)[LQ_M], const int* flags,
                              unsigned long long first, unsigned long long seam, const CellOut& fc,
                              rb200_liquid_report& r) {
    r = rb200_liquid_report{};
    const double start = f.start, dt = f.dt;
    if (!isfinite(start) || start < 0.0 || !isfinite(dt) || dt <= 0.0) return lq_error(r, RB200_LIQUID_INVALID_TIME_STEP);
    const double end = start + dt;
    if (!isfinite(end) || end <= start) return lq_error(r, RB200_LIQUID_TIME_RESOLUTION);
    if (flags[1]) return lq_error(r, RB200_LIQUID_NONFINITE_VELOCITY);
    if (!f.periodic)
        for (int q = 0; q < 6; ++q)
            if (!isfinite(f.inlet_fraction[q]) || !(f.inlet_fraction[q] >= 0.0 && f.inlet_fraction[q] <= 1.0))
                return lq_error(r, RB200_LIQUID_INVALID_INLET);
    if (flags[2]) return lq_error(r, RB200_LIQUID_INVALID_SOURCE);
    if (__double_as_longlong(start) != __double_as_longlong(L.time)) return lq_error(r, RB200_LIQUID_TIME_MISMATCH);
    if (!isfinite(f.max_courant) || f.max_courant <= 0.0 || f.max_courant > 1.0 || !isfinite(f.divergence_limit) ||
        f.divergence_limit < 0.0)
        return lq_error(r, RB200_LIQUID_INVALID_SETTINGS);
    if (L.version == ~0ull) return lq_error(r, RB200_LIQUID_VERSION_OVERFLOW);
    if (f.periodic && seam != ~0ull)
        return lq_error(r, RB200_LIQUID_PERIODIC_VELOCITY_MISMATCH, seam & ((1ull << 40) - 1), double(seam >> 40));
    const double sides[3][2] = {{g.h[1], g.h[2]}, {g.h[0], g.h[2]}, {g.h[0], g.h[1]}};
    for (int d = 0; d < 3; ++d) {
        double area = 0.0, dta = 0.0;
        if (!dev_product(sides[d][0], sides[d][1], area) || !dev_product(dt, area, dta))
            return lq_error(r, RB200_LIQUID_ARITHMETIC_FAILURE);
    }
    if (flags[0]) return lq_error(r, RB200_LIQUID_ARITHMETIC_FAILURE);
    if (first != ~0ull) {
        if (fc.code == LQ_COURANT) return lq_error(r, LQ_COURANT, first, fc.courant, f.max_courant);
        if (fc.code == LQ_BOUNDS) return lq_error(r, LQ_BOUNDS, first, fc.fraction);
        return lq_error(r, RB200_LIQUID_ARITHMETIC_FAILURE);
    }
    const double max_div = maxs[1];
    if (max_div > f.divergence_limit) return lq_error(r, RB200_LIQUID_DIVERGENCE_LIMIT, 0, max_div, f.divergence_limit);
    const double before = dd_value(sums[0]), after = dd_value(sums[1]);
    const double inward = dd_value(sums[2]), outward = dd_value(sums[3]);
    const double source_total = dd_value(sums[4]), source_abs = dd_value(sums[5]);
    const double balance = after - before + outward - inward - source_total;
    const double budget = (64.0 * DBL_EPSILON) * (fabs(before) + fabs(after) + outward + inward + source_abs);
    double mass_before = 0.0, mass_after = 0.0;
    bool ok = dev_product(L.density, before, mass_before);
    ok = ok && dev_product(L.density, after, mass_after);
    const double ledger[9] = {before, after, inward, outward, source_total, balance, budget, mass_before, mass_after};
    for (double x : ledger) ok = ok && isfinite(x);
    if (!ok) return lq_error(r, RB200_LIQUID_ARITHMETIC_FAILURE);
    if (fabs(balance) > budget) return lq_error(r, RB200_LIQUID_BALANCE_LIMIT, 0, balance, budget);
    r.stamp = rb200_liquid_stamp{L.id, L.version + 1};
    r.flow = f.flow;
    r.inlet = f.inlet;
    r.has_source = f.src ? 1 : 0;
    r.periodic = f.periodic;
    if (f.src) r.source = f.source;
    r.dt = dt;
    r.time = end;
    r.liquid_volume_before = before;
    r.liquid_volume_after = after;
    r.inward_boundary_volume = inward;
    r.outward_boundary_volume = outward;
    r.source_volume = source_total;
    r.volume_balance_error = balance;
    r.volume_rounding_budget = budget;
    r.liquid_mass_before = mass_before;
    r.liquid_mass_after = mass_after;
    r.max_outward_courant = maxs[0];
    r.actual_divergence_max = max_div;
    r.fraction_min = fmin(1.0, -maxs[2]);
    r.fraction_max = fmax(0.0, maxs[3]);
    r.dry_cells = (unsigned long long)dd_value(sums[6]);
    r.full_cells = (unsigned long long)dd_value(sums[7]);
    r.mixed_cells = (unsigned long long)g.cells - r.dry_cells - r.full_cells;
}

// Block maxima into thread 0 (lanes beyond the block's warps count as -inf,
// so that the negated minimum survives).
__device__ __forceinline__ void block_max(double (&m)[LQ_M], double (*sm)[LQ_M]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < LQ_M; ++q) m[q] = warp_reduce_max(m[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < LQ_M; ++q) sm[warp][q] = m[q];
    __syncthreads();
    if (warp == 0)
#pragma unroll
        for (int q = 0; q < LQ_M; ++q) m[q] = warp_reduce_max(lane < LQ_THREADS / 32 ? sm[lane][q] : -INFINITY);
    __syncthreads();
}

__global__ void __launch_bounds__(LQ_THREADS) k_liquid_advance(LqArgs a) {
    __shared__ BlockReduce<LQ_K, 0> red;
    __shared__ double smax[32][LQ_M];
    __shared__ bool last;
    const LiquidFlowDev& f = *a.flow;
    if (!f.active) return;
    const GridDev& g = a.g;
    LqView v;
    v.acc = a.L->frac[a.L->acc];
    v.cand = a.L->frac[a.L->acc ^ 1];
    for (int d = 0; d < 3; ++d) v.vel[d] = f.vel[d];
    v.src = f.src;
    v.dt = f.dt;
    v.volume = a.L->volume;
    v.dta[0] = f.dt * (g.h[1] * g.h[2]);
    v.dta[1] = f.dt * (g.h[0] * g.h[2]);
    v.dta[2] = f.dt * (g.h[0] * g.h[1]);
    for (int q = 0; q < 6; ++q) v.inlet[q] = f.inlet_fraction[q];
    v.max_courant = f.max_courant;
    v.periodic = f.periodic;
    for (int d = 0; d < 3; ++d) v.rh[d] = a.L->rh[d];
    v.rvol = a.L->rvolume;
    dd sums[LQ_K];
    double maxs[LQ_M] = {0.0, 0.0, -INFINITY, -INFINITY};
#pragma unroll
    for (int q = 0; q < LQ_K; ++q) sums[q] = dd{0.0, 0.0};
    bool face_bad = false, vel_bad = false, src_bad = false;
    unsigned dry = 0u, full = 0u;
    const int n0 = g.n[0], n01 = g.n[0] * g.n[1];
    // one warp per row (j, k) of cells, lanes along x: coalesced accesses and
    // one division per row instead of two per cell
    const int rows = g.n[1] * g.n[2];
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (LQ_THREADS / 32);
    for (int row = blockIdx.x * (LQ_THREADS / 32) + (threadIdx.x >> 5); row < rows; row += warps)
    for (int i = lane; i < n0; i += 32) {
        const int k = row / g.n[1], j = row - k * g.n[1];
        const int c = i + n0 * row;
        if (v.periodic) {
            // seams (src/liquid_volume.rs:530-554): a lower boundary face and
            // its upper partner carry the same velocity
            const int p3[3] = {i, j, k};
            const int low3[3] = {i + (n0 + 1) * (j + g.n[1] * k), i + n0 * (j + (g.n[1] + 1) * k), c};
            const int fs3[3] = {1, n0, n01};
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (p3[d] == 0 && v.vel[d][low3[d]] != v.vel[d][low3[d] + g.n[d] * fs3[d]])
                    atomicMin(a.sc.first + 1, ((unsigned long long)d << 40) | (unsigned long long)low3[d]);
        }
        const CellOut o = liquid_cell(g, v, i, j, k);
        face_bad |= o.face_bad;
        vel_bad |= o.vel_bad;
        src_bad |= o.src_bad;
        if (o.code) {
            atomicMin(a.sc.first, (unsigned long long)c);
            continue;
        }
        v.cand[c] = o.fraction;
        sums[0] = dd_add1(sums[0], v.volume * v.acc[c]);
        sums[1] = dd_add1(sums[1], v.volume * o.fraction);
        if (i == 0 || j == 0 || k == 0 || i + 1 == g.n[0] || j + 1 == g.n[1] || k + 1 == g.n[2]) {
            sums[2] = dd_add1(sums[2], o.inward);
            sums[3] = dd_add1(sums[3], o.outward);
        }
        if (v.src) {
            sums[4] = dd_add1(sums[4], o.source);
            sums[5] = dd_add1(sums[5], fabs(o.source));
        }
        dry += o.fraction == 0.0 ? 1u : 0u;
        full += o.fraction == 1.0 ? 1u : 0u;
        maxs[0] = fmax(maxs[0], o.courant);
        maxs[1] = fmax(maxs[1], fabs(o.div));
        maxs[2] = fmax(maxs[2], -o.fraction);
        maxs[3] = fmax(maxs[3], o.fraction);
    }
    if (__syncthreads_or(face_bad) && threadIdx.x == 0) atomicOr(&a.sc.flags[0], 1);
    if (__syncthreads_or(vel_bad) && threadIdx.x == 0) atomicOr(&a.sc.flags[1], 1);
    if (__syncthreads_or(src_bad) && threadIdx.x == 0) atomicOr(&a.sc.flags[2], 1);
    // occupancy counts (exact in a double: fewer than 2^53 cells)
    sums[6] = dd{double(__reduce_add_sync(0xffffffffu, dry)), 0.0};
    sums[7] = dd{double(__reduce_add_sync(0xffffffffu, full)), 0.0};
    if ((threadIdx.x & 31) != 0) sums[6] = sums[7] = dd{0.0, 0.0};
    double none[1] = {0.0};
    block_reduce<LQ_K, 0>(red, sums, none);
    block_max(maxs, smax);
    if (threadIdx.x == 0) {
        double* slot = a.sc.part + size_t(blockIdx.x) * LQ_STRIDE;
#pragma unroll
        for (int q = 0; q < LQ_K; ++q) {
            slot[2 * q] = sums[q].hi;
            slot[2 * q + 1] = sums[q].lo;
        }
#pragma unroll
        for (int q = 0; q < LQ_M; ++q) slot[2 * LQ_K + q] = maxs[q];
        __threadfence();
        last = atomicAdd(a.sc.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block folds every block's partials and decides
    __threadfence();
#pragma unroll
    for (int q = 0; q < LQ_K; ++q) sums[q] = dd{0.0, 0.0};
    maxs[0] = maxs[1] = 0.0;
    maxs[2] = maxs[3] = -INFINITY;
    for (int b = threadIdx.x; b < int(gridDim.x); b += LQ_THREADS) {
        const double* slot = a.sc.part + size_t(b) * LQ_STRIDE;
#pragma unroll
        for (int q = 0; q < LQ_K; ++q) sums[q] = dd_add(sums[q], dd{__ldcg(slot + 2 * q), __ldcg(slot + 2 * q + 1)});
#pragma unroll
        for (int q = 0; q < LQ_M; ++q) maxs[q] = fmax(maxs[q], __ldcg(slot + 2 * LQ_K + q));
    }
    block_reduce<LQ_K, 0>(red, sums, none);
    block_max(maxs, smax);
    if (threadIdx.x == 0) {
        int flags[3];
        for (int q = 0; q < 3; ++q) flags[q] = __ldcg(&a.sc.flags[q]);
        const unsigned long long first = __ldcg(a.sc.first);
        const unsigned long long seam = __ldcg(a.sc.first + 1);
        CellOut fc{};
        if (first != ~0ull) {
            const int c = int(first);
            const int kk = c / n01, rr = c - kk * n01, jj = rr / n0, ii = rr - jj * n0;
            fc = liquid_cell(g, v, ii, jj, kk);
        }
        liquid_decide(g, *a.L, f, v, sums, maxs, flags, first, seam, fc, *a.out);
        // scratch back to its idle state for the next interval
        *a.sc.ticket = 0u;
        a.sc.first[0] = ~0ull;
        a.sc.first[1] = ~0ull;
        for (int q = 0; q < 4; ++q) a.sc.flags[q] = 0;
    }
}

__global__ void k_liquid_commit(LiquidDev* L, const rb200_liquid_report* r) {
    if (r->error == 0 && r->stamp.version != 0) liquid_commit(L, *r);
}

// LiquidVolumeState::new checks of the fraction (src/liquid_volume.rs:284-305)
// on the device: the first invalid cell, or a failing cell-volume product,
// and the initial volume (double-double).
__global__ void __launch_bounds__(LQ_THREADS) k_liquid_check_state(GridDev g, const double* f, double volume,
                                                                   unsigned long long* first_bad,
                                                                   int* arith, double* part, unsigned* ticket,
                                                                   double* total) {
    __shared__ BlockReduce<1, 0> red;
    __shared__ bool last;
    dd s[1] = {dd{0.0, 0.0}};
    double none[1] = {0.0};
    bool bad_arith = false;
    for (int c = blockIdx.x * LQ_THREADS + threadIdx.x; c < g.cells; c += gridDim.x * LQ_THREADS) {
        const double x = f[c];
        if (!isfinite(x) || !(x >= 0.0 && x <= 1.0)) {
            atomicMin(first_bad, (unsigned long long)c);
            continue;
        }
        bool bad = false;
        prod_chk(volume, x, bad);
        bad_arith |= bad;
        s[0] = dd_add1(s[0], volume * x);
    }
    if (__syncthreads_or(bad_arith) && threadIdx.x == 0) atomicOr(arith, 1);
    block_reduce<1, 0>(red, s, none);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s[0].hi;
        part[2 * blockIdx.x + 1] = s[0].lo;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    s[0] = dd{0.0, 0.0};
    for (int b = threadIdx.x; b < int(gridDim.x); b += LQ_THREADS)
        s[0] = dd_add(s[0], dd{__ldcg(part + 2 * b), __ldcg(part + 2 * b + 1)});
    block_reduce<1, 0>(red, s, none);
    if (threadIdx.x == 0) {
        *total = dd_value(s[0]);
        *ticket = 0u;
    }
}

bool host_product(double a, double b, double* out) {
    const double v = a * b;
    *out = v;
    return std::isfinite(v) && !(v != 0.0 && std::fabs(v) < DBL_MIN) && !(v == 0.0 && a != 0.0 && b != 0.0);
}

}  // namespace

int liquid_blocks(const GridDev& g) {
    return std::max(1, std::min((g.cells + LQ_THREADS - 1) / LQ_THREADS, 148 * 8));
}

size_t liquid_partial_doubles(int blocks) { return size_t(blocks) * LQ_STRIDE; }

cudaError_t launch_liquid_advance(const GridDev& g, LiquidDev* L, const LiquidFlowDev* flow, const LiquidScratch& sc,
                                  int blocks, rb200_liquid_report* report, cudaStream_t stream) {
    LqArgs a{g, L, flow, sc, report};
    k_liquid_advance<<<blocks, LQ_THREADS, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_liquid_commit(LiquidDev* L, const rb200_liquid_report* report, cudaStream_t stream) {
    k_liquid_commit<<<1, 1, 0, stream>>>(L, report);
    return cudaGetLastError();
}

// Allocation of the scratch of one advance, in its idle state.
int liquid_scratch_alloc(LiquidScratch* sc, int blocks, cudaStream_t s) {
    if (cudaMalloc(&sc->part, liquid_partial_doubles(blocks) * 8) != cudaSuccess ||
        cudaMalloc(&sc->ticket, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&sc->first, 2 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&sc->flags, 4 * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return RB200_OUT_OF_MEMORY;
    }
    RB200_CUDA(cudaMemsetAsync(sc->ticket, 0, sizeof(unsigned), s));
    RB200_CUDA(cudaMemsetAsync(sc->first, 0xff, 2 * sizeof(unsigned long long), s));
    RB200_CUDA(cudaMemsetAsync(sc->flags, 0, 4 * sizeof(int), s));
    return RB200_OK;
}

void liquid_scratch_free(LiquidScratch* sc) {
    cudaFree(sc->part);
    cudaFree(sc->ticket);
    cudaFree(sc->first);
    cudaFree(sc->flags);
    *sc = LiquidScratch{};
}

// LiquidVolumeState::new (src/liquid_volume.rs:276-351) into device memory:
// fraction (host or device) copied to frac[0], validated on the device.
int liquid_state_create(const GridDev& g, double density, rb200_liquid_stamp stamp, double time,
                        const double* fraction, uint64_t limit, LiquidDev* h, LiquidDev** d, LiquidScratch* sc,
                        int* blocks, rb200_liquid_report* error, cudaStream_t s) {
    std::memset(h, 0, sizeof(*h));
    *d = nullptr;
    if (error) std::memset(error, 0, sizeof(*error));
    auto reject = [&](int code, uint64_t cell = 0, double actual = 0.0, double lim = 0.0) {
        if (error) {
            error->error = code;
            error->error_cell = cell;
            error->error_actual = actual;
            error->error_limit = lim;
        }
        return RB200_LIQUID_REJECTED;
    };
    if (!std::isfinite(density) || density <= 0.0) return reject(RB200_LIQUID_INVALID_DENSITY);
    // accepted and candidate fractions (the reference also counts three
    // face-transfer arrays, which the device does not keep)
    const uint64_t required = 2ull * uint64_t(g.cells) * 8ull;
    if (required > limit) return reject(RB200_LIQUID_BUFFER_LIMIT, 0, double(required), double(limit));
    *blocks = liquid_blocks(g);
    const size_t n = size_t(g.cells);
    h->density = density;
    h->volume = g.h[0] * g.h[1] * g.h[2];
    // reciprocals for div_diag's correctly rounded division (its range: 2^-500 < divisor < 2^500)
    auto recip = [](double x) { return (x > 0x1p-500 && x < 0x1p500) ? 1.0 / x : 0.0; };
    for (int d = 0; d < 3; ++d) h->rh[d] = recip(g.h[d]);
    h->rvolume = recip(h->volume);
    h->id = stamp.id;
    h->version = stamp.version;
    h->time = time;
    if (cudaMalloc(&h->frac[0], n * 8) != cudaSuccess || cudaMalloc(&h->frac[1], n * 8) != cudaSuccess ||
        cudaMalloc(d, sizeof(LiquidDev)) != cudaSuccess || liquid_scratch_alloc(sc, *blocks, s) != RB200_OK) {
        cudaGetLastError();
        return RB200_OUT_OF_MEMORY;
    }
    RB200_CUDA(cudaMemcpyAsync(h->frac[0], fraction, n * 8, cudaMemcpyDefault, s));
    RB200_CUDA(cudaMemsetAsync(h->frac[1], 0, n * 8, s));
    RB200_CUDA(cudaMemcpyAsync(*d, h, sizeof(LiquidDev), cudaMemcpyHostToDevice, s));
    double* total = sc->part + liquid_partial_doubles(*blocks) - 1;
    k_liquid_check_state<<<*blocks, LQ_THREADS, 0, s>>>(g, h->frac[0], h->volume, sc->first, sc->flags, sc->part,
                                                        sc->ticket, total);
    RB200_CUDA(cudaGetLastError());
    unsigned long long bad = 0;
    int arith = 0;
    double initial = 0.0;
    RB200_CUDA(cudaMemcpyAsync(&bad, sc->first, sizeof(bad), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaMemcpyAsync(&arith, sc->flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaMemcpyAsync(&initial, total, sizeof(double), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaMemsetAsync(sc->first, 0xff, sizeof(unsigned long long), s));
    RB200_CUDA(cudaMemsetAsync(sc->flags, 0, 4 * sizeof(int), s));
    RB200_CUDA(cudaStreamSynchronize(s));
    double mass = 0.0;
    if (bad != ~0ull) return reject(RB200_LIQUID_INVALID_FRACTION, bad);
    if (arith || !std::isfinite(initial) || !host_product(density, initial, &mass))
        return reject(RB200_LIQUID_ARITHMETIC_FAILURE);
    return RB200_OK;
}

void liquid_state_free(LiquidDev* h, LiquidDev* d, LiquidScratch* sc) {
    cudaFree(h->frac[0]);
    cudaFree(h->frac[1]);
    cudaFree(d);
    liquid_scratch_free(sc);
}

}  // namespace rb200

using namespace rb200;

struct rb200_liquid_volume {
    int device = 0;
    GridDev g{};
    LiquidDev* h_L = nullptr;        // pinned mirror of the device bookkeeping
    LiquidDev* d_L = nullptr;
    LiquidFlowDev* h_flow = nullptr; // pinned
    LiquidFlowDev* d_flow = nullptr;
    rb200_liquid_report* h_rep = nullptr;  // pinned
    rb200_liquid_report* d_rep = nullptr;
    LiquidScratch sc{};
    int blocks = 0;
    cudaStream_t stream = nullptr;
    ~rb200_liquid_volume() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        if (h_L) liquid_state_free(h_L, d_L, &sc);
        cudaFree(d_flow);
        cudaFree(d_rep);
        if (h_L) cudaFreeHost(h_L);
        if (h_flow) cudaFreeHost(h_flow);
        if (h_rep) cudaFreeHost(h_rep);
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

int rb200_liquid_create(const rb200_grid* grid, double density, rb200_liquid_stamp stamp, const double* fraction,
                        uint64_t limit, int device, rb200_liquid_volume** out, rb200_liquid_report* error) {
    if (!grid || !fraction || !out) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    if (error) std::memset(error, 0, sizeof(*error));
    GridDev g;
    int rc = make_grid_dev(grid, 1.0, &g);
    if (rc) return rc;
    RB200_CUDA(cudaSetDevice(device));
    auto* V = new rb200_liquid_volume();
    V->device = device;
    V->g = g;
    if (cudaStreamCreateWithFlags(&V->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost(&V->h_L, sizeof(LiquidDev)) != cudaSuccess ||
        cudaMallocHost(&V->h_flow, sizeof(LiquidFlowDev)) != cudaSuccess ||
        cudaMallocHost(&V->h_rep, sizeof(rb200_liquid_report)) != cudaSuccess ||
        cudaMalloc(&V->d_flow, sizeof(LiquidFlowDev)) != cudaSuccess ||
        cudaMalloc(&V->d_rep, sizeof(rb200_liquid_report)) != cudaSuccess) {
        delete V;
        cudaGetLastError();
        return RB200_OUT_OF_MEMORY;
    }
    rc = liquid_state_create(g, density, stamp, 0.0, fraction, limit, V->h_L, &V->d_L, &V->sc, &V->blocks, error,
                             V->stream);
    if (rc) {
        delete V;
        return rc;
    }
    *out = V;
    return RB200_OK;
}

void rb200_liquid_destroy(rb200_liquid_volume* V) { delete V; }

uint64_t rb200_liquid_allocated_bytes(const rb200_liquid_volume* V) { return V ? 2ull * uint64_t(V->g.cells) * 8 : 0; }

int rb200_liquid_state(const rb200_liquid_volume* V, const double** fraction, rb200_liquid_stamp* stamp,
                       double* time) {
    if (!V) return RB200_INVALID_ARGUMENT;
    if (fraction) *fraction = V->h_L->frac[V->h_L->acc];
    if (stamp) *stamp = rb200_liquid_stamp{V->h_L->id, V->h_L->version};
    if (time) *time = V->h_L->time;
    return RB200_OK;
}

int rb200_liquid_download(rb200_liquid_volume* V, double* out, size_t len) {
    if (!V || !out) return RB200_INVALID_ARGUMENT;
    if (len != size_t(V->g.cells)) return RB200_LENGTH_MISMATCH;
    cudaSetDevice(V->device);
    RB200_CUDA(cudaMemcpyAsync(out, V->h_L->frac[V->h_L->acc], len * 8, cudaMemcpyDefault, V->stream));
    RB200_CUDA(cudaStreamSynchronize(V->stream));
    return RB200_OK;
}

}  // extern "C"

namespace {

// The cancellation points of prepare_with_boundary (src/liquid_volume.rs:558-830)
// in their order: BeforeFlux once; FaceFluxSlice per z plane of the faces of
// each axis, for the periodic seam check (:575-600) and again for the face
// transfers (:604-611); CellUpdateSlice per z plane of the cells (:686-690);
// BeforeCommit once, after every check (:830).
struct VolumeCheckpoints {
    long long seam, flux, cells;  // FaceFluxSlice polls of the seam check and of the transfers; CellUpdateSlice polls
    long long total() const { return 1 + seam + flux + cells; }  // without BeforeCommit
    int stage(long long index) const {
        if (index == 0) return RB200_VOLUME_BEFORE_FLUX;
        return index <= seam + flux ? RB200_VOLUME_FACE_FLUX_SLICE : RB200_VOLUME_CELL_UPDATE_SLICE;
    }
};

VolumeCheckpoints checkpoints_of(const GridDev& g, int periodic) {
    const long long flux = (long long)g.fc[0][2] + g.fc[1][2] + g.fc[2][2];
    return VolumeCheckpoints{periodic ? flux : 0, flux, g.n[2]};
}

// How many cancellation points the reference passes before it meets the
// device's error: the validation errors precede BeforeFlux; a seam mismatch
// lies in the slice of its face; a cell's Courant or bounds failure in the
// slice of its cell; the divergence limit, the ledger and the balance limit
// after every slice. An arithmetic failure is placed after the slices: the
// device does not record which product failed.
long long checkpoints_before(const GridDev& g, const VolumeCheckpoints& cp, const rb200_liquid_report& r) {
    switch (r.error) {
        case RB200_LIQUID_PERIODIC_VELOCITY_MISMATCH: {
            const int axis = int(r.error_actual);
            long long before = 0;
            for (int a = 0; a < axis; ++a) before += g.fc[a][2];
            const long long plane = (long long)g.fc[axis][0] * g.fc[axis][1];
            return 1 + before + (long long)r.error_cell / plane + 1;
        }
        case RB200_LIQUID_COURANT_LIMIT:
        case RB200_LIQUID_FRACTION_BOUNDS:
            return 1 + cp.seam + cp.flux + (long long)r.error_cell / ((long long)g.n[0] * g.n[1]) + 1;
        case RB200_LIQUID_ARITHMETIC_FAILURE:
        case RB200_LIQUID_DIVERGENCE_LIMIT:
        case RB200_LIQUID_BALANCE_LIMIT:
            return cp.total();
        default:
            return 0;
    }
}

// One standalone interval: the inputs to the device, the transport and
// decision into the candidate array, the reference's cancellation points
// against that outcome, and the commit only when every point has passed;
// then the report and the bookkeeping back. A cancellation or an error leaves
// the accepted state untouched.
int liquid_advance_impl(rb200_liquid_volume* V, const rb200_liquid_flow* flow, const rb200_liquid_inlet* inlet,
                        rb200_liquid_stamp boundary, int periodic, const rb200_liquid_source* source,
                        const rb200_liquid_settings* settings, rb200_liquid_cancel_fn cancel, void* ctx,
                        rb200_liquid_report* report, void* stream) {
    cudaSetDevice(V->device);
    const cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : V->stream;
    LiquidFlowDev& f = *V->h_flow;
    RB200_CUDA(cudaStreamSynchronize(s));  // the pinned inputs of an earlier call are free
    f = LiquidFlowDev{};
    f.vel[0] = flow->u;
    f.vel[1] = flow->v;
    f.vel[2] = flow->w;
    f.src = source ? source->rate : nullptr;
    f.start = flow->start;
    f.dt = flow->dt;
    f.flow = flow->stamp;
    f.inlet = periodic ? boundary : inlet->stamp;
    if (source) f.source = source->stamp;
    for (int q = 0; q < 6; ++q) f.inlet_fraction[q] = periodic ? 0.0 : inlet->fraction[q];
    f.max_courant = settings->max_outward_courant;
    f.divergence_limit = settings->actual_divergence_limit;
    f.active = 1;
    f.periodic = periodic;
    RB200_CUDA(cudaMemcpyAsync(V->d_flow, V->h_flow, sizeof(LiquidFlowDev), cudaMemcpyHostToDevice, s));
    RB200_CUDA(cudaMemsetAsync(V->d_rep, 0, sizeof(rb200_liquid_report), s));
    RB200_CUDA(launch_liquid_advance(V->g, V->d_L, V->d_flow, V->sc, V->blocks, V->d_rep, s));
    if (cancel) {
        RB200_CUDA(cudaMemcpyAsync(V->h_rep, V->d_rep, sizeof(rb200_liquid_report), cudaMemcpyDeviceToHost, s));
        RB200_CUDA(cudaStreamSynchronize(s));
        const VolumeCheckpoints cp = checkpoints_of(V->g, periodic);
        const long long reach = V->h_rep->error ? checkpoints_before(V->g, cp, *V->h_rep) : cp.total() + 1;
        for (long long q = 0; q < reach; ++q) {
            const int stage = q < cp.total() ? cp.stage(q) : RB200_VOLUME_BEFORE_COMMIT;
            if (cancel(ctx, stage)) {
                *report = rb200_liquid_report{};
                report->error = RB200_LIQUID_CANCELLED;
                report->error_cell = uint64_t(stage);
                return RB200_LIQUID_REJECTED;
            }
        }
    }
    RB200_CUDA(launch_liquid_commit(V->d_L, V->d_rep, s));
    RB200_CUDA(cudaMemcpyAsync(V->h_rep, V->d_rep, sizeof(rb200_liquid_report), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaMemcpyAsync(V->h_L, V->d_L, sizeof(LiquidDev), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaStreamSynchronize(s));
    *report = *V->h_rep;
    return report->error ? RB200_LIQUID_REJECTED : RB200_OK;
}

}  // namespace

extern "C" {

// LiquidVolumeState::advance (src/liquid_volume.rs:376-387, 520-776).
int rb200_liquid_advance(rb200_liquid_volume* V, const rb200_liquid_flow* flow, const rb200_liquid_inlet* inlet,
                         const rb200_liquid_source* source, const rb200_liquid_settings* settings,
                         rb200_liquid_report* report, void* stream) {
    return rb200_liquid_advance_cancellable(V, flow, inlet, source, settings, nullptr, nullptr, report, stream);
}

int rb200_liquid_advance_cancellable(rb200_liquid_volume* V, const rb200_liquid_flow* flow,
                                     const rb200_liquid_inlet* inlet, const rb200_liquid_source* source,
                                     const rb200_liquid_settings* settings, rb200_liquid_cancel_fn cancel, void* ctx,
                                     rb200_liquid_report* report, void* stream) {
    if (!V || !flow || !inlet || !settings || !report || !flow->u || !flow->v || !flow->w)
        return RB200_INVALID_ARGUMENT;
    return liquid_advance_impl(V, flow, inlet, rb200_liquid_stamp{0, 0}, 0, source, settings, cancel, ctx, report,
                               stream);
}

// LiquidVolumeState::advance_periodic (src/liquid_volume.rs:389-406).
int rb200_liquid_advance_periodic(rb200_liquid_volume* V, const rb200_liquid_flow* flow, rb200_liquid_stamp boundary,
                                  const rb200_liquid_source* source, const rb200_liquid_settings* settings,
                                  rb200_liquid_report* report, void* stream) {
    return rb200_liquid_advance_periodic_cancellable(V, flow, boundary, source, settings, nullptr, nullptr, report,
                                                     stream);
}

int rb200_liquid_advance_periodic_cancellable(rb200_liquid_volume* V, const rb200_liquid_flow* flow,
                                              rb200_liquid_stamp boundary, const rb200_liquid_source* source,
                                              const rb200_liquid_settings* settings, rb200_liquid_cancel_fn cancel,
                                              void* ctx, rb200_liquid_report* report, void* stream) {
    if (!V || !flow || !settings || !report || !flow->u || !flow->v || !flow->w) return RB200_INVALID_ARGUMENT;
    return liquid_advance_impl(V, flow, nullptr, boundary, 1, source, settings, cancel, ctx, report, stream);
}

}  // extern "C"
