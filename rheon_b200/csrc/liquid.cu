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

#include "internal.hpp"

namespace rb200 {
namespace {

constexpr int LQ_THREADS = 256;
constexpr int LQ_K = 8;  // dd sums: before, after, inward, outward, source, |source|, dry, full
constexpr int LQ_M = 4;  // maxima: courant, |div|, -fraction (min), fraction
constexpr int LQ_STRIDE = 2 * LQ_K + LQ_M;

// rb200_liquid_error codes used on the device
enum : int { LQ_ARITH = RB200_LIQUID_ARITHMETIC_FAILURE, LQ_COURANT = RB200_LIQUID_COURANT_LIMIT,
             LQ_BOUNDS = RB200_LIQUID_FRACTION_BOUNDS };

struct LqResult {
    double sums[LQ_K];
    double maxs[LQ_M];
    int face_failed;
    int velocity_nonfinite;
    int source_nonfinite;
    int first_code;           // the first failing cell's error
    unsigned long long first_cell;
    double first_actual;      // its Courant number or fraction
};

struct LqArgs {
    GridDev g;
    const double* acc;
    double* cand;
    const float* vel[3];
    const double* src;
    double dt, volume;
    double dta[3];            // product(dt, area_d), checked on the host
    double inlet[6];
    double max_courant;
    double* part;             // [blocks][LQ_STRIDE]
    unsigned* ticket;
    unsigned long long* first_cell;  // atomicMin target, ULLONG_MAX when no cell failed
    int* flags;               // [0] face failure, [1] nonfinite velocity, [2] nonfinite source
    LqResult* out;
};

// product / quotient (src/liquid_volume.rs:879-896): overflow, a subnormal
// result or underflow to zero fails.
__device__ __forceinline__ double prod_chk(double a, double b, bool& bad) {
    const double v = a * b;
    if (!isfinite(v) || (v != 0.0 && fabs(v) < DBL_MIN) || (v == 0.0 && a != 0.0 && b != 0.0)) bad = true;
    return v;
}
__device__ __forceinline__ double quot_chk(double a, double b, bool& bad) {
    const double v = a / b;
    if (!isfinite(v) || (v != 0.0 && fabs(v) < DBL_MIN) || (v == 0.0 && a != 0.0)) bad = true;
    return v;
}

// Transfer through face p of axis d (src/liquid_volume.rs:587-639): the
// upwind donor fraction (the inlet's outside fraction on inflow through the
// box), times dt, area and velocity.
__device__ __forceinline__ double face_transfer(const LqArgs& a, int d, int i, int j, int k, double v, bool& bad) {
    const GridDev& g = a.g;
    const int p[3] = {i, j, k};
    double donor = 0.0;
    if (v > 0.0) {
        if (p[d] == 0) {
            donor = a.inlet[2 * d];
        } else {
            int q[3] = {i, j, k};
            q[d] -= 1;
            donor = a.acc[cell_idx(g, q[0], q[1], q[2])];
        }
    } else if (v < 0.0) {
        donor = p[d] == g.n[d] ? a.inlet[2 * d + 1] : a.acc[cell_idx(g, i, j, k)];
    }
    return prod_chk(prod_chk(a.dta[d], v, bad), donor, bad);
}

struct CellOut {
    double fraction, courant, div;
    double inward, outward, source;
    int code;
    bool face_bad, vel_bad, src_bad;
};

// Cell update (src/liquid_volume.rs:642-699) of cell (i, j, k).
__device__ __forceinline__ CellOut liquid_cell(const LqArgs& a, int i, int j, int k) {
    const GridDev& g = a.g;
    CellOut o{};
    const int c = cell_idx(g, i, j, k);
    o.src_bad = a.src && !isfinite(a.src[c]);
    bool bad = false;
    double amount = prod_chk(a.volume, a.acc[c], bad);
    double courant = 0.0, div = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int hi = d == 0 ? i + 1 : i, hj = d == 1 ? j + 1 : j, hk = d == 2 ? k + 1 : k;
        const float fa = a.vel[d][face_idx(g, d, i, j, k)];
        const float fb = a.vel[d][face_idx(g, d, hi, hj, hk)];
        o.vel_bad |= !isfinite(fa) || !isfinite(fb);
        const double va = double(fa), vb = double(fb);
        const double tl = face_transfer(a, d, i, j, k, va, o.face_bad);
        const double th = face_transfer(a, d, hi, hj, hk, vb, o.face_bad);
        amount += tl - th;
        // boundary faces owned by this cell: inward / outward volume (:739-757)
        const int pd = d == 0 ? i : (d == 1 ? j : k);
        if (pd == 0) {
            const double value = -tl;
            if (value < 0.0)
                o.inward += -value;
            else
                o.outward += value;
        }
        if (pd + 1 == g.n[d]) {
            const double value = th;
            if (value < 0.0)
                o.inward += -value;
            else
                o.outward += value;
        }
        courant += quot_chk(prod_chk(a.dt, fmax(vb, 0.0) - fmin(va, 0.0), bad), g.h[d], bad);
        div += quot_chk(vb - va, g.h[d], bad);
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
    const double fraction = quot_chk(amount, a.volume, bad2);
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
    const GridDev& g = a.g;
    dd sums[LQ_K];
    double maxs[LQ_M] = {0.0, 0.0, -INFINITY, -INFINITY};
#pragma unroll
    for (int q = 0; q < LQ_K; ++q) sums[q] = dd{0.0, 0.0};
    bool face_bad = false, vel_bad = false, src_bad = false;
    const int n0 = g.n[0], n01 = g.n[0] * g.n[1];
    for (int c = blockIdx.x * LQ_THREADS + threadIdx.x; c < g.cells; c += gridDim.x * LQ_THREADS) {
        const int k = c / n01, r = c - k * n01, j = r / n0, i = r - j * n0;
        const CellOut o = liquid_cell(a, i, j, k);
        face_bad |= o.face_bad;
        vel_bad |= o.vel_bad;
        src_bad |= o.src_bad;
        if (o.code) {
            atomicMin(a.first_cell, (unsigned long long)c);
            continue;
        }
        a.cand[c] = o.fraction;
        sums[0] = dd_add1(sums[0], a.volume * a.acc[c]);
        sums[1] = dd_add1(sums[1], a.volume * o.fraction);
        sums[2] = dd_add1(sums[2], o.inward);
        sums[3] = dd_add1(sums[3], o.outward);
        sums[4] = dd_add1(sums[4], o.source);
        sums[5] = dd_add1(sums[5], fabs(o.source));
        sums[6] = dd_add1(sums[6], o.fraction == 0.0 ? 1.0 : 0.0);
        sums[7] = dd_add1(sums[7], o.fraction == 1.0 ? 1.0 : 0.0);
        maxs[0] = fmax(maxs[0], o.courant);
        maxs[1] = fmax(maxs[1], fabs(o.div));
        maxs[2] = fmax(maxs[2], -o.fraction);
        maxs[3] = fmax(maxs[3], o.fraction);
    }
    if (__syncthreads_or(face_bad) && threadIdx.x == 0) atomicOr(&a.flags[0], 1);
    if (__syncthreads_or(vel_bad) && threadIdx.x == 0) atomicOr(&a.flags[1], 1);
    if (__syncthreads_or(src_bad) && threadIdx.x == 0) atomicOr(&a.flags[2], 1);
    double none[1] = {0.0};
    block_reduce<LQ_K, 0>(red, sums, none);
    block_max(maxs, smax);
    if (threadIdx.x == 0) {
        double* slot = a.part + size_t(blockIdx.x) * LQ_STRIDE;
#pragma unroll
        for (int q = 0; q < LQ_K; ++q) {
            slot[2 * q] = sums[q].hi;
            slot[2 * q + 1] = sums[q].lo;
        }
#pragma unroll
        for (int q = 0; q < LQ_M; ++q) slot[2 * LQ_K + q] = maxs[q];
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block folds every block's partials (in block order per thread)
    __threadfence();
#pragma unroll
    for (int q = 0; q < LQ_K; ++q) sums[q] = dd{0.0, 0.0};
    maxs[0] = maxs[1] = 0.0;
    maxs[2] = maxs[3] = -INFINITY;
    for (int b = threadIdx.x; b < int(gridDim.x); b += LQ_THREADS) {
        const double* slot = a.part + size_t(b) * LQ_STRIDE;
#pragma unroll
        for (int q = 0; q < LQ_K; ++q) sums[q] = dd_add(sums[q], dd{__ldcg(slot + 2 * q), __ldcg(slot + 2 * q + 1)});
#pragma unroll
        for (int q = 0; q < LQ_M; ++q) maxs[q] = fmax(maxs[q], __ldcg(slot + 2 * LQ_K + q));
    }
    block_reduce<LQ_K, 0>(red, sums, none);
    block_max(maxs, smax);
    if (threadIdx.x == 0) {
        LqResult& R = *a.out;
#pragma unroll
        for (int q = 0; q < LQ_K; ++q) R.sums[q] = dd_value(sums[q]);
#pragma unroll
        for (int q = 0; q < LQ_M; ++q) R.maxs[q] = maxs[q];
        R.face_failed = __ldcg(&a.flags[0]);
        R.velocity_nonfinite = __ldcg(&a.flags[1]);
        R.source_nonfinite = __ldcg(&a.flags[2]);
        const unsigned long long fc = __ldcg(a.first_cell);
        R.first_cell = fc;
        R.first_code = 0;
        R.first_actual = 0.0;
        if (fc != ~0ull) {
            const int c = int(fc);
            const int kk = c / n01, rr = c - kk * n01, jj = rr / n0, ii = rr - jj * n0;
            const CellOut o = liquid_cell(a, ii, jj, kk);
            R.first_code = o.code;
            R.first_actual = o.code == LQ_COURANT ? o.courant : o.fraction;
        }
        *a.ticket = 0u;
    }
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
}  // namespace rb200

using namespace rb200;

struct rb200_liquid_volume {
    int device = 0;
    GridDev g{};
    double density = 0.0;
    double volume = 0.0;
    rb200_liquid_stamp stamp{};
    double time = 0.0;
    double* frac[2] = {nullptr, nullptr};  // accepted = frac[acc]
    int acc = 0;
    int blocks = 0;
    double* part = nullptr;
    unsigned* ticket = nullptr;
    unsigned long long* first = nullptr;
    int* flags = nullptr;
    LqResult* d_out = nullptr;
    LqResult* h_out = nullptr;  // pinned
    uint64_t bytes = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    ~rb200_liquid_volume() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        cudaFree(frac[0]);
        cudaFree(frac[1]);
        cudaFree(part);
        cudaFree(ticket);
        cudaFree(first);
        cudaFree(flags);
        cudaFree(d_out);
        if (h_out) cudaFreeHost(h_out);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

void set_liquid_error(rb200_liquid_report* r, int code, uint64_t cell = 0, double actual = 0.0, double limit = 0.0) {
    if (!r) return;
    r->error = code;
    r->error_cell = cell;
    r->error_actual = actual;
    r->error_limit = limit;
}

}  // namespace

extern "C" {

int rb200_liquid_create(const rb200_grid* grid, double density, rb200_liquid_stamp stamp, const double* fraction,
                        uint64_t limit, int device, rb200_liquid_volume** out, rb200_liquid_report* error) {
    if (!grid || !fraction || !out) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    if (error) std::memset(error, 0, sizeof(*error));
    GridDev g;
    int rc = make_grid_dev(grid, 1.0, &g);
    if (rc) return rc;
    // LiquidVolumeState::new (src/liquid_volume.rs:276-351)
    if (!std::isfinite(density) || density <= 0.0) {
        set_liquid_error(error, RB200_LIQUID_INVALID_DENSITY);
        return RB200_LIQUID_REJECTED;
    }
    // accepted and candidate fractions (the reference also counts three
    // face-transfer arrays, which the device does not keep)
    const uint64_t required = 2ull * uint64_t(g.cells) * 8ull;
    if (required > limit) {
        set_liquid_error(error, RB200_LIQUID_BUFFER_LIMIT, 0, double(required), double(limit));
        return RB200_LIQUID_REJECTED;
    }
    RB200_CUDA(cudaSetDevice(device));
    auto* L = new rb200_liquid_volume();
    L->device = device;
    L->g = g;
    L->density = density;
    L->volume = g.h[0] * g.h[1] * g.h[2];
    L->stamp = stamp;
    L->blocks = std::max(1, std::min((g.cells + LQ_THREADS - 1) / LQ_THREADS, 148 * 8));
    const size_t n = size_t(g.cells);
    bool ok = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&L->frac[0], n * 8) == cudaSuccess && cudaMalloc(&L->frac[1], n * 8) == cudaSuccess &&
              cudaMalloc(&L->part, size_t(L->blocks) * LQ_STRIDE * 8) == cudaSuccess &&
              cudaMalloc(&L->ticket, sizeof(unsigned)) == cudaSuccess &&
              cudaMalloc(&L->first, sizeof(unsigned long long)) == cudaSuccess &&
              cudaMalloc(&L->flags, 4 * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&L->d_out, sizeof(LqResult)) == cudaSuccess &&
              cudaMallocHost(&L->h_out, sizeof(LqResult)) == cudaSuccess;
    if (!ok) {
        delete L;
        cudaGetLastError();
        return RB200_OUT_OF_MEMORY;
    }
    L->bytes = 2 * n * 8;
    const cudaStream_t s = L->stream;
    RB200_CUDA(cudaMemcpyAsync(L->frac[0], fraction, n * 8, cudaMemcpyDefault, s));
    RB200_CUDA(cudaMemsetAsync(L->frac[1], 0, n * 8, s));
    RB200_CUDA(cudaMemsetAsync(L->ticket, 0, sizeof(unsigned), s));
    RB200_CUDA(cudaMemsetAsync(L->first, 0xff, sizeof(unsigned long long), s));
    RB200_CUDA(cudaMemsetAsync(L->flags, 0, 4 * sizeof(int), s));
    double* total = reinterpret_cast<double*>(L->d_out);
    k_liquid_check_state<<<L->blocks, LQ_THREADS, 0, s>>>(g, L->frac[0], L->volume, L->first, L->flags, L->part,
                                                           L->ticket, total);
    RB200_CUDA(cudaGetLastError());
    unsigned long long bad = 0;
    int arith = 0;
    double initial = 0.0;
    RB200_CUDA(cudaMemcpyAsync(&bad, L->first, sizeof(bad), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaMemcpyAsync(&arith, L->flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaMemcpyAsync(&initial, total, sizeof(double), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaStreamSynchronize(s));
    double mass = 0.0;
    int code = 0;
    if (bad != ~0ull)
        code = RB200_LIQUID_INVALID_FRACTION;
    else if (arith || !std::isfinite(initial) || !host_product(density, initial, &mass))
        code = RB200_LIQUID_ARITHMETIC_FAILURE;
    if (code) {
        set_liquid_error(error, code, code == RB200_LIQUID_INVALID_FRACTION ? bad : 0);
        delete L;
        return RB200_LIQUID_REJECTED;
    }
    RB200_CUDA(cudaMemsetAsync(L->first, 0xff, sizeof(unsigned long long), s));
    RB200_CUDA(cudaMemsetAsync(L->flags, 0, 4 * sizeof(int), s));
    *out = L;
    return RB200_OK;
}

void rb200_liquid_destroy(rb200_liquid_volume* L) { delete L; }

uint64_t rb200_liquid_allocated_bytes(const rb200_liquid_volume* L) { return L ? L->bytes : 0; }

int rb200_liquid_state(const rb200_liquid_volume* L, const double** fraction, rb200_liquid_stamp* stamp,
                       double* time) {
    if (!L) return RB200_INVALID_ARGUMENT;
    if (fraction) *fraction = L->frac[L->acc];
    if (stamp) *stamp = L->stamp;
    if (time) *time = L->time;
    return RB200_OK;
}

int rb200_liquid_download(rb200_liquid_volume* L, double* out, size_t len) {
    if (!L || !out) return RB200_INVALID_ARGUMENT;
    if (len != size_t(L->g.cells)) return RB200_LENGTH_MISMATCH;
    cudaSetDevice(L->device);
    RB200_CUDA(cudaMemcpyAsync(out, L->frac[L->acc], len * 8, cudaMemcpyDefault, L->stream));
    RB200_CUDA(cudaStreamSynchronize(L->stream));
    return RB200_OK;
}

// LiquidVolumeState::advance (src/liquid_volume.rs:376-387, 520-776) with the
// checks of LiquidFlowInterval::new (:123-150), LiquidInlet::new (:84-96) and
// LiquidVolumeSource::new (:185-190), in the order a caller constructing the
// interval, the inlet and the source and then advancing meets them.
int rb200_liquid_advance(rb200_liquid_volume* L, const rb200_liquid_flow* flow, const rb200_liquid_inlet* inlet,
                         const rb200_liquid_source* source, const rb200_liquid_settings* settings,
                         rb200_liquid_report* report, void* stream) {
    if (!L || !flow || !inlet || !settings || !report || !flow->u || !flow->v || !flow->w)
        return RB200_INVALID_ARGUMENT;
    std::memset(report, 0, sizeof(*report));
    const GridDev& g = L->g;
    const double start = flow->start, dt = flow->dt;
    if (!std::isfinite(start) || start < 0.0 || !std::isfinite(dt) || dt <= 0.0) {
        set_liquid_error(report, RB200_LIQUID_INVALID_TIME_STEP);
        return RB200_LIQUID_REJECTED;
    }
    const double end = start + dt;
    if (!std::isfinite(end) || end <= start) {
        set_liquid_error(report, RB200_LIQUID_TIME_RESOLUTION);
        return RB200_LIQUID_REJECTED;
    }
    int late = 0;  // host-side errors ranked after the velocity scan
    bool inlet_bad = false;
    for (int q = 0; q < 6; ++q)
        inlet_bad |= !std::isfinite(inlet->fraction[q]) || !(inlet->fraction[q] >= 0.0 && inlet->fraction[q] <= 1.0);
    uint64_t tb, sb;
    std::memcpy(&tb, &start, 8);
    std::memcpy(&sb, &L->time, 8);
    if (tb != sb)
        late = RB200_LIQUID_TIME_MISMATCH;
    else if (!std::isfinite(settings->max_outward_courant) || settings->max_outward_courant <= 0.0 ||
             settings->max_outward_courant > 1.0 || !std::isfinite(settings->actual_divergence_limit) ||
             settings->actual_divergence_limit < 0.0)
        late = RB200_LIQUID_INVALID_SETTINGS;
    else if (L->stamp.version == ~0ull)
        late = RB200_LIQUID_VERSION_OVERFLOW;
    LqArgs a{};
    a.g = g;
    a.acc = L->frac[L->acc];
    a.cand = L->frac[L->acc ^ 1];
    a.vel[0] = flow->u;
    a.vel[1] = flow->v;
    a.vel[2] = flow->w;
    a.src = source ? source->rate : nullptr;
    a.dt = dt;
    a.volume = L->volume;
    // product(dt, area_d) is the first factor of every face transfer; it is
    // the same for all faces of an axis (src/liquid_volume.rs:551-555, 636)
    bool area_bad = false;
    const double sides[3][2] = {{g.h[1], g.h[2]}, {g.h[0], g.h[2]}, {g.h[0], g.h[1]}};
    for (int d = 0; d < 3; ++d) {
        double area = 0.0;
        area_bad |= !host_product(sides[d][0], sides[d][1], &area);
        area_bad |= !host_product(dt, area, &a.dta[d]);
    }
    for (int q = 0; q < 6; ++q) a.inlet[q] = inlet->fraction[q];
    a.max_courant = settings->max_outward_courant;
    a.part = L->part;
    a.ticket = L->ticket;
    a.first_cell = L->first;
    a.flags = L->flags;
    a.out = L->d_out;
    cudaSetDevice(L->device);
    const cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
    k_liquid_advance<<<L->blocks, LQ_THREADS, 0, s>>>(a);
    RB200_CUDA(cudaGetLastError());
    RB200_CUDA(cudaMemcpyAsync(L->h_out, L->d_out, sizeof(LqResult), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaMemsetAsync(L->first, 0xff, sizeof(unsigned long long), s));
    RB200_CUDA(cudaMemsetAsync(L->flags, 0, 4 * sizeof(int), s));
    RB200_CUDA(cudaStreamSynchronize(s));
    const LqResult R = *L->h_out;
    // outcome, in the reference's order
    int code = 0;
    if (R.velocity_nonfinite)
        code = RB200_LIQUID_NONFINITE_VELOCITY;
    else if (inlet_bad)
        code = RB200_LIQUID_INVALID_INLET;
    else if (R.source_nonfinite)
        code = RB200_LIQUID_INVALID_SOURCE;
    else if (late)
        code = late;
    else if (area_bad || R.face_failed)
        code = RB200_LIQUID_ARITHMETIC_FAILURE;
    if (code) {
        set_liquid_error(report, code);
        return RB200_LIQUID_REJECTED;
    }
    if (R.first_cell != ~0ull) {
        if (R.first_code == RB200_LIQUID_COURANT_LIMIT)
            set_liquid_error(report, R.first_code, R.first_cell, R.first_actual, settings->max_outward_courant);
        else if (R.first_code == RB200_LIQUID_FRACTION_BOUNDS)
            set_liquid_error(report, R.first_code, R.first_cell, R.first_actual);
        else
            set_liquid_error(report, RB200_LIQUID_ARITHMETIC_FAILURE);
        return RB200_LIQUID_REJECTED;
    }
    const double max_div = R.maxs[1];
    if (max_div > settings->actual_divergence_limit) {
        set_liquid_error(report, RB200_LIQUID_DIVERGENCE_LIMIT, 0, max_div, settings->actual_divergence_limit);
        return RB200_LIQUID_REJECTED;
    }
    // volume ledger (src/liquid_volume.rs:735-776)
    const double before = R.sums[0], after = R.sums[1], inward = R.sums[2], outward = R.sums[3];
    const double source_total = R.sums[4], source_abs = R.sums[5];
    const double balance = after - before + outward - inward - source_total;
    const double budget = (64.0 * DBL_EPSILON) * (std::fabs(before) + std::fabs(after) + outward + inward + source_abs);
    double mass_before = 0.0, mass_after = 0.0;
    bool arith = !host_product(L->density, before, &mass_before);
    arith = arith || !host_product(L->density, after, &mass_after);
    for (double x : {before, after, inward, outward, source_total, balance, budget, mass_before, mass_after})
        arith = arith || !std::isfinite(x);
    if (arith) {
        set_liquid_error(report, RB200_LIQUID_ARITHMETIC_FAILURE);
        return RB200_LIQUID_REJECTED;
    }
    if (std::fabs(balance) > budget) {
        set_liquid_error(report, RB200_LIQUID_BALANCE_LIMIT, 0, balance, budget);
        return RB200_LIQUID_REJECTED;
    }
    report->stamp = rb200_liquid_stamp{L->stamp.id, L->stamp.version + 1};
    report->flow = flow->stamp;
    report->inlet = inlet->stamp;
    report->has_source = source ? 1 : 0;
    if (source) report->source = source->stamp;
    report->dt = dt;
    report->time = end;
    report->liquid_volume_before = before;
    report->liquid_volume_after = after;
    report->inward_boundary_volume = inward;
    report->outward_boundary_volume = outward;
    report->source_volume = source_total;
    report->volume_balance_error = balance;
    report->volume_rounding_budget = budget;
    report->liquid_mass_before = mass_before;
    report->liquid_mass_after = mass_after;
    report->max_outward_courant = R.maxs[0];
    report->actual_divergence_max = max_div;
    report->fraction_min = std::fmin(1.0, -R.maxs[2]);
    report->fraction_max = std::fmax(0.0, R.maxs[3]);
    report->dry_cells = uint64_t(R.sums[6]);
    report->full_cells = uint64_t(R.sums[7]);
    report->mixed_cells = uint64_t(g.cells) - report->dry_cells - report->full_cells;
    // commit (src/liquid_volume.rs:514-518)
    L->acc ^= 1;
    L->time = end;
    L->stamp = report->stamp;
    return RB200_OK;
}

}  // extern "C"
