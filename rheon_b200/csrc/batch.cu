// Packed batch of fixed-box carriers stepped together with the mixed-precision
// pressure method (see batch.hpp). The step of every instance follows Rheon's
// step owner (Simulation::prepare_impl, src/simulation.rs:812-1403): dt
// policy, advection, build_rhs, the pressure solve (solve_loaded's control
// flow, src/pressure.rs:577-740, per instance, with the FP32 multigrid
// V-cycle inside FP64 flexible CG), correction with the actual divergence and
// velocity rate, the divergence and Courant gates, and the transactional
// commit. Each stage is one launch over all instances.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "advect.cuh"
#include "batch.hpp"
#include "carrier.hpp"
#include "mg_device.cuh"
#include "pcg_device.cuh"
#include "project.cuh"

namespace rb200 {
namespace {

constexpr int BT = 256;       // threads of the packed elementwise kernels
constexpr int kItems = 16;    // advected faces per thread
constexpr int kCellItems = 64;  // cells per thread of the cell passes (most reduce: a block's reduction covers 16384 cells)
constexpr int kRowsPerWarp = 16;  // rows per warp of the FCG update and finish (their reductions cover 128 rows)
constexpr int kPass1Kc = 16;   // z-march length of the direction pass
constexpr int kFineRestrictRows = 4;  // coarse rows per warp (lane group) of the finest level's restriction
constexpr int kChunk = 4;     // iterations per trip of the solve loop
constexpr int kSlotDoubles = 2 * 3 + 3;  // widest partials: the compatibility sums (3 sums, 3 maxima)
constexpr int kGeomDoubles = int(offsetof(GridDev, diag) / sizeof(double));
static_assert(offsetof(GridDev, diag) % sizeof(double) == 0, "geometry prefix");

// The entry (instance, or instance-level operation) of a packed launch this
// block works on, and the block's span within it. Entries without blocks are
// never found: the search lands on the last range that starts at or before
// the block.
__device__ __forceinline__ int batch_entry(const BatchSpans& s, Span& sp) {
    int lo = 0, hi = s.count;
    const int b = int(blockIdx.x);
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s.first[mid] <= b)
            lo = mid;
        else
            hi = mid;
    }
    sp = Span{b - s.first[lo], s.first[lo + 1] - s.first[lo]};
    return lo;
}

// The geometry and operator coefficients of a grid (everything before the
// diagonal tables, which the batch kernels do not use) into shared memory.
__device__ __forceinline__ void load_geometry(GridDev& dst, const GridDev& src) {
    double* d = reinterpret_cast<double*>(&dst);
    const double* s = reinterpret_cast<const double*>(&src);
    for (int t = threadIdx.x; t < kGeomDoubles; t += blockDim.x) d[t] = s[t];
}

template <class T>
__device__ __forceinline__ void block_copy(T& dst, const T& src) {
    static_assert(sizeof(T) % 4 == 0, "word copy");
    unsigned* d = reinterpret_cast<unsigned*>(&dst);
    const unsigned* s = reinterpret_cast<const unsigned*>(&src);
    for (int t = threadIdx.x; t < int(sizeof(T) / 4); t += blockDim.x) d[t] = s[t];
}

__device__ __forceinline__ bool running(const BatchStepDev* cd) { return cd->status == STEP_RUNNING; }

// Proceed to the correction: the solve converged, or an exact-iteration-count
// solve reached its limit.
__device__ __forceinline__ bool usable(const BatchStepDev* cd, const SolveState* st) {
    return running(cd) && (st->status == RB200_OK || (st->status == RB200_ITERATION_LIMIT && cd->iteration_limit_ok));
}

// ------------------------------------------------------------ step stages
// dt policy (src/simulation.rs:952-979): dt = min(requested, cfl/rate).
__global__ void k_b_begin(BatchInstDev* inst, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BatchStepDev* cd = inst[i].step;
    double dt = cd->requested_dt;
    if (cd->cfl > 0.0 && cd->rate > 0.0) dt = fmin(dt, cd->cfl / cd->rate);
    cd->dt = dt;
    cd->flags = 0;
    cd->skip = 0;
    cd->status = STEP_RUNNING;
    const double next = cd->time + dt;
    if (!isfinite(dt) || dt <= 0.0 || !isfinite(next) || next <= cd->time) {
        cd->status = RB200_INVALID_ARGUMENT;
        cd->skip = 1;
    }
}

template <class R>
__global__ void __launch_bounds__(BT) k_b_advect(const BatchInstDev* __restrict__ inst, const __grid_constant__ BatchSpans spans) {
    __shared__ GridDev g;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    load_geometry(g, I.g);
    __syncthreads();
    BatchStepDev* cd = I.step;
    if (!running(cd)) return;
    const int a = cd->acc, b = (a + 1) % 3;
    const Faces<float> vel{{I.faces[a][0], I.faces[a][1], I.faces[a][2]}};
    advect_velocity_body<float, R>(g, vel, cd->dt, I.faces[b][0], I.faces[b][1], I.faces[b][2], nullptr, 0.0,
                                   &cd->flags, sp);
}

__global__ void __launch_bounds__(BT) k_b_rhs(const BatchInstDev* __restrict__ inst, const __grid_constant__ BatchSpans spans) {
    __shared__ GridDev g;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    load_geometry(g, I.g);
    __syncthreads();
    BatchStepDev* cd = I.step;
    if (!running(cd)) return;
    const int b = (cd->acc + 1) % 3;
    build_rhs_body<float>(g, I.faces[b][0], I.faces[b][1], I.faces[b][2], cd->dt, I.b, &cd->flags, sp);
}

// The solver state of every instance for this step's solve (as
// k_solve_reset): flexible CG, dt from the step, skipped when the step
// already failed.
__global__ void k_b_reset(BatchInstDev* inst, int count, rb200_settings s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const BatchStepDev* cd = inst[i].step;
    SolveState init{};
    init.dt = cd->dt;
    init.relative = s.relative_residual;
    init.absolute = s.absolute_residual;
    init.divergence_limit = s.divergence_limit;
    init.max_it = s.max_iterations > 0x7fffffffull ? 0x7fffffff : int(s.max_iterations);
    init.status = ST_RUNNING;
    init.flexible = 1;
    if (cd->skip) init.flags = F_DONE | F_STOP;
    *inst[i].st = init;
}

__global__ void __launch_bounds__(BT) k_b_init_sums(const BatchInstDev* __restrict__ inst, const __grid_constant__ BatchSpans spans) {
    __shared__ GridDev g;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    load_geometry(g, I.g);
    __syncthreads();
    init_sums_body(g, I.st, I.b, I.p, I.part, sp);
}

// r <- b (INIT) or the true residual (REPLACE), r[0] = 0. The multigrid
// method forms z in its own kernels (no z vector).
__global__ void __launch_bounds__(BT) k_b_load_residual(const BatchInstDev* __restrict__ inst, const __grid_constant__ BatchSpans spans,
                                                        int mode) {
    pdl_wait();
    __shared__ GridDev g;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    load_geometry(g, I.g);
    __syncthreads();
    load_residual_body<KIND_MG>(g, I.st, I.b, I.d0, I.d1, I.r, nullptr, mode, I.part, nullptr, sp);
}

// ------------------------------------------------------------ V-cycle operations
__global__ void __launch_bounds__(MG_THREADS) k_b_smooth(const BatchLevelOp* __restrict__ ops, const __grid_constant__ BatchSpans spans,
                                                         int mode) {
    pdl_wait();
    __shared__ MgLevelDev L;
    Span sp;
    const BatchLevelOp& op = ops[batch_entry(spans, sp)];
    block_copy(L, op.L);
    __syncthreads();
    if (!mg_gate(op.st, mode)) return;
    smooth_rows<false>(L, op.r0, op.color, op.first != 0, span_warps(sp));
}

__global__ void __launch_bounds__(MG_THREADS) k_b_pair(const BatchLevelOp* __restrict__ ops, const __grid_constant__ BatchSpans spans,
                                                       int mode) {
    pdl_wait();
    extern __shared__ float4 srow[];
    __shared__ MgLevelDev L;
    Span sp;
    const BatchLevelOp& op = ops[batch_entry(spans, sp)];
    block_copy(L, op.L);
    __syncthreads();
    if (!mg_gate(op.st, mode)) return;
    const int tj = (L.n[1] + PJ - 1) / PJ;
    pair_tile<false, PJ, PK>(L, op.out, op.color, op.first != 0, (sp.block % tj) * PJ, (sp.block / tj) * PK, srow);
}

constexpr int TRAIN_THREADS = kTrainThreads;
// Half-sweeps of a train: black, red, black on the finest level (after the
// first red half-sweep going down; from the prolongation coming up).
constexpr int kTrainPhases = 3;

__global__ void __launch_bounds__(TRAIN_THREADS, 2) k_b_train(const BatchLevelOp* __restrict__ ops,
                                                           const __grid_constant__ BatchSpans spans, int mode) {
    pdl_wait();
    extern __shared__ float4 tsm[];
    __shared__ MgLevelDev L, C;
    Span sp;
    const BatchLevelOp& op = ops[batch_entry(spans, sp)];
    block_copy(L, op.L);
    block_copy(C, op.C);
    __syncthreads();
    if (!mg_gate(op.st, mode)) return;
    const int strips = (L.n[1] + op.sj - 1) / op.sj;
    train_block<kTrainPhases>(L, &C, op.out, op.color, op.start, op.sj, op.sk, sp.block % strips, sp.block / strips,
                reinterpret_cast<float*>(tsm));
}

__global__ void __launch_bounds__(MG_THREADS) k_b_restrict(const BatchLevelOp* __restrict__ ops,
                                                           const __grid_constant__ BatchSpans spans, int mode) {
    pdl_wait();
    __shared__ MgLevelDev L, C;
    Span sp;
    const BatchLevelOp& op = ops[batch_entry(spans, sp)];
    block_copy(L, op.L);
    block_copy(C, op.C);
    __syncthreads();
    if (!mg_gate(op.st, mode)) return;
    restrict_rows<false>(L, C, span_warps(sp));
}

__global__ void __launch_bounds__(MG_THREADS) k_b_prolong(const BatchLevelOp* __restrict__ ops,
                                                          const __grid_constant__ BatchSpans spans, int mode) {
    pdl_wait();
    __shared__ MgLevelDev L, C;
    Span sp;
    const BatchLevelOp& op = ops[batch_entry(spans, sp)];
    block_copy(L, op.L);
    block_copy(C, op.C);
    __syncthreads();
    if (!mg_gate(op.st, mode)) return;
    prolong_black_rows<false>(L, C, span_warps(sp));
}

// Every instance's levels of at most 32^3 cells and its coarsest solve in one
// thread-block cluster per instance (the launch's clusters are the instances
// in order): the cluster V-cycle of the single grid's multigrid (lower_body)
// on the instance's table. The first level here is never the finest, so the
// body starts from a restricted right-hand side and finishes its own last
// half-sweep.
__global__ void __launch_bounds__(MG_LOWER_THREADS, 1) k_b_lower(const BatchLowerDev* __restrict__ tab, int mode) {
    pdl_wait();
    __shared__ double bs[512];
    __shared__ float4 prow[kLowerPairRows];
    const BatchLowerDev& T = tab[blockIdx.x / cluster_size()];
    if (!mg_gate(T.st, mode)) return;  // uniform over the instance's cluster
    lower_body(T.P, nullptr, T.G, 0, bs, prow);
}

// ------------------------------------------------------------ flexible-CG passes
__global__ void __launch_bounds__(MG_THREADS, 3) k_b_pass1(const BatchInstDev* __restrict__ inst, const __grid_constant__ BatchSpans spans,
                                                        int kc_len) {
    pdl_wait();
    __shared__ GridDev g;
    __shared__ MgLevelDev L;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    load_geometry(g, I.g);
    block_copy(L, I.fine);
    __syncthreads();
    pass1_body(g, L, I.st, I.d0, I.d1, I.part, nullptr, kc_len, sp);
}

__global__ void __launch_bounds__(MG_THREADS, 3) k_b_update_first(const BatchInstDev* __restrict__ inst,
                                                               const __grid_constant__ BatchSpans spans) {
    pdl_wait();
    __shared__ GridDev g;
    __shared__ MgLevelDev L;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    load_geometry(g, I.g);
    block_copy(L, I.fine);
    __syncthreads();
    update_first_body(g, L, I.st, I.p, I.r, I.r1, I.d0, I.d1, I.part, nullptr, sp);
}

__global__ void __launch_bounds__(MG_THREADS, 3) k_b_finish(const BatchInstDev* __restrict__ inst, const __grid_constant__ BatchSpans spans,
                                                         int mode) {
    pdl_wait();
    __shared__ MgLevelDev L;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    block_copy(L, I.fine);
    __syncthreads();
    finish_red_body(L, 1, I.st, I.r, I.r1, mode, I.part, nullptr, sp);
}

// true_report (src/pressure.rs:432-456) and solve_loaded's acceptance and
// restart decisions (:686-715), as k_true_residual: t = b - K p on every cell,
// |t|^2, |t[1..]|^2 and max|t|; t is kept in the spare direction buffer for a
// restart.
__global__ void __launch_bounds__(BT) k_b_true_residual(const BatchInstDev* __restrict__ inst,
                                                        const __grid_constant__ BatchSpans spans) {
    pdl_wait();
    __shared__ GridDev g;
    __shared__ BlockReduce<2, 1> red;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    load_geometry(g, I.g);
    __syncthreads();
    SolveState* st = I.st;
    const int flags = st->flags;
    if (!(flags & F_NEED_TRUE)) return;
    double* __restrict__ spare = st->dsel ? I.d0 : I.d1;
    const double* __restrict__ b = I.b;
    const double* __restrict__ p = I.p;
    const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2], sy = n0, sz = n0 * n1;
    Neu acc;
    double gauge_sq = 0.0;
    double mx[1] = {0.0};
    for (int c = sp.block * blockDim.x + threadIdx.x; c < g.cells; c += sp.blocks * blockDim.x) {
        const int i = c % n0, j = (c / n0) % n1, k = c / sz;
        Neigh v;
        v.c = p[c];
        v.xm = i > 0 ? p[c - 1] : 0.0;
        v.xp = i + 1 < n0 ? p[c + 1] : 0.0;
        v.ym = j > 0 ? p[c - sy] : 0.0;
        v.yp = j + 1 < n1 ? p[c + sy] : 0.0;
        v.zm = k > 0 ? p[c - sz] : 0.0;
        v.zp = k + 1 < n2 ? p[c + sz] : 0.0;
        const double t = b[c] - apply_row(g, i, j, k, v);
        spare[c] = t;
        acc.add(t * t);
        if (c == 0) gauge_sq = t * t;
        mx[0] = fmax(mx[0], fabs(t));
    }
    dd sums[2] = {acc.as_dd(), dd_add1(acc.as_dd(), -gauge_sq)};
    block_reduce<2, 1>(red, sums, mx);
    if (publish_and_check_last<2, 1>(I.part, sp.block, sp.blocks, sums, mx)) {
        fold_partials<2, 1>(I.part, sp.blocks, red, sums, mx);
        if (threadIdx.x == 0) decide_true(st, nullptr, dd_value(sums[0]), dd_value(sums[1]), mx[0], flags, g.volume);
    }
}

// Whether some instance's true residual asked for a restart (the restart
// branch of a trip runs only then).
__device__ __forceinline__ int any_replace(const BatchInstDev* inst, int count) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < count; i += blockDim.x)
        if (inst[i].st->flags & F_NEED_REPLACE) atomicOr(&any, 1);
    __syncthreads();
    return any;
}

// The end of a trip of the solve loop: counts the trip for every instance and
// tells whether any instance's solve still runs. The trip count is bounded:
// an instance still running at the bound ends with an execution error instead
// of looping on.
__device__ __forceinline__ int end_trip(BatchInstDev* inst, int count, int max_trips) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        SolveState* st = inst[i].st;
        const int trips = st->trips + 1;
        st->trips = trips;
        if (st->flags & F_DONE) continue;
        if (trips >= max_trips) {
            st->status = RB200_EXECUTION;
            st->flags = st->flags | F_DONE | F_STOP;
            continue;
        }
        atomicOr(&any, 1);
    }
    __syncthreads();
    return any;
}

// Graph conditions: the restart branch's IF node and the solve's WHILE node.
__global__ void k_b_any_replace(const BatchInstDev* inst, int count, cudaGraphConditionalHandle handle) {
    const int any = any_replace(inst, count);
    if (threadIdx.x == 0) cudaGraphSetConditional(handle, any ? 1u : 0u);
}
__global__ void k_b_loop_cond(BatchInstDev* inst, int count, cudaGraphConditionalHandle handle, int max_trips) {
    const int any = end_trip(inst, count, max_trips);
    if (threadIdx.x == 0) cudaGraphSetConditional(handle, any ? 1u : 0u);
}
// The same decisions for the eager (profiled) step, read by the host.
__global__ void k_b_any_replace_out(const BatchInstDev* inst, int count, int* out) {
    const int any = any_replace(inst, count);
    if (threadIdx.x == 0) *out = any;
}
__global__ void k_b_end_trip_out(BatchInstDev* inst, int count, int max_trips, int* out) {
    const int any = end_trip(inst, count, max_trips);
    if (threadIdx.x == 0) *out = any;
}

__global__ void __launch_bounds__(BT) k_b_correct(const BatchInstDev* __restrict__ inst, const __grid_constant__ BatchSpans spans) {
    __shared__ GridDev g;
    Span sp;
    const BatchInstDev& I = inst[batch_entry(spans, sp)];
    load_geometry(g, I.g);
    __syncthreads();
    BatchStepDev* cd = I.step;
    if (!usable(cd, I.st)) return;
    const int b = (cd->acc + 1) % 3, c = (cd->acc + 2) % 3;
    correct_divergence_body<float>(g, I.p, cd->dt, I.faces[b][0], I.faces[b][1], I.faces[b][2], I.faces[c][0],
                                   I.faces[c][1], I.faces[c][2], I.part, cd->scalars, &cd->flags, sp);
}

// Gates and commit per instance (src/simulation.rs:1235-1243, :1268-1277,
// :805-811), as the single carrier's k_step_end.
__global__ void k_b_end(BatchInstDev* inst, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BatchStepDev* cd = inst[i].step;
    const SolveState* st = inst[i].st;
    const GridDev& g = inst[i].g;
    rb200_step_report& rep = cd->report;
    rep.dt = cd->dt;
    rep.pressure.iterations = uint64_t(st->it);
    rep.pressure.true_residual_l2 = st->true_l2;
    rep.pressure.true_residual_max = st->true_max;
    rep.pressure.predicted_divergence_max = st->true_div;
    rep.pressure.incompatible_sum = st->incompatible_sum;
    rep.pressure.incompatible_budget = st->incompatible_budget;
    rep.pressure.breakdown_iteration = uint64_t(st->breakdown_it);
    rep.pressure_status = st->status;
    rep.actual_divergence_max = 0.0;
    rep.velocity_rate = 0.0;
    rep.courant = 0.0;
    cd->trips = st->trips;
    int status = cd->status;
    if (status == STEP_RUNNING) {
        if (!usable(cd, st)) {
            status = st->status;
        } else if (cd->flags & VF_NONFINITE) {
            status = RB200_NONFINITE_INPUT;
        } else if (cd->flags & (VF_ARITH | VF_F32_RANGE)) {
            status = RB200_ARITHMETIC_FAILURE;
        } else {
            double rate = 0.0;
            for (int d = 0; d < 3; ++d) rate += cd->scalars[1 + d] / g.h[d];
            rep.actual_divergence_max = cd->scalars[0];
            rep.velocity_rate = rate;
            rep.courant = cd->dt * rate;
            status = RB200_OK;
            if (!cd->skip_gates) {
                if (rep.actual_divergence_max > cd->divergence_limit)
                    status = RB200_DIVERGENCE_LIMIT;
                else if (!isfinite(rep.courant))
                    status = RB200_ARITHMETIC_FAILURE;
                else if (rep.courant > cd->max_courant)
                    status = RB200_COURANT_LIMIT;
            }
            if (status == RB200_OK) {
                cd->acc = (cd->acc + 2) % 3;
                cd->time += cd->dt;
                cd->generation += 1;
                cd->rate = rate;
            }
        }
    }
    rep.time = cd->time;
    rep.generation = cd->generation;
    rep.pressure_initialization = 0;
    cd->step_status = status;
    cd->status = status;
}

// ------------------------------------------------------------ host side
int ceil_div(long long a, long long b) { return int((a + b - 1) / b); }

BatchSpans make_spans(const std::vector<int>& blocks) {
    BatchSpans s{};
    s.count = int(blocks.size());
    s.first[0] = 0;
    for (size_t e = 0; e < blocks.size(); ++e) s.first[e + 1] = s.first[e] + blocks[e];
    return s;
}
int total_blocks(const BatchSpans& s) { return s.first[s.count]; }

// Blocks of a level loop over one level: one warp per row of work items.
int level_blocks(const MgLevelDev& L, int items, int rows_per_group = 1) {
    const long rows = long(L.n[1]) * L.n[2];
    const long rpw = (32 / lanes_for(items)) * rows_per_group;
    return std::max(1, ceil_div((rows + rpw - 1) / rpw, MG_THREADS / 32));
}

template <typename... KArgs, typename... Args>
cudaError_t launch(bool pdl, void (*kernel)(KArgs...), int blocks, int threads, size_t smem, cudaStream_t s,
                   Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(blocks), 1, 1);
    cfg.blockDim = dim3(unsigned(threads), 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

enum OpKind : int { OP_SMOOTH = 0, OP_PAIR = 1, OP_RESTRICT = 2, OP_PROLONG = 3, OP_LOWER = 4, OP_TRAIN = 5 };

// Strip rows of a level's sweep trains whose shared memory fits (0: none).
constexpr int kTrainChunk = 32;  // planes per block of a batch train

// Kernel kinds of a batched step, for the profiled step's per-kind times.
enum KernelKind : int {
    KK_SMOOTH = 0, KK_PAIR, KK_RESTRICT, KK_PROLONG, KK_LOWER,  // the V-cycle operations (OpKind order)
    KK_BEGIN, KK_ADVECT, KK_RHS, KK_RESET, KK_SUMS, KK_LOAD, KK_PASS1, KK_UPDATE, KK_FINISH, KK_TRUE,
    KK_CORRECT, KK_END, KK_CONTROL,
    KK_SMOOTH_FINE, KK_PAIR_FINE, KK_RESTRICT_FINE, KK_PROLONG_FINE,  // the same on the finest level
    KK_TRAIN, KK_TRAIN_FINE,
    KK_COUNT
};
const char* const kKernelNames[KK_COUNT] = {
    "k_b_smooth", "k_b_pair", "k_b_restrict", "k_b_prolong", "k_b_lower", "k_b_begin", "k_b_advect", "k_b_rhs",
    "k_b_reset", "k_b_init_sums", "k_b_load_residual", "k_b_pass1", "k_b_update_first", "k_b_finish",
    "k_b_true_residual", "k_b_correct", "k_b_end", "loop control", "k_b_smooth (finest)", "k_b_pair (finest)",
    "k_b_restrict (finest)", "k_b_prolong (finest)", "k_b_train", "k_b_train (finest)"};

// One launch of the V-cycle program: an operation over the instances that
// take part at that point of the cycle.
struct VLaunch {
    int kind;
    int level;        // the depth of the hierarchy it works on
    size_t first_op;  // index of its first entry in the batch's op table
    BatchSpans spans;
    size_t smem;
};

}  // namespace
}  // namespace rb200

using namespace rb200;

struct rb200_batch {
    rb200_batch_config cfg{};
    int device = 0;
    int count = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t body_stream = nullptr;
    cudaStream_t replace_stream = nullptr;
    std::vector<GridDev> grids;
    char* arena = nullptr;
    size_t bytes = 0;
    std::vector<BatchInstDev> inst;
    BatchInstDev* inst_d = nullptr;
    BatchStepDev* step_d = nullptr;
    BatchStepDev* step_h = nullptr;  // pinned mirror
    std::vector<std::vector<MgLevelDev>> levels;
    std::vector<std::vector<float*>> alt;
    std::vector<const double*> dense;
    std::vector<int> lower_first;        // per instance: its first level in the cluster kernel (>= 1)
    std::vector<BatchLowerDev> lower;    // per instance: the cluster kernel's table
    BatchLowerDev* lower_d = nullptr;
    int lower_cluster = 1;               // CTAs per instance in the cluster kernel
    std::vector<int> part_blocks;
    BatchLevelOp* ops_d = nullptr;
    std::vector<BatchLevelOp> ops;
    std::vector<VLaunch> vfirst;  // V-cycle whose finest level's first half-sweep starts from r
    std::vector<VLaunch> vrest;   // V-cycle after the fused update (first half-sweep done)
    BatchSpans sp_faces{}, sp_cells{}, sp_rows{}, sp_pass1{};
    size_t pair_smem = 0;   // largest dynamic shared memory of a pair launch
    size_t train_smem = 0;  // largest dynamic shared memory of a train launch
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[4] = {};
    int fixed_nodes = 0;
    int nodes_per_trip = 0;
    bool in_flight = false;
    std::string err;

    ~rb200_batch() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        if (exec) cudaGraphExecDestroy(exec);
        cudaFree(arena);
        cudaFree(inst_d);
        cudaFree(step_d);
        cudaFree(ops_d);
        cudaFree(lower_d);
        if (step_h) cudaFreeHost(step_h);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (replace_stream) cudaStreamDestroy(replace_stream);
        if (body_stream) cudaStreamDestroy(body_stream);
        if (stream) cudaStreamDestroy(stream);
    }

    int fail(int rc, const std::string& msg) {
        err = msg;
        set_error(msg);
        return rc;
    }

};

namespace {

// Builds the V-cycle program of the batch (the level walk of
// Multigrid::enqueue with sweep trains, one launch per operation over all
// instances). Buffers per non-coarsest level: the descent's train writes the
// second buffer (the restriction reads it there), the ascent's train reads it
// and writes the level's own x, where the finest level's finish and the next
// finer level's prolongation read it; the coarsest level has one buffer.
int build_program(rb200_batch* B) {
    const int n = B->count;
    int depth = 0;  // deepest non-coarsest level
    for (int i = 0; i < n; ++i) depth = std::max(depth, int(B->levels[i].size()) - 1);
    auto with_x = [&](int i, int l, bool second) {
        MgLevelDev L = B->levels[i][l];
        if (second) L.x = B->alt[i][l];
        return L;
    };
    auto coarsest = [&](int i, int l) { return l + 1 == int(B->levels[i].size()); };
    // The final buffer of level l >= 1 once its ascent is done: the second
    // one, except on the coarsest level (the dense solve writes its x).
    auto final_x = [&](int i, int l) { return with_x(i, l, !coarsest(i, l)); };
    // The final buffer of level l after the V-cycle below it: the cluster
    // kernel's first level ends in its second buffer when it is paired.
    auto final_of = [&](int i, int l) {
        if (l == B->lower_first[i]) return with_x(i, l, B->lower[i].P.paired[0] != 0);
        return final_x(i, l);
    };
    auto add = [&](std::vector<VLaunch>& prog, int kind, int l, auto make) {
        VLaunch v{};
        v.kind = kind;
        v.level = l;
        v.first_op = B->ops.size();
        std::vector<int> blocks;
        size_t smem = 0;
        for (int i = 0; i < n; ++i) {
            // levels from lower_first on belong to the cluster kernel
            if (l >= int(B->levels[i].size()) || coarsest(i, l) || (l >= 1 && l >= B->lower_first[i])) continue;
            BatchLevelOp op{};
            op.st = B->inst[i].st;
            int nb = make(i, op);
            if (kind == OP_TRAIN) smem = std::max(smem, train_launch_smem(op.L, op.C, kTrainPhases, op.sj, op.start));
            if (kind == OP_PAIR) smem = std::max(smem, size_t(PAIR_ROWS) * size_t(op.L.n[0]) * sizeof(float));
            B->ops.push_back(op);
            blocks.push_back(nb);
        }
        if (blocks.empty()) return;
        v.spans = make_spans(blocks);
        v.smem = smem;
        (kind == OP_PAIR ? B->pair_smem : B->train_smem) =
            std::max(kind == OP_PAIR ? B->pair_smem : B->train_smem, smem);
        prog.push_back(v);
    };
    // a train of kTrainPhases half-sweeps starting with colour c0 on level l of
    // instance i, from `in` into `out`
    auto train = [&](BatchLevelOp& op, int i, int l, const MgLevelDev& in, float* out, int c0,
                     int start) {
        op.L = in;
        op.out = out;
        op.color = c0;
        op.start = start;
        op.sj = train_strip(in, B->levels[i][l + 1].n[0], kTrainPhases);
        op.sk = kTrainChunk;
        if (start == TRAIN_PROLONG) op.C = final_of(i, l + 1);
        return ceil_div(in.n[1], op.sj) * ceil_div(in.n[2], op.sk);
    };
    for (int variant = 0; variant < 2; ++variant) {
        std::vector<VLaunch>& prog = variant == 0 ? B->vfirst : B->vrest;
        // descent: the finest level by a train, the coarser ones by pairs
        for (int l = 0; l < depth; ++l) {
            if (l == 0) {
                if (variant == 0)
                    add(prog, OP_SMOOTH, 0, [&](int i, BatchLevelOp& op) {
                        op.L = with_x(i, 0, false);
                        op.r0 = B->inst[i].r;
                        op.color = 0;
                        op.first = 1;
                        return level_blocks(op.L, sweep_items(op.L));
                    });
                // black, red, black after the first red half-sweep
                add(prog, OP_TRAIN, 0, [&](int i, BatchLevelOp& op) {
                    return train(op, i, 0, with_x(i, 0, false), B->alt[i][0], 1, TRAIN_OLD);
                });
                add(prog, OP_RESTRICT, 0, [&](int i, BatchLevelOp& op) {
                    op.L = with_x(i, 0, true);
                    op.C = B->levels[i][1];
                    return level_blocks(op.C, restrict_items(op.L, op.C), kFineRestrictRows);
                });
            } else {
                // two red-black pairs from a zero correction
                add(prog, OP_PAIR, l, [&](int i, BatchLevelOp& op) {
                    op.L = with_x(i, l, false);
                    op.out = B->alt[i][l];
                    op.color = 0;
                    op.first = 1;
                    return ceil_div(op.L.n[1], PJ) * ceil_div(op.L.n[2], PK);
                });
                add(prog, OP_PAIR, l, [&](int i, BatchLevelOp& op) {
                    op.L = with_x(i, l, true);
                    op.out = B->levels[i][l].x;
                    op.color = 0;
                    return ceil_div(op.L.n[1], PJ) * ceil_div(op.L.n[2], PK);
                });
                add(prog, OP_RESTRICT, l, [&](int i, BatchLevelOp& op) {
                    op.L = with_x(i, l, false);
                    op.C = B->levels[i][l + 1];
                    return level_blocks(op.C, restrict_items(op.L, op.C));
                });
            }
        }
        // every instance's levels of at most 32^3 cells and its coarsest solve
        {
            VLaunch v{};
            v.kind = OP_LOWER;
            prog.push_back(v);
        }
        // ascent: on the coarser levels prolongation with the black
        // half-sweep, a pair, red; on the finest level a train of the
        // prolongation with the black half-sweep, red, black (its last red is
        // the finish's)
        for (int l = depth - 1; l >= 1; --l) {
            add(prog, OP_PROLONG, l, [&](int i, BatchLevelOp& op) {
                op.L = with_x(i, l, false);
                op.C = final_of(i, l + 1);
                return level_blocks(op.L, sweep_items(op.L));
            });
            add(prog, OP_PAIR, l, [&](int i, BatchLevelOp& op) {
                op.L = with_x(i, l, false);
                op.out = B->alt[i][l];
                op.color = 0;
                return ceil_div(op.L.n[1], PJ) * ceil_div(op.L.n[2], PK);
            });
            add(prog, OP_SMOOTH, l, [&](int i, BatchLevelOp& op) {
                op.L = with_x(i, l, true);
                op.color = 0;
                return level_blocks(op.L, sweep_items(op.L));
            });
        }
        add(prog, OP_TRAIN, 0, [&](int i, BatchLevelOp& op) {
            return train(op, i, 0, with_x(i, 0, true), B->levels[i][0].x, 1, TRAIN_PROLONG);
        });
    }
    return RB200_OK;
}

// Issues the batched step's kernels on one stream: in a graph capture (no
// marks) or eagerly with an event after every launch (marks: the profiled
// step). Launch errors are kept in *e; launches are counted.
struct Emit {
    rb200_batch* B;
    cudaStream_t s;
    cudaError_t* e;
    std::vector<std::pair<int, cudaEvent_t>>* marks;
    int launches = 0;

    void keep(cudaError_t r) {
        if (r != cudaSuccess && *e == cudaSuccess) *e = r;
    }
    void mark(int kind) {
        if (!marks) return;
        cudaEvent_t ev = nullptr;
        keep(cudaEventCreate(&ev));
        keep(cudaEventRecord(ev, s));
        marks->push_back({kind, ev});
    }
    template <typename... KArgs, typename... Args>
    void go(int kind, bool pdl, void (*kernel)(KArgs...), int blocks, int threads, size_t smem, Args&&... args) {
        keep(launch(pdl && !marks, kernel, blocks, threads, smem, s, std::forward<Args>(args)...));
        ++launches;
        mark(kind);
    }
    void vcycle(const std::vector<VLaunch>& prog, int mode) {
        for (const VLaunch& v : prog) {
            const BatchLevelOp* o = B->ops_d + v.first_op;
            const int nb = total_blocks(v.spans);
            const bool fine = v.level == 0;
            switch (v.kind) {
                case OP_SMOOTH:
                    go(fine ? KK_SMOOTH_FINE : KK_SMOOTH, true, k_b_smooth, nb, MG_THREADS, 0, o, v.spans, mode);
                    break;
                case OP_PAIR:
                    go(fine ? KK_PAIR_FINE : KK_PAIR, true, k_b_pair, nb, MG_THREADS, v.smem, o, v.spans, mode);
                    break;
                case OP_RESTRICT:
                    go(fine ? KK_RESTRICT_FINE : KK_RESTRICT, true, k_b_restrict, nb, MG_THREADS, 0, o, v.spans, mode);
                    break;
                case OP_PROLONG:
                    go(fine ? KK_PROLONG_FINE : KK_PROLONG, true, k_b_prolong, nb, MG_THREADS, 0, o, v.spans, mode);
                    break;
                case OP_TRAIN:
                    go(fine ? KK_TRAIN_FINE : KK_TRAIN, true, k_b_train, nb, TRAIN_THREADS, v.smem, o, v.spans, mode);
                    break;
                default: {
                    // one cluster per instance
                    cudaLaunchConfig_t cfg{};
                    cfg.gridDim = dim3(unsigned(B->count * B->lower_cluster), 1, 1);
                    cfg.blockDim = dim3(MG_LOWER_THREADS, 1, 1);
                    cfg.stream = s;
                    cudaLaunchAttribute attr[2];
                    attr[0].id = cudaLaunchAttributeClusterDimension;
                    attr[0].val.clusterDim.x = unsigned(B->lower_cluster);
                    attr[0].val.clusterDim.y = 1;
                    attr[0].val.clusterDim.z = 1;
                    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                    attr[1].val.programmaticStreamSerializationAllowed = 1;
                    cfg.attrs = attr;
                    cfg.numAttrs = marks ? 1 : 2;
                    keep(cudaLaunchKernelEx(&cfg, k_b_lower, static_cast<const BatchLowerDev*>(B->lower_d), mode));
                    ++launches;
                    mark(KK_LOWER);
                    break;
                }
            }
        }
    }
    // dt policy, advection, RHS (then the solve's timing event in a graph)
    void head() {
        const int ib = ceil_div(B->count, 128);
        go(KK_BEGIN, false, k_b_begin, ib, 128, 0, B->inst_d, B->count);
        if (B->cfg.fp32_advection)
            go(KK_ADVECT, false, k_b_advect<float>, total_blocks(B->sp_faces), BT, 0, B->inst_d, B->sp_faces);
        else
            go(KK_ADVECT, false, k_b_advect<double>, total_blocks(B->sp_faces), BT, 0, B->inst_d, B->sp_faces);
        go(KK_RHS, false, k_b_rhs, total_blocks(B->sp_cells), BT, 0, B->inst_d, B->sp_cells);
    }
    // the solve's start: state, compatibility sums, residual, first V-cycle
    void start() {
        const int ib = ceil_div(B->count, 128);
        go(KK_RESET, false, k_b_reset, ib, 128, 0, B->inst_d, B->count, B->cfg.settings);
        go(KK_SUMS, false, k_b_init_sums, total_blocks(B->sp_cells), BT, 0, B->inst_d, B->sp_cells);
        go(KK_LOAD, true, k_b_load_residual, total_blocks(B->sp_cells), BT, 0, B->inst_d, B->sp_cells,
           int(MODE_INIT));
        vcycle(B->vfirst, MODE_INIT);
        go(KK_FINISH, true, k_b_finish, total_blocks(B->sp_rows), MG_THREADS, 0, B->inst_d, B->sp_rows,
           int(MODE_INIT));
    }
    void iteration() {
        go(KK_PASS1, true, k_b_pass1, total_blocks(B->sp_pass1), MG_THREADS, 0, B->inst_d, B->sp_pass1, kPass1Kc);
        go(KK_UPDATE, true, k_b_update_first, total_blocks(B->sp_rows), MG_THREADS, 0, B->inst_d, B->sp_rows);
        vcycle(B->vrest, MODE_ITER);
        go(KK_FINISH, true, k_b_finish, total_blocks(B->sp_rows), MG_THREADS, 0, B->inst_d, B->sp_rows,
           int(MODE_ITER));
    }
    void check() {
        go(KK_TRUE, true, k_b_true_residual, total_blocks(B->sp_cells), BT, 0, B->inst_d, B->sp_cells);
    }
    void restart() {
        go(KK_LOAD, false, k_b_load_residual, total_blocks(B->sp_cells), BT, 0, B->inst_d, B->sp_cells,
           int(MODE_REPLACE));
        vcycle(B->vfirst, MODE_REPLACE);
        go(KK_FINISH, true, k_b_finish, total_blocks(B->sp_rows), MG_THREADS, 0, B->inst_d, B->sp_rows,
           int(MODE_REPLACE));
    }
    // correction, gates and commit
    void tail() {
        go(KK_CORRECT, false, k_b_correct, total_blocks(B->sp_cells), BT, 0, B->inst_d, B->sp_cells);
        go(KK_END, false, k_b_end, ceil_div(B->count, 128), 128, 0, B->inst_d, B->count);
    }
};

int max_trips(const rb200_settings& set) {
    // at least one iteration per trip of a running solve: the iteration limit
    // ends a solve before this bound, however often it restarts
    const uint64_t trips = set.max_iterations + 64;
    return trips > (1u << 24) ? (1 << 24) : int(trips);
}

int capture(rb200_batch* B) {
    cudaStream_t s = B->stream;
    const int n = B->count;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaSuccess;
    Emit E{B, s, &e, nullptr};
    RB200_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    E.head();
    E.keep(cudaEventRecordWithFlags(B->ev[0], s, cudaEventRecordExternal));
    E.start();
    const int fixed_head = E.launches;
    // the solve loop: chunks of iterations, the true-residual check, the
    // restart branch, the condition
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraph_t outer = nullptr;
    E.keep(cudaStreamGetCaptureInfo(s, &status, nullptr, &outer, &deps, &ndeps));
    cudaGraphConditionalHandle handle{};
    E.keep(cudaGraphConditionalHandleCreate(&handle, outer, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node{};
    E.keep(cudaGraphAddNode(&node, outer, deps, ndeps, &cp));
    int per_trip = 0;
    if (e == cudaSuccess) {
        cudaStream_t bs = B->body_stream;
        E.keep(cudaStreamBeginCaptureToGraph(bs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeRelaxed));
        Emit body{B, bs, &e, nullptr};
        for (int q = 0; q < kChunk; ++q) body.iteration();
        body.check();
        // the restart as an IF node: its launches run only in trips where some
        // instance restarts
        cudaStreamCaptureStatus bst;
        const cudaGraphNode_t* bdeps = nullptr;
        size_t nbdeps = 0;
        cudaGraph_t bodyg = nullptr;
        body.keep(cudaStreamGetCaptureInfo(bs, &bst, nullptr, &bodyg, &bdeps, &nbdeps));
        cudaGraphConditionalHandle rh{};
        body.keep(cudaGraphConditionalHandleCreate(&rh, bodyg, 0, cudaGraphCondAssignDefault));
        body.go(KK_CONTROL, false, k_b_any_replace, 1, 128, 0, B->inst_d, n, rh);
        body.keep(cudaStreamGetCaptureInfo(bs, &bst, nullptr, &bodyg, &bdeps, &nbdeps));
        cudaGraphNodeParams ip{};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = rh;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        cudaGraphNode_t inode{};
        body.keep(cudaGraphAddNode(&inode, bodyg, bdeps, nbdeps, &ip));
        if (e == cudaSuccess) {
            cudaStream_t rs = B->replace_stream;
            body.keep(cudaStreamBeginCaptureToGraph(rs, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                    cudaStreamCaptureModeRelaxed));
            Emit branch{B, rs, &e, nullptr};
            branch.restart();
            cudaGraph_t rbody = nullptr;
            body.keep(cudaStreamEndCapture(rs, &rbody));
            body.keep(cudaStreamUpdateCaptureDependencies(bs, &inode, 1, cudaStreamSetCaptureDependencies));
        }
        body.go(KK_CONTROL, false, k_b_loop_cond, 1, 128, 0, B->inst_d, n, handle, max_trips(B->cfg.settings));
        per_trip = body.launches;  // the restart branch's launches run rarely and are not counted
        cudaGraph_t captured = nullptr;
        E.keep(cudaStreamEndCapture(bs, &captured));
        E.keep(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    }
    E.keep(cudaEventRecordWithFlags(B->ev[1], s, cudaEventRecordExternal));
    const int before_tail = E.launches;
    E.tail();
    E.keep(cudaMemcpyAsync(B->step_h, B->step_d, sizeof(BatchStepDev) * size_t(n), cudaMemcpyDeviceToHost, s));
    E.keep(cudaGetLastError());
    cudaError_t ee = cudaStreamEndCapture(s, &graph);
    if (e != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return B->fail(RB200_EXECUTION,
                       std::string("batch step capture: ") + cudaGetErrorString(e != cudaSuccess ? e : ee));
    }
    cudaError_t ie = cudaGraphInstantiate(&B->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return B->fail(RB200_EXECUTION, std::string("batch graph instantiate: ") + cudaGetErrorString(ie));
    B->fixed_nodes = fixed_head + (E.launches - before_tail);
    B->nodes_per_trip = per_trip;
    return RB200_OK;
}

// One batched step issued eagerly (the same kernels in the same order as the
// step graph, the loop decided on the host after each trip) with an event
// after every launch; per kernel kind the summed device time and the launches.
int profiled_step(rb200_batch* B, double* kind_ms, int* kind_launches) {
    cudaStream_t s = B->stream;
    cudaError_t e = cudaSuccess;
    std::vector<std::pair<int, cudaEvent_t>> marks;
    Emit E{B, s, &e, &marks};
    int* flag_d = nullptr;
    int flag_h = 0;
    RB200_CUDA(cudaMalloc(&flag_d, sizeof(int)));
    cudaEvent_t start = nullptr;
    E.keep(cudaEventCreate(&start));
    E.keep(cudaEventRecord(start, s));
    E.head();
    E.start();
    const int bound = max_trips(B->cfg.settings);
    for (int trip = 0; e == cudaSuccess && trip < bound; ++trip) {
        for (int q = 0; q < kChunk; ++q) E.iteration();
        E.check();
        E.go(KK_CONTROL, false, k_b_any_replace_out, 1, 128, 0, B->inst_d, B->count, flag_d);
        E.keep(cudaMemcpyAsync(&flag_h, flag_d, sizeof(int), cudaMemcpyDeviceToHost, s));
        E.keep(cudaStreamSynchronize(s));
        if (flag_h) E.restart();
        E.go(KK_CONTROL, false, k_b_end_trip_out, 1, 128, 0, B->inst_d, B->count, bound, flag_d);
        E.keep(cudaMemcpyAsync(&flag_h, flag_d, sizeof(int), cudaMemcpyDeviceToHost, s));
        E.keep(cudaStreamSynchronize(s));
        if (!flag_h) break;
    }
    E.tail();
    E.keep(cudaMemcpyAsync(B->step_h, B->step_d, sizeof(BatchStepDev) * size_t(B->count), cudaMemcpyDeviceToHost, s));
    E.keep(cudaStreamSynchronize(s));
    for (int k = 0; k < KK_COUNT; ++k) {
        kind_ms[k] = 0.0;
        kind_launches[k] = 0;
    }
    cudaEvent_t prev = start;
    for (auto& m : marks) {
        float ms = 0.0f;
        if (e == cudaSuccess) E.keep(cudaEventElapsedTime(&ms, prev, m.second));
        kind_ms[m.first] += double(ms);
        kind_launches[m.first] += 1;
        prev = m.second;
    }
    for (auto& m : marks) cudaEventDestroy(m.second);
    cudaEventDestroy(start);
    cudaFree(flag_d);
    if (e != cudaSuccess) return B->fail(RB200_EXECUTION, std::string("profiled batch step: ") + cudaGetErrorString(e));
    return RB200_OK;
}

// Alignment of every buffer in the arena (16-byte vector loads, coalescing).
constexpr size_t kAlign = 256;
size_t aligned(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

int validate_upload(rb200_batch* B, int i) {
    const GridDev& g = B->grids[i];
    BatchStepDev& h = B->step_h[i];
    BatchStepDev* d = B->step_d + i;
    const int a = h.acc;
    float* const* f = B->inst[i].faces[a];
    RB200_CUDA(cudaMemsetAsync(&d->flags, 0, sizeof(int), B->stream));
    int rc = launch_face_maxima<float>(g, f[0], f[1], f[2], B->inst[i].part, B->part_blocks[i], d->scalars, &d->flags,
                                       B->stream);
    if (!rc) rc = launch_validate_faces<float>(g, f[0], f[1], f[2], &d->flags, B->stream);
    if (rc) return rc;
    RB200_CUDA(cudaMemcpyAsync(&h, d, sizeof(BatchStepDev), cudaMemcpyDeviceToHost, B->stream));
    RB200_CUDA(cudaStreamSynchronize(B->stream));
    if (h.flags & VF_NONFINITE) return RB200_NONFINITE_INPUT;
    if (h.flags & VF_WALL) return RB200_NONZERO_WALL_VELOCITY;
    double r = 0.0;
    for (int dd = 0; dd < 3; ++dd) r += h.scalars[dd] / g.h[dd];
    h.rate = r;
    h.time = 0.0;
    h.generation = 0;
    h.status = RB200_OK;
    h.flags = 0;
    RB200_CUDA(cudaMemcpyAsync(d, &h, sizeof(BatchStepDev), cudaMemcpyHostToDevice, B->stream));
    RB200_CUDA(cudaStreamSynchronize(B->stream));
    return RB200_OK;
}

}  // namespace

extern "C" {

int rb200_batch_create(const rb200_grid* grids, size_t count, const rb200_batch_config* config, rb200_batch** out) {
    if (!grids || !config || !out || count == 0) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    if (count > size_t(kBatchMax)) {
        set_error("a batch holds at most " + std::to_string(kBatchMax) + " instances");
        return RB200_UNSUPPORTED;
    }
    if (!settings_valid(&config->settings)) return RB200_INVALID_ARGUMENT;
    if (!(config->max_courant > 0.0) || !std::isfinite(config->actual_divergence_limit)) return RB200_INVALID_ARGUMENT;
    int rc = select_device(config->device);
    if (rc) return rc;
    std::unique_ptr<rb200_batch> B(new (std::nothrow) rb200_batch());
    if (!B) return RB200_OUT_OF_MEMORY;
    B->cfg = *config;
    B->device = config->device;
    B->count = int(count);
    // geometry, hierarchy and the arena's size
    size_t total = 0;
    std::vector<std::vector<double>> Gs(count);
    for (size_t i = 0; i < count; ++i) {
        GridDev g;
        if ((rc = make_grid_dev(&grids[i], config->density, &g))) return rc;
        B->grids.push_back(g);
        std::vector<MgLevelDev> lv = mg_level_geometry(g);
        if (lv.size() < 2) {
            set_error("batch instance " + std::to_string(i) + ": every axis has at most 8 cells (no hierarchy)");
            return RB200_UNSUPPORTED;
        }
        for (size_t l = 0; l + 1 < lv.size(); ++l)
            if (!mg_level_pairable(lv[l]) || (l == 0 && !train_strip(lv[0], lv[1].n[0], kTrainPhases))) {
                set_error("batch instance " + std::to_string(i) + ": level " + std::to_string(l) +
                          " rows are not a multiple of 4 cells (x extent " + std::to_string(lv[l].n[0]) + ")");
                return RB200_UNSUPPORTED;
            }
        if (!mg_coarse_pseudo_inverse(lv.back(), Gs[i])) {
            set_error("multigrid coarsest-level factorisation failed");
            return RB200_UNSUPPORTED;
        }
        B->levels.push_back(lv);
    }
    // block spans of the elementwise, row and direction passes; partials
    std::vector<int> bf, bc, br, bp;
    for (size_t i = 0; i < count; ++i) {
        const GridDev& g = B->grids[i];
        const long long faces = (long long)g.flen[0] + g.flen[1] + g.flen[2];
        bf.push_back(ceil_div(faces, BT * kItems));
        bc.push_back(ceil_div(g.cells, BT * kCellItems));
        br.push_back(ceil_div((long long)g.n[1] * g.n[2], (MG_THREADS / 32) * kRowsPerWarp));
        const int qsegs = ceil_div(g.n[0] / 4, 32);
        const long long lines = (long long)qsegs * g.n[1] * ceil_div(g.n[2], kPass1Kc);
        bp.push_back(std::max(1, ceil_div(lines, MG_THREADS / 32)));
        const int fm = std::min(ceil_div(g.flen[0], EW_THREADS), EW_BLOCKS_CAP);  // face maxima on upload
        B->part_blocks.push_back(std::max({bc.back(), br.back(), bp.back(), fm}));
    }
    B->sp_faces = make_spans(bf);
    B->sp_cells = make_spans(bc);
    B->sp_rows = make_spans(br);
    B->sp_pass1 = make_spans(bp);
    for (size_t i = 0; i < count; ++i) {
        const GridDev& g = B->grids[i];
        for (int a = 0; a < 3; ++a) total += 3 * aligned(size_t(g.flen[a]) * sizeof(float));
        total += 6 * aligned(size_t(g.cells) * sizeof(double));
        total += aligned(sizeof(SolveState)) + aligned(sizeof(unsigned));
        total += aligned(size_t(B->part_blocks[i]) * kSlotDoubles * sizeof(double));
        const auto& lv = B->levels[i];
        for (size_t l = 0; l < lv.size(); ++l)
            total += (l + 1 < lv.size() ? 3 : 2) * aligned(size_t(lv[l].cells) * sizeof(float));
        total += aligned(Gs[i].size() * sizeof(double));
    }
    RB200_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    RB200_CUDA(cudaStreamCreateWithFlags(&B->body_stream, cudaStreamNonBlocking));
    RB200_CUDA(cudaStreamCreateWithFlags(&B->replace_stream, cudaStreamNonBlocking));
    if (cudaMalloc(&B->arena, total) != cudaSuccess) {
        cudaGetLastError();
        return B->fail(RB200_OUT_OF_MEMORY, "batch arena of " + std::to_string(total) + " bytes");
    }
    B->bytes = total;
    RB200_CUDA(cudaMemsetAsync(B->arena, 0, total, B->stream));
    RB200_CUDA(cudaMalloc(&B->step_d, sizeof(BatchStepDev) * count));
    RB200_CUDA(cudaMallocHost(&B->step_h, sizeof(BatchStepDev) * count));
    std::memset(B->step_h, 0, sizeof(BatchStepDev) * count);
    char* cur = B->arena;
    auto take = [&](size_t nbytes) {
        char* p = cur;
        cur += aligned(nbytes);
        return p;
    };
    B->inst.resize(count);
    B->alt.resize(count);
    B->dense.resize(count);
    for (size_t i = 0; i < count; ++i) {
        const GridDev& g = B->grids[i];
        BatchInstDev& I = B->inst[i];
        std::memset(&I, 0, sizeof(I));
        I.g = g;
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) I.faces[b][a] = reinterpret_cast<float*>(take(size_t(g.flen[a]) * 4));
        double** vec[6] = {&I.b, &I.p, &I.r, &I.r1, &I.d0, &I.d1};
        for (double** v : vec) *v = reinterpret_cast<double*>(take(size_t(g.cells) * 8));
        I.st = reinterpret_cast<SolveState*>(take(sizeof(SolveState)));
        I.part.ticket = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
        I.part.data = reinterpret_cast<double*>(take(size_t(B->part_blocks[i]) * kSlotDoubles * 8));
        I.step = B->step_d + i;
        auto& lv = B->levels[i];
        B->alt[i].assign(lv.size(), nullptr);
        for (size_t l = 0; l < lv.size(); ++l) {
            lv[l].x = reinterpret_cast<float*>(take(size_t(lv[l].cells) * 4));
            lv[l].b = reinterpret_cast<float*>(take(size_t(lv[l].cells) * 4));
            if (l + 1 < lv.size()) B->alt[i][l] = reinterpret_cast<float*>(take(size_t(lv[l].cells) * 4));
        }
        I.fine = lv[0];
        double* G = reinterpret_cast<double*>(take(Gs[i].size() * 8));
        RB200_CUDA(cudaMemcpyAsync(G, Gs[i].data(), Gs[i].size() * 8, cudaMemcpyHostToDevice, B->stream));
        B->dense[i] = G;
        // the cluster kernel's levels: those of at most 32^3 cells below the
        // finest (at least the coarsest)
        int lf = int(lv.size()) - 1;
        while (lf > 1 && lv[lf - 1].cells <= kMgLowerCells) --lf;
        if (int(lv.size()) - lf > kMgMaxLower)
            return B->fail(RB200_UNSUPPORTED, "batch instance " + std::to_string(i) + ": hierarchy too deep");
        BatchLowerDev T{};
        T.P.count = int(lv.size()) - lf;
        for (int q = 0; q < T.P.count; ++q) {
            const MgLevelDev& L = lv[lf + q];
            T.P.lv[0][q] = L;
            T.P.lv[1][q] = L;
            T.P.paired[q] = (lf + q + 1 < int(lv.size()) && (L.n[0] & 3) == 0 && L.n[0] <= LPAIR_N0) ? 1 : 0;
            if (T.P.paired[q]) T.P.lv[1][q].x = B->alt[i][lf + q];
        }
        T.G = G;
        T.st = I.st;
        B->lower_first.push_back(lf);
        B->lower.push_back(T);
        BatchStepDev& h = B->step_h[i];
        h.max_courant = config->max_courant;
        h.divergence_limit = config->actual_divergence_limit;
        h.status = RB200_OK;
    }
    RB200_CUDA(cudaMalloc(&B->inst_d, sizeof(BatchInstDev) * count));
    RB200_CUDA(cudaMemcpyAsync(B->inst_d, B->inst.data(), sizeof(BatchInstDev) * count, cudaMemcpyHostToDevice,
                               B->stream));
    RB200_CUDA(cudaMemcpyAsync(B->step_d, B->step_h, sizeof(BatchStepDev) * count, cudaMemcpyHostToDevice,
                               B->stream));
    if ((rc = build_program(B.get()))) return rc;
    // the cluster kernel (one 1024-thread CTA per SM): the widest portable
    // cluster that keeps every instance's cluster resident at once
    int sms = 148;
    RB200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B->device));
    for (int cs : {8, 4, 2, 1})
        if (cs == 1 || B->count * cs <= sms) {
            B->lower_cluster = cs;
            break;
        }
    RB200_CUDA(cudaMalloc(&B->lower_d, sizeof(BatchLowerDev) * B->lower.size()));
    RB200_CUDA(cudaMemcpyAsync(B->lower_d, B->lower.data(), sizeof(BatchLowerDev) * B->lower.size(),
                               cudaMemcpyHostToDevice, B->stream));
    RB200_CUDA(cudaMalloc(&B->ops_d, sizeof(BatchLevelOp) * B->ops.size()));
    RB200_CUDA(cudaMemcpyAsync(B->ops_d, B->ops.data(), sizeof(BatchLevelOp) * B->ops.size(), cudaMemcpyHostToDevice,
                               B->stream));
    if (B->train_smem)
        RB200_CUDA(cudaFuncSetAttribute(k_b_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(B->train_smem)));
    if (B->pair_smem)
        RB200_CUDA(cudaFuncSetAttribute(k_b_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, int(B->pair_smem)));
    for (auto& e : B->ev) RB200_CUDA(cudaEventCreate(&e));
    RB200_CUDA(cudaStreamSynchronize(B->stream));
    if ((rc = capture(B.get()))) return rc;
    *out = B.release();
    return RB200_OK;
}

void rb200_batch_destroy(rb200_batch* batch) { delete batch; }

uint64_t rb200_batch_allocated_bytes(const rb200_batch* batch) { return batch ? uint64_t(batch->bytes) : 0; }

void* rb200_batch_stream(rb200_batch* batch) { return batch ? (void*)batch->stream : nullptr; }

const char* rb200_batch_last_error(const rb200_batch* batch) { return batch ? batch->err.c_str() : ""; }

int rb200_batch_upload(rb200_batch* batch, size_t index, const float* u, const float* v, const float* w) {
    if (!batch || !u || !v || !w) return RB200_INVALID_ARGUMENT;
    if (index >= size_t(batch->count)) return RB200_INVALID_ARGUMENT;
    if (batch->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(batch->device);
    const int i = int(index);
    const int a = batch->step_h[i].acc;
    const float* src[3] = {u, v, w};
    for (int d = 0; d < 3; ++d)
        RB200_CUDA(cudaMemcpyAsync(batch->inst[i].faces[a][d], src[d], size_t(batch->grids[i].flen[d]) * 4,
                                   cudaMemcpyDefault, batch->stream));
    return validate_upload(batch, i);
}

int rb200_batch_download(rb200_batch* batch, size_t index, float* u, float* v, float* w) {
    if (!batch || index >= size_t(batch ? batch->count : 0)) return RB200_INVALID_ARGUMENT;
    if (batch->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(batch->device);
    const int i = int(index);
    const int a = batch->step_h[i].acc;
    float* dst[3] = {u, v, w};
    for (int d = 0; d < 3; ++d)
        if (dst[d])
            RB200_CUDA(cudaMemcpyAsync(dst[d], batch->inst[i].faces[a][d], size_t(batch->grids[i].flen[d]) * 4,
                                       cudaMemcpyDefault, batch->stream));
    RB200_CUDA(cudaStreamSynchronize(batch->stream));
    return RB200_OK;
}

int rb200_batch_pressure(rb200_batch* batch, size_t index, double* out, size_t len) {
    if (!batch || !out || index >= size_t(batch->count)) return RB200_INVALID_ARGUMENT;
    if (batch->in_flight) return RB200_INVALID_ARGUMENT;
    const int i = int(index);
    if (len != size_t(batch->grids[i].cells)) return RB200_LENGTH_MISMATCH;
    cudaSetDevice(batch->device);
    RB200_CUDA(cudaMemcpyAsync(out, batch->inst[i].p, len * sizeof(double), cudaMemcpyDefault, batch->stream));
    RB200_CUDA(cudaStreamSynchronize(batch->stream));
    return RB200_OK;
}

int rb200_batch_step_async(rb200_batch* batch, const rb200_step_params* params) {
    if (!batch || !params) return RB200_INVALID_ARGUMENT;
    rb200_batch* B = batch;
    if (B->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(B->device);
    for (int i = 0; i < B->count; ++i) {
        BatchStepDev& h = B->step_h[i];
        h.requested_dt = params[i].requested_dt;
        h.cfl = params[i].cfl;
        h.iteration_limit_ok = params[i].iteration_limit_ok;
        h.skip_gates = params[i].skip_gates;
        if (params[i].buoyancy != 0.0) {
            B->err = "batched instances carry no tracer: buoyancy must be 0";
            return RB200_INVALID_ARGUMENT;
        }
    }
    // The mirror holds the device state of the last completed step (copied
    // back at the end of every step graph) with this step's parameters.
    RB200_CUDA(cudaMemcpyAsync(B->step_d, B->step_h, sizeof(BatchStepDev) * size_t(B->count), cudaMemcpyHostToDevice,
                               B->stream));
    RB200_CUDA(cudaEventRecord(B->ev[2], B->stream));
    RB200_CUDA(cudaGraphLaunch(B->exec, B->stream));
    RB200_CUDA(cudaEventRecord(B->ev[3], B->stream));
    B->in_flight = true;
    return RB200_OK;
}

int rb200_batch_step_poll(const rb200_batch* batch) {
    if (!batch || !batch->in_flight) return 0;
    cudaSetDevice(batch->device);
    return cudaEventQuery(batch->ev[3]) == cudaSuccess ? 1 : 0;
}

int rb200_batch_step_wait(rb200_batch* batch, rb200_step_report* reports, int* statuses) {
    if (!batch || !reports || !statuses) return RB200_INVALID_ARGUMENT;
    rb200_batch* B = batch;
    if (!B->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(B->device);
    B->in_flight = false;
    RB200_CUDA(cudaStreamSynchronize(B->stream));
    float ms = 0.0f;
    const bool timed = cudaEventElapsedTime(&ms, B->ev[0], B->ev[1]) == cudaSuccess;
    int trips = 0;
    for (int i = 0; i < B->count; ++i) trips = std::max(trips, B->step_h[i].trips);
    for (int i = 0; i < B->count; ++i) {
        reports[i] = B->step_h[i].report;
        if (timed) reports[i].pressure_ms = double(ms);
        reports[i].kernel_launches = uint64_t(B->fixed_nodes) + uint64_t(trips) * uint64_t(B->nodes_per_trip);
        statuses[i] = B->step_h[i].step_status;
    }
    return RB200_OK;
}

int rb200_batch_profile_step(rb200_batch* batch, const rb200_step_params* params, rb200_step_report* reports,
                             int* statuses, double* kernel_ms, int* kernel_launches, const char** kernel_names,
                             int kinds) {
    if (!batch || !params || !reports || !statuses || !kernel_ms || !kernel_launches) return RB200_INVALID_ARGUMENT;
    if (kinds < KK_COUNT) return RB200_LENGTH_MISMATCH;
    rb200_batch* B = batch;
    if (B->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(B->device);
    for (int i = 0; i < B->count; ++i) {
        BatchStepDev& h = B->step_h[i];
        h.requested_dt = params[i].requested_dt;
        h.cfl = params[i].cfl;
        h.iteration_limit_ok = params[i].iteration_limit_ok;
        h.skip_gates = params[i].skip_gates;
        if (params[i].buoyancy != 0.0) return RB200_INVALID_ARGUMENT;
    }
    RB200_CUDA(cudaMemcpyAsync(B->step_d, B->step_h, sizeof(BatchStepDev) * size_t(B->count), cudaMemcpyHostToDevice,
                               B->stream));
    int rc = profiled_step(B, kernel_ms, kernel_launches);
    if (rc) return rc;
    for (int k = 0; k < KK_COUNT; ++k)
        if (kernel_names) kernel_names[k] = kKernelNames[k];
    for (int i = 0; i < B->count; ++i) {
        reports[i] = B->step_h[i].report;
        statuses[i] = B->step_h[i].step_status;
    }
    return RB200_OK;
}

int rb200_batch_profile_kinds(void) { return KK_COUNT; }

int rb200_batch_step(rb200_batch* batch, const rb200_step_params* params, rb200_step_report* reports, int* statuses) {
    int rc = rb200_batch_step_async(batch, params);
    if (rc) return rc;
    return rb200_batch_step_wait(batch, reports, statuses);
}

}  // extern "C"
