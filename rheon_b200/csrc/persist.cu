// Persistent Jacobi-PCG: one cooperative kernel runs a whole chunk of
// iterations of PressureWorkspace::solve_loaded (src/pressure.rs:577-740)
// with the "jacobi-pcg-v1" preconditioner (:534-575), true-residual checks and
// restarts included, without returning to the host or the graph between
// passes.
//
// Each block (one per SM) owns a fixed, strided set of 32 x 8 x 8 bricks and
// is warp-specialised: one producer warp streams the bricks' slabs into a
// three-stage shared-memory ring with TMA (a stage is refilled once the 16
// consumer warps have released it through its "empty" mbarrier), and the 16
// consumer warps (512 threads, two threads per cell column, four cells each)
// compute from the ring without block-wide barriers. At the end of a phase the
// block reduces its dot products, publishes them and meets the other blocks
// at a grid barrier; every block then folds all partials in the same fixed
// order and takes the same decision on its own shared-memory copy of the
// solver state, so the blocks stay in lock-step without a second barrier.
// Block 0 writes the state back at the end of the launch.
//
// Phases per iteration (bytes per cell, f64):
//   1  d <- z + beta d (or z after a restart), q = K d, d.q      read z, d; write d          24
//   2  p += alpha d, r -= alpha K d, z = r/D, r.r, r.z           read d, p, r; write p, r, z  48
// and on a candidate:
//   3  t = b - K p, |t|_2, max|t| -> accept / stop / restart     read p, b; write t          24
//   4  (restart) r = t, z = r/D, r.z                             read t; write r, z          24
// Phase 1 forms the new direction on the fly from the z and d slabs for
// every value the stencil reads (the same z + beta*d per element), so the
// slabs are never written.
//
// Liveness: the kernel is launched cooperatively, so all blocks are
// co-resident. Every wait is bounded: a TMA or ring wait or a grid barrier
// that runs out marks the solve as failed (execution error) and raises an
// abort word that ends every other block's barrier wait, and the kernel
// returns.
#include <type_traits>

#include "pcg.hpp"
#include "slab.cuh"
#include "solve_state.cuh"

namespace rb200 {

namespace {

constexpr int PZ = 2;                        // consumer threads per cell column
constexpr int CONSUMERS = TX * TY * PZ;      // consumer threads (16 warps)
constexpr int CONSUMER_WARPS = CONSUMERS / 32;
constexpr int PT = CONSUMERS + 32;           // + one producer warp
constexpr int PZC = 8;                       // brick depth (the slab maps' box depth)
constexpr int QPT = PZC / PZ;                // cells per thread per brick
constexpr int NS = 3;                        // ring stages
using PS = Slab<PZC>;
constexpr int BOX = TX * TY * PZC;           // cells of one brick (no halo)
constexpr unsigned BOX_BYTES = unsigned(BOX) * 8u;
// A stage holds two slabs (phase 1), or one slab and two bricks (phase 2).
constexpr int STAGE = (2 * PS::SIZE > PS::SIZE + 2 * BOX) ? 2 * PS::SIZE : PS::SIZE + 2 * BOX;
constexpr size_t kPersistSmem = NS * size_t(STAGE) * sizeof(double);
constexpr unsigned kBarrierSpins = 1u << 24;
constexpr int PSTRIDE = 6;                   // doubles per block per partial set (2K + M <= 5)
constexpr int kFoldPerLane = 8;              // blocks folded per lane: grids of up to 256 blocks
constexpr int kMaxPersistBlocks = 32 * kFoldPerLane;

__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
    return v;
}
// Arrival without a return value: releases this block's writes (ordered
// before it by the block barrier); the waiting loads acquire everyone's.
__device__ __forceinline__ void red_add_release_gpu(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}
// Order this thread's generic-proxy global accesses with its (or, through a
// barrier, its block's) later TMA (async-proxy) accesses.
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

struct PersistArgs {
    GridDev g;
    SolveState* st;
    const double* b;
    double* p;
    double* r;
    double* z;
    double* d0;
    double* d1;
    double* part;      // [2][blocks][PSTRIDE]
    GridBarrier* bar;
    rb200_trace* trace;
    int budget;        // iterations this launch may start
};

// Per-block context.
struct Ctx {
    int nbx, nby, nbricks, mine;  // bricks along x, y; in total; of this block
    int bx0, by0, bz0;            // brick coordinates of this block's first brick
    int sx, sy, sz;               // the grid stride (gridDim.x bricks) as brick coordinates
    int tid, lane, tx, ty, tz;
    bool producer;
    unsigned ring;     // ring slots used so far (same count in every thread)
    unsigned long long target;  // arrival count that ends the next barrier (thread 0)
    int set;           // partial set parity
};

// Walks the block's bricks b = blockIdx.x + n * gridDim.x, keeping their
// coordinates by carries instead of divisions.
struct BrickWalk {
    int b, bx, by, bz;
    __device__ __forceinline__ explicit BrickWalk(const Ctx& c) : b(blockIdx.x), bx(c.bx0), by(c.by0), bz(c.bz0) {}
    __device__ __forceinline__ void next(const Ctx& c) {
        b += gridDim.x;
        bx += c.sx;
        int carry = bx >= c.nbx;
        bx -= carry ? c.nbx : 0;
        by += c.sy + carry;
        carry = by >= c.nby;
        by -= carry ? c.nby : 0;
        bz += c.sz + carry;
    }
    __device__ __forceinline__ int x0() const { return bx * TX; }
    __device__ __forceinline__ int y0() const { return by * TY; }
    __device__ __forceinline__ int k0() const { return bz * PZC; }
};

// One consumer thread's column of a brick: cells (i, j, k0 + qb .. + QPT - 1).
struct Col {
    int k0, kend;   // brick origin in z; cells of the brick in z
    int cc0;        // cell index of the column's first cell
    int e0;         // slab element of the column's first cell
    int bi0;        // brick (no halo) element of the column's first cell
    int mxy;        // neighbour-mask bits of x and y (src/operator.rs:813-822 order)
    bool own;       // the column lies inside the domain
};

__device__ __forceinline__ Col column(const GridDev& g, const Ctx& c, const BrickWalk& w, int qb) {
    const int x0 = w.x0(), y0 = w.y0(), k0 = w.k0();
    const int i = x0 + c.tx, j = y0 + c.ty;
    Col col;
    col.own = i < g.n[0] && j < g.n[1];
    col.k0 = k0;
    col.kend = min(PZC, g.n[2] - k0);
    col.cc0 = i + g.n[0] * (j + g.n[1] * (k0 + qb));
    col.e0 = PS::own(c.tx, c.ty, qb);
    col.bi0 = c.tx + TX * (c.ty + TY * qb);
    col.mxy = int(i > 0) | (int(i + 1 < g.n[0]) << 1) | (int(j > 0) << 2) | (int(j + 1 < g.n[1]) << 3);
    return col;
}

// Row of K applied to one cell (apply_full, src/operator.rs:400-416): the
// terms in the order X lower, X upper, Y lower, Y upper, Z lower, Z upper,
// with the x/y masks precomputed per column. ZIN: the cell has both z
// neighbours (a brick strictly inside the box in z).
template <bool ZIN = false>
__device__ __forceinline__ double row7(const GridDev& g, int mxy, int k, double cv, double xm, double xp, double ym,
                                       double yp, double zm, double zp) {
    double q = 0.0;
    if (mxy & 1) q += g.weight[0] * (cv - xm);
    if (mxy & 2) q += g.weight[0] * (cv - xp);
    if (mxy & 4) q += g.weight[1] * (cv - ym);
    if (mxy & 8) q += g.weight[1] * (cv - yp);
    if (ZIN || k > 0) q += g.weight[2] * (cv - zm);
    if (ZIN || k + 1 < g.n[2]) q += g.weight[2] * (cv - zp);
    return q;
}

__device__ __forceinline__ int zmask(const GridDev& g, int k) { return (int(k > 0) << 4) | (int(k + 1 < g.n[2]) << 5); }

// Two interleaved compensated accumulators (even and odd terms), merged in
// double-double: half the dependent-add chain of one.
struct Neu2 {
    Neu a, b;
    __device__ __forceinline__ dd as_dd() const { return dd_add(a.as_dd(), b.as_dd()); }
};

// Grid barrier: arrive (release), wait until every block of the grid has
// arrived (acquire). Returns false, with the abort word raised, when the wait
// runs out or another block aborted.
__device__ __forceinline__ bool grid_barrier(Ctx& c, GridBarrier* gb) {
    __shared__ int s_ok;
    fence_proxy_async_global();
    __syncthreads();
    if (c.tid == 0) {
        int ok = 1;
        c.target += gridDim.x;
        red_add_release_gpu(&gb->count, 1ull);
        unsigned n = 0;
        while (ld_acquire_gpu(&gb->count) < c.target) {
            if ((++n & 7u) == 0u && (*(volatile unsigned*)&gb->abort != 0u || n > kBarrierSpins)) {
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        fence_proxy_async_global();
        if (!ok) atomicExch(&gb->abort, 1u);
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Block reduction of this block's K sums and M maxima into thread 0, with the
// block's pipeline outcome `ok` and-reduced at the same barrier.
template <int K, int M>
__device__ __forceinline__ bool block_reduce_ok(BlockReduce<K, M>& sm, dd (&sums)[K > 0 ? K : 1],
                                                double (&maxs)[M > 0 ? M : 1], bool ok) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = PT / 32;
#pragma unroll
    for (int q = 0; q < K; ++q) sums[q] = warp_reduce_dd(sums[q]);
#pragma unroll
    for (int q = 0; q < M; ++q) maxs[q] = warp_reduce_max(maxs[q]);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) sm.s[warp][q] = sums[q];
#pragma unroll
        for (int q = 0; q < M; ++q) sm.m[warp][q] = maxs[q];
    }
    if (!__syncthreads_and(ok)) return false;
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) sums[q] = lane < NW ? sm.s[lane][q] : dd{0.0, 0.0};
#pragma unroll
        for (int q = 0; q < M; ++q) maxs[q] = lane < NW ? sm.m[lane][q] : 0.0;
#pragma unroll
        for (int q = 0; q < K; ++q) sums[q] = warp_reduce_dd(sums[q]);
#pragma unroll
        for (int q = 0; q < M; ++q) maxs[q] = warp_reduce_max(maxs[q]);
    }
    return true;
}

// Publish this block's K sums and M maxima, meet the other blocks, and fold
// all blocks' partials in warp 0 (lane l takes blocks l, l + 32, ... and adds
// them pairwise, then the lanes are combined by the butterfly). The fold is
// identical in every block. `ok` is this thread's pipeline outcome; a failure
// anywhere in the block fails the block before it arrives. Result valid in
// thread 0.
template <int K, int M>
__device__ __forceinline__ bool reduce_grid(Ctx& c, const PersistArgs& A, bool ok, dd (&sums)[K > 0 ? K : 1],
                                            double (&maxs)[M > 0 ? M : 1]) {
    __shared__ BlockReduce<K, M> red;
    if (!block_reduce_ok<K, M>(red, sums, maxs, ok)) return false;
    double* base = A.part + size_t(c.set) * gridDim.x * PSTRIDE;
    if (c.tid == 0) {
        double* slot = base + size_t(blockIdx.x) * PSTRIDE;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            slot[2 * q] = sums[q].hi;
            slot[2 * q + 1] = sums[q].lo;
        }
#pragma unroll
        for (int q = 0; q < M; ++q) slot[2 * K + q] = maxs[q];
    }
    c.set ^= 1;
    if (!grid_barrier(c, A.bar)) return false;
    if (c.tid < 32) {
        dd v[kFoldPerLane][K > 0 ? K : 1];
        double mv[M > 0 ? M : 1];
#pragma unroll
        for (int q = 0; q < M; ++q) mv[q] = 0.0;
#pragma unroll
        for (int u = 0; u < kFoldPerLane; ++u) {
            const int b = c.lane + 32 * u;
            const double* slot = base + size_t(b) * PSTRIDE;
            const bool have = b < int(gridDim.x);
#pragma unroll
            for (int q = 0; q < K; ++q)
                v[u][q] = have ? dd{__ldcg(slot + 2 * q), __ldcg(slot + 2 * q + 1)} : dd{0.0, 0.0};
#pragma unroll
            for (int q = 0; q < M; ++q) mv[q] = have ? fmax(mv[q], __ldcg(slot + 2 * K + q)) : mv[q];
        }
#pragma unroll
        for (int w = 1; w < kFoldPerLane; w *= 2)
#pragma unroll
            for (int u = 0; u + w < kFoldPerLane; u += 2 * w)
#pragma unroll
                for (int q = 0; q < K; ++q) v[u][q] = dd_add(v[u][q], v[u + w][q]);
#pragma unroll
        for (int q = 0; q < K; ++q) sums[q] = warp_reduce_dd(v[0][q]);
#pragma unroll
        for (int q = 0; q < M; ++q) maxs[q] = warp_reduce_max(mv[q]);
    }
    return true;
}

// Stream the block's bricks through the ring. The producer's lane 0 waits for
// a free slot and runs issue(b, slot) (which arms full[slot] and starts the
// copies); every consumer thread waits for the slot's data, runs
// body(b, slot) and its warp releases the slot. Returns this thread's outcome.
template <class Issue, class Body>
__device__ __forceinline__ bool run_bricks(Ctx& c, uint64_t* full, uint64_t* empty, Issue issue, Body body) {
    bool ok = true;
    unsigned slot_count = c.ring;
    if (c.producer) {
        if (c.lane == 0) {
            // order the data this block saw through the grid barrier before
            // the TMA (async-proxy) reads below
            fence_proxy_async_global();
            for (BrickWalk w(c); w.b < c.nbricks; w.next(c), ++slot_count) {
                const unsigned slot = slot_count % NS, phase = (slot_count / NS) & 1u;
                if (!mbar_wait_bounded(&empty[slot], phase ^ 1u)) {
                    ok = false;
                    break;
                }
                issue(w, int(slot));
            }
        }
    } else {
        for (BrickWalk w(c); w.b < c.nbricks; w.next(c), ++slot_count) {
            const unsigned slot = slot_count % NS, phase = (slot_count / NS) & 1u;
            if (!mbar_wait_bounded(&full[slot], phase)) {
                ok = false;
                break;
            }
            body(w, int(slot));
            __syncwarp();
            if (c.lane == 0) mbar_arrive(&empty[slot]);
        }
    }
    c.ring += unsigned(c.mine);
    return ok;
}

__global__ void __launch_bounds__(PT, 1) k_jacobi_persistent(const __grid_constant__ PersistArgs A,
                                                             const __grid_constant__ TmaMaps maps) {
    extern __shared__ __align__(128) double smem[];
    __shared__ SolveState sst;
    __shared__ __align__(8) uint64_t full[NS];
    __shared__ __align__(8) uint64_t empty[NS];
    __shared__ double sdiag[64], srdiag[64];
    const GridDev& g = A.g;
    Ctx c;
    c.tid = threadIdx.x;
    c.lane = c.tid & 31;
    c.producer = c.tid >= CONSUMERS;
    c.tx = c.tid & 31;
    c.ty = (c.tid >> 5) & (TY - 1);
    c.tz = (c.tid >> 8) & (PZ - 1);
    c.nbx = (g.n[0] + TX - 1) / TX;
    c.nby = (g.n[1] + TY - 1) / TY;
    c.nbricks = c.nbx * c.nby * ((g.n[2] + PZC - 1) / PZC);
    c.mine = c.nbricks > int(blockIdx.x) ? (c.nbricks - int(blockIdx.x) + int(gridDim.x) - 1) / int(gridDim.x) : 0;
    c.bx0 = int(blockIdx.x) % c.nbx;
    c.by0 = (int(blockIdx.x) / c.nbx) % c.nby;
    c.bz0 = int(blockIdx.x) / (c.nbx * c.nby);
    c.sx = int(gridDim.x) % c.nbx;
    c.sy = (int(gridDim.x) / c.nbx) % c.nby;
    c.sz = int(gridDim.x) / (c.nbx * c.nby);
    c.ring = 0u;
    c.target = 0ull;
    c.set = 0;
    if (c.tid < 64) {
        sdiag[c.tid] = g.diag[c.tid];
        srdiag[c.tid] = g.rdiag[c.tid];
    }
    if (c.tid == 0) {
        sst = *A.st;
        // every barrier of earlier launches was passed by the whole grid, so
        // the count is a multiple of the grid size plus arrivals at this
        // launch's first barrier (fewer than the grid: this block has not)
        c.target = ld_acquire_gpu(&A.bar->count) / gridDim.x * gridDim.x;
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CONSUMER_WARPS);
        }
        fence_mbar_init();
    }
    __syncthreads();
    rb200_trace* trace = blockIdx.x == 0 ? A.trace : nullptr;
    const int plane = g.n[0] * g.n[1];
    const int qb = c.tz * QPT;
    bool ok = true;
    int iters = 0;
    for (;;) {
        const int flags = sst.flags;
        if (flags & F_DONE) break;
        if (flags & F_NEED_TRUE) {
            // ---------------------------------------------- phase 3: true residual
            double* spare = sst.dsel ? A.d0 : A.d1;
            Neu2 acc;
            double gauge_sq = 0.0;  // t[0]^2 in the thread that holds cell 0
            double mx = 0.0;
            const bool mine_ok = run_bricks(
                c, full, empty,
                [&](const BrickWalk& w, int s) {
                    const int x0 = w.x0(), y0 = w.y0(), k0 = w.k0();
                    mbar_expect_tx(&full[s], PS::BYTES);
                    tma_load_slab(smem + s * STAGE, &maps.p, x0 - 2, y0 - 1, k0 - 1, &full[s]);
                },
                [&](const BrickWalk& w, int s) {
                    const double* sp = smem + s * STAGE;
                    const Col col = column(g, c, w, qb);
                    if (!col.own) return;
                    double v[QPT + 2];
#pragma unroll
                    for (int u = 0; u < QPT + 2; ++u) v[u] = sp[col.e0 + (u - 1) * PS::PLANE];
#pragma unroll
                    for (int u = 0; u < QPT; ++u) {
                        if (qb + u >= col.kend) break;
                        const int e = col.e0 + u * PS::PLANE;
                        const int cc = col.cc0 + u * plane;
                        const double kp = row7(g, col.mxy, col.k0 + qb + u, v[u + 1], sp[e - 1], sp[e + 1],
                                               sp[e - PS::SX], sp[e + PS::SX], v[u], v[u + 2]);
                        const double t = __ldcg(A.b + cc) - kp;
                        spare[cc] = t;
                        (u & 1 ? acc.b : acc.a).add(t * t);
                        if (cc == 0) gauge_sq = t * t;
                        mx = fmax(mx, fabs(t));
                    }
                });
            // |t|^2 and |t[1..]|^2 (the restart test of a seeded solve)
            dd sums[2] = {acc.as_dd(), dd_add1(acc.as_dd(), -gauge_sq)};
            double maxs[1] = {mx};
            if (!(ok = reduce_grid<2, 1>(c, A, mine_ok, sums, maxs))) break;
            if (c.tid == 0)
                decide_true(&sst, trace, dd_value(sums[0]), dd_value(sums[1]), maxs[0], flags, g.volume);
            __syncthreads();
            continue;
        }
        if (flags & F_NEED_REPLACE) {
            // ---------------------------------------------- phase 4: restart
            const double* spare = sst.dsel ? A.d0 : A.d1;
            Neu2 acc;
            if (!c.producer) {
                for (BrickWalk w(c); w.b < c.nbricks; w.next(c)) {
                    const Col col = column(g, c, w, qb);
                    if (!col.own) continue;
#pragma unroll
                    for (int u = 0; u < QPT; ++u) {
                        if (qb + u >= col.kend) break;
                        const int cc = col.cc0 + u * plane;
                        const double rc = cc == 0 ? 0.0 : __ldcg(spare + cc);
                        A.r[cc] = rc;
                        if (cc == 0) {
                            A.z[0] = 0.0;
                            continue;
                        }
                        const int m = col.mxy | zmask(g, col.k0 + qb + u);
                        const double zc = div_diag(rc, sdiag[m], srdiag[m]);
                        A.z[cc] = zc;
                        (u & 1 ? acc.b : acc.a).add(rc * zc);
                    }
                }
            }
            dd sums[1] = {acc.as_dd()};
            double none[1] = {0.0};
            if (!(ok = reduce_grid<1, 0>(c, A, true, sums, none))) break;
            if (c.tid == 0) decide_rz(&sst, trace, dd_value(sums[0]), MODE_REPLACE);
            __syncthreads();
            continue;
        }
        if (flags & F_STOP) break;  // stopped without a pending check: nothing to do
        if (iters >= A.budget) break;

        // -------------------------------------------------- phase 1: direction + K d
        {
            const bool fresh = (flags & F_REPLACED) != 0;
            const double beta = sst.beta;
            const int dsel = sst.dsel;
            double* __restrict__ dst = dsel ? A.d0 : A.d1;
            const CUtensorMap* dmap = dsel ? &maps.d1 : &maps.d0;
            Neu2 acc;
            const bool mine_ok = run_bricks(
                c, full, empty,
                [&](const BrickWalk& w, int s) {
                    const int x0 = w.x0(), y0 = w.y0(), k0 = w.k0();
                    double* sz = smem + s * STAGE;
                    mbar_expect_tx(&full[s], (fresh ? 1u : 2u) * PS::BYTES);
                    tma_load_slab(sz, &maps.z, x0 - 2, y0 - 1, k0 - 1, &full[s]);
                    if (!fresh) tma_load_slab(sz + PS::SIZE, dmap, x0 - 2, y0 - 1, k0 - 1, &full[s]);
                },
                [&](const BrickWalk& w, int s) {
                    const double* sz = smem + s * STAGE;
                    const double* sd = sz + PS::SIZE;
                    const Col col = column(g, c, w, qb);
                    if (!col.own) return;
                    // straight-line cells (no per-cell branch) so that the
                    // column's cells interleave. FRESH: d = z (after a
                    // restart); FULL: the brick is whole in z; ZIN: it lies
                    // strictly inside the box in z (no gauge cell, both z
                    // neighbours everywhere).
                    auto cells = [&](auto fresh_t, auto full_t, auto zin_t) {
                        constexpr bool FRESH = decltype(fresh_t)::value;
                        constexpr bool FULL = decltype(full_t)::value;
                        constexpr bool ZIN = decltype(zin_t)::value;
                        // the new direction at slab element e (src/pressure.rs:720-731)
                        auto dn = [&](int e) { return FRESH ? sz[e] : sz[e] + beta * sd[e]; };
                        double v[QPT + 2];
#pragma unroll
                        for (int u = 0; u < QPT + 2; ++u) v[u] = dn(col.e0 + (u - 1) * PS::PLANE);
#pragma unroll
                        for (int u = 0; u < QPT; ++u) {
                            if (!FULL && qb + u >= col.kend) break;
                            const int e = col.e0 + u * PS::PLANE;
                            const int cc = col.cc0 + u * plane;
                            const double kd = row7<ZIN>(g, col.mxy, col.k0 + qb + u, v[u + 1], dn(e - 1), dn(e + 1),
                                                        dn(e - PS::SX), dn(e + PS::SX), v[u], v[u + 2]);
                            const double qv = (!ZIN && cc == 0) ? 0.0 : kd;  // gauge row
                            dst[cc] = v[u + 1];
                            (u & 1 ? acc.b : acc.a).add(v[u + 1] * qv);
                        }
                    };
                    using T = std::true_type;
                    using F = std::false_type;
                    const bool zin = col.k0 > 0 && col.k0 + PZC < g.n[2];
                    if (fresh) {
                        if (zin)
                            cells(T{}, T{}, T{});
                        else if (col.kend == PZC)
                            cells(T{}, T{}, F{});
                        else
                            cells(T{}, F{}, F{});
                    } else {
                        if (zin)
                            cells(F{}, T{}, T{});
                        else if (col.kend == PZC)
                            cells(F{}, T{}, F{});
                        else
                            cells(F{}, F{}, F{});
                    }
                });
            dd sums[1] = {acc.as_dd()};
            double none[1] = {0.0};
            if (!(ok = reduce_grid<1, 0>(c, A, mine_ok, sums, none))) break;
            if (c.tid == 0) decide_pass1(&sst, trace, dd_value(sums[0]), flags, dsel);
            __syncthreads();
            if (sst.flags & F_DONE) continue;
        }
        // -------------------------------------------------- phase 2: update + Jacobi
        {
            const int flags2 = sst.flags;
            const double alpha = sst.alpha;
            const int dsel = sst.dsel;
            const CUtensorMap* dmap = dsel ? &maps.d1 : &maps.d0;
            Neu2 acc_rr, acc_rz;
            const bool mine_ok = run_bricks(
                c, full, empty,
                [&](const BrickWalk& w, int s) {
                    const int x0 = w.x0(), y0 = w.y0(), k0 = w.k0();
                    double* sd = smem + s * STAGE;
                    mbar_expect_tx(&full[s], PS::BYTES + 2u * BOX_BYTES);
                    tma_load_slab(sd, dmap, x0 - 2, y0 - 1, k0 - 1, &full[s]);
                    tma_load_slab(sd + PS::SIZE, &maps.p_box, x0, y0, k0, &full[s]);
                    tma_load_slab(sd + PS::SIZE + BOX, &maps.r_box, x0, y0, k0, &full[s]);
                },
                [&](const BrickWalk& w, int s) {
                    const double* sd = smem + s * STAGE;
                    const double* sp = sd + PS::SIZE;
                    const double* sr = sp + BOX;
                    const Col col = column(g, c, w, qb);
                    if (!col.own) return;
                    // straight-line cells; the rare quotient outside the
                    // fast division's range is redone after the column.
                    // Gauge row: p[0] + alpha d[0] = p[0] (d[0] = 0), and
                    // r[0] = z[0] = 0 add nothing to the sums.
                    auto cells = [&](auto full_t, auto zin_t) {
                        constexpr bool FULL = decltype(full_t)::value;
                        constexpr bool ZIN = decltype(zin_t)::value;
                        double v[QPT + 2];
                        unsigned slow = 0u;  // cells whose quotient is redone
                        // ZIN: one diagonal for the whole column
                        const int mz = col.mxy | 0x30;
                        const double Dz = sdiag[mz], yz = srdiag[mz];
#pragma unroll
                        for (int u = 0; u < QPT + 2; ++u) v[u] = sd[col.e0 + (u - 1) * PS::PLANE];
#pragma unroll
                        for (int u = 0; u < QPT; ++u) {
                            if (!FULL && qb + u >= col.kend) break;
                            const int cc = col.cc0 + u * plane;
                            const int e = col.e0 + u * PS::PLANE;
                            const int k = col.k0 + qb + u;
                            const double qv = row7<ZIN>(g, col.mxy, k, v[u + 1], sd[e - 1], sd[e + 1],
                                                        sd[e - PS::SX], sd[e + PS::SX], v[u], v[u + 2]);
                            const int bi = col.bi0 + u * (TX * TY);
                            A.p[cc] = sp[bi] + alpha * v[u + 1];
                            const double rc = (!ZIN && cc == 0) ? 0.0 : sr[bi] - alpha * qv;
                            A.r[cc] = rc;
                            (u & 1 ? acc_rr.b : acc_rr.a).add(rc * rc);
                            const int m = ZIN ? mz : (col.mxy | zmask(g, k));
                            const double y = ZIN ? yz : srdiag[m];
                            const double zc = div_diag_fast(rc, ZIN ? Dz : sdiag[m], y);
                            const bool fast = ZIN ? div_diag_range_ok(rc) : div_diag_fast_ok(rc, y);
                            slow |= fast ? 0u : 1u << u;
                            A.z[cc] = zc;
                            (u & 1 ? acc_rz.b : acc_rz.a).add(fast ? rc * zc : 0.0);
                        }
                        if (ZIN && yz == 0.0) slow = (1u << QPT) - 1u;
                        if (slow) {
                            // r / D by division; the residual is re-read
                            // from this thread's own store above
#pragma unroll
                            for (int u = 0; u < QPT; ++u) {
                                if (!FULL && qb + u >= col.kend) break;
                                if (!((slow >> u) & 1u)) continue;
                                const int cc = col.cc0 + u * plane;
                                const double rc = A.r[cc];
                                const double zc = rc / sdiag[col.mxy | zmask(g, col.k0 + qb + u)];
                                A.z[cc] = zc;
                                (u & 1 ? acc_rz.b : acc_rz.a).add(rc * zc);
                            }
                        }
                    };
                    using T = std::true_type;
                    using F = std::false_type;
                    if (col.k0 > 0 && col.k0 + PZC < g.n[2])
                        cells(T{}, T{});
                    else if (col.kend == PZC)
                        cells(T{}, F{});
                    else
                        cells(F{}, F{});
                });
            dd sums[2] = {acc_rr.as_dd(), acc_rz.as_dd()};
            double none[1] = {0.0};
            if (!(ok = reduce_grid<2, 0>(c, A, mine_ok, sums, none))) break;
            if (c.tid == 0) decide_pass2(&sst, trace, dd_value(sums[0]), dd_value(sums[1]), flags2, true);
            __syncthreads();
            ++iters;
        }
    }
    if (!ok) {
        if (c.tid == 0) {
            atomicExch(&A.bar->abort, 1u);
            A.st->status = RB200_EXECUTION;
            A.st->flags = A.st->flags | F_DONE | F_STOP;
        }
        return;
    }
    if (blockIdx.x == 0 && c.tid == 0) *A.st = sst;
}

}  // namespace

// ------------------------------------------------------------ host side
int persistent_setup(const GridDev& g, int* blocks) {
    *blocks = 0;
    RB200_CUDA(cudaFuncSetAttribute(k_jacobi_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(kPersistSmem)));
    int dev = 0, sms = 0, coop = 0, per_sm = 0;
    RB200_CUDA(cudaGetDevice(&dev));
    RB200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RB200_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    RB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi_persistent, PT, kPersistSmem));
    if (!coop || per_sm < 1) return RB200_OK;
    const int nbricks = ((g.n[0] + TX - 1) / TX) * ((g.n[1] + TY - 1) / TY) * ((g.n[2] + PZC - 1) / PZC);
    int cap = sms * per_sm;
    if (cap > kMaxPersistBlocks) cap = kMaxPersistBlocks;
    *blocks = nbricks < cap ? nbricks : cap;
    return RB200_OK;
}

size_t persistent_partial_doubles(int blocks) { return 2 * size_t(blocks) * PSTRIDE; }

cudaError_t launch_persistent(const GridDev& g, SolveState* st, const double* b, double* p, double* r, double* z,
                              double* d0, double* d1, double* part, GridBarrier* bar, rb200_trace* trace,
                              const TmaMaps& maps, int blocks, int budget, cudaStream_t s) {
    PersistArgs A{g, st, b, p, r, z, d0, d1, part, bar, trace, budget};
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(blocks), 1, 1);
    cfg.blockDim = dim3(PT, 1, 1);
    cfg.dynamicSmemBytes = kPersistSmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_jacobi_persistent, A, maps);
}

}  // namespace rb200
