// Persistent PCG: one cooperative kernel runs a whole chunk of iterations of
// PressureWorkspace::solve_loaded (src/pressure.rs:577-740) with the
// "jacobi-pcg-v1" preconditioner (:534-575), or with the red-black SGS
// preconditioner of the RBSGS method, true-residual checks and restarts
// included, without returning to the host or the graph between passes.
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
// With red-black SGS, phase 2 stores only the red y = r/D and no r.z, and two
// more phases follow it (and the restart), each after a grid barrier:
//   B  z_b = (r_b + sum w y_nb) / D_b                              read z, r; write z (black)  ~20
//   R  z_r = y_r + (sum w z_nb) / D_r, r.z                         read z, r; write z (red)    ~20
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
    int par;        // (i + j) & 1: cell k of the column is red when (par + k) is even
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
    col.par = (i + j) & 1;
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
            // Wait (bounded) until the copies of the last ring's worth of
            // issued slots have landed: when a consumer gave up early nobody
            // waits on them, and the block must not move on or exit with a
            // bulk copy into its shared memory still in flight. On the normal
            // path the consumers have waited on them already, or soon will.
            const unsigned issued = slot_count - c.ring;
            for (unsigned k = issued > unsigned(NS) ? issued - unsigned(NS) : 0u; k < issued; ++k) {
                const unsigned sc = c.ring + k;
                if (!mbar_wait_bounded(&full[sc % NS], (sc / NS) & 1u)) ok = false;
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

// Neighbour sum of the red-black SGS passes: init + w * z over the existing
// neighbours, in the order X lower, X upper, Y lower, Y upper, Z lower, Z upper
// (the order of k_rbsgs_black / k_rbsgs_red_dot), from the z slab.
__device__ __forceinline__ double rb_sum(const GridDev& g, const double* sz, int e, int m, double init) {
    double y = init;
    if (m & 1) y += g.weight[0] * sz[e - 1];
    if (m & 2) y += g.weight[0] * sz[e + 1];
    if (m & 4) y += g.weight[1] * sz[e - PS::SX];
    if (m & 8) y += g.weight[1] * sz[e + PS::SX];
    if (m & 16) y += g.weight[2] * sz[e - PS::PLANE];
    if (m & 32) y += g.weight[2] * sz[e + PS::PLANE];
    return y;
}

// Red-black SGS after r and the red y = r/D are stored: a barrier (unless the
// caller's reduction just was one), the black pass z_b = (r_b + sum w y_nb)/D_b,
// a barrier, the red pass z_r = y_r + (sum w z_nb)/D_r with r.z, and its
// decision (`mode`). Every block runs it, so the barrier sequence stays the
// same everywhere.
__device__ __forceinline__ bool rb_apply(Ctx& c, const PersistArgs& A, const TmaMaps& maps, uint64_t* full,
                                         uint64_t* empty, double* smem, const double* sdiag, const double* srdiag,
                                         SolveState& sst, rb200_trace* trace, int qb, int mode, bool barrier_first) {
    const GridDev& g = A.g;
    const int plane = g.n[0] * g.n[1];
    auto issue = [&](const BrickWalk& w, int s) {
        const int x0 = w.x0(), y0 = w.y0(), k0 = w.k0();
        double* sz = smem + s * STAGE;
        mbar_expect_tx(&full[s], PS::BYTES + BOX_BYTES);
        tma_load_slab(sz, &maps.z, x0 - 2, y0 - 1, k0 - 1, &full[s]);
        tma_load_slab(sz + PS::SIZE, &maps.r_box, x0, y0, k0, &full[s]);
    };
    double none_m[1] = {0.0};
    // the red y of every block (after the update phase its own reduction was that barrier)
    if (barrier_first && !grid_barrier(c, A.bar)) return false;
    bool mine_ok = run_bricks(c, full, empty, issue, [&](const BrickWalk& w, int s) {
        const double* sz = smem + s * STAGE;
        const double* sr = sz + PS::SIZE;
        const Col col = column(g, c, w, qb);
        if (!col.own) return;
#pragma unroll
        for (int u = 0; u < QPT; ++u) {
            if (qb + u >= col.kend) break;
            const int k = col.k0 + qb + u;
            if (((col.par + k) & 1) == 0) continue;  // red
            const int m = col.mxy | zmask(g, k);
            const int e = col.e0 + u * PS::PLANE;
            A.z[col.cc0 + u * plane] =
                div_diag(rb_sum(g, sz, e, m, sr[col.bi0 + u * (TX * TY)]), sdiag[m], srdiag[m]);
        }
    });
    if (!__syncthreads_and(mine_ok) || !grid_barrier(c, A.bar)) return false;  // every black z
    Neu2 acc;
    mine_ok = run_bricks(c, full, empty, issue, [&](const BrickWalk& w, int s) {
        const double* sz = smem + s * STAGE;
        const double* sr = sz + PS::SIZE;
        const Col col = column(g, c, w, qb);
        if (!col.own) return;
#pragma unroll
        for (int u = 0; u < QPT; ++u) {
            if (qb + u >= col.kend) break;
            const int k = col.k0 + qb + u;
            const int cc = col.cc0 + u * plane;
            if (cc == 0) continue;  // z[0] = 0 is kept
            const int e = col.e0 + u * PS::PLANE;
            double zc = sz[e];
            if (((col.par + k) & 1) == 0) {
                const int m = col.mxy | zmask(g, k);
                zc = zc + div_diag(rb_sum(g, sz, e, m, 0.0), sdiag[m], srdiag[m]);
                A.z[cc] = zc;
            }
            (u & 1 ? acc.b : acc.a).add(sr[col.bi0 + u * (TX * TY)] * zc);
        }
    });
    dd sums[1] = {acc.as_dd()};
    if (!reduce_grid<1, 0>(c, A, mine_ok, sums, none_m)) return false;
    if (c.tid == 0) decide_rz(&sst, trace, dd_value(sums[0]), mode);
    __syncthreads();
    return true;
}

#define RB_PERSIST_PRE 0
#define RB_PERSIST_KERNEL k_jacobi_persistent
#include "persist_kernel.inc"
#undef RB_PERSIST_KERNEL
#undef RB_PERSIST_PRE
#define RB_PERSIST_PRE 1
#define RB_PERSIST_KERNEL k_rbsgs_persistent
#include "persist_kernel.inc"
#undef RB_PERSIST_KERNEL
#undef RB_PERSIST_PRE

}  // namespace

// ------------------------------------------------------------ host side
int persistent_setup(const GridDev& g, int* blocks) {
    *blocks = 0;
    RB200_CUDA(cudaFuncSetAttribute(k_jacobi_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(kPersistSmem)));
    RB200_CUDA(cudaFuncSetAttribute(k_rbsgs_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(kPersistSmem)));
    int dev = 0, sms = 0, coop = 0, per_sm = 0, per_sm_rb = 0;
    RB200_CUDA(cudaGetDevice(&dev));
    RB200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RB200_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    RB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi_persistent, PT, kPersistSmem));
    RB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_rb, k_rbsgs_persistent, PT, kPersistSmem));
    if (per_sm_rb < per_sm) per_sm = per_sm_rb;
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
                              const TmaMaps& maps, int blocks, int budget, cudaStream_t s, int pre) {
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
    return pre == 1 ? cudaLaunchKernelEx(&cfg, k_rbsgs_persistent, A, maps)
                    : cudaLaunchKernelEx(&cfg, k_jacobi_persistent, A, maps);
}

}  // namespace rb200
