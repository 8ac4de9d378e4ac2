// Device-driven gauge-eliminated PCG (PressureWorkspace::solve_loaded,
// src/pressure.rs:577-740) on the sealed-box operator.
//
// One PCG iteration of the Jacobi method is two slab passes:
//   pass 1  d <- z + beta*d, q = K d, curvature = d.q           (24N bytes)
//   pass 2  q = K d re-applied from d, p += alpha*d, r -= alpha*q,
//           z = r/D stored, r.r and r.z                         (48N bytes)
// instead of the four array passes of the reference (88N); q is never stored. Scalars never leave
// the device: the last block of each pass takes solve_loaded's decision
// (alpha, beta, breakdown, candidate, restart) and writes it to SolveState.
// The true-residual check and the restart run as flag-gated kernels at the end
// of each captured chunk of iterations, so the host only launches graphs and
// polls one word per chunk.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "pcg.hpp"
#include "pcg_device.cuh"
#include "slab.cuh"
#include "solve_state.cuh"
#include "stencil.cuh"

namespace rb200 {

constexpr int EW = 256;
constexpr int EW_CAP = 148 * 8;

// ------------------------------------------------------------------ init
__global__ void __launch_bounds__(EW) k_init_sums(GridDev g, SolveState* st, const double* __restrict__ b,
                                                  double* __restrict__ p, Partials part) {
    init_sums_body(g, st, b, p, part, whole_launch());
}

template <int KIND>
__global__ void __launch_bounds__(EW) k_load_residual(GridDev g, SolveState* st, const double* b,
                                                      double* d0, double* d1, double* __restrict__ r,
                                                      double* __restrict__ z, int mode, Partials part,
                                                      rb200_trace* trace) {
    load_residual_body<KIND>(g, st, b, d0, d1, r, z, mode, part, trace, whole_launch());
}

// precondition_jacobi (src/pressure.rs:534-575) as a primitive: z = r/D on
// every row but the eliminated gauge row (z[0] = 0), and r.z over rows >= 1.
__global__ void __launch_bounds__(EW) k_precondition_jacobi(GridDev g, const double* __restrict__ r,
                                                            double* __restrict__ z, Partials part,
                                                            double* __restrict__ rz_out) {
    __shared__ BlockReduce<1, 0> sm;
    Neu acc;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.cells; c += gridDim.x * blockDim.x) {
        if (c == 0) {
            z[0] = 0.0;
            continue;
        }
        int i, j, k;
        cell_coords(g, c, i, j, k);
        const int m = diag_mask(g, i, j, k);
        const double rc = r[c];
        const double zc = div_diag(rc, g.diag[m], g.rdiag[m]);
        z[c] = zc;
        acc.add(rc * zc);
    }
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(sm, sums, none);
    if (publish_and_check_last<1, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<1, 0>(part, gridDim.x, sm, sums, none);
        if (threadIdx.x == 0) *rz_out = dd_value(sums[0]);
    }
}

// ------------------------------------------------------------ slab staging
// Stage one or two slabs of the block's brick into shared memory.
template <int ZC>
__device__ __forceinline__ void stage_issue(const GridDev& g, const TmaMaps& maps, uint64_t* bar, double* sm0,
                                            const double* src0, const CUtensorMap* m0, double* sm1,
                                            const double* src1, const CUtensorMap* m1, int x0, int y0, int k0) {
    const int tid = threadIdx.x + TX * threadIdx.y;
    if (maps.use) {
        if (tid == 0) {
            mbar_init(bar, 1);
            fence_mbar_init();
        }
        __syncthreads();
        if (tid == 0) {
            mbar_expect_tx(bar, (sm1 ? 2u : 1u) * Slab<ZC>::BYTES);
            tma_load_slab(sm0, m0, x0 - 2, y0 - 1, k0 - 1, bar);
            if (sm1) tma_load_slab(sm1, m1, x0 - 2, y0 - 1, k0 - 1, bar);
        }
    } else {
        slab_issue_rows<ZC>(g, sm0, src0, x0, y0, k0);
        if (sm1) slab_issue_rows<ZC>(g, sm1, src1, x0, y0, k0);
        cp_async_commit();
    }
}

// Wait for the staged slabs. A TMA wait that runs out records an execution
// error in the solver state, waits once more for the copy in flight, and the
// whole block returns false (the decision is block-uniform).
__device__ __forceinline__ bool stage_wait(const TmaMaps& maps, uint64_t* bar, SolveState* st) {
    bool ok = true;
    if (maps.use)
        ok = mbar_wait_bounded(bar, 0);
    else
        cp_async_wait_all();
    ok = __syncthreads_and(ok) != 0;
    if (!ok) {
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            st->status = RB200_EXECUTION;
            st->flags = st->flags | F_DONE | F_STOP;
        }
        mbar_wait_bounded(bar, 0);
        __syncthreads();
    }
    return ok;
}

// ------------------------------------------------------------ pass 1
// Direction update fused with q = K d and the curvature d.q
// (src/pressure.rs:657-668, :720-731). The slabs hold z and the old direction;
// the new direction d = z (restart) or z + beta*d is formed in shared memory
// for the whole slab (out-of-domain and gauge entries are 0 in both inputs, so
// they stay 0), then each cell's row of K d is applied.
template <int ZC>
__global__ void __launch_bounds__(TILE_THREADS) k_pass1(GridDev g, SolveState* st, const double* __restrict__ zarr,
                                                        double* d0, double* d1, double* __restrict__ qout,
                                                        const __grid_constant__ TmaMaps maps, Partials part,
                                                        rb200_trace* trace) {
    using S = Slab<ZC>;
    extern __shared__ __align__(128) double smem[];
    __shared__ BlockReduce<1, 0> red;
    __shared__ __align__(8) uint64_t bar;
    double* sz = smem;
    double* sd = smem + S::SIZE;
    const int flags = st->flags;
    if (flags & F_STOP) return;
    const bool fresh = (flags & F_REPLACED) != 0;
    const double beta = st->beta;
    const int dsel = st->dsel;
    const double* __restrict__ src = dsel ? d1 : d0;
    double* __restrict__ dst = dsel ? d0 : d1;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, k0 = blockIdx.z * ZC;
    stage_issue<ZC>(g, maps, &bar, sz, zarr, &maps.z, fresh ? nullptr : sd, src, dsel ? &maps.d1 : &maps.d0, x0,
                    y0, k0);
    if (!stage_wait(maps, &bar, st)) return;
    const int tid = threadIdx.x + TX * threadIdx.y;
    if (!fresh)
        for (int e = tid; e < S::SIZE; e += TILE_THREADS) sz[e] = sz[e] + beta * sd[e];
    __syncthreads();
    Neu acc;
    const int i = x0 + threadIdx.x, j = y0 + threadIdx.y;
    if (i < g.n[0] && j < g.n[1]) {
        const int kend = min(ZC, g.n[2] - k0);
        int e = S::own(threadIdx.x, threadIdx.y, 0);
        int c = cell_idx(g, i, j, k0);
        const int plane = g.n[0] * g.n[1];
        for (int q = 0; q < kend; ++q, e += S::PLANE, c += plane) {
            Neigh v = slab_neigh<ZC>(sz, e);
            double qv = c == 0 ? 0.0 : apply_row(g, i, j, k0 + q, v);
            dst[c] = v.c;
            if (qout) qout[c] = qv;
            acc.add(v.c * qv);
        }
    }
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(red, sums, none);
    const int nb = nblocks3();
    if (publish_and_check_last<1, 0>(part, block_id3(), nb, sums, none)) {
        fold_partials<1, 0>(part, nb, red, sums, none);
        if (tid3() == 0) decide_pass1(st, trace, dd_value(sums[0]), flags, dsel);
    }
}

// ------------------------------------------------------------ pass 2
// p += alpha*d, r -= alpha*K d (src/pressure.rs:669-680) with K d re-applied
// from the direction slab, the recursive norm, and the preconditioner's local
// part: Jacobi z = r/D with r.z (precondition_jacobi, :534-575); red-black SGS
// stores y = r/D on the red cells.
// PRE: 0 Jacobi (z = r/D and r.z here), 1 red-black SGS (y = r/D on red
// cells), 2 none (lexicographic SGS forms z in its sweeps).
template <int ZC, int PRE>
__global__ void __launch_bounds__(TILE_THREADS) k_pass2(GridDev g, SolveState* st, double* __restrict__ p,
                                                        double* __restrict__ r, double* __restrict__ z,
                                                        const double* d0, const double* d1,
                                                        const __grid_constant__ TmaMaps maps, Partials part,
                                                        rb200_trace* trace) {
    using S = Slab<ZC>;
    extern __shared__ __align__(128) double smem[];
    __shared__ BlockReduce<2, 0> red;
    __shared__ __align__(8) uint64_t bar;
    const int flags = st->flags;
    if (flags & F_STOP) return;
    const double alpha = st->alpha;
    const int dsel = st->dsel;
    const double* __restrict__ d = dsel ? d1 : d0;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, k0 = blockIdx.z * ZC;
    stage_issue<ZC>(g, maps, &bar, smem, d, dsel ? &maps.d1 : &maps.d0, nullptr, nullptr, nullptr, x0, y0, k0);
    const int i = x0 + threadIdx.x, j = y0 + threadIdx.y;
    const bool own = i < g.n[0] && j < g.n[1];
    const int kend = own ? min(ZC, g.n[2] - k0) : 0;
    const int plane = g.n[0] * g.n[1];
    const int c0 = own ? cell_idx(g, i, j, k0) : 0;
    double pv[ZC], rv[ZC];
#pragma unroll
    for (int q = 0; q < ZC; ++q) {
        if (q < kend) {
            pv[q] = p[c0 + q * plane];
            rv[q] = r[c0 + q * plane];
        }
    }
    if (!stage_wait(maps, &bar, st)) return;
    Neu acc_rr, acc_rz;
#pragma unroll
    for (int q = 0; q < ZC; ++q) {
        if (q >= kend) break;
        const int c = c0 + q * plane;
        if (c == 0) continue;  // gauge row: p[0], r[0] stay 0
        Neigh v = slab_neigh<ZC>(smem, S::own(threadIdx.x, threadIdx.y, q));
        const int k = k0 + q;
        double qv = apply_row(g, i, j, k, v);
        p[c] = pv[q] + alpha * v.c;
        double rc = rv[q] - alpha * qv;
        r[c] = rc;
        acc_rr.add(rc * rc);
        if (PRE == 0) {
            const int m = diag_mask(g, i, j, k);
            double zc = div_diag(rc, g.diag[m], g.rdiag[m]);
            z[c] = zc;
            acc_rz.add(rc * zc);
        } else if (PRE == 1 && ((i + j + k) & 1) == 0) {
            z[c] = rc / diag_at(g, i, j, k);
        }
    }
    dd sums[2] = {acc_rr.as_dd(), acc_rz.as_dd()};
    double none[1];
    block_reduce<2, 0>(red, sums, none);
    const int nb = nblocks3();
    if (publish_and_check_last<2, 0>(part, block_id3(), nb, sums, none)) {
        fold_partials<2, 0>(part, nb, red, sums, none);
        if (tid3() == 0) decide_pass2(st, trace, dd_value(sums[0]), dd_value(sums[1]), flags, PRE == 0);
    }
}

// ------------------------------------------------------------ true residual
// true_report (src/pressure.rs:432-456): t = b - K p on every cell (the gauge
// row included), |t|_2, max|t|, max|t|*dt/V; then the acceptance and restart
// decisions of solve_loaded (:686-715). t is kept in the spare direction
// buffer for a restart.
template <int ZC>
__global__ void __launch_bounds__(TILE_THREADS) k_true_residual(GridDev g, SolveState* st, const double* __restrict__ b,
                                                                const double* __restrict__ p, double* d0, double* d1,
                                                                const __grid_constant__ TmaMaps maps, Partials part,
                                                                rb200_trace* trace) {
    using S = Slab<ZC>;
    extern __shared__ __align__(128) double smem[];
    __shared__ BlockReduce<2, 1> red;
    __shared__ __align__(8) uint64_t bar;
    const int flags = st->flags;
    if (!(flags & F_NEED_TRUE)) return;
    double* __restrict__ spare = st->dsel ? d0 : d1;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, k0 = blockIdx.z * ZC;
    stage_issue<ZC>(g, maps, &bar, smem, p, &maps.p, nullptr, nullptr, nullptr, x0, y0, k0);
    if (!stage_wait(maps, &bar, st)) return;
    Neu acc;
    double gauge_sq = 0.0;  // t[0]^2 when this thread holds cell 0
    double mx[1] = {0.0};
    const int i = x0 + threadIdx.x, j = y0 + threadIdx.y;
    if (i < g.n[0] && j < g.n[1]) {
        const int kend = min(ZC, g.n[2] - k0);
        const int plane = g.n[0] * g.n[1];
        int c = cell_idx(g, i, j, k0);
        int e = S::own(threadIdx.x, threadIdx.y, 0);
        for (int q = 0; q < kend; ++q, e += S::PLANE, c += plane) {
            Neigh v = slab_neigh<ZC>(smem, e);
            double t = b[c] - apply_row(g, i, j, k0 + q, v);
            spare[c] = t;
            acc.add(t * t);
            if (c == 0) gauge_sq = t * t;
            mx[0] = fmax(mx[0], fabs(t));
        }
    }
    // the second sum leaves out the gauge row: |t[1..]|^2
    dd sums[2] = {acc.as_dd(), dd_add1(acc.as_dd(), -gauge_sq)};
    block_reduce<2, 1>(red, sums, mx);
    const int nb = nblocks3();
    if (publish_and_check_last<2, 1>(part, block_id3(), nb, sums, mx)) {
        fold_partials<2, 1>(part, nb, red, sums, mx);
        if (tid3() == 0) decide_true(st, trace, dd_value(sums[0]), dd_value(sums[1]), mx[0], flags, g.volume);
    }
}

// ------------------------------------------------------------ multigrid outer passes
// Flexible CG around the FP32 multigrid preconditioner: q = K d is formed by
// pass 1 for d.q and recomputed from d where the update and the finish need it
// (no q vector); the finish pass converts the FP32 V-cycle output to z (FP64,
// z[0] = 0), reduces r.z and z.r_old and takes the decision with the
// Polak-Ribiere beta = (z.r - z.r_old) / (z_old.r_old) (tolerant of a
// preconditioner that is symmetric only up to FP32 rounding). The residual
// before the update stays available in a second buffer. This update serves
// grids whose finest level is solved inside the cluster kernel: r stays in the
// first buffer (the V-cycle's first half-sweep reads it there) and r_old is
// copied to the second.
__global__ void __launch_bounds__(EW) k_mg_update(GridDev g, SolveState* st, double* __restrict__ p,
                                                  double* __restrict__ r, double* __restrict__ r_old,
                                                  const double* d0, const double* d1, Partials part,
                                                  rb200_trace* trace) {
    __shared__ BlockReduce<1, 0> red;
    const int flags = st->flags;
    if (flags & F_STOP) return;
    const double alpha = st->alpha;
    const double* __restrict__ d = st->dsel ? d1 : d0;
    Neu acc;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.cells; c += gridDim.x * blockDim.x) {
        if (c == 0) {
            r_old[0] = 0.0;
            continue;
        }
        int i, j, k;
        cell_coords(g, c, i, j, k);
        p[c] = p[c] + alpha * d[c];
        const double ro = r[c];
        double rc = ro - alpha * kd_at(g, d, i, j, k, c);
        r_old[c] = ro;
        r[c] = rc;
        acc.add(rc * rc);
    }
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(red, sums, none);
    if (publish_and_check_last<1, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<1, 0>(part, gridDim.x, red, sums, none);
        if (threadIdx.x == 0) {
            if (flags & F_PROFILE) return;
            int it = st->it + 1;
            st->it = it;
            double recursive_l2 = sqrt(dd_value(sums[0]));
            st->recursive_l2 = recursive_l2;
            if (trace) trace[it - 1].recursive_l2 = recursive_l2;
            if (recursive_l2 <= st->threshold || it == st->max_it) st->flags = flags | F_CANDIDATE;
        }
    }
}

// ------------------------------------------------------------ lexicographic SGS
// precondition_sgs (src/pressure.rs:467-532): forward
//   y_i = (r_i + sum_{lower d} w_d y_{i-s_d}) / D_i    (d = X, Y, Z in order)
// then reverse
//   z_i = y_i + (sum_{upper d} w_d z_{i+s_d}) / D_i
// over rows 1..N-1 (row 0 is the eliminated gauge row, z_0 = 0). Each row
// depends only on its lower (upper) neighbours, so any order that respects
// those dependencies computes the reference's lexicographic sweep bit for bit
// (the reference's own tiled wavefront, src/sgs.rs:56-104, uses the same
// fact).
//
// One launch runs both sweeps over 8^3 tiles. A block takes the next slot of
// a queue (slots 0..T-1: the tiles in wave order tx + ty + tz ascending;
// T..2T-1: the same list backwards for the reverse sweep), waits until the
// tiles it depends on are done (forward: the lower x, y, z neighbour tiles;
// reverse: the upper ones, and for the last tile of the forward order its own
// forward sweep), stages its tile and the one-cell halo it reads in shared
// memory, walks the tile's hyperplanes lx + ly + lz = l with a block barrier
// between them, stores the tile and publishes its state word (release). A
// slot only waits for slots taken before it, by blocks that are running, so
// the queue cannot deadlock whatever the number of resident blocks. The
// reverse sweep of a tile starts after the forward sweep of every tile: its
// upper neighbours' reverse sweeps come after the forward sweep of the last
// tile, which comes after every other forward sweep.
//
// Every wait is bounded: a wait that runs out raises the abort word, which
// ends every other wait, and marks the solve as failed (execution error).
constexpr int SGS_T = 8;
constexpr int SGS_THREADS = SGS_T * SGS_T * SGS_T;
constexpr unsigned kSgsSpins = 1u << 22;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Wait until tile `dep` holds a state >= need; a wait that runs out raises
// the abort word.
__device__ __forceinline__ bool sgs_wait(unsigned* ctl, int dep, unsigned need) {
    unsigned n = 0;
    while (ld_acquire_u32(ctl + 2 + dep) < need) {
        ++n;
        if ((n & 7u) == 0u && *(volatile const unsigned*)(ctl + 1) != 0u) return false;
        if (n > kSgsSpins) {
            atomicExch(ctl + 1, 1u);
            return false;
        }
        if (n > 256u) __nanosleep(64);
    }
    return true;
}

__global__ void __launch_bounds__(SGS_THREADS) k_sgs_flow(GridDev g, SolveState* st,
                                                          const double* __restrict__ r, double* z, SgsFlow f,
                                                          int mode) {
    __shared__ double zs[SGS_T + 2][SGS_T + 2][SGS_T + 2];  // the tile at [1..8], its halo at 0 and 9
    __shared__ int s_slot, s_ok;
    if (!gate(st->flags, mode)) return;
    const int nt0 = (g.n[0] + SGS_T - 1) / SGS_T, nt1 = (g.n[1] + SGS_T - 1) / SGS_T,
              nt2 = (g.n[2] + SGS_T - 1) / SGS_T;
    const int lx = threadIdx.x % SGS_T, ly = (threadIdx.x / SGS_T) % SGS_T, lz = threadIdx.x / (SGS_T * SGS_T);
    const int mine = lx + ly + lz;
    const int sy = g.n[0], sz = g.n[0] * g.n[1];
    const int slots = 2 * f.ntiles;
    if (threadIdx.x == 0) s_slot = int(atomicAdd(f.ctl, 1u));
    __syncthreads();
    int slot = s_slot;
    while (slot < slots) {
        // the next slot is taken now, its atomic overlapping this tile
        unsigned next_slot = 0;
        if (threadIdx.x == 0) next_slot = atomicAdd(f.ctl, 1u);
        const bool reverse = slot >= f.ntiles;
        const int tile = f.order[reverse ? slots - 1 - slot : slot];
        const int tx = tile % nt0, ty = (tile / nt0) % nt1, tz = tile / (nt0 * nt1);
        const int i = tx * SGS_T + lx, j = ty * SGS_T + ly, k = tz * SGS_T + lz;
        const bool in = i < g.n[0] && j < g.n[1] && k < g.n[2];
        const int c = in ? cell_idx(g, i, j, k) : 0;
        double rv = 0.0, D = 1.0, y = 0.0;
        if (in) {
            const int m = diag_mask(g, i, j, k);
            D = g.diag[m];
            y = g.rdiag[m];
            if (!reverse) rv = r[c];
        }
        if (threadIdx.x < 32) {
            // lanes 0, 1, 2 wait on the x, y, z neighbour tile at once
            const int lane = threadIdx.x;
            int dep = -1;
            unsigned need = 1u;
            if (lane < 3) {
                const int t = lane == 0 ? tx : (lane == 1 ? ty : tz);
                const int n = lane == 0 ? nt0 : (lane == 1 ? nt1 : nt2);
                const int stride = lane == 0 ? 1 : (lane == 1 ? nt0 : nt0 * nt1);
                if (!reverse) {
                    if (t > 0) dep = tile - stride;
                } else if (tx + 1 == nt0 && ty + 1 == nt1 && tz + 1 == nt2) {
                    if (lane == 0) dep = tile;  // the last tile of the forward order: its own forward sweep
                } else if (t + 1 < n) {
                    dep = tile + stride;
                    need = 2u;
                }
            }
            const bool ok = __all_sync(0xffffffffu, dep < 0 || sgs_wait(f.ctl, dep, need));
            if (lane == 0) s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) {
            if (threadIdx.x == 0) {
                atomicExch(f.ctl + 1, 1u);
                st->status = RB200_EXECUTION;
                st->flags = (st->flags | F_DONE | F_STOP) & ~F_NEED_REPLACE;
            }
            return;
        }
        double* const me = &zs[lz + 1][ly + 1][lx + 1];
        if (!reverse) {
            if (in) {
                if (c == 0) *me = __ldcg(z);  // the gauge row keeps its value
                if (lx == 0 && i > 0) zs[lz + 1][ly + 1][0] = __ldcg(z + c - 1);
                if (ly == 0 && j > 0) zs[lz + 1][0][lx + 1] = __ldcg(z + c - sy);
                if (lz == 0 && k > 0) zs[0][ly + 1][lx + 1] = __ldcg(z + c - sz);
            }
            __syncthreads();
            for (int l = 0; l < 3 * SGS_T - 2; ++l) {
                if (in && mine == l && c != 0) {
                    double value = rv;
                    if (i > 0) value += g.weight[0] * zs[lz + 1][ly + 1][lx];
                    if (j > 0) value += g.weight[1] * zs[lz + 1][ly][lx + 1];
                    if (k > 0) value += g.weight[2] * zs[lz][ly + 1][lx + 1];
                    *me = div_diag(value, D, y);
                }
                __syncthreads();
            }
        } else {
            if (in) {
                *me = __ldcg(z + c);
                if (lx == SGS_T - 1 && i + 1 < g.n[0]) zs[lz + 1][ly + 1][SGS_T + 1] = __ldcg(z + c + 1);
                if (ly == SGS_T - 1 && j + 1 < g.n[1]) zs[lz + 1][SGS_T + 1][lx + 1] = __ldcg(z + c + sy);
                if (lz == SGS_T - 1 && k + 1 < g.n[2]) zs[SGS_T + 1][ly + 1][lx + 1] = __ldcg(z + c + sz);
            }
            __syncthreads();
            for (int l = 3 * SGS_T - 3; l >= 0; --l) {
                if (in && mine == l && c != 0) {
                    double correction = 0.0;
                    if (i + 1 < g.n[0]) correction += g.weight[0] * zs[lz + 1][ly + 1][lx + 2];
                    if (j + 1 < g.n[1]) correction += g.weight[1] * zs[lz + 1][ly + 2][lx + 1];
                    if (k + 1 < g.n[2]) correction += g.weight[2] * zs[lz + 2][ly + 1][lx + 1];
                    *me = *me + div_diag(correction, D, y);
                }
                __syncthreads();
            }
        }
        if (in && c != 0) __stcg(z + c, *me);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            st_release_u32(f.ctl + 2 + tile, reverse ? 2u : 1u);
            s_slot = int(next_slot);
        }
        __syncthreads();
        slot = s_slot;
    }
}

// r.z after a lexicographic SGS application, then the preconditioner decision.
__global__ void __launch_bounds__(EW) k_sgs_dot(GridDev g, SolveState* st, const double* __restrict__ r,
                                                const double* __restrict__ z, int mode, Partials part,
                                                rb200_trace* trace, unsigned* sgs_ctl, int sgs_words) {
    __shared__ BlockReduce<1, 0> sm;
    // the sweep kernel before this one has ended: its queue starts over
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < sgs_words; t += gridDim.x * blockDim.x) sgs_ctl[t] = 0u;
    if (!gate(st->flags, mode)) return;
    Neu acc;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.cells; c += gridDim.x * blockDim.x)
        if (c != 0) acc.add(r[c] * z[c]);
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(sm, sums, none);
    if (publish_and_check_last<1, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<1, 0>(part, gridDim.x, sm, sums, none);
        if (threadIdx.x == 0) decide_rz(st, trace, dd_value(sums[0]), mode);
    }
}

// ------------------------------------------------------------ red-black SGS
// Symmetric Gauss-Seidel preconditioner in red-black order on the
// gauge-eliminated system (cell 0, red, is removed): forward reds then blacks,
// backward blacks then reds. With reds first, the forward red solve and the
// backward black solve are diagonal, so M^-1 r is
//   red:    y_r = r_r/D_r                     (stored by the pass that forms r)
//   black:  z_b = (r_b + sum_nb w * y_nb) / D_b
//   red:    z_r = y_r + (sum_nb w * z_nb) / D_r
// A symmetric M, as PCG needs; new (the reference sweeps lexicographically).
__device__ __forceinline__ bool is_black(int i, int j, int k) { return ((i + j + k) & 1) != 0; }

// Work mapping of the two passes: thread t takes cell pair m = t mod half of
// row t / half (row = j + n1 k), i.e. cells 2m and 2m + 1 of the row, one of
// each colour (half = ceil(n0 / 2); 2m + 1 may be n0 on an odd row length).
struct PairMap {
    int half, pairs;
    FastDiv by_half, by_n1;
};

static PairMap pair_map(const GridDev& g) {
    PairMap p;
    p.half = (g.n[0] + 1) / 2;
    p.pairs = p.half * g.n[1] * g.n[2];
    p.by_half = make_fastdiv(unsigned(p.half));
    p.by_n1 = make_fastdiv(unsigned(g.n[1]));
    return p;
}

// Neighbour sum of cell (i, j, k), x-, x+, y-, y+, z-, z+ (one order for both colours).
__device__ __forceinline__ double rb_neighbours(const GridDev& g, const double* __restrict__ z, int c, int i, int j,
                                                int k, double init) {
    double y = init;
    if (i > 0) y += g.weight[0] * z[c - 1];
    if (i + 1 < g.n[0]) y += g.weight[0] * z[c + 1];
    if (j > 0) y += g.weight[1] * z[c - g.n[0]];
    if (j + 1 < g.n[1]) y += g.weight[1] * z[c + g.n[0]];
    const int sz = g.n[0] * g.n[1];
    if (k > 0) y += g.weight[2] * z[c - sz];
    if (k + 1 < g.n[2]) y += g.weight[2] * z[c + sz];
    return y;
}

__global__ void __launch_bounds__(EW) k_rbsgs_black(GridDev g, PairMap pm, SolveState* st,
                                                    const double* __restrict__ r, double* __restrict__ z, int mode) {
    if (!gate(st->flags, mode)) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < pm.pairs; t += gridDim.x * blockDim.x) {
        const int row = fast_div(t, pm.by_half);
        const int m = t - row * pm.half;
        const int k = fast_div(row, pm.by_n1);
        const int j = row - k * g.n[1];
        const int i = 2 * m + ((j + k + 1) & 1);  // the black cell of the pair
        if (i >= g.n[0]) continue;
        const int c = i + g.n[0] * row;
        const int mask = diag_mask(g, i, j, k);
        z[c] = div_diag(rb_neighbours(g, z, c, i, j, k, r[c]), g.diag[mask], g.rdiag[mask]);
    }
}

__global__ void __launch_bounds__(EW) k_rbsgs_red_dot(GridDev g, PairMap pm, SolveState* st,
                                                      const double* __restrict__ r, double* __restrict__ z, int mode,
                                                      Partials part, rb200_trace* trace) {
    __shared__ BlockReduce<1, 0> sm;
    if (!gate(st->flags, mode)) return;
    Neu acc;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < pm.pairs; t += gridDim.x * blockDim.x) {
        const int row = fast_div(t, pm.by_half);
        const int m = t - row * pm.half;
        const int k = fast_div(row, pm.by_n1);
        const int j = row - k * g.n[1];
        const int ired = 2 * m + ((j + k) & 1), iblk = 2 * m + ((j + k + 1) & 1);
        const int cred = ired + g.n[0] * row, cblk = iblk + g.n[0] * row;
        if (ired < g.n[0] && cred != 0) {  // z[0] = 0 is kept by k_load_residual
            const int mask = diag_mask(g, ired, j, k);
            const double corr = rb_neighbours(g, z, cred, ired, j, k, 0.0);
            const double zc = z[cred] + div_diag(corr, g.diag[mask], g.rdiag[mask]);
            z[cred] = zc;
            acc.add(r[cred] * zc);
        }
        if (iblk < g.n[0] && cblk != 0) acc.add(r[cblk] * z[cblk]);
    }
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(sm, sums, none);
    if (publish_and_check_last<1, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<1, 0>(part, gridDim.x, sm, sums, none);
        if (threadIdx.x == 0) decide_rz(st, trace, dd_value(sums[0]), mode);
    }
}

// ------------------------------------------------------------ graph embedding
// Device-side reset of the solver state (what solve() uploads from the host).
// The seeded start of the resident carrier: p = the accepted previous
// pressure when `warm` is set.
__global__ void __launch_bounds__(EW) k_seed_pressure(int n, double* __restrict__ p, const double* __restrict__ seed,
                                                      const int* __restrict__ warm) {
    if (!*warm) return;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) p[c] = seed[c];
}

__global__ void k_solve_reset(SolveState* st, rb200_settings s, const double* __restrict__ dt_dev,
                              const int* __restrict__ skip, int flexible, const int* __restrict__ warm) {
    SolveState init{};
    init.dt = *dt_dev;
    init.relative = s.relative_residual;
    init.absolute = s.absolute_residual;
    init.divergence_limit = s.divergence_limit;
    init.max_it = s.max_iterations > 0x7fffffffull ? 0x7fffffff : int(s.max_iterations);
    init.status = ST_RUNNING;
    init.flexible = flexible;
    if (warm && *warm != 0) init.flags = F_WARM;
    if (skip && *skip != 0) init.flags = F_DONE | F_STOP;
    *st = init;
}

// Condition of the restart branch of a loop trip (an IF node): the true
// residual asked for a restart.
__global__ void k_replace_cond(const SolveState* st, cudaGraphConditionalHandle handle) {
    cudaGraphSetConditional(handle, (st->flags & F_NEED_REPLACE) ? 1u : 0u);
}

// Condition of the WHILE node: repeat while the solve is running. The trip
// count is bounded; running out of trips ends the solve with an execution
// error instead of looping on.
__global__ void k_loop_cond(SolveState* st, cudaGraphConditionalHandle handle, int max_trips) {
    const int trips = st->trips + 1;
    st->trips = trips;
    unsigned go = (st->flags & F_DONE) ? 0u : 1u;
    if (go && trips >= max_trips) {
        st->status = RB200_EXECUTION;
        st->flags = st->flags | F_DONE | F_STOP;
        go = 0u;
    }
    cudaGraphSetConditional(handle, go);
}

// ------------------------------------------------------------ host side
constexpr int ZC = 8;
constexpr size_t kSmemPass1 = 2 * size_t(Slab<ZC>::SIZE) * sizeof(double);
constexpr size_t kSmemSlab = size_t(Slab<ZC>::SIZE) * sizeof(double);

static dim3 slab_grid(const GridDev& g) {
    return dim3((g.n[0] + TX - 1) / TX, (g.n[1] + TY - 1) / TY, (g.n[2] + ZC - 1) / ZC);
}
int slab_blocks(const GridDev& g) {
    dim3 d = slab_grid(g);
    return int(d.x * d.y * d.z);
}

static int ew_blocks(int n) {
    int b = (n + EW - 1) / EW;
    return b < 1 ? 1 : (b < EW_CAP ? b : EW_CAP);
}

// Dynamic shared memory above 48 KB must be opted into per kernel.
static int set_smem_attrs() {
    RB200_CUDA(cudaFuncSetAttribute(k_pass1<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemPass1)));
    RB200_CUDA(cudaFuncSetAttribute(k_pass2<ZC, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemSlab)));
    RB200_CUDA(cudaFuncSetAttribute(k_pass2<ZC, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemSlab)));
    RB200_CUDA(cudaFuncSetAttribute(k_pass2<ZC, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemSlab)));
    RB200_CUDA(cudaFuncSetAttribute(k_true_residual<ZC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(kSmemSlab)));
    return RB200_OK;
}

struct Bufs {
    double *b, *p, *r, *z, *d0, *d1, *r1;  // r1: the multigrid method's second residual buffer
    SolveState* st;
    Partials part;
    rb200_trace* trace;
    TmaMaps maps;
    SgsFlow sgs{};
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda). The encoder validates base, strides and box on the host.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    });
    return fn;
}

// TMA slabs need a row pitch that is a multiple of 16 bytes (nx even) and, to
// stay well inside the encoder's documented limits, a grid at least one box
// large in every direction. Other grids take the cp.async path.
static bool tma_eligible(const GridDev& g) {
    return (g.n[0] % 2) == 0 && g.n[0] >= Slab<ZC>::SX && g.n[1] >= Slab<ZC>::SY && g.n[2] >= Slab<ZC>::SZ;
}

static bool encode_map(CUtensorMap* m, const double* base, const GridDev& g, const cuuint32_t box[3]) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    cuuint64_t dims[3] = {cuuint64_t(g.n[0]), cuuint64_t(g.n[1]), cuuint64_t(g.n[2])};
    cuuint64_t strides[2] = {cuuint64_t(g.n[0]) * 8, cuuint64_t(g.n[0]) * cuuint64_t(g.n[1]) * 8};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims, strides,
                     const_cast<cuuint32_t*>(box), estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

static bool encode_slab_map(CUtensorMap* m, const double* base, const GridDev& g) {
    const cuuint32_t box[3] = {cuuint32_t(Slab<ZC>::SX), cuuint32_t(Slab<ZC>::SY), cuuint32_t(Slab<ZC>::SZ)};
    return encode_map(m, base, g, box);
}

static bool encode_box_map(CUtensorMap* m, const double* base, const GridDev& g) {
    const cuuint32_t box[3] = {cuuint32_t(TX), cuuint32_t(TY), cuuint32_t(ZC)};
    return encode_map(m, base, g, box);
}

static TmaMaps make_maps(const GridDev& g, const double* z, const double* d0, const double* d1, const double* p,
                         const double* r) {
    TmaMaps m;
    std::memset(&m, 0, sizeof(m));
    if (tma_eligible(g) && encode_slab_map(&m.z, z, g) && encode_slab_map(&m.d0, d0, g) &&
        encode_slab_map(&m.d1, d1, g) && encode_slab_map(&m.p, p, g) && encode_box_map(&m.p_box, p, g) &&
        encode_box_map(&m.r_box, r, g))
        m.use = 1;
    else
        std::memset(&m, 0, sizeof(m));
    return m;
}

// One lexicographic SGS application: both sweeps in one launch, then r.z.
static int launch_sgs(const GridDev& g, const Bufs& B, int mode, cudaStream_t s) {
    k_sgs_flow<<<B.sgs.blocks, SGS_THREADS, 0, s>>>(g, B.st, B.r, B.z, B.sgs, mode);
    k_sgs_dot<<<ew_blocks(g.cells), EW, 0, s>>>(g, B.st, B.r, B.z, mode, B.part, B.trace, B.sgs.ctl,
                                                B.sgs.ntiles + 2);
    return 2;
}

// Initial residual and preconditioned start (src/pressure.rs:603-650).
// `mg` is the multigrid hierarchy of the mixed method (nullptr otherwise).
static int launch_start(const GridDev& g, int method, const Bufs& B, const Multigrid* mg, cudaStream_t s) {
    const int eb = ew_blocks(g.cells);
    k_init_sums<<<eb, EW, 0, s>>>(g, B.st, B.b, B.p, B.part);
    if (method == RB200_JACOBI_PCG_V1) {
        k_load_residual<KIND_JACOBI><<<eb, EW, 0, s>>>(g, B.st, B.b, B.d0, B.d1, B.r, B.z, MODE_INIT, B.part,
                                                       B.trace);
        return 2;
    }
    if (method == RB200_RBSGS_PCG) {
        k_load_residual<KIND_RBSGS><<<eb, EW, 0, s>>>(g, B.st, B.b, B.d0, B.d1, B.r, B.z, MODE_INIT, B.part,
                                                      B.trace);
        const PairMap pm = pair_map(g);
        const int pb = ew_blocks(pm.pairs);
        k_rbsgs_black<<<pb, EW, 0, s>>>(g, pm, B.st, B.r, B.z, MODE_INIT);
        k_rbsgs_red_dot<<<pb, EW, 0, s>>>(g, pm, B.st, B.r, B.z, MODE_INIT, B.part, B.trace);
        return 4;
    }
    k_load_residual<KIND_MG><<<eb, EW, 0, s>>>(g, B.st, B.b, B.d0, B.d1, B.r, B.z, MODE_INIT, B.part, B.trace);
    if (method == RB200_SGS_PCG_V1) return 2 + launch_sgs(g, B, MODE_INIT, s);
    int n = 2 + mg->enqueue(B.r, B.st, MODE_INIT, s);
    return n + mg->enqueue_finish(B.st, B.r, B.r1, MODE_INIT, B.part, B.trace, s);
}

// One PCG iteration (src/pressure.rs:651-734).
static int launch_iteration(const GridDev& g, int method, const Bufs& B, const Multigrid* mg, cudaStream_t s) {
    const dim3 grid = slab_grid(g), block(TX, TY, 1);
    const int eb = ew_blocks(g.cells);
    const bool flexible = method == RB200_MG_MIXED;
    if (flexible)
        mg->enqueue_pass1(g, B.st, B.d0, B.d1, B.part, B.trace, s);
    else
        k_pass1<ZC><<<grid, block, kSmemPass1, s>>>(g, B.st, B.z, B.d0, B.d1, nullptr, B.maps, B.part, B.trace);
    if (method == RB200_JACOBI_PCG_V1) {
        k_pass2<ZC, 0><<<grid, block, kSmemSlab, s>>>(g, B.st, B.p, B.r, B.z, B.d0, B.d1, B.maps, B.part,
                                                         B.trace);
        return 2;
    }
    if (method == RB200_RBSGS_PCG) {
        k_pass2<ZC, 1><<<grid, block, kSmemSlab, s>>>(g, B.st, B.p, B.r, B.z, B.d0, B.d1, B.maps, B.part,
                                                          B.trace);
        const PairMap pm = pair_map(g);
        const int pb = ew_blocks(pm.pairs);
        k_rbsgs_black<<<pb, EW, 0, s>>>(g, pm, B.st, B.r, B.z, MODE_ITER);
        k_rbsgs_red_dot<<<pb, EW, 0, s>>>(g, pm, B.st, B.r, B.z, MODE_ITER, B.part, B.trace);
        return 4;
    }
    if (method == RB200_SGS_PCG_V1) {
        k_pass2<ZC, 2><<<grid, block, kSmemSlab, s>>>(g, B.st, B.p, B.r, B.z, B.d0, B.d1, B.maps, B.part,
                                                          B.trace);
        return 2 + launch_sgs(g, B, MODE_ITER, s);
    }
    int n = 2;
    if (mg->fuses_update()) {
        mg->enqueue_update_first(g, B.st, B.p, B.r, B.r1, B.d0, B.d1, B.part, B.trace, s);
        n += mg->enqueue(B.r, B.st, MODE_ITER, s, true);
    } else {
        k_mg_update<<<eb, EW, 0, s>>>(g, B.st, B.p, B.r, B.r1, B.d0, B.d1, B.part, B.trace);
        n += mg->enqueue(B.r, B.st, MODE_ITER, s);
    }
    return n + mg->enqueue_finish(B.st, B.r, B.r1, MODE_ITER, B.part, B.trace, s);
}

// The gated true-residual check and restart (src/pressure.rs:686-715).
static int launch_check(const GridDev& g, int method, const Bufs& B, const Multigrid* mg, cudaStream_t s) {
    const dim3 grid = slab_grid(g), block(TX, TY, 1);
    const int eb = ew_blocks(g.cells);
    k_true_residual<ZC><<<grid, block, kSmemSlab, s>>>(g, B.st, B.b, B.p, B.d0, B.d1, B.maps, B.part, B.trace);
    if (method == RB200_JACOBI_PCG_V1) {
        k_load_residual<KIND_JACOBI><<<eb, EW, 0, s>>>(g, B.st, B.b, B.d0, B.d1, B.r, B.z, MODE_REPLACE, B.part,
                                                       B.trace);
        return 2;
    }
    if (method == RB200_RBSGS_PCG) {
        k_load_residual<KIND_RBSGS><<<eb, EW, 0, s>>>(g, B.st, B.b, B.d0, B.d1, B.r, B.z, MODE_REPLACE, B.part,
                                                      B.trace);
        const PairMap pm = pair_map(g);
        const int pb = ew_blocks(pm.pairs);
        k_rbsgs_black<<<pb, EW, 0, s>>>(g, pm, B.st, B.r, B.z, MODE_REPLACE);
        k_rbsgs_red_dot<<<pb, EW, 0, s>>>(g, pm, B.st, B.r, B.z, MODE_REPLACE, B.part, B.trace);
        return 4;
    }
    k_load_residual<KIND_MG><<<eb, EW, 0, s>>>(g, B.st, B.b, B.d0, B.d1, B.r, B.z, MODE_REPLACE, B.part, B.trace);
    if (method == RB200_SGS_PCG_V1) return 2 + launch_sgs(g, B, MODE_REPLACE, s);
    int n = 2 + mg->enqueue(B.r, B.st, MODE_REPLACE, s);
    return n + mg->enqueue_finish(B.st, B.r, B.r1, MODE_REPLACE, B.part, B.trace, s);
}

static SolveState initial_state(double dt, const rb200_settings& s) {
    SolveState init{};
    init.dt = dt;
    init.relative = s.relative_residual;
    init.absolute = s.absolute_residual;
    init.divergence_limit = s.divergence_limit;
    init.max_it = s.max_iterations > 0x7fffffffull ? 0x7fffffff : int(s.max_iterations);
    init.status = ST_RUNNING;
    return init;
}

static void fill_report(const SolveState& f, rb200_report* report) {
    if (!report) return;
    std::memset(report, 0, sizeof(*report));
    report->iterations = uint64_t(f.it);
    report->true_residual_l2 = f.true_l2;
    report->true_residual_max = f.true_max;
    report->predicted_divergence_max = f.true_div;
    report->incompatible_sum = f.incompatible_sum;
    report->incompatible_budget = f.incompatible_budget;
    report->breakdown_iteration = uint64_t(f.breakdown_it);
}

PcgSolver::~PcgSolver() {
    if (chunk_exec_) cudaGraphExecDestroy(chunk_exec_);
    for (auto& e : ev_)
        if (e) cudaEventDestroy(e);
    cudaFree(b_);
    cudaFree(p_);
    cudaFree(r_);
    cudaFree(d_[0]);
    cudaFree(d_[1]);
    cudaFree(z_);
    cudaFree(r1_);
    cudaFree(part_.data);
    cudaFree(part_.ticket);
    cudaFree(st_);
    cudaFree(d_trace_);
    cudaFree(gbar_);
    cudaFree(ppart_);
    cudaFree(const_cast<int*>(sgs_.order));
    cudaFree(sgs_.ctl);
    if (h_st_) cudaFreeHost(h_st_);
}

// Whether a cooperative launch of the persistent kernel can sit in a CUDA
// graph, inside the body of a WHILE conditional node (the resident carrier's
// form). Checked once per process by capturing and instantiating such a graph
// (nothing is launched).
static bool persistent_graphs_supported(PcgSolver& solver) {
    static std::once_flag once;
    static bool supported = false;
    std::call_once(once, [&] {
        cudaStream_t outer = nullptr, body_stream = nullptr;
        if (cudaStreamCreateWithFlags(&outer, cudaStreamNonBlocking) != cudaSuccess) return;
        if (cudaStreamCreateWithFlags(&body_stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaStreamDestroy(outer);
            return;
        }
        bool ok = cudaStreamBeginCapture(outer, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        cudaGraph_t graph = nullptr;
        if (ok) {
            cudaStreamCaptureStatus status;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            cudaGraph_t g = nullptr;
            ok = cudaStreamGetCaptureInfo(outer, &status, nullptr, &g, &deps, &ndeps) == cudaSuccess;
            cudaGraphConditionalHandle handle;
            ok = ok && cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
            cudaGraphNodeParams cp{};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            ok = ok && cudaGraphAddNode(&node, g, deps, ndeps, &cp) == cudaSuccess;
            if (ok) {
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                ok = cudaStreamBeginCaptureToGraph(body_stream, body, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeRelaxed) == cudaSuccess;
                if (ok) {
                    const GridDev& gd = solver.grid();
                    cudaError_t le = solver.launch_persistent_chunk(body_stream, 1);
                    cudaGraph_t captured = nullptr;
                    cudaError_t ee = cudaStreamEndCapture(body_stream, &captured);
                    (void)gd;
                    ok = le == cudaSuccess && ee == cudaSuccess;
                }
                ok = ok && cudaStreamUpdateCaptureDependencies(outer, &node, 1, cudaStreamSetCaptureDependencies) ==
                               cudaSuccess;
            }
        }
        cudaError_t end = cudaStreamEndCapture(outer, &graph);
        ok = ok && end == cudaSuccess;
        if (ok) {
            cudaGraphExec_t exec = nullptr;
            ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
            if (exec) cudaGraphExecDestroy(exec);
        }
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        cudaStreamDestroy(body_stream);
        cudaStreamDestroy(outer);
        supported = ok;
    });
    return supported;
}

// The lexicographic SGS queue: tile ids in wave order, the zeroed state
// words, and the sweep kernel's resident block count.
int PcgSolver::sgs_setup() {
    const int nt0 = (g_.n[0] + SGS_T - 1) / SGS_T, nt1 = (g_.n[1] + SGS_T - 1) / SGS_T,
              nt2 = (g_.n[2] + SGS_T - 1) / SGS_T;
    std::vector<int> order;
    order.reserve(size_t(nt0) * nt1 * nt2);
    for (int w = 0; w <= nt0 + nt1 + nt2 - 3; ++w)
        for (int tz = 0; tz < nt2; ++tz)
            for (int ty = 0; ty < nt1; ++ty) {
                const int tx = w - ty - tz;
                if (tx >= 0 && tx < nt0) order.push_back(tx + nt0 * (ty + nt1 * tz));
            }
    sgs_.ntiles = int(order.size());
    int* d_order = nullptr;
    RB200_CUDA(cudaMalloc(&d_order, order.size() * sizeof(int)));
    sgs_.order = d_order;
    RB200_CUDA(cudaMalloc(&sgs_.ctl, (order.size() + 2) * sizeof(unsigned)));
    bytes_ += order.size() * sizeof(int) + (order.size() + 2) * sizeof(unsigned);
    RB200_CUDA(cudaMemcpyAsync(d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, stream_));
    RB200_CUDA(cudaMemsetAsync(sgs_.ctl, 0, (order.size() + 2) * sizeof(unsigned), stream_));
    RB200_CUDA(cudaStreamSynchronize(stream_));
    int dev = 0, sms = 0, per_sm = 0;
    RB200_CUDA(cudaGetDevice(&dev));
    RB200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sgs_flow, SGS_THREADS, 0));
    sgs_.blocks = int(std::min<long long>(2ll * sgs_.ntiles, std::max(1ll, (long long)sms * per_sm)));
    return RB200_OK;
}

int PcgSolver::init(const GridDev& g, int method, cudaStream_t stream) {
    g_ = g;
    method_ = method;
    stream_ = stream;
    if (method < RB200_JACOBI_PCG_V1 || method > RB200_MG_MIXED) return RB200_UNSUPPORTED;
    int rc = set_smem_attrs();
    if (rc) return rc;
    part_blocks_ = std::max(slab_blocks(g), EW_CAP);
    const size_t n = size_t(g.cells);
    auto alloc = [&](double** ptr, size_t count) -> int {
        cudaError_t e = cudaMalloc(ptr, count * sizeof(double));
        if (e != cudaSuccess) {
            set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
            return RB200_OUT_OF_MEMORY;
        }
        bytes_ += count * sizeof(double);
        return RB200_OK;
    };
    if ((rc = alloc(&b_, n)) || (rc = alloc(&p_, n)) || (rc = alloc(&r_, n)) || (rc = alloc(&z_, n)) ||
        (rc = alloc(&d_[0], n)) || (rc = alloc(&d_[1], n)))
        return rc;
    if (method == RB200_MG_MIXED) {
        if ((rc = alloc(&r1_, n))) return rc;
        RB200_CUDA(cudaMemsetAsync(r1_, 0, n * sizeof(double), stream_));
        if ((rc = mg_.init(g, stream_))) return rc;
        bytes_ += mg_.bytes();
    }
    // up to 2K + M = 9 doubles per block (the init sums)
    if ((rc = alloc(&part_.data, size_t(part_blocks_) * 12))) return rc;
    RB200_CUDA(cudaMalloc(&part_.ticket, sizeof(unsigned)));
    RB200_CUDA(cudaMemsetAsync(part_.ticket, 0, sizeof(unsigned), stream_));
    RB200_CUDA(cudaMalloc(&st_, sizeof(SolveState)));
    RB200_CUDA(cudaMallocHost(&h_st_, 2 * sizeof(SolveState)));
    for (auto& e : ev_) RB200_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    maps_ = make_maps(g, z_, d_[0], d_[1], p_, r_);
    if (method == RB200_SGS_PCG_V1 && (rc = sgs_setup())) return rc;
    chunk_ = method == RB200_MG_MIXED ? 4 : (g.cells >= (1 << 20) ? 32 : 16);
    // RB200_PERSISTENT=0 in the environment keeps the per-pass kernels (a
    // diagnostic switch: both paths compute the same iteration).
    const char* persist_env = std::getenv("RB200_PERSISTENT");
    const bool persist_allowed = !(persist_env && persist_env[0] == '0');
    if ((method == RB200_JACOBI_PCG_V1 || method == RB200_RBSGS_PCG) && maps_.use && persist_allowed) {
        persist_pre_ = method == RB200_RBSGS_PCG ? 1 : 0;
        int blocks = 0;
        if ((rc = persistent_setup(g, &blocks))) return rc;
        if (blocks > 0) {
            RB200_CUDA(cudaMalloc(&gbar_, sizeof(GridBarrier)));
            RB200_CUDA(cudaMemsetAsync(gbar_, 0, sizeof(GridBarrier), stream_));
            if ((rc = alloc(&ppart_, persistent_partial_doubles(blocks)))) return rc;
            persist_blocks_ = blocks;
            if (!persistent_graphs_supported(*this)) persist_blocks_ = 0;
            else chunk_ = 64;
        }
    }
    return capture_chunk();
}

cudaError_t PcgSolver::launch_persistent_chunk(cudaStream_t s, int budget) {
    return launch_persistent(g_, st_, b_, p_, r_, z_, d_[0], d_[1], ppart_, gbar_, d_trace_, maps_, persist_blocks_,
                             budget, s, persist_pre_);
}

int PcgSolver::set_trace(rb200_trace* host, size_t capacity) {
    if (d_trace_) {
        cudaFree(d_trace_);
        d_trace_ = nullptr;
    }
    h_trace_ = host;
    trace_cap_ = host ? capacity : 0;
    if (trace_cap_) RB200_CUDA(cudaMalloc(&d_trace_, trace_cap_ * sizeof(rb200_trace)));
    if (chunk_exec_) {
        cudaGraphExecDestroy(chunk_exec_);
        chunk_exec_ = nullptr;
    }
    return capture_chunk();
}

// One chunk: `chunk_` iterations, then the gated true-residual and restart.
int PcgSolver::capture_chunk() {
    const Bufs B{b_, p_, r_, z_, d_[0], d_[1], r1_, st_, part_, d_trace_, maps_, sgs_};
    const Multigrid* mg = method_ == RB200_MG_MIXED ? &mg_ : nullptr;
    cudaGraph_t graph = nullptr;
    RB200_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    int nodes = 0;
    cudaError_t launch_err = cudaSuccess;
    if (persist_blocks_) {
        launch_err = launch_persistent(g_, st_, b_, p_, r_, z_, d_[0], d_[1], ppart_, gbar_, d_trace_, maps_,
                                       persist_blocks_, chunk_, stream_, persist_pre_);
        nodes = 1;
    } else {
        for (int q = 0; q < chunk_; ++q) nodes += launch_iteration(g_, method_, B, mg, stream_);
        nodes += launch_check(g_, method_, B, mg, stream_);
    }
    nodes_per_chunk_ = nodes;
    if (launch_err == cudaSuccess) launch_err = cudaGetLastError();
    cudaError_t end_err = cudaStreamEndCapture(stream_, &graph);
    if (launch_err != cudaSuccess || end_err != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        set_error(std::string("chunk capture: ") +
                  cudaGetErrorString(launch_err != cudaSuccess ? launch_err : end_err));
        return RB200_EXECUTION;
    }
    cudaError_t e = cudaGraphInstantiate(&chunk_exec_, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        return RB200_EXECUTION;
    }
    return RB200_OK;
}

int PcgSolver::launch_chunk(int slot) {
    RB200_CUDA(cudaGraphLaunch(chunk_exec_, stream_));
    launches_ += uint64_t(nodes_per_chunk_);
    return record_flags(slot);
}

int PcgSolver::record_flags(int slot) {
    RB200_CUDA(cudaMemcpyAsync(&h_st_[slot], st_, sizeof(SolveState), cudaMemcpyDeviceToHost, stream_));
    RB200_CUDA(cudaEventRecord(ev_[slot], stream_));
    return RB200_OK;
}

int PcgSolver::solve(double dt, const rb200_settings& s, rb200_report* report, rb200_cancel_fn cancelled,
                     void* ctx, const double* initial) {
    if (report) std::memset(report, 0, sizeof(*report));
    SolveState init = initial_state(dt, s);
    init.flexible = method_ == RB200_MG_MIXED ? 1 : 0;
    if (initial) {
        RB200_CUDA(cudaMemcpyAsync(p_, initial, size_t(g_.cells) * sizeof(double), cudaMemcpyDefault, stream_));
        init.flags |= F_WARM;
    }
    if (d_trace_ && uint64_t(init.max_it) > trace_cap_) {
        set_error("trace capacity is smaller than max_iterations");
        return RB200_INVALID_ARGUMENT;
    }
    h_st_[0] = init;
    RB200_CUDA(cudaMemcpyAsync(st_, &h_st_[0], sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
    if (d_trace_) RB200_CUDA(cudaMemsetAsync(d_trace_, 0, trace_cap_ * sizeof(rb200_trace), stream_));
    RB200_CUDA(cudaMemsetAsync(part_.ticket, 0, sizeof(unsigned), stream_));
    if (gbar_) RB200_CUDA(cudaMemsetAsync(gbar_, 0, sizeof(GridBarrier), stream_));
    launches_ += uint64_t(launch_start(g_, method_, Bufs{b_, p_, r_, z_, d_[0], d_[1], r1_, st_, part_, d_trace_, maps_, sgs_},
                                       method_ == RB200_MG_MIXED ? &mg_ : nullptr, stream_));
    RB200_CUDA(cudaGetLastError());
    // The host copy of the state must be stable before the chunk copies reuse
    // h_st_ slots.
    RB200_CUDA(cudaStreamSynchronize(stream_));
    int rc;
    if ((rc = record_flags(0))) return rc;
    if ((rc = launch_chunk(1))) return rc;
    int slot = 0, last_it = -1, stalls = 0;
    bool cancelled_now = false;
    for (;;) {
        RB200_CUDA(cudaEventSynchronize(ev_[slot]));
        const SolveState& h = h_st_[slot];
        if (h.flags & F_DONE) break;
        if (cancelled && cancelled(ctx)) {
            cancelled_now = true;
            break;
        }
        if (h.it == last_it) {
            if (++stalls > 4) {
                RB200_CUDA(cudaStreamSynchronize(stream_));
                set_error("pressure solve made no progress");
                return RB200_EXECUTION;
            }
        } else {
            stalls = 0;
            last_it = h.it;
        }
        if ((rc = launch_chunk(slot))) return rc;
        slot ^= 1;
    }
    RB200_CUDA(cudaStreamSynchronize(stream_));
    RB200_CUDA(cudaMemcpy(&h_st_[0], st_, sizeof(SolveState), cudaMemcpyDeviceToHost));
    const SolveState& f = h_st_[0];
    if (d_trace_ && h_trace_) {
        size_t n = std::min(trace_cap_, size_t(f.it));
        RB200_CUDA(cudaMemcpy(h_trace_, d_trace_, n * sizeof(rb200_trace), cudaMemcpyDeviceToHost));
    }
    fill_report(f, report);
    if (cancelled_now) return RB200_CANCELLED;
    return f.status;
}

int PcgSolver::enqueue_reset(const double* dt_dev, const int* skip, const rb200_settings& settings, cudaStream_t s,
                             const int* warm, const double* seed) {
    if (warm && seed) {
        k_seed_pressure<<<ew_blocks(g_.cells), EW, 0, s>>>(g_.cells, p_, seed, warm);
        launches_ += 1;
    }
    k_solve_reset<<<1, 1, 0, s>>>(st_, settings, dt_dev, skip, method_ == RB200_MG_MIXED ? 1 : 0,
                                  (warm && seed) ? warm : nullptr);
    RB200_CUDA(cudaMemsetAsync(part_.ticket, 0, sizeof(unsigned), s));
    if (gbar_) RB200_CUDA(cudaMemsetAsync(gbar_, 0, sizeof(GridBarrier), s));
    launches_ += 1;
    const Bufs B{b_, p_, r_, z_, d_[0], d_[1], r1_, st_, part_, d_trace_, maps_, sgs_};
    launch_start(g_, method_, B, method_ == RB200_MG_MIXED ? &mg_ : nullptr, s);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

int PcgSolver::enqueue_loop(cudaStream_t cs, cudaStream_t body_stream, const rb200_settings& settings) {
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    RB200_CUDA(cudaStreamGetCaptureInfo(cs, &status, nullptr, &graph, &deps, &ndeps));
    if (status != cudaStreamCaptureStatusActive) {
        set_error("enqueue_loop needs an active stream capture");
        return RB200_EXECUTION;
    }
    cudaGraphConditionalHandle handle;
    RB200_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    RB200_CUDA(cudaGraphAddNode(&node, graph, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    // The loop body: one chunk of iterations, the gated check, the condition.
    RB200_CUDA(cudaStreamBeginCaptureToGraph(body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    const Bufs B{b_, p_, r_, z_, d_[0], d_[1], r1_, st_, part_, d_trace_, maps_, sgs_};
    const Multigrid* mg = method_ == RB200_MG_MIXED ? &mg_ : nullptr;
    if (persist_blocks_) {
        RB200_CUDA(launch_persistent(g_, st_, b_, p_, r_, z_, d_[0], d_[1], ppart_, gbar_, d_trace_, maps_,
                                     persist_blocks_, chunk_, body_stream, persist_pre_));
    } else if (mg) {
        // The multigrid restart (a whole V-cycle) as an IF node after the
        // true-residual check: its launches run only in trips that restart.
        int nodes = 0;
        for (int q = 0; q < chunk_; ++q) nodes += launch_iteration(g_, method_, B, mg, body_stream);
        const dim3 grid = slab_grid(g_), block(TX, TY, 1);
        k_true_residual<ZC><<<grid, block, kSmemSlab, body_stream>>>(g_, B.st, B.b, B.p, B.d0, B.d1, B.maps, B.part,
                                                                      B.trace);
        cudaStreamCaptureStatus bst;
        const cudaGraphNode_t* bdeps = nullptr;
        size_t nbdeps = 0;
        cudaGraph_t bodyg = nullptr;
        RB200_CUDA(cudaStreamGetCaptureInfo(body_stream, &bst, nullptr, &bodyg, &bdeps, &nbdeps));
        cudaGraphConditionalHandle rh;
        RB200_CUDA(cudaGraphConditionalHandleCreate(&rh, bodyg, 0, cudaGraphCondAssignDefault));
        k_replace_cond<<<1, 1, 0, body_stream>>>(st_, rh);
        RB200_CUDA(cudaStreamGetCaptureInfo(body_stream, &bst, nullptr, &bodyg, &bdeps, &nbdeps));
        cudaGraphNodeParams ip{};
        ip.type = cudaGraphNodeTypeConditional;
        ip.conditional.handle = rh;
        ip.conditional.type = cudaGraphCondTypeIf;
        ip.conditional.size = 1;
        cudaGraphNode_t inode;
        RB200_CUDA(cudaGraphAddNode(&inode, bodyg, bdeps, nbdeps, &ip));
        cudaStream_t rs = nullptr;
        RB200_CUDA(cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking));
        cudaError_t ce = cudaStreamBeginCaptureToGraph(rs, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeRelaxed);
        if (ce == cudaSuccess) {
            const int eb = ew_blocks(g_.cells);
            k_load_residual<KIND_MG><<<eb, EW, 0, rs>>>(g_, B.st, B.b, B.d0, B.d1, B.r, B.z, MODE_REPLACE, B.part,
                                                        B.trace);
            mg->enqueue(B.r, B.st, MODE_REPLACE, rs);
            mg->enqueue_finish(B.st, B.r, B.r1, MODE_REPLACE, B.part, B.trace, rs);
            cudaGraph_t rbody = nullptr;
            ce = cudaStreamEndCapture(rs, &rbody);
        }
        cudaStreamDestroy(rs);
        if (ce != cudaSuccess) {
            set_error(std::string("restart branch capture: ") + cudaGetErrorString(ce));
            return RB200_EXECUTION;
        }
        RB200_CUDA(cudaStreamUpdateCaptureDependencies(body_stream, &inode, 1, cudaStreamSetCaptureDependencies));
        nodes_per_chunk_ = nodes + 2;  // the check and the branch condition (the restart runs rarely)
    } else {
        for (int q = 0; q < chunk_; ++q) launch_iteration(g_, method_, B, mg, body_stream);
        launch_check(g_, method_, B, mg, body_stream);
    }
    const uint64_t mi = settings.max_iterations;
    // Every trip of a running solve does at least one iteration (a candidate
    // stops the rest of its trip for the true-residual check), so the
    // iteration limit ends a solve before this bound does, as in the
    // reference, however often it restarts.
    const uint64_t trips = mi + 64;
    k_loop_cond<<<1, 1, 0, body_stream>>>(st_, handle, trips > (1u << 24) ? (1 << 24) : int(trips));
    cudaError_t le = cudaGetLastError();
    cudaGraph_t captured = nullptr;
    cudaError_t ee = cudaStreamEndCapture(body_stream, &captured);
    if (le != cudaSuccess || ee != cudaSuccess) {
        set_error(std::string("loop body capture: ") + cudaGetErrorString(le != cudaSuccess ? le : ee));
        return RB200_EXECUTION;
    }
    RB200_CUDA(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
    return RB200_OK;
}

int PcgSolver::profile(int which, int launches, double* avg_ms) {
    if (launches < 1 || which < 0 || which > 2) return RB200_INVALID_ARGUMENT;
    if (method_ == RB200_MG_MIXED && which == 1) return RB200_UNSUPPORTED;
    if (which == 2 && !persist_blocks_) return RB200_UNSUPPORTED;
    SolveState prof{};
    prof.rz = 1.0;
    prof.alpha = 1e-6;
    prof.beta = 0.5;
    prof.threshold = -1.0;
    prof.max_it = 0x7fffffff;
    prof.flags = F_PROFILE;
    prof.status = ST_RUNNING;
    h_st_[0] = prof;
    RB200_CUDA(cudaMemcpyAsync(st_, &h_st_[0], sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
    const bool jac = method_ == RB200_JACOBI_PCG_V1;
    const dim3 grid = slab_grid(g_), block(TX, TY, 1);
    if (which == 2) {
        // one warm iteration, then `launches` iterations in one launch
        RB200_CUDA(cudaMemsetAsync(gbar_, 0, sizeof(GridBarrier), stream_));
        RB200_CUDA(launch_persistent(g_, st_, b_, p_, r_, z_, d_[0], d_[1], ppart_, gbar_, nullptr, maps_,
                                     persist_blocks_, 1, stream_, persist_pre_));
        cudaEvent_t a, b;
        RB200_CUDA(cudaEventCreate(&a));
        RB200_CUDA(cudaEventCreate(&b));
        RB200_CUDA(cudaEventRecord(a, stream_));
        RB200_CUDA(launch_persistent(g_, st_, b_, p_, r_, z_, d_[0], d_[1], ppart_, gbar_, nullptr, maps_,
                                     persist_blocks_, launches, stream_, persist_pre_));
        RB200_CUDA(cudaEventRecord(b, stream_));
        RB200_CUDA(cudaEventSynchronize(b));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        RB200_CUDA(cudaGetLastError());
        RB200_CUDA(cudaMemcpy(&h_st_[0], st_, sizeof(SolveState), cudaMemcpyDeviceToHost));
        if (h_st_[0].status == RB200_EXECUTION) {
            set_error("persistent solver timing run failed");
            return RB200_EXECUTION;
        }
        *avg_ms = double(ms) / launches;
        return RB200_OK;
    }
    auto launch = [&]() {
        if (which == 0)
            k_pass1<ZC><<<grid, block, kSmemPass1, stream_>>>(g_, st_, z_, d_[0], d_[1], nullptr, maps_, part_, nullptr);
        else if (jac)
            k_pass2<ZC, 0><<<grid, block, kSmemSlab, stream_>>>(g_, st_, p_, r_, z_, d_[0], d_[1], maps_, part_,
                                                                   nullptr);
        else if (method_ == RB200_SGS_PCG_V1)
            k_pass2<ZC, 2><<<grid, block, kSmemSlab, stream_>>>(g_, st_, p_, r_, z_, d_[0], d_[1], maps_, part_,
                                                                   nullptr);
        else
            k_pass2<ZC, 1><<<grid, block, kSmemSlab, stream_>>>(g_, st_, p_, r_, z_, d_[0], d_[1], maps_, part_,
                                                                    nullptr);
    };
    launch();  // warm
    cudaEvent_t a, b;
    RB200_CUDA(cudaEventCreate(&a));
    RB200_CUDA(cudaEventCreate(&b));
    RB200_CUDA(cudaEventRecord(a, stream_));
    for (int q = 0; q < launches; ++q) launch();
    RB200_CUDA(cudaEventRecord(b, stream_));
    RB200_CUDA(cudaEventSynchronize(b));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    RB200_CUDA(cudaGetLastError());
    *avg_ms = double(ms) / launches;
    return RB200_OK;
}

// ProviderWorkspace's qualification of a candidate pressure
// (src/solver_provider.rs:239-270) in one pass: t = b - K p, |t|^2 and |b|^2
// (compensated), max|t|, and flags for a non-finite pressure (1) or product
// (2). out = {|t|^2, |b|^2, max|t|, flags, p[0]}.
__global__ void __launch_bounds__(EW) k_qualify_pressure(GridDev g, const double* __restrict__ b,
                                                         const double* __restrict__ p, Partials part,
                                                         double* __restrict__ out) {
    __shared__ BlockReduce<2, 2> sm;
    Neu tt, bb;
    double m[2] = {0.0, 0.0};
    const int sy = g.n[0], sz = g.n[0] * g.n[1];
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.cells; c += gridDim.x * blockDim.x) {
        int i, j, k;
        cell_coords(g, c, i, j, k);
        Neigh v;
        v.c = p[c];
        v.xm = i > 0 ? p[c - 1] : 0.0;
        v.xp = i + 1 < g.n[0] ? p[c + 1] : 0.0;
        v.ym = j > 0 ? p[c - sy] : 0.0;
        v.yp = j + 1 < g.n[1] ? p[c + sy] : 0.0;
        v.zm = k > 0 ? p[c - sz] : 0.0;
        v.zp = k + 1 < g.n[2] ? p[c + sz] : 0.0;
        if (!isfinite(v.c)) m[1] = fmax(m[1], 1.0);
        const double q = apply_row(g, i, j, k, v);
        if (!isfinite(q)) m[1] = fmax(m[1], 2.0);
        const double bc = b[c];
        const double t = bc - q;
        tt.add(t * t);
        bb.add(bc * bc);
        m[0] = fmax(m[0], fabs(t));
    }
    dd sums[2] = {tt.as_dd(), bb.as_dd()};
    block_reduce<2, 2>(sm, sums, m);
    if (publish_and_check_last<2, 2>(part, blockIdx.x, gridDim.x, sums, m)) {
        fold_partials<2, 2>(part, gridDim.x, sm, sums, m);
        if (threadIdx.x == 0) {
            out[0] = dd_value(sums[0]);
            out[1] = dd_value(sums[1]);
            out[2] = m[0];
            out[3] = m[1];
            out[4] = p[0];
        }
    }
}

int launch_qualify_pressure(const GridDev& g, const double* b, const double* p, Partials part, double* out,
                            cudaStream_t s) {
    k_qualify_pressure<<<ew_blocks(g.cells), EW, 0, s>>>(g, b, p, part, out);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

int launch_precondition_jacobi(const GridDev& g, const double* r, double* z, Partials part, double* rz_out,
                               cudaStream_t s) {
    k_precondition_jacobi<<<ew_blocks(g.cells), EW, 0, s>>>(g, r, z, part, rz_out);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}
int precondition_partials_blocks() { return EW_CAP; }

// ------------------------------------------------------------ allocation-free solve
// A Jacobi-PCG solve for callers that cannot allocate device memory: a host
// application whose device memory is owned by its own allocator under a fixed
// budget, so that a plug-in may not grow its footprint while it runs. Its
// scratch (residual, two direction buffers, preconditioned residual,
// reduction partials, solver state and ticket) lives in this fixed file-scope
// device array, which every GPU that loads the library holds until the process
// exits. It has no counterpart in the reference.
constexpr int kStaticMaxCells = 32768;   // 32^3 cells
constexpr int kStaticMaxBlocks = 2048;   // blocks of the widest pass of a solve
// Doubles of one block's reduction partials in the widest stage of a solve:
// k_init_sums publishes 3 double-double sums and 3 maxima (2 * 3 + 3); the
// other stages publish fewer (true residual 5, pass 2 4, pass 1 and the
// residual load 2).
constexpr int kStaticSlotDoubles = 2 * 3 + 3;
constexpr size_t kStaticStateDoubles = 64;
constexpr size_t kStaticPartialDoubles = size_t(kStaticMaxBlocks) * kStaticSlotDoubles;
constexpr size_t kStaticDoubles = 4 * size_t(kStaticMaxCells) + kStaticPartialDoubles + kStaticStateDoubles;
static __device__ __align__(256) double g_static_scratch[kStaticDoubles];

static_assert(sizeof(SolveState) + sizeof(unsigned) <= kStaticStateDoubles * sizeof(double),
              "state does not fit the static scratch");

// Device address of g_static_scratch per device, resolved once per device
// with that device current. In host code the symbol itself is only a host-side
// stand-in, never a device address. The cached address belongs to the
// device's primary context: after cudaDeviceReset the array may be loaded at
// another address, so a process that resets a device must not call the
// allocation-free solve on it again.
static double* static_scratch_address(int device, int* rc) {
    static std::mutex mu;
    static double* addr[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 64) {
        *rc = RB200_INVALID_ARGUMENT;
        return nullptr;
    }
    if (!addr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr) {
            set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            *rc = RB200_EXECUTION;
            return nullptr;
        }
        addr[device] = static_cast<double*>(ptr);
    }
    *rc = RB200_OK;
    return addr[device];
}

int static_solve_jacobi(const GridDev& g, const double* rhs, double* pressure, double dt, const rb200_settings& s,
                        rb200_report* report, cudaStream_t stream) {
    if (g.cells > kStaticMaxCells) {
        set_error("grid exceeds the 32768-cell limit of the allocation-free solve");
        return RB200_UNSUPPORTED;
    }
    // every stage's partials (at most kStaticSlotDoubles per block) must fit
    // the reserved region
    if (size_t(std::max(slab_blocks(g), ew_blocks(g.cells))) * kStaticSlotDoubles > kStaticPartialDoubles) {
        set_error("grid shape needs more reduction blocks than the allocation-free solve holds");
        return RB200_UNSUPPORTED;
    }
    int device = 0;
    RB200_CUDA(cudaGetDevice(&device));
    int rc = RB200_OK;
    double* base = static_scratch_address(device, &rc);
    if (rc) return rc;
    if ((rc = set_smem_attrs())) return rc;
    Bufs B;
    B.b = const_cast<double*>(rhs);  // read only
    B.p = pressure;
    B.r = base;
    B.d0 = B.r + kStaticMaxCells;
    B.d1 = B.d0 + kStaticMaxCells;
    B.z = B.d1 + kStaticMaxCells;
    B.r1 = nullptr;
    B.part.data = B.z + kStaticMaxCells;
    double* state_slot = B.part.data + kStaticPartialDoubles;
    B.st = reinterpret_cast<SolveState*>(state_slot);
    B.part.ticket = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(state_slot) + sizeof(SolveState));
    B.trace = nullptr;
    B.maps = make_maps(g, B.z, B.d0, B.d1, B.p, B.r);

    SolveState init = initial_state(dt, s);
    // The array keeps the previous call's contents: the ticket must start at 0.
    RB200_CUDA(cudaMemsetAsync(B.part.ticket, 0, sizeof(unsigned), stream));
    RB200_CUDA(cudaMemcpyAsync(B.st, &init, sizeof(SolveState), cudaMemcpyHostToDevice, stream));
    launch_start(g, RB200_JACOBI_PCG_V1, B, nullptr, stream);
    RB200_CUDA(cudaGetLastError());
    const int chunk = 16;
    int last_it = -1, stalls = 0;
    SolveState h{};
    for (;;) {
        RB200_CUDA(cudaMemcpyAsync(&h, B.st, sizeof(SolveState), cudaMemcpyDeviceToHost, stream));
        RB200_CUDA(cudaStreamSynchronize(stream));
        if (h.flags & F_DONE) break;
        if (h.it == last_it) {
            if (++stalls > 4) {
                set_error("pressure solve made no progress");
                return RB200_EXECUTION;
            }
        } else {
            stalls = 0;
            last_it = h.it;
        }
        for (int q = 0; q < chunk; ++q) launch_iteration(g, RB200_JACOBI_PCG_V1, B, nullptr, stream);
        launch_check(g, RB200_JACOBI_PCG_V1, B, nullptr, stream);
        RB200_CUDA(cudaGetLastError());
    }
    fill_report(h, report);
    return h.status;
}

}  // namespace rb200

extern "C" int rb200_pressure_solve_static(const rb200_grid* grid, double density, const double* rhs_device,
                                           double* pressure_device, size_t len, double dt,
                                           const rb200_settings* settings, rb200_report* report, void* stream) {
    using namespace rb200;
    if (!grid || !rhs_device || !pressure_device || !settings) return RB200_INVALID_ARGUMENT;
    GridDev g;
    int rc = make_grid_dev(grid, density, &g);
    if (rc) return rc;
    if (len != size_t(g.cells)) return RB200_LENGTH_MISMATCH;
    if (!std::isfinite(dt) || dt <= 0.0 || !settings_valid(settings)) return RB200_INVALID_ARGUMENT;
    return static_solve_jacobi(g, rhs_device, pressure_device, dt, *settings, report, (cudaStream_t)stream);
}
