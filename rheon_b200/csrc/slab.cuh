// Shared-memory halo slabs for the 7-point PCG passes.
//
// A block owns a TX x TY x ZC brick of cells and stages the brick plus its
// halo of one array into shared memory, then computes every cell of the brick
// from shared memory. The slab is (TX+4) x (TY+2) x (ZC+2) values: slab
// element (sx, sy, sz) holds cell (x0-2+sx, y0-1+sy, k0-1+sz). The x extent
// starts two cells left of the brick so that the TMA box starts on a 16-byte
// boundary (x0 is a multiple of 32, so x0-2 is even for 8-byte values).
//
// Loads: one TMA tiled copy (cp.async.bulk.tensor.3d, no multicast) per slab
// when the row pitch is a multiple of 16 bytes (nx even); out-of-box elements
// are zero-filled by the hardware. Otherwise a row-wise cp.async path fills the
// same layout. Halo values outside the domain are zero and never used by
// apply_row's masks.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "stencil.cuh"

namespace rb200 {

template <int ZC>
struct Slab {
    static constexpr int SX = TX + 4;
    static constexpr int SY = TY + 2;
    static constexpr int SZ = ZC + 2;
    static constexpr int SIZE = SX * SY * SZ;
    static constexpr int PLANE = SX * SY;
    static constexpr unsigned BYTES = unsigned(SIZE) * 8u;
    // slab element of the block's own cell (tx, ty, q)
    static __device__ __forceinline__ int own(int tx, int ty, int q) { return (tx + 2) + SX * ((ty + 1) + SY * (q + 1)); }
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// ------------------------------------------------------------ cp.async path
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <int ZC>
__device__ __forceinline__ void slab_issue_rows(const GridDev& g, double* sm, const double* __restrict__ src, int x0,
                                                int y0, int k0) {
    using S = Slab<ZC>;
    const int lane = threadIdx.x, warp = threadIdx.y;  // blockDim = (32, TY)
    for (int row = warp; row < S::SY * S::SZ; row += TY) {
        const int sy = row % S::SY, sz = row / S::SY;
        const int j = y0 - 1 + sy, k = k0 - 1 + sz;
        double* dst = sm + row * S::SX;
        const bool rowin = j >= 0 && j < g.n[1] && k >= 0 && k < g.n[2];
        const double* base = src + (rowin ? cell_idx(g, 0, j, k) : 0);
        for (int sx = lane; sx < S::SX; sx += 32) {
            const int i = x0 - 2 + sx;
            if (rowin && i >= 0 && i < g.n[0])
                cp_async8(dst + sx, base + i);
            else
                dst[sx] = 0.0;
        }
    }
}

// ------------------------------------------------------------ TMA path
// mbarrier waits are bounded: after kSpinLimit polls the caller gets false,
// records an execution error and gives the copy a second bounded wait.
constexpr unsigned kSpinLimit = 1u << 26;

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    for (unsigned n = 0; n < kSpinLimit; ++n)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 3-D tiled TMA load of one slab into shared memory (no multicast).
__device__ __forceinline__ void tma_load_slab(double* smem_dst, const CUtensorMap* map, int x, int y, int z,
                                              uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(smem_dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Neighbours of slab element e.
template <int ZC>
__device__ __forceinline__ Neigh slab_neigh(const double* sm, int e) {
    using S = Slab<ZC>;
    Neigh v;
    v.c = sm[e];
    v.xm = sm[e - 1];
    v.xp = sm[e + 1];
    v.ym = sm[e - S::SX];
    v.yp = sm[e + S::SX];
    v.zm = sm[e - S::PLANE];
    v.zp = sm[e + S::PLANE];
    return v;
}

// Reference-order compensated accumulation (Neumaier, src/pressure.rs:135-148)
// of one thread's terms; folded into a double-double for the block reduction.
// The rounding error of each s + x is formed branch-free by two-sum; it is
// the exact error, so it equals Neumaier's (s - t) + x or (x - t) + s and the
// compensation c is the same value bit for bit.
struct Neu {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        double t, e;
        two_sum(s, x, t, e);
        c += e;
        s = t;
    }
    __device__ __forceinline__ dd as_dd() const {
        dd r;
        two_sum(s, c, r.hi, r.lo);
        return r;
    }
};

}  // namespace rb200
