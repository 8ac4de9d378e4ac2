// Sealed-box PressureOperator primitives on the device (src/operator.rs).
// Each kernel keeps the reference's per-element operation order; the library
// is built with -fmad=false so no multiply-add is fused.
#include "internal.hpp"
#include "project.cuh"
#include "stencil.cuh"

namespace rb200 {


static inline int ew_blocks(long long n) {
    long long b = (n + EW_THREADS - 1) / EW_THREADS;
    if (b < 1) b = 1;
    return int(b < EW_BLOCKS_CAP ? b : EW_BLOCKS_CAP);
}

int partials_blocks_needed(const GridDev& g) {
    MarchGrid m1 = march_grid(g.n, 1);
    int need = m1.nblocks;  // the deepest split any marching kernel may use
    return need > EW_BLOCKS_CAP ? need : EW_BLOCKS_CAP;
}

// ------------------------------------------------------------ apply_full
__global__ void __launch_bounds__(TILE_THREADS) k_apply_full(GridDev g, int zc, const double* __restrict__ p,
                                                              double* __restrict__ out, int* flags) {
    march(
        g, zc, [&](int c, int, int, int) { return p[c]; },
        [&](int c, int i, int j, int k, const Neigh& v) {
            double q = apply_row(g, i, j, k, v);
            if (!isfinite(q)) atomicOr(flags, VF_ARITH);
            out[c] = q;
        });
}

int launch_apply_full(const GridDev& g, const double* p, double* out, int* flags, cudaStream_t s) {
    MarchGrid m = march_grid(g.n, 16);
    k_apply_full<<<m.grid, m.block, 0, s>>>(g, m.zc, p, out, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

// ------------------------------------------------------------ finiteness
// validate_cells (src/operator.rs:840-848): every value finite.
__global__ void k_check_finite(const double* __restrict__ x, int n, int* flags) {
    int local = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        if (!isfinite(x[c])) local = VF_NONFINITE;
    if (local) atomicOr(flags, local);
}

int launch_check_finite(const double* x, int n, int* flags, cudaStream_t s) {
    k_check_finite<<<ew_blocks(n), EW_THREADS, 0, s>>>(x, n, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

// ------------------------------------------------------------ validation
// validate_velocity (src/operator.rs:850-875): finite, wall-normal faces zero.
template <class T>
__global__ void k_validate_faces(GridDev g, const T* __restrict__ u, const T* __restrict__ v,
                                 const T* __restrict__ w, int* flags) {
    const long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    int local = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int a = 0;
        long long f = t;
        if (f >= g.flen[0]) {
            f -= g.flen[0];
            a = 1;
            if (f >= g.flen[1]) {
                f -= g.flen[1];
                a = 2;
            }
        }
        const T* src = a == 0 ? u : (a == 1 ? v : w);
        T x = src[f];
        if (!isfinite(double(x))) local |= VF_NONFINITE;
        int fi = int(f % g.fc[a][0]);
        int fj = int((f / g.fc[a][0]) % g.fc[a][1]);
        int fk = int(f / ((long long)g.fc[a][0] * g.fc[a][1]));
        if (is_wall_face(g, a, fi, fj, fk) && x != T(0)) local |= VF_WALL;
    }
    if (local) atomicOr(flags, local);
}

template <class T>
int launch_validate_faces(const GridDev& g, const T* u, const T* v, const T* w, int* flags,
                          cudaStream_t s) {
    long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    k_validate_faces<T><<<ew_blocks(total), EW_THREADS, 0, s>>>(g, u, v, w, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

// ------------------------------------------------------------ build_rhs
template <class T>
__global__ void k_build_rhs(GridDev g, const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w,
                            double dt, double* __restrict__ out, int* flags) {
    build_rhs_body<T>(g, u, v, w, dt, out, flags, whole_launch());
}

template <class T>
int launch_build_rhs(const GridDev& g, const T* u, const T* v, const T* w, double dt, double* out,
                     int* flags, cudaStream_t s) {
    k_build_rhs<T><<<ew_blocks(g.cells), EW_THREADS, 0, s>>>(g, u, v, w, dt, out, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

template <class T>
__global__ void k_divergence(GridDev g, const T* __restrict__ u, const T* __restrict__ v,
                             const T* __restrict__ w, double* __restrict__ out, int* flags) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.cells; c += gridDim.x * blockDim.x) {
        int i, j, k;
        cell_coords(g, c, i, j, k);
        double value = cell_divergence<T>(
            g, double(u[face_idx(g, 0, i, j, k)]), double(u[face_idx(g, 0, i + 1, j, k)]),
            double(v[face_idx(g, 1, i, j, k)]), double(v[face_idx(g, 1, i, j + 1, k)]),
            double(w[face_idx(g, 2, i, j, k)]), double(w[face_idx(g, 2, i, j, k + 1)]));
        if (!isfinite(value)) atomicOr(flags, VF_ARITH);
        out[c] = value;
    }
}

template <class T>
int launch_divergence(const GridDev& g, const T* u, const T* v, const T* w, double* out,
                      int* flags, cudaStream_t s) {
    k_divergence<T><<<ew_blocks(g.cells), EW_THREADS, 0, s>>>(g, u, v, w, out, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

template <class T>
__global__ void k_correct(GridDev g, const double* __restrict__ p, double dt, T* u, T* v, T* w,
                          int* flags) {
    const long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    const int s[3] = {1, g.n[0], g.n[0] * g.n[1]};
    int local = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int a = 0;
        long long f = t;
        if (f >= g.flen[0]) {
            f -= g.flen[0];
            a = 1;
            if (f >= g.flen[1]) {
                f -= g.flen[1];
                a = 2;
            }
        }
        int fi = int(f % g.fc[a][0]);
        int fj = int((f / g.fc[a][0]) % g.fc[a][1]);
        int fk = int(f / ((long long)g.fc[a][0] * g.fc[a][1]));
        if (is_wall_face(g, a, fi, fj, fk)) continue;
        T* dst = a == 0 ? u : (a == 1 ? v : w);
        int c = cell_idx(g, fi, fj, fk);
        dst[f] = corrected<T>(g, a, dst[f], p[c], p[c - s[a]], dt, local);
    }
    if (local) atomicOr(flags, local);
}

template <class T>
int launch_correct(const GridDev& g, const double* p, double dt, T* u, T* v, T* w, int* flags,
                   cudaStream_t s) {
    long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    k_correct<T><<<ew_blocks(total), EW_THREADS, 0, s>>>(g, p, dt, u, v, w, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

// ------------------------------------------------------------ fused epilogue
template <class T>
__global__ void __launch_bounds__(EW_THREADS) k_correct_divergence(GridDev g, const double* __restrict__ p, double dt,
                                                                   const T* __restrict__ iu, const T* __restrict__ iv,
                                                                   const T* __restrict__ iw, T* __restrict__ ou,
                                                                   T* __restrict__ ov, T* __restrict__ ow,
                                                                   Partials part, double* out_scalars, int* flags) {
    correct_divergence_body<T>(g, p, dt, iu, iv, iw, ou, ov, ow, part, out_scalars, flags, whole_launch());
}

template <class T>
int launch_correct_divergence(const GridDev& g, const double* p, double dt, const T* const in[3],
                              T* const out[3], Partials part, int nblocks_cap, double* out_scalars,
                              int* flags, cudaStream_t s) {
    int nb = ew_blocks(g.cells);
    if (nb > nblocks_cap) nb = nblocks_cap;
    k_correct_divergence<T><<<nb, EW_THREADS, 0, s>>>(g, p, dt, in[0], in[1], in[2], out[0], out[1],
                                                      out[2], part, out_scalars, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

template <class T>
__global__ void __launch_bounds__(EW_THREADS) k_face_maxima(GridDev g, const T* __restrict__ u,
                                                            const T* __restrict__ v, const T* __restrict__ w,
                                                            Partials part, double* out_scalars, int* flags) {
    __shared__ BlockReduce<0, 3> sm;
    double mx[3] = {0.0, 0.0, 0.0};
    int local = 0;
    const T* f3[3] = {u, v, w};
#pragma unroll
    for (int a = 0; a < 3; ++a)
        for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.flen[a]; f += gridDim.x * blockDim.x) {
            double x = double(f3[a][f]);
            if (!isfinite(x)) local |= VF_NONFINITE;
            mx[a] = fmax(mx[a], fabs(x));
        }
    if (local) atomicOr(flags, local);
    dd none[1];
    block_reduce<0, 3>(sm, none, mx);
    if (publish_and_check_last<0, 3>(part, blockIdx.x, gridDim.x, none, mx)) {
        fold_partials<0, 3>(part, gridDim.x, sm, none, mx);
        if (threadIdx.x == 0)
            for (int q = 0; q < 3; ++q) out_scalars[q] = mx[q];
    }
}

template <class T>
int launch_face_maxima(const GridDev& g, const T* u, const T* v, const T* w, Partials part,
                       int nblocks_cap, double* out_scalars, int* flags, cudaStream_t s) {
    int nb = ew_blocks(g.flen[0]);
    if (nb > nblocks_cap) nb = nblocks_cap;
    k_face_maxima<T><<<nb, EW_THREADS, 0, s>>>(g, u, v, w, part, out_scalars, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

// The momentum witness of a supplied projection
// (composition/projection.rs:515-542): each face of the supplied velocity must
// equal, bit for bit, the input velocity corrected with the supplied pressure
// (walls unchanged). The lowest mismatching face index of each axis is kept.
template <class T>
__global__ void k_projection_witness(GridDev g, const double* __restrict__ p, double dt, const T* __restrict__ iu,
                                     const T* __restrict__ iv, const T* __restrict__ iw, const T* __restrict__ su,
                                     const T* __restrict__ sv, const T* __restrict__ sw,
                                     unsigned long long* __restrict__ first) {
    const long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    const int s[3] = {1, g.n[0], g.n[0] * g.n[1]};
    int local = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int a = 0;
        long long f = t;
        if (f >= g.flen[0]) {
            f -= g.flen[0];
            a = 1;
            if (f >= g.flen[1]) {
                f -= g.flen[1];
                a = 2;
            }
        }
        const T* in = a == 0 ? iu : (a == 1 ? iv : iw);
        const T* sup = a == 0 ? su : (a == 1 ? sv : sw);
        int fi = int(f % g.fc[a][0]);
        int fj = int((f / g.fc[a][0]) % g.fc[a][1]);
        int fk = int(f / ((long long)g.fc[a][0] * g.fc[a][1]));
        T expect = in[f];
        if (!is_wall_face(g, a, fi, fj, fk)) {
            const int c = cell_idx(g, fi, fj, fk);
            expect = corrected<T>(g, a, expect, p[c], p[c - s[a]], dt, local);
        }
        const T got = sup[f];
        bool same;
        if (sizeof(T) == 4)
            same = __float_as_uint(float(expect)) == __float_as_uint(float(got));
        else
            same = __double_as_longlong(double(expect)) == __double_as_longlong(double(got));
        if (!same) atomicMin(&first[a], (unsigned long long)f);
    }
}

template <class T>
int launch_projection_witness(const GridDev& g, const double* p, double dt, const T* const in[3],
                              const T* const sup[3], unsigned long long* first, cudaStream_t s) {
    const long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    k_projection_witness<T><<<ew_blocks(total), EW_THREADS, 0, s>>>(g, p, dt, in[0], in[1], in[2], sup[0], sup[1],
                                                                    sup[2], first);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

#define RB200_INSTANTIATE(T)                                                                        \
    template int launch_validate_faces<T>(const GridDev&, const T*, const T*, const T*, int*,       \
                                          cudaStream_t);                                            \
    template int launch_build_rhs<T>(const GridDev&, const T*, const T*, const T*, double, double*, \
                                     int*, cudaStream_t);                                           \
    template int launch_divergence<T>(const GridDev&, const T*, const T*, const T*, double*, int*,  \
                                      cudaStream_t);                                                \
    template int launch_correct<T>(const GridDev&, const double*, double, T*, T*, T*, int*,         \
                                   cudaStream_t);                                                   \
    template int launch_correct_divergence<T>(const GridDev&, const double*, double,                \
                                              const T* const[3], T* const[3], Partials, int,        \
                                              double*, int*, cudaStream_t);                         \
    template int launch_face_maxima<T>(const GridDev&, const T*, const T*, const T*, Partials, int, \
                                       double*, int*, cudaStream_t);                                \
    template int launch_projection_witness<T>(const GridDev&, const double*, double, const T* const[3], \
                                              const T* const[3], unsigned long long*, cudaStream_t);
RB200_INSTANTIATE(float)
RB200_INSTANTIATE(double)
#undef RB200_INSTANTIATE

}  // namespace rb200
