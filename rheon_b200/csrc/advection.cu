// Standalone semi-Lagrangian advection kernels (src/advection.rs); the device
// bodies are in advect.cuh.
#include "advect.cuh"

namespace rb200 {

template <class T, class R>
__global__ void __launch_bounds__(ADV_THREADS, 3) k_advect_velocity(GridDev g, Faces<T> vel, double dt, T* ou, T* ov, T* ow,
                                                                 const float* __restrict__ tracer, double gb,
                                                                 int* flags) {
    advect_velocity_body<T, R>(g, vel, dt, ou, ov, ow, tracer, gb, flags, whole_launch());
}

template <class T, class R>
__global__ void __launch_bounds__(ADV_THREADS) k_advect_tracer(GridDev g, const float* __restrict__ old, Faces<T> vel,
                                                               double dt, float* __restrict__ out, int* flags) {
    advect_tracer_body<T, R>(g, old, vel, dt, out, flags, whole_launch());
}

template <class T>
int launch_advect_velocity(const GridDev& g, const T* u, const T* v, const T* w, double dt, T* ou,
                           T* ov, T* ow, const float* tracer, double gb, int* flags, cudaStream_t s,
                           bool fp32_math) {
    long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    long long blocks = (total + ADV_THREADS - 1) / ADV_THREADS;
    if (blocks > 148 * 64) blocks = 148 * 64;
    Faces<T> vel{{u, v, w}};
    if (fp32_math)
        k_advect_velocity<T, float><<<int(blocks), ADV_THREADS, 0, s>>>(g, vel, dt, ou, ov, ow, tracer, gb, flags);
    else
        k_advect_velocity<T, double><<<int(blocks), ADV_THREADS, 0, s>>>(g, vel, dt, ou, ov, ow, tracer, gb, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

template <class T>
int launch_advect_tracer(const GridDev& g, const float* old, const T* u, const T* v, const T* w,
                         double dt, float* out, int* flags, cudaStream_t s, bool fp32_math) {
    long long blocks = ((long long)g.cells + ADV_THREADS - 1) / ADV_THREADS;
    if (blocks > 148 * 64) blocks = 148 * 64;
    Faces<T> vel{{u, v, w}};
    if (fp32_math)
        k_advect_tracer<T, float><<<int(blocks), ADV_THREADS, 0, s>>>(g, old, vel, dt, out, flags);
    else
        k_advect_tracer<T, double><<<int(blocks), ADV_THREADS, 0, s>>>(g, old, vel, dt, out, flags);
    RB200_CUDA(cudaGetLastError());
    return RB200_OK;
}

template int launch_advect_velocity<float>(const GridDev&, const float*, const float*, const float*,
                                           double, float*, float*, float*, const float*, double,
                                           int*, cudaStream_t, bool);
template int launch_advect_velocity<double>(const GridDev&, const double*, const double*,
                                            const double*, double, double*, double*, double*,
                                            const float*, double, int*, cudaStream_t, bool);
template int launch_advect_tracer<float>(const GridDev&, const float*, const float*, const float*,
                                         const float*, double, float*, int*, cudaStream_t, bool);
template int launch_advect_tracer<double>(const GridDev&, const float*, const double*,
                                          const double*, const double*, double, float*, int*,
                                          cudaStream_t, bool);

}  // namespace rb200
