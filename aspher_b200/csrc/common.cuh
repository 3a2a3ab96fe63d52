// Shared device helpers: complex arithmetic on float2/double2, error
// plumbing and deterministic block reductions.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

namespace asb {

// ---- complex vector types --------------------------------------------------
template <typename T> struct cvec;
template <> struct cvec<float> { using type = float2; };
template <> struct cvec<double> { using type = double2; };
template <typename T> using cplx = typename cvec<T>::type;

template <typename T>
__host__ __device__ __forceinline__ cplx<T> mk(T x, T y) {
    cplx<T> r; r.x = x; r.y = y; return r;
}
template <typename V>
__host__ __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V>
__host__ __device__ __forceinline__ V csub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename V>
__host__ __device__ __forceinline__ V cmul(V a, V b) {
    V r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename V>
__host__ __device__ __forceinline__ V cmulc(V a, V b) {
    V r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename V>
__host__ __device__ __forceinline__ V cconj(V a) { V r; r.x = a.x; r.y = -a.y; return r; }
template <typename V, typename S>
__host__ __device__ __forceinline__ V cscale(V a, S s) { V r; r.x = a.x * s; r.y = a.y * s; return r; }
// multiply by -i (forward) or +i (inverse): DIR = -1 forward, +1 inverse
template <int DIR, typename V>
__host__ __device__ __forceinline__ V mul_i(V a) {
    V r;
    if (DIR < 0) { r.x = a.y; r.y = -a.x; }   // * (-i)
    else         { r.x = -a.y; r.y = a.x; }   // * (+i)
    return r;
}

// ---- reductions ------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide reduction of NV doubles with a fixed tree (deterministic for a
// fixed blockDim). op: 0 = sum, 1 = min, 2 = max per slot (kinds[i]).
// Result valid in thread 0. scratch must hold 32*NV doubles.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], const int (&kinds)[NV],
                                             double* scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double x = v[i];
        x = kinds[i] == 0 ? warp_sum(x) : (kinds[i] == 1 ? warp_min(x) : warp_max(x));
        if (lane == 0) scratch[wid * NV + i] = x;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            const double id = kinds[i] == 0 ? 0.0 : (kinds[i] == 1 ? (double)INFINITY : -(double)INFINITY);
            double x = lane < nw ? scratch[lane * NV + i] : id;
            x = kinds[i] == 0 ? warp_sum(x) : (kinds[i] == 1 ? warp_min(x) : warp_max(x));
            v[i] = x;
        }
    }
    __syncthreads();
}

}  // namespace asb
