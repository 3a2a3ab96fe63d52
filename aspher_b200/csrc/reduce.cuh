// Deterministic grid reductions: every block reduces its values with a fixed
// warp tree, writes them to `partials`, and the last block to finish (an
// atomic ticket) sums the partials in block order.  For a fixed grid the
// result is bitwise reproducible run to run.
#pragma once

#include "common.cuh"

namespace asb {

constexpr int kRedThreads = 256;
// the vector passes run kMaxBlocks / 2 = 4 x 148 blocks: with at most 64
// registers per thread all of them are resident at once (one wave)
constexpr int kRedMinBlocks = 4;
// upper bound on the grid of the vector-pass reducing kernels
constexpr int kMaxBlocks = 1184;
// partials per instance of a batched solve: 8 values for the largest grid of
// any reducing kernel -- the row kernels of an 8192-row transform run up to
// 8192 blocks (reductions fused into their stores)
constexpr int kMaxRowBlocks = 8192;
constexpr int kPartStride = kMaxRowBlocks * 8;

template <int NV>
__device__ __forceinline__ void ident_init(double (&v)[NV], const int (&kinds)[NV]) {
#pragma unroll
    for (int i = 0; i < NV; ++i)
        v[i] = kinds[i] == 0 ? 0.0 : (kinds[i] == 1 ? (double)INFINITY : -(double)INFINITY);
}

__device__ __forceinline__ double red_op(int kind, double a, double b) {
    return kind == 0 ? a + b : (kind == 1 ? fmin(a, b) : fmax(a, b));
}

// Returns true in every thread of the last block; thread 0 of that block then
// holds the grid totals in v.  `counter` must be 0 at kernel start; the last
// block resets it.
template <int NV>
__device__ bool grid_reduce_last(double (&v)[NV], const int (&kinds)[NV], double* partials,
                                 unsigned* counter) {
    __shared__ double scratch[32 * NV];
    __shared__ bool am_last;
    block_reduce<NV>(v, kinds, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) partials[(size_t)blockIdx.x * NV + i] = v[i];
        __threadfence();
        const unsigned prev = atomicAdd(counter, 1u);
        am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double acc[NV];
    ident_init<NV>(acc, kinds);
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int i = 0; i < NV; ++i)
            acc[i] = red_op(kinds[i], acc[i], __ldcg(&partials[(size_t)b * NV + i]));
    }
    block_reduce<NV>(acc, kinds, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] = acc[i];
        *counter = 0u;
    }
    return true;
}

}  // namespace asb
