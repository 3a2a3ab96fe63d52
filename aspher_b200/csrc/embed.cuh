// Embedded grids: the caller's Nl x Nl field as the top-left block of the
// power-of-two Ns x Ns compute field (row pitch Nl outside, Ns inside).
// Scalar element accesses only: an odd Nl leaves caller rows at every
// alignment.
#pragma once

#include <cuda_runtime.h>

namespace asb {

// Gap value of the cells outside the caller's block in an embedded solve:
// never the minimum of v = S p + g0, never penetrating, and every product
// p * pad that a reduction forms is 0 * pad = 0.  Finite in FP32 with room
// for the identification step's trial z = p - s g (s a compliance scale).
constexpr double kEmbedPadGap = 1e20;

// dst (B compute fields) <- src (B caller fields), cells outside the block
// set to `pad`
template <typename Ts, typename Td>
__global__ void k_embed(int Nl, int Ns, int B, const Ts* __restrict__ src, Td* __restrict__ dst,
                        Td pad) {
    const long n = (long)Ns * Ns, nl = (long)Nl * Nl;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n * B;
         i += (long)gridDim.x * blockDim.x) {
        const long b = i / n, r = i - b * n;
        const int y = (int)(r / Ns), x = (int)(r - (long)y * Ns);
        dst[i] = (x < Nl && y < Nl) ? (Td)src[b * nl + (long)y * Nl + x] : pad;
    }
}

// dst (B caller fields) <- the blocks of src (B compute fields)
template <typename Ts, typename Td>
__global__ void k_extract(int Nl, int Ns, int B, const Ts* __restrict__ src,
                          Td* __restrict__ dst) {
    const long n = (long)Ns * Ns, nl = (long)Nl * Nl;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nl * B;
         i += (long)gridDim.x * blockDim.x) {
        const long b = i / nl, r = i - b * nl;
        const int y = (int)(r / Nl), x = (int)(r - (long)y * Nl);
        dst[i] = (Td)src[b * n + (long)y * Ns + x];
    }
}

// one compute field: v on the block, 0 outside
template <typename T>
__global__ void k_fill_block(int Nl, int Ns, T* __restrict__ x, T v) {
    const long n = (long)Ns * Ns;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int y = (int)(i / Ns), x0 = (int)(i - (long)y * Ns);
        x[i] = (x0 < Nl && y < Nl) ? v : T(0);
    }
}

inline int embed_grid(long n) {
    const long b = (n + 255) / 256;
    return (int)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace asb
