// Host-side launchers of the FFT pass kernels (fft_kernels.cuh): launch
// shape of variant V, dynamic shared memory (with the opt-in attribute set
// once per kernel and device), persistent grids for the staged forms, and
// gridDim.y = B instances.  Shared by the operators' translation units.
#pragma once

#include "fft_kernels.cuh"
#include "ops.hpp"

namespace asb {

// small sizes collapse to variant 0
__host__ __device__ constexpr int vclamp(int L, int V) { return L >= 128 ? V : 0; }

// max dynamic shared memory + max-shared carveout, once per kernel per device
void fft_attrs(const void* func, int bytes);
// CTAs of a persistent pass kernel: at most occupancy x SMs, at most `units`
int persistent_blocks(const void* func, int threads, int smem, int units);

// B > 1: gridDim.y = B instances (functors / gates / spectrum per instance)
template <typename T, int LR, bool PAD, int V, class Load, class Store>
void launch_row_fwd(Load ld, Store st, int nrows, cudaStream_t s, const int* gate, int B = 1) {
    constexpr int rb = row_rb_v<T>(LR, V), thr = row_threads<T>(LR, V);
    constexpr int sm = row_fwd_smem<T, LR, PAD, V, Load>();
    auto k = row_fwd_kernel<T, LR, PAD, V, Load, Store>;
    fft_attrs((const void*)k, sm);
    const int units = (nrows + rb - 1) / rb;
    const int gx = row_fwd_staged<T, LR, PAD, V, Load::kRaw>()
                       ? persistent_blocks((const void*)k, thr, sm, units) : units;
    k<<<dim3(gx, B), thr, sm, s>>>(ld, st, nrows, tw<T>(LR), tw<T>(2 * LR), gate);
}
template <typename T, int LR, bool PAD, int V, class Load, class Store>
void launch_row_inv(Load ld, Store st, int nrows, cudaStream_t s, const int* gate, int B = 1) {
    constexpr int rb = row_rb_v<T>(LR, V), thr = row_threads<T>(LR, V);
    constexpr int sm = row_inv_smem<T, LR, PAD, V, Load>();
    auto k = row_inv_kernel<T, LR, PAD, V, Load, Store>;
    fft_attrs((const void*)k, sm);
    const int units = (nrows + rb - 1) / rb;
    const int gx = row_inv_staged<T, LR, PAD, V, Load::kTiled>()
                       ? persistent_blocks((const void*)k, thr, sm, units) : units;
    k<<<dim3(gx, B), thr, sm, s>>>(ld, st, nrows, tw<T>(LR), tw<T>(2 * LR), gate);
}
template <typename T, int LC, int NCM1, bool PAD, int V, class Mult>
void launch_col(cplx<T>* spec, int nrows, Mult m, cudaStream_t s, const int* gate, int B = 1) {
    constexpr int ct = col_ct_v<T>(LC, NCM1, V), thr = col_threads<T>(LC, NCM1, V);
    constexpr int sm = col_smem_total<T, LC, NCM1, PAD, V>();
    auto k = col_kernel<T, LC, NCM1, PAD, V, Mult>;
    fft_attrs((const void*)k, sm);
    const int gx = col_staged<T, LC, NCM1, PAD, V>()
                       ? persistent_blocks((const void*)k, thr, sm, NCM1 / ct + 1)
                       : NCM1 / ct + 1;
    k<<<dim3(gx, B), thr, sm, s>>>(spec, nrows, m, tw<T>(LC), gate);
}


}  // namespace asb
