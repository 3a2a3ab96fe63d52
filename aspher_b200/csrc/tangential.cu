// Tangential (Cerruti) FFT operator: u = C q with q = [q_x; q_y] and
// u = [u_x; u_y] stacked (N = Ns^2 each, natural flat order iy*Ns + ix).
//
// Reference: TangentialFFTOperator (include/tangential_operator.hpp:32-57,
// src/tangential_operator.cpp:10-140) over CerrutiKernel
// (include/cerruti_kernel.hpp:35-61, src/cerruti_kernel.cpp:114-128).  The
// three influence tables -- xx (even in each axis), yy(dx, dy) = xx(dy, dx)
// and xy (odd in each axis, 0 on the axes) -- are embedded in wrap-around
// order on the (2Ns)^2 grid like the Love table of the free-space operator;
// each is even under joint negation, so all three spectra are real, and the
// apply is
//   U(k) = Kxx(k) Qx(k) + Kxy(k) Qy(k),   V(k) = Kxy(k) Qx(k) + Kyy(k) Qy(k).
//
// Device form.  Build (FP64): the xx and xy tables by a kernel
// (kernel_tables.cuh), their spectra by the same two real-row passes through
// a transposed buffer as the free-space Kh (each row of an even table
// transforms to a real row, of an odd table to an imaginary one; the part
// that must vanish is tracked and checked against 1e-10 of the kept one, as
// the reference checks max|Im| <= 1e-10 max|Re|), stored canonically for
// kx, ky in [0, Ns] (xx even and xy odd in ky); Kyy is the transpose of the
// canonical Kxx.  Apply: both fields' rows in one row_fwd launch
// (gridDim.y = 2), one column kernel that transforms a column of each field,
// mixes them through shared memory and transforms both back, both fields'
// rows in one row_inv launch: 3 launches, the spectrum of each field read
// and written once per pass.  q and u may alias (q is consumed by the first
// pass before u is written).
#include "../../include/aspher_b200.h"
#include "embed.cuh"
#include "fft_kernels.cuh"
#include "fft_launch.cuh"
#include "functors.cuh"
#include "kernel_tables.cuh"
#include "ops.hpp"
#include "reduce.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <string>
#include <vector>

namespace asb {
namespace {

// largest supported grid: a column pair of 2 Ns points per field in one
// CTA's shared memory for FP64 (and the FP32 form kept to the same sizes)
constexpr int kTanMaxNs = 2048;

__global__ void k_cerruti_tables(double* __restrict__ xx, double* __restrict__ xy, int Ns,
                                 double h, double pref, double prefnu, double nu) {
    const long n = (long)Ns * Ns;
    const double a = 0.5 * h;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int dy = (int)(i / Ns), dx = (int)(i % Ns);
        xx[i] = pref * cerruti_uxx_dev(dx * h, dy * h, a, a, nu);
        xy[i] = prefnu * cerruti_uxy_dev(dx * h, dy * h, a, a);
    }
}

// the table t[|dy| * Ns + |dx|] embedded in wrap-around order on the M x M
// grid (offset d >= 0 at d, d < 0 at M + d, row / column Ns zero); odd:
// the sign of an odd-in-each-axis table restored from the offsets' signs
struct LoadEmbeddedSigned {
    static constexpr bool kTiled = false;
    static constexpr bool kRaw = false;
    const double* tab;
    int Ns, M;
    int odd;
    __device__ __forceinline__ double at(int iy, int ix) const {
        if (iy == Ns || ix == Ns) return 0.0;
        const int dy = iy < Ns ? iy : iy - M;
        const int dx = ix < Ns ? ix : ix - M;
        const double v = tab[(size_t)(dy < 0 ? -dy : dy) * Ns + (dx < 0 ? -dx : dx)];
        return (odd && ((dx < 0) != (dy < 0))) ? -v : v;
    }
    __device__ __forceinline__ double2 operator()(int row, int n) const {
        return make_double2(at(row, 2 * n), at(row, 2 * n + 1));
    }
};

// Row-pass output of the spectrum build: the kept part of X (real for an even
// row, imaginary for an odd one; times `scale`) into the transposed buffer
// (pass A) or the canonical spectrum (pass B, times norm); the maxima of the
// discarded and the kept parts tracked for the realness check.
struct StorePartTracked {
    double* out_t;  // pass A: (Ns+1) x M, transposed
    int M;
    double* canon;  // pass B: canonical [ky][kx], kx, ky in [0, Ns]
    int nk;
    int imag;       // keep Im X (odd rows)
    double scale;   // norm (and sign) of the kept part
    unsigned long long* maxbits;  // [0] max |discarded|, [1] max |kept|
    static constexpr bool kFinish = true;
    static constexpr bool kTiled = false;
    mutable double md, mk;
    __device__ __forceinline__ void operator()(int row, int k, double2 X) const {
        const double keep = imag ? X.y : X.x, drop = imag ? X.x : X.y;
        if (out_t) out_t[(size_t)k * M + row] = keep * scale;
        else canon[(size_t)k * nk + row] = keep * scale;
        md = fmax(md, fabs(drop));
        mk = fmax(mk, fabs(keep));
    }
    __device__ void finish(double* scratch) const {
        double v[2] = {md, mk};
        const int kinds[2] = {2, 2};
        block_reduce<2>(v, kinds, scratch);
        if (threadIdx.x == 0) {
            atomicMax(&maxbits[0], (unsigned long long)__double_as_longlong(v[0]));
            atomicMax(&maxbits[1], (unsigned long long)__double_as_longlong(v[1]));
        }
    }
};

// The three spectra for the column kernel: K(kx, ky) at ky folded to
// kf <= Ns, tiled by the column-pass tile width ct: [kx/ct][kf][kx % ct]
// (a column's values contiguous for ct = 1); Kyy is the transpose of Kxx.
template <typename T>
__global__ void k_tan_retile(int Ns, int ncols, const double* __restrict__ cxx,
                             const double* __restrict__ cxy, int ct, T* __restrict__ kxx,
                             T* __restrict__ kyy, T* __restrict__ kxy) {
    const int nk = Ns + 1;
    const long n = (long)ncols * nk;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int kx = (int)(i / nk), kf = (int)(i % nk);
        const size_t at = (size_t)(kx / ct) * nk * ct + (size_t)kf * ct + (kx % ct);
        if (kx > Ns) {  // padding columns of the last tile
            kxx[at] = T(0);
            kyy[at] = T(0);
            kxy[at] = T(0);
            continue;
        }
        kxx[at] = (T)cxx[(size_t)kf * nk + kx];
        kyy[at] = (T)cxx[(size_t)kx * nk + kf];
        kxy[at] = (T)cxy[(size_t)kf * nk + kx];
    }
}

// columns per field of one column-pass CTA: both fields' columns (2 ct of
// them, interleaved in shared memory) in at most 512 threads and the
// shared memory of one CTA
template <typename T>
__host__ __device__ constexpr int tan_ct(int LC, int Ns) {
    const int tt = LC / col_rpt<T>(LC, 0);
    int ct = 16;
    while (ct > 1 && (2 * ct * tt > 512 || ct > Ns || col_smem<T>(LC, 2 * ct) > kSmemPerSM))
        ct >>= 1;
    return ct;
}

// two FFT workspaces of the column-pair kernel fit one CTA
template <typename T>
__host__ __device__ constexpr bool col_pair_pp(int LC, int CT) {
    return 2 * align16(col_smem<T>(LC, 2 * CT)) <= kSmemPerSM;
}

// Row-pass launch variant of the tangential apply (its rows are the free-
// space operator's zero-padded transforms, two fields as gridDim.y = 2),
// measured on B200 with the column-pair kernel: FP32 the free-space
// defaults (2048: 0.220 -> 0.210 ms per apply against variant 0, 256: 0.028
// -> 0.024 ms); FP64 variant 1 up to 512, else 0 (variant 2, the free-space
// default at 2048, took the two-field apply from 0.396 to 0.441 ms)
template <typename T>
__host__ __device__ constexpr int tan_row_variant(int Ns) {
    return vclamp(Ns, sizeof(T) == 4 ? (Ns <= 512 ? 2 : 1) : (Ns <= 512 ? 1 : 0));
}

template <typename T>
struct TanMix {
    const T* kxx;
    const T* kyy;
    const T* kxy;
    int nk, ct, M;
    // field f's output at (kx, ky) from its own forward transform a and the
    // other field's b: Kxx a + Kxy b (f = 0) or Kyy a + Kxy b (f = 1); the
    // field picks an array, not a branch (the two fields share warps)
    __device__ __forceinline__ cplx<T> operator()(int f, cplx<T> a, cplx<T> b, int kx,
                                                  int ky) const {
        const bool lo = ky <= (M >> 1);
        const int kf = lo ? ky : M - ky;
        const size_t at = (size_t)(kx / ct) * nk * ct + (size_t)kf * ct + (kx % ct);
        const T* own = f ? kyy : kxx;
        const T xy = __ldg(&kxy[at]);
        const T wxy = lo ? xy : -xy;  // odd in ky
        const T w = __ldg(&own[at]);
        return mk<T>(w * a.x + wxy * b.x, w * a.y + wxy * b.y);
    }
};

// Column pass of both fields: CT columns of each field per CTA (interleaved
// as 2 CT transforms: field c / CT, column c % CT); per column the pruned
// forward transform (upper half zero), the 2x2 mix with the other field's
// column through shared memory, the inverse transform keeping rows < Ns.
template <typename T, int LC, int CT>
__global__ void __launch_bounds__(2 * CT * (LC / col_rpt<T>(LC, 0)))
col_pair_kernel(cplx<T>* __restrict__ spec, long bsp, int nrows, TanMix<T> mix,
                const cplx<T>* __restrict__ tw_lc) {
    constexpr int RPT = col_rpt<T>(LC, 0);
    constexpr int TT = LC / RPT;
    constexpr int S = 2 * CT;
    // second FFT workspace (elements from sm) where two fit one CTA, else 0:
    // the round trips alternate between them (one barrier each), and the
    // exchange of the two fields' spectra uses the one the forward
    // transform's last round trip did not read
    constexpr int ALT = col_pair_pp<T>(LC, CT) ? align16(col_smem<T>(LC, S)) / (int)sizeof(cplx<T>)
                                               : 0;
    constexpr int PX = ALT ? ping_pong_next<LC, RPT>(0) : 0;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* xs = sm + (PX ? ALT : 0);
    const int c = threadIdx.x % S, t = threadIdx.x / S;
    const int f = c / CT, cc = c % CT;
    const int tile = blockIdx.x;
    cplx<T>* base = spec + f * bsp + (size_t)tile * nrows * CT;
    cplx<T> v[RPT];
#pragma unroll
    for (int m = 0; m < RPT; ++m)
        v[m] = m >= RPT / 2 ? mk<T>(0, 0) : base[(size_t)(t + m * TT) * CT + cc];
    block_fft<T, LC, RPT, -1, S, true, ALT>(v, t, sm, c, tw_lc);
    // every thread publishes its column's spectrum, then reads the other
    // field's column at the same kx (the forward transform's last stage ran
    // in registers; with one workspace, after every thread's last read of it)
    if constexpr (ALT == 0) __syncthreads();
#pragma unroll
    for (int m = 0; m < RPT; ++m) xs[smaddr(t + m * TT, S, c)] = v[m];
    __syncthreads();
    const int pc = f ? c - CT : c + CT;
    const int kx = tile * CT + cc;
#pragma unroll
    for (int m = 0; m < RPT; ++m) {
        const int ky = t + m * TT;
        v[m] = mix(f, v[m], xs[smaddr(ky, S, pc)], kx, ky);
    }
    // one workspace: reused by the inverse transform; two: the inverse
    // starts in the other one and reaches xs after its first barrier
    if constexpr (ALT == 0) __syncthreads();
    block_fft<T, LC, RPT, +1, S, false, ALT, ALT ? (PX ^ 1) : 0>(v, t, sm, c, tw_lc);
#pragma unroll
    for (int m = 0; m < RPT / 2; ++m) base[(size_t)(t + m * TT) * CT + cc] = v[m];
}

}  // namespace

struct TanOperator {
    // Ns: the compute grid (a power of two in [16, 2048]); Nl: the caller's
    // side.  Nl < Ns (a side that is not a power of two >= 16) runs
    // embedded: the caller's cells are the top-left block of the compute
    // grid, the Cerruti tables at the caller's cell size L / Nl, so the
    // padded convolution of a field that is zero outside the block is the
    // tangential operator of the Nl grid on the block
    int Ns = 0, Nl = 0;
    double L = 1.0, E = 1.0, nu = 0.3;
    bool embedded() const { return Nl != Ns; }
    // embedded: two-field compute-grid scratch of the caller-facing apply
    void* emb_q = nullptr;
    void* emb_u = nullptr;
    // caller-facing apply: q, u hold 2 Nl^2 values
    void apply_caller(bool dbl, const void* q, void* u, cudaStream_t s);
    int device = 0;
    double max_im_ratio = 0.0;
    double* tab_xx = nullptr;  // FP64 tables [dy][dx], dx, dy in [0, Ns)
    double* tab_xy = nullptr;
    // tiled spectra per precision: [0] FP32, [1] FP64; each 3 arrays
    void* kt[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int ct[2] = {1, 1};
    void* spec[2] = {nullptr, nullptr};  // two fields' half spectra per precision

    TanOperator(int Ns_, double L_, double E_, double nu_);
    ~TanOperator() { release(); }
    void release();
    void matvec(bool dbl, const void* q, void* u, cudaStream_t s);

    template <typename T, int NS>
    void apply(const T* q, T* u, cudaStream_t s);
    template <int NS>
    void build();
};

template <int NS>
void TanOperator::build() {
    constexpr int LR = NS, M = 2 * NS;
    const size_t nk = (size_t)NS + 1;
    double *cxx = nullptr, *cxy = nullptr, *yt = nullptr;
    unsigned long long* mx = nullptr;
    ASB_CUDA(cudaMalloc(&cxx, nk * nk * sizeof(double)));
    ASB_CUDA(cudaMalloc(&cxy, nk * nk * sizeof(double)));
    ASB_CUDA(cudaMalloc(&yt, nk * M * sizeof(double)));
    ASB_CUDA(cudaMalloc(&mx, 8 * sizeof(unsigned long long)));
    ASB_CUDA(cudaMemset(mx, 0, 8 * sizeof(unsigned long long)));
    const double norm = 1.0 / ((double)M * (double)M);
    for (int odd = 0; odd < 2; ++odd) {
        const LoadEmbeddedSigned emb{odd ? tab_xy : tab_xx, NS, M, odd};
        unsigned long long* mb = mx + 4 * odd;
        // pass A: rows of the embedded table -> transposed (real part of an
        // even row, imaginary part of an odd one)
        StorePartTracked sa{yt, M, nullptr, 0, odd, 1.0, mb, 0.0, 0.0};
        launch_row_fwd<double, LR, false, 0>(emb, sa, M, nullptr, nullptr);
        // pass B: rows of the transposed buffer; for the odd table the two
        // imaginary factors give K = -Im(X_B)
        StorePartTracked sb{nullptr, M, odd ? cxy : cxx, (int)nk, odd, odd ? -norm : norm,
                            mb + 2, 0.0, 0.0};
        launch_row_fwd<double, LR, false, 0>(LoadRealRows<double>{yt, M, 0}, sb, NS + 1, nullptr,
                                             nullptr);
        ASB_CUDA(cudaGetLastError());
    }
    unsigned long long h[8];
    ASB_CUDA(cudaMemcpy(h, mx, sizeof(h), cudaMemcpyDeviceToHost));
    double v[8];
    for (int i = 0; i < 8; ++i) std::memcpy(&v[i], &h[i], sizeof(double));
    max_im_ratio = 0.0;
    bool broken = false;
    for (int i = 0; i < 8; i += 2) {
        const double r = v[i + 1] > 0 ? v[i] / v[i + 1] : 0.0;
        max_im_ratio = r > max_im_ratio ? r : max_im_ratio;
        broken = broken || v[i] > 1e-10 * v[i + 1];
    }
    ASB_CUDA(cudaFree(yt));
    ASB_CUDA(cudaFree(mx));
    if (broken) {
        cudaFree(cxx);
        cudaFree(cxy);
        throw Error(ASPHER_EBUILD, "TangentialFFTOperator: spectrum parity broken "
                                   "(wrap-around embedding)");
    }
    // tiled copies per precision, for the column pass's tile width
    ct[0] = tan_ct<float>(2 * NS, NS);
    ct[1] = tan_ct<double>(2 * NS, NS);
    for (int dbl = 0; dbl < 2; ++dbl) {
        const int c = ct[dbl];
        const int ncols = (NS / c + 1) * c;
        const size_t es = dbl ? sizeof(double) : sizeof(float);
        for (int j = 0; j < 3; ++j) ASB_CUDA(cudaMalloc(&kt[dbl][j], (size_t)ncols * nk * es));
        if (dbl)
            k_tan_retile<double><<<592, 256>>>(NS, ncols, cxx, cxy, c, (double*)kt[1][0],
                                               (double*)kt[1][1], (double*)kt[1][2]);
        else
            k_tan_retile<float><<<592, 256>>>(NS, ncols, cxx, cxy, c, (float*)kt[0][0],
                                              (float*)kt[0][1], (float*)kt[0][2]);
        ASB_CUDA(cudaGetLastError());
        const size_t bsp = (size_t)(LR / c + 1) * NS * c;
        ASB_CUDA(cudaMalloc(&spec[dbl], 2 * bsp * (dbl ? sizeof(double2) : sizeof(float2))));
    }
    ASB_CUDA(cudaDeviceSynchronize());
    ASB_CUDA(cudaFree(cxx));
    ASB_CUDA(cudaFree(cxy));
}

#define ASB_TAN_SIZE_SWITCH(NSV, ...)                                       \
    switch (NSV) {                                                          \
        case 16: { constexpr int NS = 16; __VA_ARGS__; } break;             \
        case 32: { constexpr int NS = 32; __VA_ARGS__; } break;             \
        case 64: { constexpr int NS = 64; __VA_ARGS__; } break;             \
        case 128: { constexpr int NS = 128; __VA_ARGS__; } break;           \
        case 256: { constexpr int NS = 256; __VA_ARGS__; } break;           \
        case 512: { constexpr int NS = 512; __VA_ARGS__; } break;           \
        case 1024: { constexpr int NS = 1024; __VA_ARGS__; } break;         \
        case 2048: { constexpr int NS = 2048; __VA_ARGS__; } break;         \
        default: throw Error(ASPHER_EINVAL, "tangential operator: grid_size must be a power of " \
                                            "two in [16, 2048]");           \
    }

TanOperator::TanOperator(int Ns_, double L_, double E_, double nu_)
    : Ns(Ns_), Nl(Ns_), L(L_), E(E_), nu(nu_) {
    if (Nl < 2 || Nl > kTanMaxNs)
        throw Error(ASPHER_EINVAL, "tangential operator: grid_size must be in [2, 2048]");
    if (!is_pow2(Nl) || Nl < 16) {  // embedded in the next power of two
        int nc = 16;
        while (nc < Nl) nc *= 2;
        Ns = nc;
    }
    if (!(L > 0.0) || !std::isfinite(L)) throw Error(ASPHER_EINVAL, "domain_size must be positive");
    if (!(E > 0.0) || !std::isfinite(E)) throw Error(ASPHER_EINVAL, "E_star must be positive");
    if (!(nu >= 0.0 && nu < 1.0)) throw Error(ASPHER_EINVAL, "nu must be in [0, 1)");
    std::lock_guard<std::recursive_mutex> setup(setup_mutex());
    ASB_CUDA(cudaGetDevice(&device));
    (void)tw_table(false, 2);
    const size_t n = (size_t)Ns * Ns;
    try {
        ASB_CUDA(cudaMalloc(&tab_xx, n * sizeof(double)));
        ASB_CUDA(cudaMalloc(&tab_xy, n * sizeof(double)));
        // CerrutiKernel (cerruti_kernel.cpp:114-128): h = L / Ns, a = h / 2,
        // prefactors 1 / (pi E* (1 - nu)) and nu times it (h = L / Nl: the
        // caller's cell size; tables for offsets up to the compute grid)
        const double h = L / Nl, pref = 1.0 / (M_PI * E * (1.0 - nu));
        k_cerruti_tables<<<592, 256>>>(tab_xx, tab_xy, Ns, h, pref, nu * pref, nu);
        ASB_CUDA(cudaGetLastError());
        ASB_TAN_SIZE_SWITCH(Ns, build<NS>());
    } catch (...) {
        release();
        throw;
    }
}

void TanOperator::release() {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    cudaFree(tab_xx);
    cudaFree(tab_xy);
    tab_xx = tab_xy = nullptr;
    cudaFree(emb_q);
    cudaFree(emb_u);
    emb_q = emb_u = nullptr;
    for (int d = 0; d < 2; ++d) {
        for (int j = 0; j < 3; ++j) {
            cudaFree(kt[d][j]);
            kt[d][j] = nullptr;
        }
        cudaFree(spec[d]);
        spec[d] = nullptr;
    }
    if (cur != device) cudaSetDevice(cur);
}

template <typename T, int NS>
void TanOperator::apply(const T* q, T* u, cudaStream_t s) {
    constexpr int LR = NS, LC = 2 * NS;
    constexpr int CT = tan_ct<T>(LC, NS);
    const int dbl = sizeof(T) == 8;
    const long N = (long)NS * NS;
    const long bsp = (long)(LR / CT + 1) * NS * CT;
    cplx<T>* sp = static_cast<cplx<T>*>(spec[dbl]);
    // both fields' rows (instances 0 = q_x, 1 = q_y)
    constexpr int RV = tan_row_variant<T>(NS);
    launch_row_fwd<T, LR, true, RV>(LoadRealRows<T>{q, NS, N}, StoreTiled<T>{sp, NS, CT, bsp}, NS,
                                   s, nullptr, 2);
    {
        constexpr int thr = 2 * CT * (LC / col_rpt<T>(LC, 0));
        constexpr int sm = col_pair_pp<T>(LC, CT) ? 2 * align16(col_smem<T>(LC, 2 * CT))
                                                  : col_smem<T>(LC, 2 * CT);
        auto k = col_pair_kernel<T, LC, CT>;
        fft_attrs((const void*)k, sm);
        const TanMix<T> mix{static_cast<const T*>(kt[dbl][0]), static_cast<const T*>(kt[dbl][1]),
                            static_cast<const T*>(kt[dbl][2]), NS + 1, CT, LC};
        k<<<NS / CT + 1, thr, sm, s>>>(sp, bsp, NS, mix, tw<T>(LC));
    }
    launch_row_inv<T, LR, true, RV>(LoadTiled<T>{sp, NS, CT, bsp}, StoreRealRows<T>{u, NS, N}, NS,
                                   s, nullptr, 2);
    count_launches(3);
    ASB_CUDA(cudaGetLastError());
}

void TanOperator::matvec(bool dbl, const void* q, void* u, cudaStream_t s) {
    if (dbl) {
        ASB_TAN_SIZE_SWITCH(Ns, (apply<double, NS>((const double*)q, (double*)u, s)));
    } else {
        ASB_TAN_SIZE_SWITCH(Ns, (apply<float, NS>((const float*)q, (float*)u, s)));
    }
}

void TanOperator::apply_caller(bool dbl, const void* q, void* u, cudaStream_t s) {
    if (!embedded()) {
        matvec(dbl, q, u, s);
        return;
    }
    const long n = (long)Ns * Ns, nl = (long)Nl * Nl;
    if (!emb_q) {
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        ASB_CUDA(cudaMalloc(&emb_q, 2 * n * sizeof(double)));
        ASB_CUDA(cudaMalloc(&emb_u, 2 * n * sizeof(double)));
    }
    if (dbl) {
        k_embed<double, double><<<embed_grid(2 * n), 256, 0, s>>>(Nl, Ns, 2, (const double*)q,
                                                                  (double*)emb_q, 0.0);
        matvec(true, emb_q, emb_u, s);
        k_extract<double, double><<<embed_grid(2 * nl), 256, 0, s>>>(Nl, Ns, 2,
                                                                     (const double*)emb_u,
                                                                     (double*)u);
    } else {
        k_embed<float, float><<<embed_grid(2 * n), 256, 0, s>>>(Nl, Ns, 2, (const float*)q,
                                                                (float*)emb_q, 0.0f);
        matvec(false, emb_q, emb_u, s);
        k_extract<float, float><<<embed_grid(2 * nl), 256, 0, s>>>(Nl, Ns, 2,
                                                                   (const float*)emb_u, (float*)u);
    }
    count_launches(2);
    ASB_CUDA(cudaGetLastError());
}

}  // namespace asb

// ============================================================================
// Tangential projected CG (reference: src/friction_solve.cpp:1-688,
// include/friction_solve.hpp:14-109): the vector Polonsky-Keer iteration for
//   min 1/2 q'C q - sum_i q_i . delta    s.t. |q_i| <= s_i   (displacement)
// with the two-metric projection (the outward-radial part of the direction
// dropped at bound points), the beta restart on stick / slip partition
// changes, best-iterate tracking and the steepest-descent fallback; force
// control mean(q) = q_bar by the reference's outer Newton / Broyden
// iteration on the rigid shift with the terminal exact-load correction; the
// local KKT check on the returned state.  Double precision (as the
// reference: double-only), unpreconditioned.  The vector passes run on the
// device with deterministic FP64 reductions (per-block partials summed in a
// fixed order by one block); the scalar control flow of each iteration runs
// on the host, as in the reference.
// ============================================================================
namespace asb {
namespace {

constexpr int kTanThreads = 256;
constexpr int kTanMaxBlocks = 512;

__device__ __forceinline__ bool tan_interior(double qx, double qy, double si) {
    return hypot(qx, qy) < si * (1.0 - 1e-9);  // friction_solve.cpp:13-15
}

// block partials of NV values (kinds: 0 sum, 1 max) -> part[blockIdx.x * NV + j]
template <int NV>
__device__ __forceinline__ void tan_block_out(double (&v)[NV], const int (&kind)[NV],
                                              double* part) {
    __shared__ double sh[NV][kTanThreads / 32];
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double a = v[j];
        for (int o = 16; o > 0; o >>= 1) {
            const double b = __shfl_down_sync(0xffffffffu, a, o);
            a = kind[j] ? fmax(a, b) : a + b;
        }
        if ((threadIdx.x & 31) == 0) sh[j][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double a = sh[j][0];
            for (int w = 1; w < kTanThreads / 32; ++w) a = kind[j] ? fmax(a, sh[j][w]) : a + sh[j][w];
            part[blockIdx.x * NV + j] = a;
        }
    }
}

// one block: out[j] = fold of part[b * nv + j] over b in block order
struct TanKinds {  // per value: 0 sum, 1 max
    int k[8];
};
__global__ void k_tan_fold(const double* __restrict__ part, int nb, int nv, TanKinds kinds,
                           double* __restrict__ out) {
    const int j = threadIdx.x;
    if (j >= nv) return;
    const int kind = kinds.k[j];
    double a = kind ? -INFINITY : 0.0;
    for (int b = 0; b < nb; ++b) {
        const double x = part[b * nv + j];
        a = kind ? fmax(a, x) : a + x;
    }
    out[j] = a;
}

#define TAN_LOOP(N) \
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (N); i += (long)gridDim.x * blockDim.x)

// initial iterate: q_init clamped to the disks and zeroed off A, or 0
__global__ void k_tan_start(long N, const double* __restrict__ s, const double* __restrict__ q0,
                            double* __restrict__ q) {
    TAN_LOOP(N) {
        double qx = q0 ? q0[i] : 0.0, qy = q0 ? q0[N + i] : 0.0;
        const double si = s[i];
        if (!(si > 0.0)) {
            qx = qy = 0.0;
        } else {
            const double qn = hypot(qx, qy);
            if (qn > si) {
                const double f = si / qn;
                qx *= f;
                qy *= f;
            }
        }
        q[i] = qx;
        q[N + i] = qy;
    }
}

// residual g = u + u_hist - delta on A and the KKT stationarity error
// (friction_solve.cpp:93-125): [0] e, [1] max |g|
// The per-iteration scalars of the loop kernels live in device memory (a
// TanScalars record) so that the kernel sequences of an iteration can be
// captured once and replayed as CUDA graphs.
struct TanScalars {
    double beta;    // conjugate-direction weight (k_tan_tupd)
    double tau;     // step (k_tan_qupd)
    double skip;    // nonzero: k_tan_qupd leaves q unchanged
    double dx, dy;  // the imposed shift (k_tan_eval)
};

// residual g = u + u_hist - delta on A and the KKT stationarity error
// (friction_solve.cpp:93-125): [0] e, [1] max |g|
__global__ void __launch_bounds__(kTanThreads) k_tan_eval(
    long N, const double* __restrict__ s, const double* __restrict__ q,
    const double* __restrict__ u, const double* __restrict__ hist,
    const TanScalars* __restrict__ sc, double* __restrict__ g, double* part) {
    const double dx = sc->dx, dy = sc->dy;
    double v[2] = {0.0, 0.0};
    TAN_LOOP(N) {
        const double si = s[i];
        if (!(si > 0.0)) {
            g[i] = 0.0;
            g[N + i] = 0.0;
            continue;
        }
        const double gx = u[i] + (hist ? hist[i] : 0.0) - dx;
        const double gy = u[N + i] + (hist ? hist[N + i] : 0.0) - dy;
        g[i] = gx;
        g[N + i] = gy;
        const double gn = hypot(gx, gy);
        v[1] = fmax(v[1], gn);
        const double qx = q[i], qy = q[N + i];
        const double qn = hypot(qx, qy);
        if (tan_interior(qx, qy, si)) {
            v[0] += (si - qn) * gn;
        } else {
            const double hx = qx / qn, hy = qy / qn;
            const double gpar = gx * hx + gy * hy;
            v[0] += si * (hypot(gx - gpar * hx, gy - gpar * hy) + fmax(0.0, gpar));
        }
    }
    const int kind[2] = {0, 1};
    tan_block_out<2>(v, kind, part);
}

// direction source z = chi_A g with the bound points' negative radial part
// dropped (two-metric projection, friction_solve.cpp:74-90) and the dots
// [0] G = sum z.g, [1] G_pr = sum z.(g - g_prev) (friction_solve.cpp:212-221)
__global__ void __launch_bounds__(kTanThreads) k_tan_dir(
    long N, const double* __restrict__ s, const double* __restrict__ q,
    const double* __restrict__ g, const double* __restrict__ gp, double* __restrict__ z,
    double* part) {
    double v[2] = {0.0, 0.0};
    TAN_LOOP(N) {
        const double si = s[i];
        if (!(si > 0.0)) {
            z[i] = 0.0;
            z[N + i] = 0.0;
            continue;
        }
        double zx = g[i], zy = g[N + i];
        const double qx = q[i], qy = q[N + i];
        if (!tan_interior(qx, qy, si)) {
            const double qn = hypot(qx, qy);
            const double hx = qx / qn, hy = qy / qn;
            const double zpar = zx * hx + zy * hy;
            if (zpar < 0.0) {
                zx -= zpar * hx;
                zy -= zpar * hy;
            }
        }
        z[i] = zx;
        z[N + i] = zy;
        v[0] += zx * g[i] + zy * g[N + i];
        v[1] += zx * (g[i] - gp[i]) + zy * (g[N + i] - gp[N + i]);
    }
    const int kind[2] = {0, 0};
    tan_block_out<2>(v, kind, part);
}

// t = chi_A (z + beta t)
__global__ void k_tan_tupd(long N, const double* __restrict__ s, const double* __restrict__ z,
                           const TanScalars* __restrict__ sc, double* __restrict__ t) {
    const double beta = sc->beta;
    TAN_LOOP(N) {
        const bool a = s[i] > 0.0;
        t[i] = a ? z[i] + beta * t[i] : 0.0;
        t[N + i] = a ? z[N + i] + beta * t[N + i] : 0.0;
    }
}

// [0] num = sum_A g.t, [1] den = sum_A r.t (friction_solve.cpp:234-241)
__global__ void __launch_bounds__(kTanThreads) k_tan_numden(
    long N, const double* __restrict__ s, const double* __restrict__ g,
    const double* __restrict__ t, const double* __restrict__ r, double* part) {
    double v[2] = {0.0, 0.0};
    TAN_LOOP(N) {
        if (!(s[i] > 0.0)) continue;
        v[0] += g[i] * t[i] + g[N + i] * t[N + i];
        v[1] += r[i] * t[i] + r[N + i] * t[N + i];
    }
    const int kind[2] = {0, 0};
    tan_block_out<2>(v, kind, part);
}

// q <- clamp(q - tau t) on A; [0] partition changed (max)
// (friction_solve.cpp:258-276)
__global__ void __launch_bounds__(kTanThreads) k_tan_qupd(
    long N, const double* __restrict__ s, const double* __restrict__ t,
    const TanScalars* __restrict__ sc, double* __restrict__ q, double* part) {
    if (sc->skip != 0.0) return;  // no update this iteration (partials unused)
    const double tau = sc->tau;
    double v[1] = {0.0};
    TAN_LOOP(N) {
        const double si = s[i];
        if (!(si > 0.0)) continue;
        const bool was = tan_interior(q[i], q[N + i], si);
        double qx = q[i] - tau * t[i], qy = q[N + i] - tau * t[N + i];
        const double qn = hypot(qx, qy);
        const bool clamp = qn > si;
        if (clamp) {
            const double f = si / qn;
            qx *= f;
            qy *= f;
        }
        q[i] = qx;
        q[N + i] = qy;
        const bool is = !clamp && tan_interior(qx, qy, si);
        if (was != is) v[0] = 1.0;
    }
    const int kind[1] = {1};
    tan_block_out<1>(v, kind, part);
}

// [0] sum qx, [1] sum qy, [2] stick, [3] slip, [4] open (friction_solve.cpp:285-303)
__global__ void __launch_bounds__(kTanThreads) k_tan_classify(
    long N, const double* __restrict__ s, const double* __restrict__ q, double* part) {
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    TAN_LOOP(N) {
        v[0] += q[i];
        v[1] += q[N + i];
        const double si = s[i];
        if (!(si > 0.0)) v[4] += 1.0;
        else if (tan_interior(q[i], q[N + i], si)) v[2] += 1.0;
        else v[3] += 1.0;
    }
    const int kind[5] = {0, 0, 0, 0, 0};
    tan_block_out<5>(v, kind, part);
}

// local KKT quantities (friction_solve.cpp:316-370): [0] cone, [1] stick,
// [2] slip, [3] proj (max), [4] sum qx, [5] sum qy
__global__ void __launch_bounds__(kTanThreads) k_tan_kkt(
    long N, const double* __restrict__ s, const double* __restrict__ q,
    const double* __restrict__ u, const double* __restrict__ hist, double dx, double dy,
    double rho, double s_ref, double w_ref, double* part) {
    double v[6] = {-INFINITY, 0.0, 0.0, 0.0, 0.0, 0.0};
    TAN_LOOP(N) {
        const double qx = q[i], qy = q[N + i];
        v[4] += qx;
        v[5] += qy;
        const double si = s[i];
        const double qn = hypot(qx, qy);
        if (si <= 0.0) {
            v[0] = fmax(v[0], qn / s_ref);
            continue;
        }
        v[0] = fmax(v[0], (qn - si) / s_ref);
        const double gx = u[i] + (hist ? hist[i] : 0.0) - dx;
        const double gy = u[N + i] + (hist ? hist[N + i] : 0.0) - dy;
        const double zx = qx - rho * gx, zy = qy - rho * gy;
        const double zn = hypot(zx, zy);
        const double f = (zn > si && zn > 0.0) ? si / zn : 1.0;
        v[3] = fmax(v[3], hypot(qx - f * zx, qy - f * zy) / s_ref);
        const double wx = -gx, wy = -gy;
        if (tan_interior(qx, qy, si)) {
            v[1] = fmax(v[1], hypot(wx, wy) / w_ref);
        } else {
            const double hx = qx / qn, hy = qy / qn;
            const double wpar = wx * hx + wy * hy;
            v[2] = fmax(v[2], (hypot(wx - wpar * hx, wy - wpar * hy) + fmax(0.0, -wpar)) / w_ref);
        }
    }
    const int kind[6] = {1, 1, 1, 1, 0, 0};
    tan_block_out<6>(v, kind, part);
}

// [0] max s, [1] max |u_x| over the first N (the compliance scale of q = (s, 0))
// on the caller's Nl x Nl block of the Ns x Ns grid
__global__ void __launch_bounds__(kTanThreads) k_tan_scales(long N, int Nl, int Ns,
                                                            const double* __restrict__ s,
                                                            const double* __restrict__ u,
                                                            double* part) {
    double v[2] = {0.0, 0.0};
    TAN_LOOP(N) {
        v[0] = fmax(v[0], s[i]);
        if (Nl == Ns || (i / Ns < Nl && i % Ns < Nl)) v[1] = fmax(v[1], fabs(u[i]));
    }
    const int kind[2] = {1, 1};
    tan_block_out<2>(v, kind, part);
}

// qs = [s; 0]
__global__ void k_tan_sfield(long N, const double* __restrict__ s, double* __restrict__ qs) {
    TAN_LOOP(N) {
        qs[i] = s[i];
        qs[N + i] = 0.0;
    }
}

// terminal exact-load correction pass (friction_solve.cpp:635-660): [0] sum
// qx, [1] sum qy, [2] interior points of A
__global__ void __launch_bounds__(kTanThreads) k_tan_loadsums(long N, const double* __restrict__ s,
                                                              const double* __restrict__ q,
                                                              double* part) {
    double v[3] = {0.0, 0.0, 0.0};
    TAN_LOOP(N) {
        v[0] += q[i];
        v[1] += q[N + i];
        if (s[i] > 0.0 && tan_interior(q[i], q[N + i], s[i])) v[2] += 1.0;
    }
    const int kind[3] = {0, 0, 0};
    tan_block_out<3>(v, kind, part);
}
__global__ void k_tan_loadfix(long N, const double* __restrict__ s, double ax, double ay,
                              double* __restrict__ q) {
    TAN_LOOP(N) {
        const double si = s[i];
        if (!(si > 0.0) || !tan_interior(q[i], q[N + i], si)) continue;
        double qx = q[i] + ax, qy = q[N + i] + ay;
        const double qn = hypot(qx, qy);
        if (qn > si) {
            const double f = si / qn;
            qx *= f;
            qy *= f;
        }
        q[i] = qx;
        q[N + i] = qy;
    }
}

struct V2 {
    double x = 0.0, y = 0.0;
};
inline double v2norm(V2 a) { return std::hypot(a.x, a.y); }

// One inner solve's outcome (the fields of TangentialResult the driver reads)
struct DispOut {
    int status = ST_MAX_ITERATIONS;
    std::string reason;
    int iterations = 0;
    double error = 0.0;
    V2 q_mean;
    int n_stick = 0, n_slip = 0, n_open = 0;
};

// Device workspace and the inner (displacement-control) solve.
struct TanSolver {
    TanOperator& op;
    cudaStream_t st;
    long N;
    int grid;
    double *q = nullptr, *u = nullptr, *g = nullptr, *gp = nullptr, *z = nullptr, *t = nullptr,
           *r = nullptr, *qbest = nullptr, *qw = nullptr;
    // block partials: part (the reduction just launched), part_dir (the
    // direction pass's dots, folded with the evaluation's), part_q (the
    // partition flag of the last update, folded with the next iteration's)
    double* part = nullptr;
    double* part_dir = nullptr;
    double* part_q = nullptr;
    double* red = nullptr;    // folded results
    double* red_h = nullptr;  // pinned host copy
    // the loop kernels' scalars: written on the host (pinned), copied to the
    // device by the iteration's first node
    TanScalars* sc_d = nullptr;
    TanScalars* sc_h = nullptr;
    // The two kernel sequences of an iteration, captured once (on a private
    // stream: a caller's legacy stream cannot capture) and replayed on st:
    // [0] the previous iteration's update, the apply, the evaluation, the
    // direction pass and their folds; [1] the direction update, the apply of
    // t, the line-search dots and their fold.  Their buffers and the scalars
    // record are fixed for the solver's lifetime.
    cudaGraph_t seg_graph[2] = {nullptr, nullptr};
    cudaGraphExec_t seg_exec[2] = {nullptr, nullptr};
    bool seg_ran[2] = {false, false};
    const double* s = nullptr;
    const double* hist = nullptr;
    double Stotal = 0.0;
    // the caller's cell count (mean tractions, open cells); N for the
    // operator's own grid, Nl^2 for an embedded one
    double ncells = 0.0;

    TanSolver(TanOperator& o, cudaStream_t s_) : op(o), st(s_) {
        N = (long)op.Ns * op.Ns;
        ncells = (double)op.Nl * (double)op.Nl;
        grid = (int)std::min<long>(kTanMaxBlocks, (N + kTanThreads - 1) / kTanThreads);
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        double** vs[] = {&q, &u, &g, &gp, &z, &t, &r, &qbest, &qw};
        for (double** v : vs) ASB_CUDA(cudaMalloc((void**)v, 2 * N * sizeof(double)));
        ASB_CUDA(cudaMalloc((void**)&part, (size_t)3 * kTanMaxBlocks * 8 * sizeof(double)));
        part_dir = part + (size_t)kTanMaxBlocks * 8;
        part_q = part + (size_t)2 * kTanMaxBlocks * 8;
        ASB_CUDA(cudaMalloc((void**)&red, 8 * sizeof(double)));
        ASB_CUDA(cudaMallocHost((void**)&red_h, 8 * sizeof(double)));
        ASB_CUDA(cudaMalloc((void**)&sc_d, sizeof(TanScalars)));
        ASB_CUDA(cudaMallocHost((void**)&sc_h, sizeof(TanScalars)));
        *sc_h = TanScalars{};
    }
    ~TanSolver() {
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        for (int k = 0; k < 2; ++k) {
            if (seg_exec[k]) cudaGraphExecDestroy(seg_exec[k]);
            if (seg_graph[k]) cudaGraphDestroy(seg_graph[k]);
        }
        double* vs[] = {q, u, g, gp, z, t, r, qbest, qw, part, red};
        for (double* v : vs) cudaFree(v);
        cudaFree(sc_d);
        cudaFreeHost(red_h);
        cudaFreeHost(sc_h);
    }
    // fold the block partials `src` (nv values, kinds) into red[at ...]
    void fold_into(const double* src, int nv, std::initializer_list<int> kind, int at,
                   cudaStream_t ss = nullptr) {
        TanKinds k{};
        int j = 0;
        for (int v : kind) k.k[j++] = v;
        k_tan_fold<<<1, 32, 0, ss ? ss : st>>>(src, grid, nv, k, red + at);
        count_launches(1);
    }
    // the scalars record, host -> device (pinned source, read when the copy
    // runs: the host writes it only while no segment is in flight)
    void put_scalars(cudaStream_t ss) {
        ASB_CUDA(cudaMemcpyAsync(sc_d, sc_h, sizeof(TanScalars), cudaMemcpyHostToDevice, ss));
    }
    // segment 0 of iteration k >= 1 (iteration 0 has no update to apply and
    // runs its evaluation eagerly): gp <- g (the previous iteration's g), the
    // previous iteration's update unless sc.skip, then the evaluation and the
    // direction pass; red[0..4] = e, max |g|, G, G_pr, partition flag
    void enqueue_seg0(cudaStream_t ss) {
        ASB_CUDA(cudaMemcpyAsync(gp, g, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice, ss));
        put_scalars(ss);
        k_tan_qupd<<<grid, kTanThreads, 0, ss>>>(N, s, t, sc_d, q, part_q);
        op.matvec(true, q, u, ss);
        k_tan_eval<<<grid, kTanThreads, 0, ss>>>(N, s, q, u, hist, sc_d, g, part);
        k_tan_dir<<<grid, kTanThreads, 0, ss>>>(N, s, q, g, gp, z, part_dir);
        count_launches(3);
        fold_into(part, 2, {0, 1}, 0, ss);
        fold_into(part_dir, 2, {0, 0}, 2, ss);
        fold_into(part_q, 1, {1}, 4, ss);
        ASB_CUDA(cudaMemcpyAsync(red_h, red, 5 * sizeof(double), cudaMemcpyDeviceToHost, ss));
    }
    // segment 1: t = chi_A (z + beta t), r = S t, red[0..1] = num, den
    void enqueue_seg1(cudaStream_t ss) {
        put_scalars(ss);
        k_tan_tupd<<<grid, kTanThreads, 0, ss>>>(N, s, z, sc_d, t);
        op.matvec(true, t, r, ss);
        k_tan_numden<<<grid, kTanThreads, 0, ss>>>(N, s, g, t, r, part);
        count_launches(2);
        fold_into(part, 2, {0, 0}, 0, ss);
        ASB_CUDA(cudaMemcpyAsync(red_h, red, 2 * sizeof(double), cudaMemcpyDeviceToHost, ss));
    }
    // run segment k and wait for it: the first time kernel by kernel (every
    // kernel in it then has been loaded and set up outside any capture),
    // then captured once and replayed
    const double* run_seg(int k) {
        if (!seg_ran[k]) {
            if (k == 0) enqueue_seg0(st);
            else enqueue_seg1(st);
            ASB_CUDA(cudaGetLastError());
            ASB_CUDA(cudaStreamSynchronize(st));
            seg_ran[k] = true;
            return red_h;
        }
        if (!seg_exec[k]) {
            std::lock_guard<std::recursive_mutex> setup(setup_mutex());
            cudaStream_t cs = nullptr;
            ASB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            ASB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
            try {
                if (k == 0) enqueue_seg0(cs);
                else enqueue_seg1(cs);
            } catch (...) {
                cudaGraph_t partial = nullptr;
                cudaStreamEndCapture(cs, &partial);
                if (partial) cudaGraphDestroy(partial);
                cudaGetLastError();
                cudaStreamDestroy(cs);
                throw;
            }
            ASB_CUDA(cudaStreamEndCapture(cs, &seg_graph[k]));
            ASB_CUDA(cudaStreamDestroy(cs));
            ASB_CUDA(cudaGraphInstantiate(&seg_exec[k], seg_graph[k], 0));
        }
        ASB_CUDA(cudaGraphLaunch(seg_exec[k], st));
        count_launches(1);
        ASB_CUDA(cudaStreamSynchronize(st));
        return red_h;
    }
    // bring red[0 .. n) to the host (one synchronisation)
    const double* fetch(int n) {
        ASB_CUDA(cudaMemcpyAsync(red_h, red, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        ASB_CUDA(cudaStreamSynchronize(st));
        return red_h;
    }
    // fold the partials of the last reduction kernel (nv values, kinds) and
    // bring them to the host
    const double* fold(int nv, std::initializer_list<int> kind) {
        fold_into(part, nv, kind, 0);
        return fetch(nv);
    }
    void apply(const double* x, double* y) { op.matvec(true, x, y, st); }

    // friction_solve.cpp:26-306 (unpreconditioned)
    DispOut solve_disp(V2 dt, double tol, int max_iter, bool use_pr, const double* q_init,
                       double g_floor) {
        DispOut res;
        k_tan_start<<<grid, kTanThreads, 0, st>>>(N, s, q_init, q);
        ASB_CUDA(cudaMemsetAsync(t, 0, 2 * N * sizeof(double), st));
        ASB_CUDA(cudaMemsetAsync(gp, 0, 2 * N * sizeof(double), st));
        ASB_CUDA(cudaMemcpyAsync(qbest, q, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        count_launches(1);
        double err_best = 1e300, G_old = 1.0, delta_conj = 0.0, g_scale = 0.0, best_err = 1e300;
        int stall = 0;
        const int stall_limit = 200;
        int it = 0;
        // The iteration's kernels run as two segments (enqueue_seg0 / seg1),
        // one host synchronisation each.  Segment 0 applies the previous
        // iteration's update first, so a loop that stops (converged,
        // stalled, out of iterations) never evaluates an update it would
        // discard: q returns to the best evaluated iterate below either way.
        // Every value and decision is the plain loop's.
        sc_h->dx = dt.x;
        sc_h->dy = dt.y;
        sc_h->skip = 1.0;
        bool q_flag_pending = false;  // segment 0 folds an update's partition flag
        // iteration 0: no update to apply
        put_scalars(st);
        apply(q, u);
        k_tan_eval<<<grid, kTanThreads, 0, st>>>(N, s, q, u, hist, sc_d, g, part);
        k_tan_dir<<<grid, kTanThreads, 0, st>>>(N, s, q, g, gp, z, part_dir);
        count_launches(2);
        fold_into(part, 2, {0, 1}, 0);
        fold_into(part_dir, 2, {0, 0}, 2);
        const double* ev = fetch(4);
        for (it = 0; it < max_iter; ++it) {
            if (it > 0) {
                ev = run_seg(0);
                if (q_flag_pending) delta_conj = ev[4] > 0.0 ? 0.0 : 1.0;
                q_flag_pending = false;
            }
            const double e = ev[0], gmax = ev[1], G = ev[2], G_pr = ev[3];
            if (it == 0) g_scale = std::max(gmax > 0.0 ? gmax : 1.0, g_floor);
            res.error = e / (Stotal * g_scale);
            if (res.error < err_best) {
                err_best = res.error;
                ASB_CUDA(cudaMemcpyAsync(qbest, q, 2 * N * sizeof(double),
                                         cudaMemcpyDeviceToDevice, st));
            }
            if (res.error < tol) {
                res.status = ST_CONVERGED;
                break;
            }
            if (res.error < best_err * (1.0 - 1e-4)) {
                best_err = res.error;
                stall = 0;
            } else if (++stall >= stall_limit) {
                res.status = ST_STAGNATED;
                res.reason = "stall";
                break;
            }
            double num = 0.0, den = 0.0;
            for (int attempt = 0;; ++attempt) {
                // a retry reuses z, G, G_pr: q, g and gp are unchanged
                if (attempt == 1) delta_conj = 0.0;  // steepest descent
                sc_h->beta = delta_conj * (use_pr ? std::max(0.0, G_pr / G_old) : G / G_old);
                G_old = G > 0.0 ? G : 1.0;
                const double* nd = run_seg(1);
                num = nd[0];
                den = nd[1];
                if (num > 0.0 || attempt == 1) break;
            }
            if (den <= 0.0 || num <= 0.0) {
                delta_conj = 0.0;
                sc_h->skip = 1.0;
                continue;
            }
            sc_h->tau = num / den;
            sc_h->skip = 0.0;
            q_flag_pending = true;
        }
        // the best iterate seen (friction_solve.cpp:278-283)
        ASB_CUDA(cudaMemcpyAsync(q, qbest, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        res.error = err_best;
        res.iterations = it;
        classify(res);
        return res;
    }
    void classify(DispOut& res) {
        k_tan_classify<<<grid, kTanThreads, 0, st>>>(N, s, q, part);
        count_launches(1);
        const double* c = fold(5, {0, 0, 0, 0, 0});
        res.q_mean.x = c[0] / ncells;
        res.q_mean.y = c[1] / ncells;
        res.n_stick = (int)c[2];
        res.n_slip = (int)c[3];
        // the cells outside an embedded grid's block are open (s = 0) and
        // not the caller's
        res.n_open = (int)(c[4] - ((double)N - ncells));
    }
};

}  // namespace

// solve_tangential (friction_solve.cpp:375-688) with the local KKT check of
// check_tangential_kkt (:309-371); q_out receives the returned traction.
// Fields in the operator's compute-grid layout (see solve_tangential).
void solve_tangential_core(TanOperator& op, const double* s, bool force_control, double tx,
                           double ty, double tol, int max_iter, bool use_pr, double kkt_tol,
                           const double* q_init, const double* u_hist, double* q_out,
                           aspher_tan_result& out, cudaStream_t st) {
    const long N = (long)op.Ns * op.Ns;
    TanSolver S(op, st);
    S.s = s;
    S.hist = u_hist;
    // A = {s > 0}, its count and total; negative thresholds rejected
    {
        std::vector<double> sh(N);
        ASB_CUDA(cudaMemcpyAsync(sh.data(), s, N * sizeof(double), cudaMemcpyDeviceToHost, st));
        ASB_CUDA(cudaStreamSynchronize(st));
        double Stotal = 0.0, smin = 0.0;
        long nA = 0;
        for (long i = 0; i < N; ++i) {
            smin = std::min(smin, sh[i]);
            if (sh[i] > 0.0) {
                ++nA;
                Stotal += sh[i];
            }
        }
        if (smin < 0.0) throw Error(ASPHER_EINVAL, "solve_tangential: negative threshold");
        if (nA == 0) throw Error(ASPHER_EINVAL, "solve_tangential: s == 0 everywhere");
        S.Stotal = Stotal;
    }
    const double kt = kkt_tol > 0.0 ? kkt_tol : 1e-2;
    const V2 target{tx, ty};
    std::memset(&out, 0, sizeof(out));

    auto finish = [&](DispOut& r, V2 delta_used, int iterations) {
        // check_tangential_kkt: rho from the operator's own compliance scale
        k_tan_sfield<<<S.grid, kTanThreads, 0, st>>>(N, s, S.z);
        S.apply(S.z, S.r);
        k_tan_scales<<<S.grid, kTanThreads, 0, st>>>(N, op.Nl, op.Ns, s, S.r, S.part);
        count_launches(2);
        const double* sc = S.fold(2, {1, 1});
        const double s_ref = std::max(sc[0], 1e-300), w_ref = std::max(sc[1], 1e-300);
        const double rho = s_ref / w_ref;
        S.apply(S.q, S.u);
        k_tan_kkt<<<S.grid, kTanThreads, 0, st>>>(N, s, S.q, S.u, u_hist, delta_used.x,
                                                  delta_used.y, rho, s_ref, w_ref, S.part);
        count_launches(1);
        const double* k = S.fold(6, {1, 1, 1, 1, 0, 0});
        out.cone_violation = std::max(0.0, k[0]);
        out.stick_residual = k[1];
        out.slip_residual = k[2];
        out.proj_residual = k[3];
        const V2 qm{k[4] / S.ncells, k[5] / S.ncells};
        out.force_error = force_control ? v2norm({qm.x - target.x, qm.y - target.y}) / s_ref : 0.0;
        out.rho = rho;
        out.s_ref = s_ref;
        out.w_ref = w_ref;
        out.kkt_tol = kt;
        const bool kkt_ok = out.cone_violation <= 1e-9 && out.proj_residual <= kt &&
                            out.force_error <= kt && std::isfinite(out.proj_residual);
        int status = r.status;
        std::string reason = r.reason;
        if (!kkt_ok) {
            if (status == ST_CONVERGED) status = ST_VERIFICATION_FAILED;
            if (reason.empty()) reason = "local_kkt";
        }
        const bool conv = kkt_ok && (status == ST_CONVERGED || status == ST_STAGNATED);
        if (conv) {
            status = ST_CONVERGED;
            reason.clear();
            if (out.proj_residual > 0.1 * kt) reason = "local_kkt_near_tolerance";
        }
        out.status = status;
        out.converged = conv ? 1 : 0;
        std::snprintf(out.status_reason, sizeof(out.status_reason), "%s", reason.c_str());
        out.iterations = iterations;
        out.error = r.error;
        out.delta_t[0] = delta_used.x;
        out.delta_t[1] = delta_used.y;
        out.q_mean[0] = r.q_mean.x;
        out.q_mean[1] = r.q_mean.y;
        out.n_stick = r.n_stick;
        out.n_slip = r.n_slip;
        out.n_open = r.n_open;
        ASB_CUDA(cudaMemcpyAsync(q_out, S.q, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice,
                                 st));
        ASB_CUDA(cudaStreamSynchronize(st));
    };

    if (!force_control) {
        DispOut r = S.solve_disp(target, tol, max_iter, use_pr, q_init, 0.0);
        finish(r, target, r.iterations);
        return;
    }

    // force control (friction_solve.cpp:460-688)
    const double q_limit = S.Stotal / S.ncells;
    if (v2norm(target) >= q_limit)
        throw Error(ASPHER_EINVAL, "solve_tangential: |q_bar| >= mean(s) -- at or beyond the "
                                   "gross-slip limit, no equilibrium exists");
    if (v2norm(target) == 0.0 && !u_hist && !q_init) {  // trivial: q = 0, delta = 0
        DispOut r = S.solve_disp(V2{}, tol, 1, use_pr, nullptr, 0.0);
        r.status = ST_CONVERGED;
        finish(r, V2{}, r.iterations);
        return;
    }
    // full-stick 2x2 stiffness from two eps-probes (cold, no history) or
    // differential probes around the starting shift (with history)
    double K[2][2] = {{0, 0}, {0, 0}};
    int total_it = 0;
    {
        k_tan_sfield<<<S.grid, kTanThreads, 0, st>>>(N, s, S.z);
        S.apply(S.z, S.r);
        k_tan_scales<<<S.grid, kTanThreads, 0, st>>>(N, op.Nl, op.Ns, s, S.r, S.part);
        count_launches(2);
        const double u_scale = S.fold(2, {1, 1})[1];
        if (u_scale <= 0.0)
            throw Error(ASPHER_ECUDA, "solve_tangential: degenerate tangential operator");
        const double eps = 1e-4 * u_scale;
        if (!u_hist) {
            double ep = eps;
            for (int tries = 0; tries < 2; ++tries) {
                DispOut px = S.solve_disp(V2{ep, 0.0}, tol, max_iter, use_pr, nullptr, 0.0);
                DispOut py = S.solve_disp(V2{0.0, ep}, tol, max_iter, use_pr, nullptr, 0.0);
                const int slip = px.n_slip + py.n_slip;
                const int cand = px.n_slip + px.n_stick + py.n_slip + py.n_stick;
                if (tries == 0 && slip > cand / 5) {
                    ep *= 0.5;
                    continue;
                }
                K[0][0] = px.q_mean.x / ep;
                K[1][0] = px.q_mean.y / ep;
                K[0][1] = py.q_mean.x / ep;
                K[1][1] = py.q_mean.y / ep;
                total_it = px.iterations + py.iterations;
                break;
            }
        } else {
            DispOut base = S.solve_disp(V2{}, tol, max_iter, use_pr, q_init, 0.0);
            ASB_CUDA(cudaMemcpyAsync(S.qw, S.q, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice,
                                     st));
            DispOut px = S.solve_disp(V2{eps, 0.0}, tol, max_iter, use_pr, S.qw, 0.0);
            ASB_CUDA(cudaMemcpyAsync(S.qw, S.q, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice,
                                     st));
            DispOut py = S.solve_disp(V2{0.0, eps}, tol, max_iter, use_pr, S.qw, 0.0);
            K[0][0] = (px.q_mean.x - base.q_mean.x) / eps;
            K[1][0] = (px.q_mean.y - base.q_mean.y) / eps;
            K[0][1] = (py.q_mean.x - base.q_mean.x) / eps;
            K[1][1] = (py.q_mean.y - base.q_mean.y) / eps;
            total_it = base.iterations + px.iterations + py.iterations;
            if (K[0][0] * K[1][1] - K[0][1] * K[1][0] <= 0.0)
                throw Error(ASPHER_ECUDA, "solve_tangential: probe stiffness degenerate");
        }
    }
    auto det = [](const double (&A)[2][2]) { return A[0][0] * A[1][1] - A[0][1] * A[1][0]; };
    auto solve2 = [&](const double (&A)[2][2], V2 b) {  // A^-1 b
        const double d = det(A);
        return V2{(A[1][1] * b.x - A[0][1] * b.y) / d, (-A[1][0] * b.x + A[0][0] * b.y) / d};
    };
    const double ftol = 1e-8;
    const int outer_max = 40;
    const double target_scale = v2norm(target) > 0.0 ? v2norm(target) : q_limit;
    V2 delta = solve2(K, target), delta_prev, F_prev;
    bool have_prev = false, have_warm = q_init != nullptr, best_converged = false;
    if (q_init)
        ASB_CUDA(cudaMemcpyAsync(S.qw, q_init, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice,
                                 st));
    double F_best = 1e300;
    V2 delta_best = delta;
    DispOut best;
    // the best outer iterate's traction
    struct DevBuf {
        double* p = nullptr;
        ~DevBuf() { cudaFree(p); }
    } keep;
    ASB_CUDA(cudaMalloc((void**)&keep.p, 2 * N * sizeof(double)));
    double* qkeep = keep.p;
    {
        for (int outer = 0; outer < outer_max; ++outer) {
            DispOut inner = S.solve_disp(delta, tol, max_iter, use_pr, have_warm ? S.qw : nullptr,
                                         0.0);
            total_it += inner.iterations;
            const V2 F{inner.q_mean.x - target.x, inner.q_mean.y - target.y};
            ASB_CUDA(cudaMemcpyAsync(S.qw, S.q, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice,
                                     st));
            have_warm = true;
            if (v2norm(F) < F_best) {
                F_best = v2norm(F);
                delta_best = delta;
                best_converged = inner.status == ST_CONVERGED;
                best = inner;
                ASB_CUDA(cudaMemcpyAsync(qkeep, S.q, 2 * N * sizeof(double),
                                         cudaMemcpyDeviceToDevice, st));
            }
            if (v2norm(F) <= ftol * target_scale) break;
            if (have_prev && v2norm({F.x - F_prev.x, F.y - F_prev.y}) <=
                                 1e-3 * std::max(v2norm(F), 1e-300))
                break;
            if (have_prev) {  // Broyden: K <- K + ((dF - K dd) dd^T) / |dd|^2
                const V2 dd{delta.x - delta_prev.x, delta.y - delta_prev.y};
                const double dd2 = dd.x * dd.x + dd.y * dd.y;
                if (dd2 > 0.0) {
                    const V2 Kdd{K[0][0] * dd.x + K[0][1] * dd.y, K[1][0] * dd.x + K[1][1] * dd.y};
                    const V2 w{(F.x - F_prev.x) - Kdd.x, (F.y - F_prev.y) - Kdd.y};
                    double Ku[2][2] = {{K[0][0] + w.x * dd.x / dd2, K[0][1] + w.x * dd.y / dd2},
                                       {K[1][0] + w.y * dd.x / dd2, K[1][1] + w.y * dd.y / dd2}};
                    if (det(Ku) > 1e-6 * std::abs(det(K)))
                        for (int a = 0; a < 2; ++a)
                            for (int b = 0; b < 2; ++b) K[a][b] = Ku[a][b];
                }
            }
            delta_prev = delta;
            F_prev = F;
            have_prev = true;
            const V2 step = solve2(K, F);
            if (!std::isfinite(step.x) || !std::isfinite(step.y))
                throw Error(ASPHER_ECUDA, "solve_tangential: force-control step not finite");
            delta.x -= step.x;
            delta.y -= step.y;
        }
        // terminal exact-load enforcement on the best outer iterate
        ASB_CUDA(cudaMemcpyAsync(S.q, qkeep, 2 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        for (int pass = 0; pass < 3; ++pass) {
            k_tan_loadsums<<<S.grid, kTanThreads, 0, st>>>(N, s, S.q, S.part);
            count_launches(1);
            const double* ls = S.fold(3, {0, 0, 0});
            const double cx = target.x * S.ncells - ls[0], cy = target.y * S.ncells - ls[1];
            const double ni = ls[2];
            if (ni <= 0.0 || (std::abs(cx) + std::abs(cy)) <= 1e-14 * S.ncells * target_scale)
                break;
            k_tan_loadfix<<<S.grid, kTanThreads, 0, st>>>(N, s, cx / ni, cy / ni, S.q);
            count_launches(1);
        }
        S.classify(best);
        best.status = (best_converged && F_best <= 1e-3 * target_scale) ? ST_CONVERGED
                                                                          : ST_STAGNATED;
        if (best.status != ST_CONVERGED) best.reason = "outer force iteration";
        else best.reason.clear();
        finish(best, delta_best, total_it);
    }
}

// The caller's fields (s: Nl^2 thresholds; q_init, u_hist, q_out: 2 Nl^2)
// around the core: for an embedded operator they are copied into
// compute-grid fields whose cells outside the caller's block have s = 0
// (open: the solve never gives them traction, as the reference never does
// an open cell) and zero warm start and history, and the traction's block is
// copied back.
void solve_tangential(TanOperator& op, const double* s, bool force_control, double tx,
                      double ty, double tol, int max_iter, bool use_pr, double kkt_tol,
                      const double* q_init, const double* u_hist, double* q_out,
                      aspher_tan_result& out, cudaStream_t st) {
    if (!op.embedded()) {
        solve_tangential_core(op, s, force_control, tx, ty, tol, max_iter, use_pr, kkt_tol,
                              q_init, u_hist, q_out, out, st);
        return;
    }
    const long n = (long)op.Ns * op.Ns;
    std::vector<double*> bufs;
    auto alloc = [&](long count) {
        double* p = nullptr;
        ASB_CUDA(cudaMallocAsync((void**)&p, (size_t)count * sizeof(double), st));
        bufs.push_back(p);
        return p;
    };
    auto embed = [&](const double* src, int fields) -> const double* {
        if (!src) return nullptr;
        double* d = alloc(fields * n);
        k_embed<double, double><<<embed_grid(fields * n), 256, 0, st>>>(op.Nl, op.Ns, fields,
                                                                         src, d, 0.0);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
        return d;
    };
    try {
        const double* sc = embed(s, 1);
        const double* qi = embed(q_init, 2);
        const double* uh = embed(u_hist, 2);
        double* qc = alloc(2 * n);
        solve_tangential_core(op, sc, force_control, tx, ty, tol, max_iter, use_pr, kkt_tol, qi,
                              uh, qc, out, st);
        k_extract<double, double><<<embed_grid(2 * (long)op.Nl * op.Nl), 256, 0, st>>>(
            op.Nl, op.Ns, 2, qc, q_out);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
    } catch (...) {
        for (double* p : bufs) cudaFreeAsync(p, st);
        throw;
    }
    for (double* p : bufs) cudaFreeAsync(p, st);
    ASB_CUDA(cudaStreamSynchronize(st));
}

}  // namespace asb

struct aspher_tan_op {
    asb::TanOperator* impl;
};

extern "C" {

int aspher_tan_create(int grid_size, double domain_size, double E_star, double nu,
                      aspher_tan_op** out) {
    try {
        if (!out) throw asb::Error(ASPHER_EINVAL, "aspher_tan_create: out is NULL");
        *out = nullptr;
        auto* op = new aspher_tan_op{nullptr};
        try {
            op->impl = new asb::TanOperator(grid_size, domain_size, E_star, nu);
        } catch (...) {
            delete op;
            throw;
        }
        *out = op;
        return ASPHER_OK;
    } catch (const asb::Error& e) {
        asb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        asb::set_last_error(e.what());
        return ASPHER_ECUDA;
    }
}

int aspher_tan_destroy(aspher_tan_op* op) {
    if (op) {
        delete op->impl;
        delete op;
    }
    return ASPHER_OK;
}

int aspher_tan_matvec(aspher_tan_op* op, int dtype, const void* q_dev, void* u_dev,
                      void* stream) {
    try {
        if (!op || !op->impl || !q_dev || !u_dev)
            throw asb::Error(ASPHER_EINVAL, "aspher_tan_matvec: NULL argument");
        if (((uintptr_t)q_dev | (uintptr_t)u_dev) % 16)
            throw asb::Error(ASPHER_EINVAL, "aspher_tan_matvec: buffers must be 16-byte aligned");
        if (dtype != ASPHER_F32 && dtype != ASPHER_F64)
            throw asb::Error(ASPHER_EINVAL, "aspher_tan_matvec: dtype must be F32 or F64");
        op->impl->apply_caller(dtype == ASPHER_F64, q_dev, u_dev,
                               static_cast<cudaStream_t>(stream));
        return ASPHER_OK;
    } catch (const asb::Error& e) {
        asb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        asb::set_last_error(e.what());
        return ASPHER_ECUDA;
    }
}

int aspher_solve_tangential(aspher_tan_op* op, const double* s_dev, int force_control,
                            double target_x, double target_y, double tol, int max_iter,
                            int use_pr, double kkt_tol, const double* q_init_dev,
                            const double* u_hist_dev, double* q_dev, aspher_tan_result* res,
                            void* stream) {
    try {
        if (!op || !op->impl || !s_dev || !q_dev || !res)
            throw asb::Error(ASPHER_EINVAL, "aspher_solve_tangential: NULL argument");
        if (((uintptr_t)s_dev | (uintptr_t)q_dev | (uintptr_t)q_init_dev |
             (uintptr_t)u_hist_dev) % 16)
            throw asb::Error(ASPHER_EINVAL, "aspher_solve_tangential: buffers must be 16-byte aligned");
        if (!(tol > 0.0)) throw asb::Error(ASPHER_EINVAL, "aspher_solve_tangential: tol must be positive");
        if (max_iter < 1) throw asb::Error(ASPHER_EINVAL, "aspher_solve_tangential: max_iter must be >= 1");
        asb::solve_tangential(*op->impl, s_dev, force_control != 0, target_x, target_y, tol,
                              max_iter, use_pr != 0, kkt_tol, q_init_dev, u_hist_dev, q_dev, *res,
                              static_cast<cudaStream_t>(stream));
        return ASPHER_OK;
    } catch (const asb::Error& e) {
        asb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        asb::set_last_error(e.what());
        return ASPHER_ECUDA;
    }
}

int aspher_tan_max_im_ratio(const aspher_tan_op* op, double* out) {
    if (!op || !op->impl || !out) {
        asb::set_last_error("aspher_tan_max_im_ratio: NULL argument");
        return ASPHER_EINVAL;
    }
    *out = op->impl->max_im_ratio;
    return ASPHER_OK;
}

// CerrutiKernel's signed offset tables (xx, yy, xy) for offsets dx, dy in
// (-Ns, Ns), row-major [dy + Ns - 1][dx + Ns - 1], copied to host memory.
int aspher_tan_tables(const aspher_tan_op* op, double* xx_host, double* yy_host,
                      double* xy_host) {
    try {
        if (!op || !op->impl || !xx_host || !yy_host || !xy_host)
            throw asb::Error(ASPHER_EINVAL, "aspher_tan_tables: NULL argument");
        // the caller's offsets |d| < Nl of the tables (pitch: the compute grid)
        const int Ns = op->impl->Nl, P = op->impl->Ns;
        std::vector<double> xx((size_t)P * P), xy((size_t)P * P);
        ASB_CUDA(cudaMemcpy(xx.data(), op->impl->tab_xx, xx.size() * sizeof(double),
                            cudaMemcpyDeviceToHost));
        ASB_CUDA(cudaMemcpy(xy.data(), op->impl->tab_xy, xy.size() * sizeof(double),
                            cudaMemcpyDeviceToHost));
        const int W = 2 * Ns - 1;
        for (int dy = -(Ns - 1); dy < Ns; ++dy)
            for (int dx = -(Ns - 1); dx < Ns; ++dx) {
                const int ax = dx < 0 ? -dx : dx, ay = dy < 0 ? -dy : dy;
                const size_t at = (size_t)(dy + Ns - 1) * W + (dx + Ns - 1);
                xx_host[at] = xx[(size_t)ay * P + ax];
                yy_host[at] = xx[(size_t)ax * P + ay];
                const double v = xy[(size_t)ay * P + ax];
                xy_host[at] = (dx == 0 || dy == 0) ? 0.0 : (((dx > 0) == (dy > 0)) ? v : -v);
            }
        return ASPHER_OK;
    } catch (const asb::Error& e) {
        asb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        asb::set_last_error(e.what());
        return ASPHER_ECUDA;
    }
}

}  // extern "C"
