// Load / store / multiplier functors of the row and column kernels shared by
// the operators (operators.cu) and the allocation-free entry point.
#pragma once

#include "fft_kernels.cuh"

namespace asb {

// Every functor offsets by blockIdx.y * bs (elements): instance blockIdx.y
// of a batched launch (bs = 0 or gridDim.y = 1 for a single field).
// The PK loop's pressure with the pending load rescale of instance
// blockIdx.y (PkState::scale / scale_add): Real(x f) + a.
template <typename T>
__device__ __forceinline__ T pending_scale(const PkState* sc, T x) {
    const PkState* sb = sc + blockIdx.y;
    return x * (T)__ldg(&sb->scale) + (T)__ldg(&sb->scale_add);
}

template <typename T>
struct LoadRealRows {  // z[n] = (x[row*pitch + 2n], x[row*pitch + 2n + 1])
    const T* x;
    int pitch;
    long bs;
    // optional: x is the PK loop's pressure, scaled by the pending load
    // rescale of sc[blockIdx.y] as it is loaded
    const PkState* sc = nullptr;
    static constexpr bool kTiled = false;
    static constexpr bool kRaw = true;  // plain rows: the row kernel may stage them
    __device__ __forceinline__ cplx<T> fix(cplx<T> v) const {
        if (sc) {
            v.x = pending_scale(sc, v.x);
            v.y = pending_scale(sc, v.y);
        }
        return v;
    }
    __device__ __forceinline__ cplx<T> operator()(int row, int n) const {
        return fix(*reinterpret_cast<const cplx<T>*>(x + blockIdx.y * bs + (size_t)row * pitch +
                                                      2 * n));
    }
};

template <typename T>
struct StoreRealRows {
    T* y;
    int pitch;
    long bs;
    static constexpr bool kFinish = false;
    static constexpr bool kTiled = false;
    __device__ __forceinline__ void operator()(int row, int n, cplx<T> z) const {
        *reinterpret_cast<cplx<T>*>(y + blockIdx.y * bs + (size_t)row * pitch + 2 * n) = z;
    }
    __device__ void finish(double*) const {}
};

// FP64 rows in, FP32 pairs out: x - x0 (x0 optional), rounded once.  The
// defect-corrected FP64 apply (Operator::matvec_defect) transforms this
// difference in FP32.
struct LoadDiffRows {
    static constexpr bool kTiled = false;
    static constexpr bool kRaw = false;
    const double* x;
    const double* x0;
    int pitch;
    long bs;
    // optional: x is the PK loop's pressure with a pending load rescale
    // (see LoadRealRows)
    const PkState* sc = nullptr;
    __device__ __forceinline__ cplx<float> operator()(int row, int n) const {
        const size_t i = blockIdx.y * bs + (size_t)row * pitch + 2 * n;
        double2 v = *reinterpret_cast<const double2*>(x + i);
        if (sc) {
            v.x = pending_scale(sc, v.x);
            v.y = pending_scale(sc, v.y);
        }
        if (x0) {
            const double2 w = *reinterpret_cast<const double2*>(x0 + i);
            v.x -= w.x;
            v.y -= w.y;
        }
        return mk<float>((float)v.x, (float)v.y);
    }
};

// FP32 pairs in, FP64 rows out: y = y0 + z (y0 optional).
struct StoreAddRows {
    static constexpr bool kFinish = false;
    static constexpr bool kTiled = false;
    double* y;
    const double* y0;
    int pitch;
    long bs;
    __device__ __forceinline__ void operator()(int row, int n, cplx<float> z) const {
        const size_t i = blockIdx.y * bs + (size_t)row * pitch + 2 * n;
        double2 o = make_double2((double)z.x, (double)z.y);
        if (y0) {
            const double2 w = *reinterpret_cast<const double2*>(y0 + i);
            o.x += w.x;
            o.y += w.y;
        }
        *reinterpret_cast<double2*>(y + i) = o;
    }
    __device__ void finish(double*) const {}
};

template <typename T>
struct StoreTiled {
    cplx<T>* base;
    int nrows, ct;
    long bs;
    static constexpr bool kFinish = false;
    static constexpr bool kTiled = true;  // row kernels store whole tile chunks
    __device__ __forceinline__ void operator()(int row, int k, cplx<T> X) const {
        base[blockIdx.y * bs + (size_t)(k / ct) * nrows * ct + (size_t)row * ct + (k % ct)] = X;
    }
    __device__ void finish(double*) const {}
};

template <typename T>
struct LoadTiled {
    const cplx<T>* base;
    int nrows, ct;
    long bs;
    static constexpr bool kTiled = true;  // row kernels load whole tile chunks
    static constexpr bool kRaw = false;
    __device__ __forceinline__ cplx<T> operator()(int row, int k) const {
        return base[blockIdx.y * bs + (size_t)(k / ct) * nrows * ct + (size_t)row * ct +
                    (k % ct)];
    }
};

// Free-space multiplier: real Kh, even-folded in ky, tiled like the spectrum
// with ct columns per tile and Ns+1 rows.
template <typename T>
struct KhMult {
    const T* kh;
    int nk;  // Ns + 1 rows
    int M;   // padded length 2 Ns
    int ct;
    __device__ __forceinline__ cplx<T> operator()(cplx<T> X, int kx, int ky) const {
        const int kf = ky <= (M >> 1) ? ky : M - ky;
        const T w = __ldg(&kh[(size_t)(kx / ct) * nk * ct + (size_t)kf * ct + (kx % ct)]);
        return cscale(X, w);
    }
};

// Periodic multiplier: scale / |m| in FP64, cast to T (periodic_fft_operator.cpp:34-47).
template <typename T>
struct PeriodicMult {
    double scale;
    int Ns;
    __device__ __forceinline__ cplx<T> operator()(cplx<T> X, int kx, int ky) const {
        const int my = ky < (Ns + 1) / 2 ? ky : ky - Ns;
        const double m2 = (double)kx * kx + (double)my * my;
        const T w = m2 > 0.0 ? (T)(scale / sqrt(m2)) : T(0);
        return cscale(X, w);
    }
};

}  // namespace asb
