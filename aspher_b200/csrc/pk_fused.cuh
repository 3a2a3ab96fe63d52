// Pieces of the PK iteration that run inside the operator's row kernels.
//
// The second apply of an iteration, r = S t, is bracketed by two vector
// passes of the reference loop (contact_solver.cpp:440-478): the direction
// update t = chi_C(z_f + beta t) just before it and the sums of r (rsum,
// num, den) just after.  LoadTupd computes the new t inside the forward row
// kernel's load (writing t, g_prev and, when asked, the best-pressure copy
// as it goes, and feeding t to the transform), and StoreRden consumes r in
// the inverse row kernel's store (r itself is never written): two passes
// and the r round trip leave the iteration.  Both read instance
// blockIdx.y's state and fields (batched launches).
#pragma once

#include "common.cuh"
#include "pk_state.hpp"
#include "reduce.cuh"

namespace asb {

__device__ __forceinline__ void set_halt(PkState* st, int h) {
    st->halt = h;
    st->skip_mv1 = 1;
}

// Scalar tail of the rsum / den pass (thread 0 of the last block).
// acc = {sum_C r, sum_C g t, sum_C r t, sum_C t};
// den = sum_C Real(r - rm) t, linear in rm: sum_C r t - rm sum_C t.
template <typename T>
__device__ inline void rden_tail(PkState* st, const double (&acc)[4]) {
    st->mv++;
    if (st->copy_best) {
        st->copy_best = 0;
        st->have_best = 1;
    }
    st->rsum = acc[0];
    st->num = acc[1];
    st->rmean = (double)(T)(st->nc ? acc[0] / st->nc : 0.0);
    const double den = acc[2] - st->rmean * acc[3], num = acc[1];
    st->den = den;
    if (den > 0.0 && isfinite(den) && isfinite(num)) {
        const T tau = (T)(num / den);
        st->tau = (double)tau;
        st->tau_ov = st->gg > 0.0 ? (double)(T)(num * num / (den * st->gg)) : (double)tau;
    } else {
        set_halt(st, H_IDENT);  // no usable direction: identification step
    }
}

// Row-kernel load: z[n] = (t[2n], t[2n+1]) of the updated direction
//   t = contact ? Real(z_f + beta t) : 0,  z_f = precond ? Real(z - zmean) : g,
// with g = Real(v - Real(alpha)) centred on the fly; also g_prev = g and,
// when copy_best is set, best = p.
template <typename T>
struct LoadTupd {
    static constexpr bool kTiled = false;
    static constexpr bool kRaw = false;
    const T* z;
    const T* g;  // v (uncentred)
    T* gprev;
    T* t;
    const uint8_t* mask;
    const T* p;
    T* best;
    const PkState* st;
    int pitch;
    int precond;
    long bs;  // batch stride (elements)
    __device__ __forceinline__ cplx<T> operator()(int row, int n) const {
        const PkState* sb = st + blockIdx.y;
        const T zm = (T)sb->zmean, beta = (T)sb->beta, aT = (T)sb->alpha;
        const size_t i = blockIdx.y * bs + (size_t)row * pitch + 2 * n;
        const uchar2 m = *reinterpret_cast<const uchar2*>(mask + i);
        const cplx<T> gv = *reinterpret_cast<const cplx<T>*>(g + i);
        const cplx<T> tv = *reinterpret_cast<const cplx<T>*>(t + i);
        const T g0 = gv.x - aT, g1 = gv.y - aT;
        T f0 = g0, f1 = g1;
        if (precond) {
            const cplx<T> zv = *reinterpret_cast<const cplx<T>*>(z + i);
            f0 = (T)(zv.x - zm);
            f1 = (T)(zv.y - zm);
        }
        const cplx<T> tn = mk<T>(m.x ? (T)(f0 + beta * tv.x) : T(0),
                                 m.y ? (T)(f1 + beta * tv.y) : T(0));
        *reinterpret_cast<cplx<T>*>(t + i) = tn;
        *reinterpret_cast<cplx<T>*>(gprev + i) = mk<T>(g0, g1);
        if (sb->copy_best)
            *reinterpret_cast<cplx<T>*>(best + i) = *reinterpret_cast<const cplx<T>*>(p + i);
        return tn;
    }
};

// Row-kernel store: accumulates the rsum / den sums of r = S t over the
// contact set; finish() runs the grid reduction and rden_tail.
template <typename T>
struct StoreRden {
    static constexpr bool kTiled = false;
    static constexpr bool kFinish = true;
    const T* g;  // v (uncentred)
    const T* t;
    const uint8_t* mask;
    PkState* st;
    double* part;
    int pitch;
    long bs;
    double a0, a1, a2, a3;
    __device__ __forceinline__ void operator()(int row, int n, cplx<T> r) {
        const T aT = (T)st[blockIdx.y].alpha;
        const size_t i = blockIdx.y * bs + (size_t)row * pitch + 2 * n;
        const uchar2 m = *reinterpret_cast<const uchar2*>(mask + i);
        const cplx<T> gv = *reinterpret_cast<const cplx<T>*>(g + i);
        const cplx<T> tv = *reinterpret_cast<const cplx<T>*>(t + i);
        if (m.x) {
            const double td = (double)tv.x;
            a0 += (double)r.x;
            a1 += (double)(T)(gv.x - aT) * td;
            a2 += (double)r.x * td;
            a3 += td;
        }
        if (m.y) {
            const double td = (double)tv.y;
            a0 += (double)r.y;
            a1 += (double)(T)(gv.y - aT) * td;
            a2 += (double)r.y * td;
            a3 += td;
        }
    }
    __device__ void finish(double*) {
        double a[4] = {a0, a1, a2, a3};
        const int kinds[4] = {0, 0, 0, 0};
        PkState* sb = st + blockIdx.y;
        double* pb = part + (size_t)blockIdx.y * kPartStride;
        if (grid_reduce_last<4>(a, kinds, pb, &sb->counter[4]) && threadIdx.x == 0)
            rden_tail<T>(sb, a);
    }
};

}  // namespace asb
