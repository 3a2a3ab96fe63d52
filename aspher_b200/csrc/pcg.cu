// Polonsky-Keer projected CG with certified termination on the device.
//
// Reference: solve_contact_impl<Real> (src/contact_solver.cpp:150-587),
// project_load_simplex (:31-60), identification step (:314-364),
// evaluate()/refine_contact_mean (:69-99, :260-303).  Real = T in {float,
// double}; every reduction is accumulated in FP64 as in the reference.
//
// One CG iteration is the kernel sequence
//   [apply p->u] eval1 eval2 [precond] dots tupd [apply t->r] rsum den pupd rescale
// where each pass is one HBM sweep and each reduction's scalar logic runs in
// the last block of its pass (see pk_state.hpp).  The host enqueues several
// iterations between synchronisations; once a pass sets `halt`, the rest are
// no-ops.
#include "../../include/aspher_b200.h"
#include "ops.hpp"
#include "pk_state.hpp"
#include "pcg.hpp"
#include "reduce.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

namespace asb {

// ---- vector helpers ------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void ld4(const T* __restrict__ p, long i4, T (&a)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(p) + i4);
        a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
    } else {
        const double2 v0 = __ldg(reinterpret_cast<const double2*>(p) + 2 * i4);
        const double2 v1 = __ldg(reinterpret_cast<const double2*>(p) + 2 * i4 + 1);
        a[0] = v0.x; a[1] = v0.y; a[2] = v1.x; a[3] = v1.y;
    }
}
// load through L2 without the read-only path (for arrays written earlier in
// the same kernel sequence by other kernels it does not matter; kept plain)
template <typename T>
__device__ __forceinline__ void ldp4(const T* p, long i4, T (&a)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 v = reinterpret_cast<const float4*>(p)[i4];
        a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
    } else {
        const double2 v0 = reinterpret_cast<const double2*>(p)[2 * i4];
        const double2 v1 = reinterpret_cast<const double2*>(p)[2 * i4 + 1];
        a[0] = v0.x; a[1] = v0.y; a[2] = v1.x; a[3] = v1.y;
    }
}
template <typename T>
__device__ __forceinline__ void st4(T* p, long i4, const T (&a)[4]) {
    if constexpr (sizeof(T) == 4) {
        reinterpret_cast<float4*>(p)[i4] = make_float4(a[0], a[1], a[2], a[3]);
    } else {
        reinterpret_cast<double2*>(p)[2 * i4] = make_double2(a[0], a[1]);
        reinterpret_cast<double2*>(p)[2 * i4 + 1] = make_double2(a[2], a[3]);
    }
}
__device__ __forceinline__ void ldm4(const uint8_t* m, long i4, uint8_t (&a)[4]) {
    const uchar4 v = reinterpret_cast<const uchar4*>(m)[i4];
    a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
}
__device__ __forceinline__ void stm4(uint8_t* m, long i4, const uint8_t (&a)[4]) {
    reinterpret_cast<uchar4*>(m)[i4] = make_uchar4(a[0], a[1], a[2], a[3]);
}

#define GRID_LOOP4(N) \
    for (long i4 = blockIdx.x * (long)blockDim.x + threadIdx.x; i4 < (N) / 4; i4 += (long)gridDim.x * blockDim.x)

__device__ __forceinline__ void set_halt(PkState* st, int h) {
    st->halt = h;
    st->skip_mv1 = 1;
}

// ---- evaluate() -----------------------------------------------------------------
// pass 1: v = u + (g0 - gshift) -> g; sum of v over p>0, count, min v.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_eval1(const PkParams* __restrict__ Pp, PkState* st, const T* u,
                                                       const T* g0, const T* p, T* g,
                                                       double* part, int final_mode) {
    const PkParams& P = *Pp;
    if (!final_mode && st->halt) return;
    const T gs = (T)P.gshift;
    double acc[3] = {0.0, 0.0, (double)INFINITY};
    GRID_LOOP4(P.N) {
        T uu[4], gg0[4], pp[4], vv[4];
        ldp4(u, i4, uu);
        ldp4(g0, i4, gg0);
        ldp4(p, i4, pp);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const T v = uu[j] + (gg0[j] - gs);
            vv[j] = v;
            const double vd = (double)v;
            acc[2] = fmin(acc[2], vd);
            if (pp[j] > T(0)) { acc[0] += vd; acc[1] += 1.0; }
        }
        st4(g, i4, vv);
    }
    const int kinds[3] = {0, 0, 1};
    if (grid_reduce_last<3>(acc, kinds, part, &st->counter[0]) && threadIdx.x == 0) {
        if (!final_mode) {
            if (!st->u_fresh) st->mv++;
            st->u_fresh = 0;
            st->skip_mv1 = 0;
        }
        const int nc = (int)acc[1];
        st->nc = nc;
        st->gsum = acc[0];
        st->vmin = acc[2];
        st->alpha = nc ? acc[0] / nc : acc[2];
        st->gmin = acc[2] - st->alpha;
    }
}

// pass 2: centre g, certificate sums, contact mask; last block runs the
// convergence test and the best/stall bookkeeping (contact_solver.cpp:379-412).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_eval2(const PkParams* __restrict__ Pp, PkState* st, const T* p, T* g,
                                                       uint8_t* mask, double* part, double* hist,
                                                       int final_mode) {
    const PkParams& P = *Pp;
    if (!final_mode && st->halt) return;
    const T aT = (T)st->alpha, gmT = (T)st->gmin;
    double acc[5] = {0, 0, 0, 0, 0};  // pv, gcs, e, Gc, psum
    GRID_LOOP4(P.N) {
        T pp[4], gv[4];
        uint8_t mm[4];
        ldp4(p, i4, pp);
        ldp4(g, i4, gv);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double pd = (double)pp[j];
            acc[0] += pd * (double)gv[j];
            const T gi = gv[j] - aT;
            gv[j] = gi;
            const double gid = (double)gi;
            if (pd > 0.0) acc[1] += gid;
            acc[2] += pd * fabs(gid);
            acc[3] += pd * (double)(gi - gmT);
            acc[4] += pd;
            mm[j] = pp[j] > T(0) ? 1 : 0;
        }
        st4(g, i4, gv);
        stm4(mask, i4, mm);
    }
    const int kinds[5] = {0, 0, 0, 0, 0};
    if (grid_reduce_last<5>(acc, kinds, part, &st->counter[1]) && threadIdx.x == 0) {
        const int nc = st->nc;
        double alpha = st->alpha, gmin = st->gmin;
        if (nc > 0) {  // refine_contact_mean (contact_solver.cpp:94-99)
            const double d = acc[1] / nc;
            alpha += d;
            gmin -= d;
        }
        const double PG = P.P_total * P.g_ref;
        st->alpha_ref = alpha;
        st->gmin_ref = gmin;
        st->pv = acc[0];
        st->gcs = acc[1];
        st->pk = acc[2] / PG;
        st->G = acc[3];
        st->fw = acc[3] / PG;
        st->pen = fmax(0.0, -gmin) / P.g_ref;
        st->psum = acc[4];
        st->load = fabs(acc[4] - P.P_total) / P.P_total;
        st->finite = isfinite(st->gsum) && isfinite(st->vmin) && isfinite(acc[4]) &&
                     isfinite(acc[2]) && isfinite(acc[3]);
        if (final_mode) return;
        if (!st->finite) {
            st->status = ST_NONFINITE;
            set_halt(st, H_FINAL);
            return;
        }
        if (P.record_history && hist) hist[st->it] = st->pk;
        if (st->load <= P.load_tol && st->fw <= P.tol && st->pen <= P.tol) {
            st->status = ST_CONVERGED;
            st->u_fresh = 1;
            set_halt(st, H_FINAL);
            return;
        }
        const double merit = fmax(st->fw, st->pen);
        if (P.keep_best && merit < st->best_merit) {
            st->best_merit = merit;
            st->copy_best = 1;
        }
        if (merit < st->seen_merit * (1.0 - 1e-4)) {
            st->seen_merit = merit;
            st->stall = 0;
        } else if (++st->stall >= P.stall_limit) {
            set_halt(st, H_STALL);
            return;
        }
        if (nc < 2) set_halt(st, H_IDENT);
    }
}

// ---- stencil preconditioner (stencil_precond.cpp:63-109) ---------------------
// z = T(sum_t w_t gc(i + d_t)) on contact, gc = contact ? g - gmean : 0 with
// periodic wrap; the contact mean of z is removed downstream (dots/tupd read
// z - zmean).  2-D tile of 64 x 16 outputs with an R-cell halo in shared memory.
constexpr int kStX = 64, kStY = 16, kMaxR = 4;

template <typename T>
__global__ void __launch_bounds__(256) k_stencil(const PkParams* __restrict__ Pp, PkState* st, StencilTaps taps,
                                                 const T* g, const uint8_t* mask, T* z,
                                                 double* part, int gated) {
    const PkParams& P = *Pp;
    if (gated && st->halt) return;
    __shared__ double tile[(kStY + 2 * kMaxR) * (kStX + 2 * kMaxR)];
    const int Ns = P.Ns, R = taps.R;
    const int TW = kStX + 2 * R, TH = kStY + 2 * R;
    const double gmean = st->nc ? st->gcs / st->nc : 0.0;
    const int ntx = (Ns + kStX - 1) / kStX, nty = (Ns + kStY - 1) / kStY;
    double acc[1] = {0.0};
    for (int tid = blockIdx.x; tid < ntx * nty; tid += gridDim.x) {
        const int tx0 = (tid % ntx) * kStX, ty0 = (tid / ntx) * kStY;
        for (int idx = threadIdx.x; idx < TW * TH; idx += blockDim.x) {
            const int ly = idx / TW, lx = idx % TW;
            int gy = ty0 + ly - R, gx = tx0 + lx - R;
            gy = gy < 0 ? gy + Ns : (gy >= Ns ? gy - Ns : gy);
            gx = gx < 0 ? gx + Ns : (gx >= Ns ? gx - Ns : gx);
            const size_t j = (size_t)gy * Ns + gx;
            tile[ly * TW + lx] = mask[j] ? (double)g[j] - gmean : 0.0;
        }
        __syncthreads();
        for (int o = threadIdx.x; o < kStX * kStY; o += blockDim.x) {
            const int ly = o / kStX, lx = o % kStX;
            const int gy = ty0 + ly, gx = tx0 + lx;
            if (gy >= Ns || gx >= Ns) continue;
            const size_t i = (size_t)gy * Ns + gx;
            if (!mask[i]) { z[i] = T(0); continue; }
            double a = 0.0;
            for (int t = 0; t < taps.n; ++t)
                a += taps.w[t] * tile[(ly + R + taps.dy[t]) * TW + (lx + R + taps.dx[t])];
            z[i] = (T)a;
            acc[0] += a;
        }
        __syncthreads();
    }
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[2]) && threadIdx.x == 0) {
        st->zmean = st->nc ? (double)(T)(acc[0] / st->nc) : 0.0;
        st->pc++;
    }
}

inline int stencil_grid(int Ns) {
    const int n = ((Ns + kStX - 1) / kStX) * ((Ns + kStY - 1) / kStY);
    return n < kMaxBlocks ? n : kMaxBlocks;
}

// ---- CG passes (contact_solver.cpp:420-501) ------------------------------------
template <typename T>
__device__ __forceinline__ T zfinal(const PkParams& P, T z, T g, T zm) {
    return P.precond ? (T)(z - zm) : g;
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_dots(const PkParams* __restrict__ Pp, PkState* st, const T* z,
                                                      const T* g, const T* gprev,
                                                      const uint8_t* mask, double* part) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T zm = (T)st->zmean;
    double acc[3] = {0, 0, 0};  // G, G_pr, gg
    GRID_LOOP4(P.N) {
        T zz[4], gv[4], gp[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(g, i4, gv);
        ldp4(gprev, i4, gp);
        if (P.precond) ldp4(z, i4, zz);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!mm[j]) continue;
            const T zf = zfinal(P, zz[j], gv[j], zm);
            const double gd = (double)gv[j];
            acc[0] += (double)zf * gd;
            acc[1] += (double)zf * (double)(gv[j] - gp[j]);
            acc[2] += gd * gd;
        }
    }
    const int kinds[3] = {0, 0, 0};
    if (grid_reduce_last<3>(acc, kinds, part, &st->counter[3]) && threadIdx.x == 0) {
        const double G_old = st->G_old;
        const double bv = (G_old != 0.0) ? (P.use_pr ? fmax(0.0, acc[1] / G_old) : acc[0] / G_old)
                                         : 0.0;
        st->beta = (double)((T)st->delta * (T)bv);
        st->G_old = acc[0];
        st->gg = acc[2];
    }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_tupd(const PkParams* __restrict__ Pp, PkState* st, const T* z,
                                                      const T* g, T* gprev, T* t,
                                                      const uint8_t* mask, const T* p, T* best) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T zm = (T)st->zmean, beta = (T)st->beta;
    const int cb = st->copy_best;
    GRID_LOOP4(P.N) {
        T zz[4], gv[4], tt[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(g, i4, gv);
        ldp4(t, i4, tt);
        if (P.precond) ldp4(z, i4, zz);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            tt[j] = mm[j] ? (T)(zfinal(P, zz[j], gv[j], zm) + beta * tt[j]) : T(0);
        st4(t, i4, tt);
        st4(gprev, i4, gv);
        if (cb) {
            T pp[4];
            ldp4(p, i4, pp);
            st4(best, i4, pp);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_rsum(const PkParams* __restrict__ Pp, PkState* st, const T* r,
                                                      const T* g, const T* t,
                                                      const uint8_t* mask, double* part) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    double acc[2] = {0, 0};
    GRID_LOOP4(P.N) {
        T rr[4], gv[4], tt[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(r, i4, rr);
        ldp4(g, i4, gv);
        ldp4(t, i4, tt);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!mm[j]) continue;
            acc[0] += (double)rr[j];
            acc[1] += (double)gv[j] * (double)tt[j];
        }
    }
    const int kinds[2] = {0, 0};
    if (grid_reduce_last<2>(acc, kinds, part, &st->counter[4]) && threadIdx.x == 0) {
        st->mv++;
        if (st->copy_best) {
            st->copy_best = 0;
            st->have_best = 1;
        }
        st->rsum = acc[0];
        st->num = acc[1];
        st->rmean = (double)(T)(st->nc ? acc[0] / st->nc : 0.0);
    }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_den(const PkParams* __restrict__ Pp, PkState* st, const T* r,
                                                     const T* t, const uint8_t* mask,
                                                     double* part) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T rm = (T)st->rmean;
    double acc[1] = {0};
    GRID_LOOP4(P.N) {
        T rr[4], tt[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(r, i4, rr);
        ldp4(t, i4, tt);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (mm[j]) acc[0] += (double)(T)(rr[j] - rm) * (double)tt[j];
    }
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[5]) && threadIdx.x == 0) {
        const double den = acc[0], num = st->num;
        st->den = den;
        if (den > 0.0 && isfinite(den) && isfinite(num)) {
            const T tau = (T)(num / den);
            st->tau = (double)tau;
            st->tau_ov = st->gg > 0.0 ? (double)(T)(num * num / (den * st->gg)) : (double)tau;
        } else {
            set_halt(st, H_IDENT);  // no usable direction: identification step
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_pupd(const PkParams* __restrict__ Pp, PkState* st, T* p, const T* t,
                                                      const T* g, double* part) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T tau = (T)st->tau, tov = (T)st->tau_ov;
    double acc[2] = {0, 0};  // changed (max), total
    GRID_LOOP4(P.N) {
        T pp[4], tt[4], gv[4];
        ldp4(p, i4, pp);
        ldp4(t, i4, tt);
        ldp4(g, i4, gv);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T pi = pp[j];
            const bool was = pi > T(0);
            if (was) {
                const T q = pi - tau * tt[j];
                pi = q < T(0) ? T(0) : q;
            }
            if (pi == T(0) && gv[j] < T(0)) pi -= tov * gv[j];
            if ((pi > T(0)) != was) acc[0] = 1.0;
            pp[j] = pi;
            acc[1] += (double)pi;
        }
        st4(p, i4, pp);
    }
    const int kinds[2] = {2, 0};
    if (grid_reduce_last<2>(acc, kinds, part, &st->counter[6]) && threadIdx.x == 0) {
        st->delta = acc[0] > 0.0 ? 0.0 : 1.0;
        st->total = acc[1];
        if (acc[1] > 0.0) {
            st->scale = (double)(T)(P.P_total / acc[1]);
            st->fill = 0;
        } else {
            st->fill = 1;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_rescale(const PkParams* __restrict__ Pp, PkState* st, T* p,
                                                         double* part) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    const int fill = st->fill;
    const T f = (T)st->scale, pb = (T)P.p_bar;
    GRID_LOOP4(P.N) {
        T pp[4];
        ldp4(p, i4, pp);
#pragma unroll
        for (int j = 0; j < 4; ++j) pp[j] = fill ? pb : pp[j] * f;
        st4(p, i4, pp);
    }
    double acc[1] = {0};
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[7]) && threadIdx.x == 0) {
        st->it++;
        if (st->it >= P.max_iter) set_halt(st, H_FINAL);  // status stays max_iterations
    }
}

// ---- host-driven helpers (identification step, validation, outputs) -----------
// generic reduction: mode 0: [min g0, max g0, nonfinite count]
//                    1: [sum x]
//                    2: f_cur = sum p(0.5u + g0s), pp = sum p^2, pu = sum p u
//                    3: f_try = sum z(0.5r + g0s), gd = sum g (z - p)
//                    4: count/sum of x > theta
//                    5: objective = sum p(0.5u + g0s)
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_reduce(const PkParams* __restrict__ Pp, PkState* st, int mode,
                                                        const T* a, const T* b, const T* c,
                                                        const T* d, double theta,
                                                        double* part) {
    const PkParams& P = *Pp;
    const T gs = (T)P.gshift;
    double acc[3] = {0, 0, 0};
    if (mode == 0) { acc[0] = (double)INFINITY; acc[1] = -(double)INFINITY; }
    GRID_LOOP4(P.N) {
        T A[4], B[4], C[4], D[4];
        ldp4(a, i4, A);
        if (b) ldp4(b, i4, B);
        if (c) ldp4(c, i4, C);
        if (d) ldp4(d, i4, D);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double x = (double)A[j];
            switch (mode) {
                case 0:
                    acc[0] = fmin(acc[0], x);
                    acc[1] = fmax(acc[1], x);
                    if (!isfinite(x)) acc[2] += 1.0;
                    break;
                case 1: acc[0] += x; break;
                case 2:  // a=p b=u c=g0
                case 5:
                    acc[0] += x * (0.5 * (double)B[j] + (double)(T)(C[j] - gs));
                    acc[1] += x * x;
                    acc[2] += x * (double)B[j];
                    break;
                case 3:  // a=z b=r c=g0 d=g ; p in `d`? see host: d=g, p via theta-less extra
                    acc[0] += x * (0.5 * (double)B[j] + (double)(T)(C[j] - gs));
                    break;
                case 4:
                    if (x > theta) { acc[0] += x; acc[1] += 1.0; }
                    break;
            }
        }
    }
    int kinds[3] = {0, 0, 0};
    if (mode == 0) { kinds[0] = 1; kinds[1] = 2; }
    if (grid_reduce_last<3>(acc, kinds, part, &st->counter[8]) && threadIdx.x == 0) {
        st->red[0] = acc[0];
        st->red[1] = acc[1];
        st->red[2] = acc[2];
    }
}

// gd = sum double(g) * double(z - p)  (contact_solver.cpp:345-346)
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_gd(const PkParams* __restrict__ Pp, PkState* st, const T* g,
                                                    const T* z, const T* p, double* part) {
    const PkParams& P = *Pp;
    double acc[1] = {0};
    GRID_LOOP4(P.N) {
        T G[4], Z[4], Pp[4];
        ldp4(g, i4, G);
        ldp4(z, i4, Z);
        ldp4(p, i4, Pp);
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[0] += (double)G[j] * (double)(T)(Z[j] - Pp[j]);
    }
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[9]) && threadIdx.x == 0)
        st->red[3] = acc[0];
}

template <typename T>
__global__ void k_axpy_trial(long N, T* z, const T* p, const T* g, T s) {
    GRID_LOOP4(N) {
        T Pp[4], G[4], Z[4];
        ldp4(p, i4, Pp);
        ldp4(g, i4, G);
#pragma unroll
        for (int j = 0; j < 4; ++j) Z[j] = Pp[j] - s * G[j];
        st4(z, i4, Z);
    }
}

template <typename T>
__global__ void k_threshold(long N, T* z, T th) {
    GRID_LOOP4(N) {
        T Z[4];
        ldp4(z, i4, Z);
#pragma unroll
        for (int j = 0; j < 4; ++j) Z[j] = Z[j] > th ? (T)(Z[j] - th) : T(0);
        st4(z, i4, Z);
    }
}

template <typename T>
__global__ void k_fill(long N, T* x, T v) {
    GRID_LOOP4(N) {
        T X[4] = {v, v, v, v};
        st4(x, i4, X);
    }
}

template <typename T>
__global__ void k_clamp_pos(long N, T* x, const T* src) {
    GRID_LOOP4(N) {
        T X[4];
        ldp4(src, i4, X);
#pragma unroll
        for (int j = 0; j < 4; ++j) X[j] = X[j] < T(0) ? T(0) : X[j];  // cwiseMax(0)
        st4(x, i4, X);
    }
}

template <typename T>
__global__ void k_scale(long N, T* x, T f) {
    GRID_LOOP4(N) {
        T X[4];
        ldp4(x, i4, X);
#pragma unroll
        for (int j = 0; j < 4; ++j) X[j] = X[j] * f;
        st4(x, i4, X);
    }
}

template <typename T>
__global__ void k_to_f64(long N, double* out, const T* x) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        out[i] = (double)x[i];
}

// out = float(x - datum): the FP32 stage's gap, centred before the cast so a
// large datum is not rounded into the field (nested_solve.cpp:871-917)
__global__ void k_center_cast(long N, float* out, const double* x, double datum) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        out[i] = (float)(x[i] - datum);
}
__global__ void k_cast_f32(long N, float* out, const double* x) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        out[i] = (float)x[i];
}

// z[C] -= T(zmean) (the standalone preconditioner entry point)
template <typename T>
__global__ void k_sub_zmean(long N, T* z, const uint8_t* mask, const PkState* st) {
    const T zm = (T)st->zmean;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        if (mask[i]) z[i] = z[i] - zm;
}

// contact sum / count of g for the standalone preconditioner
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_gmean(long N, PkState* st, const T* g,
                                                       const uint8_t* mask, double* part) {
    double acc[2] = {0, 0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
        if (mask[i]) { acc[0] += (double)g[i]; acc[1] += 1.0; }
    const int kinds[2] = {0, 0};
    if (grid_reduce_last<2>(acc, kinds, part, &st->counter[10]) && threadIdx.x == 0) {
        st->gcs = acc[0];
        st->nc = (int)acc[1];
    }
}

// ---- device-side loop control -------------------------------------------------------
// Last kernel of the graph body: keep looping while no pass has set `halt`.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const PkState* st) {
    cudaGraphSetConditional(h, st->halt == H_RUN ? 1u : 0u);
}

// ---- host driver -----------------------------------------------------------------
namespace {

int red_grid(long N) {
    long g = (N / 4 + kRedThreads - 1) / kRedThreads;
    if (g > kMaxBlocks / 2) g = kMaxBlocks / 2;
    if (g < 1) g = 1;
    return (int)g;
}

// Per-operator, per-precision solver context: the CG workspace, the device
// parameter block and the instantiated loop graph (a while-conditional node
// whose body is one CG iteration), reused by every solve with the same
// preconditioner configuration.
template <typename T>
struct SolverCtx : SolverCtxBase {
    Operator& op;
    long N = 0;
    T *p = nullptr, *t = nullptr, *u = nullptr, *g = nullptr, *gprev = nullptr, *z = nullptr,
      *r = nullptr, *best = nullptr;
    T* g0c = nullptr;  // the solve's gap, copied in so the loop graph is reusable
    uint8_t* mask = nullptr;
    double* part = nullptr;
    double* hist = nullptr;
    int hist_cap = 0;
    PkState* st = nullptr;
    PkParams* Pd = nullptr;
    StencilTaps taps{};
    int precond = -1, radius = -1;
    int grid = 1;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    // Private non-blocking stream: the loop graph is captured and launched
    // here (the legacy NULL stream a caller may pass cannot be captured);
    // entry and exit are fenced to the caller's stream with events.
    cudaStream_t ws = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;

    explicit SolverCtx(Operator& o) : op(o) {
        ASB_CUDA(cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking));
        ASB_CUDA(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
        ASB_CUDA(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
        N = (long)o.Ns * o.Ns;
        const size_t b = (size_t)N * sizeof(T);
        T** vecs[] = {&p, &t, &u, &g, &gprev, &z, &r, &best, &g0c};
        for (T** v : vecs) ASB_CUDA(cudaMalloc((void**)v, b));
        ASB_CUDA(cudaMalloc((void**)&mask, (size_t)N));
        ASB_CUDA(cudaMalloc((void**)&part, kMaxBlocks * 8 * sizeof(double)));
        ASB_CUDA(cudaMalloc((void**)&st, sizeof(PkState)));
        ASB_CUDA(cudaMalloc((void**)&Pd, sizeof(PkParams)));
        ASB_CUDA(cudaMemset(st, 0, sizeof(PkState)));
        grid = red_grid(N);
        (void)o.spectrum(sizeof(T) == 8, nullptr);  // allocate before any capture
    }
    ~SolverCtx() override {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        void* all[] = {p, t, u, g, gprev, z, r, best, g0c, mask, part, hist, st, Pd};
        for (void* v : all)
            if (v) cudaFree(v);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (ws) cudaStreamDestroy(ws);
    }
    size_t bytes() const override {
        return (9 * sizeof(T) + 1) * (size_t)N + hist_cap * sizeof(double) +
               kMaxBlocks * 8 * sizeof(double);
    }
    void ensure_hist(int cap) {
        if (cap <= hist_cap) return;
        if (hist) ASB_CUDA(cudaFree(hist));
        ASB_CUDA(cudaMalloc((void**)&hist, (size_t)cap * sizeof(double)));
        hist_cap = cap;
        drop_graph();  // the graph bakes the history pointer
    }
    void invalidate() override { drop_graph(); }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    void configure(int pc, int R) {
        if (pc == precond && (pc != 1 || R == radius)) return;
        if (pc == 1) taps = make_stencil_taps(op.Ns, R);
        precond = pc;
        radius = R;
        drop_graph();
    }

    void apply(const T* x, T* y, const int* gate, cudaStream_t s) {
        op.matvec(sizeof(T) == 8, x, y, s, gate);
    }
    void precond_apply(const int* gate, cudaStream_t s) {
        if (precond == 1) {
            k_stencil<T><<<stencil_grid(op.Ns), 256, 0, s>>>(Pd, st, taps, g, mask, z, part,
                                                            gate != nullptr);
            count_launches(1);
            ASB_CUDA(cudaGetLastError());
        } else if (precond == 2) {
            fourier_precond_pk<T>(op, g, mask, st, z, part, s, gate);
        }
    }
    // one CG iteration (the common path), every pass gated on the device
    void enqueue_iteration(const T* g0, cudaStream_t s) {
        apply(p, u, &st->skip_mv1, s);
        k_eval1<T><<<grid, kRedThreads, 0, s>>>(Pd, st, u, g0, p, g, part, 0);
        k_eval2<T><<<grid, kRedThreads, 0, s>>>(Pd, st, p, g, mask, part, hist, 0);
        if (precond > 0) precond_apply(&st->halt, s);
        k_dots<T><<<grid, kRedThreads, 0, s>>>(Pd, st, z, g, gprev, mask, part);
        k_tupd<T><<<grid, kRedThreads, 0, s>>>(Pd, st, z, g, gprev, t, mask, p, best);
        apply(t, r, &st->halt, s);
        k_rsum<T><<<grid, kRedThreads, 0, s>>>(Pd, st, r, g, t, mask, part);
        k_den<T><<<grid, kRedThreads, 0, s>>>(Pd, st, r, t, mask, part);
        k_pupd<T><<<grid, kRedThreads, 0, s>>>(Pd, st, p, t, g, part);
        k_rescale<T><<<grid, kRedThreads, 0, s>>>(Pd, st, p, part);
        count_launches(8);
        ASB_CUDA(cudaGetLastError());
    }
    // Graph: while (halt == H_RUN) { iteration }.  The g0 pointer is baked
    // in, so the graph is rebuilt when a solve passes another gap buffer.
    const T* graph_g0 = nullptr;
    void build_graph(const T* g0, cudaStream_t s) {
        drop_graph();
        ASB_CUDA(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle h;
        ASB_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        ASB_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ASB_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeRelaxed));
        enqueue_iteration(g0, s);
        k_loop_cond<<<1, 1, 0, s>>>(h, st);
        cudaGraph_t captured = nullptr;
        ASB_CUDA(cudaStreamEndCapture(s, &captured));
        ASB_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        graph_g0 = g0;
    }
    // (Re)build the loop graph if needed.  Before capturing, one fully gated
    // iteration runs eagerly (every kernel returns at entry) so that all
    // function attributes are set outside the capture.  Clobbers st; the
    // caller writes the initial state afterwards.
    void ensure_graph(const T* g0, cudaStream_t s) {
        if (exec && graph_g0 == g0) return;
        PkState gated;
        std::memset(&gated, 0, sizeof(gated));
        gated.halt = H_FINAL;
        gated.skip_mv1 = 1;
        ASB_CUDA(cudaMemcpyAsync(st, &gated, sizeof(PkState), cudaMemcpyHostToDevice, s));
        enqueue_iteration(g0, s);
        ASB_CUDA(cudaStreamSynchronize(s));
        build_graph(g0, s);
    }
    void launch_graph(cudaStream_t s) {
        ASB_CUDA(cudaGraphLaunch(exec, s));
        count_launches(1);
    }
};

template <typename T>
struct Solver {
    SolverCtx<T>& c;
    PkParams P{};
    cudaStream_t s;
    PkState h{};  // host mirror
    const T* g0 = nullptr;
    long long mv_host = 0;

    cudaStream_t caller;
    // All work runs on the context's private stream, ordered after the
    // caller's pending work and before the caller's later work.
    Solver(SolverCtx<T>& ctx, cudaStream_t st) : c(ctx), s(ctx.ws), caller(st) {
        ASB_CUDA(cudaEventRecord(c.ev_in, caller));
        ASB_CUDA(cudaStreamWaitEvent(s, c.ev_in, 0));
    }
    ~Solver() {
        if (cudaEventRecord(c.ev_out, s) == cudaSuccess) cudaStreamWaitEvent(caller, c.ev_out, 0);
    }

    void read_state() {
        ASB_CUDA(cudaMemcpyAsync(&h, c.st, sizeof(PkState), cudaMemcpyDeviceToHost, s));
        ASB_CUDA(cudaStreamSynchronize(s));
    }
    void write_state() {
        ASB_CUDA(cudaMemcpyAsync(c.st, &h, sizeof(PkState), cudaMemcpyHostToDevice, s));
        ASB_CUDA(cudaStreamSynchronize(s));
    }
    // results of the helper reductions live in st->red; only that slice is
    // read back so the host mirror `h` is never clobbered mid-update
    void read_red(double (&r)[8]) {
        ASB_CUDA(cudaMemcpyAsync(r, c.st->red, sizeof(r), cudaMemcpyDeviceToHost, s));
        ASB_CUDA(cudaStreamSynchronize(s));
    }
    double reduce(int mode, const T* a, const T* b, const T* cc, const T* d, double theta,
                  double* out3 = nullptr) {
        k_reduce<T><<<c.grid, kRedThreads, 0, s>>>(c.Pd, c.st, mode, a, b, cc, d, theta, c.part);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
        double r[8];
        read_red(r);
        if (out3) { out3[0] = r[0]; out3[1] = r[1]; out3[2] = r[2]; }
        return r[0];
    }

    // project_load_simplex on c.z (contact_solver.cpp:31-60)
    void project_simplex(double P_total) {
        const long N = P.N;
        double ssum = reduce(1, c.z, nullptr, nullptr, nullptr, 0.0);
        long nact = N;
        double theta = (ssum - P_total) / (double)nact;
        for (int pass = 0; pass < 64; ++pass) {
            double o[3];
            reduce(4, c.z, nullptr, nullptr, nullptr, theta, o);
            const long n2 = (long)o[1];
            if (n2 == 0) break;
            if (n2 == nact) break;
            nact = n2;
            ssum = o[0];
            theta = (ssum - P_total) / (double)nact;
        }
        k_threshold<T><<<c.grid, kRedThreads, 0, s>>>(N, c.z, (T)theta);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
    }

    // identification step (contact_solver.cpp:314-364); host mirror h is current
    bool identification_step(double& s_id, int& id_steps) {
        double o[3];
        reduce(2, c.p, c.u, g0, nullptr, 0.0, o);
        const double f_cur = o[0];
        if (!(s_id > 0.0)) {
            const double pp = o[1], pu = o[2];
            s_id = (pu > 0.0 && pp > 0.0) ? pp / pu : 1.0;
        }
        for (int trial = 0; trial < 12; ++trial) {
            k_axpy_trial<T><<<c.grid, kRedThreads, 0, s>>>(P.N, c.z, c.p, c.g, (T)s_id);
            count_launches(1);
            project_simplex(P.P_total);
            c.apply(c.z, c.r, nullptr, s);
            mv_host++;
            reduce(3, c.z, c.r, g0, nullptr, 0.0, o);
            const double f_try = o[0];
            k_gd<T><<<c.grid, kRedThreads, 0, s>>>(c.Pd, c.st, c.g, c.z, c.p, c.part);
            count_launches(1);
            double rr[8];
            read_red(rr);
            const double gd = rr[3];
            if (std::isfinite(f_try) && gd < 0.0 && f_try <= f_cur + 1e-4 * gd) {
                const size_t b = (size_t)P.N * sizeof(T);
                ASB_CUDA(cudaMemcpyAsync(c.p, c.z, b, cudaMemcpyDeviceToDevice, s));
                ASB_CUDA(cudaMemcpyAsync(c.u, c.r, b, cudaMemcpyDeviceToDevice, s));
                ASB_CUDA(cudaMemsetAsync(c.t, 0, b, s));
                ASB_CUDA(cudaMemsetAsync(c.gprev, 0, b, s));
                h.u_fresh = 1;
                h.delta = 0.0;
                h.G_old = 1.0;
                ++id_steps;
                if (trial == 0) s_id *= 2.0;
                return true;
            }
            s_id *= 0.25;
        }
        return false;
    }

    void run(const aspher_solve_opts& o, const T* g0_, double p_bar, const T* p_init,
             double* pressure, double* disp, double* gap, double* hist_host, int hist_cap,
             aspher_result& res) {
        const auto t_start = std::chrono::steady_clock::now();
        const int Ns = c.op.Ns;
        const long N = (long)Ns * Ns;
        // the caller's gap is read once into the context (zero-copy is not
        // needed on a 180 GB device, and a fixed address keeps the graph valid)
        if (g0_ != c.g0c)
            ASB_CUDA(cudaMemcpyAsync(c.g0c, g0_, (size_t)N * sizeof(T), cudaMemcpyDeviceToDevice,
                                     s));
        g0 = c.g0c;
        constexpr bool is_double = sizeof(T) == 8;
        if (!(p_bar > 0.0) || !std::isfinite(p_bar))
            throw Error(ASPHER_EINVAL, "solve_contact: empty gap or p_bar <= 0");
        if (!(o.tol > 0.0)) throw Error(ASPHER_EINVAL, "solve_contact: tol must be positive");
        if (o.max_iter < 0) throw Error(ASPHER_EINVAL, "solve_contact: max_iter must be >= 0");
        if (o.precond < 0 || o.precond > 2) throw Error(ASPHER_EINVAL, "solve_contact: bad precond");
        c.configure(o.precond, o.precond_radius);
        if (o.record_history) c.ensure_hist(o.max_iter + 1);
        P.N = N;
        P.Ns = Ns;
        // validation before any operator apply (contact_solver.cpp:159-168)
        double mm[3];
        ASB_CUDA(cudaMemcpyAsync(c.Pd, &P, sizeof(PkParams), cudaMemcpyHostToDevice, s));
        reduce(0, g0, nullptr, nullptr, nullptr, 0.0, mm);
        if (mm[2] > 0.0) throw Error(ASPHER_EINVAL, "solve_contact: g0 contains non-finite values");
        const double P_total = (double)(T)p_bar * (double)N;
        const double gmin_v = mm[0], gmax_v = mm[1];
        double g_ref = o.g_ref;
        if (!(g_ref > 0.0)) g_ref = gmax_v - gmin_v;
        if (!(g_ref > 0.0)) g_ref = 1.0;
        const double p_ref = o.p_ref > 0.0 ? o.p_ref : (double)(T)p_bar;
        const double load_tol = o.load_tol > 0.0 ? o.load_tol : (is_double ? 1e-12 : 5e-7);
        const double tol = o.tol;
        const double req_tol = o.requested_tol > 0.0 ? o.requested_tol : tol;
        double datum = 0.0;
        bool subtract = false;
        if (o.datum_mode == ASPHER_DATUM_AUTOMATIC) {
            datum = gmin_v + 0.5 * (gmax_v - gmin_v);
            subtract = true;
        } else if (o.datum_mode == ASPHER_DATUM_SOLVER) {
            datum = o.datum;
            subtract = true;
        } else {
            datum = o.datum;
        }
        P.max_iter = o.max_iter;
        P.stall_limit = o.stall_limit > 0 ? o.stall_limit : 200;
        P.keep_best = o.keep_best;
        P.record_history = o.record_history && c.hist_cap > 0;
        P.use_pr = o.use_pr;
        P.precond = o.precond;
        P.P_total = P_total;
        P.g_ref = g_ref;
        P.tol = tol;
        P.load_tol = load_tol;
        P.p_bar = (double)(T)p_bar;
        P.gshift = subtract ? (double)(T)datum : 0.0;
        ASB_CUDA(cudaMemcpyAsync(c.Pd, &P, sizeof(PkParams), cudaMemcpyHostToDevice, s));

        // initial pressure (contact_solver.cpp:204-223)
        const T pb = (T)p_bar;
        if (p_init) {
            k_clamp_pos<T><<<c.grid, kRedThreads, 0, s>>>(N, c.p, p_init);
            count_launches(1);
            const double ssum = reduce(1, c.p, nullptr, nullptr, nullptr, 0.0);
            if (ssum > 0.0) k_scale<T><<<c.grid, kRedThreads, 0, s>>>(N, c.p, (T)(P_total / ssum));
            else k_fill<T><<<c.grid, kRedThreads, 0, s>>>(N, c.p, pb);
        } else {
            k_fill<T><<<c.grid, kRedThreads, 0, s>>>(N, c.p, pb);
        }
        count_launches(1);
        ASB_CUDA(cudaMemsetAsync(c.t, 0, (size_t)N * sizeof(T), s));
        ASB_CUDA(cudaMemsetAsync(c.gprev, 0, (size_t)N * sizeof(T), s));
        ASB_CUDA(cudaMemsetAsync(c.z, 0, (size_t)N * sizeof(T), s));
        std::memset(&h, 0, sizeof(h));
        h.G_old = 1.0;
        h.delta = 0.0;
        h.best_merit = std::numeric_limits<double>::infinity();
        h.seen_merit = std::numeric_limits<double>::infinity();
        h.status = ST_MAX_ITERATIONS;
        h.halt = o.max_iter > 0 ? H_RUN : H_FINAL;
        h.skip_mv1 = h.halt ? 1 : 0;
        c.ensure_graph(g0, s);
        write_state();

        double s_id = 0.0;
        int forced_id = 0, id_steps = 0;
        std::string reason;
        while (h.halt == H_RUN) {
            c.launch_graph(s);
            read_state();
            if (h.halt == H_RUN || h.halt == H_FINAL) break;
            if (h.copy_best) {
                ASB_CUDA(cudaMemcpyAsync(c.best, c.p, (size_t)N * sizeof(T),
                                         cudaMemcpyDeviceToDevice, s));
                h.copy_best = 0;
                h.have_best = 1;
            }
            if (h.halt == H_STALL) {
                if (forced_id < 3 && identification_step(s_id, id_steps)) {
                    ++forced_id;
                    h.stall = 0;
                } else {
                    h.status = ST_STAGNATED;
                    reason = "stall";
                    h.halt = H_FINAL;
                    break;
                }
            } else if (h.halt == H_IDENT) {
                if (!identification_step(s_id, id_steps)) {
                    h.status = ST_NONPOSITIVE_CURVATURE;
                    h.halt = H_FINAL;
                    break;
                }
            }
            // resume: the loop body's end increments the iteration counter
            h.it++;
            h.mv += mv_host;
            mv_host = 0;
            if (h.it >= o.max_iter) {
                h.halt = H_FINAL;
                break;
            }
            h.halt = H_RUN;
            h.skip_mv1 = h.u_fresh ? 1 : 0;
            write_state();
        }
        h.mv += mv_host;
        mv_host = 0;
        int status = h.status;
        // ---- final, freshly evaluated diagnostics (contact_solver.cpp:518-586)
        bool returned_best = false;
        if (status != ST_CONVERGED && o.keep_best && h.have_best) {
            const double merit = std::max(h.fw, h.pen);
            if (!(merit <= h.best_merit)) {
                ASB_CUDA(cudaMemcpyAsync(c.p, c.best, (size_t)N * sizeof(T),
                                         cudaMemcpyDeviceToDevice, s));
                h.u_fresh = 0;
                returned_best = true;
            }
        }
        if (!h.u_fresh) {
            c.apply(c.p, c.u, nullptr, s);
            h.mv++;
        }
        h.halt = H_FINAL;
        write_state();
        k_eval1<T><<<c.grid, kRedThreads, 0, s>>>(c.Pd, c.st, c.u, g0, c.p, c.g, c.part, 1);
        k_eval2<T><<<c.grid, kRedThreads, 0, s>>>(c.Pd, c.st, c.p, c.g, c.mask, c.part, nullptr, 1);
        count_launches(2);
        ASB_CUDA(cudaGetLastError());
        read_state();
        if (!h.finite && status != ST_NONFINITE) status = ST_NONFINITE;
        if (status == ST_CONVERGED && !(h.load <= load_tol && h.fw <= tol && h.pen <= tol)) {
            status = ST_VERIFICATION_FAILED;
            reason = "final_check";
        }
        if (status == ST_CONVERGED && req_tol < tol && !o.allow_tolerance_relaxation) {
            if (!(h.fw <= req_tol && h.pen <= req_tol)) {
                status = ST_STAGNATED;
                reason = "precision_limit";
            }
        }
        double ob[3];
        reduce(5, c.p, c.u, g0, nullptr, 0.0, ob);
        k_to_f64<T><<<c.grid, kRedThreads, 0, s>>>(N, pressure, c.p);
        count_launches(1);
        if (!o.light) {
            if (disp) { k_to_f64<T><<<c.grid, kRedThreads, 0, s>>>(N, disp, c.u); count_launches(1); }
            if (gap) { k_to_f64<T><<<c.grid, kRedThreads, 0, s>>>(N, gap, c.g); count_launches(1); }
        }
        ASB_CUDA(cudaGetLastError());
        int hl = 0;
        if (o.record_history && hist_host && hist_cap > 0 && c.hist_cap > 0) {
            hl = std::min(h.it, hist_cap);
            if (hl > 0)
                ASB_CUDA(cudaMemcpyAsync(hist_host, c.hist, hl * sizeof(double),
                                         cudaMemcpyDeviceToHost, s));
        }
        ASB_CUDA(cudaStreamSynchronize(s));

        std::memset(&res, 0, sizeof(res));
        res.status = status;
        std::strncpy(res.status_reason, reason.c_str(), sizeof(res.status_reason) - 1);
        res.iterations = h.it;
        res.converged = status == ST_CONVERGED;
        res.contact_fraction = (double)h.nc / (double)N;
        res.mean_pressure = h.psum / (double)N;
        res.approach = h.alpha_ref + datum;
        res.objective = ob[0] + datum * P_total;
        res.error = h.pk;
        res.pk_error = h.pk;
        res.fw_gap = h.G;
        res.fw_error = h.fw;
        res.load_error = h.load;
        res.pressure_violation = 0.0;
        res.penetration_error = h.pen;
        res.requested_tol = req_tol;
        res.effective_tol = tol;
        res.p_ref = p_ref;
        res.g_ref = g_ref;
        res.matvec_count = h.mv;
        res.precond_count = h.pc;
        res.identification_steps = id_steps;
        res.returned_best = returned_best;
        res.history_len = hl;
        const long long rb = sizeof(T);
        res.mem_cg_state = 7LL * N * rb;
        res.mem_best_iterate = o.keep_best ? N * rb : 0;
        res.mem_contact_mask = N;
        res.mem_output_arrays = (rb == 8 ? 0 : N * 8LL) + (o.light ? 0 : 2LL * N * 8);
        res.mem_peak = res.mem_cg_state + res.mem_best_iterate + res.mem_contact_mask +
                       res.mem_output_arrays;
        res.time_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start)
                             .count();
    }
};

template <typename T>
SolverCtx<T>& get_ctx(Operator& op) {
    std::shared_ptr<SolverCtxBase>& slot = sizeof(T) == 8 ? op.ctx_d : op.ctx_f;
    if (!slot) slot = std::make_shared<SolverCtx<T>>(op);
    return static_cast<SolverCtx<T>&>(*slot);
}

}  // namespace

namespace {
// w(dx, dy) of the |k| kernel on the Nw^2 grid: the c2r of |k| (DC zeroed) by
// direct summation over the half spectrum (kx = 0 and Nw/2 counted once).
long double kgrid_value(int Nw, int dx, int dy) {
    const int nh = Nw / 2 + 1;
    long double acc = 0.0L;
    const long double tp = 2.0L * 3.14159265358979323846264338327950288L / Nw;
    for (int ky = 0; ky < Nw; ++ky) {
        const int kof = ky < Nw / 2 ? ky : ky - Nw;
        for (int kx = 0; kx < nh; ++kx) {
            if (kx == 0 && ky == 0) continue;
            const long double mag = std::sqrt((long double)kx * kx + (long double)kof * kof);
            const long double wt = (kx == 0 || 2 * kx == Nw) ? 1.0L : 2.0L;
            acc += wt * mag * std::cos(tp * ((long double)kx * dx + (long double)ky * dy));
        }
    }
    return acc;
}
std::mutex g_taps_mu;
std::map<std::pair<int, int>, StencilTaps> g_taps_cache;
}  // namespace

StencilTaps make_stencil_taps(int Ns, int R) {
    if (R < 1) throw Error(ASPHER_EINVAL, "stencil radius must be >= 1");
    if (R > kMaxR) throw Error(ASPHER_EINVAL, "stencil radius must be <= 4");
    if (2 * R + 1 > Ns) throw Error(ASPHER_EINVAL, "stencil radius too large for the grid");
    // The kernel shape is taken on min(Ns, 512) (stencil_precond.cpp:199-220).
    const int Nw = Ns < 512 ? Ns : 512;
    {
        std::lock_guard<std::mutex> lk(g_taps_mu);
        auto it = g_taps_cache.find({Nw, R});
        if (it != g_taps_cache.end()) return it->second;
    }
    StencilTaps t{};
    t.R = R;
    t.n = 0;
    const long double c0 = kgrid_value(Nw, 0, 0);
    std::map<std::pair<int, int>, double> uniq;  // w depends on (|dx|, |dy|) only
    for (int dy = -R; dy <= R; ++dy)
        for (int dx = -R; dx <= R; ++dx) {
            if (dx * dx + dy * dy > R * R) continue;
            const std::pair<int, int> key{std::abs(dx), std::abs(dy)};
            auto u = uniq.find(key);
            double v;
            if (dx == 0 && dy == 0) v = 1.0;
            else if (u != uniq.end()) v = u->second;
            else v = uniq[key] = (double)(kgrid_value(Nw, key.first, key.second) / c0);
            t.dx[t.n] = dx;
            t.dy[t.n] = dy;
            t.w[t.n] = v;
            ++t.n;
        }
    std::lock_guard<std::mutex> lk(g_taps_mu);
    g_taps_cache[{Nw, R}] = t;
    return t;
}

template <typename T>
void solve_impl(Operator& op, const aspher_solve_opts& o, const void* g0, double p_bar,
                const void* p_init, double* pressure, double* disp, double* gap, double* hist,
                int hist_cap, aspher_result& res, cudaStream_t s) {
    Solver<T> S(get_ctx<T>(op), s);
    S.run(o, (const T*)g0, p_bar, (const T*)p_init, pressure, disp, gap, hist, hist_cap, res);
}
template void solve_impl<float>(Operator&, const aspher_solve_opts&, const void*, double,
                                const void*, double*, double*, double*, double*, int,
                                aspher_result&, cudaStream_t);
template void solve_impl<double>(Operator&, const aspher_solve_opts&, const void*, double,
                                 const void*, double*, double*, double*, double*, int,
                                 aspher_result&, cudaStream_t);


// FP32 stage + FP64 polish (the reference's float_then_double staging,
// nested_solve.cpp:871-974, on one level): the gap is centred by its
// midpoint datum and cast to FP32 on the device, the FP32 PK solve runs to
// float_tol with FP64 reductions, and -- when polish -- an FP64 PK solve
// warm-started from that pressure certifies the requested tol.
void solve_mixed(Operator& op, const aspher_solve_opts& o, const double* g0, double p_bar,
                 const double* p_init, double float_tol, int polish, double* pressure,
                 double* disp, double* gap, aspher_result& res, aspher_result* res_float,
                 cudaStream_t s) {
    SolverCtx<double>& cd = get_ctx<double>(op);
    SolverCtx<float>& cf = get_ctx<float>(op);
    const long N = (long)op.Ns * op.Ns;
    // FP64 statistics of the gap (validation before any apply)
    double mm[3];
    {
        Solver<double> probe(cd, s);
        probe.P.N = N;
        probe.P.Ns = op.Ns;
        ASB_CUDA(cudaMemcpyAsync(cd.Pd, &probe.P, sizeof(PkParams), cudaMemcpyHostToDevice,
                                 probe.s));
        probe.reduce(0, g0, nullptr, nullptr, nullptr, 0.0, mm);
    }
    if (mm[2] > 0.0) throw Error(ASPHER_EINVAL, "solve_contact: g0 contains non-finite values");
    const double datum = o.datum_mode == ASPHER_DATUM_AUTOMATIC ? mm[0] + 0.5 * (mm[1] - mm[0])
                                                                 : o.datum;
    double g_ref = o.g_ref;
    if (!(g_ref > 0.0)) g_ref = mm[1] - mm[0];
    if (!(g_ref > 0.0)) g_ref = 1.0;
    const int grid = red_grid(N);
    k_center_cast<<<grid, kRedThreads, 0, s>>>(N, cf.g0c, g0, o.datum_mode == ASPHER_DATUM_CALLER ? 0.0 : datum);
    count_launches(1);
    float* pinit_f = nullptr;
    if (p_init) {
        pinit_f = cf.r;  // scratch: read by the FP32 solve before r is first written
        k_cast_f32<<<grid, kRedThreads, 0, s>>>(N, pinit_f, p_init);
        count_launches(1);
    }
    ASB_CUDA(cudaGetLastError());
    aspher_solve_opts of = o;
    of.dtype = ASPHER_F32;
    of.tol = float_tol;
    of.requested_tol = polish ? float_tol : (o.requested_tol > 0.0 ? o.requested_tol : o.tol);
    of.allow_tolerance_relaxation = polish ? 1 : o.allow_tolerance_relaxation;
    of.datum_mode = ASPHER_DATUM_CALLER;
    of.datum = datum;
    of.g_ref = g_ref;
    of.light = polish ? 1 : o.light;
    aspher_result rf;
    {
        Solver<float> S(cf, s);
        S.run(of, cf.g0c, p_bar, pinit_f, pressure, polish ? nullptr : disp,
              polish ? nullptr : gap, nullptr, 0, rf);
    }
    if (res_float) *res_float = rf;
    if (!polish) {
        res = rf;
        return;
    }
    aspher_solve_opts od = o;
    od.dtype = ASPHER_F64;
    od.datum_mode = ASPHER_DATUM_SOLVER;
    od.datum = datum;
    od.g_ref = g_ref;
    {
        Solver<double> S(cd, s);
        S.run(od, g0, p_bar, pressure, pressure, disp, gap, nullptr, 0, res);
    }
    // the reported work is the sum of both stages (nested_solve.cpp:445-450)
    res.iterations += rf.iterations;
    res.matvec_count += rf.matvec_count;
    res.precond_count += rf.precond_count;
    res.identification_steps += rf.identification_steps;
    res.time_total += rf.time_total;
}

// Standalone preconditioner apply: z = M^-1 g on contact, contact-mean removed.
template <typename T>
void precond_apply_impl(Operator& op, int precond, int radius, const T* g,
                        const uint8_t* mask, T* z, cudaStream_t s) {
    const long N = (long)op.Ns * op.Ns;
    PkState* st = nullptr;
    double* part = nullptr;
    ASB_CUDA(cudaMallocAsync((void**)&st, sizeof(PkState), s));
    ASB_CUDA(cudaMallocAsync((void**)&part, kMaxBlocks * 8 * sizeof(double), s));
    ASB_CUDA(cudaMemsetAsync(st, 0, sizeof(PkState), s));
    PkParams P{};
    P.N = N;
    P.Ns = op.Ns;
    P.precond = precond;
    PkParams* Pd = nullptr;
    ASB_CUDA(cudaMallocAsync((void**)&Pd, sizeof(PkParams), s));
    ASB_CUDA(cudaMemcpyAsync(Pd, &P, sizeof(PkParams), cudaMemcpyHostToDevice, s));
    const int grid = red_grid(N);
    k_gmean<T><<<grid, kRedThreads, 0, s>>>(N, st, g, mask, part);
    if (precond == 1) {
        StencilTaps taps = make_stencil_taps(op.Ns, radius);
        k_stencil<T><<<stencil_grid(op.Ns), 256, 0, s>>>(Pd, st, taps, g, mask, z, part, 0);
        count_launches(1);
    } else {
        fourier_precond_pk<T>(op, g, mask, st, z, part, s, nullptr);
    }
    k_sub_zmean<T><<<grid, kRedThreads, 0, s>>>(N, z, mask, st);
    count_launches(2);
    ASB_CUDA(cudaGetLastError());
    ASB_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(st, s);
    cudaFreeAsync(part, s);
    cudaFreeAsync(Pd, s);
    ASB_CUDA(cudaStreamSynchronize(s));
}
template void precond_apply_impl<float>(Operator&, int, int, const float*, const uint8_t*, float*,
                                        cudaStream_t);
template void precond_apply_impl<double>(Operator&, int, int, const double*, const uint8_t*,
                                         double*, cudaStream_t);

}  // namespace asb
