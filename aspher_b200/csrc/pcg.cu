// Polonsky-Keer projected CG with certified termination on the device.
//
// Reference: solve_contact_impl<Real> (src/contact_solver.cpp:150-587),
// project_load_simplex (:31-60), identification step (:314-364),
// evaluate()/refine_contact_mean (:69-99, :260-303).  Real = T in {float,
// double}; every reduction is accumulated in FP64 as in the reference.
//
// One CG iteration is the kernel sequence
//   [apply p->u] eval [evalpk] stencil+dots tupd [apply t->r] rden pupd
// where each pass is one HBM sweep and each reduction's scalar logic runs in
// the last block of its pass (see pk_state.hpp).  The loop is a CUDA graph
// with a while node; once a pass sets `halt`, the rest of the iteration is a
// no-op.  Every kernel serves B instances at once (gridDim.y = B, instance
// blockIdx.y reading its own parameters, state, partials and fields).
#include "../../include/aspher_b200.h"
#include "ops.hpp"
#include "pk_state.hpp"
#include "pcg.hpp"
#include "embed.cuh"
#include "reduce.cuh"

#include <algorithm>
#include <map>
#include <tuple>
#include <utility>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
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


// ---- evaluate() -----------------------------------------------------------------
// The gap buffer holds v = u + (g0 - gshift) uncentred after k_eval; every
// later consumer centres on the fly with gc(), which is bit-identical to the
// reference's stored g = Real(v - Real(alpha)) (contact_solver.cpp:283-285),
// so centring costs no pass of its own.
template <typename T>
__device__ __forceinline__ T gc(T v, T aT) { return v - aT; }

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

// The pending load rescale of an instance (PkState::scale / scale_add),
// read once at kernel entry: the iterate is Real(x f) + a of the stored x
// (bit-identical to the reference's p(i) *= f, where a = 0).
template <typename T>
struct PScale {
    T f, a;
    __device__ explicit PScale(const PkState* st) : f((T)st->scale), a((T)st->scale_add) {}
    __device__ __forceinline__ T operator()(T x) const { return x * f + a; }
};

// One pass for evaluate() (contact_solver.cpp:263-303): v -> g buffer, the
// contact mask, and the sums whose last-block logic is the certificate, the
// convergence test and the best/stall bookkeeping (contact_solver.cpp:379-412).
// The second-pass sums of the reference are linear in the centring, so they
// come from first-pass sums:
//   gcs = sum_C Real(v - a)            -> sum_C v - n_C a
//   G   = sum p Real(Real(v - a) - m)  -> sum p v - (a + m) sum p
// with a = Real(alpha), m = Real(gmin) (equal up to the rounding of each
// Real difference; in FP64 to ~1e-16 relative).  pk = sum p |g| is not
// linear; k_evalpk computes it when a history is recorded and at the end.
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_eval(const PkParams* __restrict__ Pp, PkState* st,
                                                      const T* u, const T* g0, const T* p, T* g,
                                                      uint8_t* mask, double* part,
                                                      int final_mode) {
    // instance blockIdx.y of a batched solve (0 when unbatched)
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    u += bo_;
    g0 += bo_;
    p += bo_;
    g += bo_;
    mask += bo_;
    const PkParams& P = *Pp;
    if (!final_mode && st->halt) return;
    const T gs = (T)P.gshift;
    const PScale<T> ps(st);
    double acc[5] = {0.0, 0.0, (double)INFINITY, 0.0, 0.0};  // sum_C v, n_C, min v, pv, psum
    GRID_LOOP4(P.N) {
        T uu[4], gg0[4], pp[4], vv[4];
        uint8_t mm[4];
        ldp4(u, i4, uu);
        ldp4(g0, i4, gg0);
        ldp4(p, i4, pp);
#pragma unroll
        for (int j = 0; j < 4; ++j) pp[j] = ps(pp[j]);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const T v = uu[j] + (gg0[j] - gs);
            vv[j] = v;
            const double vd = (double)v, pd = (double)pp[j];
            acc[2] = fmin(acc[2], vd);
            if (pp[j] > T(0)) { acc[0] += vd; acc[1] += 1.0; }
            acc[3] += pd * vd;
            acc[4] += pd;
            mm[j] = pp[j] > T(0) ? 1 : 0;
        }
        st4(g, i4, vv);
        stm4(mask, i4, mm);
    }
    const int kinds[5] = {0, 0, 1, 0, 0};
    if (grid_reduce_last<5>(acc, kinds, part, &st->counter[0]) && threadIdx.x == 0) {
        if (!final_mode) {
            if (!st->u_fresh) st->mv++;
            st->u_fresh = 0;
            st->skip_mv1 = 0;
            st->pk_due = 1;
        }
        const int nc = (int)acc[1];
        const double alpha = nc ? acc[0] / nc : acc[2];
        const double gmin = acc[2] - alpha;
        const double aT = (double)(T)alpha, gmT = (double)(T)gmin;
        const double gcs = acc[0] - (double)nc * aT;
        st->nc = nc;
        st->gsum = acc[0];
        st->vmin = acc[2];
        st->alpha = alpha;
        st->gmin = gmin;
        double ar = alpha, gr = gmin;
        if (nc > 0) {  // refine_contact_mean (contact_solver.cpp:94-99)
            const double d = gcs / nc;
            ar += d;
            gr -= d;
        }
        const double PG = P.P_total * P.g_ref;
        const double G = acc[3] - (aT + gmT) * acc[4];
        st->alpha_ref = ar;
        st->gmin_ref = gr;
        st->pv = acc[3];
        st->gcs = gcs;
        st->G = G;
        st->fw = G / PG;
        st->pen = fmax(0.0, -gr) / P.g_ref;
        st->psum = acc[4];
        st->load = fabs(acc[4] - P.P_total) / P.P_total;
        st->finite = isfinite(acc[0]) && isfinite(acc[2]) && isfinite(acc[4]) && isfinite(acc[3]);
        if (final_mode) return;
        if (!st->finite) {
            st->status = ST_NONFINITE;
            set_halt(st, H_FINAL);
            return;
        }
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

// pk = sum p |g| / (P g_ref) (the reference's legacy error, reported and
// recorded in the history); runs after k_eval of a recorded iteration
// (pk_due) or in final mode.
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_evalpk(const PkParams* __restrict__ Pp, PkState* st,
                                                        const T* p, const T* g, double* part,
                                                        double* hist, int final_mode) {
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    p += bo_;
    g += bo_;
    const PkParams& P = *Pp;
    if (!final_mode && !st->pk_due) return;
    const T aT = (T)st->alpha;
    const PScale<T> ps(st);
    double acc[1] = {0.0};
    GRID_LOOP4(P.N) {
        T pp[4], gv[4];
        ldp4(p, i4, pp);
        ldp4(g, i4, gv);
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[0] += (double)ps(pp[j]) * fabs((double)gc(gv[j], aT));
    }
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[12]) && threadIdx.x == 0) {
        st->pk = acc[0] / (P.P_total * P.g_ref);
        st->finite = st->finite && isfinite(acc[0]);
        if (final_mode) return;
        st->pk_due = 0;
        if (P.record_history && hist) hist[blockIdx.y * P.hist_stride + st->it] = st->pk;
    }
}

// g <- centred gap (materialised for the host-side branches and the output)
template <typename T>
__global__ void k_center(const PkParams* __restrict__ Pp, const PkState* st, T* g) {
    Pp += blockIdx.y;
    st += blockIdx.y;
    g += (long)blockIdx.y * Pp->N;
    const T aT = (T)st->alpha;
    GRID_LOOP4(Pp->N) {
        T gv[4];
        ldp4(g, i4, gv);
#pragma unroll
        for (int j = 0; j < 4; ++j) gv[j] = gc(gv[j], aT);
        st4(g, i4, gv);
    }
}

// PR+ / FR ratio from G = <zf, g>, G_pr = <zf, g - g_prev> (contact_solver.cpp:420-446);
// beta = Real(delta) * Real(ratio) is formed by the caller
__device__ __forceinline__ void beta_update(const PkParams& P, PkState* st, double G, double Gpr,
                                            double gg) {
    const double G_old = st->G_old;
    const double bv = (G_old != 0.0) ? (P.use_pr ? fmax(0.0, Gpr / G_old) : G / G_old) : 0.0;
    st->G_old = G;
    st->gg = gg;
    st->bv = bv;
}

// ---- stencil preconditioner (stencil_precond.cpp:63-109) ---------------------
// z = T(sum_t w_t gc(i + d_t)) on contact, gc = contact ? g - gmean : 0 with
// periodic wrap; the contact mean of z is removed downstream.  A CTA of 256
// threads owns a 64 x 32 tile of outputs whose (64 + 2R) x (32 + 2R) halo
// of centred values sits in shared memory (FP64, as the reference
// accumulates); thread (x, q) computes the 8 outputs (x, 8q .. 8q + 7) with
// the disc's taps unrolled at compile time (R is a template parameter) and
// summed in the reference's tap order (dy-major, dx-minor).
constexpr int kStX = 64, kStY = 32, kStRows = 8, kMaxR = 4;

// the disc's weights by signed offset, w[dy + kMaxR][dx + kMaxR] (even in
// each offset on an even kernel grid; on an odd one the reference's
// wavenumber convention leaves them slightly uneven)
struct StencilW {
    double w[2 * kMaxR + 1][2 * kMaxR + 1];
};

// LAZY: g holds v uncentred (the solve loop; centred by Real(alpha) on the
// fly), else g is used as given (standalone preconditioner, adjoint).
// DOTS: also the CG dots of the loop -- with zf = Real(z - zm) the
// contact-mean-free direction,
//   G = sum_C zf g,  G_pr = sum_C zf Real(g - gprev),  gg = sum_C g^2,
// from sums linear in zm (zm is this pass's own reduction):
//   G = sum_C z g - zm sum_C g,  G_pr = sum_C z (g - gprev) - zm sum_C (g - gprev).
template <typename T, int R, bool LAZY, bool DOTS>
__global__ void __launch_bounds__(256) k_stencil_t(const PkParams* __restrict__ Pp, PkState* st,
                                                   StencilW W, const T* g, const T* gprev,
                                                   const uint8_t* mask, T* z, double* part,
                                                   int gated) {
    // instance blockIdx.y of a batched solve (0 when unbatched)
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    g += bo_;
    mask += bo_;
    z += bo_;
    if (DOTS) gprev += bo_;
    const PkParams& P = *Pp;
    if (gated && st->halt) return;
    constexpr int TW = kStX + 2 * R, TH = kStY + 2 * R;
    __shared__ double tile[TH * TW];
    // Nw: the periodic grid of the wrap (the caller's side; Ns, the row
    // pitch, unless the operator is embedded)
    const int Ns = P.Ns, Nw = P.Nl;
    // halo coordinates run from -R to the last tile's end (up to 63 + R past
    // Nw); 2R + 1 <= Nw
    auto wrap = [Nw](int v) { return v < 0 ? v + Nw : v % Nw; };
    const double gmean = st->nc ? st->gcs / st->nc : 0.0;
    const T aT = LAZY ? (T)st->alpha : T(0);
    const int ntx = (Nw + kStX - 1) / kStX, nty = (Nw + kStY - 1) / kStY;
    const int tx = threadIdx.x % kStX, tq = threadIdx.x / kStX;
    // sum z (unrounded), sum zT g, sum g, sum zT (g - gp), sum (g - gp), sum g^2
    double acc[DOTS ? 6 : 1];
#pragma unroll
    for (int i = 0; i < (DOTS ? 6 : 1); ++i) acc[i] = 0.0;
    // each thread issues all of its loads before it uses any (none depends
    // on another), so a tile costs about one memory latency, not one per
    // element
    constexpr int NL = (TW * TH + 255) / 256;  // halo elements per thread
    for (int tid = blockIdx.x; tid < ntx * nty; tid += gridDim.x) {
        const int tx0 = (tid % ntx) * kStX, ty0 = (tid / ntx) * kStY;
        T hv[NL];
        uint8_t hm[NL];
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int idx = threadIdx.x + u * 256;
            if (idx < TW * TH) {
                const int ly = idx / TW, lx = idx - ly * TW;
                const int gy = wrap(ty0 + ly - R), gx = wrap(tx0 + lx - R);
                const size_t j = (size_t)gy * Ns + gx;
                hm[u] = mask[j];
                hv[u] = g[j];
            }
        }
        const int x = tx0 + tx;
        const bool xin = x < Nw;
        uint8_t om[kStRows];
        T og[kStRows], op[kStRows];
#pragma unroll
        for (int k = 0; k < kStRows; ++k) {
            const int y = ty0 + tq * kStRows + k;
            const bool in = xin && y < Nw;
            const size_t i = (size_t)(in ? y : 0) * Ns + (in ? x : 0);
            om[k] = in ? mask[i] : 0;
            og[k] = g[i];
            if constexpr (DOTS) op[k] = gprev[i];
        }
#pragma unroll
        for (int u = 0; u < NL; ++u) {
            const int idx = threadIdx.x + u * 256;
            if (idx < TW * TH)
                tile[idx] = hm[u] ? (double)(LAZY ? (T)(hv[u] - aT) : hv[u]) - gmean : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kStRows; ++k) {
            const int ly = tq * kStRows + k, y = ty0 + ly;
            if (!xin || y >= Nw) continue;
            const size_t i = (size_t)y * Ns + x;
            if (!om[k]) {
                z[i] = T(0);
                continue;
            }
            double a = 0.0;
#pragma unroll
            for (int dy = -R; dy <= R; ++dy)
#pragma unroll
                for (int dx = -R; dx <= R; ++dx)
                    if (dx * dx + dy * dy <= R * R)
                        a += W.w[dy + kMaxR][dx + kMaxR] *
                             tile[(ly + R + dy) * TW + (tx + R + dx)];
            const T zT = (T)a;
            z[i] = zT;
            acc[0] += a;
            if constexpr (DOTS) {
                const T gi = LAZY ? (T)(og[k] - aT) : og[k];
                const double gd = (double)gi, dg = (double)(T)(gi - op[k]);
                acc[1] += (double)zT * gd;
                acc[2] += gd;
                acc[3] += (double)zT * dg;
                acc[4] += dg;
                acc[5] += gd * gd;
            }
        }
        __syncthreads();
    }
    int kinds[DOTS ? 6 : 1];
#pragma unroll
    for (int i = 0; i < (DOTS ? 6 : 1); ++i) kinds[i] = 0;
    if (grid_reduce_last<DOTS ? 6 : 1>(acc, kinds, part, &st->counter[2]) && threadIdx.x == 0) {
        const double zmean = st->nc ? (double)(T)(acc[0] / st->nc) : 0.0;
        st->zmean = zmean;
        st->pc++;
        if constexpr (DOTS) {
            beta_update(P, st, acc[1] - zmean * acc[2], acc[3] - zmean * acc[4], acc[5]);
            st->beta = (double)((T)st->delta * (T)st->bv);
        }
    }
}

// Register-blocked form for Ns >= 128 (the tile form above serves smaller
// grids): a warp owns a 128-wide segment of a 32-row strip, lane l the four
// consecutive columns x0 = seg*128 + 4l .. x0+3.  It streams the strip's
// rows top to bottom through a window of 2R+1 rows of centred values in
// registers (one float4 / double2x2 load of g and one uchar4 of the mask per
// new row); horizontal neighbours come from the adjacent lanes by shuffles
// and, at the segment edges, from the strip's halo columns staged in shared
// memory once per strip.  No block-wide barrier inside the strip.
constexpr int kSwSeg = 128, kSwRows = 32, kSwWarps = 4;

template <typename T, int R, bool LAZY, bool DOTS>
__global__ void __launch_bounds__(32 * kSwWarps) k_stencil_w(const PkParams* __restrict__ Pp,
                                                             PkState* st, StencilW W, const T* g,
                                                             const T* gprev, const uint8_t* mask,
                                                             T* z, double* part, int gated,
                                                             int rows) {
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    g += bo_;
    mask += bo_;
    z += bo_;
    if (DOTS) gprev += bo_;
    const PkParams& P = *Pp;
    if (gated && st->halt) return;
    constexpr int WR = 2 * R + 1;            // window rows
    constexpr int HR = kSwRows + 2 * R;      // halo rows of the longest strip
    __shared__ double halo[kSwWarps][HR][2 * R];
    const int Ns = P.Ns, msk = Ns - 1;
    const double gmean = st->nc ? st->gcs / st->nc : 0.0;
    const T aT = LAZY ? (T)st->alpha : T(0);
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nseg = Ns / kSwSeg, nstrips = nseg * (Ns / rows);
    auto centred = [&](uint8_t m, T v) -> double {
        return m ? (double)(LAZY ? (T)(v - aT) : v) - gmean : 0.0;
    };
    auto load4 = [&](const T* base, size_t i, T (&o)[4]) {
        if constexpr (sizeof(T) == 4) {
            const float4 q = *reinterpret_cast<const float4*>(base + i);
            o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w;
        } else {
            const double2 q0 = *reinterpret_cast<const double2*>(base + i);
            const double2 q1 = *reinterpret_cast<const double2*>(base + i + 2);
            o[0] = q0.x; o[1] = q0.y; o[2] = q1.x; o[3] = q1.y;
        }
    };
    double acc[DOTS ? 6 : 1];
#pragma unroll
    for (int i = 0; i < (DOTS ? 6 : 1); ++i) acc[i] = 0.0;
    for (int sw = blockIdx.x * kSwWarps + wib; sw < nstrips; sw += gridDim.x * kSwWarps) {
        const int seg = sw % nseg, y0 = (sw / nseg) * rows;
        const int xs = seg * kSwSeg, x0 = xs + 4 * lane;
        // the strip's halo columns (R left of the segment, R right), centred
        for (int e = lane; e < (rows + 2 * R) * 2 * R; e += 32) {
            const int hr = e / (2 * R), c = e - hr * (2 * R);
            const int x = (c < R ? xs - R + c : xs + kSwSeg + (c - R)) & msk;
            const size_t j = (size_t)((y0 - R + hr) & msk) * Ns + x;
            halo[wib][hr][c] = centred(mask[j], g[j]);
        }
        __syncwarp();
        double win[WR][4];
        uint32_t wmk[WR];  // the window rows' masks, 4 bytes
        // raw loads of one row (issued a step ahead of their use, so a row's
        // load latency hides behind the previous row's arithmetic)
        auto fetch = [&](int y, T (&v)[4], uint32_t& m4) {
            const size_t i = (size_t)(y & msk) * Ns + x0;
            m4 = *reinterpret_cast<const uint32_t*>(mask + i);
            load4(g, i, v);
        };
        auto put = [&](const T (&v)[4], uint32_t m4, double (&w)[4], uint32_t& mk) {
#pragma unroll
            for (int j = 0; j < 4; ++j) w[j] = centred((m4 >> (8 * j)) & 0xff, v[j]);
            mk = m4;
        };
#pragma unroll
        for (int r = 1; r < WR; ++r) {
            T v[4];
            uint32_t m4;
            fetch(y0 - R + r - 1, v, m4);
            put(v, m4, win[r], wmk[r]);
        }
        T nv[4], np[4];
        uint32_t nm;
        fetch(y0 + R, nv, nm);
        if constexpr (DOTS) load4(gprev, (size_t)y0 * Ns + x0, np);
        for (int k = 0; k < rows; ++k) {
#pragma unroll
            for (int r = 0; r + 1 < WR; ++r) {
#pragma unroll
                for (int j = 0; j < 4; ++j) win[r][j] = win[r + 1][j];
                wmk[r] = wmk[r + 1];
            }
            put(nv, nm, win[WR - 1], wmk[WR - 1]);
            T gp[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) gp[j] = np[j];
            if (k + 1 < rows) {
                fetch(y0 + k + 1 + R, nv, nm);
                if constexpr (DOTS) load4(gprev, (size_t)(y0 + k + 1) * Ns + x0, np);
            }
            // value at column offset d (in [-R, 3 + R]) of window row r
            auto at = [&](int r, int d) -> double {
                if (d >= 0 && d < 4) return win[r][d];
                double own, v;
                if (d < 0) {
                    own = win[r][4 + d];  // lane-1 holds it at index 4 + d
                    v = __shfl_up_sync(0xffffffffu, own, 1);
                    if (lane == 0) v = halo[wib][k + r][R + d];
                } else {
                    own = win[r][d - 4];  // lane+1 holds it at index d - 4
                    v = __shfl_down_sync(0xffffffffu, own, 1);
                    if (lane == 31) v = halo[wib][k + r][R + (d - 4)];
                }
                return v;
            };
            const int y = y0 + k;
            const size_t i = (size_t)y * Ns + x0;
            double a[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int dy = -R; dy <= R; ++dy) {
#pragma unroll
                for (int dx = -R; dx <= R; ++dx) {
                    if (dx * dx + dy * dy > R * R) continue;
                    const double w = W.w[dy + kMaxR][dx + kMaxR];
#pragma unroll
                    for (int j = 0; j < 4; ++j) a[j] += w * at(R + dy, j + dx);
                }
            }
            const uint32_t mc = wmk[R];
            T zo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool on = (mc >> (8 * j)) & 0xff;
                zo[j] = on ? (T)a[j] : T(0);
                if (on) acc[0] += a[j];
            }
            if constexpr (sizeof(T) == 4) {
                *reinterpret_cast<float4*>(z + i) = make_float4(zo[0], zo[1], zo[2], zo[3]);
            } else {
                *reinterpret_cast<double2*>(z + i) = make_double2(zo[0], zo[1]);
                *reinterpret_cast<double2*>(z + i + 2) = make_double2(zo[2], zo[3]);
            }
            if constexpr (DOTS) {
                T gv[4];
                load4(g, i, gv);  // loaded R rows ago: a cache hit
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (!((mc >> (8 * j)) & 0xff)) continue;
                    const T gi = LAZY ? (T)(gv[j] - aT) : gv[j];
                    const double gd = (double)gi, dg = (double)(T)(gi - gp[j]);
                    acc[1] += (double)zo[j] * gd;
                    acc[2] += gd;
                    acc[3] += (double)zo[j] * dg;
                    acc[4] += dg;
                    acc[5] += gd * gd;
                }
            }
        }
        __syncwarp();  // the halo buffer is refilled by the next strip
    }
    int kinds[DOTS ? 6 : 1];
#pragma unroll
    for (int i = 0; i < (DOTS ? 6 : 1); ++i) kinds[i] = 0;
    if (grid_reduce_last<DOTS ? 6 : 1>(acc, kinds, part, &st->counter[2]) && threadIdx.x == 0) {
        const double zmean = st->nc ? (double)(T)(acc[0] / st->nc) : 0.0;
        st->zmean = zmean;
        st->pc++;
        if constexpr (DOTS) {
            beta_update(P, st, acc[1] - zmean * acc[2], acc[3] - zmean * acc[4], acc[5]);
            st->beta = (double)((T)st->delta * (T)st->bv);
        }
    }
}

inline int num_sms() {
    int dev = 0, n = 0;
    ASB_CUDA(cudaGetDevice(&dev));
    ASB_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n > 0 ? n : 1;
}

inline int stencil_grid(int Ns) {
    const int n = ((Ns + kStX - 1) / kStX) * ((Ns + kStY - 1) / kStY);
    return n < kMaxRowBlocks ? n : kMaxRowBlocks;
}

StencilW stencil_weights(const StencilTaps& taps) {
    StencilW W{};
    for (int t = 0; t < taps.n; ++t)
        W.w[taps.dy[t] + kMaxR][taps.dx[t] + kMaxR] = taps.w[t];
    return W;
}

// launch of the stencil pass for the runtime radius R in [1, kMaxR]: the
// register-window kernel for Ns >= 128, the tile kernel below that and for
// embedded grids (Nl < Ns: the wrap is at the caller's side Nl)
template <typename T, bool LAZY, bool DOTS>
void launch_stencil(int R, int Ns, int Nl, dim3 grid, cudaStream_t s, const PkParams* Pp,
                    PkState* st, const StencilW& W, const T* g, const T* gprev,
                    const uint8_t* mask, T* z, double* part, int gated) {
    if (Ns >= kSwSeg && Nl == Ns) {
        // strips of 32, 16 or 8 rows: the longest that still gives every SM
        // 12 or more warps (a shorter strip re-reads more halo rows; at
        // Ns=2048 16-row strips measured 1 % faster per solve than 8 or 32)
        int rows = kSwRows;
        const long want = 12L * num_sms();
        while (rows > 8 && (long)(Ns / kSwSeg) * (Ns / rows) * grid.y < want) rows /= 2;
        const int strips = (Ns / kSwSeg) * (Ns / rows);
        int nb = (strips + kSwWarps - 1) / kSwWarps;
        if (nb > kMaxRowBlocks) nb = kMaxRowBlocks;
        const dim3 gw(nb, grid.y);
        switch (R) {
            case 1: k_stencil_w<T, 1, LAZY, DOTS><<<gw, 32 * kSwWarps, 0, s>>>(Pp, st, W, g, gprev, mask, z, part, gated, rows); break;
            case 2: k_stencil_w<T, 2, LAZY, DOTS><<<gw, 32 * kSwWarps, 0, s>>>(Pp, st, W, g, gprev, mask, z, part, gated, rows); break;
            case 3: k_stencil_w<T, 3, LAZY, DOTS><<<gw, 32 * kSwWarps, 0, s>>>(Pp, st, W, g, gprev, mask, z, part, gated, rows); break;
            case 4: k_stencil_w<T, 4, LAZY, DOTS><<<gw, 32 * kSwWarps, 0, s>>>(Pp, st, W, g, gprev, mask, z, part, gated, rows); break;
            default: throw Error(ASPHER_EINVAL, "stencil radius must be in [1, 4]");
        }
        count_launches(1);
        return;
    }
    switch (R) {
        case 1: k_stencil_t<T, 1, LAZY, DOTS><<<grid, 256, 0, s>>>(Pp, st, W, g, gprev, mask, z, part, gated); break;
        case 2: k_stencil_t<T, 2, LAZY, DOTS><<<grid, 256, 0, s>>>(Pp, st, W, g, gprev, mask, z, part, gated); break;
        case 3: k_stencil_t<T, 3, LAZY, DOTS><<<grid, 256, 0, s>>>(Pp, st, W, g, gprev, mask, z, part, gated); break;
        case 4: k_stencil_t<T, 4, LAZY, DOTS><<<grid, 256, 0, s>>>(Pp, st, W, g, gprev, mask, z, part, gated); break;
        default: throw Error(ASPHER_EINVAL, "stencil radius must be in [1, 4]");
    }
    count_launches(1);
}

// ---- CG passes (contact_solver.cpp:420-501) ------------------------------------
template <typename T>
__device__ __forceinline__ T zfinal(const PkParams& P, T z, T g, T zm) {
    return P.precond ? (T)(z - zm) : g;
}

// dots for the unpreconditioned and the FFT-preconditioned loops (z from the
// preconditioner; g centred on the fly)
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_dots(const PkParams* __restrict__ Pp, PkState* st, const T* z,
                                                      const T* g, const T* gprev,
                                                      const uint8_t* mask, double* part) {
    // instance blockIdx.y of a batched solve (0 when unbatched)
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    z += bo_;
    g += bo_;
    gprev += bo_;
    mask += bo_;
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T zm = (T)st->zmean, aT = (T)st->alpha;
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
            const T gi = gc(gv[j], aT);
            const T zf = zfinal(P, zz[j], gi, zm);
            const double gd = (double)gi;
            acc[0] += (double)zf * gd;
            acc[1] += (double)zf * (double)(T)(gi - gp[j]);
            acc[2] += gd * gd;
        }
    }
    const int kinds[3] = {0, 0, 0};
    if (grid_reduce_last<3>(acc, kinds, part, &st->counter[3]) && threadIdx.x == 0) {
        beta_update(P, st, acc[0], acc[1], acc[2]);
        st->beta = (double)((T)st->delta * (T)st->bv);
    }
}

// Direction update t = chi_C(z_f + beta t), g_prev = g (and best = p when
// copy_best) before the t apply; k_rden consumes r after it.
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_tupd(const PkParams* __restrict__ Pp, PkState* st, const T* z,
                                                      const T* g, T* gprev, T* t,
                                                      const uint8_t* mask, const T* p, T* best) {
    // instance blockIdx.y of a batched solve (0 when unbatched)
    Pp += blockIdx.y;
    st += blockIdx.y;
    const long bo_ = (long)blockIdx.y * Pp->N;
    z += bo_;
    g += bo_;
    gprev += bo_;
    t += bo_;
    mask += bo_;
    p += bo_;
    best += bo_;
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T zm = (T)st->zmean, beta = (T)st->beta, aT = (T)st->alpha;
    const int cb = st->copy_best;
    const PScale<T> ps(st);
    GRID_LOOP4(P.N) {
        T zz[4], gv[4], tt[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(g, i4, gv);
        ldp4(t, i4, tt);
        if (P.precond) ldp4(z, i4, zz);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            gv[j] = gc(gv[j], aT);
            tt[j] = mm[j] ? (T)(zfinal(P, zz[j], gv[j], zm) + beta * tt[j]) : T(0);
        }
        st4(t, i4, tt);
        st4(gprev, i4, gv);
        if (cb) {
            T pp[4];
            ldp4(p, i4, pp);
#pragma unroll
            for (int j = 0; j < 4; ++j) pp[j] = ps(pp[j]);
            st4(best, i4, pp);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_rden(const PkParams* __restrict__ Pp, PkState* st, const T* r,
                                                      const T* g, const T* t,
                                                      const uint8_t* mask, double* part) {
    // instance blockIdx.y of a batched solve (0 when unbatched)
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    r += bo_;
    g += bo_;
    t += bo_;
    mask += bo_;
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T aT = (T)st->alpha;
    double acc[4] = {0, 0, 0, 0};  // sum_C r, sum_C g t, sum_C r t, sum_C t
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
            const double td = (double)tt[j];
            acc[0] += (double)rr[j];
            acc[1] += (double)gc(gv[j], aT) * td;
            acc[2] += (double)rr[j] * td;
            acc[3] += td;
        }
    }
    const int kinds[4] = {0, 0, 0, 0};
    if (grid_reduce_last<4>(acc, kinds, part, &st->counter[4]) && threadIdx.x == 0)
        rden_tail<T>(st, acc);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_pupd(const PkParams* __restrict__ Pp, PkState* st, T* p, const T* t,
                                                      const T* g, double* part) {
    // instance blockIdx.y of a batched solve (0 when unbatched)
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    p += bo_;
    t += bo_;
    g += bo_;
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T tau = (T)st->tau, tov = (T)st->tau_ov, aT = (T)st->alpha;
    // every block reads the pending rescale here, before it arrives at the
    // last-block counter; only the last block's tail rewrites it
    const PScale<T> ps(st);
    double acc[2] = {0, 0};  // changed (max), total
    GRID_LOOP4(P.N) {
        T pp[4], tt[4], gv[4];
        ldp4(p, i4, pp);
        ldp4(t, i4, tt);
        ldp4(g, i4, gv);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T pi = ps(pp[j]);
            const T gi = gc(gv[j], aT);
            const bool was = pi > T(0);
            if (was) {
                const T q = pi - tau * tt[j];
                pi = q < T(0) ? T(0) : q;
            }
            if (pi == T(0) && gi < T(0)) pi -= tov * gi;
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
        // the load rescale (contact_solver.cpp:489-500), pending until the
        // next consumer of p forms it
        if (acc[1] > 0.0) {
            st->scale = (double)(T)(P.P_total / acc[1]);
            st->scale_add = 0.0;
            st->fill = 0;
        } else if (P.Nl != P.Ns) {  // every p is 0, embedded: the host fills the block
            st->scale = 1.0;
            st->scale_add = 0.0;
            st->fill = 2;
            set_halt(st, H_FILL);
        } else {  // every p is 0: p = p_bar
            st->scale = 1.0;
            st->scale_add = (double)(T)P.p_bar;
            st->fill = 1;
        }
        st->it++;
        if (st->it >= P.max_iter) set_halt(st, H_FINAL);  // status stays max_iterations
    }
}

// The pending load rescale applied to the stored pressure of every instance
// of the launch (before the host reads p), leaving scale 1 and fill 0.
// Reads the state of all blocks before the last block resets it.
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_materialize(
    const PkParams* __restrict__ Pp, PkState* st, T* p, double* part) {
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    p += bo_;
    const PkParams& P = *Pp;
    const PScale<T> ps(st);
    const bool identity = ps.f == T(1) && ps.a == T(0);
    if (!identity) {
        GRID_LOOP4(P.N) {
            T pp[4];
            ldp4(p, i4, pp);
#pragma unroll
            for (int j = 0; j < 4; ++j) pp[j] = ps(pp[j]);
            st4(p, i4, pp);
        }
    }
    double acc[1] = {0};
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[7]) && threadIdx.x == 0) {
        st->scale = 1.0;
        st->scale_add = 0.0;
        st->fill = 0;
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
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_reduce(const PkParams* __restrict__ Pp, PkState* st, int mode,
                                                        const T* a, const T* b, const T* c,
                                                        const T* d, double theta,
                                                        double* part) {
    // instance blockIdx.y of a batched launch (0 when unbatched)
    Pp += blockIdx.y;
    st += blockIdx.y;
    part += (size_t)blockIdx.y * kPartStride;
    const long bo_ = (long)blockIdx.y * Pp->N;
    if (a) a += bo_;
    if (b) b += bo_;
    if (c) c += bo_;
    if (d) d += bo_;
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
                    if (P.Nl != P.Ns) {  // embedded: the caller's block only
                        const long e = 4 * i4 + j;
                        if (e / P.Ns >= P.Nl || e % P.Ns >= P.Nl) break;
                    }
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
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_gd(const PkParams* __restrict__ Pp, PkState* st, const T* g,
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
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_gmean(long N, PkState* st, const T* g,
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
// Last kernel of the graph body of instances [0, n) (a range of the batch):
// keep looping while both end instances are running.  When an end instance
// halts the host continues with the loop graph of the smaller range that
// covers the instances still running, so halted instances at the ends stop
// costing gated blocks.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, const PkState* st, int n) {
    if (threadIdx.x == 0)
        cudaGraphSetConditional(h, (st[0].halt == H_RUN && st[n - 1].halt == H_RUN) ? 1u : 0u);
}

// ---- host driver -----------------------------------------------------------------
namespace {

int red_grid(long N) {
    long g = (N / 4 + kRedThreads - 1) / kRedThreads;
    if (g > kMaxBlocks / 2) g = kMaxBlocks / 2;
    if (g < 1) g = 1;
    return (int)g;
}

// The FP64 polish stage of a mixed solve runs its loop applies
// defect-corrected (Operator::matvec_defect: FP32 transforms of p - p0 and of
// t around one exact FP64 apply of p0).

// Per-operator, per-precision solver context: the CG workspace of up to
// `cap` instances (fields back to back), the device parameter and state
// blocks, and the instantiated loop graph (a while-conditional node whose
// body is one CG iteration of all instances), reused by every solve with the
// same preconditioner configuration and batch size.
template <typename T>
struct SolverCtx : SolverCtxBase {
    Operator& op;
    int cap = 1;
    long N = 0;
    T *p = nullptr, *t = nullptr, *u = nullptr, *g = nullptr, *gprev = nullptr, *z = nullptr,
      *r = nullptr, *best = nullptr;
    T* g0c = nullptr;  // the solves' gaps, copied in so the loop graph is reusable
    uint8_t* mask = nullptr;
    double* part = nullptr;
    double* hist = nullptr;
    int hist_cap = 0;  // entries per instance
    PkState* st = nullptr;
    PkParams* Pd = nullptr;
    void* spec = nullptr;  // spectrum scratch of cap instances (cap > 1 only)
    StencilTaps taps{};
    StencilW W{};
    int precond = -1, radius = -1;
    int grid = 1;
    bool with_hist = false;  // the loop body records pk per iteration (k_evalpk)
    // Defect-corrected applies (FP64 contexts, the polish stage of a mixed
    // solve): u = u0 + S_32(p - p0) and r = S_32(t), with p0 the stage's
    // starting pressure and u0 = S p0 from one exact FP64 apply.
    bool defect = false;
    double* p0 = nullptr;
    double* u0 = nullptr;
    // instantiated loop graphs, keyed by (apply mode: plain / defect-
    // corrected, first instance, number of instances): the graph of the
    // instance range [lo, lo + n) of a batch
    struct LoopGraph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
    };
    std::map<std::tuple<int, int, int>, LoopGraph> graphs;
    // Private non-blocking stream: the loop graph is captured and launched
    // here (the legacy NULL stream a caller may pass cannot be captured);
    // entry and exit are fenced to the caller's stream with events.
    cudaStream_t ws = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;

    SolverCtx(Operator& o, int capacity) : op(o), cap(capacity) {
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        ASB_CUDA(cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking));
        ASB_CUDA(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
        ASB_CUDA(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
        N = (long)o.Ns * o.Ns;
        const size_t b = (size_t)cap * N * sizeof(T);
        T** vecs[] = {&p, &t, &u, &g, &gprev, &z, &r, &best, &g0c};
        for (T** v : vecs) ASB_CUDA(cudaMalloc((void**)v, b));
        ASB_CUDA(cudaMalloc((void**)&mask, (size_t)cap * N));
        ASB_CUDA(cudaMalloc((void**)&part, (size_t)cap * kPartStride * sizeof(double)));
        ASB_CUDA(cudaMalloc((void**)&st, (size_t)cap * sizeof(PkState)));
        ASB_CUDA(cudaMalloc((void**)&Pd, (size_t)cap * sizeof(PkParams)));
        ASB_CUDA(cudaMemset(st, 0, (size_t)cap * sizeof(PkState)));
        ASB_CUDA(cudaMemset(z, 0, b));
        grid = red_grid(N);
        // spectra allocated before any capture; none for a precision whose
        // applies do not exist at this size (FP64 above 8192: this context
        // then only holds the FP64 fields of a mixed solve)
        const bool has_apply = o.supports(sizeof(T) == 8);
        if (has_apply) (void)o.spectrum(sizeof(T) == 8, nullptr);
        if (cap > 1 && has_apply) {
            const size_t sb = o.spectrum_bytes(sizeof(T) == 8) * (size_t)cap;
            ASB_CUDA(cudaMalloc(&spec, sb));
            ASB_CUDA(cudaMemset(spec, 0, sb));
        }
    }
    ~SolverCtx() override {
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        drop_graph();
        void* all[] = {p, t, u, g, gprev, z, r, best, g0c, mask, part, hist, st, Pd, spec, p0, u0};
        for (void* v : all)
            if (v) cudaFree(v);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (ws) cudaStreamDestroy(ws);
    }
    size_t bytes() const override {
        return (size_t)cap * ((9 * sizeof(T) + 1) * (size_t)N + hist_cap * sizeof(double) +
                              kPartStride * sizeof(double));
    }
    void invalidate() override { drop_graph(); }
    void ensure_hist(int per_instance) {
        if (per_instance <= hist_cap) return;
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        if (hist) ASB_CUDA(cudaFree(hist));
        ASB_CUDA(cudaMalloc((void**)&hist, (size_t)cap * per_instance * sizeof(double)));
        hist_cap = per_instance;
        drop_graph();  // the graph bakes the history pointer
    }
    void drop_graph() {
        for (auto& kv : graphs) {
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
        }
        graphs.clear();
    }
    // The context seen from instance b0 on: every per-instance pointer
    // offset to b0 (restored on destruction), so enqueue_iteration(s, n)
    // captures the iteration of instances [b0, b0 + n) with gridDim.y = n.
    struct InstanceView {
        SolverCtx& c;
        T *p, *t, *u, *g, *gprev, *z, *r, *best, *g0c;
        uint8_t* mask;
        double *part, *p0, *u0;
        PkState* st;
        PkParams* Pd;
        InstanceView(SolverCtx& cx, int b0)
            : c(cx), p(cx.p), t(cx.t), u(cx.u), g(cx.g), gprev(cx.gprev), z(cx.z), r(cx.r),
              best(cx.best), g0c(cx.g0c), mask(cx.mask), part(cx.part), p0(cx.p0), u0(cx.u0),
              st(cx.st), Pd(cx.Pd) {
            const size_t o = (size_t)b0 * cx.N;
            T** vs[] = {&cx.p, &cx.t, &cx.u, &cx.g, &cx.gprev, &cx.z, &cx.r, &cx.best, &cx.g0c};
            for (T** v : vs) *v += o;
            cx.mask += o;
            cx.part += (size_t)b0 * kPartStride;
            if (cx.p0) cx.p0 += o;
            if (cx.u0) cx.u0 += o;
            cx.st += b0;
            cx.Pd += b0;
        }
        ~InstanceView() {
            c.p = p; c.t = t; c.u = u; c.g = g; c.gprev = gprev; c.z = z; c.r = r;
            c.best = best; c.g0c = g0c; c.mask = mask; c.part = part; c.p0 = p0; c.u0 = u0;
            c.st = st; c.Pd = Pd;
        }
    };
    // switch the loop's applies between exact and defect-corrected (FP64
    // contexts only); allocates p0 / u0 on first use, outside any capture
    void set_defect(bool on) {
        if (on && sizeof(T) != 8) throw Error(ASPHER_EINVAL, "defect correction needs FP64");
        if (on && !p0) {
            std::lock_guard<std::recursive_mutex> setup(setup_mutex());
            ASB_CUDA(cudaMalloc((void**)&p0, (size_t)cap * N * sizeof(double)));
            ASB_CUDA(cudaMalloc((void**)&u0, (size_t)cap * N * sizeof(double)));
            (void)op.spectrum(false, nullptr);  // the FP32 scratch of unbatched applies
        }
        defect = on;
    }
    void set_hist(bool on) {
        if (on == with_hist) return;
        with_hist = on;
        drop_graph();
    }
    void configure(int pc, int R) {
        if (pc == precond && (pc != 1 || R == radius)) return;
        if (pc == 2 && op.embedded()) {
            if (op.Nl % 2)
                throw Error(ASPHER_EINVAL, "precond 'fourier-fft' on a grid that is not a power "
                                           "of two needs an even grid_size (use 'fourier', the "
                                           "stencil, on this grid)");
            op.ensure_precond_spectrum();  // set-up before any capture
        }
        if (pc == 1) {
            taps = make_stencil_taps(op.Nl, R);
            W = stencil_weights(taps);
        }
        precond = pc;
        radius = R;
        drop_graph();
    }
    T* at(T* v, int b) const { return v + (size_t)b * N; }

    // B instances: gates per instance, spectrum of the batch when B > 1
    void apply(const T* x, T* y, const int* gate, cudaStream_t s, int B,
               const PkState* sc = nullptr) {
        op.matvec(sizeof(T) == 8, x, y, s, gate, B, B > 1 ? spec : nullptr, sc);
    }
    // one CG iteration of B instances (the common path), every pass gated
    // per instance on the device:
    //   [apply p->u] eval (evalpk) | stencil+dots  or  [precond] dots |
    //   tupd [apply t->r] rden | pupd (load rescale pending, formed by the
    //   next consumers of p)
    // the loop's two applies: u = S p (gated by skip_mv1) and r = S t
    void apply_u(cudaStream_t s, int B) {
        if constexpr (sizeof(T) == 8) {
            if (defect) {
                op.matvec_defect(p, p0, u, u0, s, &st->skip_mv1, B, B > 1 ? spec : nullptr, st);
                return;
            }
        }
        // p carries its pending load rescale (formed as it is loaded)
        apply(p, u, &st->skip_mv1, s, B, st);
    }
    void apply_r(cudaStream_t s, int B) {
        if constexpr (sizeof(T) == 8) {
            if (defect) {
                op.matvec_defect(t, nullptr, r, nullptr, s, &st->halt, B, B > 1 ? spec : nullptr);
                return;
            }
        }
        apply(t, r, &st->halt, s, B);
    }
    void enqueue_iteration(cudaStream_t s, int B) {
        const dim3 gr(grid, B);
        int n = 0;
        apply_u(s, B);
        k_eval<T><<<gr, kRedThreads, 0, s>>>(Pd, st, u, g0c, p, g, mask, part, 0);
        ++n;
        if (with_hist) {
            k_evalpk<T><<<gr, kRedThreads, 0, s>>>(Pd, st, p, g, part, hist, 0);
            ++n;
        }
        if (precond == 1) {
            launch_stencil<T, true, true>(radius, op.Ns, op.Nl, dim3(stencil_grid(op.Nl), B), s, Pd, st, W, g,
                                          gprev, mask, z, part, 1);
            ++n;
        } else {
            if (precond == 2)
                fourier_precond_pk<T>(op, g, mask, st, z, part, s, &st->halt, B,
                                      B > 1 ? spec : nullptr);
            k_dots<T><<<gr, kRedThreads, 0, s>>>(Pd, st, z, g, gprev, mask, part);
            ++n;
        }
        k_tupd<T><<<gr, kRedThreads, 0, s>>>(Pd, st, z, g, gprev, t, mask, p, best);
        apply_r(s, B);
        k_rden<T><<<gr, kRedThreads, 0, s>>>(Pd, st, r, g, t, mask, part);
        n += 2;
        k_pupd<T><<<gr, kRedThreads, 0, s>>>(Pd, st, p, t, g, part);
        count_launches(n + 1);
        ASB_CUDA(cudaGetLastError());
    }
    // g <- centred gap for instance b (or all B when b < 0)
    void center(cudaStream_t s, int B, int b = -1) {
        if (b < 0)
            k_center<T><<<dim3(grid, B), kRedThreads, 0, s>>>(Pd, st, g);
        else
            k_center<T><<<grid, kRedThreads, 0, s>>>(Pd + b, st + b, at(g, b));
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
    }
    // capture the loop graph of instances [lo, lo + n); the caller holds
    // setup_mutex()
    void build_graph(cudaStream_t s, int lo, int n) {
        LoopGraph& lg = graphs[std::make_tuple((int)defect, lo, n)];
        if (lg.exec) cudaGraphExecDestroy(lg.exec);
        if (lg.graph) cudaGraphDestroy(lg.graph);
        lg = LoopGraph{};
        ASB_CUDA(cudaGraphCreate(&lg.graph, 0));
        cudaGraphConditionalHandle h;
        ASB_CUDA(cudaGraphConditionalHandleCreate(&h, lg.graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        ASB_CUDA(cudaGraphAddNode(&node, lg.graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ASB_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeRelaxed));
        try {
            InstanceView view(*this, lo);
            enqueue_iteration(s, n);
            k_loop_cond<<<1, 32, 0, s>>>(h, st, n);
        } catch (...) {
            // leave no capture open on the stream, then report the failure
            cudaGraph_t partial = nullptr;
            cudaStreamEndCapture(s, &partial);
            cudaGetLastError();
            drop_graph();
            throw;
        }
        cudaGraph_t captured = nullptr;
        ASB_CUDA(cudaStreamEndCapture(s, &captured));
        ASB_CUDA(cudaGraphInstantiate(&lg.exec, lg.graph, 0));
    }
    // Build the loop graph of instances [lo, lo + n) if needed.  Before
    // capturing, one fully gated iteration of those instances runs eagerly
    // (every kernel returns at entry) so that all function attributes are set
    // outside the capture: it clobbers their device states, which the caller
    // writes afterwards.  The capture holds setup_mutex(): no other host
    // thread may synchronise the device (a set-up call) while this stream is
    // capturing.
    bool has_graph(int lo, int n) const {
        auto it = graphs.find(std::make_tuple((int)defect, lo, n));
        return it != graphs.end() && it->second.exec;
    }
    void ensure_graph(cudaStream_t s, int lo, int n) {
        if (has_graph(lo, n)) return;
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        std::vector<PkState> gated(n);
        std::memset(gated.data(), 0, n * sizeof(PkState));
        for (auto& x : gated) {
            x.halt = H_FINAL;
            x.skip_mv1 = 1;
        }
        ASB_CUDA(cudaMemcpyAsync(st + lo, gated.data(), n * sizeof(PkState),
                                 cudaMemcpyHostToDevice, s));
        {
            InstanceView view(*this, lo);
            enqueue_iteration(s, n);
        }
        ASB_CUDA(cudaStreamSynchronize(s));
        build_graph(s, lo, n);
    }
    // one iteration of instances [lo, lo + n) launched kernel by kernel
    void launch_eager(cudaStream_t s, int lo, int n) {
        InstanceView view(*this, lo);
        enqueue_iteration(s, n);
    }
    void launch_graph(cudaStream_t s, int lo, int n) {
        ASB_CUDA(cudaGraphLaunch(graphs.at(std::make_tuple((int)defect, lo, n)).exec, s));
        count_launches(1);
    }
};

// One instance's host-side bookkeeping in a (possibly batched) solve.
struct InstHost {
    double p_bar = 0.0, P_total = 0.0, g_ref = 1.0, p_ref = 0.0, datum = 0.0;
    double s_id = 0.0;
    int forced_id = 0, id_steps = 0;
    std::string reason;
    long long mv_host = 0;
    bool returned_best = false;
    int status = ST_MAX_ITERATIONS;
};

template <typename T>
struct Solver {
    SolverCtx<T>& c;
    cudaStream_t s;
    cudaStream_t caller;
    int B = 1;
    std::vector<PkParams> P;
    std::vector<PkState> h;  // host mirrors
    std::vector<InstHost> ih;

    // All work runs on the context's private stream, ordered after the
    // caller's pending work and before the caller's later work.
    Solver(SolverCtx<T>& ctx, cudaStream_t st, int batch = 1)
        : c(ctx), s(ctx.ws), caller(st), B(batch), P(batch), h(batch), ih(batch) {
        ASB_CUDA(cudaEventRecord(c.ev_in, caller));
        ASB_CUDA(cudaStreamWaitEvent(s, c.ev_in, 0));
    }
    ~Solver() {
        if (cudaEventRecord(c.ev_out, s) == cudaSuccess) cudaStreamWaitEvent(caller, c.ev_out, 0);
    }

    // p = v on the caller's cells (0 outside the block of an embedded grid)
    void fill_p(T* p, T v) {
        if (c.op.embedded())
            k_fill_block<T><<<embed_grid(c.N), 256, 0, s>>>(c.op.Nl, c.op.Ns, p, v);
        else
            k_fill<T><<<c.grid, kRedThreads, 0, s>>>(c.N, p, v);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
    }
    void read_states() {
        ASB_CUDA(cudaMemcpyAsync(h.data(), c.st, B * sizeof(PkState), cudaMemcpyDeviceToHost, s));
        ASB_CUDA(cudaStreamSynchronize(s));
    }
    void write_states() {
        ASB_CUDA(cudaMemcpyAsync(c.st, h.data(), B * sizeof(PkState), cudaMemcpyHostToDevice, s));
        ASB_CUDA(cudaStreamSynchronize(s));
    }
    void write_params() {
        ASB_CUDA(cudaMemcpyAsync(c.Pd, P.data(), B * sizeof(PkParams), cudaMemcpyHostToDevice, s));
    }
    // results of the helper reductions live in st[b].red; only that slice is
    // read back so the host mirrors are never clobbered mid-update
    void read_red(int b, double (&r)[8]) {
        ASB_CUDA(cudaMemcpyAsync(r, c.st[b].red, sizeof(r), cudaMemcpyDeviceToHost, s));
        ASB_CUDA(cudaStreamSynchronize(s));
    }
    // reduction of instance b (pointers are instance b's fields)
    double reduce(int b, int mode, const T* a, const T* bb, const T* cc, const T* d, double theta,
                  double* out3 = nullptr) {
        k_reduce<T><<<c.grid, kRedThreads, 0, s>>>(c.Pd + b, c.st + b, mode, a, bb, cc, d, theta,
                                                 c.part + (size_t)b * kPartStride);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
        double r[8];
        read_red(b, r);
        if (out3) { out3[0] = r[0]; out3[1] = r[1]; out3[2] = r[2]; }
        return r[0];
    }

    // project_load_simplex on instance b's z (contact_solver.cpp:31-60)
    void project_simplex(int b, double P_total) {
        const long N = c.N;
        T* z = c.at(c.z, b);
        double ssum = reduce(b, 1, z, nullptr, nullptr, nullptr, 0.0);
        long nact = N;
        double theta = (ssum - P_total) / (double)nact;
        for (int pass = 0; pass < 64; ++pass) {
            double o[3];
            reduce(b, 4, z, nullptr, nullptr, nullptr, theta, o);
            const long n2 = (long)o[1];
            if (n2 == 0) break;
            if (n2 == nact) break;
            nact = n2;
            ssum = o[0];
            theta = (ssum - P_total) / (double)nact;
        }
        k_threshold<T><<<c.grid, kRedThreads, 0, s>>>(N, z, (T)theta);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
    }

    // identification step of instance b (contact_solver.cpp:314-364); reads
    // the centred gap (the caller materialises it first)
    bool identification_step(int b) {
        InstHost& I = ih[b];
        PkState& H = h[b];
        T *p = c.at(c.p, b), *u = c.at(c.u, b), *g = c.at(c.g, b), *z = c.at(c.z, b),
          *r = c.at(c.r, b), *t = c.at(c.t, b), *gp = c.at(c.gprev, b);
        const T* g0 = c.at(c.g0c, b);
        double o[3];
        reduce(b, 2, p, u, g0, nullptr, 0.0, o);
        const double f_cur = o[0];
        if (!(I.s_id > 0.0)) {
            const double pp = o[1], pu = o[2];
            I.s_id = (pu > 0.0 && pp > 0.0) ? pp / pu : 1.0;
        }
        for (int trial = 0; trial < 12; ++trial) {
            k_axpy_trial<T><<<c.grid, kRedThreads, 0, s>>>(c.N, z, p, g, (T)I.s_id);
            count_launches(1);
            project_simplex(b, I.P_total);
            c.op.matvec(sizeof(T) == 8, z, r, s, nullptr);  // unbatched scratch
            I.mv_host++;
            reduce(b, 3, z, r, g0, nullptr, 0.0, o);
            const double f_try = o[0];
            k_gd<T><<<c.grid, kRedThreads, 0, s>>>(c.Pd + b, c.st + b, g, z, p,
                                                 c.part + (size_t)b * kPartStride);
            count_launches(1);
            double rr[8];
            read_red(b, rr);
            const double gd = rr[3];
            if (std::isfinite(f_try) && gd < 0.0 && f_try <= f_cur + 1e-4 * gd) {
                const size_t bytes = (size_t)c.N * sizeof(T);
                ASB_CUDA(cudaMemcpyAsync(p, z, bytes, cudaMemcpyDeviceToDevice, s));
                ASB_CUDA(cudaMemcpyAsync(u, r, bytes, cudaMemcpyDeviceToDevice, s));
                ASB_CUDA(cudaMemsetAsync(t, 0, bytes, s));
                ASB_CUDA(cudaMemsetAsync(gp, 0, bytes, s));
                H.u_fresh = 1;
                H.delta = 0.0;
                H.G_old = 1.0;
                ++I.id_steps;
                if (trial == 0) I.s_id *= 2.0;
                return true;
            }
            I.s_id *= 0.25;
        }
        return false;
    }

    // Solve B instances that share the operator and the options.  g0s[b],
    // p_inits[b] (nullable) are device fields of T; outputs FP64 (disps /
    // gaps / hist only honoured for B == 1).  datum_b / gref_b (nullable):
    // per-instance datum and g_ref overriding opts' (used with the datum
    // modes solver / caller).
    void run(const aspher_solve_opts& o, const T* const* g0s, const double* p_bars,
             const T* const* p_inits, double* const* pressures, double* disp, double* gap,
             double* hist_host, int hist_cap, aspher_result* res,
             const double* datum_b = nullptr, const double* gref_b = nullptr,
             bool defect = false) {
        const auto t_start = std::chrono::steady_clock::now();
        const int Ns = c.op.Ns;
        const long N = (long)Ns * Ns;
        // the caller's cell count: the load P = p_bar n_grid and the reported
        // fractions (contact_solver.cpp:623-625,1003-1004); N but for
        // embedded operators, whose fields hold the caller's block in
        // compute-grid layout (gap kEmbedPadGap, pressure 0 outside it)
        const bool emb = c.op.embedded();
        const double n_grid = (double)c.op.Nl * (double)c.op.Nl;
        constexpr bool is_double = sizeof(T) == 8;
        if (B < 1 || B > c.cap) throw Error(ASPHER_EINVAL, "solve: batch size out of range");
        for (int b = 0; b < B; ++b)
            if (!(p_bars[b] > 0.0) || !std::isfinite(p_bars[b]))
                throw Error(ASPHER_EINVAL, "solve_contact: empty gap or p_bar <= 0");
        if (!(o.tol > 0.0)) throw Error(ASPHER_EINVAL, "solve_contact: tol must be positive");
        if (o.max_iter < 0) throw Error(ASPHER_EINVAL, "solve_contact: max_iter must be >= 0");
        if (o.precond < 0 || o.precond > 2) throw Error(ASPHER_EINVAL, "solve_contact: bad precond");
        c.configure(o.precond, o.precond_radius);
        const bool rec = o.record_history && B == 1 && hist_host && hist_cap > 0;
        if (rec) c.ensure_hist(o.max_iter + 1);
        c.set_hist(rec);
        // the caller's gaps are read once into the context (a fixed address
        // keeps the graph valid)
        for (int b = 0; b < B; ++b) {
            P[b] = PkParams{};
            P[b].N = N;
            P[b].Ns = Ns;
            P[b].Nl = c.op.Nl;
            if (g0s[b] != c.at(c.g0c, b))
                ASB_CUDA(cudaMemcpyAsync(c.at(c.g0c, b), g0s[b], (size_t)N * sizeof(T),
                                         cudaMemcpyDeviceToDevice, s));
        }
        write_params();
        // validation before any operator apply (contact_solver.cpp:159-168):
        // min, max and non-finite count of every gap in one batched pass
        k_reduce<T><<<dim3(c.grid, B), kRedThreads, 0, s>>>(c.Pd, c.st, 0, c.g0c, nullptr, nullptr,
                                                          nullptr, 0.0, c.part);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
        read_states();
        const double load_tol = o.load_tol > 0.0 ? o.load_tol : (is_double ? 1e-12 : 5e-7);
        const double tol = o.tol;
        const double req_tol = o.requested_tol > 0.0 ? o.requested_tol : tol;
        for (int b = 0; b < B; ++b) {
            InstHost& I = ih[b];
            const double gmin_v = h[b].red[0], gmax_v = h[b].red[1];
            if (h[b].red[2] > 0.0)
                throw Error(ASPHER_EINVAL, "solve_contact: g0 contains non-finite values");
            I.p_bar = p_bars[b];
            I.P_total = (double)(T)p_bars[b] * n_grid;
            double g_ref = gref_b ? gref_b[b] : o.g_ref;
            if (!(g_ref > 0.0)) g_ref = gmax_v - gmin_v;
            if (!(g_ref > 0.0)) g_ref = 1.0;
            I.g_ref = g_ref;
            I.p_ref = o.p_ref > 0.0 ? o.p_ref : (double)(T)p_bars[b];
            bool subtract = false;
            if (o.datum_mode == ASPHER_DATUM_AUTOMATIC) {
                I.datum = gmin_v + 0.5 * (gmax_v - gmin_v);
                subtract = true;
            } else if (o.datum_mode == ASPHER_DATUM_SOLVER) {
                I.datum = datum_b ? datum_b[b] : o.datum;
                subtract = true;
            } else {
                I.datum = datum_b ? datum_b[b] : o.datum;
            }
            PkParams& Q = P[b];
            Q.max_iter = o.max_iter;
            Q.stall_limit = o.stall_limit > 0 ? o.stall_limit : 200;
            Q.keep_best = o.keep_best;
            Q.record_history = rec ? 1 : 0;
            Q.hist_stride = c.hist_cap;
            Q.use_pr = o.use_pr;
            Q.precond = o.precond;
            Q.P_total = I.P_total;
            Q.g_ref = g_ref;
            Q.tol = tol;
            Q.load_tol = load_tol;
            Q.p_bar = (double)(T)p_bars[b];
            Q.gshift = subtract ? (double)(T)I.datum : 0.0;
        }
        write_params();

        // initial pressures (contact_solver.cpp:204-223)
        for (int b = 0; b < B; ++b) {
            T* p = c.at(c.p, b);
            const T pb = (T)p_bars[b];
            if (p_inits && p_inits[b]) {
                k_clamp_pos<T><<<c.grid, kRedThreads, 0, s>>>(N, p, p_inits[b]);
                count_launches(1);
                const double ssum = reduce(b, 1, p, nullptr, nullptr, nullptr, 0.0);
                if (ssum > 0.0)
                    k_scale<T><<<c.grid, kRedThreads, 0, s>>>(N, p, (T)(ih[b].P_total / ssum));
                else
                    fill_p(p, pb);
            } else {
                fill_p(p, pb);
            }
            count_launches(1);
        }
        const size_t vb = (size_t)B * N * sizeof(T);
        ASB_CUDA(cudaMemsetAsync(c.t, 0, vb, s));
        ASB_CUDA(cudaMemsetAsync(c.gprev, 0, vb, s));
        ASB_CUDA(cudaMemsetAsync(c.z, 0, vb, s));
        for (int b = 0; b < B; ++b) {
            PkState& H = h[b];
            std::memset(&H, 0, sizeof(H));
            H.scale = 1.0;  // no load rescale pending
            H.G_old = 1.0;
            H.delta = 0.0;
            H.best_merit = std::numeric_limits<double>::infinity();
            H.seen_merit = std::numeric_limits<double>::infinity();
            H.status = ST_MAX_ITERATIONS;
            H.halt = o.max_iter > 0 ? H_RUN : H_FINAL;
            H.skip_mv1 = H.halt ? 1 : 0;
        }
        // defect-corrected applies (a polish stage): p0 = the starting
        // pressures, u0 = S p0 by one exact FP64 apply of all instances
        c.set_defect(defect);
        if constexpr (sizeof(T) == 8) {
            if (defect) {
                ASB_CUDA(cudaMemcpyAsync(c.p0, c.p, (size_t)B * N * sizeof(double),
                                         cudaMemcpyDeviceToDevice, s));
                c.apply(c.p0, c.u0, nullptr, s, B);
                for (int b = 0; b < B; ++b) ih[b].mv_host += 1;
            }
        }
        const bool eager = o.loop_mode == 1;
        if (o.loop_mode != 0 && !eager) throw Error(ASPHER_EINVAL, "solve_contact: bad loop_mode");
        if (!eager) c.ensure_graph(s, 0, B);
        write_states();
        // loop_mode 1: the loop body's kernels launched one by one, the end
        // instances' halt flags read back after each iteration (the graph's
        // while condition, evaluated on the host)
        auto run_eager = [&](int lo, int n) {
            int hv[2];
            do {
                c.launch_eager(s, lo, n);
                ASB_CUDA(cudaMemcpyAsync(&hv[0], &c.st[lo].halt, sizeof(int),
                                         cudaMemcpyDeviceToHost, s));
                ASB_CUDA(cudaMemcpyAsync(&hv[1], &c.st[lo + n - 1].halt, sizeof(int),
                                         cudaMemcpyDeviceToHost, s));
                ASB_CUDA(cudaStreamSynchronize(s));
            } while (hv[0] == H_RUN && hv[1] == H_RUN);
        };

        // ---- the loop: device-driven, the host services rare branches
        auto any_running = [&]() {
            for (int b = 0; b < B; ++b)
                if (h[b].halt == H_RUN) return true;
            return false;
        };
        while (any_running()) {
            // the loop graph of the smallest instance range that covers
            // every running instance: halted instances outside it launch
            // no (gated) blocks
            int lo = -1, hi = -1;
            for (int b = 0; b < B; ++b)
                if (h[b].halt == H_RUN) {
                    if (lo < 0) lo = b;
                    hi = b;
                }
            const int n = hi - lo + 1;
            if (eager) {
                run_eager(lo, n);
            } else {
                if (!c.has_graph(lo, n)) {
                    c.ensure_graph(s, lo, n);  // clobbers st[lo, lo + n)
                    write_states();
                }
                c.launch_graph(s, lo, n);
            }
            // the host takes over: form the pending load rescale of p
            k_materialize<T><<<dim3(c.grid, n), kRedThreads, 0, s>>>(
                c.Pd + lo, c.st + lo, c.at(c.p, lo), c.part + (size_t)lo * kPartStride);
            count_launches(1);
            read_states();
            bool changed = false;
            for (int b = 0; b < B; ++b) {
                PkState& H = h[b];
                InstHost& I = ih[b];
                if (H.fill == 2) {
                    // an embedded solve's p = p_bar (contact_solver.cpp:498-500)
                    // on the caller's block; the iteration counter already
                    // moved on
                    fill_p(c.at(c.p, b), (T)I.p_bar);
                    H.fill = 0;
                    H.u_fresh = 0;
                    if (H.halt == H_FILL) {
                        H.halt = H_RUN;
                        H.skip_mv1 = 0;
                    }
                    changed = true;
                    continue;
                }
                if (H.halt != H_STALL && H.halt != H_IDENT) continue;
                changed = true;
                if (H.copy_best) {
                    ASB_CUDA(cudaMemcpyAsync(c.at(c.best, b), c.at(c.p, b), (size_t)N * sizeof(T),
                                             cudaMemcpyDeviceToDevice, s));
                    H.copy_best = 0;
                    H.have_best = 1;
                }
                c.center(s, B, b);  // the identification step reads the centred gap
                bool resume = true;
                if (H.halt == H_STALL) {
                    if (I.forced_id < 3 && identification_step(b)) {
                        ++I.forced_id;
                        H.stall = 0;
                    } else {
                        H.status = ST_STAGNATED;
                        I.reason = "stall";
                        H.halt = H_FINAL;
                        resume = false;
                    }
                } else if (!identification_step(b)) {
                    H.status = ST_NONPOSITIVE_CURVATURE;
                    H.halt = H_FINAL;
                    resume = false;
                }
                if (!resume) continue;
                // the loop body's end increments the iteration counter
                H.it++;
                H.mv += I.mv_host;
                I.mv_host = 0;
                if (H.it >= o.max_iter) {
                    H.halt = H_FINAL;
                    continue;
                }
                H.halt = H_RUN;
                H.skip_mv1 = H.u_fresh ? 1 : 0;
            }
            if (changed) write_states();
        }

        // ---- final, freshly evaluated diagnostics (contact_solver.cpp:518-586)
        for (int b = 0; b < B; ++b) {
            PkState& H = h[b];
            InstHost& I = ih[b];
            H.mv += I.mv_host;
            I.mv_host = 0;
            I.status = H.status;
            if (I.status != ST_CONVERGED && o.keep_best && H.have_best) {
                const double merit = std::max(H.fw, H.pen);
                if (!(merit <= H.best_merit)) {
                    ASB_CUDA(cudaMemcpyAsync(c.at(c.p, b), c.at(c.best, b), (size_t)N * sizeof(T),
                                             cudaMemcpyDeviceToDevice, s));
                    H.u_fresh = 0;
                    I.returned_best = true;
                }
            }
            // the certificate is evaluated from an exact apply: a
            // defect-corrected u is recomputed
            const bool fresh = H.u_fresh && !c.defect;
            if (!fresh) H.mv++;
            H.skip_mv1 = fresh ? 1 : 0;  // gates the final apply per instance
            H.halt = H_FINAL;
        }
        write_states();
        c.apply(c.p, c.u, &c.st->skip_mv1, s, B);
        k_eval<T><<<dim3(c.grid, B), kRedThreads, 0, s>>>(c.Pd, c.st, c.u, c.g0c, c.p, c.g, c.mask,
                                                        c.part, 1);
        k_evalpk<T><<<dim3(c.grid, B), kRedThreads, 0, s>>>(c.Pd, c.st, c.p, c.g, c.part, nullptr,
                                                          1);
        count_launches(2);
        ASB_CUDA(cudaGetLastError());
        read_states();
        // objective sum p (0.5 u + g0s) of every instance in one batched pass
        k_reduce<T><<<dim3(c.grid, B), kRedThreads, 0, s>>>(c.Pd, c.st, 5, c.p, c.u, c.g0c, nullptr,
                                                          0.0, c.part);
        count_launches(1);
        std::vector<PkState> ob(B);
        ASB_CUDA(cudaMemcpyAsync(ob.data(), c.st, B * sizeof(PkState), cudaMemcpyDeviceToHost, s));
        for (int b = 0; b < B; ++b) {
            k_to_f64<T><<<c.grid, kRedThreads, 0, s>>>(N, pressures[b], c.at(c.p, b));
            count_launches(1);
        }
        if (B == 1 && !o.light) {
            if (disp) { k_to_f64<T><<<c.grid, kRedThreads, 0, s>>>(N, disp, c.u); count_launches(1); }
            if (gap) {
                c.center(s, 1);
                k_to_f64<T><<<c.grid, kRedThreads, 0, s>>>(N, gap, c.g);
                count_launches(1);
            }
        }
        ASB_CUDA(cudaGetLastError());
        int hl = 0;
        if (rec) {
            hl = std::min(h[0].it, hist_cap);
            if (hl > 0)
                ASB_CUDA(cudaMemcpyAsync(hist_host, c.hist, hl * sizeof(double),
                                         cudaMemcpyDeviceToHost, s));
        }
        ASB_CUDA(cudaStreamSynchronize(s));
        const double secs =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        for (int b = 0; b < B; ++b) {
            const PkState& H = h[b];
            const InstHost& I = ih[b];
            int status = I.status;
            std::string reason = I.reason;
            if (!H.finite && status != ST_NONFINITE) status = ST_NONFINITE;
            if (status == ST_CONVERGED && !(H.load <= load_tol && H.fw <= tol && H.pen <= tol)) {
                status = ST_VERIFICATION_FAILED;
                reason = "final_check";
            }
            if (status == ST_CONVERGED && req_tol < tol && !o.allow_tolerance_relaxation) {
                if (!(H.fw <= req_tol && H.pen <= req_tol)) {
                    status = ST_STAGNATED;
                    reason = "precision_limit";
                }
            }
            aspher_result& R = res[b];
            std::memset(&R, 0, sizeof(R));
            R.status = status;
            std::strncpy(R.status_reason, reason.c_str(), sizeof(R.status_reason) - 1);
            R.iterations = H.it;
            R.converged = status == ST_CONVERGED;
            R.contact_fraction = (double)H.nc / n_grid;
            R.mean_pressure = H.psum / n_grid;
            R.approach = H.alpha_ref + I.datum;
            R.objective = ob[b].red[0] + I.datum * I.P_total;
            R.error = H.pk;
            R.pk_error = H.pk;
            R.fw_gap = H.G;
            R.fw_error = H.fw;
            R.load_error = H.load;
            R.pressure_violation = 0.0;
            R.penetration_error = H.pen;
            R.requested_tol = req_tol;
            R.effective_tol = tol;
            R.p_ref = I.p_ref;
            R.g_ref = I.g_ref;
            R.matvec_count = H.mv;
            R.precond_count = H.pc;
            R.identification_steps = I.id_steps;
            R.returned_best = I.returned_best;
            R.history_len = b == 0 ? hl : 0;
            const long long rb = sizeof(T);
            R.mem_cg_state = 7LL * N * rb;
            R.mem_best_iterate = o.keep_best ? N * rb : 0;
            R.mem_contact_mask = N;
            R.mem_output_arrays = (rb == 8 ? 0 : N * 8LL) + (o.light ? 0 : 2LL * N * 8);
            R.mem_peak = R.mem_cg_state + R.mem_best_iterate + R.mem_contact_mask +
                         R.mem_output_arrays;
            R.time_total = secs;
        }
    }
};

template <typename T>
SolverCtx<T>& get_ctx(Operator& op, int cap = 1) {
    std::shared_ptr<SolverCtxBase>& slot = sizeof(T) == 8 ? op.ctx_d : op.ctx_f;
    if (!slot || static_cast<SolverCtx<T>&>(*slot).cap < cap) {
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        slot.reset();  // free the smaller workspace first
        slot = std::make_shared<SolverCtx<T>>(op, cap);
    }
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
    // w depends on (|dx|, |dy|) only on an even Nw; on an odd one the
    // reference's wavenumber convention (ky < Nw/2 ? ky : ky - Nw) makes the
    // kernel slightly uneven, and the reference reads it at the signed
    // offsets (stencil_precond.cpp:211-216)
    const bool even = Nw % 2 == 0;
    std::map<std::pair<int, int>, double> uniq;
    for (int dy = -R; dy <= R; ++dy)
        for (int dx = -R; dx <= R; ++dx) {
            if (dx * dx + dy * dy > R * R) continue;
            const std::pair<int, int> key = even ? std::make_pair(std::abs(dx), std::abs(dy))
                                                 : std::make_pair(dx, dy);
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

// Embedded operators: the caller's Nl x Nl fields copied into compute-grid
// temporaries (gaps padded with kEmbedPadGap, pressures with 0) on the
// caller's stream before a solve, and the outputs' blocks copied back after
// it; stream-ordered allocations, freed on exit.  For other operators every
// call passes its pointer through.
struct EmbedIO {
    Operator& op;
    cudaStream_t s;
    std::vector<void*> bufs;
    EmbedIO(Operator& o, cudaStream_t st) : op(o), s(st) {}
    ~EmbedIO() {
        for (void* p : bufs) cudaFreeAsync(p, s);
    }
    long n() const { return (long)op.Ns * op.Ns; }
    template <typename T>
    T* alloc() {
        void* p = nullptr;
        ASB_CUDA(cudaMallocAsync(&p, (size_t)n() * sizeof(T), s));
        bufs.push_back(p);
        return static_cast<T*>(p);
    }
    template <typename T>
    const T* in(const T* src, T pad) {
        if (!src || !op.embedded()) return src;
        T* d = alloc<T>();
        k_embed<T, T><<<embed_grid(n()), 256, 0, s>>>(op.Nl, op.Ns, 1, src, d, pad);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
        return d;
    }
    double* out(double* dst) { return dst && op.embedded() ? alloc<double>() : dst; }
    void back(const double* tmp, double* dst) {
        if (!dst || !op.embedded()) return;
        k_extract<double, double><<<embed_grid((long)op.Nl * op.Nl), 256, 0, s>>>(op.Nl, op.Ns, 1,
                                                                                 tmp, dst);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
    }
};

template <typename T>
void solve_impl(Operator& op, const aspher_solve_opts& o, const void* g0, double p_bar,
                const void* p_init, double* pressure, double* disp, double* gap, double* hist,
                int hist_cap, aspher_result& res, cudaStream_t s, bool polish_stage) {
    EmbedIO io(op, s);
    const T* g = io.in((const T*)g0, (T)kEmbedPadGap);
    const T* pi = io.in((const T*)p_init, T(0));
    double *pr = io.out(pressure), *ds = io.out(disp), *gp = io.out(gap);
    {
        Solver<T> S(get_ctx<T>(op), s);
        const bool defect = sizeof(T) == 8 && polish_stage && p_init;
        S.run(o, &g, &p_bar, &pi, &pr, ds, gp, hist, hist_cap, &res, nullptr, nullptr, defect);
    }
    io.back(pr, pressure);
    io.back(ds, disp);
    io.back(gp, gap);
}
template void solve_impl<float>(Operator&, const aspher_solve_opts&, const void*, double,
                                const void*, double*, double*, double*, double*, int,
                                aspher_result&, cudaStream_t, bool);
template void solve_impl<double>(Operator&, const aspher_solve_opts&, const void*, double,
                                 const void*, double*, double*, double*, double*, int,
                                 aspher_result&, cudaStream_t, bool);

namespace {
// FP64 min / max / non-finite count of B FP64 gaps (validation before any
// apply), the FP32 stage's datum and g_ref per instance, and the centred FP32
// copies of the gaps in the FP32 context.
void mixed_prepare(Operator& op, const aspher_solve_opts& o, int B, const double* const* g0s,
                   std::vector<double>& datum, std::vector<double>& gref, cudaStream_t s) {
    SolverCtx<double>& cd = get_ctx<double>(op, B);
    SolverCtx<float>& cf = get_ctx<float>(op, B);
    const long N = (long)op.Ns * op.Ns;
    datum.assign(B, 0.0);
    gref.assign(B, 0.0);
    Solver<double> probe(cd, s, B);
    for (int b = 0; b < B; ++b) {
        probe.P[b].N = N;
        probe.P[b].Ns = op.Ns;
        probe.P[b].Nl = op.Nl;
    }
    probe.write_params();
    for (int b = 0; b < B; ++b) {
        double mm[3];
        probe.reduce(b, 0, g0s[b], nullptr, nullptr, nullptr, 0.0, mm);
        if (mm[2] > 0.0) throw Error(ASPHER_EINVAL, "solve_contact: g0 contains non-finite values");
        datum[b] = o.datum_mode == ASPHER_DATUM_AUTOMATIC ? mm[0] + 0.5 * (mm[1] - mm[0]) : o.datum;
        double g_ref = o.g_ref;
        if (!(g_ref > 0.0)) g_ref = mm[1] - mm[0];
        if (!(g_ref > 0.0)) g_ref = 1.0;
        gref[b] = g_ref;
        // on the caller's stream: the FP32 solve's stream waits for it
        k_center_cast<<<red_grid(N), kRedThreads, 0, s>>>(
            N, cf.at(cf.g0c, b), g0s[b], o.datum_mode == ASPHER_DATUM_CALLER ? 0.0 : datum[b]);
        count_launches(1);
    }
    ASB_CUDA(cudaGetLastError());
}

aspher_solve_opts float_stage_opts(const aspher_solve_opts& o, double float_tol, int polish) {
    aspher_solve_opts of = o;
    of.dtype = ASPHER_F32;
    of.tol = float_tol;
    of.requested_tol = polish ? float_tol : (o.requested_tol > 0.0 ? o.requested_tol : o.tol);
    of.allow_tolerance_relaxation = polish ? 1 : o.allow_tolerance_relaxation;
    of.datum_mode = ASPHER_DATUM_CALLER;
    return of;
}

// the reported work is the sum of both stages (nested_solve.cpp:445-450)
void add_stage(aspher_result& r, const aspher_result& rf) {
    r.iterations += rf.iterations;
    r.matvec_count += rf.matvec_count;
    r.precond_count += rf.precond_count;
    r.identification_steps += rf.identification_steps;
    r.time_total += rf.time_total;
}
}  // namespace

// FP32 stage + FP64 polish (the reference's float_then_double staging,
// nested_solve.cpp:871-974, on one level): the gap is centred by its
// midpoint datum and cast to FP32 on the device, the FP32 PK solve runs to
// float_tol with FP64 reductions, and -- when polish -- an FP64 PK solve
// warm-started from that pressure certifies opts.tol (the caller may ask
// for a polish tolerance below the requested one).
namespace {
void solve_mixed_core(Operator& op, const aspher_solve_opts& o, const double* g0, double p_bar,
                      const double* p_init, double float_tol, int polish, double* pressure,
                      double* disp, double* gap, aspher_result& res, aspher_result* res_float,
                      cudaStream_t s) {
    std::vector<double> datum, gref;
    mixed_prepare(op, o, 1, &g0, datum, gref, s);
    SolverCtx<double>& cd = get_ctx<double>(op);
    SolverCtx<float>& cf = get_ctx<float>(op);
    const long N = (long)op.Ns * op.Ns;
    const float* pinit_f = nullptr;
    if (p_init) {
        pinit_f = cf.r;  // scratch: read by the FP32 solve before r is first written
        k_cast_f32<<<red_grid(N), kRedThreads, 0, s>>>(N, cf.r, p_init);
        count_launches(1);
        ASB_CUDA(cudaGetLastError());
    }
    aspher_solve_opts of = float_stage_opts(o, float_tol, polish);
    of.light = polish ? 1 : o.light;
    aspher_result rf;
    {
        Solver<float> S(cf, s);
        const float* g0f = cf.g0c;
        S.run(of, &g0f, &p_bar, &pinit_f, &pressure, polish ? nullptr : disp,
              polish ? nullptr : gap, nullptr, 0, &rf, datum.data(), gref.data());
    }
    if (res_float) *res_float = rf;
    if (!polish) {
        res = rf;
        return;
    }
    aspher_solve_opts od = o;
    od.dtype = ASPHER_F64;
    od.datum_mode = ASPHER_DATUM_SOLVER;
    {
        Solver<double> S(cd, s);
        const double* pw = pressure;
        S.run(od, &g0, &p_bar, &pw, &pressure, disp, gap, nullptr, 0, &res, datum.data(),
              gref.data(), true);
    }
    add_stage(res, rf);
}
}  // namespace

void solve_mixed(Operator& op, const aspher_solve_opts& o, const double* g0, double p_bar,
                 const double* p_init, double float_tol, int polish, double* pressure,
                 double* disp, double* gap, aspher_result& res, aspher_result* res_float,
                 cudaStream_t s) {
    EmbedIO io(op, s);
    const double* g = io.in(g0, kEmbedPadGap);
    const double* pi = io.in(p_init, 0.0);
    double *pr = io.out(pressure), *ds = io.out(disp), *gp = io.out(gap);
    solve_mixed_core(op, o, g, p_bar, pi, float_tol, polish, pr, ds, gp, res, res_float, s);
    io.back(pr, pressure);
    io.back(ds, disp);
    io.back(gp, gap);
}

// Batched solve of B instances sharing the operator and the options, in one
// loop graph (per-instance gates = convergence masks).
template <typename T>
void solve_batch_impl(Operator& op, const aspher_solve_opts& o, int B, const void* const* g0s,
                      const double* p_bars, const void* const* p_inits, double* const* pressures,
                      aspher_result* res, cudaStream_t s) {
    if (B < 1) throw Error(ASPHER_EINVAL, "solve_batch: batch must be >= 1");
    EmbedIO io(op, s);
    std::vector<const T*> g(B), pi(B);
    std::vector<double*> pr(B);
    for (int b = 0; b < B; ++b) {
        g[b] = io.in(static_cast<const T*>(g0s[b]), (T)kEmbedPadGap);
        pi[b] = p_inits ? io.in(static_cast<const T*>(p_inits[b]), T(0)) : nullptr;
        pr[b] = io.out(pressures[b]);
    }
    {
        Solver<T> S(get_ctx<T>(op, B), s, B);
        aspher_solve_opts ob = o;
        if (B > 1) ob.light = 1;
        S.run(ob, g.data(), p_bars, p_inits ? pi.data() : nullptr, pr.data(), nullptr, nullptr,
              nullptr, 0, res);
    }
    for (int b = 0; b < B; ++b) io.back(pr[b], pressures[b]);
}
template void solve_batch_impl<float>(Operator&, const aspher_solve_opts&, int, const void* const*,
                                      const double*, const void* const*, double* const*,
                                      aspher_result*, cudaStream_t);
template void solve_batch_impl<double>(Operator&, const aspher_solve_opts&, int,
                                       const void* const*, const double*, const void* const*,
                                       double* const*, aspher_result*, cudaStream_t);

namespace {
void solve_batch_mixed_core(Operator& op, const aspher_solve_opts& o, int B,
                            const double* const* g0s, const double* p_bars, double float_tol,
                            int polish, double* const* pressures, aspher_result* res,
                            aspher_result* res_float, cudaStream_t s);
}  // namespace

// Batched FP32 stage + FP64 polish (solve_mixed for B instances).
void solve_batch_mixed(Operator& op, const aspher_solve_opts& o, int B, const double* const* g0s,
                       const double* p_bars, double float_tol, int polish,
                       double* const* pressures, aspher_result* res, aspher_result* res_float,
                       cudaStream_t s) {
    if (B < 1) throw Error(ASPHER_EINVAL, "solve_batch: batch must be >= 1");
    EmbedIO io(op, s);
    std::vector<const double*> gv(B);
    std::vector<double*> prv(B);
    for (int b = 0; b < B; ++b) {
        gv[b] = io.in(g0s[b], kEmbedPadGap);
        prv[b] = io.out(pressures[b]);
    }
    solve_batch_mixed_core(op, o, B, gv.data(), p_bars, float_tol, polish, prv.data(), res,
                           res_float, s);
    for (int b = 0; b < B; ++b) io.back(prv[b], pressures[b]);
}

namespace {
void solve_batch_mixed_core(Operator& op, const aspher_solve_opts& o, int B,
                            const double* const* g0s, const double* p_bars, double float_tol,
                            int polish, double* const* pressures, aspher_result* res,
                            aspher_result* res_float, cudaStream_t s) {
    std::vector<double> datum, gref;
    mixed_prepare(op, o, B, g0s, datum, gref, s);
    SolverCtx<double>& cd = get_ctx<double>(op, B);
    SolverCtx<float>& cf = get_ctx<float>(op, B);
    aspher_solve_opts of = float_stage_opts(o, float_tol, polish);
    of.light = 1;
    std::vector<aspher_result> rf(B);
    {
        Solver<float> S(cf, s, B);
        std::vector<const float*> gf(B);
        for (int b = 0; b < B; ++b) gf[b] = cf.at(cf.g0c, b);
        S.run(of, gf.data(), p_bars, nullptr, pressures, nullptr, nullptr, nullptr, 0, rf.data(),
              datum.data(), gref.data());
    }
    if (res_float)
        for (int b = 0; b < B; ++b) res_float[b] = rf[b];
    if (!polish) {
        for (int b = 0; b < B; ++b) res[b] = rf[b];
        return;
    }
    aspher_solve_opts od = o;
    od.dtype = ASPHER_F64;
    od.datum_mode = ASPHER_DATUM_SOLVER;
    od.light = 1;
    {
        Solver<double> S(cd, s, B);
        std::vector<const double*> pw(pressures, pressures + B);
        S.run(od, g0s, p_bars, pw.data(), pressures, nullptr, nullptr, nullptr, 0, res,
              datum.data(), gref.data(), true);
    }
    for (int b = 0; b < B; ++b) add_stage(res[b], rf[b]);
}
}  // namespace

// Standalone preconditioner apply: z = M^-1 g on contact, contact-mean removed.
template <typename T>
void precond_apply_impl(Operator& op, int precond, int radius, const T* g_in,
                        const uint8_t* mask_in, T* z_out, cudaStream_t s) {
    if (op.embedded() && precond != 1) {
        if (op.Nl % 2)
            throw Error(ASPHER_EINVAL, "precond 'fourier-fft' on a grid that is not a power of "
                                       "two needs an even grid_size");
        op.ensure_precond_spectrum();
    }
    const long N = (long)op.Ns * op.Ns;
    // embedded: g and the contact flags into compute-grid fields (0 outside
    // the caller's block: no contact there), z's block copied back
    const T* g = g_in;
    const uint8_t* mask = mask_in;
    T* z = z_out;
    void* tmp[3] = {nullptr, nullptr, nullptr};
    if (op.embedded()) {
        ASB_CUDA(cudaMallocAsync(&tmp[0], (size_t)N * sizeof(T), s));
        ASB_CUDA(cudaMallocAsync(&tmp[1], (size_t)N, s));
        ASB_CUDA(cudaMallocAsync(&tmp[2], (size_t)N * sizeof(T), s));
        k_embed<T, T><<<embed_grid(N), 256, 0, s>>>(op.Nl, op.Ns, 1, g_in, (T*)tmp[0], T(0));
        k_embed<uint8_t, uint8_t><<<embed_grid(N), 256, 0, s>>>(op.Nl, op.Ns, 1, mask_in,
                                                                (uint8_t*)tmp[1], 0);
        count_launches(2);
        g = (const T*)tmp[0];
        mask = (const uint8_t*)tmp[1];
        z = (T*)tmp[2];
    }
    PkState* st = nullptr;
    double* part = nullptr;
    ASB_CUDA(cudaMallocAsync((void**)&st, sizeof(PkState), s));
    ASB_CUDA(cudaMallocAsync((void**)&part, kPartStride * sizeof(double), s));
    ASB_CUDA(cudaMemsetAsync(st, 0, sizeof(PkState), s));  // alpha = 0: g used as given
    PkParams P{};
    P.N = N;
    P.Ns = op.Ns;
    P.Nl = op.Nl;
    P.precond = precond;
    PkParams* Pd = nullptr;
    ASB_CUDA(cudaMallocAsync((void**)&Pd, sizeof(PkParams), s));
    ASB_CUDA(cudaMemcpyAsync(Pd, &P, sizeof(PkParams), cudaMemcpyHostToDevice, s));
    const int grid = red_grid(N);
    k_gmean<T><<<grid, kRedThreads, 0, s>>>(N, st, g, mask, part);
    if (precond == 1) {
        StencilTaps taps = make_stencil_taps(op.Nl, radius);
        launch_stencil<T, false, false>(radius, op.Ns, op.Nl, dim3(stencil_grid(op.Nl)), s, Pd,
                                        st, stencil_weights(taps), g, nullptr, mask, z, part, 0);
    } else {
        fourier_precond_pk<T>(op, g, mask, st, z, part, s, nullptr);
    }
    k_sub_zmean<T><<<grid, kRedThreads, 0, s>>>(N, z, mask, st);
    count_launches(2);
    if (op.embedded()) {
        k_extract<T, T><<<embed_grid((long)op.Nl * op.Nl), 256, 0, s>>>(op.Nl, op.Ns, 1, z, z_out);
        count_launches(1);
        for (void* v : tmp) cudaFreeAsync(v, s);
    }
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

// ---- adjoint of a converged solve ------------------------------------------------
// No reference counterpart.  At a converged solve with contact set
// C = {p > 0} the KKT system restricted to C,
//     S_CC p_C - alpha 1 = -g0_C,   1^T p_C = P,
// is linear in (g0, P), so for a loss L(p) with w = dL/dp the adjoint pair
// (lam, mu) solves the symmetric system
//     S_CC lam - mu 1 = w_C,   1^T lam = 0,
// and dL/dg0 = -lam on C (0 off C), dL/dP = -mu, dL/dp_bar = -mu N.  lam is
// found by CG on V = {x : x = 0 off C, sum_C x = 0} with the projected
// operator Pi S Pi and the projected stencil preconditioner (the PK solve's
// own Pi M Pi); mu = mean_C(S lam - w) once lam has converged.  Nothing of
// the forward iterates is needed (they are not stored).
//
// The state reuses PkState: nc / gcs (= 0) / zmean / pc for the stencil
// kernel, halt / it / status for the loop, G_old = previous r.z, beta,
// tau = step length, gg = |r|^2, total = |r0|^2, rmean = contact mean of q,
// alpha = contact mean of w.
namespace {

template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_adj_init(const PkParams* __restrict__ Pp, PkState* st,
                                                          const double* p, const double* w,
                                                          uint8_t* mask, T* wT, double* part) {
    const PkParams& P = *Pp;
    double acc[2] = {0.0, 0.0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P.N; i += (long)gridDim.x * blockDim.x) {
        const bool c = p[i] > 0.0;
        const T wi = (T)w[i];
        mask[i] = c ? 1 : 0;
        wT[i] = wi;
        if (c) { acc[0] += (double)wi; acc[1] += 1.0; }
    }
    const int kinds[2] = {0, 0};
    if (grid_reduce_last<2>(acc, kinds, part, &st->counter[0]) && threadIdx.x == 0) {
        st->nc = (int)acc[1];
        st->alpha = st->nc ? acc[0] / st->nc : 0.0;
        st->gcs = 0.0;
        st->halt = st->nc < 2 ? H_FINAL : H_RUN;
        st->status = st->nc < 2 ? ST_NONPOSITIVE_CURVATURE : ST_MAX_ITERATIONS;
    }
}

// r = Pi w, lam = d = 0, |r0|^2
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_adj_r0(const PkParams* __restrict__ Pp, PkState* st,
                                                        const uint8_t* mask, const T* wT, T* r,
                                                        T* lam, T* d, double* part) {
    const PkParams& P = *Pp;
    const T wm = (T)st->alpha;
    double acc[1] = {0.0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P.N; i += (long)gridDim.x * blockDim.x) {
        const T ri = mask[i] ? (T)(wT[i] - wm) : T(0);
        r[i] = ri;
        lam[i] = T(0);
        d[i] = T(0);
        acc[0] += (double)ri * (double)ri;
    }
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[1]) && threadIdx.x == 0) {
        st->total = acc[0];
        st->gg = acc[0];
        st->it = 0;
        st->G_old = 0.0;
        if (!(acc[0] > 0.0)) {  // w is constant on C: lam = 0 solves exactly
            st->status = ST_CONVERGED;
            st->halt = H_FINAL;
        }
    }
}

// rz = <Pi z, r>, beta = rz / rz_old; z = r when unpreconditioned
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_adj_rz(const PkParams* __restrict__ Pp, PkState* st,
                                                        const T* z, const T* r,
                                                        const uint8_t* mask, double* part) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T zm = (T)st->zmean;
    double acc[1] = {0.0};
    GRID_LOOP4(P.N) {
        T zz[4], rr[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(r, i4, rr);
        ldp4(z, i4, zz);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (mm[j]) acc[0] += (double)(T)(zz[j] - zm) * (double)rr[j];
    }
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[3]) && threadIdx.x == 0) {
        st->beta = (st->it > 0 && st->G_old != 0.0) ? (double)(T)(acc[0] / st->G_old) : 0.0;
        st->G_old = acc[0];
        if (!(acc[0] > 0.0) || !isfinite(acc[0])) {  // preconditioner lost definiteness
            st->status = isfinite(acc[0]) ? ST_NONPOSITIVE_CURVATURE : ST_NONFINITE;
            st->halt = H_FINAL;
        }
    }
}

// d = Pi z + beta d on C
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_adj_d(const PkParams* __restrict__ Pp, const PkState* st,
                                                       const T* z, const uint8_t* mask, T* d) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T zm = (T)st->zmean, beta = (T)st->beta;
    GRID_LOOP4(P.N) {
        T zz[4], dd[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(z, i4, zz);
        ldp4(d, i4, dd);
#pragma unroll
        for (int j = 0; j < 4; ++j) dd[j] = mm[j] ? (T)((T)(zz[j] - zm) + beta * dd[j]) : T(0);
        st4(d, i4, dd);
    }
}

// a = rz / <d, q>, qm = contact mean of q (q = S d)
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_adj_dq(const PkParams* __restrict__ Pp, PkState* st,
                                                        const T* d, const T* q,
                                                        const uint8_t* mask, double* part) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    double acc[2] = {0.0, 0.0};
    GRID_LOOP4(P.N) {
        T dd[4], qq[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(d, i4, dd);
        ldp4(q, i4, qq);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (mm[j]) { acc[0] += (double)dd[j] * (double)qq[j]; acc[1] += (double)qq[j]; }
    }
    const int kinds[2] = {0, 0};
    if (grid_reduce_last<2>(acc, kinds, part, &st->counter[4]) && threadIdx.x == 0) {
        st->rmean = (double)(T)(acc[1] / st->nc);
        if (acc[0] > 0.0 && isfinite(acc[0])) {
            st->tau = (double)(T)(st->G_old / acc[0]);
        } else {
            st->status = isfinite(acc[0]) ? ST_NONPOSITIVE_CURVATURE : ST_NONFINITE;
            st->halt = H_FINAL;
        }
    }
}

// lam += a d; r -= a Pi q; convergence |r| <= tol |r0|
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_adj_upd(const PkParams* __restrict__ Pp, PkState* st,
                                                         const T* d, const T* q,
                                                         const uint8_t* mask, T* lam, T* r,
                                                         double* part) {
    const PkParams& P = *Pp;
    if (st->halt) return;
    const T a = (T)st->tau, qm = (T)st->rmean;
    double acc[1] = {0.0};
    GRID_LOOP4(P.N) {
        T dd[4], qq[4], ll[4], rr[4];
        uint8_t mm[4];
        ldm4(mask, i4, mm);
        ldp4(d, i4, dd);
        ldp4(q, i4, qq);
        ldp4(lam, i4, ll);
        ldp4(r, i4, rr);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!mm[j]) { rr[j] = T(0); continue; }
            ll[j] = ll[j] + a * dd[j];
            rr[j] = rr[j] - a * (T)(qq[j] - qm);
            acc[0] += (double)rr[j] * (double)rr[j];
        }
        st4(lam, i4, ll);
        st4(r, i4, rr);
    }
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[5]) && threadIdx.x == 0) {
        st->gg = acc[0];
        st->it++;
        if (!isfinite(acc[0])) {
            st->status = ST_NONFINITE;
            st->halt = H_FINAL;
        } else if (acc[0] <= P.tol * P.tol * st->total) {
            st->status = ST_CONVERGED;
            st->halt = H_FINAL;
        } else if (st->it >= P.max_iter) {
            st->halt = H_FINAL;
        }
    }
}

// mu = mean_C(S lam - w); grad_g0 = -lam on C (0 off C), FP64
template <typename T>
__global__ void __launch_bounds__(kRedThreads, kRedMinBlocks) k_adj_out(const PkParams* __restrict__ Pp, PkState* st,
                                                         const T* q, const T* wT, const T* lam,
                                                         const uint8_t* mask, double* grad,
                                                         double* part) {
    const PkParams& P = *Pp;
    double acc[1] = {0.0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P.N; i += (long)gridDim.x * blockDim.x) {
        const bool c = mask[i] != 0;
        grad[i] = c ? -(double)lam[i] : 0.0;
        if (c) acc[0] += (double)q[i] - (double)wT[i];
    }
    const int kinds[1] = {0};
    if (grid_reduce_last<1>(acc, kinds, part, &st->counter[6]) && threadIdx.x == 0)
        st->red[0] = st->nc ? acc[0] / st->nc : 0.0;
}

}  // namespace

template <typename T>
void adjoint_core(Operator& op, const double* p, const double* w, double tol, int max_iter,
                  int precond, int radius, double* grad_g0, double* grad_pbar,
                  aspher_adjoint_info* info, cudaStream_t s) {
    if (!(tol > 0.0)) throw Error(ASPHER_EINVAL, "adjoint: tol must be positive");
    if (max_iter < 1) throw Error(ASPHER_EINVAL, "adjoint: max_iter must be >= 1");
    if (precond != ASPHER_PRECOND_NONE && precond != ASPHER_PRECOND_STENCIL)
        throw Error(ASPHER_EINVAL, "adjoint: precond must be NONE or STENCIL");
    const auto t0 = std::chrono::steady_clock::now();
    const long N = (long)op.Ns * op.Ns;
    const size_t vb = (size_t)N * sizeof(T);
    StencilW W{};
    if (precond == ASPHER_PRECOND_STENCIL) W = stencil_weights(make_stencil_taps(op.Nl, radius));
    T *wT = nullptr, *r = nullptr, *z = nullptr, *d = nullptr, *q = nullptr, *lam = nullptr;
    uint8_t* mask = nullptr;
    double* part = nullptr;
    PkState* st = nullptr;
    PkParams* Pd = nullptr;
    T** vecs[] = {&wT, &r, &z, &d, &q, &lam};
    for (T** v : vecs) ASB_CUDA(cudaMallocAsync((void**)v, vb, s));
    ASB_CUDA(cudaMallocAsync((void**)&mask, (size_t)N, s));
    ASB_CUDA(cudaMallocAsync((void**)&part, kPartStride * sizeof(double), s));
    ASB_CUDA(cudaMallocAsync((void**)&st, sizeof(PkState), s));
    ASB_CUDA(cudaMallocAsync((void**)&Pd, sizeof(PkParams), s));
    ASB_CUDA(cudaMemsetAsync(st, 0, sizeof(PkState), s));
    PkParams P{};
    P.N = N;
    P.Ns = op.Ns;
    P.Nl = op.Nl;
    P.tol = tol;
    P.max_iter = max_iter;
    P.precond = precond;
    ASB_CUDA(cudaMemcpyAsync(Pd, &P, sizeof(P), cudaMemcpyHostToDevice, s));
    const int grid = red_grid(N);
    k_adj_init<T><<<grid, kRedThreads, 0, s>>>(Pd, st, p, w, mask, wT, part);
    k_adj_r0<T><<<grid, kRedThreads, 0, s>>>(Pd, st, mask, wT, r, lam, d, part);
    count_launches(2);
    ASB_CUDA(cudaGetLastError());
    PkState h{};
    auto read = [&]() {
        ASB_CUDA(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s));
        ASB_CUDA(cudaStreamSynchronize(s));
    };
    read();
    while (h.halt == H_RUN) {
        for (int k = 0; k < 16; ++k) {  // kernels return at entry once halted
            const T* zz = r;
            if (precond == ASPHER_PRECOND_STENCIL) {
                launch_stencil<T, false, false>(radius, op.Ns, op.Nl, dim3(stencil_grid(op.Nl)),
                                                s, Pd, st, W, r, nullptr, mask, z, part, 1);
                zz = z;
            }
            k_adj_rz<T><<<grid, kRedThreads, 0, s>>>(Pd, st, zz, r, mask, part);
            k_adj_d<T><<<grid, kRedThreads, 0, s>>>(Pd, st, zz, mask, d);
            op.matvec(sizeof(T) == 8, d, q, s, &st->halt);
            k_adj_dq<T><<<grid, kRedThreads, 0, s>>>(Pd, st, d, q, mask, part);
            k_adj_upd<T><<<grid, kRedThreads, 0, s>>>(Pd, st, d, q, mask, lam, r, part);
            count_launches(4);
        }
        ASB_CUDA(cudaGetLastError());
        read();
    }
    op.matvec(sizeof(T) == 8, lam, q, s, nullptr);
    k_adj_out<T><<<grid, kRedThreads, 0, s>>>(Pd, st, q, wT, lam, mask, grad_g0, part);
    count_launches(1);
    ASB_CUDA(cudaGetLastError());
    read();
    const double mu = h.red[0];
    if (grad_pbar) *grad_pbar = -mu * (double)op.Nl * (double)op.Nl;  // P = p_bar Nl^2
    if (info) {
        std::memset(info, 0, sizeof(*info));
        info->status = h.status;
        info->iterations = h.it;
        info->residual = h.total > 0.0 ? std::sqrt(h.gg / h.total) : 0.0;
        info->contact_count = h.nc;
        info->mu = mu;
        info->time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    void* all[] = {wT, r, z, d, q, lam, mask, part, st, Pd};
    for (void* v : all) cudaFreeAsync(v, s);
    ASB_CUDA(cudaStreamSynchronize(s));
}
// the caller's fields around the core (embedded operators: p and w into
// compute-grid fields that are 0 outside the caller's block, so the contact
// set and the constraint are the caller's; dL/dg0's block copied back)
template <typename T>
void adjoint_impl(Operator& op, const double* p, const double* w, double tol, int max_iter,
                  int precond, int radius, double* grad_g0, double* grad_pbar,
                  aspher_adjoint_info* info, cudaStream_t s) {
    EmbedIO io(op, s);
    const double* pc = io.in(p, 0.0);
    const double* wc = io.in(w, 0.0);
    double* gc = io.out(grad_g0);
    adjoint_core<T>(op, pc, wc, tol, max_iter, precond, radius, gc, grad_pbar, info, s);
    io.back(gc, grad_g0);
    ASB_CUDA(cudaStreamSynchronize(s));
}
template void adjoint_impl<float>(Operator&, const double*, const double*, double, int, int, int,
                                  double*, double*, aspher_adjoint_info*, cudaStream_t);
template void adjoint_impl<double>(Operator&, const double*, const double*, double, int, int, int,
                                   double*, double*, aspher_adjoint_info*, cudaStream_t);

}  // namespace asb
