// Nested-grid (cascadic) driver for the fft / periodic backends.
//
// Reference: solve_contact_nested (src/nested_solve.cpp:518-990) with
// stencil_for_level (:27-39), restrict_field (:42-54) and prolong_field
// (:57-71).  Levels coarsest * 2^k .. Ns; the gap is restricted by 2x2 block
// averages on the device; each level solves with its own operator (taken from
// a per-process cache keyed by backend, Ns, L, E*, device) and is
// warm-started by injecting the coarser pressure; one datum and one g_ref =
// max(range(g0), p_bar L / E*) serve every level.  Precision policy (A09):
// double, float (FP32 levels, float floor) or float_then_double (FP32
// levels, then an FP64 polish of the finest level at the requested tol).
#include "../../include/aspher_b200.h"
#include "common.cuh"
#include "ops.hpp"
#include "pcg.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace asb {

__global__ void k_restrict(int Ns, const double* __restrict__ f, double* __restrict__ out) {
    const int c = Ns / 2;
    const long n = (long)c * c;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int iy = (int)(i / c), ix = (int)(i % c);
        const long x0 = 2 * ix, y0 = 2 * iy;
        out[i] = 0.25 * (((f[y0 * Ns + x0] + f[y0 * Ns + x0 + 1]) + f[(y0 + 1) * Ns + x0]) +
                         f[(y0 + 1) * Ns + x0 + 1]);
    }
}

__global__ void k_prolong(int Nc, const double* __restrict__ pc, double* __restrict__ out) {
    const int f = 2 * Nc;
    const long n = (long)Nc * Nc;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int iy = (int)(i / Nc), ix = (int)(i % Nc);
        const double v = pc[i];
        const long x0 = 2 * ix, y0 = 2 * iy;
        out[y0 * f + x0] = v;
        out[y0 * f + x0 + 1] = v;
        out[(y0 + 1) * f + x0] = v;
        out[(y0 + 1) * f + x0 + 1] = v;
    }
}

__global__ void k_minmax_f64(long n, const double* __restrict__ x, double* out3) {
    // single block: min, max, count of non-finite values
    double mn = INFINITY, mx = -INFINITY, nf = 0.0;
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = x[i];
        mn = fmin(mn, v);
        mx = fmax(mx, v);
        if (!isfinite(v)) nf += 1.0;
    }
    __shared__ double s[3][32];
    mn = warp_min(mn);
    mx = warp_max(mx);
    nf = warp_sum(nf);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s[0][wid] = mn; s[1][wid] = mx; s[2][wid] = nf; }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x / 32;
        mn = lane < nw ? s[0][lane] : INFINITY;
        mx = lane < nw ? s[1][lane] : -INFINITY;
        nf = lane < nw ? s[2][lane] : 0.0;
        mn = warp_min(mn);
        mx = warp_max(mx);
        nf = warp_sum(nf);
        if (lane == 0) { out3[0] = mn; out3[1] = mx; out3[2] = nf; }
    }
}

// ---- active set (restricted levels) ------------------------------------------
// Reference: active_level and dilate_mask (src/nested_solve.cpp:72-100,
// 103-518), restricted PK solve_contact_active_impl (src/contact_solver.cpp:
// 595-1040).  The restricted PK runs as the full-grid device solve with the
// gap outside the candidate set raised to kNoContactGap: those cells can then
// never carry pressure (their gradient is huge and positive, so neither the
// projection nor the overlap correction or the identification step activates
// them), never set the minimum gradient, and contribute p v = 0 to every sum,
// which is the restricted problem and its certificate (min over the
// candidates).  Datum and g_ref come from the caller, as in the reference.
constexpr double kNoContactGap = 1e30;

__global__ void k_cand_seed(long n2, const double* __restrict__ p, uint8_t* __restrict__ m) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2;
         i += (long)gridDim.x * blockDim.x)
        m[i] = p[i] > 0.0 ? 1 : 0;
}

// Chebyshev (square) dilation by r, clamped at the grid edges: a max filter
// along rows (k_dilate_rows) then along columns (k_dilate_cols).
__global__ void k_dilate_rows(int n, int r, const uint8_t* __restrict__ in,
                              uint8_t* __restrict__ out) {
    const long n2 = (long)n * n;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2;
         i += (long)gridDim.x * blockDim.x) {
        const int iy = (int)(i / n), ix = (int)(i % n);
        const int x0 = ix - r < 0 ? 0 : ix - r, x1 = ix + r > n - 1 ? n - 1 : ix + r;
        const uint8_t* row = in + (long)iy * n;
        uint8_t v = 0;
        for (int x = x0; x <= x1 && !v; ++x) v = row[x];
        out[i] = v;
    }
}
__global__ void k_dilate_cols(int n, int r, const uint8_t* __restrict__ in,
                              uint8_t* __restrict__ out) {
    const long n2 = (long)n * n;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2;
         i += (long)gridDim.x * blockDim.x) {
        const int iy = (int)(i / n), ix = (int)(i % n);
        const int y0 = iy - r < 0 ? 0 : iy - r, y1 = iy + r > n - 1 ? n - 1 : iy + r;
        uint8_t v = 0;
        for (int y = y0; y <= y1 && !v; ++y) v = in[(long)y * n + ix];
        out[i] = v;
    }
}

// m |= (coarse gap, injected from the (n/2)^2 level below) < delta
__global__ void k_cand_gap(int n, const double* __restrict__ cg, double delta,
                           uint8_t* __restrict__ m) {
    const long n2 = (long)n * n;
    const int c = n / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2;
         i += (long)gridDim.x * blockDim.x) {
        const int iy = (int)(i / n), ix = (int)(i % n);
        if (cg[(long)(iy / 2) * c + ix / 2] < delta) m[i] = 1;
    }
}

__global__ void k_mask_or(long n2, const uint8_t* __restrict__ v, uint8_t* __restrict__ m) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2;
         i += (long)gridDim.x * blockDim.x)
        if (v[i]) m[i] = 1;
}

__global__ void k_masked_gap(long n2, const double* __restrict__ g, const uint8_t* __restrict__ m,
                             double* __restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2;
         i += (long)gridDim.x * blockDim.x)
        out[i] = m[i] ? g[i] : kNoContactGap;
}

__global__ void k_cast_f32(long n2, const double* __restrict__ x, float* __restrict__ y) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2;
         i += (long)gridDim.x * blockDim.x)
        y[i] = (float)x[i];
}

// The global check of a restricted solution (the reference's streamed
// verification, nested_solve.cpp:273-309): with u = S p over the whole grid,
// v = u + (g - gsub); per block the minimum of v over the grid and over the
// candidates and the number of violations (outside the candidates,
// v - a < vthresh; marked in viol); optionally the fields disp = u and
// gap = v - a.  part: 3 doubles per block.
template <typename T>
__global__ void k_active_verify(long n2, const T* __restrict__ u, const double* __restrict__ g,
                                double gsub, double a, double vthresh,
                                const uint8_t* __restrict__ m, uint8_t* __restrict__ viol,
                                double* __restrict__ disp, double* __restrict__ gap,
                                double* __restrict__ part) {
    double mg = INFINITY, ml = INFINITY, nv = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n2;
         i += (long)gridDim.x * blockDim.x) {
        const double ui = (double)u[i];
        const double v = ui + (g[i] - gsub);
        mg = fmin(mg, v);
        const bool cand = m[i] != 0;
        if (cand) ml = fmin(ml, v);
        const bool bad = !cand && v - a < vthresh;
        viol[i] = bad ? 1 : 0;
        nv += bad ? 1.0 : 0.0;
        if (disp) disp[i] = ui;
        if (gap) gap[i] = v - a;
    }
    __shared__ double sh[3][32];
    mg = warp_min(mg);
    ml = warp_min(ml);
    nv = warp_sum(nv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[0][wid] = mg; sh[1][wid] = ml; sh[2][wid] = nv; }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x / 32;
        mg = lane < nw ? sh[0][lane] : INFINITY;
        ml = lane < nw ? sh[1][lane] : INFINITY;
        nv = lane < nw ? sh[2][lane] : 0.0;
        mg = warp_min(mg);
        ml = warp_min(ml);
        nv = warp_sum(nv);
        if (lane == 0) {
            part[3 * blockIdx.x] = mg;
            part[3 * blockIdx.x + 1] = ml;
            part[3 * blockIdx.x + 2] = nv;
        }
    }
}

namespace {

std::mutex g_cache_mu;
std::map<std::tuple<int, int, double, double, int>, std::shared_ptr<Operator>> g_op_cache;

}  // namespace

std::shared_ptr<Operator> cached_operator(int kind, int Ns, double L, double E) {
    int dev = 0;
    ASB_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(kind, Ns, L, E, dev);
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        auto it = g_op_cache.find(key);
        if (it != g_op_cache.end()) return it->second;
    }
    auto op = std::make_shared<Operator>(kind, Ns, L, E);
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_op_cache[key] = op;
    return op;
}

void clear_operator_cache() {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_op_cache.clear();
}

// nested_solve.cpp:27-39
bool stencil_for_level(int engine, bool precond, double prev_occupancy, double occupancy_max) {
    if (!precond) return false;
    switch (engine) {
        case 1: return true;   // stencil
        case 2: return false;  // fft
        default: return prev_occupancy < 0.0 || prev_occupancy < occupancy_max;
    }
}

namespace {

inline int lgrid(long n2) { return (int)std::min(1184L, (n2 + 255) / 256); }

void dilate(int n, int r, uint8_t* m, uint8_t* tmp, cudaStream_t s) {
    if (r <= 0) return;
    const long n2 = (long)n * n;
    k_dilate_rows<<<lgrid(n2), 256, 0, s>>>(n, r, m, tmp);
    k_dilate_cols<<<lgrid(n2), 256, 0, s>>>(n, r, tmp, m);
    count_launches(2);
}

// One restricted level (reference active_level, src/nested_solve.cpp:118-518):
// candidates = dilate(p_init > 0) | (coarse gap < delta), then up to
// active_max_rounds of [restricted solve at tol/2 -> global check -> add the
// dilated violations], and the full-grid solve warm-started from the last
// restricted pressure when no round certifies.  o carries the level's
// options (tol, datum, g_ref, precond, light); p_init (the prolonged coarse
// pressure) and coarse_gap ((n/2)^2, the level below's gap field) are read
// only.  Outputs as solve_impl; r.iterations is the level's total.
void active_level(Operator& op, const aspher_solve_opts& o, bool level_float, const double* glvl,
                  double p_bar, double lvl_tol, const aspher_nested_opts& np, int n,
                  const double* p_init, const double* coarse_gap, double g_ref, double datum,
                  double* p_out, double* dout, double* gout, double* hout, int hist_cap,
                  aspher_result& r, cudaStream_t s) {
    using clk = std::chrono::steady_clock;
    const long n2 = (long)n * n;
    const int gb = lgrid(n2);
    double t_cand = 0.0;
    uint8_t *cm = nullptr, *tmp = nullptr, *viol = nullptr;
    double *ga = nullptr, *pw = nullptr, *part = nullptr, *mm_d = nullptr;
    void* u = nullptr;
    float* p32 = nullptr;
    auto release = [&]() {
        for (void* v : {(void*)cm, (void*)tmp, (void*)viol, (void*)ga, (void*)pw, (void*)part,
                        (void*)mm_d, u, (void*)p32})
            if (v) cudaFreeAsync(v, s);
    };
    try {
        ASB_CUDA(cudaMallocAsync((void**)&cm, n2, s));
        ASB_CUDA(cudaMallocAsync((void**)&tmp, n2, s));
        ASB_CUDA(cudaMallocAsync((void**)&viol, n2, s));
        ASB_CUDA(cudaMallocAsync((void**)&ga, n2 * sizeof(double), s));
        ASB_CUDA(cudaMallocAsync((void**)&pw, n2 * sizeof(double), s));
        ASB_CUDA(cudaMallocAsync((void**)&part, 3 * (size_t)gb * sizeof(double), s));
        ASB_CUDA(cudaMallocAsync((void**)&mm_d, 3 * sizeof(double), s));
        ASB_CUDA(cudaMallocAsync(&u, n2 * (level_float ? sizeof(float) : sizeof(double)), s));
        if (level_float) ASB_CUDA(cudaMallocAsync((void**)&p32, n2 * sizeof(float), s));

        // the level gap's range sets delta and the violation threshold
        k_minmax_f64<<<1, 1024, 0, s>>>(n2, glvl, mm_d);
        double mm[3];
        ASB_CUDA(cudaMemcpyAsync(mm, mm_d, sizeof(mm), cudaMemcpyDeviceToHost, s));
        ASB_CUDA(cudaStreamSynchronize(s));
        const double g_scale = mm[1] > mm[0] ? mm[1] - mm[0] : 1.0;
        const double delta = np.active_delta * g_scale;
        const double vthresh = -lvl_tol * g_scale;
        const double P_total = p_bar * (double)n2;

        auto tc = clk::now();
        k_cand_seed<<<gb, 256, 0, s>>>(n2, p_init, cm);
        count_launches(1);
        dilate(n, np.active_halo, cm, tmp, s);
        k_cand_gap<<<gb, 256, 0, s>>>(n, coarse_gap, delta, cm);
        count_launches(1);
        ASB_CUDA(cudaMemcpyAsync(pw, p_init, n2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        ASB_CUDA(cudaGetLastError());
        ASB_CUDA(cudaStreamSynchronize(s));
        t_cand += std::chrono::duration<double>(clk::now() - tc).count();

        int it_total = 0, rounds = 0, hist_used = 0;
        bool certified = false;
        aspher_result rr;
        std::memset(&rr, 0, sizeof(rr));
        std::vector<double> ph(3 * (size_t)gb);
        while (rounds < np.active_max_rounds) {
            ++rounds;
            k_masked_gap<<<gb, 256, 0, s>>>(n2, glvl, cm, ga);
            count_launches(1);
            // restricted solve at half the level tolerance: with every outside
            // gap >= -tol/2 g_scale the global certificate gains at most tol/2
            aspher_solve_opts ao = o;
            ao.tol = 0.5 * lvl_tol;
            ao.requested_tol = lvl_tol;
            ao.allow_tolerance_relaxation = 1;
            ao.light = 1;
            ao.keep_best = 1;
            ao.g_ref = g_ref;
            ao.datum = datum;
            ao.datum_mode = ASPHER_DATUM_SOLVER;
            double* hh = (hout && o.record_history && hist_used < hist_cap) ? hout + hist_used : nullptr;
            ao.record_history = hh ? 1 : 0;
            if (level_float) {
                aspher_result dummy;
                solve_mixed(op, ao, ga, p_bar, pw, ao.tol, 0, p_out, nullptr, nullptr, rr, &dummy,
                            s);
            } else {
                ao.dtype = ASPHER_F64;
                solve_impl<double>(op, ao, ga, p_bar, pw, p_out, nullptr, nullptr, hh,
                                   hist_cap - hist_used, rr, s);
            }
            if (hh) hist_used += rr.history_len;
            it_total += rr.iterations;

            // global check from a fresh full-grid apply of the restricted pressure
            tc = clk::now();
            if (level_float) {
                k_cast_f32<<<gb, 256, 0, s>>>(n2, p_out, p32);
                count_launches(1);
                op.apply_caller(false, p32, u, s);
            } else {
                op.apply_caller(true, p_out, u, s);
            }
            const double a = rr.approach - datum;  // centred approach
            if (level_float)
                k_active_verify<float><<<gb, 256, 0, s>>>(n2, (const float*)u, glvl, datum, a,
                                                          vthresh, cm, viol, nullptr, nullptr, part);
            else
                k_active_verify<double><<<gb, 256, 0, s>>>(n2, (const double*)u, glvl, datum, a,
                                                           vthresh, cm, viol, nullptr, nullptr,
                                                           part);
            count_launches(1);
            ASB_CUDA(cudaGetLastError());
            ASB_CUDA(cudaMemcpyAsync(ph.data(), part, ph.size() * sizeof(double),
                                     cudaMemcpyDeviceToHost, s));
            ASB_CUDA(cudaStreamSynchronize(s));
            double vmin_glob = INFINITY, vmin_loc = INFINITY, nviol = 0.0;
            for (int b = 0; b < gb; ++b) {
                vmin_glob = std::min(vmin_glob, ph[3 * b]);
                vmin_loc = std::min(vmin_loc, ph[3 * b + 1]);
                nviol += ph[3 * b + 2];
            }
            // G_glob = G_loc + P (vmin_loc - vmin_glob), both terms >= 0
            const double G_glob = rr.fw_gap + P_total * (vmin_loc - vmin_glob);
            const double fw_glob = G_glob / (P_total * g_ref);
            const double pen_glob = std::max(0.0, -(vmin_glob - a)) / g_ref;
            rr.fw_gap = G_glob;
            rr.fw_error = fw_glob;
            rr.penetration_error = pen_glob;
            rr.effective_tol = lvl_tol;
            t_cand += std::chrono::duration<double>(clk::now() - tc).count();
            if (rr.status == ASPHER_CONVERGED && nviol == 0.0 && fw_glob <= lvl_tol &&
                pen_glob <= lvl_tol) {
                certified = true;
                break;
            }
            if (nviol == 0.0) break;  // nothing to add: the fallback decides
            // add the dilated violations and resume from this pressure
            tc = clk::now();
            dilate(n, np.active_halo, viol, tmp, s);
            k_mask_or<<<gb, 256, 0, s>>>(n2, viol, cm);
            count_launches(1);
            ASB_CUDA(cudaMemcpyAsync(pw, p_out, n2 * sizeof(double), cudaMemcpyDeviceToDevice,
                                     s));
            ASB_CUDA(cudaStreamSynchronize(s));
            t_cand += std::chrono::duration<double>(clk::now() - tc).count();
        }

        bool fallback = false;
        if (!certified) {
            // full-grid solve warm-started from the last restricted pressure
            ASB_CUDA(cudaMemcpyAsync(pw, p_out, n2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
            aspher_solve_opts fo = o;
            fo.tol = lvl_tol;
            fo.allow_tolerance_relaxation = 1;
            fo.keep_best = !o.light;
            fo.g_ref = g_ref;
            fo.datum = datum;
            fo.datum_mode = ASPHER_DATUM_SOLVER;
            double* hh = (hout && o.record_history && hist_used < hist_cap) ? hout + hist_used : nullptr;
            fo.record_history = hh ? 1 : 0;
            if (level_float) {
                aspher_result dummy;
                solve_mixed(op, fo, glvl, p_bar, pw, lvl_tol, 0, p_out, dout, gout, rr, &dummy, s);
            } else {
                fo.dtype = ASPHER_F64;
                solve_impl<double>(op, fo, glvl, p_bar, pw, p_out, dout, gout, hh,
                                   hist_cap - hist_used, rr, s);
            }
            if (hh) hist_used += rr.history_len;
            it_total += rr.iterations;
            fallback = true;
        } else if (!o.light && (dout || gout)) {
            // the fields from the certifying apply (u still holds it)
            const double a = rr.approach - datum;
            if (level_float)
                k_active_verify<float><<<gb, 256, 0, s>>>(n2, (const float*)u, glvl, datum, a,
                                                          vthresh, cm, viol, dout, gout, part);
            else
                k_active_verify<double><<<gb, 256, 0, s>>>(n2, (const double*)u, glvl, datum, a,
                                                           vthresh, cm, viol, dout, gout, part);
            count_launches(1);
            ASB_CUDA(cudaGetLastError());
        }
        rr.iterations = it_total;
        rr.history_len = hist_used;
        // an uncertified restricted result never reports success (the
        // fallback carries its own global certificate)
        if (!certified && !fallback && rr.status == ASPHER_CONVERGED) {
            rr.status = ASPHER_VERIFICATION_FAILED;
            std::strncpy(rr.status_reason, "global_check", sizeof(rr.status_reason) - 1);
        }
        rr.converged = rr.status == ASPHER_CONVERGED;
        rr.active_rounds = rounds;
        rr.active_fallback = fallback ? 1 : 0;
        rr.time_candidate = t_cand;
        r = rr;
        release();
        ASB_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        release();
        throw;
    }
}

}  // namespace

void solve_nested(int kind, int Ns, double L, double E, const double* g0, double p_bar,
                  const aspher_nested_opts& np, double* pressure, double* disp, double* gap,
                  double* hist_host, int hist_cap, aspher_result& res, aspher_stage* stages,
                  int stage_cap, int* nstages, cudaStream_t s) {
    using clk = std::chrono::steady_clock;
    const auto t_nested = clk::now();
    auto pow2 = [](long v) { return v > 0 && (v & (v - 1)) == 0; };
    // ---- validation before any allocation or iteration (nested_solve.cpp:523-617)
    if (Ns <= 0) throw Error(ASPHER_EINVAL, "solve_contact_nested: Ns must be positive");
    if (!(L > 0.0) || !std::isfinite(L)) throw Error(ASPHER_EINVAL, "solve_contact_nested: L must be positive");
    if (!(E > 0.0) || !std::isfinite(E)) throw Error(ASPHER_EINVAL, "solve_contact_nested: E_star must be positive");
    if (!(p_bar > 0.0) || !std::isfinite(p_bar))
        throw Error(ASPHER_EINVAL, "solve_contact_nested: p_nominal must be positive");
    if (!(np.tol > 0.0) || !std::isfinite(np.tol))
        throw Error(ASPHER_EINVAL, "solve_contact_nested: tol must be positive");
    if (np.max_iter < 0) throw Error(ASPHER_EINVAL, "solve_contact_nested: max_iter must be >= 0");
    if (np.coarsest <= 0) throw Error(ASPHER_EINVAL, "solve_contact_nested: coarsest must be positive");
    if (np.coarsest > Ns) throw Error(ASPHER_EINVAL, "solve_contact_nested: coarsest > Ns");
    if (np.leaf_side <= 0 || !pow2(np.leaf_side))
        throw Error(ASPHER_EINVAL, "solve_contact_nested: leaf_side must be a positive power of two");
    if (!(np.coarse_tol > 0.0)) throw Error(ASPHER_EINVAL, "solve_contact_nested: coarse_tol must be positive");
    if (!(np.precond_occupancy_max > 0.0))
        throw Error(ASPHER_EINVAL, "solve_contact_nested: precond_occupancy_max must be > 0");
    if (!(np.float_floor > 0.0)) throw Error(ASPHER_EINVAL, "solve_contact_nested: float_floor must be positive");
    if (np.precond_engine < 0 || np.precond_engine > 2)
        throw Error(ASPHER_EINVAL, "precond_engine must be 'auto', 'stencil' or 'fft'");
    int policy = np.precision;  // 0 defer, 1 double, 2 float, 3 float_then_double
    if (policy == 0) policy = np.single_precision ? 2 : 1;
    if (policy < 1 || policy > 3) throw Error(ASPHER_EINVAL, "precision must be 'double', 'float', 'float_then_double' or ''");
    const bool any_float = policy != 1;
    if (np.active_set) {  // nested_solve.cpp:567-580,593-597
        if (np.active_halo < 0)
            throw Error(ASPHER_EINVAL, "solve_contact_nested: active_halo must be >= 0");
        if (np.active_max_rounds < 1)
            throw Error(ASPHER_EINVAL, "solve_contact_nested: active_max_rounds must be >= 1");
        if (!(np.active_delta >= 0.0))
            throw Error(ASPHER_EINVAL, "solve_contact_nested: active_delta must be >= 0");
        if (!(np.active_occupancy_max > 0.0))
            throw Error(ASPHER_EINVAL, "solve_contact_nested: active_occupancy_max must be > 0");
        if (policy == 3)
            throw Error(ASPHER_EINVAL, "solve_contact_nested: float_then_double does not route "
                                       "its polish through the active-set path; use float or "
                                       "double with active_set=true");
    }
    std::vector<int> levels;
    for (int n = np.coarsest; n <= Ns; n *= 2) levels.push_back(n);
    if (levels.empty() || levels.back() != Ns)
        throw Error(ASPHER_EINVAL, "solve_contact_nested: Ns must equal coarsest * 2^k");
    // levels that are not powers of two >= 16 run on embedded operators;
    // the FFT preconditioner engine needs power-of-two levels
    const int engine0 = (kind == OP_PERIODIC && np.precond_engine == 0) ? 2 : np.precond_engine;
    for (int n : levels) {
        if (n > kMaxNs) throw Error(ASPHER_EINVAL, "solve_contact_nested: Ns must be <= 16384");
        if (np.precond && engine0 == 2 && (!pow2(n) || n < 16) && n % 2)
            throw Error(ASPHER_EINVAL, "solve_contact_nested: the fft preconditioner engine needs "
                                       "even levels (use precond_engine='stencil')");
    }
    if (np.active_set && levels.size() < 2)
        throw Error(ASPHER_EINVAL, "solve_contact_nested: active_set needs a coarse level "
                                   "(Ns > coarsest)");

    const long N = (long)Ns * Ns;
    // gap statistics (FP64) -> datum and g_ref (nested_solve.cpp:634-636)
    double* mm_d = nullptr;
    ASB_CUDA(cudaMallocAsync((void**)&mm_d, 3 * sizeof(double), s));
    k_minmax_f64<<<1, 1024, 0, s>>>(N, g0, mm_d);
    count_launches(1);
    double mm[3];
    ASB_CUDA(cudaMemcpyAsync(mm, mm_d, sizeof(mm), cudaMemcpyDeviceToHost, s));
    ASB_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(mm_d, s);
    if (mm[2] > 0.0) throw Error(ASPHER_EINVAL, "solve_contact_nested: gap contains non-finite values");
    const double datum = mm[0] + 0.5 * (mm[1] - mm[0]);
    const double g_ref = std::max(mm[1] - mm[0], p_bar * L / E);

    // restriction hierarchy (coarse levels only; the finest reads g0)
    const int ncoarse = (int)levels.size() - 1;
    std::vector<double*> gaps(ncoarse, nullptr);
    for (int i = ncoarse - 1; i >= 0; --i) {
        const int n = levels[i];
        ASB_CUDA(cudaMallocAsync((void**)&gaps[i], (size_t)n * n * sizeof(double), s));
        const double* src = (i == ncoarse - 1) ? g0 : gaps[i + 1];
        k_restrict<<<std::min(1184L, ((long)n * n + 255) / 256), 256, 0, s>>>(2 * n, src, gaps[i]);
        count_launches(1);
    }
    ASB_CUDA(cudaGetLastError());

    double* p_init = nullptr;   // prolonged pressure for the current level (FP64)
    double* p_lvl = nullptr;    // current level's pressure output (FP64)
    double* coarse_gap = nullptr;  // gap field of the level below (active set only)
    double* gap_keep = nullptr;    // this level's gap field, kept for the next level
    double t_build = 0.0, t_coarse = 0.0, t_candidate = 0.0;
    double prev_occupancy = -1.0;
    int ns = 0;
    auto record = [&](const std::string& name, const char* prec, double req, double eff,
                      const aspher_result& r) {
        if (stages && ns < stage_cap) {
            aspher_stage& st = stages[ns];
            std::memset(&st, 0, sizeof(st));
            std::strncpy(st.name, name.c_str(), sizeof(st.name) - 1);
            std::strncpy(st.precision, prec, sizeof(st.precision) - 1);
            st.q = np.q;
            st.requested_tol = req;
            st.effective_tol = eff;
            st.iterations = r.iterations;
            st.matvec_count = r.matvec_count;
            st.seconds = r.time_total;
            st.status = r.status;
            st.fw_error = r.fw_error;
            st.penetration_error = r.penetration_error;
        }
        ++ns;
    };
    try {
        for (size_t li = 0; li < levels.size(); ++li) {
            const int n = levels[li];
            const long Nl = (long)n * n;
            const bool finest = li + 1 == levels.size();
            const auto tb = clk::now();
            std::shared_ptr<Operator> op = cached_operator(kind, n, L, E);
            // periodic: `auto` means the FFT engine (nested_solve.cpp:717-721)
            const int engine = (kind == OP_PERIODIC && np.precond_engine == 0) ? 2 : np.precond_engine;
            bool use_stencil = stencil_for_level(engine, np.precond != 0, prev_occupancy,
                                                 np.precond_occupancy_max);
            // an odd embedded level has no FFT preconditioner: under `auto`
            // it keeps the stencil where the reference would switch
            if (!use_stencil && np.precond && engine == 0 && op->embedded() && n % 2)
                use_stencil = true;
            const int r_lvl = std::min({np.precond_radius, std::max(1, n / 4), np.leaf_side});
            const int pc = use_stencil ? ASPHER_PRECOND_STENCIL
                                       : (np.precond ? ASPHER_PRECOND_FFT : ASPHER_PRECOND_NONE);
            if (use_stencil) (void)make_stencil_taps(n, r_lvl);  // validate + cache up front
            t_build += std::chrono::duration<double>(clk::now() - tb).count();

            const double* glvl = finest ? g0 : gaps[li];
            const bool polish_after = finest && policy == 3;
            double lvl_tol = finest ? np.tol : np.coarse_tol;
            if (polish_after) lvl_tol = np.float_floor;
            else if (any_float) lvl_tol = std::max(lvl_tol, np.float_floor);
            // a level that the next one restricts keeps its gap field (the
            // next candidate set is built from it); whether the next level is
            // restricted is predicted from the occupancy of the level below
            // (nested_solve.cpp:752-787)
            const bool gate_open_next = prev_occupancy < 0.0 ||
                                        prev_occupancy < np.active_occupancy_max;
            const bool keep_gap = np.active_set && !finest && gate_open_next &&
                                  (np.active_all_levels || li + 2 == levels.size());
            const bool light = finest ? (np.light_result != 0) : !keep_gap;
            const bool use_active = np.active_set && p_init && coarse_gap &&
                                    prev_occupancy < np.active_occupancy_max &&
                                    (finest || np.active_all_levels);

            aspher_solve_opts o;
            aspher_solve_opts_default(&o);
            o.tol = lvl_tol;
            o.requested_tol = finest ? np.tol : np.coarse_tol;
            o.max_iter = np.max_iter;
            o.use_pr = np.use_pr;
            o.light = light;
            o.record_history = finest && np.record_error_history;
            o.keep_best = !light;
            o.allow_tolerance_relaxation = (!finest || polish_after || np.allow_tolerance_relaxation);
            o.g_ref = g_ref;
            o.datum = datum;
            o.precond = pc;
            o.precond_radius = r_lvl;

            ASB_CUDA(cudaMallocAsync((void**)&p_lvl, (size_t)Nl * sizeof(double), s));
            double* dout = finest ? disp : nullptr;
            double* gout = finest ? gap : nullptr;
            if (keep_gap) {
                ASB_CUDA(cudaMallocAsync((void**)&gap_keep, (size_t)Nl * sizeof(double), s));
                gout = gap_keep;
            }
            double* hout = o.record_history ? hist_host : nullptr;
            aspher_result r;
            std::memset(&r, 0, sizeof(r));
            if (use_active) {
                active_level(*op, o, any_float, glvl, p_bar, lvl_tol, np, n, p_init, coarse_gap,
                             g_ref, datum, p_lvl, dout, gout, hout, hist_cap, r, s);
                r.requested_tol = o.requested_tol;
                t_candidate += r.time_candidate;
                record(std::string(finest ? "finest:" : "coarse:") + std::to_string(n) +
                           "(active)",
                       any_float ? "float" : "double", o.requested_tol, o.tol, r);
            } else if (any_float) {
                // FP32 level: datum removed inside the cast (nested_solve.cpp:871-917)
                o.datum_mode = ASPHER_DATUM_SOLVER;
                if (polish_after) {
                    aspher_result rf;
                    solve_mixed(*op, o, glvl, p_bar, p_init, lvl_tol, 0, p_lvl, nullptr, nullptr,
                                rf, nullptr, s);
                    // solve_mixed with polish=0 returns the FP32 stage in rf
                    record("finest:" + std::to_string(n), "float", o.requested_tol, o.tol, rf);
                    aspher_solve_opts od = o;
                    od.tol = np.tol;
                    od.requested_tol = np.tol;
                    od.light = np.light_result;
                    od.keep_best = !np.light_result;
                    od.allow_tolerance_relaxation = np.allow_tolerance_relaxation;
                    od.datum_mode = ASPHER_DATUM_SOLVER;
                    od.dtype = ASPHER_F64;
                    solve_impl<double>(*op, od, glvl, p_bar, p_lvl, p_lvl, dout, gout, hout,
                                       hist_cap, r, s, /*polish_stage=*/true);
                    record("polish:" + std::to_string(n), "double", np.tol, np.tol, r);
                    r.iterations += rf.iterations;
                    r.matvec_count += rf.matvec_count;
                    r.precond_count += rf.precond_count;
                    r.time_total += rf.time_total;
                } else {
                    aspher_result dummy;
                    solve_mixed(*op, o, glvl, p_bar, p_init, lvl_tol, 0, p_lvl, dout, gout, r,
                                &dummy, s);
                    record(std::string(finest ? "finest:" : "coarse:") + std::to_string(n),
                           "float", o.requested_tol, o.tol, r);
                }
            } else {
                o.datum_mode = ASPHER_DATUM_SOLVER;
                o.dtype = ASPHER_F64;
                solve_impl<double>(*op, o, glvl, p_bar, p_init, p_lvl, dout, gout, hout,
                                   hist_cap, r, s);
                record(std::string(finest ? "finest:" : "coarse:") + std::to_string(n), "double",
                       o.requested_tol, o.tol, r);
            }
            prev_occupancy = r.contact_fraction;
            if (p_init) {
                cudaFreeAsync(p_init, s);
                p_init = nullptr;
            }
            if (coarse_gap) {  // consumed by this level
                cudaFreeAsync(coarse_gap, s);
                coarse_gap = nullptr;
            }
            if (gap_keep) {
                coarse_gap = gap_keep;
                gap_keep = nullptr;
            }
            if (!finest) {
                t_coarse += r.time_total;
                ASB_CUDA(cudaMallocAsync((void**)&p_init, (size_t)4 * Nl * sizeof(double), s));
                k_prolong<<<std::min(1184L, (Nl + 255) / 256), 256, 0, s>>>(n, p_lvl, p_init);
                count_launches(1);
                ASB_CUDA(cudaGetLastError());
                cudaFreeAsync(gaps[li], s);
                gaps[li] = nullptr;
                cudaFreeAsync(p_lvl, s);
                p_lvl = nullptr;
            } else {
                ASB_CUDA(cudaMemcpyAsync(pressure, p_lvl, (size_t)Nl * sizeof(double),
                                         cudaMemcpyDeviceToDevice, s));
                res = r;
            }
        }
    } catch (...) {
        for (double* gp : gaps) if (gp) cudaFreeAsync(gp, s);
        if (p_init) cudaFreeAsync(p_init, s);
        if (p_lvl) cudaFreeAsync(p_lvl, s);
        if (coarse_gap) cudaFreeAsync(coarse_gap, s);
        if (gap_keep) cudaFreeAsync(gap_keep, s);
        throw;
    }
    if (p_lvl) cudaFreeAsync(p_lvl, s);
    if (coarse_gap) cudaFreeAsync(coarse_gap, s);
    ASB_CUDA(cudaStreamSynchronize(s));
    if (nstages) *nstages = std::min(ns, stage_cap);
    res.time_build = t_build;
    res.time_coarse = t_coarse;
    res.time_candidate = t_candidate;
    res.time_total = std::chrono::duration<double>(clk::now() - t_nested).count();
}

}  // namespace asb
