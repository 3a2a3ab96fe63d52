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
    if (np.active_set)
        throw Error(ASPHER_EINVAL, "solve_contact_nested: active_set requires backend='h2' "
                                   "(masked matvec)");
    std::vector<int> levels;
    for (int n = np.coarsest; n <= Ns; n *= 2) levels.push_back(n);
    if (levels.empty() || levels.back() != Ns)
        throw Error(ASPHER_EINVAL, "solve_contact_nested: Ns must equal coarsest * 2^k");
    for (int n : levels)
        if (!pow2(n) || n < 16)
            throw Error(ASPHER_EINVAL, "solve_contact_nested: every level must be a power of two "
                                       ">= 16 on this device path");

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
    double t_build = 0.0, t_coarse = 0.0;
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
            const bool use_stencil = stencil_for_level(engine, np.precond != 0, prev_occupancy,
                                                       np.precond_occupancy_max);
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
            const bool light = finest ? (np.light_result != 0) : true;

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
            double* hout = o.record_history ? hist_host : nullptr;
            aspher_result r;
            if (any_float) {
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
        throw;
    }
    if (p_lvl) cudaFreeAsync(p_lvl, s);
    ASB_CUDA(cudaStreamSynchronize(s));
    if (nstages) *nstages = std::min(ns, stage_cap);
    res.time_build = t_build;
    res.time_coarse = t_coarse;
    res.time_total = std::chrono::duration<double>(clk::now() - t_nested).count();
}

}  // namespace asb
