// C-ABI entry points of the solver and the preconditioners.
#include "../../include/aspher_b200.h"
#include "ops.hpp"
#include "pcg.hpp"

#include <cstring>

struct aspher_op {
    asb::Operator* impl;
};

#define ASB_API_BEGIN try {
#define ASB_API_END                                               \
    }                                                             \
    catch (const asb::Error& e) {                                 \
        asb::set_last_error(e.what());                            \
        return e.code;                                            \
    }                                                             \
    catch (const std::exception& e) {                             \
        asb::set_last_error(e.what());                            \
        return ASPHER_ECUDA;                                      \
    }                                                             \
    catch (...) {                                                 \
        asb::set_last_error("unknown error");                     \
        return ASPHER_ECUDA;                                      \
    }

extern "C" {

const char* aspher_status_string(int s) {
    switch (s) {
        case ASPHER_CONVERGED: return "converged";
        case ASPHER_STAGNATED: return "stagnated";
        case ASPHER_MAX_ITERATIONS: return "max_iterations";
        case ASPHER_NONPOSITIVE_CURVATURE: return "nonpositive_curvature";
        case ASPHER_NONFINITE: return "nonfinite";
        case ASPHER_VERIFICATION_FAILED: return "verification_failed";
        case ASPHER_RESOURCE_LIMIT: return "resource_limit";
    }
    return "unknown";
}

void aspher_solve_opts_default(aspher_solve_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-8;
    o->requested_tol = 0.0;
    o->max_iter = 5000;
    o->use_pr = 1;
    o->light = 0;
    o->record_history = 0;
    o->keep_best = 1;
    o->load_tol = 0.0;
    o->stall_limit = 200;
    o->allow_tolerance_relaxation = 0;
    o->precond = ASPHER_PRECOND_NONE;
    o->precond_radius = 2;
    o->p_ref = 0.0;
    o->g_ref = 0.0;
    o->datum_mode = ASPHER_DATUM_AUTOMATIC;
    o->datum = 0.0;
    o->dtype = ASPHER_F64;
}

int aspher_solve(aspher_op* op, const aspher_solve_opts* opts, const void* g0_dev, double p_bar,
                 const void* p_init_dev, double* pressure_dev, double* displacement_dev,
                 double* gap_dev, double* history_host, int history_cap, aspher_result* res,
                 void* stream) {
    ASB_API_BEGIN
    if (!op || !op->impl || !opts || !g0_dev || !pressure_dev || !res)
        throw asb::Error(ASPHER_EINVAL, "aspher_solve: NULL argument");
    if (opts->dtype != ASPHER_F32 && opts->dtype != ASPHER_F64)
        throw asb::Error(ASPHER_EINVAL, "aspher_solve: dtype must be F32 or F64");
    const uintptr_t a = (uintptr_t)g0_dev | (uintptr_t)pressure_dev |
                        (uintptr_t)p_init_dev | (uintptr_t)displacement_dev |
                        (uintptr_t)gap_dev;
    if (a % 16) throw asb::Error(ASPHER_EINVAL, "aspher_solve: buffers must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (opts->dtype == ASPHER_F64)
        asb::solve_impl<double>(*op->impl, *opts, g0_dev, p_bar, p_init_dev, pressure_dev,
                                displacement_dev, gap_dev, history_host, history_cap, *res, s);
    else
        asb::solve_impl<float>(*op->impl, *opts, g0_dev, p_bar, p_init_dev, pressure_dev,
                               displacement_dev, gap_dev, history_host, history_cap, *res, s);
    return ASPHER_OK;
    ASB_API_END
}

int aspher_solve_mixed(aspher_op* op, const aspher_solve_opts* opts, const double* g0_dev,
                       double p_bar, const double* p_init_dev, double float_tol, int polish,
                       double* pressure_dev, double* displacement_dev, double* gap_dev,
                       aspher_result* res, aspher_result* res_float, void* stream) {
    ASB_API_BEGIN
    if (!op || !op->impl || !opts || !g0_dev || !pressure_dev || !res)
        throw asb::Error(ASPHER_EINVAL, "aspher_solve_mixed: NULL argument");
    if (!(float_tol > 0.0)) throw asb::Error(ASPHER_EINVAL, "aspher_solve_mixed: float_tol must be positive");
    const uintptr_t a = (uintptr_t)g0_dev | (uintptr_t)pressure_dev | (uintptr_t)p_init_dev |
                        (uintptr_t)displacement_dev | (uintptr_t)gap_dev;
    if (a % 16) throw asb::Error(ASPHER_EINVAL, "aspher_solve_mixed: buffers must be 16-byte aligned");
    asb::solve_mixed(*op->impl, *opts, g0_dev, p_bar, p_init_dev, float_tol, polish, pressure_dev,
                     displacement_dev, gap_dev, *res, res_float, static_cast<cudaStream_t>(stream));
    return ASPHER_OK;
    ASB_API_END
}

int aspher_solve_batch(aspher_op* op, const aspher_solve_opts* opts, int batch,
                       const void* const* g0_devs, const double* p_bars,
                       const void* const* p_init_devs, double* const* pressure_devs,
                       aspher_result* res, void* stream) {
    ASB_API_BEGIN
    if (!op || !op->impl || !opts || !g0_devs || !p_bars || !pressure_devs || !res)
        throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch: NULL argument");
    if (batch < 1) throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch: batch must be >= 1");
    for (int b = 0; b < batch; ++b) {
        if (!g0_devs[b] || !pressure_devs[b])
            throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch: NULL field");
        const uintptr_t a = (uintptr_t)g0_devs[b] | (uintptr_t)pressure_devs[b] |
                            (uintptr_t)(p_init_devs ? p_init_devs[b] : nullptr);
        if (a % 16) throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch: buffers must be 16-byte aligned");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (opts->dtype == ASPHER_F64)
        asb::solve_batch_impl<double>(*op->impl, *opts, batch, g0_devs, p_bars, p_init_devs,
                                      pressure_devs, res, s);
    else if (opts->dtype == ASPHER_F32)
        asb::solve_batch_impl<float>(*op->impl, *opts, batch, g0_devs, p_bars, p_init_devs,
                                     pressure_devs, res, s);
    else
        throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch: dtype must be F32 or F64");
    return ASPHER_OK;
    ASB_API_END
}

int aspher_solve_batch_mixed(aspher_op* op, const aspher_solve_opts* opts, int batch,
                             const double* const* g0_devs, const double* p_bars, double float_tol,
                             int polish, double* const* pressure_devs, aspher_result* res,
                             aspher_result* res_float, void* stream) {
    ASB_API_BEGIN
    if (!op || !op->impl || !opts || !g0_devs || !p_bars || !pressure_devs || !res)
        throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch_mixed: NULL argument");
    if (batch < 1) throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch_mixed: batch must be >= 1");
    if (!(float_tol > 0.0))
        throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch_mixed: float_tol must be positive");
    for (int b = 0; b < batch; ++b) {
        if (!g0_devs[b] || !pressure_devs[b])
            throw asb::Error(ASPHER_EINVAL, "aspher_solve_batch_mixed: NULL field");
        if (((uintptr_t)g0_devs[b] | (uintptr_t)pressure_devs[b]) % 16)
            throw asb::Error(ASPHER_EINVAL,
                             "aspher_solve_batch_mixed: buffers must be 16-byte aligned");
    }
    asb::solve_batch_mixed(*op->impl, *opts, batch, g0_devs, p_bars, float_tol, polish,
                           pressure_devs, res, res_float, static_cast<cudaStream_t>(stream));
    return ASPHER_OK;
    ASB_API_END
}

int aspher_adjoint(aspher_op* op, int dtype, const double* p_dev, const double* w_dev,
                   double tol, int max_iter, int precond, int precond_radius,
                   double* grad_g0_dev, double* grad_pbar, aspher_adjoint_info* info,
                   void* stream) {
    ASB_API_BEGIN
    if (!op || !op->impl || !p_dev || !w_dev || !grad_g0_dev)
        throw asb::Error(ASPHER_EINVAL, "aspher_adjoint: NULL argument");
    if (((uintptr_t)p_dev | (uintptr_t)w_dev | (uintptr_t)grad_g0_dev) % 16)
        throw asb::Error(ASPHER_EINVAL, "aspher_adjoint: buffers must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == ASPHER_F64)
        asb::adjoint_impl<double>(*op->impl, p_dev, w_dev, tol, max_iter, precond,
                                  precond_radius, grad_g0_dev, grad_pbar, info, s);
    else if (dtype == ASPHER_F32)
        asb::adjoint_impl<float>(*op->impl, p_dev, w_dev, tol, max_iter, precond,
                                 precond_radius, grad_g0_dev, grad_pbar, info, s);
    else
        throw asb::Error(ASPHER_EINVAL, "aspher_adjoint: dtype must be F32 or F64");
    return ASPHER_OK;
    ASB_API_END
}

int aspher_precond_apply(aspher_op* op, int precond, int radius, int dtype, const void* g_dev,
                         const uint8_t* contact_dev, void* z_dev, void* stream) {
    ASB_API_BEGIN
    if (!op || !op->impl || !g_dev || !contact_dev || !z_dev)
        throw asb::Error(ASPHER_EINVAL, "aspher_precond_apply: NULL argument");
    if (precond != ASPHER_PRECOND_STENCIL && precond != ASPHER_PRECOND_FFT)
        throw asb::Error(ASPHER_EINVAL, "aspher_precond_apply: precond must be STENCIL or FFT");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == ASPHER_F64)
        asb::precond_apply_impl<double>(*op->impl, precond, radius, (const double*)g_dev,
                                        contact_dev, (double*)z_dev, s);
    else if (dtype == ASPHER_F32)
        asb::precond_apply_impl<float>(*op->impl, precond, radius, (const float*)g_dev,
                                       contact_dev, (float*)z_dev, s);
    else
        throw asb::Error(ASPHER_EINVAL, "aspher_precond_apply: dtype must be F32 or F64");
    return ASPHER_OK;
    ASB_API_END
}

void aspher_nested_opts_default(aspher_nested_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-8;
    o->max_iter = 20000;
    o->use_pr = 1;
    o->coarsest = 64;
    o->q = 6;
    o->leaf_side = 8;
    o->precond = 1;
    o->precond_engine = 0;
    o->precond_radius = 2;
    o->precond_occupancy_max = 0.4;
    o->coarse_tol = 1e-4;
    o->single_precision = 0;
    o->precision = 0;
    o->float_floor = 2e-6;
    o->allow_tolerance_relaxation = 0;
    o->light_result = 0;
    o->record_error_history = 0;
    o->active_set = 0;
    o->active_delta = 0.05;
    o->active_halo = 2;
    o->active_max_rounds = 5;
    o->active_all_levels = 1;
    o->active_occupancy_max = 0.4;
}

int aspher_solve_nested(int backend, int grid_size, double domain_size, double E_star,
                        const double* g0_dev, double p_bar, const aspher_nested_opts* opts,
                        double* pressure_dev, double* displacement_dev, double* gap_dev,
                        double* history_host, int history_cap, aspher_result* res,
                        aspher_stage* stages, int stage_cap, int* nstages, void* stream) {
    ASB_API_BEGIN
    if (!opts || !g0_dev || !pressure_dev || !res)
        throw asb::Error(ASPHER_EINVAL, "aspher_solve_nested: NULL argument");
    if (backend != ASPHER_BACKEND_FFT && backend != ASPHER_BACKEND_PERIODIC)
        throw asb::Error(ASPHER_EINVAL, "solve_contact_nested: backend must be 'fft' or "
                                        "'periodic' on this build");
    const uintptr_t a = (uintptr_t)g0_dev | (uintptr_t)pressure_dev |
                        (uintptr_t)displacement_dev | (uintptr_t)gap_dev;
    if (a % 16) throw asb::Error(ASPHER_EINVAL, "aspher_solve_nested: buffers must be 16-byte aligned");
    asb::solve_nested(backend, grid_size, domain_size, E_star, g0_dev, p_bar, *opts, pressure_dev,
                      displacement_dev, gap_dev, history_host, history_cap, *res, stages,
                      stage_cap, nstages, static_cast<cudaStream_t>(stream));
    return ASPHER_OK;
    ASB_API_END
}

int aspher_stencil_for_level(int engine, int precond, double prev_occupancy,
                             double occupancy_max) {
    return asb::stencil_for_level(engine, precond != 0, prev_occupancy, occupancy_max) ? 1 : 0;
}

int aspher_operator_cache_clear(void) {
    ASB_API_BEGIN
    asb::clear_operator_cache();
    return ASPHER_OK;
    ASB_API_END
}

int aspher_stencil_taps(int grid_size, int radius, int* dx, int* dy, double* w, int cap,
                        int* ntaps) {
    ASB_API_BEGIN
    if (!dx || !dy || !w || !ntaps) throw asb::Error(ASPHER_EINVAL, "aspher_stencil_taps: NULL");
    const asb::StencilTaps t = asb::make_stencil_taps(grid_size, radius);
    const int n = t.n < cap ? t.n : cap;
    for (int i = 0; i < n; ++i) {
        dx[i] = t.dx[i];
        dy[i] = t.dy[i];
        w[i] = t.w[i];
    }
    *ntaps = t.n;
    return ASPHER_OK;
    ASB_API_END
}

}  // extern "C"
