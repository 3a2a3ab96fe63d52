// C-ABI harness around the reference's own hot-path C++ (TEST INFRASTRUCTURE).
//
// oracle/Makefile compiles this file together with the UNMODIFIED reference
// sources, read in place from the reference tree (src/contact_solver.cpp,
// src/fft_operator.cpp, src/periodic_fft_operator.cpp,
// src/boussinesq_kernel.cpp, src/stencil_precond.cpp,
// src/fourier_precond.cpp with the vendored pocketfft,
// src/cerruti_kernel.cpp), against the
// project's Eigen-API shim (oracle/eigen_shim), into oracle/_ref/
// libaspher_ref.so.  Only tests/, __graft_entry__.smoke() and bench.py's
// reference / CPU-baseline legs load it (oracle/ref.py), as the checker and
// the timed CPU baseline; the product never does.
//
// The wiring restates python/bindings.cpp:115-214 (ContactSolver: operator
// per backend, precond "fourier" = StencilPreconditioner(Ns, 2),
// "fourier-fft" = FourierPreconditioner(Ns)) and src/contact_solver.cpp:
// 1051-1082 (solve_contact -> solve_contact_impl<double> with default
// SolveOptions), plus the float working precision of solve_contact_impl
// <float> with matvec_single_into / apply_single_into that the reference's
// nested driver uses for its float stages (src/nested_solve.cpp:871-917).
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "boussinesq_kernel.hpp"
#include "cerruti_kernel.hpp"
#include "contact_solver.hpp"
#include "fft_engine.hpp"
#include "friction_solve.hpp"
#include "fft_operator.hpp"
#include "fourier_precond.hpp"
#include "periodic_fft_operator.hpp"
#include "stencil_precond.hpp"

namespace {

thread_local std::string g_err;

struct RefOp {
    int backend = 0;  // 0 fft (free space), 1 periodic
    int Ns = 0;
    std::unique_ptr<hmc::BoussinesqKernel> kernel;
    std::unique_ptr<hmc::FFTOperator> fft;
    std::unique_ptr<hmc::PeriodicFFTOperator> periodic;
    std::unique_ptr<hmc::StencilPreconditioner> stencil;
    std::unique_ptr<hmc::FourierPreconditioner> fourier;

    template <class Real>
    void apply(const hmc::VecT<Real>& x, hmc::VecT<Real>& y) const {
        if constexpr (std::is_same_v<Real, double>) {
            if (backend == 0) fft->matvec_into(x, y);
            else periodic->matvec_into(x, y);
        } else {
            if (backend == 0) fft->matvec_single_into(x, y);
            else periodic->matvec_single_into(x, y);
        }
    }
};

// Fixed layout of the scalar results (aref_solve's `out`, 24 doubles).
enum {
    R_STATUS = 0, R_ITER, R_CONVERGED, R_CONTACT, R_MEAN_P, R_APPROACH, R_OBJECTIVE,
    R_ERROR, R_FW_GAP, R_FW_ERROR, R_LOAD_ERROR, R_PVIOL, R_PEN_ERROR, R_REQ_TOL,
    R_EFF_TOL, R_P_REF, R_G_REF, R_MATVECS, R_PRECONDS, R_IDENT, R_RETURNED_BEST,
    R_TIME, R_HISTORY_LEN, R_NSCALARS
};

template <class Real>
int solve_t(RefOp* op, const double* g0, double p_bar, const hmc::SolveOptions& opt,
            int precond, int radius, const double* p_init, double* pressure, double* disp,
            double* gap, double* out, double* history, int history_cap, char* status_out) {
    const int64_t N = int64_t(op->Ns) * op->Ns;
    hmc::VecT<Real> g(N);
    for (int64_t i = 0; i < N; ++i) g(i) = Real(g0[i]);
    hmc::MatVecIntoT<Real> S = [op](const hmc::VecT<Real>& x, hmc::VecT<Real>& y) {
        op->apply<Real>(x, y);
    };
    hmc::PrecondIntoT<Real> pc;
    if (precond == 1) {
        if (!op->stencil || op->stencil->radius() != radius)
            op->stencil = std::make_unique<hmc::StencilPreconditioner>(op->Ns, radius);
        hmc::StencilPreconditioner* sp = op->stencil.get();
        pc = [sp](const hmc::VecT<Real>& gg, const std::vector<std::uint8_t>& c,
                  hmc::VecT<Real>& z) {
            if constexpr (std::is_same_v<Real, double>) sp->apply_into(gg, c, z);
            else sp->apply_single_into(gg, c, z);
        };
    } else if (precond == 2) {
        if (!op->fourier) op->fourier = std::make_unique<hmc::FourierPreconditioner>(op->Ns);
        hmc::FourierPreconditioner* fp = op->fourier.get();
        pc = [fp](const hmc::VecT<Real>& gg, const std::vector<std::uint8_t>& c,
                  hmc::VecT<Real>& z) {
            if constexpr (std::is_same_v<Real, double>) fp->apply_into(gg, c, z);
            else fp->apply_single_into(gg, c, z);
        };
    }
    hmc::VecT<Real> p0;
    if (p_init) {
        p0.resize(N);
        for (int64_t i = 0; i < N; ++i) p0(i) = Real(p_init[i]);
    }
    hmc::ContactResult r = hmc::solve_contact_impl<Real>(S, g, Real(p_bar), opt, pc,
                                                         p_init ? &p0 : nullptr);
    std::memcpy(pressure, r.pressure.data(), sizeof(double) * N);
    if (disp && r.displacement.size() == N)
        std::memcpy(disp, r.displacement.data(), sizeof(double) * N);
    if (gap && r.gap.size() == N) std::memcpy(gap, r.gap.data(), sizeof(double) * N);
    out[R_STATUS] = double(int(r.status));
    out[R_ITER] = r.iterations;
    out[R_CONVERGED] = r.converged ? 1.0 : 0.0;
    out[R_CONTACT] = r.contact_fraction;
    out[R_MEAN_P] = r.mean_pressure;
    out[R_APPROACH] = r.approach;
    out[R_OBJECTIVE] = r.objective;
    out[R_ERROR] = r.error;
    out[R_FW_GAP] = r.fw_gap;
    out[R_FW_ERROR] = r.fw_error;
    out[R_LOAD_ERROR] = r.load_error;
    out[R_PVIOL] = r.pressure_violation;
    out[R_PEN_ERROR] = r.penetration_error;
    out[R_REQ_TOL] = r.requested_tol;
    out[R_EFF_TOL] = r.effective_tol;
    out[R_P_REF] = r.p_ref;
    out[R_G_REF] = r.g_ref;
    out[R_MATVECS] = double(r.matvec_count);
    out[R_PRECONDS] = double(r.precond_count);
    out[R_IDENT] = r.identification_steps;
    out[R_RETURNED_BEST] = r.returned_best ? 1.0 : 0.0;
    out[R_TIME] = r.time_total;
    const int nh = int(r.error_history.size());
    out[R_HISTORY_LEN] = nh;
    if (history)
        for (int i = 0; i < nh && i < history_cap; ++i) history[i] = r.error_history[i];
    std::snprintf(status_out, 64, "%s", r.status_reason.c_str());
    return 0;
}

// The tangential FFT operator, restated from src/tangential_operator.cpp:
// 18-140 on the reference's own FFT engine (fft_engine.hpp) and Cerruti
// tables: that file itself cannot be compiled here (it includes the H2
// operator, which needs far more of Eigen than the stand-in has).  Checked
// against the dense Cerruti block in tests/test_tangential_oracle.py.
struct RefTangential {
    int Ns, M, nh;
    hmc::CerrutiKernel kernel;
    std::vector<double> Kxx, Kyy, Kxy;  // (nh x M), 1/M^2 folded in
    mutable Eigen::MatrixXd G1, G2;
    mutable Eigen::MatrixXcd C1, C2;
    mutable hmc::fft::SquareR2C<double> f1, f2;

    RefTangential(int Ns_, double L, double E, double nu)
        : Ns(Ns_), M(2 * Ns_), nh(Ns_ + 1), kernel(Ns_, L, E, nu) {
        Eigen::MatrixXd K(M, M);
        Eigen::MatrixXcd Kc(nh, M);
        hmc::fft::SquareR2C<double> plan;
        plan.bind(M, K.data(), Kc.data());
        const double norm = 1.0 / (double(M) * double(M));
        auto harvest = [&](int which, std::vector<double>& out) {
            for (int iy = 0; iy < M; ++iy)
                for (int ix = 0; ix < M; ++ix) {
                    const int dy = iy < Ns ? iy : iy - M, dx = ix < Ns ? ix : ix - M;
                    double v = 0.0;
                    if (iy != Ns && ix != Ns)
                        v = which == 0 ? kernel.xx_offset(dx, dy)
                                       : which == 1 ? kernel.yy_offset(dx, dy)
                                                    : kernel.xy_offset(dx, dy);
                    K(ix, iy) = v;
                }
            plan.fwd();
            out.resize(size_t(nh) * M);
            for (int ky = 0; ky < M; ++ky)
                for (int kx = 0; kx < nh; ++kx) out[size_t(ky) * nh + kx] = norm * Kc(kx, ky).real();
        };
        harvest(0, Kxx);
        harvest(1, Kyy);
        harvest(2, Kxy);
        G1.resize(M, M);
        G2.resize(M, M);
        C1.resize(nh, M);
        C2.resize(nh, M);
        f1.bind(M, G1.data(), C1.data(), Ns);
        f2.bind(M, G2.data(), C2.data(), Ns);
    }
    void apply(const Eigen::VectorXd& q, Eigen::VectorXd& u) const {
        const int N = Ns * Ns;
        if (u.size() != 2 * N) u.resize(2 * N);
        for (int iy = 0; iy < Ns; ++iy)
            for (int ix = 0; ix < M; ++ix) {
                G1(ix, iy) = ix < Ns ? q(iy * Ns + ix) : 0.0;
                G2(ix, iy) = ix < Ns ? q(N + iy * Ns + ix) : 0.0;
            }
        f1.fwd();
        f2.fwd();
        for (int ky = 0; ky < M; ++ky)
            for (int kx = 0; kx < nh; ++kx) {
                const size_t at = size_t(ky) * nh + kx;
                const std::complex<double> a = C1(kx, ky), b = C2(kx, ky);
                C1(kx, ky) = Kxx[at] * a + Kxy[at] * b;
                C2(kx, ky) = Kxy[at] * a + Kyy[at] * b;
            }
        f1.inv();
        f2.inv();
        for (int iy = 0; iy < Ns; ++iy)
            for (int ix = 0; ix < Ns; ++ix) {
                u(iy * Ns + ix) = G1(ix, iy);
                u(N + iy * Ns + ix) = G2(ix, iy);
            }
    }
};

}  // namespace

extern "C" {

const char* aref_last_error(void) { return g_err.c_str(); }

int aref_nscalars(void) { return R_NSCALARS; }

int aref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void aref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// ContactSolver(grid_size, domain_size, E_star, backend) for "fft" (0) and
// "periodic" (1): python/bindings.cpp:119-148.
void* aref_op_create(int backend, int Ns, double L, double E_star) {
    try {
        auto op = std::make_unique<RefOp>();
        op->backend = backend;
        op->Ns = Ns;
        if (backend == 0) {
            op->kernel = std::make_unique<hmc::BoussinesqKernel>(Ns, L, E_star);
            op->fft = std::make_unique<hmc::FFTOperator>(*op->kernel);
            op->fft->build();
        } else if (backend == 1) {
            op->periodic = std::make_unique<hmc::PeriodicFFTOperator>(Ns, L, E_star);
        } else {
            throw std::invalid_argument("backend must be 0 (fft) or 1 (periodic)");
        }
        return op.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void aref_op_destroy(void* h) { delete static_cast<RefOp*>(h); }

// y = S x, FP64 (matvec_into) or FP32 (matvec_single_into)
int aref_op_matvec(void* h, int dtype, const void* x, void* y) {
    try {
        RefOp* op = static_cast<RefOp*>(h);
        const int64_t N = int64_t(op->Ns) * op->Ns;
        if (dtype == 1) {
            hmc::VecT<double> xv(N), yv;
            std::memcpy(xv.data(), x, sizeof(double) * N);
            op->apply<double>(xv, yv);
            std::memcpy(y, yv.data(), sizeof(double) * N);
        } else {
            hmc::VecT<float> xv(N), yv;
            std::memcpy(xv.data(), x, sizeof(float) * N);
            op->apply<float>(xv, yv);
            std::memcpy(y, yv.data(), sizeof(float) * N);
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// The Ns*Ns Love table T[dy*Ns+dx] (fft backend): BoussinesqKernel::entry
int aref_love_table(void* h, double* out) {
    RefOp* op = static_cast<RefOp*>(h);
    if (!op->kernel) {
        g_err = "no Love table on the periodic backend";
        return -1;
    }
    const int Ns = op->Ns;
    for (int dy = 0; dy < Ns; ++dy)
        for (int dx = 0; dx < Ns; ++dx) out[int64_t(dy) * Ns + dx] = op->kernel->entry_offset(dx, dy);
    return 0;
}

// z = M^-1 g on the contact set: precond 1 = StencilPreconditioner(Ns,
// radius).apply_into, 2 = FourierPreconditioner(Ns).apply_into (FP64)
int aref_precond_apply(void* h, int precond, int radius, const double* g, const uint8_t* contact,
                       double* z) {
    try {
        RefOp* op = static_cast<RefOp*>(h);
        const int64_t N = int64_t(op->Ns) * op->Ns;
        hmc::VecT<double> gv(N), zv;
        std::memcpy(gv.data(), g, sizeof(double) * N);
        std::vector<std::uint8_t> c(contact, contact + N);
        if (precond == 1) {
            hmc::StencilPreconditioner sp(op->Ns, radius);
            sp.apply_into(gv, c, zv);
        } else {
            if (!op->fourier) op->fourier = std::make_unique<hmc::FourierPreconditioner>(op->Ns);
            op->fourier->apply_into(gv, c, zv);
        }
        std::memcpy(z, zv.data(), sizeof(double) * N);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// solve_contact_impl<Real> (src/contact_solver.cpp:150-587); dtype 1 =
// double (ContactSolver.solve), 0 = float.  opt[] holds the SolveOptions
// fields in this order (entries past nopt keep the reference defaults):
//   tol, max_iter, use_pr, light, record_history, keep_best, stall_limit,
//   scales.g_ref, scales.p_ref, load_tol
// precond: 0 none, 1 stencil (radius), 2 full-grid Fourier.  Returns 0, or -1
// with the reference's std::invalid_argument message (aref_last_error).
int aref_solve(void* h, int dtype, const double* g0, double p_bar, const double* opt, int nopt,
               int precond, int radius, const double* p_init, double* pressure, double* disp,
               double* gap, double* out, double* history, int history_cap, char* status_reason) {
    try {
        RefOp* op = static_cast<RefOp*>(h);
        hmc::SolveOptions o;
        auto has = [&](int i) { return i < nopt; };
        if (has(0)) o.tol = opt[0];
        if (has(1)) o.max_iter = int(opt[1]);
        if (has(2)) o.use_pr = opt[2] != 0.0;
        if (has(3)) o.light = opt[3] != 0.0;
        if (has(4)) o.record_history = opt[4] != 0.0;
        if (has(5)) o.keep_best = opt[5] != 0.0;
        if (has(6)) o.stall_limit = int(opt[6]);
        if (has(7)) o.scales.g_ref = opt[7];
        if (has(8)) o.scales.p_ref = opt[8];
        if (has(9)) o.load_tol = opt[9];
        if (dtype == 1)
            return solve_t<double>(op, g0, p_bar, o, precond, radius, p_init, pressure, disp,
                                   gap, out, history, history_cap, status_reason);
        return solve_t<float>(op, g0, p_bar, o, precond, radius, p_init, pressure, disp, gap,
                              out, history, history_cap, status_reason);
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// CerrutiKernel(Ns, L, E*, nu) (src/cerruti_kernel.cpp:114-128): the signed
// offset tables xx_offset / xy_offset / yy_offset for offsets dx, dy in
// (-Ns, Ns), written row-major as out[(dy + Ns - 1) * (2 Ns - 1) + dx + Ns - 1]
int aref_cerruti_tables(int Ns, double L, double E_star, double nu, double* xx, double* yy,
                        double* xy) {
    try {
        hmc::CerrutiKernel C(Ns, L, E_star, nu);
        const int W = 2 * Ns - 1;
        for (int dy = -(Ns - 1); dy < Ns; ++dy)
            for (int dx = -(Ns - 1); dx < Ns; ++dx) {
                const int64_t at = int64_t(dy + Ns - 1) * W + dx + Ns - 1;
                xx[at] = C.xx_offset(dx, dy);
                yy[at] = C.yy_offset(dx, dy);
                xy[at] = C.xy_offset(dx, dy);
            }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// The element-integrated Cerruti brackets (src/cerruti_kernel.cpp:64-112)
double aref_cerruti_uxx(double x, double y, double a, double b, double nu) {
    return hmc::cerruti_uxx(x, y, a, b, nu);
}
double aref_cerruti_uxy(double x, double y, double a, double b) {
    return hmc::cerruti_uxy(x, y, a, b);
}

void* aref_tan_create(int Ns, double L, double E_star, double nu) {
    try {
        return new RefTangential(Ns, L, E_star, nu);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}
void aref_tan_destroy(void* h) { delete static_cast<RefTangential*>(h); }
int aref_tan_matvec(void* h, const double* q, double* u) {
    const RefTangential* t = static_cast<RefTangential*>(h);
    const int64_t n2 = 2 * int64_t(t->Ns) * t->Ns;
    hmc::VecT<double> qv(n2), uv;
    std::memcpy(qv.data(), q, sizeof(double) * n2);
    t->apply(qv, uv);
    std::memcpy(u, uv.data(), sizeof(double) * n2);
    return 0;
}

// solve_tangential (src/friction_solve.cpp:375-688) on the tangential FFT
// operator, unpreconditioned: displacement control (force_control = 0,
// target = the rigid shift) or force control (target = the mean traction).
// out[] = status, iterations, converged, error, delta_t x/y, q_mean x/y,
// n_stick, n_slip, n_open, cone_violation, stick_residual, slip_residual,
// proj_residual, force_error, rho, s_ref, w_ref, kkt_tol
int aref_solve_tangential(void* h, const double* s, int force_control, double tx, double ty,
                          double tol, int max_iter, int use_pr, double kkt_tol,
                          const double* q_init, double* q_out, double* out,
                          char* status_reason) {
    try {
        const RefTangential* t = static_cast<RefTangential*>(h);
        const int N = t->Ns * t->Ns;
        Eigen::VectorXd sv(N), qi;
        std::memcpy(sv.data(), s, sizeof(double) * N);
        if (q_init) {
            qi.resize(2 * N);
            std::memcpy(qi.data(), q_init, sizeof(double) * 2 * N);
        }
        hmc::TanMatVecInto C = [t](const Eigen::VectorXd& q, Eigen::VectorXd& u) { t->apply(q, u); };
        hmc::TangentialResult r =
            hmc::solve_tangential(C, sv, force_control != 0, Eigen::Vector2d(tx, ty), tol,
                                  max_iter, use_pr != 0, {}, q_init ? &qi : nullptr, nullptr,
                                  0.0, nullptr, nullptr, kkt_tol);
        std::memcpy(q_out, r.q.data(), sizeof(double) * 2 * N);
        const double v[] = {double(int(r.status)), double(r.iterations), r.converged ? 1.0 : 0.0,
                            r.error, r.delta_t(0), r.delta_t(1), r.q_mean(0), r.q_mean(1),
                            double(r.n_stick), double(r.n_slip), double(r.n_open),
                            r.cone_violation, r.stick_residual, r.slip_residual, r.proj_residual,
                            r.force_error, r.rho, r.s_ref, r.w_ref, r.kkt_tol};
        std::memcpy(out, v, sizeof(v));
        std::snprintf(status_reason, 64, "%s", r.status_reason.c_str());
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

const char* aref_status_string(int s) { return hmc::to_string(static_cast<hmc::SolveStatus>(s)); }

// project_load_simplex<double> (src/contact_solver.cpp:31-60), in place
double aref_project_simplex(double* y, int64_t n, double P_total) {
    hmc::VecT<double> v(n);
    std::memcpy(v.data(), y, sizeof(double) * n);
    const double theta = hmc::project_load_simplex<double>(v, P_total);
    std::memcpy(y, v.data(), sizeof(double) * n);
    return theta;
}

}  // extern "C"
