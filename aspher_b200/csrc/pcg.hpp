// Internal declarations of the solver translation unit.
#pragma once

#include "../../include/aspher_b200.h"
#include "ops.hpp"
#include "pk_state.hpp"

namespace asb {

// Stencil taps of the l2 disc |d| <= R (R <= 4: at most 49 taps).
struct StencilTaps {
    int n;
    int R;
    int dx[64];
    int dy[64];
    double w[64];
};
StencilTaps make_stencil_taps(int Ns, int R);

// Full-grid |k| preconditioner inside a PK solve: centre g (held as v and
// centred by Real(st->alpha) on the fly) on the contact mask by
// st->gcs / st->nc, transform, multiply by |k|/Ns^2 (FP32 table values,
// fourier_precond.cpp:12-28), gather on contact into z and leave T(contact
// mean of z) in st->zmean (st->pc incremented).  Kernels return at entry
// when gate != nullptr and gate[b * kGateStride] != 0 (instance b of B;
// spec: B spectra, or nullptr for the operator's own when B = 1).
// Defined in operators.cu.
template <typename T>
void fourier_precond_pk(Operator& op, const T* g, const uint8_t* mask, PkState* st, T* z,
                        double* part, cudaStream_t s, const int* gate, int B = 1,
                        void* spec = nullptr);

// polish_stage: the solve refines p_init (the FP64 stage of a mixed or
// nested float_then_double solve); its loop applies may then be
// defect-corrected (see Operator::matvec_defect)
template <typename T>
void solve_impl(Operator& op, const aspher_solve_opts& o, const void* g0, double p_bar,
                const void* p_init, double* pressure, double* disp, double* gap, double* hist,
                int hist_cap, aspher_result& res, cudaStream_t s, bool polish_stage = false);

void solve_mixed(Operator& op, const aspher_solve_opts& o, const double* g0, double p_bar,
                 const double* p_init, double float_tol, int polish, double* pressure,
                 double* disp, double* gap, aspher_result& res, aspher_result* res_float,
                 cudaStream_t s);

void solve_nested(int kind, int Ns, double L, double E, const double* g0, double p_bar,
                  const aspher_nested_opts& np, double* pressure, double* disp, double* gap,
                  double* hist_host, int hist_cap, aspher_result& res, aspher_stage* stages,
                  int stage_cap, int* nstages, cudaStream_t s);
bool stencil_for_level(int engine, bool precond, double prev_occupancy, double occupancy_max);
void clear_operator_cache();

template <typename T>
void solve_batch_impl(Operator& op, const aspher_solve_opts& o, int B, const void* const* g0s,
                      const double* p_bars, const void* const* p_inits, double* const* pressures,
                      aspher_result* res, cudaStream_t s);
void solve_batch_mixed(Operator& op, const aspher_solve_opts& o, int B, const double* const* g0s,
                       const double* p_bars, double float_tol, int polish,
                       double* const* pressures, aspher_result* res, aspher_result* res_float,
                       cudaStream_t s);

void solve_many(int n, const aspher_problem* problems, const aspher_many_opts& o,
                aspher_result* res, aspher_result* res_float, cudaStream_t s);

template <typename T>
void adjoint_impl(Operator& op, const double* p, const double* w, double tol, int max_iter,
                  int precond, int radius, double* grad_g0, double* grad_pbar,
                  aspher_adjoint_info* info, cudaStream_t s);

template <typename T>
void precond_apply_impl(Operator& op, int precond, int radius, const T* g, const uint8_t* mask,
                        T* z, cudaStream_t s);

}  // namespace asb
