/*
 * aspher_b200 -- C ABI of the B200 (sm_100a) FFT-operator contact solve.
 *
 * This is the drop-in boundary for ASPHER's backend="fft" / "periodic"
 * normal-contact path.  Each entry point names the reference interface it
 * replaces (paths relative to the reference project).  Conventions:
 *   - plain pointers and sizes only; every array argument named *_dev is a
 *     device pointer on the current CUDA device, 16-byte aligned;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy stream);
 *   - every function returns ASPHER_OK (0) or a negative error code and
 *     leaves a message readable through aspher_last_error() (thread-local);
 *     no C++ exception crosses this boundary;
 *   - numerical outcomes of a solve are NOT errors: they are reported in
 *     aspher_result.status (the reference's SolveStatus taxonomy);
 *   - handles are not thread-safe: one operator per host thread / stream,
 *     as for the reference's operators (include/fft_operator.hpp:42-44).
 */
#ifndef ASPHER_B200_H
#define ASPHER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ASPHER_B200_ABI_VERSION 3

/* ---- error codes ------------------------------------------------------- */
#define ASPHER_OK 0
#define ASPHER_EINVAL (-1)   /* invalid argument (reference: std::invalid_argument) */
#define ASPHER_ECUDA (-2)    /* CUDA runtime / launch failure */
#define ASPHER_EBUILD (-3)   /* operator build check failed (fft_operator.cpp:57-60) */
#define ASPHER_ETIMEOUT (-4) /* a bounded device wait gave up */

/* ---- enums -------------------------------------------------------------- */
enum aspher_backend { ASPHER_BACKEND_FFT = 0, ASPHER_BACKEND_PERIODIC = 1 };
enum aspher_dtype { ASPHER_F32 = 0, ASPHER_F64 = 1 };
/* precond: reference python/bindings.cpp:193-214 ("fourier" is the stencil) */
enum aspher_precond {
    ASPHER_PRECOND_NONE = 0,
    ASPHER_PRECOND_STENCIL = 1, /* StencilPreconditioner (include/stencil_precond.hpp:50) */
    ASPHER_PRECOND_FFT = 2      /* FourierPreconditioner (include/fourier_precond.hpp:33) */
};
/* SolveStatus, reference include/contact_solver.hpp:13-21 */
enum aspher_status {
    ASPHER_CONVERGED = 0,
    ASPHER_STAGNATED = 1,
    ASPHER_MAX_ITERATIONS = 2,
    ASPHER_NONPOSITIVE_CURVATURE = 3,
    ASPHER_NONFINITE = 4,
    ASPHER_VERIFICATION_FAILED = 5,
    ASPHER_RESOURCE_LIMIT = 6
};
/* SolveScales::DatumMode, reference include/contact_solver.hpp:138-144 */
enum aspher_datum_mode { ASPHER_DATUM_AUTOMATIC = 0, ASPHER_DATUM_SOLVER = 1, ASPHER_DATUM_CALLER = 2 };

int aspher_abi_version(void);
const char* aspher_last_error(void);
/* Number of CUDA kernel launches this library has issued in this process
 * (a CUDA-graph launch counts once); for launch accounting in benchmarks.
 * No reference counterpart. */
int64_t aspher_launch_count(void);
/* to_string(SolveStatus), reference src/contact_solver.cpp:12-23 */
const char* aspher_status_string(int status);

/* ---- operators ---------------------------------------------------------- */
typedef struct aspher_op aspher_op;

/* Replaces BoussinesqKernel(Ns, L, E*) + FFTOperator(kernel).build()
 * (include/boussinesq_kernel.hpp:26, include/fft_operator.hpp:47-52) for
 * backend FFT and PeriodicFFTOperator(Ns, L, E*)
 * (include/periodic_fft_operator.hpp:26) for backend PERIODIC.  The Love
 * table and its FP64 spectrum are built on the device; synchronous.
 * grid_size in [2, 16384]; at 16384 only FP32 applies and solves exist
 * (FP64 ones return ASPHER_EINVAL).  A grid_size that is not a power of two
 * >= 16 runs embedded: its cells are the top-left block of the next
 * power-of-two grid's free-space pipeline, whose kernel table is the Love
 * table at cell size domain_size / grid_size (FFT) or the real-space kernel
 * of the periodic symbol on the grid_size torus (PERIODIC); every entry
 * point still takes grid_size^2 fields.  Creation flags need a power of
 * two >= 16 and the FFT preconditioner an even grid_size (ASPHER_EINVAL
 * otherwise). */
int aspher_op_create(int backend, int grid_size, double domain_size, double E_star,
                     aspher_op** out);
/* The same with creation flags (the survey's aspher_op_create(kind, Ns, L,
 * Estar, flags, ...)): ASPHER_OPF_SPLIT_COLUMNS computes the free-space
 * column pass as two half-length transforms and ASPHER_OPF_SPLIT_KH builds
 * the FP64 kernel spectrum from even / odd row samples at every grid_size
 * >= 256 -- the forms that FP64 at 8192 and 16384 need, selectable at
 * smaller sizes so that they can be checked against the one-CTA forms.
 * Results equal aspher_op_create's to rounding; flags = 0 is
 * aspher_op_create.  Unknown flag bits return ASPHER_EINVAL. */
#define ASPHER_OPF_SPLIT_COLUMNS 1
#define ASPHER_OPF_SPLIT_KH 2
int aspher_op_create_ex(int backend, int grid_size, double domain_size, double E_star,
                        int flags, aspher_op** out);
int aspher_op_destroy(aspher_op* op);

/* y = S x over Ns*Ns values of `dtype` (F64: FFTOperator::matvec_into,
 * include/fft_operator.hpp:57; F32: matvec_single_into, :62; periodic:
 * include/periodic_fft_operator.hpp:32,35).  x and y may alias.  Async on
 * `stream`. */
int aspher_op_matvec(aspher_op* op, int dtype, const void* x_dev, void* y_dev, void* stream);

/* FFTInfo, reference include/fft_operator.hpp:13-25 */
typedef struct {
    int backend;
    int grid_size;
    int padded_side;
    int64_t n;
    int64_t bytes_spectrum;
    int64_t bytes_scratch;
    int64_t bytes_total;
    double max_im_ratio; /* build-time max|Im|/max|Re| of the kernel spectrum */
} aspher_op_info;
int aspher_op_get_info(const aspher_op* op, aspher_op_info* info);

/* Launch variants of the three FFT passes (row variant: registers per thread
 * and rows per CTA of the two row passes; column variant: registers per
 * thread, columns per CTA and CTAs per SM of the column pass).  Variants
 * 0..3; the half-spectrum layout follows the column variant's tile width.
 * No reference counterpart (the reference's FFT engine has no launch shape). */
int aspher_op_set_variants(aspher_op* op, int dtype, int row_variant, int col_variant);
int aspher_op_get_variants(const aspher_op* op, int dtype, int* row_variant, int* col_variant,
                           int* col_tile);
/* Autotuner: times every variant pair (reps applies each, L2 flushed between
 * applies) on this operator, keeps the fastest and records it for every
 * operator of the same backend / precision / grid_size created later in the
 * process.  Synchronous; allocates temporary device buffers.  No reference
 * counterpart. */
int aspher_op_autotune(aspher_op* op, int dtype, int reps, int* row_variant, int* col_variant,
                       double* best_ms);

/* Copies the Ns*Ns FP64 Love table T[dy*Ns+dx] (BoussinesqKernel::table_,
 * src/boussinesq_kernel.cpp:97-106) to host memory.  FFT backend only. */
int aspher_op_love_table(const aspher_op* op, double* host_out);

/* z = M^-1 g on the contact set (contact_dev: Ns*Ns bytes, nonzero = in
 * contact), centred and mean-zeroed on it: StencilPreconditioner::apply_into
 * (include/stencil_precond.hpp:64, radius >= 1) or
 * FourierPreconditioner::apply_into (include/fourier_precond.hpp:46).
 * Synchronous. */
int aspher_precond_apply(aspher_op* op, int precond, int radius, int dtype, const void* g_dev,
                         const uint8_t* contact_dev, void* z_dev, void* stream);

/* Stencil taps (StencilPreconditioner::tap_dx/tap_dy/tap_w,
 * include/stencil_precond.hpp:57-60) for grid_size and radius; writes at
 * most `cap` taps and returns their count in *ntaps. */
int aspher_stencil_taps(int grid_size, int radius, int* dx, int* dy, double* w, int cap,
                        int* ntaps);

/* ---- solve -------------------------------------------------------------- */
/* SolveOptions + SolveScales, reference include/contact_solver.hpp:134-191 */
typedef struct {
    double tol;
    double requested_tol;   /* 0 -> tol */
    int max_iter;
    int use_pr;             /* Polak-Ribiere+ (1) or Fletcher-Reeves (0) */
    int light;              /* skip displacement / gap outputs */
    int record_history;
    int keep_best;
    double load_tol;        /* 0 -> 1e-12 (F64) / 5e-7 (F32) */
    int stall_limit;        /* <= 0 -> 200 */
    int allow_tolerance_relaxation;
    int precond;            /* enum aspher_precond */
    int precond_radius;     /* stencil radius (2 -> 13 taps) */
    double p_ref;           /* <= 0 -> p_bar */
    double g_ref;           /* <= 0 -> range(g0) */
    int datum_mode;         /* enum aspher_datum_mode */
    double datum;
    int dtype;              /* working precision Real: ASPHER_F32 / ASPHER_F64 */
    int loop_mode;          /* 0: the iterations in a CUDA-graph while loop (default);
                               1: the same kernels launched one by one (for
                               per-kernel profilers, which cannot see inside
                               graphs with conditional nodes) */
} aspher_solve_opts;

/* Fills the reference defaults (SolveOptions{} and solve_contact(...)'s
 * arguments: tol 1e-8, max_iter 5000, use_pr, keep_best, F64). */
void aspher_solve_opts_default(aspher_solve_opts* o);

/* ContactResult, reference include/contact_solver.hpp:25-123 */
typedef struct {
    int status;              /* enum aspher_status */
    char status_reason[32];  /* "", "stall", "precision_limit", "final_check" */
    int iterations;
    int converged;
    double contact_fraction; /* Python `contact_area` */
    double mean_pressure;
    double approach;
    double objective;
    double error;            /* == pk_error */
    double pk_error;
    double fw_gap;
    double fw_error;
    double load_error;
    double pressure_violation;
    double penetration_error;
    double requested_tol;
    double effective_tol;
    double p_ref;
    double g_ref;
    int64_t matvec_count;
    int64_t precond_count;
    int identification_steps;
    int returned_best;
    int history_len;         /* entries written to history_out */
    double time_total;       /* seconds, host wall clock around the solve */
    int64_t mem_cg_state;    /* Memory, contact_solver.hpp:75-81 */
    int64_t mem_best_iterate;
    int64_t mem_contact_mask;
    int64_t mem_output_arrays;
    int64_t mem_peak;
    double time_build;       /* nested driver: operator construction, seconds */
    double time_coarse;      /* nested driver: coarse-level solves, seconds */
    int active_rounds;       /* nested active set: restricted rounds of the finest level */
    int active_fallback;     /* nested active set: the full-grid fallback solve ran */
    double time_candidate;   /* nested active set: candidate-set work, seconds */
} aspher_result;

/* solve_contact_impl<Real> (include/contact_solver.hpp:244-249; reference
 * src/contact_solver.cpp:150-587) with the operator of `op`, the
 * preconditioner selected in opts, and Real = opts->dtype:
 *   g0_dev        : Ns*Ns values of opts->dtype (read only)
 *   p_init_dev    : NULL or Ns*Ns values of opts->dtype (warm start; read only)
 *   pressure_dev  : Ns*Ns FP64 output (required)
 *   displacement_dev, gap_dev : Ns*Ns FP64 outputs or NULL (skipped when light)
 *   history_host  : NULL or host array of history_cap doubles (per-iteration
 *                   pk error when opts->record_history)
 * Invalid input returns ASPHER_EINVAL before any operator apply
 * (contact_solver.cpp:159-168).  Synchronous with respect to the host. */
int aspher_solve(aspher_op* op, const aspher_solve_opts* opts, const void* g0_dev, double p_bar,
                 const void* p_init_dev, double* pressure_dev, double* displacement_dev,
                 double* gap_dev, double* history_host, int history_cap, aspher_result* res,
                 void* stream);

/* Mixed-precision solve: FP32 operator/CG with FP64-accumulated reductions
 * to float_tol, then (polish != 0) an FP64 PK solve warm-started from it that
 * certifies opts->tol on the FP64 operator.  This is the reference's
 * float_then_double staging (src/nested_solve.cpp:871-974,
 * include/nested_solve.hpp:53-68) applied to one grid.  g0_dev and
 * p_init_dev are FP64 (opts->dtype is ignored); the gap is centred by its
 * datum and cast to FP32 on the device.  *res holds the final stage with
 * iterations / matvec / precond counts summed over both stages;
 * res_float (nullable) receives the FP32 stage alone.  Synchronous. */
int aspher_solve_mixed(aspher_op* op, const aspher_solve_opts* opts, const double* g0_dev,
                       double p_bar, const double* p_init_dev, double float_tol, int polish,
                       double* pressure_dev, double* displacement_dev, double* gap_dev,
                       aspher_result* res, aspher_result* res_float, void* stream);

/* Batched solves: `batch` independent problems on the same operator and
 * options (per-problem gap, p_bar, warm start and pressure output) solved
 * together, every kernel of the loop launched once for the whole batch with
 * one CUDA-graph loop and per-problem convergence masks.  Each problem's
 * result is the result aspher_solve / aspher_solve_mixed would return for it
 * alone, up to reduction order.  Arrays of pointers live in host memory and
 * point to device fields; outputs are pressures only (light).  No reference
 * counterpart (the reference solves one problem per call).  Synchronous. */
int aspher_solve_batch(aspher_op* op, const aspher_solve_opts* opts, int batch,
                       const void* const* g0_devs, const double* p_bars,
                       const void* const* p_init_devs, double* const* pressure_devs,
                       aspher_result* res, void* stream);
int aspher_solve_batch_mixed(aspher_op* op, const aspher_solve_opts* opts, int batch,
                             const double* const* g0_devs, const double* p_bars, double float_tol,
                             int polish, double* const* pressure_devs, aspher_result* res,
                             aspher_result* res_float, void* stream);

/* ---- many problems of uneven size and backend ------------------------------ */
/* One problem of aspher_solve_many: the survey's aspher_problem of the
 * batch entry aspher_solve_batch(n, const aspher_problem*, aspher_result*,
 * stream), whose one-operator form keeps that name above.  Buffers are the
 * caller's: g0_dev (Ns*Ns FP64 gap) and pressure_dev (Ns*Ns FP64 output) on
 * the current device, 16-byte aligned. */
typedef struct {
    int backend;           /* ASPHER_BACKEND_FFT / ASPHER_BACKEND_PERIODIC */
    int grid_size;         /* in [2, 16384] (see aspher_op_create) */
    double domain_size;    /* <= 0: 1 */
    double E_star;         /* <= 0: 1 */
    const double* g0_dev;
    double p_bar;
    double* pressure_dev;
} aspher_problem;

enum aspher_many_precision {
    ASPHER_MANY_DOUBLE = 0,           /* FP64 solves (the reference's) */
    ASPHER_MANY_FLOAT = 1,            /* FP32 operator / CG, FP64 reductions */
    ASPHER_MANY_FLOAT_THEN_DOUBLE = 2 /* FP32 to float_tol, FP64 polish to polish_tol */
};

/* Options shared by every problem of a call. */
typedef struct {
    int precision;        /* enum aspher_many_precision */
    double tol;           /* requested certificate */
    double float_tol;     /* FP32 stage target (<= 0: tol) */
    double polish_tol;    /* FP64 polish certificate, in (0, tol] (<= 0: tol) */
    int max_iter;         /* per stage (<= 0: 5000) */
    int precond;          /* enum aspher_precond */
    int precond_radius;   /* stencil radius (<= 0: 2) */
    int concurrent;       /* groups run concurrently on their own streams */
} aspher_many_opts;

/* Fills the defaults: float_then_double, tol 1e-6, float_tol = polish_tol
 * = tol, max_iter 5000, stencil preconditioner of radius 2, concurrent. */
void aspher_many_opts_default(aspher_many_opts* o);

/* n independent solves of any (backend, grid_size, domain_size, E_star) in
 * one call.  No reference counterpart (the reference solves one problem per
 * call).  The library groups the problems by operator (operators from the
 * per-process cache of aspher_solve_nested), solves each group as one
 * batched solve (aspher_solve_batch / aspher_solve_batch_mixed: one CUDA-
 * graph loop, per-problem convergence masks), and runs the groups
 * concurrently, longest first, each on its own stream of a per-device pool
 * driven by its own host thread.  res[i] (and res_float[i], nullable: the
 * FP32 stage alone) is problem i's result, the result aspher_solve_batch
 * would give it (light: pressure only).  The groups wait for the caller's
 * earlier work on `stream` and later work on `stream` waits for them.
 * Invalid problems return ASPHER_EINVAL (the message names the problem)
 * before any device work.  Synchronous. */
int aspher_solve_many(int n, const aspher_problem* problems, const aspher_many_opts* opts,
                      aspher_result* res, aspher_result* res_float, void* stream);

/* ---- adjoint of a converged solve ------------------------------------------ */
/* No reference counterpart (the reference has no derivative of the solve).
 * With C = {p > 0} the contact set of a converged solve of (op, g0, p_bar)
 * and w = dL/dp, solves  S_CC lam - mu 1 = w_C,  sum_C lam = 0  by CG on the
 * contact set (the same operator; optional stencil preconditioner) and
 * returns dL/dg0 = -lam (0 off C) and dL/dp_bar = -mu N.  p_dev, w_dev and
 * grad_g0_dev are FP64 device fields of N entries; dtype (ASPHER_F32 /
 * ASPHER_F64) is the working precision of the CG (reductions always FP64).
 * tol: relative residual |r| <= tol |r0|.  Synchronous. */
typedef struct {
    int status;        /* aspher_status: CONVERGED, MAX_ITERATIONS, ... */
    int iterations;
    int contact_count; /* |C| */
    int reserved;
    double residual;   /* final |r| / |r0| */
    double mu;         /* the load multiplier */
    double time;       /* seconds */
} aspher_adjoint_info;

int aspher_adjoint(aspher_op* op, int dtype, const double* p_dev, const double* w_dev,
                   double tol, int max_iter, int precond, int precond_radius,
                   double* grad_g0_dev, double* grad_pbar, aspher_adjoint_info* info,
                   void* stream);

/* Allocation-free doubly periodic apply, y = S x (no counterpart in the
 * reference).  For callers that cannot allocate device memory: real-time
 * loops that must not block in the allocator, and applications whose own
 * allocator owns all GPU memory.  Same
 * result as aspher_op_matvec on a PERIODIC operator of the same grid_size,
 * domain_size and E_star, without an operator handle: the scratch is a
 * static 8.65 MB device array and grid_size must be a power of two in
 * [16, 1024]; larger sizes return ASPHER_EINVAL.  With CUDA's lazy module
 * loading (the default since CUDA 12.2) the 8.65 MB are allocated by the
 * driver in the first call on each device and held until the process exits:
 * make that first call before a host allocator reserves the GPU's memory, or
 * set CUDA_MODULE_LOADING=EAGER.  The first call on a device also sets it up
 * (make it before any stream capture).  `stream` must belong to the current
 * device.  All calls share the scratch: calls that overlap on the GPU race.
 * x_dev and y_dev must not alias.  Async on `stream`. */
int aspher_periodic_matvec_noalloc(int grid_size, double domain_size, double E_star, int dtype,
                                   const void* x_dev, void* y_dev, void* stream);

/* ---- tangential (Cerruti) operator ------------------------------------------ */
typedef struct aspher_tan_op aspher_tan_op;

/* Replaces CerrutiKernel(Ns, L, E*, nu) + TangentialFFTOperator(kernel).build()
 * (include/cerruti_kernel.hpp:35-61, include/tangential_operator.hpp:32-57;
 * src/cerruti_kernel.cpp:114-128, src/tangential_operator.cpp:18-77): the
 * Cerruti tables and their three real spectra built on the device in FP64,
 * with the reference's realness check (ASPHER_EBUILD when it fails).
 * grid_size in [2, 2048] (one that is not a power of two >= 16 runs
 * embedded in the next power of two, as for aspher_op_create; every entry
 * point still takes 2 grid_size^2 fields); nu in [0, 1).  Synchronous. */
int aspher_tan_create(int grid_size, double domain_size, double E_star, double nu,
                      aspher_tan_op** out);
int aspher_tan_destroy(aspher_tan_op* op);

/* u = C q (TangentialFFTOperator::matvec_into,
 * include/tangential_operator.hpp:41-42): q = [q_x; q_y] and u = [u_x; u_y],
 * 2 Ns*Ns values of `dtype` each (F64, or F32 with the spectra in FP32),
 * stacked as the reference's dense block [[XX, XY], [XY, YY]] expects.  q
 * and u may alias.  Async on `stream`. */
int aspher_tan_matvec(aspher_tan_op* op, int dtype, const void* q_dev, void* u_dev,
                      void* stream);

/* Build-time max |discarded part| / max |kept part| over the three spectra
 * (the reference's realness check, tangential_operator.cpp:52-59). */
int aspher_tan_max_im_ratio(const aspher_tan_op* op, double* out);

/* CerrutiKernel::xx_offset / yy_offset / xy_offset (cerruti_kernel.hpp:44-58)
 * for dx, dy in (-Ns, Ns), copied to host arrays of (2 Ns - 1)^2 doubles,
 * row-major [dy + Ns - 1][dx + Ns - 1]. */
int aspher_tan_tables(const aspher_tan_op* op, double* xx_host, double* yy_host,
                      double* xy_host);

/* TangentialResult (include/friction_solve.hpp:14-44) */
typedef struct {
    int status;              /* enum aspher_status */
    char status_reason[48];  /* "", "stall", "local_kkt", "outer force iteration",
                                "local_kkt_near_tolerance" */
    int iterations;
    int converged;
    double error;            /* the iteration's KKT stationarity metric */
    double delta_t[2];       /* rigid shift (the force-control multiplier) */
    double q_mean[2];        /* grid-mean traction */
    int n_stick, n_slip, n_open;
    double cone_violation;   /* max(0, |q_i| - s_i) / s_ref */
    double stick_residual;   /* max |w_i| over stick / w_ref */
    double slip_residual;    /* max(|w_perp|, (-w.qhat)+) over slip / w_ref */
    double proj_residual;    /* ||q - proj[q - rho g]||_inf / s_ref */
    double force_error;      /* |q_mean - q_bar| / s_ref (force control) */
    double rho, s_ref, w_ref, kkt_tol;
} aspher_tan_result;

/* solve_tangential (include/friction_solve.hpp:62-76, src/friction_solve.cpp:
 * 375-688) on the operator of `op`, unpreconditioned, FP64:
 *   displacement control (force_control = 0): min 1/2 q'Cq - sum q_i.delta,
 *     |q_i| <= s_i, with delta = (target_x, target_y);
 *   force control: the same with mean(q) = (target_x, target_y), by the
 *     reference's outer Newton / Broyden iteration on the rigid shift.
 * s_dev: Ns*Ns thresholds (>= 0; open points s = 0); q_init_dev (nullable,
 * 2 Ns*Ns) a warm start; u_hist_dev (nullable, 2 Ns*Ns) the history term
 * added to u; q_dev: 2 Ns*Ns output.  kkt_tol <= 0: 1e-2 (the reference's
 * default local-KKT acceptance).  Synchronous. */
int aspher_solve_tangential(aspher_tan_op* op, const double* s_dev, int force_control,
                            double target_x, double target_y, double tol, int max_iter,
                            int use_pr, double kkt_tol, const double* q_init_dev,
                            const double* u_hist_dev, double* q_dev, aspher_tan_result* res,
                            void* stream);

/* ---- nested-grid driver ---------------------------------------------------- */
/* NestedParams, reference include/nested_solve.hpp:11-119 (the fields that
 * apply to the fft / periodic backends; the H2 q / leaf_side are kept for
 * signature compatibility, leaf_side still clamps the stencil radius). */
typedef struct {
    double tol;
    int max_iter;
    int use_pr;
    int coarsest;
    int q;
    int leaf_side;
    int precond;               /* bool */
    int precond_engine;        /* 0 auto, 1 stencil, 2 fft */
    int precond_radius;
    double precond_occupancy_max;
    double coarse_tol;
    int single_precision;      /* legacy spelling of precision = float */
    int precision;             /* 0 defer to single_precision, 1 double, 2 float, 3 float_then_double */
    double float_floor;
    int allow_tolerance_relaxation;
    int light_result;
    int record_error_history;
    int active_set;            /* restricted (active-set) levels; the reference
                                  has them for h2 only (nested_solve.cpp:608-617) */
    double active_delta;       /* candidates: coarse gap < delta * range(level gap) */
    int active_halo;           /* Chebyshev dilation radius of candidates / violations */
    int active_max_rounds;     /* restricted rounds before the full-grid fallback */
    int active_all_levels;     /* restrict every level with a coarser one, not only the finest */
    double active_occupancy_max; /* restrict only below this contact fraction */
} aspher_nested_opts;

/* ContactResult::Stage, reference include/contact_solver.hpp:100-113 */
typedef struct {
    char name[32];             /* "coarse:128", "finest:2048", "polish:2048" */
    char precision[8];         /* "float" | "double" */
    int q;
    double requested_tol;
    double effective_tol;
    int iterations;
    int64_t matvec_count;
    double seconds;
    int status;
    double fw_error;
    double penetration_error;
    int precond_dropped;
} aspher_stage;

/* Fills the reference defaults (python/bindings.cpp:836-853). */
void aspher_nested_opts_default(aspher_nested_opts* o);

/* solve_contact_nested for backend FFT / PERIODIC (include/nested_solve.hpp:146-151,
 * reference src/nested_solve.cpp:518-990).  g0_dev: Ns*Ns FP64 gap on the
 * device (read only); outputs as for aspher_solve.  Operators of every
 * level come from a per-process cache keyed by (backend, Ns, L, E*, device).
 * stages (nullable) receives up to stage_cap entries, *nstages their count.
 * Synchronous. */
int aspher_solve_nested(int backend, int grid_size, double domain_size, double E_star,
                        const double* g0_dev, double p_bar, const aspher_nested_opts* opts,
                        double* pressure_dev, double* displacement_dev, double* gap_dev,
                        double* history_host, int history_cap, aspher_result* res,
                        aspher_stage* stages, int stage_cap, int* nstages, void* stream);

/* stencil_for_level (include/nested_solve.hpp:132-133): which preconditioner
 * engine a level uses; engine 0 auto, 1 stencil, 2 fft.  Returns 0 / 1. */
int aspher_stencil_for_level(int engine, int precond, double prev_occupancy,
                             double occupancy_max);

/* Drops the cached per-level operators of aspher_solve_nested. */
int aspher_operator_cache_clear(void);

#ifdef __cplusplus
}
#endif

#endif /* ASPHER_B200_H */
