// Device-resident state of one Polonsky-Keer solve.
//
// The per-iteration control flow of solve_contact_impl (reference
// src/contact_solver.cpp:375-515) runs on the device: every vector pass ends
// with a deterministic last-block reduction whose thread 0 applies the
// scalar logic of that step (certificate, best/stall bookkeeping, beta, tau,
// support change, load rescale) and writes the results here.  Rare branches
// (forced identification step, |C| < 2, no positive curvature) set `halt`;
// every later kernel of the iteration then returns at entry, and the host
// takes over at its next synchronisation point.
#pragma once

#include <cstdint>

namespace asb {

// H_FILL: every p became 0 in an embedded solve; the host sets p = p_bar on
// the caller's block (the fill of the cells outside it would be wrong)
enum Halt : int { H_RUN = 0, H_FINAL = 1, H_STALL = 2, H_IDENT = 3, H_FILL = 4 };

enum Status : int {
    ST_CONVERGED = 0,
    ST_STAGNATED = 1,
    ST_MAX_ITERATIONS = 2,
    ST_NONPOSITIVE_CURVATURE = 3,
    ST_NONFINITE = 4,
    ST_VERIFICATION_FAILED = 5,
    ST_RESOURCE_LIMIT = 6
};

// Solve constants, passed by value to every kernel.
struct PkParams {
    long N;
    int Ns;
    // the caller's grid side: Ns, or (embedded operators) the side of the
    // top-left block of the Ns x Ns field that holds the caller's cells
    int Nl;
    int max_iter;
    int stall_limit;
    int keep_best;
    int record_history;
    int use_pr;
    int precond;  // 0 none, 1 stencil, 2 fft
    double P_total;
    double g_ref;
    double tol;
    double load_tol;
    double p_bar;
    double gshift;  // datum subtracted on the fly (0 in caller mode)
    long hist_stride;  // history entries per instance (batched solves)
};

struct PkState {
    // evaluate() -- contact_solver.cpp:260-303
    double alpha, gmin;  // alpha: one-pass mean (g is centred by Real(alpha)); refined below
    double alpha_ref, gmin_ref;
    double gsum, vmin;
    double pk, G, fw, pen, psum, pv, load, gcs;
    int nc;
    int finite;
    // control
    int halt;
    int it;
    int u_fresh;
    int skip_mv1;  // gate of the first apply of an iteration: halt || u_fresh
    int stall, forced_id;
    int copy_best, have_best;
    int status;
    int fill;  // total <= 0: the pressure is p_bar everywhere (pending, see scale);
               // 2: an embedded solve's fill, done by the host (H_FILL)
    int pk_due;  // k_eval ran; k_evalpk records this iteration's pk
    double best_merit, seen_merit;
    // CG recurrences
    double G_old, delta, beta, gg, bv;  // bv: PR+ / FR ratio before the delta gate
    double zmean;  // preconditioner output contact mean
    double rsum, num, rmean, den, tau, tau_ov;
    double total;
    // the load rescale p <- p P / sum p (contact_solver.cpp:491-497) is
    // applied lazily: the iterate is Real(x * scale) + scale_add of the
    // stored x, every consumer in the loop forms it (bit-identical to the
    // reference's p(i) *= f: scale_add is 0 then), and the host materialises
    // it whenever it takes over (scale 1, scale_add 0 afterwards).  The
    // reference's p = p_bar fill (every p zero after the update) is scale 1,
    // scale_add p_bar.
    double scale, scale_add;
    // identification / helpers: generic reduction results
    double red[8];
    // last-block counters, one per kernel kind (reset by the last block)
    unsigned counter[16];
    long long mv, pc;
};

}  // namespace asb
