"""Adjoint of the converged contact solve -- TEST INFRASTRUCTURE ONLY.

The reference has no derivative of its solve, so there is no reference code
to restate here; this module states the mathematics the CUDA adjoint
(``aspher_adjoint``) implements, by a dense direct solve instead of CG, so
the two can be compared, and it is itself pinned against central finite
differences of the oracle's FP64 solve (``tests/test_adjoint.py``).
Parity with the reference is not applicable (no counterpart).

At a converged solve of  min 1/2 p^T S p + p^T g0,  p >= 0,  sum p = P
(``src/contact_solver.cpp:150-587``) with contact set C = {p > 0} and strict
complementarity, the KKT conditions restricted to C,

    S_CC p_C - alpha 1 = -g0_C,      1^T p_C = P,

are linear in (g0, P).  For a loss L(p) with w = dL/dp the adjoint pair
solves the symmetric system

    [ S_CC  -1 ] [lam]   [w_C]
    [ -1^T   0 ] [mu ] = [ 0 ]

and dL/dg0_C = -lam, dL/dg0 = 0 off C, dL/dP = -mu (P = p_bar N, so
dL/dp_bar = -mu N).
"""

import numpy as np


def operator_matrix(matvec, N):
    """Dense symmetric S from N applies (small grids only)."""
    S = np.empty((N, N))
    e = np.zeros(N)
    for j in range(N):
        e[j] = 1.0
        S[:, j] = matvec(e)
        e[j] = 0.0
    return 0.5 * (S + S.T)


def adjoint_dense(S, p, w):
    """(dL/dg0, dL/dP) for the converged pressure p and w = dL/dp."""
    p = np.asarray(p, np.float64).reshape(-1)
    w = np.asarray(w, np.float64).reshape(-1)
    C = np.flatnonzero(p > 0.0)
    n = C.size
    A = np.zeros((n + 1, n + 1))
    A[:n, :n] = S[np.ix_(C, C)]
    A[:n, n] = -1.0
    A[n, :n] = -1.0
    rhs = np.zeros(n + 1)
    rhs[:n] = w[C]
    sol = np.linalg.solve(A, rhs)
    grad = np.zeros_like(p)
    grad[C] = -sol[:n]
    return grad, -sol[n]
