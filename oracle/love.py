"""Love (1929) cell integral and the Boussinesq influence table (oracle).

Test infrastructure only (see ``oracle/__init__.py``).  Restates
``src/boussinesq_kernel.cpp:44-106`` of the reference, vectorised over numpy
arrays with the same branch structure and the same order of the four corner
terms, so the values agree with the reference's scalar code to a few ulp.
"""

import numpy as np

# Multipole switch radius in units of max(a, b): boussinesq_kernel.cpp:44.
LOVE_FAR_SWITCH = 1500.0
_HUGE_ARG = 1e150


def asinh_diff(u, v, du):
    """asinh(u) - asinh(v) without cancellation, du = u - v known exactly.

    boussinesq_kernel.cpp:60-69: asinh(u sqrt(1+v^2) - v sqrt(1+u^2)), with the
    inner difference taken through its conjugate when u and v share a sign.
    """
    u, v, du = np.broadcast_arrays(np.asarray(u, dtype=np.float64),
                                   np.asarray(v, dtype=np.float64),
                                   np.asarray(du, dtype=np.float64))
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        huge = (np.abs(u) > _HUGE_ARG) | (np.abs(v) > _HUGE_ARG)
        su = np.sqrt(1.0 + u * u)
        sv = np.sqrt(1.0 + v * v)
        den = u * sv + v * su
        conj = (u * v > 0.0) & (den != 0.0)
        w = np.where(conj, du * (u + v) / np.where(den != 0.0, den, 1.0),
                     u * sv - v * su)
        out = np.where(huge, np.arcsinh(u) - np.arcsinh(v), np.arcsinh(w))
    return out


def _term(t, s1, s2, ds):
    """t * [asinh(s1/|t|) - asinh(s2/|t|)] with the removable t -> 0 limit."""
    c = np.abs(t)
    safe = np.where(t == 0.0, 1.0, c)
    val = t * asinh_diff(s1 / safe, s2 / safe, ds / safe)
    return np.where(t == 0.0, 0.0, val)


def love_uz(x, y, a, b):
    """Integral of 1/|r - r'| over [-a,a]x[-b,b] seen from (x, y).

    boussinesq_kernel.cpp:71-95: parity folding, the asinh rearrangement and
    the two-term multipole expansion past LOVE_FAR_SWITCH * max(a, b).
    """
    x = np.abs(np.asarray(x, dtype=np.float64))
    y = np.abs(np.asarray(y, dtype=np.float64))
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    x, y, a, b = np.broadcast_arrays(x, y, a, b)
    m = np.where(a > b, a, b)
    r2 = x * x + y * y
    far = r2 > (LOVE_FAR_SWITCH * m) * (LOVE_FAR_SWITCH * m)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.sqrt(r2)
        A = 4.0 * a * b
        quad = (a * a * (3.0 * x * x - r2) + b * b * (3.0 * y * y - r2)) / (
            6.0 * r2 * r2)
        far_val = A * (1.0 + quad) / r
    xp, xm, yp, ym = x + a, x - a, y + b, y - b
    da, db = 2.0 * a, 2.0 * b
    near_val = (((_term(xp, yp, ym, db) + _term(yp, xp, xm, da))
                 + _term(xm, ym, yp, -db)) + _term(ym, xm, xp, -da))
    out = np.where(far, far_val, near_val)
    return out if out.ndim else float(out)


def boussinesq_table(Ns, L, E_star):
    """T[dy, dx] = love_uz(dx h, dy h, h/2, h/2) / (pi E*), h = L / Ns.

    boussinesq_kernel.cpp:97-106 (table stored row-major, index dy*Ns + dx).
    """
    h = L / Ns
    a = 0.5 * h
    scale = 1.0 / (np.pi * E_star)
    d = np.arange(Ns, dtype=np.float64)
    xx = (d * h)[None, :]
    yy = (d * h)[:, None]
    return scale * love_uz(xx, yy, a, a)


def assemble_dense(Ns, L, E_star):
    """Dense S_ij = T(|ix-jx|, |iy-jy|): boussinesq_kernel.cpp:108-115."""
    T = boussinesq_table(Ns, L, E_star)
    idx = np.arange(Ns * Ns)
    ix, iy = idx % Ns, idx // Ns
    return T[np.abs(iy[:, None] - iy[None, :]), np.abs(ix[:, None] - ix[None, :])]
