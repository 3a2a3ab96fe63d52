// Element-integrated surface kernels on the device (FP64): the Love cell
// integral of the normal (Boussinesq) operator and the Cerruti brackets of
// the tangential operator.
//
// Love (1929): the integral of 1/|r - r'| over the cell [-a,a] x [-b,b]
// seen from (x, y) (reference: src/boussinesq_kernel.cpp:44-95): parity
// folding, the stable asinh differences, the two-term multipole expansion
// past 1500 max(a, b).  Cerruti (reference: src/cerruti_kernel.cpp:1-112):
// ylog = the integral of (x - xi)^2 / rho^3 in the same stable asinh form
// with its own multipole branch past 1500 max(a, b), the u_xx bracket
// (1 - nu) Love + nu ylog, and the mixed bracket, the integral of
// (x - xi)(y - eta) / rho^3, in its rationalised form (a product of positive
// factors, odd in x and y).  The branch structure and switch radii are the
// reference's: the table values are defined by them.  CUDA's asinh / sqrt /
// hypot are called.
#pragma once

#include <cuda_runtime.h>

namespace asb {

__device__ inline double asinh_diff_dev(double u, double v, double du) {
    if (fabs(u) > 1e150 || fabs(v) > 1e150) return asinh(u) - asinh(v);
    const double su = sqrt(1.0 + u * u), sv = sqrt(1.0 + v * v);
    const double den = u * sv + v * su;
    const double w = (u * v > 0.0 && den != 0.0) ? du * (u + v) / den : u * sv - v * su;
    return asinh(w);
}

__device__ __forceinline__ double love_term(double t, double s1, double s2, double ds) {
    if (t == 0.0) return 0.0;
    const double c = fabs(t);
    return t * asinh_diff_dev(s1 / c, s2 / c, ds / c);
}

__device__ inline double love_uz_dev(double x, double y, double a, double b) {
    x = fabs(x);
    y = fabs(y);
    const double m = a > b ? a : b;
    const double r2 = x * x + y * y;
    const double sw = 1500.0 * m;
    if (r2 > sw * sw) {
        const double r = sqrt(r2);
        const double A = 4.0 * a * b;
        const double quad = (a * a * (3.0 * x * x - r2) + b * b * (3.0 * y * y - r2)) /
                            (6.0 * r2 * r2);
        return A * (1.0 + quad) / r;
    }
    const double xp = x + a, xm = x - a, yp = y + b, ym = y - b;
    const double da = 2.0 * a, db = 2.0 * b;
    return love_term(xp, yp, ym, db) + love_term(yp, xp, xm, da) +
           love_term(xm, ym, yp, -db) + love_term(ym, xm, xp, -da);
}


// ylog: the integral of (x - xi)^2 / rho^3 over the cell (x, y >= 0)
__device__ inline double cerruti_ylog_dev(double x, double y, double a, double b) {
    const double mmax = a > b ? a : b;
    const double r2 = x * x + y * y;
    const double sw = 1500.0 * mmax;
    if (r2 > sw * sw) {
        const double r = sqrt(r2);
        const double r3 = r2 * r, r5 = r3 * r2, r7 = r5 * r2;
        const double A = 4.0 * a * b;
        const double x2 = x * x, y2 = y * y;
        return A * (x2 / r3 + (a * a / 6.0) * (2.0 / r3 - 15.0 * x2 / r5 + 15.0 * x2 * x2 / r7) +
                    (b * b / 6.0) * (-3.0 * x2 / r5 + 15.0 * x2 * y2 / r7));
    }
    const double k = x + a, l = x - a, m = y + b, n = y - b;
    return love_term(m, k, l, 2.0 * a) + love_term(n, l, k, -2.0 * a);
}

// the u_x bracket of a unit q_x traction: (1 - nu) Love + nu ylog
__device__ inline double cerruti_uxx_dev(double x, double y, double a, double b, double nu) {
    x = fabs(x);
    y = fabs(y);
    return (1.0 - nu) * love_uz_dev(x, y, a, b) + nu * cerruti_ylog_dev(x, y, a, b);
}

// the mixed bracket, odd in x and in y (0 on the axes)
__device__ inline double cerruti_uxy_dev(double x, double y, double a, double b) {
    const double xa = fabs(x), ya = fabs(y);
    const double k = xa + a, l = xa - a, m = ya + b, n = ya - b;
    const double Rkm = hypot(k, m), Rkn = hypot(k, n), Rlm = hypot(l, m), Rln = hypot(l, n);
    const double num = 16.0 * a * b * xa * ya * (1.0 / (Rkn + Rln) + 1.0 / (Rkm + Rlm));
    const double den = (Rlm + Rln) * (Rkn + Rkm);
    const double mag = den > 0.0 ? num / den : 0.0;
    return ((x >= 0.0) == (y >= 0.0)) ? mag : -mag;
}

}  // namespace asb
