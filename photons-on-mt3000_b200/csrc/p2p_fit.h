// Polynomial for the FP32 forms of the pair kernel.
//
// g(x) = erfc(x) + (2/sqrt(pi)) x exp(-x^2) is written as g(x) = 1 - x^3 H(x^2);
// H is fitted on [0, umax] (umax = x_cut^2) by Chebyshev interpolation and
// handed to the kernels as monomials in t = u - u0, u0 = umax / 2 (Horner in
// a variable centred on the interval keeps the FP32 evaluation error near
// the fit error). Fixed-size arrays: no heap allocation.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>

#include "p2p_internal.h"

namespace p2p {

// H(u) = (1 - g(x)) / x^3 with x = sqrt(u). Near 0, where 1 - g cancels, the
// power series (4/sqrt(pi)) sum (-1)^n u^n / (n! (2n+3)) is used; it follows
// from g'(x) = -(4/sqrt(pi)) x^2 exp(-x^2).
inline double h_exact(double u) {
    const double k = 4.0 / std::sqrt(M_PI);
    if (u < 0.25) {
        double term = 1.0, sum = 0.0;
        for (int n = 0; n < 30; ++n) {
            sum += term / (2 * n + 3);
            term *= -u / (n + 1);
        }
        return k * sum;
    }
    const double x = std::sqrt(u);
    const double g = std::erfc(x) + (2.0 / std::sqrt(M_PI)) * x * std::exp(-u);
    return (1.0 - g) / (x * x * x);
}

struct PolyFit {
    int degree = 0;
    int ncoef_kernel = 0;  // coefficients the kernel instance evaluates (degree + 1)
    double u0 = 0, umax = 0;
    double max_err = 0;    // max over [0, umax] of sqrt(u) * |P(u) - H(u)|
    float coef[kMaxCoef] = {0};
};

// The smallest degree in {8, 10, 12, 14, 16, 20} whose interpolation error,
// weighted by x (the pair force error scales as x * dH), is below tol.
inline PolyFit fit_h(double umax, double tol) {
    static const int kDegrees[] = {8, 10, 12, 14, 16, 20};
    PolyFit best;
    const double half = 0.5 * umax;
    for (int D : kDegrees) {
        const int n = D + 1;
        double fj[kMaxCoef], cheb[kMaxCoef], mono[kMaxCoef], c[kMaxCoef];
        double tkm1[kMaxCoef], tk[kMaxCoef], tkp1[kMaxCoef];
        for (int j = 0; j < n; ++j) fj[j] = h_exact(half * (1.0 + std::cos(M_PI * (j + 0.5) / n)));
        for (int k = 0; k < n; ++k) {
            double s = 0;
            for (int j = 0; j < n; ++j) s += fj[j] * std::cos(M_PI * k * (j + 0.5) / n);
            cheb[k] = (k == 0 ? 1.0 : 2.0) * s / n;
        }
        // Chebyshev series -> monomials in tau = t / half
        for (int m = 0; m < n; ++m) mono[m] = tkm1[m] = tk[m] = 0.0;
        tkm1[0] = 1.0;           // T0
        if (n > 1) tk[1] = 1.0;  // T1
        for (int k = 0; k < n; ++k) {
            const double *T = (k == 0) ? tkm1 : tk;
            for (int m = 0; m < n; ++m) mono[m] += cheb[k] * T[m];
            if (k >= 1) {
                for (int m = 0; m < n; ++m) tkp1[m] = -tkm1[m];
                for (int m = 0; m + 1 < n; ++m) tkp1[m + 1] += 2.0 * tk[m];
                std::memcpy(tkm1, tk, sizeof(double) * n);
                std::memcpy(tk, tkp1, sizeof(double) * n);
            }
        }
        double sc = 1.0;
        for (int m = 0; m < n; ++m) {
            c[m] = mono[m] / sc;
            sc *= half;
        }
        double err = 0;
        for (int q = 0; q <= 4000; ++q) {
            const double u = umax * q / 4000.0;
            const double t = u - half;
            double h = c[n - 1];
            for (int m = n - 2; m >= 0; --m) h = h * t + c[m];
            err = std::max(err, std::sqrt(u) * std::fabs(h - h_exact(u)));
        }
        best.degree = D;
        best.u0 = half;
        best.umax = umax;
        best.max_err = err;
        std::memset(best.coef, 0, sizeof(best.coef));
        for (int m = 0; m < n; ++m) best.coef[m] = (float)c[m];
        best.ncoef_kernel = n;
        if (err <= tol) break;
    }
    return best;
}

// Polynomial domain of the FP32 forms: x in [0, x_cut], or [0, 4] without a
// cutoff (g(4) ~ 5e-7 of its value at 0).
inline double fit_umax(double x_cut) {
    const double xmax = x_cut > 0.0 ? x_cut : 4.0;
    return xmax * xmax;
}

}  // namespace p2p
