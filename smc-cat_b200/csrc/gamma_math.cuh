// Incomplete gamma, its inverse and the discrete-gamma rate categories, for
// host and device code alike (the device-side shape move re-discretises the
// rates): the series / continued-fraction evaluation of P(a, x) (Numerical
// Recipes 6.2), Halley iterations for its inverse from a Wilson-Hilferty or
// small-x start, and Acklam's rational approximation of the normal quantile
// for that start.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define SMCCAT_HD __host__ __device__
#else
#define SMCCAT_HD
#endif

namespace smccat {

// Series for P(a, x), valid and fast for x < a + 1.
SMCCAT_HD inline double gm_p_series(double a, double x, double lpre) {
    double term = 1.0 / a, sum = term, ap = a;
    for (int n = 0; n < 1000000; ++n) {
        ap += 1.0;
        term *= x / ap;
        sum += term;
        if (fabs(term) <= fabs(sum) * 1e-17) break;
    }
    return sum * exp(lpre);
}

// Continued fraction for Q(a, x) (modified Lentz), valid for x >= a + 1.
SMCCAT_HD inline double gm_q_fraction(double a, double x, double lpre) {
    const double tiny = 1e-300;
    double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
    for (int i = 1; i < 1000000; ++i) {
        const double an = -i * (i - a);
        b += 2.0;
        d = an * d + b;
        if (fabs(d) < tiny) d = tiny;
        c = b + an / c;
        if (fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (fabs(del - 1.0) <= 1e-17) break;
    }
    return exp(lpre) * h;
}

// Acklam's rational approximation of the standard normal quantile.
SMCCAT_HD inline double gm_normal_quantile(double p) {
    const double a0 = -3.969683028665376e+01, a1 = 2.209460984245205e+02, a2 = -2.759285104469687e+02,
                 a3 = 1.383577518672690e+02, a4 = -3.066479806614716e+01, a5 = 2.506628277459239e+00;
    const double b0 = -5.447609879822406e+01, b1 = 1.615858368580409e+02, b2 = -1.556989798598866e+02,
                 b3 = 6.680131188771972e+01, b4 = -1.328068155288572e+01;
    const double c0 = -7.784894002430293e-03, c1 = -3.223964580411365e-01, c2 = -2.400758277161838e+00,
                 c3 = -2.549732539343734e+00, c4 = 4.374664141464968e+00, c5 = 2.938163982698783e+00;
    const double d0 = 7.784695709041462e-03, d1 = 3.224671290700398e-01, d2 = 2.445134137142996e+00,
                 d3 = 3.754408661907416e+00;
    const double lo = 0.02425, hi = 1.0 - lo;
    if (p < lo) {
        const double q = sqrt(-2.0 * log(p));
        return (((((c0 * q + c1) * q + c2) * q + c3) * q + c4) * q + c5) /
               ((((d0 * q + d1) * q + d2) * q + d3) * q + 1.0);
    }
    if (p > hi) {
        const double q = sqrt(-2.0 * log(1.0 - p));
        return -(((((c0 * q + c1) * q + c2) * q + c3) * q + c4) * q + c5) /
               ((((d0 * q + d1) * q + d2) * q + d3) * q + 1.0);
    }
    const double q = p - 0.5, r = q * q;
    return (((((a0 * r + a1) * r + a2) * r + a3) * r + a4) * r + a5) * q /
           (((((b0 * r + b1) * r + b2) * r + b3) * r + b4) * r + 1.0);
}

// Regularized lower incomplete gamma P(a, x).
SMCCAT_HD inline double gm_gamma_p(double a, double x) {
    if (!(x > 0.0)) return 0.0;
    const double lpre = -x + a * log(x) - lgamma(a);
    return (x < a + 1.0) ? gm_p_series(a, x, lpre) : 1.0 - gm_q_fraction(a, x, lpre);
}

// Quantile of the standard gamma: x with P(a, x) = p.
SMCCAT_HD inline double gm_gamma_p_inv(double a, double p) {
    if (!(p > 0.0)) return 0.0;
    if (!(p < 1.0)) return INFINITY;
    const double lga = lgamma(a);
    // Start: x^a / Gamma(a+1) ~ p for small x; Wilson-Hilferty otherwise.
    double x;
    const double xs = exp((log(p) + lgamma(a + 1.0)) / a);
    if (a < 1.0 && xs < 1.0) {
        x = xs;
    } else {
        const double z = gm_normal_quantile(p);
        const double w = 1.0 - 1.0 / (9.0 * a) + z / (3.0 * sqrt(a));
        x = a * w * w * w;
        if (!(x > 0.0)) x = xs;
    }
    for (int it = 0; it < 200; ++it) {
        const double f = gm_gamma_p(a, x) - p;
        const double lf1 = -x + (a - 1.0) * log(x) - lga;
        const double f1 = exp(lf1);
        if (!(f1 > 0.0) || !isfinite(f1)) break;
        const double u = f / f1;
        const double f2_over_f1 = (a - 1.0) / x - 1.0;
        const double dx = u / (1.0 - 0.5 * fmin(1.0, u * f2_over_f1));  // Halley
        double nx = x - dx;
        if (!(nx > 0.0)) nx = 0.5 * x;
        const double step = fabs(nx - x);
        x = nx;
        if (step <= 1e-15 * x) break;
    }
    return x;
}

// discretizeGamma (src/core/Miscellaneous.hpp:22-37): the R midpoint
// quantiles (2i+1)/(2R) of Gamma(shape, scale 1/shape), rescaled to mean 1.
SMCCAT_HD inline void gm_discretize_gamma(double shape, int R, double* out) {
    if (R <= 1) {
        out[0] = 1.0;
        return;
    }
    const double interval = 1.0 / (2.0 * R);
    double tot = 0.0;
    for (int i = 0; i < R; ++i) {
        out[i] = gm_gamma_p_inv(shape, (2.0 * i + 1.0) * interval) / shape;
        tot += out[i];
    }
    const double f = R / tot;
    for (int i = 0; i < R; ++i) out[i] *= f;
}

}  // namespace smccat
