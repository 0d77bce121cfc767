// Host-side numerics: incomplete gamma, its inverse (Halley iterations from a
// Wilson-Hilferty / small-x start) and the discrete-gamma rate categories.
#include "host_math.h"

#include <cmath>

namespace smccat {

namespace {

// Series for P(a, x), valid and fast for x < a + 1.
double p_series(double a, double x, double lpre) {
    double term = 1.0 / a, sum = term, ap = a;
    for (int n = 0; n < 1000000; ++n) {
        ap += 1.0;
        term *= x / ap;
        sum += term;
        if (std::fabs(term) <= std::fabs(sum) * 1e-17) break;
    }
    return sum * std::exp(lpre);
}

// Continued fraction for Q(a, x) (modified Lentz), valid for x >= a + 1.
double q_fraction(double a, double x, double lpre) {
    const double tiny = 1e-300;
    double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
    for (int i = 1; i < 1000000; ++i) {
        const double an = -i * (i - a);
        b += 2.0;
        d = an * d + b;
        if (std::fabs(d) < tiny) d = tiny;
        c = b + an / c;
        if (std::fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) <= 1e-17) break;
    }
    return std::exp(lpre) * h;
}

// Acklam's rational approximation of the standard normal quantile.
double normal_quantile(double p) {
    static const double a[] = {-3.969683028665376e+01, 2.209460984245205e+02,
                               -2.759285104469687e+02, 1.383577518672690e+02,
                               -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[] = {-5.447609879822406e+01, 1.615858368580409e+02,
                               -1.556989798598866e+02, 6.680131188771972e+01,
                               -1.328068155288572e+01};
    static const double c[] = {-7.784894002430293e-03, -3.223964580411365e-01,
                               -2.400758277161838e+00, -2.549732539343734e+00,
                               4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[] = {7.784695709041462e-03, 3.224671290700398e-01,
                               2.445134137142996e+00, 3.754408661907416e+00};
    const double lo = 0.02425, hi = 1.0 - lo;
    if (p < lo) {
        const double q = std::sqrt(-2.0 * std::log(p));
        return (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
               ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    }
    if (p > hi) {
        const double q = std::sqrt(-2.0 * std::log(1.0 - p));
        return -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
               ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    }
    const double q = p - 0.5, r = q * q;
    return (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
           (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
}

const double kLG[190] = {
    0.425093, 0.276818, 0.751878, 0.395144, 0.123954, 5.076149, 2.489084, 0.534551,
    0.528768, 0.062556, 0.969894, 2.807908, 1.695752, 0.523386, 0.084808, 1.038545,
    0.363970, 0.541712, 5.243870, 0.003499, 4.128591, 2.066040, 0.390192, 1.437645,
    0.844926, 0.569265, 0.267959, 0.348847, 0.358858, 2.426601, 4.509238, 0.927114,
    0.640543, 4.813505, 0.423881, 0.311484, 0.149830, 0.126991, 0.191503, 0.010690,
    0.320627, 0.072854, 0.044265, 0.008705, 0.108882, 0.395337, 0.301848, 0.068427,
    0.015076, 0.594007, 0.582457, 0.069673, 0.044261, 0.366317, 4.145067, 0.536518,
    6.326067, 2.145078, 0.282959, 0.013266, 3.234294, 1.807177, 0.296636, 0.697264,
    0.159069, 0.137500, 1.124035, 0.484133, 0.371004, 0.025548, 0.893680, 1.672569,
    0.173735, 0.139538, 0.442472, 4.273607, 6.312358, 0.656604, 0.253701, 0.052722,
    0.089525, 0.017416, 1.105251, 0.035855, 0.018811, 0.089586, 0.682139, 1.112727,
    2.592692, 0.023918, 1.798853, 1.177651, 0.332533, 0.161787, 0.394456, 0.075382,
    0.624294, 0.419409, 0.196961, 0.508851, 0.078281, 0.249060, 0.390322, 0.099849,
    0.094464, 4.727182, 0.858151, 4.008358, 1.240275, 2.784478, 1.223828, 0.611973,
    1.739990, 0.990012, 0.064105, 0.182287, 0.748683, 0.346960, 0.361819, 1.338132,
    2.139501, 0.578987, 2.000679, 0.425860, 1.143480, 1.080136, 0.604545, 0.129836,
    0.584262, 1.033739, 0.302936, 1.136863, 2.020366, 0.165001, 0.571468, 6.472279,
    0.180717, 0.593607, 0.045376, 0.029890, 0.670128, 0.236199, 0.077852, 0.268491,
    0.597054, 0.111660, 0.619632, 0.049906, 0.696175, 2.457121, 0.095131, 0.248862,
    0.140825, 0.218959, 0.314440, 0.612025, 0.135107, 1.165532, 0.257336, 0.120037,
    0.054679, 5.306834, 0.232523, 0.299648, 0.131932, 0.481306, 7.803902, 0.089613,
    0.400547, 0.245841, 3.151815, 2.547870, 0.170887, 0.083688, 0.037967, 1.959291,
    0.210332, 0.245034, 0.076701, 0.119013, 10.649107, 1.702745, 0.185202, 1.898718,
    0.654683, 0.296501, 0.098369, 2.188158, 0.189510, 0.249313,
};

}  // namespace

double gamma_p(double a, double x) {
    if (!(x > 0.0)) return 0.0;
    const double lpre = -x + a * std::log(x) - std::lgamma(a);
    return (x < a + 1.0) ? p_series(a, x, lpre) : 1.0 - q_fraction(a, x, lpre);
}

double gamma_p_inv(double a, double p) {
    if (!(p > 0.0)) return 0.0;
    if (!(p < 1.0)) return INFINITY;
    const double lga = std::lgamma(a);
    // Start: x^a / Gamma(a+1) ~ p for small x; Wilson-Hilferty otherwise.
    double x;
    const double xs = std::exp((std::log(p) + std::lgamma(a + 1.0)) / a);
    if (a < 1.0 && xs < 1.0) {
        x = xs;
    } else {
        const double z = normal_quantile(p);
        const double w = 1.0 - 1.0 / (9.0 * a) + z / (3.0 * std::sqrt(a));
        x = a * w * w * w;
        if (!(x > 0.0)) x = xs;
    }
    for (int it = 0; it < 200; ++it) {
        const double f = gamma_p(a, x) - p;
        const double lf1 = -x + (a - 1.0) * std::log(x) - lga;
        const double f1 = std::exp(lf1);
        if (!(f1 > 0.0) || !std::isfinite(f1)) break;
        const double u = f / f1;
        const double f2_over_f1 = (a - 1.0) / x - 1.0;
        double dx = u / (1.0 - 0.5 * std::fmin(1.0, u * f2_over_f1));  // Halley
        double nx = x - dx;
        if (!(nx > 0.0)) nx = 0.5 * x;
        const double step = std::fabs(nx - x);
        x = nx;
        if (step <= 1e-15 * x) break;
    }
    return x;
}

void discretize_gamma(double shape, int R, double* out) {
    if (R <= 1) {
        out[0] = 1.0;
        return;
    }
    const double interval = 1.0 / (2.0 * R);
    double tot = 0.0;
    for (int i = 0; i < R; ++i) {
        out[i] = gamma_p_inv(shape, (2.0 * i + 1.0) * interval) / shape;
        tot += out[i];
    }
    const double f = R / tot;
    for (int i = 0; i < R; ++i) out[i] *= f;
}

const double* lg_exchangeabilities() { return kLG; }

}  // namespace smccat
