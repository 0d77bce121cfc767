// Host-side numerics of the B200 engine (no device code).
#pragma once
#include <cstdint>

namespace smccat {

// Regularized lower incomplete gamma P(a, x).
double gamma_p(double a, double x);

// Quantile of the standard gamma: x with P(a, x) = p.
double gamma_p_inv(double a, double p);

// discretizeGamma (src/core/Miscellaneous.hpp:22-37): the R midpoint
// quantiles (2i+1)/(2R) of Gamma(shape, scale 1/shape), rescaled to mean 1.
void discretize_gamma(double shape, int R, double* out);

// LG exchangeabilities in the reference's 190-vector order
// (src/analysis/RateMatrices.hpp:7-111): pairs (i, j) for i = 1..19, j < i.
const double* lg_exchangeabilities();

}  // namespace smccat
