// Learned CAT class proposal: a per-(site, class) scoring MLP.
//
// Input (kMlpIn = 44 floats) for site s and class k: the residue frequencies
// of column s over the taxa (20, gaps / X / ? excluded) and its fraction of
// non-residue cells (1); the class's stationary distribution pi_k (20);
// log n_k (1); sum_i freq_i log pi_k,i (1); one zero pad. Two ReLU hidden
// layers of kMlpHid units and a linear score; a site's proposal over its
// particle's classes is the softmax of the scores.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace smccat {

constexpr int kMlpIn = 44;
constexpr int kMlpHid = 128;
constexpr int kMlpW1 = 0;                            // [kMlpIn][kMlpHid]
constexpr int kMlpB1 = kMlpW1 + kMlpIn * kMlpHid;    // [kMlpHid]
constexpr int kMlpW2 = kMlpB1 + kMlpHid;             // [kMlpHid][kMlpHid]
constexpr int kMlpB2 = kMlpW2 + kMlpHid * kMlpHid;   // [kMlpHid]
constexpr int kMlpW3 = kMlpB2 + kMlpHid;             // [kMlpHid]
constexpr int kMlpB3 = kMlpW3 + kMlpHid;             // [1]
constexpr int kMlpParams = kMlpB3 + 1;
constexpr int kSiteFeat = 21;

}  // namespace smccat
