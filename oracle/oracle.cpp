// Smc-CAT likelihood oracle -- TEST INFRASTRUCTURE ONLY.
//
// A plain FP64 CPU restatement of the reference's likelihood hot path. It is
// used by tests/ as the parity checker, by __graft_entry__.smoke() as the
// checker, and by bench.py as the timed CPU baseline (the reference's own
// OpenMP-over-particles structure). Nothing in the product links or calls it.
//
// Parity status: parity unpinned. The reference ships no tests or golden
// vectors, and it cannot be compiled on this machine (its arithmetic lives in
// Eigen >= 3.4 and Boost.Math, neither installed), so this restatement is
// checked instead against golden vectors produced by an independent
// numpy/scipy restatement (tests/golden/make_golden.py) that follows the
// reference's own formulas -- general complex eigendecomposition + inverse for
// P(t) (Eigen::EigenSolver's role, here LAPACK dgeev) and the gamma quantile
// (Boost's role, here scipy) -- and against the LG table parsed from the
// reference source.
//
// Reference files (paths inside the Smc-CAT project):
//   src/analysis/RateMatrices.hpp            LG table, lower-triangle order
//   src/core/Miscellaneous.hpp               discretizeGamma, computeNextStep
//   src/analysis/TransitionProbabilityClass.cpp  Q, eigen, P(t), softmax
//   src/analysis/Particle.cpp                tips, refreshLikelihood, lnPrior,
//                                             gibbsPartitionMove
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int NS = 20;   // amino-acid states
constexpr int NB = 190;  // exchangeability pairs

// ---------------------------------------------------------------------------
// LG exchangeabilities (Le & Gascuel 2008), lower triangle row by row:
// row i (i = 1..19) lists the pairs (i, j) for j = 0..i-1. This is exactly the
// order of the reference's 190-vector (RateMatrices.hpp:97-111).
// State order ARNDCQEGHILKMFPSTWYV (Alignment.cpp:7-31).
const double kLGLower[NB] = {
    0.425093,
    0.276818, 0.751878,
    0.395144, 0.123954, 5.076149,
    2.489084, 0.534551, 0.528768, 0.062556,
    0.969894, 2.807908, 1.695752, 0.523386, 0.084808,
    1.038545, 0.363970, 0.541712, 5.243870, 0.003499, 4.128591,
    2.066040, 0.390192, 1.437645, 0.844926, 0.569265, 0.267959, 0.348847,
    0.358858, 2.426601, 4.509238, 0.927114, 0.640543, 4.813505, 0.423881, 0.311484,
    0.149830, 0.126991, 0.191503, 0.010690, 0.320627, 0.072854, 0.044265, 0.008705, 0.108882,
    0.395337, 0.301848, 0.068427, 0.015076, 0.594007, 0.582457, 0.069673, 0.044261, 0.366317,
    4.145067,
    0.536518, 6.326067, 2.145078, 0.282959, 0.013266, 3.234294, 1.807177, 0.296636, 0.697264,
    0.159069, 0.137500,
    1.124035, 0.484133, 0.371004, 0.025548, 0.893680, 1.672569, 0.173735, 0.139538, 0.442472,
    4.273607, 6.312358, 0.656604,
    0.253701, 0.052722, 0.089525, 0.017416, 1.105251, 0.035855, 0.018811, 0.089586, 0.682139,
    1.112727, 2.592692, 0.023918, 1.798853,
    1.177651, 0.332533, 0.161787, 0.394456, 0.075382, 0.624294, 0.419409, 0.196961, 0.508851,
    0.078281, 0.249060, 0.390322, 0.099849, 0.094464,
    4.727182, 0.858151, 4.008358, 1.240275, 2.784478, 1.223828, 0.611973, 1.739990, 0.990012,
    0.064105, 0.182287, 0.748683, 0.346960, 0.361819, 1.338132,
    2.139501, 0.578987, 2.000679, 0.425860, 1.143480, 1.080136, 0.604545, 0.129836, 0.584262,
    1.033739, 0.302936, 1.136863, 2.020366, 0.165001, 0.571468, 6.472279,
    0.180717, 0.593607, 0.045376, 0.029890, 0.670128, 0.236199, 0.077852, 0.268491, 0.597054,
    0.111660, 0.619632, 0.049906, 0.696175, 2.457121, 0.095131, 0.248862, 0.140825,
    0.218959, 0.314440, 0.612025, 0.135107, 1.165532, 0.257336, 0.120037, 0.054679, 5.306834,
    0.232523, 0.299648, 0.131932, 0.481306, 7.803902, 0.089613, 0.400547, 0.245841, 3.151815,
    2.547870, 0.170887, 0.083688, 0.037967, 1.959291, 0.210332, 0.245034, 0.076701, 0.119013,
    10.649107, 1.702745, 0.185202, 1.898718, 0.654683, 0.296501, 0.098369, 2.188158, 0.189510,
    0.249313,
};

// ---------------------------------------------------------------------------
// Regularized lower incomplete gamma P(a, x): series for x < a + 1, Lentz
// continued fraction for Q otherwise (the classic split, Numerical Recipes 6.2).
double gamma_p(double a, double x) {
    if (x <= 0.0) return 0.0;
    const double lpre = -x + a * std::log(x) - std::lgamma(a);
    if (x < a + 1.0) {
        double ap = a, term = 1.0 / a, sum = term;
        for (int n = 0; n < 100000; ++n) {
            ap += 1.0;
            term *= x / ap;
            sum += term;
            if (std::fabs(term) < std::fabs(sum) * 1e-17) break;
        }
        return sum * std::exp(lpre);
    }
    const double tiny = 1e-300;
    double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
    for (int i = 1; i < 100000; ++i) {
        const double an = -i * (i - a);
        b += 2.0;
        d = an * d + b;
        if (std::fabs(d) < tiny) d = tiny;
        c = b + an / c;
        if (std::fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < 1e-17) break;
    }
    return 1.0 - std::exp(lpre) * h;
}

// Inverse of P(a, .): bracket, bisect in log space, then Newton polish.
double gamma_p_inv(double a, double p) {
    if (p <= 0.0) return 0.0;
    double hi = 1.0;
    while (gamma_p(a, hi) < p) hi *= 2.0;
    double lo = hi * 0.5;
    while (lo > 1e-300 && gamma_p(a, lo) > p) lo *= 0.5;
    for (int it = 0; it < 200; ++it) {
        const double mid = std::sqrt(lo * hi);
        if (gamma_p(a, mid) < p) lo = mid; else hi = mid;
        if (hi - lo <= 1e-16 * hi) break;
    }
    double x = std::sqrt(lo * hi);
    for (int it = 0; it < 3; ++it) {
        const double f = gamma_p(a, x) - p;
        const double dens = std::exp(-x + (a - 1.0) * std::log(x) - std::lgamma(a));
        if (dens <= 0.0 || !std::isfinite(dens)) break;
        const double nx = x - f / dens;
        if (!(nx > 0.0) || !std::isfinite(nx)) break;
        x = nx;
    }
    return x;
}

// ---------------------------------------------------------------------------
// Symmetric eigendecomposition by cyclic Jacobi rotations (row-by-row sweep,
// Rutishauser's stable rotation formulas). A is destroyed; V gets the
// eigenvectors as columns, w the eigenvalues.
void jacobi_eigen(double* A, double* V, double* w, int n) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) off += A[i * n + j] * A[i * n + j];
        if (off == 0.0) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[p * n + q];
                if (apq == 0.0) continue;
                const double app = A[p * n + p], aqq = A[q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                double t = 1.0 / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                if (theta < 0.0) t = -t;
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {  // columns p, q
                    const double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {  // rows p, q
                    const double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                A[p * n + q] = A[q * n + p] = 0.0;
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
        }
    }
    for (int i = 0; i < n; ++i) w[i] = A[i * n + i];
}

// Spectral data of one class: P(t) = L diag(exp(lambda t)) Rm with
// L = diag(pi)^-1/2 U and Rm = U^T diag(pi)^1/2.
struct Spectral {
    double lam[NS];
    double L[NS * NS];
    double Rm[NS * NS];
};

// softmax of the logits: TransitionProbabilityClass.cpp:101-109.
void softmax20(const double* logits, double* pi) {
    double tot = 0.0;
    for (int i = 0; i < NS; ++i) { pi[i] = std::exp(logits[i]); tot += pi[i]; }
    for (int i = 0; i < NS; ++i) pi[i] /= tot;
}

// Q exactly as recomputeEigens builds it (TransitionProbabilityClass.cpp:50-75):
// Q(i,j) = exp(b_ij) * pi_j, diagonal = -row sum, divided by sum_i pi_i(-Q_ii).
void rate_matrix(const double* base, const double* pi, double* Q) {
    std::memset(Q, 0, sizeof(double) * NS * NS);
    int c = 0;
    for (int i = 1; i < NS; ++i)
        for (int j = 0; j < i; ++j, ++c) {
            const double e = std::exp(base[c]);
            Q[i * NS + j] = e;
            Q[j * NS + i] = e;
        }
    for (int i = 0; i < NS; ++i)
        for (int j = 0; j < NS; ++j) Q[i * NS + j] *= pi[j];
    for (int i = 0; i < NS; ++i) {
        double off = 0.0;
        for (int j = 0; j < NS; ++j) if (j != i) off += Q[i * NS + j];
        Q[i * NS + i] = -off;
    }
    double mean = 0.0;
    for (int i = 0; i < NS; ++i) mean += -Q[i * NS + i] * pi[i];
    for (int k = 0; k < NS * NS; ++k) Q[k] /= mean;
}

// The reference diagonalises Q with a general complex solver. Q is
// reversible, so S = D^1/2 Q D^-1/2 is symmetric with the same (real)
// spectrum; P(t) = D^-1/2 U e^{Lt} U^T D^1/2 is the same matrix.
void spectral(const double* base, const double* pi, Spectral* sp) {
    double Q[NS * NS], S[NS * NS], U[NS * NS];
    rate_matrix(base, pi, Q);
    double sq[NS];
    for (int i = 0; i < NS; ++i) sq[i] = std::sqrt(pi[i]);
    for (int i = 0; i < NS; ++i)
        for (int j = 0; j < NS; ++j) S[i * NS + j] = sq[i] * Q[i * NS + j] / sq[j];
    for (int i = 0; i < NS; ++i)  // exact symmetry before rotating
        for (int j = i + 1; j < NS; ++j) {
            const double m = 0.5 * (S[i * NS + j] + S[j * NS + i]);
            S[i * NS + j] = S[j * NS + i] = m;
        }
    jacobi_eigen(S, U, sp->lam, NS);
    for (int i = 0; i < NS; ++i)
        for (int k = 0; k < NS; ++k) {
            sp->L[i * NS + k] = U[i * NS + k] / sq[i];
            sp->Rm[k * NS + i] = U[i * NS + k] * sq[i];
        }
}

// recomputeTransitionProbs (TransitionProbabilityClass.cpp:83-95): P(t*r).
void transition(const Spectral& sp, double t, double* P) {
    double e[NS];
    for (int k = 0; k < NS; ++k) e[k] = std::exp(sp.lam[k] * t);
    for (int i = 0; i < NS; ++i)
        for (int j = 0; j < NS; ++j) {
            double s = 0.0;
            for (int k = 0; k < NS; ++k) s += sp.L[i * NS + k] * e[k] * sp.Rm[k * NS + j];
            P[i * NS + j] = s;
        }
}

// ---------------------------------------------------------------------------
// Tree helpers on the flat parent array (tips 0..T-1, internal T..2T-2).
struct FlatTree {
    int N = 0, root = -1;
    std::vector<int> kids;  // 2 per node (-1 for tips), ascending id
    std::vector<int> post;  // all nodes, children before parents
};

bool build_tree(int T, const int32_t* parent, FlatTree* t) {
    const int N = 2 * T - 1;
    t->N = N;
    t->kids.assign(2 * N, -1);
    t->root = -1;
    std::vector<int> nk(N, 0);
    for (int n = 0; n < N; ++n) {
        const int p = parent[n];
        if (p < 0) { if (t->root >= 0) return false; t->root = n; continue; }
        if (p < T || p >= N || nk[p] >= 2) return false;
        t->kids[2 * p + nk[p]++] = n;
    }
    if (t->root < T) return false;
    for (int n = T; n < N; ++n) {
        if (nk[n] != 2) return false;
        if (t->kids[2 * n] > t->kids[2 * n + 1]) std::swap(t->kids[2 * n], t->kids[2 * n + 1]);
    }
    t->post.clear();
    std::vector<std::pair<int, int>> st;  // (node, next child)
    st.push_back({t->root, 0});
    while (!st.empty()) {
        auto& top = st.back();
        const int n = top.first;
        if (n >= T && top.second < 2) {
            const int c = t->kids[2 * n + top.second++];
            st.push_back({c, 0});
        } else {
            t->post.push_back(n);
            st.pop_back();
        }
    }
    return (int)t->post.size() == N;
}

// Tip encoding + invariance flags: Particle.cpp:44-73. A column is invariant
// iff every taxon carries the same code (so an all-gap column is invariant
// and a gap differs from a residue); its invariant character is that code if
// it is a residue, else 0.
void tip_encode(const uint8_t* codes, int T, int S, double* isInv, int32_t* invChar) {
    for (int s = 0; s < S; ++s) {
        const int c1 = codes[s];
        double inv = 1.0;
        for (int t = 0; t < T; ++t) if (codes[t * S + s] != c1) inv = 0.0;
        isInv[s] = inv;
        invChar[s] = (inv == 1.0 && c1 < 20) ? c1 : 0;
    }
}

struct State {
    int T, S, R, K;
    const uint8_t* codes;
    const int32_t* parent;
    const double* branch;
    const double* base;
    const double* logits;  // K x 20
    const int32_t* assign; // S
    double pinv;
    const double* rates;   // R
};

// refreshLikelihood(true) (Particle.cpp:530-675) for one particle state.
// Returns lnL; optionally writes per-site log-likelihoods.
double lnl_full(const State& st, double* site_out) {
    const int T = st.T, S = st.S, R = st.R, K = st.K, N = 2 * T - 1;
    FlatTree tree;
    if (!build_tree(T, st.parent, &tree)) return std::numeric_limits<double>::quiet_NaN();
    std::vector<std::vector<int>> members(K);
    for (int s = 0; s < S; ++s) {
        const int k = st.assign[s];
        if (k < 0 || k >= K) return std::numeric_limits<double>::quiet_NaN();
        members[k].push_back(s);
    }
    // Classes: stationary, spectral data, P for every node and rate
    // (Particle.cpp:537-548).
    std::vector<double> pi(K * NS);
    std::vector<double> P((size_t)K * N * R * NS * NS);
    for (int k = 0; k < K; ++k) {
        softmax20(st.logits + k * NS, &pi[k * NS]);
        Spectral sp;
        spectral(st.base, &pi[k * NS], &sp);
        for (int n = 0; n < N; ++n)
            for (int r = 0; r < R; ++r)
                transition(sp, st.branch[n] * st.rates[r],
                           &P[(((size_t)k * N + n) * R + r) * NS * NS]);
    }
    // Conditional likelihoods [node][site*R + r][20] and rescale [node][site*R + r].
    const size_t SR = (size_t)S * R;
    std::vector<double> CL((size_t)N * SR * NS, 0.0);
    std::vector<double> resc((size_t)N * SR, 0.0);
    for (int t = 0; t < T; ++t)
        for (int s = 0; s < S; ++s) {
            const int code = st.codes[t * S + s];
            for (int r = 0; r < R; ++r) {
                double* v = &CL[((size_t)t * SR + s * R + r) * NS];
                if (code < 20) v[code] = 1.0;
                else for (int i = 0; i < NS; ++i) v[i] = 1.0;
            }
        }
    double work[NS];
    for (int n : tree.post) {
        if (n < T) continue;
        double* pN = &CL[(size_t)n * SR * NS];
        for (size_t i = 0; i < SR * NS; ++i) pN[i] = 1.0;
        for (int ci = 0; ci < 2; ++ci) {
            const int d = tree.kids[2 * n + ci];
            const double* pD = &CL[(size_t)d * SR * NS];
            for (int k = 0; k < K; ++k)
                for (int r = 0; r < R; ++r) {
                    const double* Pm = &P[(((size_t)k * N + d) * R + r) * NS * NS];
                    for (int c : members[k]) {
                        const double* x = &pD[((size_t)c * R + r) * NS];
                        for (int i = 0; i < NS; ++i) work[i] = 0.0;
                        for (int j = 0; j < NS; ++j) {
                            const double xj = x[j];
                            for (int i = 0; i < NS; ++i) work[i] += Pm[i * NS + j] * xj;
                        }
                        double* y = &pN[((size_t)c * R + r) * NS];
                        for (int i = 0; i < NS; ++i) y[i] *= work[i];
                    }
                }
        }
        // Per (site, rate) max-rescaling (Particle.cpp:614-624).
        for (size_t c = 0; c < SR; ++c) {
            double* y = &pN[c * NS];
            double mx = y[0];
            for (int i = 1; i < NS; ++i) mx = std::max(mx, y[i]);
            for (int i = 0; i < NS; ++i) y[i] /= mx;
            resc[(size_t)n * SR + c] = std::log(mx);
        }
    }
    // Root reduction (Particle.cpp:634-674): no 1/R weight, +I mixing.
    std::vector<double> isInv(S);
    std::vector<int32_t> invChar(S);
    tip_encode(st.codes, T, S, isInv.data(), invChar.data());
    const double* pR = &CL[(size_t)tree.root * SR * NS];
    const double inv_scale = 1.0 - st.pinv;
    double lnL = 0.0;
    std::vector<double> logs(R);
    for (int k = 0; k < K; ++k) {
        const double* pk = &pi[k * NS];
        for (int c : members[k]) {
            double mx = -INFINITY;
            for (int r = 0; r < R; ++r) {
                const double* v = &pR[((size_t)c * R + r) * NS];
                double s = 0.0;
                for (int i = 0; i < NS; ++i) s += pk[i] * v[i];
                double l = std::log(s);
                for (int n = 0; n < N; ++n) l += resc[(size_t)n * SR + c * R + r];
                logs[r] = l;
                if (l > mx) mx = l;
            }
            double se = 0.0;
            for (int r = 0; r < R; ++r) se += std::exp(logs[r] - mx);
            const double lse = mx + std::log(se);
            const double site = std::exp(lse) * inv_scale + st.pinv * pk[invChar[c]] * isInv[c];
            const double ls = std::log(site);
            if (site_out) site_out[c] = ls;
            lnL += ls;
        }
    }
    return lnL;
}

// Single-site likelihood of site `site` under a class with stationary `pi`
// (the per-class loop body of gibbsPartitionMove, Particle.cpp:857-933, in its
// corrected form: the tip vector of `site` itself, rescalers read at the
// stride they were written). Returns log of the +I-mixed site likelihood.
double site_lnl_class(const State& st, const FlatTree& tree, const double* pi,
                      const Spectral& sp, int site, const double* isInv,
                      const int32_t* invChar) {
    const int T = st.T, R = st.R, N = 2 * T - 1;
    std::vector<double> CL((size_t)N * R * NS, 0.0);
    std::vector<double> resc((size_t)N * R, 0.0);
    double P[NS * NS], work[NS];
    for (int n : tree.post) {
        double* pN = &CL[(size_t)n * R * NS];
        if (n < T) {
            const int code = st.codes[n * st.S + site];
            for (int r = 0; r < R; ++r)
                for (int i = 0; i < NS; ++i)
                    pN[r * NS + i] = (code < 20) ? (i == code ? 1.0 : 0.0) : 1.0;
            continue;
        }
        for (int i = 0; i < R * NS; ++i) pN[i] = 1.0;
        for (int ci = 0; ci < 2; ++ci) {
            const int d = tree.kids[2 * n + ci];
            for (int r = 0; r < R; ++r) {
                transition(sp, st.branch[d] * st.rates[r], P);
                const double* x = &CL[((size_t)d * R + r) * NS];
                for (int i = 0; i < NS; ++i) work[i] = 0.0;
                for (int j = 0; j < NS; ++j)
                    for (int i = 0; i < NS; ++i) work[i] += P[i * NS + j] * x[j];
                for (int i = 0; i < NS; ++i) pN[r * NS + i] *= work[i];
            }
        }
        for (int r = 0; r < R; ++r) {
            double* y = &pN[r * NS];
            double mx = y[0];
            for (int i = 1; i < NS; ++i) mx = std::max(mx, y[i]);
            for (int i = 0; i < NS; ++i) y[i] /= mx;
            resc[(size_t)n * R + r] = std::log(mx);
        }
    }
    const double* pR = &CL[(size_t)tree.root * R * NS];
    std::vector<double> logs(R);
    double mx = -INFINITY;
    for (int r = 0; r < R; ++r) {
        double s = 0.0;
        for (int i = 0; i < NS; ++i) s += pi[i] * pR[r * NS + i];
        double l = std::log(s);
        for (int n = 0; n < N; ++n) l += resc[(size_t)n * R + r];
        logs[r] = l;
        mx = std::max(mx, l);
    }
    double se = 0.0;
    for (int r = 0; r < R; ++r) se += std::exp(logs[r] - mx);
    const double lse = mx + std::log(se);
    const double v = std::exp(lse) * (1.0 - st.pinv) + st.pinv * pi[invChar[site]] * isInv[site];
    return std::log(v);
}

double log_normal_pdf(double z) { return -0.5 * z * z - 0.5 * std::log(2.0 * M_PI); }

double log_gamma_pdf(double x, double shape, double scale) {
    return (shape - 1.0) * std::log(x) - x / scale - std::lgamma(shape) - shape * std::log(scale);
}

}  // namespace

extern "C" {

// 190-vector of the LG model as the reference stores it for LG runs
// (Particle.cpp:84-94; recomputeEigens exponentiates each entry).
void orc_lg_base(double* out) { std::memcpy(out, kLGLower, sizeof(kLGLower)); }

double orc_gamma_p(double a, double x) { return gamma_p(a, x); }

// Quantile of Gamma(shape, scale): boost::math::quantile in discretizeGamma.
double orc_gamma_quantile(double shape, double scale, double p) {
    return scale * gamma_p_inv(shape, p);
}

// discretizeGamma (Miscellaneous.hpp:22-37): midpoint quantiles of
// Gamma(shape, 1/shape) at (2i+1)/(2R), rescaled to mean 1.
void orc_discretize_gamma(double shape, int R, double* out) {
    const double interval = 1.0 / (2.0 * R);
    double tot = 0.0;
    for (int i = 0; i < R; ++i) {
        out[i] = orc_gamma_quantile(shape, 1.0 / shape, (i * 2.0 + 1.0) * interval);
        tot += out[i];
    }
    const double f = R / tot;
    for (int i = 0; i < R; ++i) out[i] *= f;
}

void orc_softmax20(const double* logits, double* pi) { softmax20(logits, pi); }

void orc_rate_matrix(const double* base, const double* pi, double* Q) { rate_matrix(base, pi, Q); }

// P(t) for one class given the base vector and stationary distribution.
void orc_transition(const double* base, const double* pi, double t, double* P) {
    Spectral sp;
    spectral(base, pi, &sp);
    transition(sp, t, P);
}

// Eigenvalues (ascending) of the normalised Q.
void orc_eigenvalues(const double* base, const double* pi, double* lam) {
    Spectral sp;
    spectral(base, pi, &sp);
    std::sort(sp.lam, sp.lam + NS);
    std::memcpy(lam, sp.lam, sizeof(sp.lam));
}

void orc_tip_encode(const uint8_t* codes, int T, int S, double* isInv, int32_t* invChar) {
    tip_encode(codes, T, S, isInv, invChar);
}

// Post-order of a flat tree (children before parents); returns 0 on success.
int orc_postorder(int T, const int32_t* parent, int32_t* post) {
    FlatTree t;
    if (!build_tree(T, parent, &t)) return -1;
    for (int i = 0; i < t.N; ++i) post[i] = t.post[i];
    return 0;
}

// lnL of one particle state (full refresh). site_out (S doubles) may be null.
double orc_lnl(int T, int S, int R, const uint8_t* codes, const int32_t* parent,
               const double* branch, const double* base, int K, const double* logits,
               const int32_t* assign, double pinv, const double* rates, double* site_out) {
    State st{T, S, R, K, codes, parent, branch, base, logits, assign, pinv, rates};
    return lnl_full(st, site_out);
}

// refreshLikelihood(true) over a batch of particles with the reference's
// OpenMP-over-particles structure (main.cpp:295, schedule(dynamic)).
// Per-particle arrays are packed: parent/branch [np][2T-1], base [np][190],
// logits [np][kmax][20], assign [np][S], pinv [np], rates [np][R].
void orc_lnl_batch(int np, int T, int S, int R, const uint8_t* codes, const int32_t* parent,
                   const double* branch, const double* base, const int32_t* K, int kmax,
                   const double* logits, const int32_t* assign, const double* pinv,
                   const double* rates, double* out, int nthreads) {
    const int N = 2 * T - 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic)
#endif
    for (int p = 0; p < np; ++p) {
        State st{T, S, R, K[p], codes, parent + (size_t)p * N, branch + (size_t)p * N,
                 base + (size_t)p * NB, logits + (size_t)p * kmax * NS,
                 assign + (size_t)p * S, pinv[p], rates + (size_t)p * R};
        out[p] = lnl_full(st, nullptr);
    }
}

int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Particle::lnPrior (Particle.cpp:484-517). `lg` selects whether the 190
// N(0,1) terms are included; logits are the K class logit vectors.
double orc_ln_prior(int T, int S, int R, int lg, const double* branch, double shape,
                    const double* base, int K, const double* logits, const int32_t* counts,
                    double dpp_alpha) {
    const int N = 2 * T - 1;
    double lnP = 0.0;
    double len = 0.0;
    for (int n = 0; n < N; ++n) len += branch[n];
    lnP += log_gamma_pdf(len, (double)(N - 1), 1.0 / 10.0);
    if (R > 1) lnP += log_gamma_pdf(shape, 3.0, 2.0);
    if (!lg)
        for (int i = 0; i < NB; ++i) lnP += log_normal_pdf(base[i]);
    lnP += std::log(dpp_alpha) * K;
    for (int k = 0; k < K; ++k) {
        for (int i = 0; i < NS; ++i) lnP += log_normal_pdf(logits[k * NS + i]);
        lnP += std::lgamma((double)counts[k]);
    }
    lnP += std::lgamma(dpp_alpha) - std::lgamma(dpp_alpha + S);
    return lnP;
}

// computeNextStep (Miscellaneous.hpp:42-109): bisection on the temperature
// for the target ESS, then weight update and normalisation.
void orc_next_step(int np, double* raw_w, const double* lnl, double* norm_w, double* ess,
                   double target_ess, double* cur_temp, double last_temp) {
    std::vector<double> tw(np), ew(np);
    auto ess_at = [&](double temp) {
        for (int n = 0; n < np; ++n) tw[n] = raw_w[n] + (temp - last_temp) * lnl[n];
        const double mx = *std::max_element(tw.begin(), tw.end());
        double tot = 0.0;
        for (int n = 0; n < np; ++n) { ew[n] = std::exp(tw[n] - mx); tot += ew[n]; }
        double sq = 0.0;
        for (int n = 0; n < np; ++n) { ew[n] /= tot; sq += ew[n] * ew[n]; }
        return 1.0 / sq;
    };
    double low = last_temp, high = 1.0;
    while (high - low > 1e-5) {
        const double mid = 0.5 * (low + high);
        if (ess_at(mid) > target_ess) low = mid; else high = mid;
    }
    *cur_temp = high;
    for (int n = 0; n < np; ++n) raw_w[n] = raw_w[n] + (high - last_temp) * lnl[n];
    const double mx = *std::max_element(raw_w, raw_w + np);
    double tot = 0.0;
    for (int n = 0; n < np; ++n) { norm_w[n] = std::exp(raw_w[n] - mx); tot += norm_w[n]; }
    double sq = 0.0;
    for (int n = 0; n < np; ++n) { norm_w[n] /= tot; sq += norm_w[n] * norm_w[n]; }
    *ess = 1.0 / sq;
}

// One Neal-Algorithm-8 weight vector (gibbsPartitionMove, Particle.cpp:808-941,
// corrected form). `assign` is the state with `site` already removed from its
// class (classes with zero members are expected to have been dropped by the
// caller); `aux_logits` holds m auxiliary classes. Writes K + m unnormalised
// log weights: temp * site lnL + log n_k, or + log(alpha / m) for the aux.
void orc_gibbs_weights(int T, int S, int R, const uint8_t* codes, const int32_t* parent,
                       const double* branch, const double* base, int K, const double* logits,
                       const int32_t* counts, double pinv, const double* rates, int site,
                       int m, const double* aux_logits, double temp, double dpp_alpha,
                       double* out) {
    State st{T, S, R, K, codes, parent, branch, base, logits, nullptr, pinv, rates};
    FlatTree tree;
    build_tree(T, parent, &tree);
    std::vector<double> isInv(S);
    std::vector<int32_t> invChar(S);
    tip_encode(codes, T, S, isInv.data(), invChar.data());
    const double alpha_split = std::log(dpp_alpha / m);
    for (int k = 0; k < K + m; ++k) {
        const double* lg = (k < K) ? logits + k * NS : aux_logits + (k - K) * NS;
        double pi[NS];
        softmax20(lg, pi);
        Spectral sp;
        spectral(base, pi, &sp);
        const double l = site_lnl_class(st, tree, pi, sp, site, isInv.data(), invChar.data()) * temp;
        out[k] = l + ((k < K) ? std::log((double)counts[k]) : alpha_split);
    }
}

}  // extern "C"
