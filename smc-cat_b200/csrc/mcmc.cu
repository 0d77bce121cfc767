// Rejuvenation MCMC driver and SMC weight step of the B200 engine.
//
// The reference runs Mcmc::operator() (Mcmc.cpp:25-73) once per particle,
// particles spread over OpenMP threads (main.cpp:295-312), and every MH step
// calls refreshLikelihood() on that one particle. Here all particles of a
// range advance in lockstep: at every step each unfinished particle makes its
// next proposal on the host mirror (the reference's move rules, Tree.cpp and
// Particle.cpp), one batched dirty refresh evaluates every proposal on the
// device, and the MH test (tempered likelihood + lnPrior + Hastings) decides
// per particle; accept/reject only flips workspace indices.
//
// computeNextStep (Miscellaneous.hpp:42-109) runs on the device in FP64 on
// the log-likelihoods already resident there.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include "engine_internal.h"
#include "gibbs.h"
#include "host_math.h"
#include "smccat.h"

namespace smccat {
namespace {

int mfail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

// Move kinds in the reference's UpdateType order (Particle.hpp:18-30).
enum Kind {
    ADAPTIVE_NNI = 0, NNI = 1, SPR = 2, BRANCH_LENGTH = 3, SCALE_SUBTREE = 4, INVAR = 5,
    RATE_SHAPE = 6, STATIONARY_SINGLE = 7, RATE_MATRIX_SINGLE = 8, RATE_MATRIX_FULL = 9
};

// Registry entries of main.cpp:55-106.
enum Family { FAM_TREE, FAM_STATIONARY, FAM_SHAPE, FAM_INVAR, FAM_RATE_MATRIX };

struct Split {
    uint64_t w[2];
    bool operator==(const Split& o) const { return w[0] == o.w[0] && w[1] == o.w[1]; }
};
struct SplitHash {
    size_t operator()(const Split& s) const { return std::hash<uint64_t>()(s.w[0] * 0x9E3779B97F4A7C15ull ^ s.w[1]); }
};

struct Tuning {
    smccat_tuning t;
    std::vector<double> chol;  // 190 x 190 lower triangular, row-major
    std::unordered_map<Split, double, SplitHash> split_post;
};

std::unordered_map<const smccat_ctx*, Tuning>& tunings() {
    static std::unordered_map<const smccat_ctx*, Tuning> m;
    return m;
}

std::mutex& tunings_mu() {
    static std::mutex mu;
    return mu;
}

// Per-context MCMC settings (entries stay valid: unordered_map never moves
// its nodes; a context's entry is erased by smccat_destroy).
Tuning& tuning_of(const smccat_ctx* c) {
    std::lock_guard<std::mutex> lk(tunings_mu());
    auto& m = tunings();
    auto it = m.find(c);
    if (it != m.end()) return it->second;
    Tuning tn;
    tn.t = smccat_tuning{0.01, 1.0, 1.0, 1.0, 0.25, 0.25, 100.0, 0.01};  // Particle.hpp:87-94, 106
    tn.chol.assign(190 * 190, 0.0);
    for (int i = 0; i < 190; ++i) tn.chol[i * 190 + i] = 0.5;         // Particle.hpp:93
    return m.emplace(c, std::move(tn)).first->second;
}

using Rng = std::mt19937_64;

double unif(Rng& g) { return std::generate_canonical<double, 53>(g); }

double normal(Rng& g, double sd) { return std::normal_distribution<double>(0.0, sd)(g); }

double beta_draw(Rng& g, double a, double b) {
    const double x = std::gamma_distribution<double>(a, 1.0)(g);
    const double y = std::gamma_distribution<double>(b, 1.0)(g);
    return x / (x + y);
}

double beta_lpdf(double x, double a, double b) {
    return std::lgamma(a + b) - std::lgamma(a) - std::lgamma(b) + (a - 1.0) * std::log(x) +
           (b - 1.0) * std::log1p(-x);
}

double gamma_lpdf(double x, double shape, double scale) {
    return (shape - 1.0) * std::log(x) - x / scale - std::lgamma(shape) - shape * std::log(scale);
}

double normal_lpdf(double z) { return -0.5 * z * z - 0.91893853320467274178; }

// Working copy of one particle's tree with child lists in id order.
struct WTree {
    int T, N, root;
    std::vector<int32_t> parent;
    std::vector<double> branch;
    std::vector<int32_t> kids;  // 2 per node
    void load(const Mirror& m, int T_) {
        T = T_;
        N = 2 * T - 1;
        root = m.root;
        parent = m.parent;
        branch = m.branch;
        kids = m.kids;
    }
    void rebuild_kids() {
        std::vector<int> nk(N, 0);
        std::fill(kids.begin(), kids.end(), -1);
        for (int n = 0; n < N; ++n)
            if (parent[n] >= 0) kids[2 * parent[n] + nk[parent[n]]++] = n;
        for (int n = T; n < N; ++n)
            if (kids[2 * n] > kids[2 * n + 1]) std::swap(kids[2 * n], kids[2 * n + 1]);
    }
    bool in_subtree(int x, int r) const {  // Tree.hpp:29-34
        for (; x >= 0; x = parent[x])
            if (x == r) return true;
        return false;
    }
    int uniform_node(Rng& g) const { return std::min(N - 1, (int)(unif(g) * N)); }
    // chooseNodeFromSet (Tree.cpp:614-623) over the (ordered) children of n.
    int choose_child(Rng& g, int n) const { return kids[2 * n + std::min(1, (int)(unif(g) * 2))]; }
    // Clade bit sets of every node, canonicalised so that taxon 0 is set
    // (Tree.cpp:485-519).
    std::vector<Split> splits() const {
        std::vector<Split> s(N, Split{{0, 0}});
        std::vector<int> order;
        order.reserve(N);
        std::vector<int> st{root};
        while (!st.empty()) {
            const int n = st.back();
            st.pop_back();
            order.push_back(n);
            if (n >= T) { st.push_back(kids[2 * n]); st.push_back(kids[2 * n + 1]); }
        }
        for (int i = N - 1; i >= 0; --i) {
            const int n = order[i];
            if (n < T) s[n].w[n >> 6] |= 1ull << (n & 63);
            else for (int c = 0; c < 2; ++c) {
                s[n].w[0] |= s[kids[2 * n + c]].w[0];
                s[n].w[1] |= s[kids[2 * n + c]].w[1];
            }
        }
        Split full{{0, 0}};
        for (int t = 0; t < T; ++t) full.w[t >> 6] |= 1ull << (t & 63);
        for (auto& x : s)
            if (!(x.w[0] & 1ull)) { x.w[0] = ~x.w[0] & full.w[0]; x.w[1] = ~x.w[1] & full.w[1]; }
        return s;
    }
};

int popcount2(const Split& s) { return __builtin_popcountll(s.w[0]) + __builtin_popcountll(s.w[1]); }

// Adaptive-NNI node weights (Tree.cpp:676-694): epsilon + (1 - posterior of
// the node's split), or epsilon + 1 when the split is absent or trivial.
std::vector<double> annI_weights(const WTree& t, const Tuning& tn, double* total) {
    std::vector<double> w(t.N, 0.0);
    const auto sp = t.splits();
    *total = 0.0;
    for (int n = t.T; n < t.N; ++n) {
        if (n == t.root) continue;
        double v = tn.t.adaptive_nni_epsilon;
        const int cnt = popcount2(sp[n]);
        auto it = (cnt == 1 || cnt == t.T - 1) ? tn.split_post.end() : tn.split_post.find(sp[n]);
        v += (it != tn.split_post.end()) ? 1.0 - it->second : 1.0;
        w[n] = v;
        *total += v;
    }
    return w;
}

struct Proposal {
    int kind = -1;
    double hastings = 0.0;
};

// One proposal on particle p (Particle::treeMove etc.), applied through the
// engine's edit calls so the dirty sets follow.
int propose(smccat_ctx* c, int p, int family, Rng& g, const Tuning& tn, Proposal* out) {
    const Slot& s = slot_of(c, p);
    const Mirror& m = s.cur;
    const Dims& d = dims_of(c);
    out->hastings = 0.0;
    if (family == FAM_TREE) {
        WTree t;
        t.load(m, d.T);
        const double u = unif(g);  // Particle.cpp:680-701
        if (u < 0.5 && u >= 0.4) {  // SPR, Tree.cpp:768-812
            int x;
            do { x = t.uniform_node(g); } while (x == t.root || x < t.T);
            const int sch = t.choose_child(g, x);
            const int sib = (t.kids[2 * x] == sch) ? t.kids[2 * x + 1] : t.kids[2 * x];
            int a;
            do { a = t.uniform_node(g); } while (t.in_subtree(a, x) || a == t.root);
            const int a_par = t.parent[a];
            const int gpar = t.parent[x];
            t.parent[sib] = gpar;
            t.parent[x] = (a_par == x) ? gpar : a_par;
            t.parent[a] = x;
            out->kind = SPR;
            return smccat_set_topology(c, p, t.parent.data(), t.branch.data());
        }
        if (u < 0.4) {  // NNI (u < 0.1) or adaptive NNI, Tree.cpp:625-766
            int x;
            double sel = 0.0, tot = 0.0;
            std::vector<double> w;
            if (u < 0.1) {
                do { x = t.uniform_node(g); } while (x == t.root || x < t.T);
                out->kind = NNI;
            } else {
                w = annI_weights(t, tn, &tot);
                const double r = unif(g);
                double cum = 0.0;
                x = -1;
                for (int n = t.T; n < t.N; ++n) {
                    if (n == t.root) continue;
                    cum += w[n] / tot;
                    x = n;
                    if (r <= cum) break;
                }
                sel = w[x] / tot;
                out->kind = ADAPTIVE_NNI;
            }
            const int a = t.parent[x];
            const int n1 = t.choose_child(g, x);
            (void)unif(g);  // the reference draws from the one-element sibling set too
            const int n2 = (t.kids[2 * a] == x) ? t.kids[2 * a + 1] : t.kids[2 * a];
            t.parent[n1] = a;
            t.parent[n2] = x;
            if (out->kind == ADAPTIVE_NNI) {
                t.rebuild_kids();
                double tot2 = 0.0;
                const auto w2 = annI_weights(t, tn, &tot2);
                out->hastings = std::log(w2[x] / tot2) - std::log(sel);
            }
            return smccat_set_topology(c, p, t.parent.data(), t.branch.data());
        }
        int x;
        do { x = t.uniform_node(g); } while (x == t.root);
        if (u < 0.9) {  // scaleBranchMove, Tree.cpp:553-578
            const double sc = std::exp(tn.t.scale_delta * (unif(g) - 0.5));
            const double nb = t.branch[x] * sc;
            out->kind = BRANCH_LENGTH;
            out->hastings = std::log(sc);
            return smccat_set_branch_lengths(c, p, 1, &x, &nb);
        }
        // scaleSubtreeMove, Tree.cpp:580-612
        const double sc = std::exp(tn.t.subtree_scale_delta * (unif(g) - 0.5));
        std::vector<int32_t> nodes;
        std::vector<double> lens;
        std::vector<int> st{x};
        while (!st.empty()) {
            const int n = st.back();
            st.pop_back();
            nodes.push_back(n);
            lens.push_back(t.branch[n] * sc);
            if (n >= t.T) { st.push_back(t.kids[2 * n]); st.push_back(t.kids[2 * n + 1]); }
        }
        out->kind = SCALE_SUBTREE;
        out->hastings = nodes.size() * std::log(sc);
        return smccat_set_branch_lengths(c, p, (int)nodes.size(), nodes.data(), lens.data());
    }
    if (family == FAM_STATIONARY) {
        // Particle::stationaryMove (Particle.cpp:734-742) with the shift applied
        // to the class's logit: the reference shifts pi and then recomputes pi
        // from the unchanged logits, which makes its move a no-op.
        const int k = std::min(m.K - 1, (int)(unif(g) * m.K));
        const int i = std::min(19, (int)(unif(g) * 20));
        double lg[kStates];
        std::memcpy(lg, &m.logits[(size_t)k * kStates], sizeof(lg));
        lg[i] += normal(g, tn.t.stationary_delta);
        out->kind = STATIONARY_SINGLE;
        return smccat_set_class_logits(c, p, k, lg);
    }
    if (family == FAM_SHAPE) {  // Particle::shapeMove, Particle.cpp:768-783
        const double sc = std::exp(tn.t.shape_delta * (unif(g) - 0.5));
        out->kind = RATE_SHAPE;
        out->hastings = std::log(sc);
        return smccat_set_shape(c, p, m.shape * sc);
    }
    if (family == FAM_INVAR) {  // Particle::invarMove, Particle.cpp:744-766
        const double al = tn.t.invar_alpha;
        const double cur = m.pinv;
        const double a = al + 1.0, b = al / cur - a + 2.0;
        double nv = beta_draw(g, a, b);
        nv = std::min(std::max(nv, 1e-300), 1.0 - 1e-16);
        const double b2 = al / nv - a + 2.0;
        out->kind = INVAR;
        out->hastings = beta_lpdf(cur, a, b2) - beta_lpdf(nv, a, b);
        return smccat_set_pinv(c, p, nv);
    }
    // Particle::rateMatrixMove (Particle.cpp:706-732); the new exchangeabilities
    // take effect at once (the reference only updates its eigensystems later).
    std::vector<double> base = m.base;
    if (unif(g) < 0.25) {
        double z[kBase];
        for (int i = 0; i < kBase; ++i) z[i] = normal(g, 1.0);
        for (int i = 0; i < kBase; ++i) {
            double sacc = 0.0;
            for (int j = 0; j <= i; ++j) sacc += tn.chol[i * kBase + j] * z[j];
            base[i] += sacc;
        }
        out->kind = RATE_MATRIX_FULL;
    } else {
        const int i = std::min(kBase - 1, (int)(kBase * unif(g)));
        base[i] += normal(g, 1.0) * tn.t.rate_matrix_delta;
        out->kind = RATE_MATRIX_SINGLE;
    }
    return smccat_set_base(c, p, base.data());
}

// Particle::lnPrior (Particle.cpp:484-517) of the current mirror state.
double ln_prior(const smccat_ctx* c, int p, const Tuning& tn) {
    const Slot& s = slot_of(c, p);
    const Mirror& m = s.cur;
    const Dims& d = dims_of(c);
    double len = 0.0;
    for (int n = 0; n < d.N; ++n) len += m.branch[n];
    double lnp = gamma_lpdf(len, (double)(d.N - 1), 0.1);
    if (d.R > 1) lnp += gamma_lpdf(m.shape, 3.0, 2.0);
    if (!(model_flags_of(c) & SMCCAT_MODEL_LG))
        for (int i = 0; i < kBase; ++i) lnp += normal_lpdf(m.base[i]);
    std::vector<int> cnt(m.K, 0);
    for (int v : s.assign) cnt[v]++;
    const double alpha = tn.t.dpp_alpha;
    int kk = 0;
    for (int k = 0; k < m.K; ++k) {
        if (cnt[k] == 0) continue;  // an empty class carries no prior mass
        ++kk;
        for (int i = 0; i < kStates; ++i) lnp += normal_lpdf(m.logits[(size_t)k * kStates + i]);
        lnp += std::lgamma((double)cnt[k]);
    }
    lnp += std::log(alpha) * kk;
    lnp += std::lgamma(alpha) - std::lgamma(alpha + d.S);
    return lnp;
}

// ---------------------------------------------------------------------------
// computeNextStep on the device: one CTA, fixed-order FP64 reductions.
constexpr int kStepThreads = 1024;

__device__ double block_reduce(double v, double* sh, bool is_max) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int o = kStepThreads / 2; o > 0; o >>= 1) {
        if (t < o) sh[t] = is_max ? fmax(sh[t], sh[t + o]) : sh[t] + sh[t + o];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__device__ double ess_at(const double* w, const double* lnl, int n, double temp, double last,
                         double* sh) {
    double mx = -INFINITY;
    for (int i = threadIdx.x; i < n; i += kStepThreads) mx = fmax(mx, w[i] + (temp - last) * lnl[i]);
    mx = block_reduce(mx, sh, true);
    double tot = 0.0;
    for (int i = threadIdx.x; i < n; i += kStepThreads) tot += exp(w[i] + (temp - last) * lnl[i] - mx);
    tot = block_reduce(tot, sh, false);
    double sq = 0.0;
    for (int i = threadIdx.x; i < n; i += kStepThreads) {
        const double e = exp(w[i] + (temp - last) * lnl[i] - mx) / tot;
        sq += e * e;
    }
    sq = block_reduce(sq, sh, false);
    return 1.0 / sq;
}

__global__ void __launch_bounds__(kStepThreads) smc_step_kernel(double* w, const double* lnl, int n,
                                                                double target, double last,
                                                                double* normw, double* out) {
    __shared__ double sh[kStepThreads];
    double low = last, high = 1.0;
    for (int it = 0; it < 200 && high - low > 1e-5; ++it) {
        const double mid = 0.5 * (low + high);
        if (ess_at(w, lnl, n, mid, last, sh) > target) low = mid;
        else high = mid;
    }
    const double temp = high;
    for (int i = threadIdx.x; i < n; i += kStepThreads) w[i] = w[i] + (temp - last) * lnl[i];
    __syncthreads();
    double mx = -INFINITY;
    for (int i = threadIdx.x; i < n; i += kStepThreads) mx = fmax(mx, w[i]);
    mx = block_reduce(mx, sh, true);
    double tot = 0.0;
    for (int i = threadIdx.x; i < n; i += kStepThreads) tot += exp(w[i] - mx);
    tot = block_reduce(tot, sh, false);
    double sq = 0.0;
    for (int i = threadIdx.x; i < n; i += kStepThreads) {
        const double e = exp(w[i] - mx) / tot;
        normw[i] = e;
        sq += e * e;
    }
    sq = block_reduce(sq, sh, false);
    if (threadIdx.x == 0) { out[0] = temp; out[1] = 1.0 / sq; }
}

}  // namespace

void mcmc_release(const smccat_ctx* c) {
    std::lock_guard<std::mutex> lk(tunings_mu());
    tunings().erase(c);
}

void split_table(const smccat_ctx* c, std::vector<uint64_t>* keys, std::vector<double>* prob) {
    const auto& mp = tuning_of(c).split_post;
    std::vector<std::pair<Split, double>> v(mp.begin(), mp.end());
    std::sort(v.begin(), v.end(), [](const auto& x, const auto& y) {
        return x.first.w[0] != y.first.w[0] ? x.first.w[0] < y.first.w[0] : x.first.w[1] < y.first.w[1];
    });
    keys->resize(2 * v.size());
    prob->resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        (*keys)[2 * i] = v[i].first.w[0];
        (*keys)[2 * i + 1] = v[i].first.w[1];
        (*prob)[i] = v[i].second;
    }
}

}  // namespace smccat

using namespace smccat;

extern "C" {

int smccat_set_tuning(smccat_ctx* c, const smccat_tuning* t) {
    if (!c || !t) return mfail(SMCCAT_EINVAL, "null argument");
    if (!(t->invar_alpha > 0.0) || !(t->dpp_alpha > 0.0)) return mfail(SMCCAT_EINVAL, "bad tuning");
    tuning_of(c).t = *t;
    return SMCCAT_OK;
}

int smccat_get_tuning(smccat_ctx* c, smccat_tuning* t) {
    if (!c || !t) return mfail(SMCCAT_EINVAL, "null argument");
    *t = tuning_of(c).t;
    return SMCCAT_OK;
}

int smccat_set_rate_cholesky(smccat_ctx* c, const double* lower190) {
    if (!c || !lower190) return mfail(SMCCAT_EINVAL, "null argument");
    auto& ch = tuning_of(c).chol;
    for (int i = 0; i < 190; ++i)
        for (int j = 0; j < 190; ++j) ch[i * 190 + j] = (j <= i) ? lower190[i * 190 + j] : 0.0;
    return SMCCAT_OK;
}

int smccat_get_rate_cholesky(smccat_ctx* c, double* lower190) {
    if (!c || !lower190) return mfail(SMCCAT_EINVAL, "null argument");
    const auto& ch = tuning_of(c).chol;
    std::copy(ch.begin(), ch.end(), lower190);
    return SMCCAT_OK;
}

int smccat_set_split_posteriors(smccat_ctx* c, int32_t n, const uint64_t* bits, const double* prob) {
    if (!c || n < 0 || (n > 0 && (!bits || !prob))) return mfail(SMCCAT_EINVAL, "null argument");
    auto& mp = tuning_of(c).split_post;
    mp.clear();
    for (int i = 0; i < n; ++i) mp[Split{{bits[2 * i], bits[2 * i + 1]}}] = prob[i];
    return SMCCAT_OK;
}

int smccat_resample_tune(smccat_ctx* c, int32_t first, int32_t count, const double* w, double u,
                         int32_t copy, int32_t* anc_out) {
    NvtxRange range("smccat_resample_tune");
    if (!c || !w || !anc_out) return mfail(SMCCAT_EINVAL, "null argument");
    if (first < 0 || count < 1) return mfail(SMCCAT_EINVAL, "bad range");
    if (!(u >= 0.0 && u < 1.0)) return mfail(SMCCAT_EINVAL, "u must be in [0, 1)");
    for (int i = 0; i < count; ++i)
        if (!slot_of(c, first + i).loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
    const Dims& d = dims_of(c);
    const int flags = model_flags_of(c);
    // Systematic resampling, main.cpp:178-192 (same walk, same arithmetic).
    std::vector<int> a;
    a.reserve(count);
    {
        double cumulative = w[0];
        int k = 0;
        double ruler = u / static_cast<double>(count);
        const double step = 1.0 / static_cast<double>(count);
        while ((int)a.size() < count) {
            if (ruler <= cumulative) {
                a.push_back(k);
                ruler += step;
            } else if (++k >= count) {
                k = count - 1;
                cumulative = 1.0;
            } else {
                cumulative += w[k];
            }
        }
    }
    // Proposal tuning over the resampled population, main.cpp:197-291.
    // Variances are population variances (boost::accumulators tag::variance).
    struct Var {
        double n = 0, s = 0, s2 = 0;
        void add(double x) { n += 1; s += x; s2 += x * x; }
        double var() const { const double m = s / n; return s2 / n - m * m; }
    } shape_v, branch_v, stat_v;
    double pinv_mean = 0.0;
    std::vector<double> xtx;
    const bool gtr = !(flags & SMCCAT_MODEL_LG);
    if (gtr) xtx.assign(kBase * kBase, 0.0);
    for (int n : a) {
        const Mirror& m = slot_of(c, first + n).cur;
        shape_v.add(std::log(m.shape));
        pinv_mean += m.pinv;
        for (int x = 0; x < d.N; ++x)
            if (x != m.root) branch_v.add(std::log(m.branch[x]));  // every non-root branch
        for (int k = 0; k < m.K; ++k)
            for (int j = 0; j < kStates; ++j) stat_v.add(m.logits[(size_t)k * kStates + j]);
        if (gtr)  // X^T X of the base vectors, uncentred as in main.cpp:249
            for (int i = 0; i < kBase; ++i)
                for (int j = 0; j < kBase; ++j) xtx[i * kBase + j] += m.base[i] * m.base[j];
    }
    pinv_mean /= static_cast<double>(count);
    Tuning& tn = tuning_of(c);
    double shrink_diag = 0.0;
    if (gtr) {
        const double scale = (2.38 * 2.38) / 190.0 * 0.21, shrink = 0.2;
        for (double& v : xtx) v *= scale;
        for (int i = 0; i < kBase; ++i) shrink_diag += xtx[i * kBase + i];
        shrink_diag = shrink_diag / 190.0 * shrink;
        for (double& v : xtx) v *= 1.0 - shrink;
        for (int i = 0; i < kBase; ++i) xtx[i * kBase + i] += shrink_diag + 1e-6;
        // Cholesky (LLT), lower triangle in place.
        for (int j = 0; j < kBase; ++j) {
            double dj = xtx[j * kBase + j];
            for (int k = 0; k < j; ++k) dj -= xtx[j * kBase + k] * xtx[j * kBase + k];
            if (!(dj > 0.0)) return mfail(SMCCAT_ENUMERIC, "rate-matrix covariance is not positive definite");
            dj = std::sqrt(dj);
            xtx[j * kBase + j] = dj;
            for (int i = j + 1; i < kBase; ++i) {
                double v = xtx[i * kBase + j];
                for (int k = 0; k < j; ++k) v -= xtx[i * kBase + k] * xtx[j * kBase + k];
                xtx[i * kBase + j] = v / dj;
            }
        }
        for (int i = 0; i < kBase; ++i)
            for (int j = i + 1; j < kBase; ++j) xtx[i * kBase + j] = 0.0;
        tn.chol = xtx;
        tn.t.rate_matrix_delta = std::max(shrink_diag, 0.01);
    }
    tn.t.shape_delta = std::max(0.5 * shape_v.var(), 0.01);
    tn.t.scale_delta = std::max(branch_v.var(), 0.01);
    tn.t.subtree_scale_delta = tn.t.scale_delta;
    tn.t.stationary_delta = std::max(stat_v.var(), 0.01);
    if ((flags & SMCCAT_MODEL_INVAR) && pinv_mean > 0.0) tn.t.invar_alpha = pinv_mean * 0.5;
    // computeSplitPosteriors over the assignments (main.cpp:203-207).
    std::vector<double> mult(count, 0.0);
    for (int n : a) mult[n] += 1.0 / static_cast<double>(count);
    int32_t nsplit = 0;
    if (d.T <= 128) {
        const int rc = smccat_compute_split_posteriors(c, first, count, mult.data(), 0, &nsplit, nullptr,
                                                       nullptr);
        if (rc) return rc;
    }
    for (int i = 0; i < count; ++i) anc_out[i] = a[i];
    if (!copy) return SMCCAT_OK;
    // copyFromSerialized of each ancestor into its new slot (main.cpp:299-301).
    const size_t N = d.N, S = d.S, K = d.Kmax;
    std::vector<int32_t> par(count * N), nk(count), asg(count * S);
    std::vector<double> br(count * N), base(count * kBase), lg(count * K * kStates), pv(count), sh(count);
    int rc = smccat_get_particles(c, first, count, par.data(), br.data(), base.data(), nk.data(), lg.data(),
                                  asg.data(), pv.data(), sh.data());
    if (rc) return rc;
    std::vector<int32_t> par2(count * N), nk2(count), asg2(count * S);
    std::vector<double> br2(count * N), base2(count * kBase), lg2(count * K * kStates), pv2(count), sh2(count);
    for (int i = 0; i < count; ++i) {
        const int f = a[i];
        std::copy(&par[f * N], &par[f * N] + N, &par2[i * N]);
        std::copy(&br[f * N], &br[f * N] + N, &br2[i * N]);
        std::copy(&base[f * kBase], &base[f * kBase] + kBase, &base2[i * kBase]);
        std::copy(&lg[f * K * kStates], &lg[f * K * kStates] + K * kStates, &lg2[i * K * kStates]);
        std::copy(&asg[f * S], &asg[f * S] + S, &asg2[i * S]);
        nk2[i] = nk[f];
        pv2[i] = pv[f];
        sh2[i] = sh[f];
    }
    return smccat_set_particles(c, first, count, par2.data(), br2.data(), base2.data(), nk2.data(),
                                lg2.data(), asg2.data(), pv2.data(), sh2.data());
}

int smccat_compute_split_posteriors(smccat_ctx* c, int32_t first, int32_t count,
                                    const double* weights, int32_t cap, int32_t* n_out,
                                    uint64_t* bits, double* prob) {
    if (!c || !n_out) return mfail(SMCCAT_EINVAL, "null argument");
    const Dims& d = dims_of(c);
    if (d.T > 128) return mfail(SMCCAT_EINVAL, "split bit sets hold at most 128 taxa");
    if (first < 0 || count < 1 || cap < 0) return mfail(SMCCAT_EINVAL, "bad range");
    for (int i = 0; i < count; ++i)
        if (!slot_of(c, first + i).loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
    auto less = [](const Split& a, const Split& b) {
        return a.w[1] != b.w[1] ? a.w[1] < b.w[1] : a.w[0] < b.w[0];
    };
    std::unordered_map<Split, double, SplitHash> acc;
    for (int i = 0; i < count; ++i) {  // particle order fixes the summation order
        WTree t;
        t.load(slot_of(c, first + i).cur, d.T);
        const std::vector<Split> sp = t.splits();
        std::vector<Split> set;
        set.reserve(sp.size());
        for (int n = 0; n < t.N; ++n)
            if (n != t.root) set.push_back(sp[n]);
        std::sort(set.begin(), set.end(), less);
        set.erase(std::unique(set.begin(), set.end()), set.end());
        const double w = weights ? weights[i] : 1.0 / count;
        for (const Split& x : set) acc[x] += w;
    }
    tuning_of(c).split_post = acc;
    *n_out = (int32_t)acc.size();
    if (bits && prob) {
        std::vector<std::pair<Split, double>> v(acc.begin(), acc.end());
        std::sort(v.begin(), v.end(), [&](const auto& a, const auto& b) {
            return a.second != b.second ? a.second > b.second : less(a.first, b.first);
        });
        const int m = std::min<int>(cap, (int)v.size());
        for (int i = 0; i < m; ++i) {
            bits[2 * i] = v[i].first.w[0];
            bits[2 * i + 1] = v[i].first.w[1];
            prob[i] = v[i].second;
        }
    }
    return SMCCAT_OK;
}

int smccat_ln_prior(smccat_ctx* c, int32_t first, int32_t count, double* out) {
    if (!c || !out) return mfail(SMCCAT_EINVAL, "null argument");
    const Tuning& tn = tuning_of(c);
    for (int i = 0; i < count; ++i) {
        const Slot& s = slot_of(c, first + i);
        if (!s.loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
        out[i] = ln_prior(c, first + i, tn);
    }
    return SMCCAT_OK;
}

int smccat_propose(smccat_ctx* c, int32_t p, int32_t family, uint64_t seed, int32_t* kind,
                   double* hastings) {
    if (!c) return mfail(SMCCAT_EINVAL, "null context");
    if (p < 0 || !slot_of(c, p).loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
    if (family < SMCCAT_FAMILY_TREE || family > SMCCAT_FAMILY_RATE_MATRIX)
        return mfail(SMCCAT_EINVAL, "unknown move family");
    if (family == SMCCAT_FAMILY_INVAR && !(slot_of(c, p).cur.pinv > 0.0))
        return mfail(SMCCAT_EINVAL, "invariant-site move needs pinv > 0");
    Rng g(seed);
    Proposal pr;
    const int rc = propose(c, p, family, g, tuning_of(c), &pr);
    if (rc) return rc;
    if (kind) *kind = pr.kind;
    if (hastings) *hastings = pr.hastings;
    return SMCCAT_OK;
}

int smccat_rejuvenate(smccat_ctx* c, int32_t first, int32_t count, int32_t iterations,
                      double temperature, uint64_t seed, smccat_move_stats* stats) {
    NvtxRange range("smccat_rejuvenate");
    if (!c) return mfail(SMCCAT_EINVAL, "null context");
    if (iterations < 0 || count < 0 || first < 0) return mfail(SMCCAT_EINVAL, "bad range");
    const Dims& d = dims_of(c);
    const int flags = model_flags_of(c);
    const Tuning& tn = tuning_of(c);
    for (int i = 0; i < count; ++i) {
        const Slot& s = slot_of(c, first + i);
        if (!s.loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
        if (s.pending) return mfail(SMCCAT_ESTATE, "particle has uncommitted edits");
    }
    // The move registry of main.cpp:55-106: (weight, repeat count, family).
    struct Entry { double w; int family; };
    std::vector<Entry> reg{{3.0, FAM_TREE}, {1.0, FAM_STATIONARY}};
    if (d.R > 1) reg.push_back({1.0, FAM_SHAPE});
    if (flags & SMCCAT_MODEL_INVAR) reg.push_back({1.0, FAM_INVAR});
    if (!(flags & SMCCAT_MODEL_LG)) reg.push_back({1.0, FAM_RATE_MATRIX});
    double wt = 0.0;
    for (auto& e : reg) wt += e.w;
    std::vector<double> cum;  // Mcmc::initMoveProbs, Mcmc.cpp:15-23
    double acc = 0.0;
    for (auto& e : reg) { acc += e.w; cum.push_back(acc / wt); }
    auto repeats = [&](int family, int p) -> int {
        switch (family) {
            case FAM_TREE: return (int)(d.T * 0.25);
            case FAM_STATIONARY: return slot_of(c, p).cur.K * 2;
            case FAM_SHAPE: return 2;
            case FAM_INVAR: return 2;
            default: return 5;
        }
    };
    struct PS {
        Rng g;
        int iter = 0, family = 0, left = 0;
        bool done = false;
        double lik = 0.0, prior = 0.0;
        Proposal pr;
    };
    std::vector<PS> ps(count);
    for (int i = 0; i < count; ++i) ps[i].g.seed(seed * 0x9E3779B97F4A7C15ull + (uint64_t)(first + i) + 1);
    smccat_move_stats st{};
    // Mcmc.cpp:34-37: current likelihood (root reduction) and prior.
    int rc = refresh_internal(c, first, count, SMCCAT_REFRESH_DIRTY, nullptr);
    if (rc) return rc;
    std::vector<double> lnl(count);
    rc = smccat_get_lnl(c, first, count, lnl.data());
    if (rc) return rc;
#pragma omp parallel for schedule(static) num_threads(host_team()) if (count >= kParallelParticles)
    for (int i = 0; i < count; ++i) {
        ps[i].lik = lnl[i] * temperature;
        ps[i].prior = ln_prior(c, first + i, tn);
    }
    std::vector<uint8_t> active(count), mask(count);
    std::vector<int> prc(count);
    std::vector<std::string> perr(count);
    std::vector<double> nprior(count);
    for (;;) {
        // Proposals on the host mirrors; each particle has its own generator
        // and touches only its own slot, so they run in parallel.
#pragma omp parallel for schedule(dynamic, 8) num_threads(host_team()) if (count >= kParallelParticles)
        for (int i = 0; i < count; ++i) {
            PS& q = ps[i];
            active[i] = 0;
            prc[i] = SMCCAT_OK;
            while (!q.done && q.left == 0) {
                if (q.iter == iterations) { q.done = true; break; }
                const double u = unif(q.g);  // Mcmc.cpp:40-50
                int j = 0;
                while (j + 1 < (int)cum.size() && !(u < cum[j])) ++j;
                q.family = reg[j].family;
                q.left = repeats(q.family, first + i);
                q.iter++;
            }
            if (q.done) continue;
            const int r = propose(c, first + i, q.family, q.g, tn, &q.pr);
            if (r) {
                prc[i] = r;
                perr[i] = smccat_last_error();  // the message is per thread
                continue;
            }
            q.left--;
            active[i] = 1;
        }
        int n_active = 0;
        for (int i = 0; i < count; ++i) {
            if (prc[i]) return mfail(prc[i], perr[i]);
            n_active += active[i];
        }
        if (n_active == 0) break;
        rc = refresh_internal(c, first, count, SMCCAT_REFRESH_DIRTY, active.data());
        if (rc) return rc;
        rc = smccat_get_lnl(c, first, count, lnl.data());
        if (rc) return rc;
        st.lockstep_steps++;
#pragma omp parallel for schedule(static) num_threads(host_team()) if (count >= kParallelParticles)
        for (int i = 0; i < count; ++i)
            if (active[i]) nprior[i] = ln_prior(c, first + i, tn);
        for (int i = 0; i < count; ++i) {
            mask[i] = 1;
            if (!active[i]) continue;
            PS& q = ps[i];
            const double nlik = lnl[i] * temperature;
            const double ratio = (nprior[i] + nlik) - (q.prior + q.lik) + q.pr.hastings;  // Mcmc.cpp:57-60
            const bool ok = std::log(unif(q.g)) <= ratio;
            mask[i] = ok ? 1 : 0;
            st.proposed[q.pr.kind]++;
            if (ok) {
                st.accepted[q.pr.kind]++;
                q.prior = nprior[i];
                q.lik = nlik;
            }
        }
        rc = smccat_accept(c, first, count, mask.data());
        if (rc) return rc;
    }
    if (stats) *stats = st;
    return SMCCAT_OK;
}

}  // extern "C"

namespace {

// Runs the device Gibbs kernel on the listed particles. In weights mode
// (site >= 0) only writes the weight vector of particle list[0] and changes
// nothing; otherwise installs the new class sets and refreshes. With
// `learned_updates` > 0 the learned-proposal MH move runs instead of Gibbs.
int run_gibbs(smccat_ctx* c, const std::vector<int>& list, double temperature, uint64_t seed,
              int site, const double* aux, double* weights_out, smccat_gibbs_stats* stats,
              int learned_updates = 0, smccat_learned_stats* lstats = nullptr) {
    const Dims& d = dims_of(c);
    const int n = (int)list.size();
    if (n == 0) return SMCCAT_OK;
    const float* site_feat = nullptr;
    const void* mlp = nullptr;
    if (learned_updates > 0) {
        mlp = learned_inference_weights(c, &site_feat);
        if (!mlp) return mfail(SMCCAT_ESTATE, "the learned proposal has not been trained");
    }
    const int naux = gibbs_aux();
    const int Kcap = d.Kmax + 64;
    const int ks = Kcap + naux;
    std::vector<GibbsPart> parts(n);
    std::vector<GibbsNode> tree((size_t)n * d.NI);
    std::vector<int32_t> assign((size_t)n * d.S);
    int nslots = 1;
    std::vector<double> branch((size_t)n * d.N), base((size_t)n * kBase), logits((size_t)n * ks * kStates, 0.0);
    std::vector<double> auxv((size_t)n * naux * kStates, 0.0);
    for (int j = 0; j < n; ++j) {
        const Slot& s = slot_of(c, list[j]);
        const Mirror& m = s.cur;
        GibbsPart& g = parts[j];
        g.p = list[j];
        g.K = m.K;
        g.n_iter = learned_updates > 0 ? learned_updates : (site >= 0 ? 1 : d.S / 2);  // Particle.cpp:791
        g.fixed_site = site;
        g.pinv = m.pinv;
        for (int r = 0; r < kMaxRates; ++r) g.rates[r] = m.rates[r];
        // Stash slots from a free list: a node's result takes a free slot and
        // its internal children's slots are freed once it has read them.
        std::vector<int> slot_of_node(d.N, -1), free_slots;
        int used = 0;
        for (int q = 0; q < d.NI; ++q) {
            const int x = m.post[q];
            GibbsNode& g = tree[(size_t)j * d.NI + q];
            g.n = x;
            for (int ci = 0; ci < 2; ++ci) {
                const int ch = m.kids[2 * x + ci];
                g.c[ci] = ch;
                g.sc[ci] = ch >= d.T ? slot_of_node[ch] : -1;
                if (ch >= d.T && slot_of_node[ch] < 0)
                    return mfail(SMCCAT_ESTATE, "internal post-order lists a parent before its child");
                if (ch >= d.T) free_slots.push_back(slot_of_node[ch]);
            }
            if (free_slots.empty()) free_slots.push_back(used++);
            g.so = free_slots.back();
            free_slots.pop_back();
            g.pad[0] = g.pad[1] = 0;
            slot_of_node[x] = g.so;
        }
        nslots = std::max(nslots, used);
        std::copy(m.branch.begin(), m.branch.end(), branch.begin() + (size_t)j * d.N);
        std::copy(m.base.begin(), m.base.end(), base.begin() + (size_t)j * kBase);
        std::copy(m.logits.begin(), m.logits.begin() + (size_t)m.K * kStates,
                  logits.begin() + (size_t)j * ks * kStates);
        std::copy(s.assign.begin(), s.assign.end(), assign.begin() + (size_t)j * d.S);
        if (aux) std::copy(aux, aux + naux * kStates, auxv.begin() + (size_t)j * naux * kStates);
    }
    void* stv = nullptr;
    int rc = smccat_get_stream(c, &stv);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stv);
    // A Gibbs pass evaluates the drawn site under every class at every
    // iteration, the learned move under two. For the classes the particles
    // enter with, those values are evaluated beforehand for every site in one
    // batched pruning pass per class (the SIMT pruning kernels' evaluation
    // mode, into the partial workspaces the committed state does not use) and
    // read from a table: a pass changes assignments only, never a class.
    const int pfirst = *std::min_element(list.begin(), list.end());
    const int prange = *std::max_element(list.begin(), list.end()) - pfirst + 1;
    DeviceView view;
    bool use_table = false;
    if (site < 0 && device_view(c, pfirst, prange, &view) == SMCCAT_OK)
        use_table = view.pa.wt == nullptr && prune_variant_has_eval(d.R, view.fp32, view.variant);
    std::vector<PartHdr> ehdr;
    std::vector<NodeJob> enodes;
    std::vector<int32_t> emap;
    std::vector<uint8_t> esws;
    int kmax_list = 0;
    if (use_table) {
        ehdr.assign(prange, PartHdr{});
        enodes.assign((size_t)prange * d.NI, NodeJob{0, 0, 0, 0});
        emap.assign(prange, -1);
        esws.assign((size_t)prange * d.Kmax, 0);
        for (int q = 0; q < prange; ++q) {
            const Mirror& m = slot_of(c, pfirst + q).cur;
            std::copy(m.sws.begin(), m.sws.end(), &esws[(size_t)q * d.Kmax]);
        }
        for (int j = 0; j < n; ++j) {
            const int q = list[j] - pfirst;
            const Mirror& m = slot_of(c, list[j]).cur;
            emap[q] = j;
            kmax_list = std::max(kmax_list, m.K);
            PartHdr& h = ehdr[q];
            h.node_off = q * d.NI;
            h.node_cnt = (int)m.post.size();
            h.root = m.root;
            h.root_ws = 1 - m.clws[m.root];
            h.active = 1;
            h.num_classes = m.K;
            h.cls_only = -1;
            h.pinv = m.pinv;
            for (int r = 0; r < kMaxRates; ++r) h.rates[r] = m.rates[r];
            for (int x = 0; x < (int)m.post.size(); ++x) {
                const int nd = m.post[x], c1 = m.kids[2 * nd], c2 = m.kids[2 * nd + 1];
                int ws = 1 - m.clws[nd];
                if (c1 >= d.T) ws |= (1 - m.clws[c1]) << 1;
                if (c2 >= d.T) ws |= (1 - m.clws[c2]) << 2;
                ws |= m.pws[c1] << 3;
                ws |= m.pws[c2] << 4;
                enodes[(size_t)q * d.NI + x] = NodeJob{nd, c1, c2, ws};
            }
        }
    }
    // Device buffers for this call (inputs, outputs and kernel scratch).
    const int n_iter = parts[0].n_iter;
    if (n_iter >= (1 << 24)) return mfail(SMCCAT_EINVAL, "too many site iterations in one call");
    const size_t scratch = gibbs_scratch_doubles(d, n, Kcap, n_iter, nslots, true);
    size_t bytes = 0;
    auto carve = [&](size_t b) { const size_t o = bytes; bytes += (b + 255) & ~size_t(255); return o; };
    const size_t o_parts = carve(sizeof(GibbsPart) * n), o_tree = carve(tree.size() * sizeof(GibbsNode)),
                 o_branch = carve(branch.size() * 8), o_base = carve(base.size() * 8),
                 o_logits = carve(logits.size() * 8), o_assign = carve(assign.size() * 4),
                 o_counts = carve((size_t)n * ks * 4), o_kout = carve((size_t)n * 4),
                 o_aux = carve(auxv.size() * 8), o_w = carve((size_t)n * ks * 8),
                 o_status = carve(4), o_scr = carve(scratch * 8), o_acc = carve((size_t)n * 4),
                 o_prop = carve((size_t)n * 4);
    size_t o_ehdr = 0, o_enodes = 0, o_emap = 0, o_table = 0;
    // A table-mode Gibbs pass runs in rounds (classes opened into table slots
    // get their columns between rounds): per-particle resume state, the
    // transition-matrix jobs of every particle's branches and the per-round
    // evaluation classes.
    const bool rounds = use_table && learned_updates == 0;
    const int nbr = d.N - 1, nchunk = (nbr + kPmChunk - 1) / kPmChunk;
    size_t o_rit = 0, o_rk = 0, o_born = 0, o_pjobs = 0, o_pmjobs = 0, o_ekp = 0;
    std::vector<int32_t> rit(n, 0), rk(n), born(n, -1);
    std::vector<PJob> pjobs;
    // Table mode also lists each particle's drawn sites (the table is filled
    // for those only): row qrow[j] = list[j] - first of [prange][S].
    size_t o_qrow = 0, o_flags = 0, o_elist = 0, o_env = 0;
    std::vector<int32_t> qrow(n);
    for (int j = 0; j < n; ++j) qrow[j] = list[j] - pfirst;
    if (use_table) {
        o_ehdr = carve(sizeof(PartHdr) * ehdr.size());
        o_enodes = carve(sizeof(NodeJob) * enodes.size());
        o_emap = carve(4 * emap.size());
        o_table = carve((size_t)n * d.Kmax * d.S * 8);
        o_qrow = carve((size_t)n * 4);
        o_flags = carve((size_t)n * d.S);
        o_elist = carve((size_t)prange * d.S * 4);
        o_env = carve((size_t)prange * 4);
    }
    if (rounds) {
        o_rit = carve((size_t)n * 4);
        o_rk = carve((size_t)n * 4);
        o_born = carve((size_t)n * 4);
        o_pjobs = carve(sizeof(PJob) * (size_t)n * nbr);
        o_pmjobs = carve(sizeof(PmJob) * (size_t)n * nchunk);
        o_ekp = carve((size_t)prange * 4);
        pjobs.reserve((size_t)n * nbr);
        for (int j = 0; j < n; ++j) {
            const Mirror& m = slot_of(c, list[j]).cur;
            rk[j] = m.K;
            for (int x = 0; x < d.N; ++x)
                if (x != m.root) pjobs.push_back(PJob{list[j], x, m.pws[x], 0, m.branch[x]});
        }
    }
    char* dbuf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dbuf, bytes, st);
    if (e != cudaSuccess) return mfail(SMCCAT_ENOMEM, std::string("gibbs buffers: ") + cudaGetErrorString(e));
    std::vector<int32_t> counts((size_t)n * ks), kout(n);
    std::vector<double> wout((size_t)n * ks);
    int status = 0;
    auto up = [&](size_t o, const void* src, size_t b) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(dbuf + o, src, b, cudaMemcpyHostToDevice, st);
    };
    auto down = [&](void* dst, size_t o, size_t b) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst, dbuf + o, b, cudaMemcpyDeviceToHost, st);
    };
    up(o_parts, parts.data(), sizeof(GibbsPart) * n);
    up(o_tree, tree.data(), tree.size() * sizeof(GibbsNode));
    up(o_branch, branch.data(), branch.size() * 8);
    up(o_base, base.data(), base.size() * 8);
    up(o_logits, logits.data(), logits.size() * 8);
    up(o_assign, assign.data(), assign.size() * 4);
    up(o_aux, auxv.data(), auxv.size() * 8);
    if (e == cudaSuccess) e = cudaMemsetAsync(dbuf + o_status, 0, 4, st);
    if (rounds) {
        up(o_rit, rit.data(), (size_t)n * 4);
        up(o_rk, rk.data(), (size_t)n * 4);
        up(o_born, born.data(), (size_t)n * 4);
        up(o_pjobs, pjobs.data(), sizeof(PJob) * pjobs.size());
    }
    PruneArgs pa{};
    if (use_table) {
        up(o_ehdr, ehdr.data(), sizeof(PartHdr) * ehdr.size());
        up(o_enodes, enodes.data(), sizeof(NodeJob) * enodes.size());
        up(o_emap, emap.data(), 4 * emap.size());
        // The committed workspace bytes (a host-side reject since the last
        // refresh may have left the device array on the rejected ones).
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(const_cast<uint8_t*>(view.sws) + (size_t)pfirst * d.Kmax, esws.data(),
                                esws.size(), cudaMemcpyHostToDevice, st);
        pa = view.pa;
        pa.hdr = reinterpret_cast<const PartHdr*>(dbuf + o_ehdr);
        pa.nodes = reinterpret_cast<const NodeJob*>(dbuf + o_enodes);
        pa.eval_map = reinterpret_cast<const int32_t*>(dbuf + o_emap);
        pa.eval_out = reinterpret_cast<double*>(dbuf + o_table);
        pa.eval_perm = reinterpret_cast<const int32_t*>(dbuf + o_elist);
        pa.eval_nv = reinterpret_cast<const int32_t*>(dbuf + o_env);
        up(o_qrow, qrow.data(), (size_t)n * 4);
        if (e == cudaSuccess) e = cudaMemsetAsync(dbuf + o_elist, 0, (size_t)prange * d.S * 4, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(dbuf + o_env, 0, (size_t)prange * 4, st);
    }
    if (e == cudaSuccess) {
        GibbsArgs a{};
        a.d = d;
        a.count = n;
        a.Kcap = Kcap;
        a.temp = temperature;
        a.alpha = tuning_of(c).t.dpp_alpha;
        a.seed = seed;
        a.parts = reinterpret_cast<const GibbsPart*>(dbuf + o_parts);
        a.nodes = reinterpret_cast<const GibbsNode*>(dbuf + o_tree);
        a.nslots = nslots;
        a.branch = reinterpret_cast<const double*>(dbuf + o_branch);
        a.base = reinterpret_cast<const double*>(dbuf + o_base);
        a.logits = reinterpret_cast<double*>(dbuf + o_logits);
        a.assign = reinterpret_cast<int32_t*>(dbuf + o_assign);
        a.counts = reinterpret_cast<int32_t*>(dbuf + o_counts);
        a.kout = reinterpret_cast<int32_t*>(dbuf + o_kout);
        a.aux_in = aux ? reinterpret_cast<const double*>(dbuf + o_aux) : nullptr;
        a.weights_out = reinterpret_cast<double*>(dbuf + o_w);
        a.codes = codes_device(c);
        a.isinv = isinv_device(c);
        a.invchar = invchar_device(c);
        a.status = reinterpret_cast<int*>(dbuf + o_status);
        a.wait_limit = wait_limit_of(c);
        a.table = use_table ? reinterpret_cast<const double*>(dbuf + o_table) : nullptr;
        a.Kt = d.Kmax;
        double* scr = reinterpret_cast<double*>(dbuf + o_scr);
        if (rounds) {
            a.resume_it = reinterpret_cast<int32_t*>(dbuf + o_rit);
            a.resume_kcur = reinterpret_cast<int32_t*>(dbuf + o_rk);
            a.born = reinterpret_cast<int32_t*>(dbuf + o_born);
            a.eng_spec = const_cast<double*>(view.spec);
            a.eng_sws = view.sws;
        }
        if (use_table) {
            // The pass's drawn sites first (they do not depend on the chain),
            // then the table for those sites only, then the pass.
            e = learned_updates > 0 ? launch_draw_sites(a, n_iter, scr, st) : launch_gibbs_aux(a, n_iter, scr, st);
            if (e == cudaSuccess)
                e = launch_visited_sites(a, n_iter, scr, reinterpret_cast<const int32_t*>(dbuf + o_qrow),
                                         reinterpret_cast<uint8_t*>(dbuf + o_flags),
                                         reinterpret_cast<int32_t*>(dbuf + o_elist),
                                         reinterpret_cast<int32_t*>(dbuf + o_env), st);
            for (int k = 0; k < kmax_list && e == cudaSuccess; ++k) {
                pa.eval_k = k;
                e = launch_prune(pa, view.ntiles, view.variant, st);
            }
            pa.eval_k = -1;
        }
        if (e == cudaSuccess) {
            if (learned_updates > 0)
                e = launch_learned_move(a, n_iter, mlp, site_feat, reinterpret_cast<int32_t*>(dbuf + o_acc),
                                        reinterpret_cast<int32_t*>(dbuf + o_prop), scr, st);
            else if (use_table)
                e = launch_gibbs_resume(a, n_iter, scr, st);
            else
                e = launch_gibbs(a, n_iter, scr, st);
        }
        // Rounds: the classes the last round opened into table slots get
        // their transition matrices and table columns (the pruning kernels'
        // evaluation mode, one class per particle), then the particles resume.
        // Each round opens at least one class, so there are at most Kmax.
        std::vector<int32_t> ekp(prange);
        std::vector<PmJob> mj;
        PruneArgs pb = pa;
        pb.eval_k = -1;
        pb.eval_kp = reinterpret_cast<const int32_t*>(dbuf + o_ekp);
        for (int round = 0; rounds && round <= d.Kmax && e == cudaSuccess; ++round) {
            down(born.data(), o_born, (size_t)n * 4);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) break;
            mj.clear();
            std::fill(ekp.begin(), ekp.end(), -1);
            for (int j = 0; j < n; ++j) {
                if (born[j] < 0) continue;
                const int q = list[j] - pfirst;
                ekp[q] = born[j];
                for (int c0 = 0; c0 < nbr; c0 += kPmChunk)
                    mj.push_back(PmJob{q, born[j], j * nbr + c0, std::min(kPmChunk, nbr - c0)});
            }
            if (mj.empty()) break;
            up(o_pmjobs, mj.data(), sizeof(PmJob) * mj.size());
            up(o_ekp, ekp.data(), (size_t)prange * 4);
            if (e == cudaSuccess)
                e = launch_pmat(reinterpret_cast<const PmJob*>(dbuf + o_pmjobs), (int)mj.size(),
                                reinterpret_cast<const PJob*>(dbuf + o_pjobs), pa.hdr, pfirst, view.sws,
                                view.spec, view.Pm, view.fp32, d, st);
            if (e == cudaSuccess) e = launch_prune(pb, view.ntiles, view.variant, st);
            if (e == cudaSuccess) e = launch_gibbs_resume(a, n_iter, scr, st);
        }
    }
    down(assign.data(), o_assign, assign.size() * 4);
    down(counts.data(), o_counts, counts.size() * 4);
    down(kout.data(), o_kout, kout.size() * 4);
    down(logits.data(), o_logits, logits.size() * 8);
    down(wout.data(), o_w, wout.size() * 8);
    down(&status, o_status, 4);
    std::vector<int32_t> nacc(n, 0), nprop(n, 0);
    if (learned_updates > 0) {
        down(nacc.data(), o_acc, (size_t)n * 4);
        down(nprop.data(), o_prop, (size_t)n * 4);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(dbuf, st);
    if (e != cudaSuccess) return mfail(SMCCAT_ECUDA, std::string("gibbs: ") + cudaGetErrorString(e));
    // The table's pruning launches report through the engine's status word:
    // read and clear it here, so that it neither leaks into the next refresh
    // nor goes unreported.
    if (use_table) {
        int es = 0;
        e = cudaMemcpy(&es, view.status, sizeof(int), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && es) e = cudaMemset(view.status, 0, sizeof(int));
        if (e != cudaSuccess) return mfail(SMCCAT_ECUDA, std::string("gibbs: ") + cudaGetErrorString(e));
        if (es & 2) status |= 8;
    }
    if (lstats) {
        *lstats = smccat_learned_stats{};
        for (int j = 0; j < n; ++j) { lstats->proposed += nprop[j]; lstats->accepted += nacc[j]; }
    }
    if (status & 8) return mfail(SMCCAT_ETIMEOUT, "a bounded device wait gave up during the reassignment");
    if (site >= 0) {
        const int K = slot_of(c, list[0]).cur.K;
        for (int k = 0; k < K; ++k) weights_out[k] = wout[k];
        if (learned_updates == 0)
            for (int j = 0; j < naux; ++j) weights_out[K + j] = wout[K + j];
        return SMCCAT_OK;
    }
    if (status & 4) return mfail(SMCCAT_ENOMEM, "Gibbs reassignment ran out of class slots");
    // Compact the surviving classes and install the new assignments
    // (the reference erases empty classes as it goes, Particle.cpp:817-821).
    int first = *std::min_element(list.begin(), list.end());
    int last = *std::max_element(list.begin(), list.end());
    std::vector<uint8_t> act(last - first + 1, 0);
    smccat_gibbs_stats gs{};
    for (int j = 0; j < n; ++j) {
        const int p = list[j];
        const Slot& s = slot_of(c, p);
        std::vector<int> remap(ks, -1);
        int K = 0;
        for (int k = 0; k < kout[j]; ++k)
            if (counts[(size_t)j * ks + k] > 0) remap[k] = K++;
        if (K > d.Kmax) return mfail(SMCCAT_ENOMEM, "Gibbs reassignment exceeded max_classes");
        std::vector<double> nl((size_t)d.Kmax * kStates, 0.0);
        for (int k = 0; k < kout[j]; ++k)
            if (remap[k] >= 0)
                std::copy(&logits[((size_t)j * ks + k) * kStates], &logits[((size_t)j * ks + k + 1) * kStates],
                          nl.begin() + (size_t)remap[k] * kStates);
        std::vector<int32_t> na(d.S);
        for (int x = 0; x < d.S; ++x) na[x] = remap[assign[(size_t)j * d.S + x]];
        gs.classes_before += s.cur.K;
        gs.classes_after += K;
        gs.created += std::max(0, kout[j] - s.cur.K);
        const Mirror m = s.cur;  // copy: set_particles replaces the slot
        const int32_t kk = K;
        const double pv = m.pinv, sh = m.shape;
        rc = smccat_set_particles(c, p, 1, m.parent.data(), m.branch.data(), m.base.data(), &kk,
                                  nl.data(), na.data(), &pv, &sh);
        if (rc) return rc;
        act[p - first] = 1;
    }
    // refreshLikelihood(true) after the move (main.cpp:303-306).
    rc = refresh_internal(c, first, last - first + 1, SMCCAT_REFRESH_FULL, act.data());
    if (rc) return rc;
    gs.particles = n;
    if (stats) *stats = gs;
    return SMCCAT_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// Particles per reassignment call: the call's device buffers, dominated by the
// class table (Kmax x S doubles per particle), take at most half of the free
// device memory. A pass's random streams are keyed by particle, so splitting
// the particles into calls changes nothing in the result.
size_t reassign_chunk(const smccat_ctx* c) {
    if (reassign_group_of(c) > 0) return (size_t)reassign_group_of(c);
    const Dims& d = dims_of(c);
    size_t freeb = 0, total = 0;
    if (cudaSetDevice(device_of(c)) != cudaSuccess || cudaMemGetInfo(&freeb, &total) != cudaSuccess ||
        freeb == 0)
        return 1;
    const size_t per = (size_t)d.Kmax * d.S * 8 + (size_t)d.S * 64 +
                       (size_t)(d.Kmax + 64 + gibbs_aux()) * (kSpecStride + 2 * kStates) * 8 +
                       ((size_t)1 << 20);
    return std::max<size_t>(1, freeb / 2 / per);
}

}  // namespace

extern "C" {

int smccat_gibbs(smccat_ctx* c, int32_t first, int32_t count, const uint8_t* mask, double temperature,
                 uint64_t seed, smccat_gibbs_stats* stats) {
    NvtxRange range("smccat_gibbs");
    if (!c || first < 0 || count < 0) return mfail(SMCCAT_EINVAL, "bad argument");
    if (!(model_flags_of(c) & SMCCAT_MODEL_CAT)) return mfail(SMCCAT_EINVAL, "Gibbs reassignment needs SMCCAT_MODEL_CAT");
    std::vector<int> list;
    for (int i = 0; i < count; ++i) {
        if (mask && !mask[i]) continue;
        const Slot& s = slot_of(c, first + i);
        if (!s.loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
        if (s.pending) return mfail(SMCCAT_ESTATE, "particle has uncommitted edits");
        list.push_back(first + i);
    }
    const size_t chunk = reassign_chunk(c);
    smccat_gibbs_stats total{};
    for (size_t b = 0; b < list.size() || b == 0; b += chunk) {
        const std::vector<int> part(list.begin() + b, list.begin() + std::min(list.size(), b + chunk));
        smccat_gibbs_stats gs{};
        const int rc = run_gibbs(c, part, temperature, seed, -1, nullptr, nullptr, &gs);
        if (rc) return rc;
        total.particles += gs.particles;
        total.classes_before += gs.classes_before;
        total.classes_after += gs.classes_after;
        total.created += gs.created;
        if (list.empty()) break;
    }
    if (stats) *stats = total;
    return SMCCAT_OK;
}

int smccat_learned_move(smccat_ctx* c, int32_t first, int32_t count, const uint8_t* mask,
                        int32_t updates, double temperature, uint64_t seed,
                        smccat_learned_stats* stats) {
    NvtxRange range("smccat_learned_move");
    if (!c || first < 0 || count < 0 || updates < 1) return mfail(SMCCAT_EINVAL, "bad argument");
    if (!(model_flags_of(c) & SMCCAT_MODEL_CAT)) return mfail(SMCCAT_EINVAL, "the learned move needs SMCCAT_MODEL_CAT");
    if (dims_of(c).R > 2 * 4) return mfail(SMCCAT_EINVAL, "the learned move supports at most 8 rates");
    std::vector<int> list;
    for (int i = 0; i < count; ++i) {
        if (mask && !mask[i]) continue;
        const Slot& s = slot_of(c, first + i);
        if (!s.loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
        if (s.pending) return mfail(SMCCAT_ESTATE, "particle has uncommitted edits");
        list.push_back(first + i);
    }
    const size_t chunk = reassign_chunk(c);
    smccat_learned_stats total{};
    for (size_t b = 0; b < list.size() || b == 0; b += chunk) {
        const std::vector<int> part(list.begin() + b, list.begin() + std::min(list.size(), b + chunk));
        smccat_learned_stats ls{};
        const int rc = run_gibbs(c, part, temperature, seed, -1, nullptr, nullptr, nullptr, updates, &ls);
        if (rc) return rc;
        total.proposed += ls.proposed;
        total.accepted += ls.accepted;
        if (list.empty()) break;
    }
    if (stats) *stats = total;
    return SMCCAT_OK;
}

int smccat_learned_scores(smccat_ctx* c, int32_t p, int32_t site, double* out) {
    if (!c || !out || p < 0 || p >= particles_of(c)) return mfail(SMCCAT_EINVAL, "bad argument");
    if (!(model_flags_of(c) & SMCCAT_MODEL_CAT)) return mfail(SMCCAT_EINVAL, "the learned move needs SMCCAT_MODEL_CAT");
    if (dims_of(c).R > 2 * 4) return mfail(SMCCAT_EINVAL, "the learned move supports at most 8 rates");
    if (site < 0 || site >= dims_of(c).S) return mfail(SMCCAT_EINVAL, "site out of range");
    const Slot& s = slot_of(c, p);
    if (!s.loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
    return run_gibbs(c, {p}, 1.0, 0, site, nullptr, out, nullptr, 1, nullptr);
}

int smccat_gibbs_weights(smccat_ctx* c, int32_t p, int32_t site, const double* aux_logits,
                         double temperature, double* out) {
    if (!c || !aux_logits || !out || p < 0 || p >= particles_of(c)) return mfail(SMCCAT_EINVAL, "bad argument");
    const Slot& s = slot_of(c, p);
    if (!s.loaded) return mfail(SMCCAT_ESTATE, "particle has no state loaded");
    if (site < 0 || site >= dims_of(c).S) return mfail(SMCCAT_EINVAL, "site out of range");
    return run_gibbs(c, {p}, temperature, 0, site, aux_logits, out, nullptr);
}

int smccat_smc_step(smccat_ctx* c, int32_t first, int32_t count, double* raw_weights,
                    double target_ess, double last_temp, double* cur_temp, double* ess,
                    double* norm_weights) {
    NvtxRange range("smccat_smc_step");
    if (!c || !raw_weights || !cur_temp || !ess || !norm_weights || count < 1 || first < 0)
        return mfail(SMCCAT_EINVAL, "bad argument");
    void* stv = nullptr;
    int rc = smccat_get_stream(c, &stv);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stv);
    // Scratch: the weights, normalised weights and two scalars, taken from a
    // small device buffer owned by this call.
    double* dbuf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dbuf, sizeof(double) * (2 * (size_t)count + 2), st);
    if (e != cudaSuccess) return mfail(SMCCAT_ENOMEM, cudaGetErrorString(e));
    const double* dlnl = lnl_device(c);
    double out[2] = {0, 0};
    if (!rc) {
        e = cudaMemcpyAsync(dbuf, raw_weights, sizeof(double) * count, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            smc_step_kernel<<<1, kStepThreads, 0, st>>>(dbuf, dlnl + first, count, target_ess, last_temp,
                                                        dbuf + count, dbuf + 2 * count);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(raw_weights, dbuf, sizeof(double) * count, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(norm_weights, dbuf + count, sizeof(double) * count, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, dbuf + 2 * count, sizeof(out), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaFreeAsync(dbuf, st);
    if (rc) return rc;
    if (e != cudaSuccess) return mfail(SMCCAT_ECUDA, cudaGetErrorString(e));
    *cur_temp = out[0];
    *ess = out[1];
    return SMCCAT_OK;
}

}  // extern "C"
