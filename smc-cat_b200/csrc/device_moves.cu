// Tree moves on the device, a whole sweep captured as one CUDA graph.
//
// The host MCMC driver (mcmc.cu) proposes every move on host mirrors and packs
// each step's plan on the host. Here the reference's whole tree-move mixture,
// Particle::treeMove (Particle.cpp:677-701) -- NNI 0.1, adaptive NNI 0.3,
// SPR 0.1, branch scale 0.4, subtree scale 0.1 (Tree.cpp:553-812) -- runs for
// every particle of a range in lockstep with nothing on the host between steps:
//
//   dm_propose_kernel   one thread per particle: Philox draws, the edit of the
//                       flattened tree (branch lengths; or parent / child
//                       table entries, logged for undo), the dirty sets, the
//                       plan in post-order with the next workspaces, the
//                       tree-length prior change and the log Hastings ratio.
//                       Adaptive NNI weighs nodes by their split's posterior,
//                       looked up by binary search in a sorted split table;
//   pmat_kernel, prune_kernel, reduce_kernel
//                       the engine's kernels on that device-built plan, with
//                       launch shapes fixed by the range (empty job slots exit);
//   dm_mh_kernel        one thread per particle: Metropolis-Hastings on
//                       temperature * lnL + lnPrior + log Hastings (Mcmc.cpp:57-60);
//                       accept commits the new workspaces, reject restores the
//                       branch lengths or replays the table undo log (the dirty
//                       work sits in the other workspace, as on the host path).
//
// A sweep of B steps is B repetitions of this fixed sequence, captured into a
// CUDA graph and launched once. At the end the host mirrors take the final
// trees (children and post-order regenerated from the parent tables), branch
// lengths and committed workspaces back.
//
// smccat_mcmc_sweep runs the reference's whole Mcmc::operator() (Mcmc.cpp:25-73)
// this way: each particle's sequence of moves -- a draw from the registry of
// main.cpp:55-106 per iteration, repeated its count of times -- is drawn on
// the host first, and every step of the sweep then runs that step's move for
// each particle: the tree mixture above, or a parameter move
// (Particle.cpp:706-783): invarMove (beta proposal on pinv; only the root
// reduction reruns), shapeMove (rates re-discretised on the device, every
// matrix and partial rebuilt), stationaryMove (one logit of one class shifted,
// that class re-decomposed, every matrix and partial rebuilt) or
// rateMatrixMove (one exchangeability, or all of them through the Cholesky
// factor; every class re-decomposed, everything rebuilt). dm_spec_kernel
// re-decomposes the classes a step touches; the MH kernel restores the
// parameters (and the spectral workspaces) of rejected proposals.
//
// Partials invalidated by a topology move: the moved node and its ancestors,
// and for SPR also the old parent's ancestors. (The reference's SPRMove marks
// only the new path, Tree.cpp:803-807, leaving the old parent's partials stale
// until the next full refresh; the host path and this one mark both.)
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <math.h>

#include <algorithm>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "gamma_math.cuh"
#include "kernels.h"
#include "smccat.h"
#include "spectral.cuh"

namespace smccat {
namespace {

constexpr int kDmThreads = 64;  // one thread per particle (generator set-up)
constexpr int kDmWarps = 4;     // particles per proposal / MH block (one warp each)
constexpr int kUndo = 8;  // table edits of one move (SPR: 6, NNI: 4)

// Move kinds, numbered like SMCCAT_MOVE_*.
constexpr int kAnni = 0, kNni = 1, kSpr = 2, kBranch = 3, kSubtree = 4, kInvar = 5, kShape = 6,
              kStationary = 7, kRateSingle = 8, kRateFull = 9;
constexpr int kKinds = 10;
// Registry families, numbered like SMCCAT_FAMILY_*; -1 in a schedule = idle.
constexpr int kFamTree = 0, kFamStationary = 1, kFamShape = 2, kFamInvar = 3, kFamRate = 4;

struct DmArgs {
    Dims d;
    int first, count, nchunk;
    int32_t* parent;     // [count][N]
    int32_t* kids;       // [count][2N]
    int32_t* ulog;       // [count][2 kUndo] (table index, old value); index >= N is kids[index - N]
    int32_t* nlog;       // [count]
    double* branch;      // [count][N]
    uint8_t* clws;       // [count][N] committed partial workspace of each node
    uint8_t* pws;        // [count][N] committed transition-matrix workspace
    uint8_t* cur_clws;   // [count][N] workspaces of this step's proposal
    uint8_t* cur_pws;
    uint8_t* dirty;      // [count][N] bit 0: P, bit 1: partial, bit 2: on the first path
    int32_t* undo_node;  // [count][N] scaled nodes, walk order
    double* undo_len;    // [count][N] their previous lengths
    int32_t* nundo;      // [count]
    int32_t* kind;       // [count] SMCCAT_MOVE_* of this step's move
    double* extra;       // [count] lnPrior change + log Hastings ratio
    const uint64_t* skeys;  // [nsplit][2] canonical splits, sorted
    const double* sprob;    // [nsplit]
    int nsplit;
    bool use_splits;     // T <= 128: splits fit two words
    const PartHdr* hdr0; // [count] root, classes, pinv, rates
    PartHdr* hdr;        // [count] this step's
    NodeJob* nodes;      // [count][NI]
    PJob* pjobs;         // [count][N]
    PmJob* mjobs;        // [count][Kmax][nchunk]
    curandStatePhilox4_32_10_t* rng;  // [count]
    double* lnl;         // engine arrays, [max_particles]
    double* lnl_old;
    unsigned long long* stats;  // proposed / accepted per move kind (2 x kKinds)
    double scale_delta, subtree_delta, anni_eps, temp;
    // Whole-registry sweeps (sched != null); tree-only sweeps leave these null.
    const int8_t* sched;    // [count][nsched] family of each step, -1 = idle
    int nsched, step;
    PartHdr* hdr0w;         // hdr0, writable: accepted pinv / rates are committed here
    double* base;           // [count][kBase] exchangeabilities
    double* logits;         // [count][Kmax][kStates]
    double* shape;          // [count]
    double* shape_new;      // [count] this step's proposal
    double* undo_base;      // [count][kBase] exchangeabilities before a rate-matrix proposal
    double* undo_logit;     // [count] the shifted logit's previous value
    int32_t* undo_k;        // [count] class and state of the shifted logit (k * kStates + i)
    uint8_t* sws;           // engine's spectral workspace array [max_particles][Kmax]
    const double* spec;     // engine's spectral records
    uint8_t* spec_flip;     // [count][Kmax] classes this step re-decomposes
    const double* chol;     // [kBase][kBase] lower-triangular proposal factor
    double shape_delta, stationary_delta, rate_delta, invar_alpha;
    int lg, R;
};

__global__ void dm_init_kernel(curandStatePhilox4_32_10_t* rng, int count, int first, unsigned long long seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) curand_init(seed, (unsigned long long)(first + i), 0ull, &rng[i]);
}

// Posterior of a canonical split, or -1 when the table does not hold it.
__device__ double split_lookup(const DmArgs& a, uint64_t w0, uint64_t w1) {
    int lo = 0, hi = a.nsplit;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const uint64_t k0 = a.skeys[2 * mid], k1 = a.skeys[2 * mid + 1];
        if (k0 < w0 || (k0 == w0 && k1 < w1)) lo = mid + 1;
        else hi = mid;
    }
    if (lo < a.nsplit && a.skeys[2 * lo] == w0 && a.skeys[2 * lo + 1] == w1) return a.sprob[lo];
    return -1.0;
}

// Adaptive-NNI weight of a node whose clade is (c0, c1) (Tree.cpp:676-694):
// epsilon + 1 - posterior of its split, epsilon + 1 when the split is absent
// or trivial. Splits are canonicalised to contain taxon 0.
__device__ double anni_weight(const DmArgs& a, uint64_t c0, uint64_t c1) {
    double v = a.anni_eps;
    if (!a.use_splits) return v + 1.0;
    const int T = a.d.T;
    const uint64_t f0 = T >= 64 ? ~0ull : (1ull << T) - 1;
    const uint64_t f1 = T <= 64 ? 0ull : (T >= 128 ? ~0ull : (1ull << (T - 64)) - 1);
    if (!(c0 & 1ull)) { c0 = ~c0 & f0; c1 = ~c1 & f1; }
    const int cnt = __popcll(c0) + __popcll(c1);
    const double pr = (cnt == 1 || cnt == T - 1) ? -1.0 : split_lookup(a, c0, c1);
    return v + (pr >= 0.0 ? 1.0 - pr : 1.0);
}

// Shared-memory bytes one particle's proposal needs (per warp): the tree
// tables, and the normal draws of a rate-matrix proposal.
__host__ __device__ inline size_t dm_warp_bytes(int N) {
    return ((size_t)N * (8 + 16 + 8 + 4 * 6 + 3) + 8 * kBase + 15) & ~size_t(15);
}

__device__ __forceinline__ double dm_unif(curandStatePhilox4_32_10_t* rs) {
    return 1.0 - curand_uniform_double(rs);  // [0, 1)
}

// Gamma(a, 1) variate: Marsaglia and Tsang's squeeze method (a >= 1; for
// a < 1 the Gamma(a + 1) draw times U^(1/a)). The rejection loop is bounded;
// its acceptance rate is above 95%.
__device__ double dm_gamma(curandStatePhilox4_32_10_t* rs, double a) {
    double boost = 1.0;
    if (a < 1.0) {
        boost = pow(dm_unif(rs) + 1e-300, 1.0 / a);
        a += 1.0;
    }
    const double dd = a - 1.0 / 3.0, cc = 1.0 / sqrt(9.0 * dd);
    for (int it = 0; it < 1000; ++it) {
        const double x = curand_normal_double(rs);
        double v = 1.0 + cc * x;
        if (v <= 0.0) continue;
        v = v * v * v;
        const double u = dm_unif(rs);
        if (u < 1.0 - 0.0331 * x * x * x * x) return dd * v * boost;
        if (log(u + 1e-300) < 0.5 * x * x + dd * (1.0 - v + log(v))) return dd * v * boost;
    }
    return dd * boost;
}

__device__ __forceinline__ double dm_beta_lpdf(double x, double a, double b) {
    return lgamma(a + b) - lgamma(a) - lgamma(b) + (a - 1.0) * log(x) + (b - 1.0) * log1p(-x);
}

__device__ __forceinline__ double dm_gamma_lpdf(double x, double shape, double scale) {
    return (shape - 1.0) * log(x) - x / scale - lgamma(shape) - shape * log(scale);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One warp per particle. The particle's tables are staged in shared memory;
// lane 0 makes the move (the tree walks are sequential), the lanes share the
// O(N) passes, the adaptive-NNI split lookups and the plan writes.
__global__ void __launch_bounds__(kDmWarps * 32) dm_propose_kernel(DmArgs a) {
    extern __shared__ __align__(16) unsigned char dm_smem[];
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= a.count) return;  // whole warps leave together
    const Dims& d = a.d;
    const int N = d.N, T = d.T, NI = d.NI;
    const int family = a.sched ? a.sched[(size_t)i * a.nsched + a.step] : kFamTree;
    if (a.spec_flip)
        for (int k = lane; k < d.Kmax; k += 32) a.spec_flip[(size_t)i * d.Kmax + k] = 0;
    if (family < 0) {  // this particle's sweep is over: nothing to evaluate
        PmJob* mj = a.mjobs + (size_t)i * d.Kmax * a.nchunk;
        for (int e = lane; e < d.Kmax * a.nchunk; e += 32) mj[e] = PmJob{i, 0, 0, 0};
        if (lane == 0) {
            PartHdr h = a.hdr0[i];
            h.node_off = i * NI;
            h.node_cnt = 0;
            h.active = 0;
            a.hdr[i] = h;
            a.kind[i] = -1;
            a.nlog[i] = 0;
            a.nundo[i] = 0;
        }
        return;
    }
    unsigned char* base = dm_smem + (size_t)(threadIdx.x >> 5) * dm_warp_bytes(N);
    double* br = reinterpret_cast<double*>(base);     // N
    uint64_t* cl = reinterpret_cast<uint64_t*>(br + N);  // 2N
    double* wn = reinterpret_cast<double*>(cl + 2 * N);  // N
    int32_t* par = reinterpret_cast<int32_t*>(wn + N);   // N
    int32_t* kids = par + N;                             // 2N
    int32_t* stk = kids + 2 * N;                         // N
    int32_t* ord = stk + N;                              // N
    int32_t* un = ord + N;                               // N
    uint8_t* dirty = reinterpret_cast<uint8_t*>(un + N); // N
    uint8_t* cc = dirty + N;                             // N
    uint8_t* cp = cc + N;                                // N
    double* zz = reinterpret_cast<double*>(base + (((size_t)N * (8 + 16 + 8 + 4 * 6 + 3) + 7) & ~size_t(7)));  // kBase
    int32_t* gpar = a.parent + (size_t)i * N;
    int32_t* gkids = a.kids + (size_t)i * 2 * N;
    double* gbr = a.branch + (size_t)i * N;
    const PartHdr h0 = a.hdr0[i];
    const int root = h0.root;

    double l0 = 0.0;
    for (int n = lane; n < N; n += 32) {
        par[n] = gpar[n];
        kids[2 * n] = gkids[2 * n];
        kids[2 * n + 1] = gkids[2 * n + 1];
        br[n] = gbr[n];
        dirty[n] = 0;
        l0 += br[n];
    }
    const double L0 = warp_sum(l0);
    __syncwarp();

    curandStatePhilox4_32_10_t rs;
    int kind = 0;
    if (lane == 0) {
        rs = a.rng[i];
        if (family == kFamTree) {
            const double u = 1.0 - curand_uniform_double(&rs);  // Particle.cpp:680-701
            kind = u < 0.1 ? kNni : u < 0.4 ? kAnni : u < 0.5 ? kSpr : u < 0.9 ? kBranch : kSubtree;
        } else if (family == kFamStationary) {
            kind = kStationary;
        } else if (family == kFamShape) {
            kind = kShape;
        } else if (family == kFamInvar) {
            kind = kInvar;
        } else {  // Particle.cpp:706-732: the full (Cholesky) proposal a quarter of the time
            kind = dm_unif(&rs) < 0.25 ? kRateFull : kRateSingle;
        }
        if (kind == kAnni && a.use_splits) {  // clades bottom-up over a pre-order walk
            int top = 0, cnt = 0;
            stk[top++] = root;
            while (top > 0 && cnt < N) {
                const int n = stk[--top];
                ord[cnt++] = n;
                if (n >= T && top + 2 <= N) { stk[top++] = kids[2 * n]; stk[top++] = kids[2 * n + 1]; }
            }
            for (int q = cnt - 1; q >= 0; --q) {
                const int n = ord[q];
                if (n < T) {
                    cl[2 * n] = n < 64 ? 1ull << n : 0ull;
                    cl[2 * n + 1] = n >= 64 ? 1ull << (n - 64) : 0ull;
                } else {
                    const int k1 = kids[2 * n], k2 = kids[2 * n + 1];
                    cl[2 * n] = cl[2 * k1] | cl[2 * k2];
                    cl[2 * n + 1] = cl[2 * k1 + 1] | cl[2 * k2 + 1];
                }
            }
        }
    }
    kind = __shfl_sync(0xffffffffu, kind, 0);
    __syncwarp();
    if (kind == kAnni) {  // node weights, the lookups spread over the lanes
        for (int n = T + lane; n < N; n += 32)
            if (n != root) wn[n] = a.use_splits ? anni_weight(a, cl[2 * n], cl[2 * n + 1]) : a.anni_eps + 1.0;
        __syncwarp();
    }

    int nord = 0, nch = 0, local_k = -1;
    unsigned long long rate_key = 0;
    double hastings = 0.0, dprior = 0.0;
    double new_pinv = a.hdr0[i].pinv;
    double new_rates[kMaxRates];
    for (int r = 0; r < kMaxRates; ++r) new_rates[r] = a.hdr0[i].rates[r];
    if (lane == 0) {
        int32_t* lg = a.ulog + (size_t)i * 2 * kUndo;
        double* gul = a.undo_len + (size_t)i * N;
        auto unif = [&]() { return 1.0 - curand_uniform_double(&rs); };  // [0, 1)
        auto uniform_node = [&]() { return min(N - 1, (int)(unif() * N)); };
        // A uniform node other than the root (internal only if `internal`);
        // after 64 misses the first admissible id (probability below 1e-12).
        auto pick = [&](bool internal) {
            int x = root;
            for (int t = 0; t < 64 && (x == root || (internal && x < T)); ++t) x = uniform_node();
            if (x == root || (internal && x < T))
                for (int n = internal ? T : 0; n < N; ++n)
                    if (n != root) { x = n; break; }
            return x;
        };
        auto in_subtree = [&](int y, int r) {  // Tree.hpp:29-34
            for (int g = 0; y >= 0 && g <= N; y = par[y], ++g)
                if (y == r) return true;
            return false;
        };
        int nlog = 0;
        auto set_par = [&](int n, int v) {
            lg[2 * nlog] = n; lg[2 * nlog + 1] = par[n]; ++nlog;
            par[n] = v;
        };
        auto set_kid = [&](int k, int v) {
            lg[2 * nlog] = N + k; lg[2 * nlog + 1] = kids[k]; ++nlog;
            kids[k] = v;
        };
        // Dirty partials on two root paths, recorded children first: the path
        // of `b` up to where it meets the path of `pa`, then the path of `pa`.
        auto mark_paths = [&](int pa, int b) {
            for (int y = pa, g = 0; y >= 0 && g < N; y = par[y], ++g) dirty[y] |= 2 | 4;
            for (int y = b, g = 0; y >= 0 && g < N && !(dirty[y] & 4); y = par[y], ++g) {
                dirty[y] |= 2;
                if (nord < N) ord[nord++] = y;
            }
            for (int y = pa, g = 0; y >= 0 && g < N; y = par[y], ++g)
                if (nord < N) ord[nord++] = y;
        };

        if (kind == kNni || kind == kAnni) {
            // NNIMove / adaptiveNNIMove (Tree.cpp:625-766): one child n1 of x
            // trades places with x's sibling n2; branch lengths stay with
            // their nodes, so no transition matrix changes.
            int x;
            double sel = 0.0, tot = 0.0;
            if (kind == kNni) {
                x = pick(true);
            } else {
                for (int n = T; n < N; ++n)
                    if (n != root) tot += wn[n];
                const double r = unif();
                double cum = 0.0;
                x = -1;
                for (int n = T; n < N; ++n) {
                    if (n == root) continue;
                    cum += wn[n] / tot;
                    x = n;
                    if (r <= cum) break;
                }
                sel = wn[x] / tot;
            }
            const int pa = par[x];
            const int s1 = min(1, (int)(unif() * 2));
            const int n1 = kids[2 * x + s1];
            const int s2 = kids[2 * pa] == x ? 1 : 0;
            const int n2 = kids[2 * pa + s2];
            set_par(n1, pa);
            set_par(n2, x);
            set_kid(2 * pa + s2, n1);
            set_kid(2 * x + s1, n2);
            if (kind == kAnni) {
                // Only x's clade changes: it loses n1's taxa and gains n2's.
                double w2 = a.anni_eps + 1.0;
                if (a.use_splits)
                    w2 = anni_weight(a, (cl[2 * x] & ~cl[2 * n1]) | cl[2 * n2],
                                     (cl[2 * x + 1] & ~cl[2 * n1 + 1]) | cl[2 * n2 + 1]);
                double tot2 = 0.0;
                for (int n = T; n < N; ++n)
                    if (n != root) tot2 += n == x ? w2 : wn[n];
                hastings = log(w2 / tot2) - log(sel);
            }
            mark_paths(pa, x);
        } else if (kind == kSpr) {
            // SPRMove (Tree.cpp:768-812): prune the subtree of x's child (x
            // comes with it, x's other child sib takes x's place) and regraft
            // x on the branch above a node an outside it.
            const int x = pick(true);
            const int s1 = min(1, (int)(unif() * 2));
            const int sib = kids[2 * x + 1 - s1];
            int an = -1;
            for (int t = 0; t < 256 && an < 0; ++t) {
                const int c = uniform_node();
                if (c != root && !in_subtree(c, x)) an = c;
            }
            if (an < 0)  // x's parent or sibling always qualifies
                for (int n = 0; n < N && an < 0; ++n)
                    if (n != root && !in_subtree(n, x)) an = n;
            const int gp = par[x];
            set_kid(2 * gp + (kids[2 * gp] == x ? 0 : 1), sib);
            set_par(sib, gp);
            const int ap = par[an];
            set_kid(2 * ap + (kids[2 * ap] == an ? 0 : 1), x);
            set_par(x, ap);
            set_kid(2 * x + 1 - s1, an);
            set_par(an, x);
            mark_paths(gp, x);
        } else if (kind >= kInvar) {
            // Parameter moves (Particle.cpp:706-783).
            const int K = h0.num_classes;
            uint8_t* flip = a.spec_flip + (size_t)i * d.Kmax;
            double* lgt = a.logits + (size_t)i * d.Kmax * kStates;
            double* bs = a.base + (size_t)i * kBase;
            if (kind == kInvar) {
                // invarMove: beta proposal centred on the current pinv.
                const double al = a.invar_alpha, cur = h0.pinv;
                const double aa = al + 1.0, bb = al / cur - aa + 2.0;
                const double x = dm_gamma(&rs, aa), y = dm_gamma(&rs, bb);
                double nv = x / (x + y);
                nv = fmin(fmax(nv, 1e-300), 1.0 - 1e-16);
                const double b2 = al / nv - aa + 2.0;
                hastings = dm_beta_lpdf(cur, aa, b2) - dm_beta_lpdf(nv, aa, bb);
                new_pinv = nv;
            } else {
                if (kind == kShape) {
                    // shapeMove: multiplicative proposal, rates re-discretised.
                    const double sc = exp(a.shape_delta * (dm_unif(&rs) - 0.5));
                    const double old = a.shape[i], nw = old * sc;
                    a.shape_new[i] = nw;
                    gm_discretize_gamma(nw, a.R, new_rates);
                    hastings = log(sc);
                    dprior = dm_gamma_lpdf(nw, 3.0, 2.0) - dm_gamma_lpdf(old, 3.0, 2.0);
                } else if (kind == kStationary) {
                    // stationaryMove, with the shift applied to the class's logit.
                    const int k = min(K - 1, (int)(dm_unif(&rs) * K));
                    const int st = min(kStates - 1, (int)(dm_unif(&rs) * kStates));
                    const double old = lgt[(size_t)k * kStates + st];
                    const double nw = old + curand_normal_double(&rs) * a.stationary_delta;
                    lgt[(size_t)k * kStates + st] = nw;
                    a.undo_k[i] = k * kStates + st;
                    a.undo_logit[i] = old;
                    dprior = -0.5 * (nw * nw - old * old);
                    flip[k] = 1;
                    local_k = k;
                } else {
                    // rateMatrixMove: one entry, or all through the Cholesky
                    // factor (the product runs over the lanes below).
                    double* ub = a.undo_base + (size_t)i * kBase;
                    for (int x = 0; x < kBase; ++x) ub[x] = bs[x];
                    if (kind == kRateFull) {
                        // The 190 N(0, 1) draws come from a stream of their own,
                        // keyed from this one, spread over the lanes below.
                        rate_key = ((unsigned long long)curand(&rs) << 32) | curand(&rs);
                    } else {
                        const int x = min(kBase - 1, (int)(kBase * dm_unif(&rs)));
                        const double old = bs[x];
                        const double nw = old + curand_normal_double(&rs) * a.rate_delta;
                        bs[x] = nw;
                        if (!a.lg) dprior = -0.5 * (nw * nw - old * old);
                    }
                    for (int k = 0; k < K; ++k) flip[k] = 1;
                }
                // Every transition matrix and partial is rebuilt: all non-root
                // nodes' matrices, all internal nodes in a post-order
                // (a reversed pre-order: each node after its children). A
                // stationary move rebuilds its class alone, class-locally: the
                // node workspaces stay (no dirty flags), that class's byte of
                // the spectral-workspace array flips its own workspaces.
                int top = 0, cnt = 0;
                stk[top++] = root;
                while (top > 0 && cnt < N) {
                    const int n = stk[--top];
                    un[cnt++] = n;
                    if (n >= T && top + 2 <= N) { stk[top++] = kids[2 * n]; stk[top++] = kids[2 * n + 1]; }
                }
                for (int q = cnt - 1; q >= 0; --q)
                    if (un[q] >= T && nord < N) ord[nord++] = un[q];
                nch = 0;
                for (int n = 0; n < N; ++n) {
                    dirty[n] = kind == kStationary ? 0 : (n != root ? 1 : 0) | (n >= T ? 2 : 0);
                    if (n != root) un[nch++] = n;
                }
            }
        } else {
            // scaleBranchMove / scaleSubtreeMove (Tree.cpp:553-612): x's
            // branch, or every branch of x's subtree (walk order: pre-order
            // with the second child first; reversed it is a post-order).
            const bool subtree = kind == kSubtree;
            const int x = pick(false);
            const double sc = exp((subtree ? a.subtree_delta : a.scale_delta) * (unif() - 0.5));
            int top = 0;
            stk[top++] = x;
            while (top > 0) {  // every node is pushed once: top <= N, nch <= N
                const int n = stk[--top];
                un[nch] = n;
                gul[nch] = br[n];
                ++nch;
                br[n] *= sc;
                dirty[n] |= 1;
                if (subtree && n >= T) {
                    stk[top++] = kids[2 * n];
                    stk[top++] = kids[2 * n + 1];
                }
            }
            if (subtree)
                for (int q = nch - 1; q >= 0; --q)
                    if (un[q] >= T) {
                        dirty[un[q]] |= 2;
                        if (nord < N) ord[nord++] = un[q];
                    }
            for (int y = par[x], g = 0; y >= 0 && g < N; y = par[y], ++g) {
                dirty[y] |= 2;
                if (nord < N) ord[nord++] = y;
            }
            hastings = nch * log(sc);
        }
        a.nlog[i] = nlog;
        a.nundo[i] = (kind == kBranch || kind == kSubtree) ? nch : 0;
        a.kind[i] = kind;
        a.rng[i] = rs;
    }
    nord = __shfl_sync(0xffffffffu, nord, 0);
    nch = __shfl_sync(0xffffffffu, nch, 0);
    local_k = __shfl_sync(0xffffffffu, local_k, 0);
    __syncwarp();
    if (kind == kRateFull) {
        // z ~ N(0, I) (lane l draws z[l], z[l + 32], ... from subsequence l of
        // the move's stream), then base += L z over the lanes (L lower
        // triangular), and the N(0, 1) prior change of the exchangeabilities.
        rate_key = __shfl_sync(0xffffffffu, rate_key, 0);
        curandStatePhilox4_32_10_t zr;
        curand_init(rate_key, (unsigned long long)lane, 0ull, &zr);
        for (int x = lane; x < kBase; x += 32) zz[x] = curand_normal_double(&zr);
        __syncwarp();
        double* bs = a.base + (size_t)i * kBase;
        double dp = 0.0;
        for (int x = lane; x < kBase; x += 32) {
            double acc = 0.0;
            for (int j = 0; j <= x; ++j) acc = fma(a.chol[(size_t)x * kBase + j], zz[j], acc);
            const double old = bs[x], nw = old + acc;
            bs[x] = nw;
            dp += -0.5 * (nw * nw - old * old);
        }
        dp = warp_sum(dp);
        if (lane == 0 && !a.lg) dprior = dp;
    }
    if (kind >= kStationary) {  // the re-decomposed classes take their other spectral workspace
        const uint8_t* flip = a.spec_flip + (size_t)i * d.Kmax;
        const uint8_t fl = kind == kStationary ? (kSwsSpec | kSwsCl | kSwsP) : kSwsSpec;
        for (int k = lane; k < d.Kmax; k += 32)
            if (flip[k]) a.sws[(size_t)(a.first + i) * d.Kmax + k] ^= fl;
    }
    __syncwarp();

    // Next workspaces, the tree and the dirty flags back to global memory.
    const uint8_t* kc = a.clws + (size_t)i * N;
    const uint8_t* kp = a.pws + (size_t)i * N;
    uint8_t* gcc = a.cur_clws + (size_t)i * N;
    uint8_t* gcp = a.cur_pws + (size_t)i * N;
    uint8_t* gdirty = a.dirty + (size_t)i * N;
    double l1 = 0.0;
    for (int n = lane; n < N; n += 32) {
        const uint8_t f = dirty[n];
        cc[n] = (f & 2) ? 1 - kc[n] : kc[n];
        cp[n] = (f & 1) ? 1 - kp[n] : kp[n];
        gcc[n] = cc[n];
        gcp[n] = cp[n];
        gdirty[n] = f;
        gpar[n] = par[n];
        gkids[2 * n] = kids[2 * n];
        gkids[2 * n + 1] = kids[2 * n + 1];
        gbr[n] = br[n];
        l1 += br[n];
    }
    const double L1 = warp_sum(l1);
    __syncwarp();
    // Plan: the recorded dirty internal nodes, each after its dirty children.
    NodeJob* nj = a.nodes + (size_t)i * NI;
    const int nn = min(nord, NI);
    for (int q = lane; q < nn; q += 32) {
        const int n = ord[q];
        const int c1 = kids[2 * n], c2 = kids[2 * n + 1];
        int ws = cc[n];
        if (c1 >= T) ws |= cc[c1] << 1;
        if (c2 >= T) ws |= cc[c2] << 2;
        ws |= cp[c1] << 3;
        ws |= cp[c2] << 4;
        nj[q] = NodeJob{n, c1, c2, ws};
    }
    PJob* pj = a.pjobs + (size_t)i * N;
    int32_t* gun = a.undo_node + (size_t)i * N;
    for (int q = lane; q < nch; q += 32) {
        pj[q] = PJob{a.first + i, un[q], cp[un[q]], 0, br[un[q]]};
        gun[q] = un[q];
    }
    PmJob* mj = a.mjobs + (size_t)i * d.Kmax * a.nchunk;
    for (int e = lane; e < d.Kmax * a.nchunk; e += 32) {
        const int k = e / a.nchunk, c = e - k * a.nchunk;
        const bool cls_on = local_k >= 0 ? k == local_k : k < h0.num_classes;
        const int nj_k = cls_on ? max(0, min(kPmChunk, nch - kPmChunk * c)) : 0;
        mj[e] = PmJob{i, k, i * N + kPmChunk * c, nj_k};
    }
    if (lane == 0) {
        PartHdr h = h0;
        h.node_off = i * NI;
        h.node_cnt = nn;
        h.root_ws = cc[root];
        h.active = 1;
        h.cls_only = local_k;
        h.pinv = new_pinv;
        for (int r = 0; r < kMaxRates; ++r) h.rates[r] = new_rates[r];
        a.hdr[i] = h;
        // Tree-length prior Gamma(2T-2, scale 1/10) (Particle.cpp:484-517),
        // the parameter priors' change and the Hastings ratio.
        a.extra[i] = (N - 2) * (log(L1) - log(L0)) - (L1 - L0) / 0.1 + dprior + hastings;
    }
}

// One warp per (particle, class) slot: re-decompose the classes a step's
// proposal marked, into the spectral workspace the proposal switched them to,
// starting from the committed record in the other workspace (the same class
// before the proposal's small change).
__global__ void __launch_bounds__(32) dm_spec_kernel(DmArgs a) {
    const int i = blockIdx.x / a.d.Kmax, k = blockIdx.x - i * a.d.Kmax;
    if (!a.spec_flip[(size_t)i * a.d.Kmax + k]) return;
    const size_t pk = (size_t)(a.first + i) * a.d.Kmax + k;
    const int half = a.sws[pk] & kSwsSpec;
    double* spec = const_cast<double*>(a.spec);
    __shared__ SpecWork w;
    spectral_decompose_warp_warm(a.base + (size_t)i * kBase, a.logits + ((size_t)i * a.d.Kmax + k) * kStates,
                                 spec + (pk * 2 + (half ^ 1)) * kSpecStride, spec + (pk * 2 + half) * kSpecStride,
                                 w);
}

// One warp per particle: lane 0 draws the decision, the lanes commit the
// workspaces or restore the branch lengths; lane 0 replays the table log.
__global__ void __launch_bounds__(kDmWarps * 32) dm_mh_kernel(DmArgs a) {
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= a.count) return;  // whole warps leave together
    const int N = a.d.N, p = a.first + i;
    const int kind = a.kind[i];
    if (kind < 0) return;  // idle this step
    int ok = 0;
    if (lane == 0) {
        curandStatePhilox4_32_10_t rs = a.rng[i];
        const double ratio = a.temp * (a.lnl[p] - a.lnl_old[p]) + a.extra[i];
        ok = log(curand_uniform_double(&rs)) <= ratio;  // NaN ratios reject
        a.rng[i] = rs;
        atomicAdd(&a.stats[2 * kind], 1ull);
        if (ok) {
            a.lnl_old[p] = a.lnl[p];
            atomicAdd(&a.stats[2 * kind + 1], 1ull);
        } else {
            a.lnl[p] = a.lnl_old[p];
            int32_t* par = a.parent + (size_t)i * N;
            int32_t* kids = a.kids + (size_t)i * 2 * N;
            const int32_t* lg = a.ulog + (size_t)i * 2 * kUndo;
            for (int q = a.nlog[i] - 1; q >= 0; --q) {
                const int x = lg[2 * q];
                if (x < N) par[x] = lg[2 * q + 1];
                else kids[x - N] = lg[2 * q + 1];
            }
        }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (ok) {
        const uint8_t* dirty = a.dirty + (size_t)i * N;
        uint8_t* kc = a.clws + (size_t)i * N;
        uint8_t* kp = a.pws + (size_t)i * N;
        for (int n = lane; n < N; n += 32) {
            const uint8_t f = dirty[n];
            if (f & 2) kc[n] = a.cur_clws[(size_t)i * N + n];
            if (f & 1) kp[n] = a.cur_pws[(size_t)i * N + n];
        }
        // Accepted parameters: pinv and rates become the committed header;
        // exchangeabilities, logits and spectral workspaces already are.
        if (lane == 0 && (kind == kInvar || kind == kShape)) {
            a.hdr0w[i].pinv = a.hdr[i].pinv;
            for (int r = 0; r < kMaxRates; ++r) a.hdr0w[i].rates[r] = a.hdr[i].rates[r];
            if (kind == kShape) a.shape[i] = a.shape_new[i];
        }
    } else {
        // The scaled nodes are distinct: their lengths restore in any order.
        double* br = a.branch + (size_t)i * N;
        const int32_t* un = a.undo_node + (size_t)i * N;
        const double* ul = a.undo_len + (size_t)i * N;
        for (int q = lane; q < a.nundo[i]; q += 32) br[un[q]] = ul[q];
        // Rejected parameters: previous exchangeabilities or logit, and the
        // re-decomposed classes back on their previous spectral workspace.
        if (kind == kRateSingle || kind == kRateFull)
            for (int x = lane; x < kBase; x += 32) a.base[(size_t)i * kBase + x] = a.undo_base[(size_t)i * kBase + x];
        if (kind == kStationary && lane == 0)
            a.logits[(size_t)i * a.d.Kmax * kStates + a.undo_k[i]] = a.undo_logit[i];
        if (kind >= kStationary) {
            const uint8_t fl = kind == kStationary ? (kSwsSpec | kSwsCl | kSwsP) : kSwsSpec;
            const uint8_t* flip = a.spec_flip + (size_t)i * a.d.Kmax;
            for (int k = lane; k < a.d.Kmax; k += 32)
                if (flip[k]) a.sws[(size_t)p * a.d.Kmax + k] ^= fl;
        }
    }
}

int dm_fail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

// A device-resident sweep of `steps` lockstep MH steps on [first, first+count).
// sched (count x steps, row-major) gives each particle's move family per step
// (-1 = idle); null runs the tree mixture at every step. kind_stats gets
// proposed / accepted counts per move kind (2 x kKinds).
int device_sweep(smccat_ctx* c, int first, int count, int steps, const std::vector<int8_t>* sched,
                 double temperature, uint64_t seed, int use_graph, unsigned long long* kind_stats) {
    const Dims& d = dims_of(c);
    if (first < 0 || count < 1 || steps < 0) return dm_fail(SMCCAT_EINVAL, "bad range");
    for (int i = 0; i < count; ++i) {
        const Slot& s = slot_of(c, first + i);
        if (!s.loaded) return dm_fail(SMCCAT_ESTATE, "particle has no state loaded");
        if (s.pending || s.full) return dm_fail(SMCCAT_ESTATE, "particle has unrefreshed or uncommitted edits");
    }
    DeviceView v;
    int rc = device_view(c, first, count, &v);
    if (rc) return rc;
    smccat_tuning tn;
    rc = smccat_get_tuning(c, &tn);
    if (rc) return rc;
    const int N = d.N, NI = d.NI, nchunk = (N + kPmChunk - 1) / kPmChunk;
    const bool use_splits = d.T <= 128;
    std::vector<uint64_t> skeys;
    std::vector<double> sprob;
    if (use_splits) split_table(c, &skeys, &sprob);
    const int nsplit = (int)sprob.size();

    // Host images of the trees and committed workspaces.
    std::vector<int32_t> par((size_t)count * N), kids((size_t)count * 2 * N);
    std::vector<double> br((size_t)count * N);
    std::vector<uint8_t> clws((size_t)count * N), pws((size_t)count * N);
    std::vector<PartHdr> hdr0(count);
    // The committed spectral workspaces: the device array holds what the last
    // refresh shipped, which a later reject on the host path may have undone.
    std::vector<uint8_t> sws0((size_t)count * d.Kmax);
    for (int i = 0; i < count; ++i) {
        const Mirror& m = slot_of(c, first + i).cur;
        std::copy(m.sws.begin(), m.sws.end(), &sws0[(size_t)i * d.Kmax]);
        std::copy(m.parent.begin(), m.parent.end(), &par[(size_t)i * N]);
        std::copy(m.kids.begin(), m.kids.end(), &kids[(size_t)i * 2 * N]);
        std::copy(m.branch.begin(), m.branch.end(), &br[(size_t)i * N]);
        std::copy(m.clws.begin(), m.clws.end(), &clws[(size_t)i * N]);
        std::copy(m.pws.begin(), m.pws.end(), &pws[(size_t)i * N]);
        PartHdr& h = hdr0[i];
        std::memset(&h, 0, sizeof(h));
        h.root = m.root;
        h.num_classes = m.K;
        h.cls_only = -1;
        h.pinv = m.pinv;
        for (int r = 0; r < kMaxRates; ++r) h.rates[r] = m.rates[r];
    }

    // One context-owned device buffer carved into the argument arrays.
    DmArgs a{};
    a.d = d;
    a.first = first;
    a.count = count;
    a.nchunk = nchunk;
    a.lnl = v.lnl;
    a.lnl_old = v.lnl_old;
    a.scale_delta = tn.scale_delta;
    a.subtree_delta = tn.subtree_scale_delta;
    a.anni_eps = tn.adaptive_nni_epsilon;
    a.temp = temperature;
    a.nsplit = nsplit;
    a.use_splits = use_splits;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off = (off + bytes + 255) & ~size_t(255); return o; };
    const size_t cN = (size_t)count * N;
    const size_t o_par = take(cN * 4), o_kids = take(2 * cN * 4), o_log = take((size_t)count * 2 * kUndo * 4),
                 o_nlog = take((size_t)count * 4), o_sk = take((size_t)std::max(nsplit, 1) * 16),
                 o_sp = take((size_t)std::max(nsplit, 1) * 8), o_br = take(cN * 8), o_clws = take(cN),
                 o_pws = take(cN), o_cc = take(cN), o_cp = take(cN), o_dirty = take(cN),
                 o_un = take(cN * 4), o_ul = take(cN * 8), o_nundo = take((size_t)count * 4),
                 o_kind = take((size_t)count * 4), o_extra = take((size_t)count * 8),
                 o_hdr0 = take((size_t)count * sizeof(PartHdr)), o_hdr = take((size_t)count * sizeof(PartHdr)),
                 o_nodes = take((size_t)count * NI * sizeof(NodeJob)), o_pj = take(cN * sizeof(PJob)),
                 o_mj = take((size_t)count * d.Kmax * nchunk * sizeof(PmJob)),
                 o_rng = take((size_t)count * sizeof(curandStatePhilox4_32_10_t)),
                 o_stats = take(2 * kKinds * 8);
    // Parameter state of whole-registry sweeps.
    const bool params = sched != nullptr;
    const size_t cK = (size_t)count * d.Kmax;
    size_t o_sched = 0, o_base = 0, o_logits = 0, o_shape = 0, o_shape_new = 0, o_ubase = 0,
           o_ulogit = 0, o_uk = 0, o_flip = 0, o_chol = 0;
    if (params) {
        o_sched = take((size_t)count * steps);
        o_base = take((size_t)count * kBase * 8);
        o_logits = take(cK * kStates * 8);
        o_shape = take((size_t)count * 8);
        o_shape_new = take((size_t)count * 8);
        o_ubase = take((size_t)count * kBase * 8);
        o_ulogit = take((size_t)count * 8);
        o_uk = take((size_t)count * 4);
        o_flip = take(cK);
        o_chol = take((size_t)kBase * kBase * 8);
    }
    unsigned char* buf = moves_buffer(c, off);
    if (!buf) return dm_fail(SMCCAT_ENOMEM, "device-move buffers: out of device memory");
    a.parent = reinterpret_cast<int32_t*>(buf + o_par);
    a.kids = reinterpret_cast<int32_t*>(buf + o_kids);
    a.ulog = reinterpret_cast<int32_t*>(buf + o_log);
    a.nlog = reinterpret_cast<int32_t*>(buf + o_nlog);
    a.skeys = reinterpret_cast<const uint64_t*>(buf + o_sk);
    a.sprob = reinterpret_cast<const double*>(buf + o_sp);
    a.branch = reinterpret_cast<double*>(buf + o_br);
    a.clws = buf + o_clws;
    a.pws = buf + o_pws;
    a.cur_clws = buf + o_cc;
    a.cur_pws = buf + o_cp;
    a.dirty = buf + o_dirty;
    a.undo_node = reinterpret_cast<int32_t*>(buf + o_un);
    a.undo_len = reinterpret_cast<double*>(buf + o_ul);
    a.nundo = reinterpret_cast<int32_t*>(buf + o_nundo);
    a.kind = reinterpret_cast<int32_t*>(buf + o_kind);
    a.extra = reinterpret_cast<double*>(buf + o_extra);
    a.hdr0 = reinterpret_cast<const PartHdr*>(buf + o_hdr0);
    a.hdr = reinterpret_cast<PartHdr*>(buf + o_hdr);
    a.nodes = reinterpret_cast<NodeJob*>(buf + o_nodes);
    a.pjobs = reinterpret_cast<PJob*>(buf + o_pj);
    a.mjobs = reinterpret_cast<PmJob*>(buf + o_mj);
    a.rng = reinterpret_cast<curandStatePhilox4_32_10_t*>(buf + o_rng);
    a.stats = reinterpret_cast<unsigned long long*>(buf + o_stats);
    std::vector<double> h_base, h_logits, h_shape, h_chol;
    if (params) {
        a.sched = reinterpret_cast<const int8_t*>(buf + o_sched);
        a.nsched = steps;
        a.hdr0w = reinterpret_cast<PartHdr*>(buf + o_hdr0);
        a.base = reinterpret_cast<double*>(buf + o_base);
        a.logits = reinterpret_cast<double*>(buf + o_logits);
        a.shape = reinterpret_cast<double*>(buf + o_shape);
        a.shape_new = reinterpret_cast<double*>(buf + o_shape_new);
        a.undo_base = reinterpret_cast<double*>(buf + o_ubase);
        a.undo_logit = reinterpret_cast<double*>(buf + o_ulogit);
        a.undo_k = reinterpret_cast<int32_t*>(buf + o_uk);
        a.spec_flip = buf + o_flip;
        a.chol = reinterpret_cast<const double*>(buf + o_chol);
        a.sws = const_cast<uint8_t*>(v.sws);
        a.spec = v.spec;
        a.shape_delta = tn.shape_delta;
        a.stationary_delta = tn.stationary_delta;
        a.rate_delta = tn.rate_matrix_delta;
        a.invar_alpha = tn.invar_alpha;
        a.lg = (model_flags_of(c) & SMCCAT_MODEL_LG) ? 1 : 0;
        a.R = d.R;
        h_base.resize((size_t)count * kBase);
        h_logits.assign(cK * kStates, 0.0);
        h_shape.resize(count);
        h_chol.resize((size_t)kBase * kBase);
        for (int i = 0; i < count; ++i) {
            const Mirror& m = slot_of(c, first + i).cur;
            std::copy(m.base.begin(), m.base.end(), &h_base[(size_t)i * kBase]);
            std::copy(m.logits.begin(), m.logits.begin() + (size_t)m.K * kStates,
                      &h_logits[(size_t)i * d.Kmax * kStates]);
            h_shape[i] = m.shape;
        }
        rc = smccat_get_rate_cholesky(c, h_chol.data());
        if (rc) return rc;
    }

    cudaStream_t st = v.st;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto finish = [&](int code, const std::string& msg) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamSynchronize(st);
        if (code) set_last_error(msg);
        return code;
    };
#define DM_CK(call)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return finish(SMCCAT_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
    DM_CK(cudaMemcpyAsync(a.parent, par.data(), cN * 4, cudaMemcpyHostToDevice, st));
    DM_CK(cudaMemcpyAsync(a.kids, kids.data(), 2 * cN * 4, cudaMemcpyHostToDevice, st));
    DM_CK(cudaMemcpyAsync(a.branch, br.data(), cN * 8, cudaMemcpyHostToDevice, st));
    DM_CK(cudaMemcpyAsync(a.clws, clws.data(), cN, cudaMemcpyHostToDevice, st));
    DM_CK(cudaMemcpyAsync(a.pws, pws.data(), cN, cudaMemcpyHostToDevice, st));
    DM_CK(cudaMemcpyAsync(buf + o_hdr0, hdr0.data(), (size_t)count * sizeof(PartHdr), cudaMemcpyHostToDevice, st));
    DM_CK(cudaMemsetAsync(a.stats, 0, 2 * kKinds * 8, st));
    DM_CK(cudaMemcpyAsync(const_cast<uint8_t*>(v.sws) + (size_t)first * d.Kmax, sws0.data(), sws0.size(),
                          cudaMemcpyHostToDevice, st));
    if (params) {
        DM_CK(cudaMemcpyAsync(buf + o_sched, sched->data(), (size_t)count * steps, cudaMemcpyHostToDevice, st));
        DM_CK(cudaMemcpyAsync(a.base, h_base.data(), h_base.size() * 8, cudaMemcpyHostToDevice, st));
        DM_CK(cudaMemcpyAsync(a.logits, h_logits.data(), h_logits.size() * 8, cudaMemcpyHostToDevice, st));
        DM_CK(cudaMemcpyAsync(a.shape, h_shape.data(), h_shape.size() * 8, cudaMemcpyHostToDevice, st));
        DM_CK(cudaMemcpyAsync(buf + o_chol, h_chol.data(), h_chol.size() * 8, cudaMemcpyHostToDevice, st));
        DM_CK(cudaMemsetAsync(a.spec_flip, 0, cK, st));
    }
    if (nsplit > 0) {
        DM_CK(cudaMemcpyAsync(buf + o_sk, skeys.data(), (size_t)nsplit * 16, cudaMemcpyHostToDevice, st));
        DM_CK(cudaMemcpyAsync(buf + o_sp, sprob.data(), (size_t)nsplit * 8, cudaMemcpyHostToDevice, st));
    }
    const int grid = (count + kDmThreads - 1) / kDmThreads;
    // Proposal blocks: kDmWarps particles each, fewer when their shared
    // memory would exceed the per-block limit.
    int dev = 0, smem_max = 0;
    DM_CK(cudaGetDevice(&dev));
    DM_CK(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t wbytes = dm_warp_bytes(N);
    const int pwarps = (int)std::min<size_t>(kDmWarps, (size_t)smem_max / wbytes);
    if (pwarps < 1) return finish(SMCCAT_EINVAL, "too many taxa for the device tree sweep");
    const size_t psmem = (size_t)pwarps * wbytes;
    if (psmem > 48 * 1024)
        DM_CK(cudaFuncSetAttribute(dm_propose_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem));
    const int pgrid = (count + pwarps - 1) / pwarps;
    dm_init_kernel<<<grid, kDmThreads, 0, st>>>(a.rng, count, first, (unsigned long long)seed);
    DM_CK(cudaGetLastError());
    DM_CK(cudaStreamSynchronize(st));  // the host images may go out of scope only after their copies

    PruneArgs pa = v.pa;
    pa.hdr = a.hdr;
    pa.nodes = a.nodes;
    const int nmjobs = count * d.Kmax * nchunk;
    auto step = [&](int k) -> cudaError_t {
        DmArgs ak = a;
        ak.step = k;
        dm_propose_kernel<<<pgrid, 32 * pwarps, psmem, st>>>(ak);
        cudaError_t x = cudaGetLastError();
        if (x == cudaSuccess && params) {
            dm_spec_kernel<<<count * d.Kmax, 32, 0, st>>>(ak);
            x = cudaGetLastError();
        }
        if (x == cudaSuccess) x = launch_pmat(a.mjobs, nmjobs, a.pjobs, a.hdr, first, v.sws, v.spec, v.Pm, v.fp32, d, st);
        if (x == cudaSuccess) x = launch_prune(pa, v.ntiles, v.variant, st);
        if (x == cudaSuccess) x = launch_reduce(v.tile_off, pa.partial, a.hdr, first, count, v.lnl, v.status, st);
        if (x == cudaSuccess) {
            dm_mh_kernel<<<(count + kDmWarps - 1) / kDmWarps, 32 * kDmWarps, 0, st>>>(ak);
            x = cudaGetLastError();
        }
        return x;
    };
    if (steps > 0) {
        if (use_graph) {
            DM_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            cudaError_t x = cudaSuccess;
            for (int k = 0; k < steps && x == cudaSuccess; ++k) x = step(k);
            const cudaError_t y = cudaStreamEndCapture(st, &graph);
            DM_CK(x);
            DM_CK(y);
            DM_CK(cudaGraphInstantiate(&exec, graph, 0));
            DM_CK(cudaGraphLaunch(exec, st));
        } else {
            for (int k = 0; k < steps; ++k) DM_CK(step(k));
        }
    }
    unsigned long long h_stats[2 * kKinds];
    int status = 0;
    std::vector<uint8_t> h_sws;
    if (params) {
        h_sws.resize(cK);
        DM_CK(cudaMemcpyAsync(h_base.data(), a.base, h_base.size() * 8, cudaMemcpyDeviceToHost, st));
        DM_CK(cudaMemcpyAsync(h_logits.data(), a.logits, h_logits.size() * 8, cudaMemcpyDeviceToHost, st));
        DM_CK(cudaMemcpyAsync(h_shape.data(), a.shape, h_shape.size() * 8, cudaMemcpyDeviceToHost, st));
        DM_CK(cudaMemcpyAsync(hdr0.data(), buf + o_hdr0, (size_t)count * sizeof(PartHdr), cudaMemcpyDeviceToHost, st));
        DM_CK(cudaMemcpyAsync(h_sws.data(), v.sws + (size_t)first * d.Kmax, cK, cudaMemcpyDeviceToHost, st));
    }
    DM_CK(cudaMemcpyAsync(h_stats, a.stats, sizeof(h_stats), cudaMemcpyDeviceToHost, st));
    DM_CK(cudaMemcpyAsync(&status, v.status, sizeof(int), cudaMemcpyDeviceToHost, st));
    DM_CK(cudaMemcpyAsync(br.data(), a.branch, cN * 8, cudaMemcpyDeviceToHost, st));
    DM_CK(cudaMemcpyAsync(par.data(), a.parent, cN * 4, cudaMemcpyDeviceToHost, st));
    DM_CK(cudaMemcpyAsync(clws.data(), a.clws, cN, cudaMemcpyDeviceToHost, st));
    DM_CK(cudaMemcpyAsync(pws.data(), a.pws, cN, cudaMemcpyDeviceToHost, st));
    DM_CK(cudaStreamSynchronize(st));
    if (status) {
        DM_CK(cudaMemset(v.status, 0, sizeof(int)));
        return finish(status & 2 ? SMCCAT_ETIMEOUT : SMCCAT_ENUMERIC,
                      status & 2 ? "a pruning warp gave up waiting for its transition matrices"
                                 : "a log-likelihood came out NaN");
    }
    // The host mirrors take the final committed state back; children and
    // post-order are regenerated from the parent tables.
    for (int i = 0; i < count; ++i) {
        Mirror tree;
        if (!rebuild_tree(d.T, &par[(size_t)i * N], &tree))
            return finish(SMCCAT_ENUMERIC, "device tree moves left an invalid tree");
        Slot& s = slot_mut(c, first + i);
        for (Mirror* m : {&s.cur, &s.old}) {
            m->parent = tree.parent;
            m->kids = tree.kids;
            m->post = tree.post;
            m->root = tree.root;
            std::copy(&br[(size_t)i * N], &br[(size_t)i * N] + N, m->branch.begin());
            std::copy(&clws[(size_t)i * N], &clws[(size_t)i * N] + N, m->clws.begin());
            std::copy(&pws[(size_t)i * N], &pws[(size_t)i * N] + N, m->pws.begin());
            if (params) {
                std::copy(&h_base[(size_t)i * kBase], &h_base[(size_t)i * kBase] + kBase, m->base.begin());
                std::copy(&h_logits[(size_t)i * d.Kmax * kStates],
                          &h_logits[(size_t)i * d.Kmax * kStates] + (size_t)m->K * kStates, m->logits.begin());
                m->shape = h_shape[i];
                m->pinv = hdr0[i].pinv;
                for (int r = 0; r < kMaxRates; ++r) m->rates[r] = hdr0[i].rates[r];
                std::copy(&h_sws[(size_t)i * d.Kmax], &h_sws[(size_t)i * d.Kmax] + d.Kmax, m->sws.begin());
            }
        }
    }
    if (kind_stats)
        for (int k = 0; k < 2 * kKinds; ++k) kind_stats[k] = h_stats[k];
    return finish(SMCCAT_OK, "");
#undef DM_CK
}

}  // namespace
}  // namespace smccat

using namespace smccat;

extern "C" int smccat_tree_sweep(smccat_ctx* c, int32_t first, int32_t count, int32_t steps,
                                 double temperature, uint64_t seed, int32_t use_graph,
                                 int64_t* stats) {
    NvtxRange range("smccat_tree_sweep");
    if (!c) return dm_fail(SMCCAT_EINVAL, "null context");
    unsigned long long ks[2 * kKinds];
    const int rc = device_sweep(c, first, count, steps, nullptr, temperature, seed, use_graph, ks);
    if (rc) return rc;
    if (stats)
        for (int k = 0; k < 10; ++k) stats[k] = (int64_t)ks[k];
    return SMCCAT_OK;
}

extern "C" int smccat_mcmc_sweep(smccat_ctx* c, int32_t first, int32_t count, int32_t iterations,
                                 double temperature, uint64_t seed, int32_t use_graph,
                                 smccat_move_stats* stats) {
    NvtxRange range("smccat_mcmc_sweep");
    if (!c) return dm_fail(SMCCAT_EINVAL, "null context");
    if (first < 0 || count < 1 || iterations < 0) return dm_fail(SMCCAT_EINVAL, "bad range");
    const Dims& d = dims_of(c);
    const int flags = model_flags_of(c);
    for (int i = 0; i < count; ++i) {
        const Slot& s = slot_of(c, first + i);
        if (!s.loaded) return dm_fail(SMCCAT_ESTATE, "particle has no state loaded");
        if ((flags & SMCCAT_MODEL_INVAR) && !(s.cur.pinv > 0.0))
            return dm_fail(SMCCAT_EINVAL, "invariant-site move needs pinv > 0");
    }
    // The registry of main.cpp:55-106 (weight, family), Mcmc::initMoveProbs
    // (Mcmc.cpp:15-23), and each particle's step sequence: per iteration one
    // draw from the registry, repeated its count of times (Mcmc.cpp:40-56).
    struct Entry { double w; int family; };
    std::vector<Entry> reg{{3.0, kFamTree}, {1.0, kFamStationary}};
    if (d.R > 1) reg.push_back({1.0, kFamShape});
    if (flags & SMCCAT_MODEL_INVAR) reg.push_back({1.0, kFamInvar});
    if (!(flags & SMCCAT_MODEL_LG)) reg.push_back({1.0, kFamRate});
    double wt = 0.0;
    for (auto& e : reg) wt += e.w;
    std::vector<double> cum;
    double acc = 0.0;
    for (auto& e : reg) { acc += e.w; cum.push_back(acc / wt); }
    std::vector<std::vector<int8_t>> seq(count);
    size_t steps = 0;
    for (int i = 0; i < count; ++i) {
        std::mt19937_64 g(seed * 0x9E3779B97F4A7C15ull + (uint64_t)(first + i) + 1);
        const int K = slot_of(c, first + i).cur.K;
        for (int it = 0; it < iterations; ++it) {
            const double u = std::generate_canonical<double, 53>(g);
            int fam = reg.back().family;
            for (size_t j = 0; j < cum.size(); ++j)
                if (u < cum[j]) { fam = reg[j].family; break; }
            const int rep = fam == kFamTree ? (int)(d.T * 0.25) : fam == kFamStationary ? 2 * K
                          : fam == kFamRate ? 5 : 2;
            seq[i].insert(seq[i].end(), rep, (int8_t)fam);
        }
        steps = std::max(steps, seq[i].size());
    }
    std::vector<int8_t> sched((size_t)count * steps, (int8_t)-1);
    for (int i = 0; i < count; ++i) std::copy(seq[i].begin(), seq[i].end(), &sched[(size_t)i * steps]);
    unsigned long long ks[2 * kKinds];
    const int rc = device_sweep(c, first, count, (int)steps, &sched, temperature, seed, use_graph, ks);
    if (rc) return rc;
    if (stats) {
        *stats = smccat_move_stats{};
        for (int k = 0; k < kKinds; ++k) {
            stats->proposed[k] = ks[2 * k];
            stats->accepted[k] = ks[2 * k + 1];
        }
        stats->lockstep_steps = steps;
    }
    return SMCCAT_OK;
}
