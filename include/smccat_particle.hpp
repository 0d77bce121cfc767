/*
 * smccat_particle.hpp -- the reference's C++ particle / MCMC interface on top
 * of the C-ABI (smccat.h), header-only, C++17.
 *
 * Smc-CAT's hot path is driven through `class Particle`
 * (src/analysis/Particle.hpp:48-94) and the MCMC functor `class Mcmc`
 * (src/analysis/Mcmc.hpp:15-26); its SMC driver (src/main.cpp) keeps one
 * Particle per OpenMP thread, copies particle states in and out with
 * copyFromSerialized / writeToSerialized, and calls mcmc(particle, iterations,
 * temperature). This header keeps those names, signatures and semantics so
 * such a driver compiles against the B200 engine:
 *
 *   - smccat::Particle has the reference's constructor
 *     Particle(seed, aln, nR, initInvar, lg, cat), its move methods (each
 *     returns the log Hastings ratio and leaves the edit pending),
 *     refreshLikelihood(force), lnLikelihood(), lnPrior(), accept(), reject(),
 *     copy, copyFromSerialized / writeToSerialized, the getters, and the public
 *     tunables and move counters. A Particle built with that constructor owns
 *     a one-slot engine context on its own; a Particle built from a
 *     ParticleBatch is a view of one slot of a shared context.
 *   - smccat::Mcmc has emplaceMove / initMoveProbs / operator()(Particle&,
 *     iterations, tempering) with the reference's loop (Mcmc.cpp:25-73), plus
 *     an overload on a whole ParticleBatch that runs the engine's batched
 *     rejuvenation (smccat_rejuvenate: the reference's move registry,
 *     main.cpp:55-106, every particle in lockstep on the GPU).
 *   - standardMoves() registers the reference's registry (main.cpp:55-106).
 *
 * Differences a caller sees, all at the boundary:
 *   - No Eigen / Boost types: vectors are std::array / std::vector; a split is
 *     two 64-bit taxon words (at most 128 taxa) instead of a dynamic_bitset.
 *   - SerializedParticle (SerializedParticle.hpp:8-17) carries the tree as a
 *     parent array and per-node branch lengths instead of a Newick string
 *     (Newick I/O is not part of the likelihood path); `stationaries` are the
 *     classes' logits, as in the reference.
 *   - The random streams are std::mt19937, so draws differ from Boost's.
 *   - Errors throw smccat::Error (with the C-ABI status code) instead of
 *     exiting the process.
 *   - Tunables are pushed to the context before each proposal; particles that
 *     share a ParticleBatch share one set (the reference's driver sets the same
 *     values on every particle, main.cpp:197-291).
 */
#ifndef SMCCAT_PARTICLE_HPP
#define SMCCAT_PARTICLE_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <limits>
#include <memory>
#include <random>
#include <set>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <vector>

#include "smccat.h"

namespace smccat {

class Error : public std::runtime_error {
   public:
    Error(int code, const std::string& msg)
        : std::runtime_error("smccat error " + std::to_string(code) + ": " + msg), code_(code) {}
    int code() const { return code_; }

   private:
    int code_;
};

inline void check(int rc) {
    if (rc != SMCCAT_OK) throw Error(rc, smccat_last_error());
}

/* Particle.hpp:18-30 */
enum UpdateType {
    ADAPTIVE_NNI = 0,
    NNI = 1,
    SPR = 2,
    BRANCH_LENGTH = 3,
    SCALE_SUBTREE = 4,
    INVAR = 5,
    RATE_SHAPE = 6,
    STATIONARY_SINGLE = 7,
    RATE_MATRIX_SINGLE = 8,
    RATE_MATRIX_FULL = 9,
    NO_MOVE = 10
};

static const std::array<std::string, 10> MoveNames = {
    "Adaptive NNI", "NNI", "SPR", "Branch Length", "Scale Subtree",
    "Proportion Invariant", "Rate Shape", "Stationary", "Rate Matrix Single", "Rate Matrix Full"};

/* An alignment in the reference's residue codes (Alignment.cpp:7-31:
 * ARNDCQEGHILKMFPSTWYV = 0..19, '-' = 20, 'X' = 21, '?' = 22), held in
 * memory. Reading FASTA files is not part of the likelihood path; build one
 * from sequences or from codes. */
class Alignment {
   public:
    /* Residue code of a character, -1 if it is not in the reference's table. */
    static int encode(char ch) {
        static const char* kResidues = "ARNDCQEGHILKMFPSTWYV";
        for (int i = 0; i < 20; ++i)
            if (kResidues[i] == ch) return i;
        if (ch == '-') return 20;
        if (ch == 'X') return 21;
        if (ch == '?') return 22;
        return -1;
    }

    /* One sequence per taxon, all the same length (the reference exits on a
     * ragged alignment or an unknown character, Alignment.cpp:79-96). */
    Alignment(std::vector<std::string> names, const std::vector<std::string>& sequences)
        : names_(std::move(names)) {
        if (sequences.empty() || sequences.size() != names_.size())
            throw Error(SMCCAT_EINVAL, "one sequence per taxon name is needed");
        numTaxa_ = (int)sequences.size();
        numChar_ = (int)sequences[0].size();
        codes_.resize((size_t)numTaxa_ * numChar_);
        for (int t = 0; t < numTaxa_; ++t) {
            if ((int)sequences[t].size() != numChar_)
                throw Error(SMCCAT_EINVAL, "sequence " + names_[t] + " has a different length");
            for (int s = 0; s < numChar_; ++s) {
                const int c = encode(sequences[t][s]);
                if (c < 0) throw Error(SMCCAT_EINVAL, "unknown residue in sequence " + names_[t]);
                codes_[(size_t)t * numChar_ + s] = (uint8_t)c;
            }
        }
    }

    /* codes: [numTaxa][numChar] row-major, values 0..22. */
    Alignment(std::vector<std::string> names, std::vector<uint8_t> codes, int numChar)
        : names_(std::move(names)), codes_(std::move(codes)), numChar_(numChar) {
        numTaxa_ = (int)names_.size();
        if (numChar_ < 1 || codes_.size() != (size_t)numTaxa_ * numChar_)
            throw Error(SMCCAT_EINVAL, "codes must hold numTaxa x numChar values");
        for (uint8_t c : codes_)
            if (c > 22) throw Error(SMCCAT_EINVAL, "alignment code > 22");
    }

    int operator()(int taxon, int site) const { return codes_[(size_t)taxon * numChar_ + site]; }
    int getNumChar() const { return numChar_; }
    int getNumTaxa() const { return numTaxa_; }
    const std::vector<std::string>& getTaxaNames() const { return names_; }
    const uint8_t* codes() const { return codes_.data(); }

   private:
    std::vector<std::string> names_;
    std::vector<uint8_t> codes_;
    int numChar_ = 0, numTaxa_ = 0;
};

/* A split: the taxa on one side of an edge, taxa 0..63 in w[0] and 64..127 in
 * w[1], canonicalised so that taxon 0 is set (Tree.cpp:511-516). */
struct Split {
    uint64_t w[2] = {0, 0};
    bool operator==(const Split& o) const { return w[0] == o.w[0] && w[1] == o.w[1]; }
    bool operator<(const Split& o) const { return w[0] < o.w[0] || (w[0] == o.w[0] && w[1] < o.w[1]); }
};
struct SplitHash {
    size_t operator()(const Split& s) const { return std::hash<uint64_t>()(s.w[0] * 0x9E3779B97F4A7C15ull ^ s.w[1]); }
};
using SplitPosteriors = std::unordered_map<Split, double, SplitHash>;

/* SerializedParticle.hpp:8-17 with the tree as arrays over the 2T-1 node ids
 * (tips 0..T-1 in alignment order, internal T..2T-2, parent[root] = -1). */
struct SerializedParticle {
    std::vector<int32_t> parent;
    std::vector<double> branchLengths;           /* per node id; the root's is unused */
    std::vector<int> assignments;                /* class of each site           */
    std::vector<int> categorySize;               /* sites per class              */
    std::vector<std::array<double, 20>> stationaries;  /* each class's logits    */
    std::array<double, 190> baseMatrix{};        /* log-exchangeabilities        */
    double pInvar = 0.0;
    double shape = 1.0;
};

/* One engine context: a batch of particle slots resident on one GPU. */
class ParticleBatch {
   public:
    struct Options {
        int maxClasses = 128;                /* per-particle class capacity (CAT) */
        int precision = SMCCAT_PREC_FP64;    /* or SMCCAT_PREC_FP32               */
        int device = 0;
        bool patterns = false;               /* site-pattern compression          */
    };

    ParticleBatch(const Alignment& aln, int numParticles, int nR, bool invar, bool lg, bool cat)
        : ParticleBatch(aln, numParticles, nR, invar, lg, cat, Options()) {}
    ParticleBatch(const Alignment& aln, int numParticles, int nR, bool invar, bool lg, bool cat,
                  Options o)
        : numTaxa_(aln.getNumTaxa()), numChar_(aln.getNumChar()), numRates_(nR), size_(numParticles),
          invar_(invar), lg_(lg), cat_(cat), maxClasses_(cat ? o.maxClasses : 1) {
        smccat_config cfg{};
        cfg.num_taxa = numTaxa_;
        cfg.num_sites = numChar_;
        cfg.num_rates = nR;
        cfg.max_particles = numParticles;
        cfg.max_classes = maxClasses_;
        cfg.model_flags = (lg ? SMCCAT_MODEL_LG : 0) | (invar ? SMCCAT_MODEL_INVAR : 0) |
                          (cat ? SMCCAT_MODEL_CAT : 0) | (o.patterns ? SMCCAT_MODEL_PATTERNS : 0);
        cfg.precision = o.precision;
        cfg.device = o.device;
        check(smccat_create(&cfg, aln.codes(), &ctx_));
    }
    ~ParticleBatch() {
        if (ctx_) smccat_destroy(ctx_);
    }
    ParticleBatch(const ParticleBatch&) = delete;
    ParticleBatch& operator=(const ParticleBatch&) = delete;

    smccat_ctx* ctx() const { return ctx_; }
    int size() const { return size_; }
    int numTaxa() const { return numTaxa_; }
    int numChar() const { return numChar_; }
    int numRates() const { return numRates_; }
    int maxClasses() const { return maxClasses_; }
    bool invar() const { return invar_; }
    bool lg() const { return lg_; }
    bool cat() const { return cat_; }

    /* refreshLikelihood(force) of every slot in one batched call. */
    void refreshLikelihood(bool force = false) {
        check(smccat_refresh(ctx_, 0, size_, force ? SMCCAT_REFRESH_FULL : SMCCAT_REFRESH_DIRTY));
    }
    std::vector<double> lnLikelihoods() const {
        std::vector<double> out(size_);
        check(smccat_get_lnl(ctx_, 0, size_, out.data()));
        return out;
    }

    /* Tunables of the context, written only when they change. */
    void setTuning(const smccat_tuning& t) {
        if (haveTuning_ && std::equal(reinterpret_cast<const double*>(&t),
                                      reinterpret_cast<const double*>(&t) + 8,
                                      reinterpret_cast<const double*>(&tuning_)))
            return;
        check(smccat_set_tuning(ctx_, &t));
        tuning_ = t;
        haveTuning_ = true;
    }
    void setRateCholesky(const std::vector<double>& lower) {
        if (lower == cholesky_) return;
        if (lower.size() != 190u * 190u) throw Error(SMCCAT_EINVAL, "the Cholesky factor is 190 x 190");
        check(smccat_set_rate_cholesky(ctx_, lower.data()));
        cholesky_ = lower;
    }
    /* The split posteriors the adaptive NNI move reads. */
    void setSplitPosteriors(const SplitPosteriors& sp) {
        std::vector<std::pair<Split, double>> v(sp.begin(), sp.end());
        std::sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        if (v == splits_) return;
        std::vector<uint64_t> bits(2 * v.size());
        std::vector<double> prob(v.size());
        for (size_t i = 0; i < v.size(); ++i) {
            bits[2 * i] = v[i].first.w[0];
            bits[2 * i + 1] = v[i].first.w[1];
            prob[i] = v[i].second;
        }
        check(smccat_set_split_posteriors(ctx_, (int32_t)v.size(), bits.data(), prob.data()));
        splits_ = std::move(v);
    }

   private:
    smccat_ctx* ctx_ = nullptr;
    int numTaxa_, numChar_, numRates_, size_;
    bool invar_, lg_, cat_;
    int maxClasses_;
    smccat_tuning tuning_{};
    bool haveTuning_ = false;
    std::vector<double> cholesky_;
    std::vector<std::pair<Split, double>> splits_;
};

/* class Particle (Particle.hpp:48-125) as a view of one slot of an engine
 * context. Move methods propose on the slot and leave the edit pending; the
 * caller refreshes and accepts or rejects, as with the reference. */
class Particle {
   public:
    Particle(void) = delete;

    /* Particle::Particle + initialize (Particle.cpp:21-183): a random state
     * (random tree, LG or N(0,1) exchangeabilities, pinv ~ U(0,1) with +I,
     * shape ~ Gamma(3, 2) with nR > 1, a CRP(0.01) class partition with CAT)
     * drawn from `seed`, in a one-slot context of its own. */
    Particle(int seed, Alignment& aln, int nR = 1, bool initInvar = false, bool lg = true,
             bool cat = true)
        : own_(std::make_shared<ParticleBatch>(aln, 1, nR, initInvar, lg, cat)), batch_(own_.get()),
          slot_(0), rng_((uint32_t)seed) {
        setup();
        initialize(initInvar, cat);
    }

    /* A view of slot `slot` of `batch`, with no state loaded yet: call
     * initialize() or copyFromSerialized() first. */
    Particle(int seed, ParticleBatch& batch, int slot) : batch_(&batch), slot_(slot), rng_((uint32_t)seed) {
        if (slot < 0 || slot >= batch.size()) throw Error(SMCCAT_EINVAL, "slot out of range");
        setup();
    }

    double getPInvar() const { return read().pInvar; }
    double getShape() const { return read().shape; }

    /* Neal's Algorithm 8 reassignment (Particle.cpp:785-995) followed by the
     * full refresh the driver makes after it (main.cpp:303-306). Returns +inf,
     * as the reference does outside an MH setting. */
    double gibbsPartitionMove(double tempering) {
        const uint8_t mask = 1;
        smccat_gibbs_stats st{};
        check(smccat_gibbs(ctx(), slot_, 1, &mask, tempering, next_seed(), &st));
        return std::numeric_limits<double>::infinity();
    }
    double invarMove() { return propose(SMCCAT_FAMILY_INVAR); }
    double rateMatrixMove() {
        batch_->setRateCholesky(rateMatrixCholesky);
        return propose(SMCCAT_FAMILY_RATE_MATRIX);
    }
    double shapeMove() { return propose(SMCCAT_FAMILY_SHAPE); }
    double stationaryMove() { return propose(SMCCAT_FAMILY_STATIONARY); }
    double treeMove(const SplitPosteriors& splitPosterior) {
        batch_->setSplitPosteriors(splitPosterior);
        return propose(SMCCAT_FAMILY_TREE);
    }

    double lnLikelihood() {
        double v = 0.0;
        check(smccat_get_lnl(ctx(), slot_, 1, &v));
        return v;
    }
    double lnPrior() {
        syncTuning();
        double v = 0.0;
        check(smccat_ln_prior(ctx(), slot_, 1, &v));
        return v;
    }

    std::mt19937& getRng() { return rng_; }
    std::array<double, 190> getBaseMatrix() const { return read().baseMatrix; }
    int getNumCategories() const { return (int)read().stationaries.size(); }
    int getNumNodes() const { return numNodes_; }
    int getNumRates() const { return batch_->numRates(); }
    /* Tree::getSplitSet (Tree.cpp:485-541): every non-root node's taxon set,
     * canonicalised to contain taxon 0. */
    std::set<Split> getSplitSet() const {
        const SerializedParticle sp = read();
        const int T = batch_->numTaxa(), N = numNodes_;
        std::vector<Split> clade(N);
        for (int t = 0; t < T; ++t) clade[t].w[t >> 6] = 1ull << (t & 63);
        // Children before parents: internal nodes by decreasing depth.
        std::vector<int> depth(N, 0), order;
        for (int n = 0; n < N; ++n) {
            int d = 0;
            for (int y = sp.parent[n]; y >= 0 && d <= N; y = sp.parent[y]) ++d;
            depth[n] = d;
            if (n >= T) order.push_back(n);
        }
        std::sort(order.begin(), order.end(), [&](int a, int b) { return depth[a] > depth[b]; });
        for (int n : order)
            for (int x = 0; x < N; ++x)
                if (sp.parent[x] == n) { clade[n].w[0] |= clade[x].w[0]; clade[n].w[1] |= clade[x].w[1]; }
        const uint64_t f0 = T >= 64 ? ~0ull : (1ull << T) - 1;
        const uint64_t f1 = T <= 64 ? 0ull : (T >= 128 ? ~0ull : (1ull << (T - 64)) - 1);
        std::set<Split> out;
        for (int n = 0; n < N; ++n) {
            if (sp.parent[n] < 0) continue;
            Split s = clade[n];
            if (!(s.w[0] & 1ull)) { s.w[0] = ~s.w[0] & f0; s.w[1] = ~s.w[1] & f1; }
            out.insert(s);
        }
        return out;
    }
    std::vector<double> getRates() const {
        std::vector<double> r(getNumRates(), 1.0);
        if (r.size() > 1) check(smccat_discretize_gamma(getShape(), (int32_t)r.size(), r.data()));
        return r;
    }
    std::vector<std::array<double, 20>> getCategories() const { return read().stationaries; }
    std::vector<int> getAssignments() const { return read().assignments; }

    /* Particle::accept / reject (Particle.cpp:343-478): the engine keeps the
     * new state or restores the old one by flipping workspace indices. */
    void accept() {
        const uint8_t m = 1;
        check(smccat_accept(ctx(), slot_, 1, &m));
        if (currentMove_ != NO_MOVE) {
            moveCount[currentMove_]++;
            acceptCount[currentMove_]++;
        }
        currentMove_ = NO_MOVE;
    }
    void reject() {
        const uint8_t m = 0;
        check(smccat_accept(ctx(), slot_, 1, &m));
        if (currentMove_ != NO_MOVE) moveCount[currentMove_]++;
        currentMove_ = NO_MOVE;
    }

    /* Particle::copy (Particle.cpp:185-216): take p's state. */
    void copy(Particle& p) {
        SerializedParticle sp;
        p.writeToSerialized(sp);
        copyFromSerialized(sp);
    }
    /* Particle::copyFromSerialized (Particle.cpp:218-300): load the state and
     * refreshLikelihood(true), which commits it. */
    void copyFromSerialized(SerializedParticle& sp) {
        const int T = batch_->numTaxa(), N = numNodes_, S = batch_->numChar();
        const int K = (int)sp.stationaries.size();
        if ((int)sp.parent.size() != N || (int)sp.branchLengths.size() != N || (int)sp.assignments.size() != S)
            throw Error(SMCCAT_EINVAL, "serialized particle does not match the alignment");
        if (K < 1 || K > batch_->maxClasses()) throw Error(SMCCAT_EINVAL, "class count out of range");
        (void)T;
        std::vector<double> logits((size_t)batch_->maxClasses() * 20, 0.0);
        for (int k = 0; k < K; ++k) std::copy(sp.stationaries[k].begin(), sp.stationaries[k].end(), &logits[(size_t)k * 20]);
        const int32_t nk = K;
        std::vector<int32_t> assign(sp.assignments.begin(), sp.assignments.end());
        check(smccat_set_particles(ctx(), slot_, 1, sp.parent.data(), sp.branchLengths.data(),
                                   sp.baseMatrix.data(), &nk, logits.data(), assign.data(), &sp.pInvar,
                                   &sp.shape));
        refreshLikelihood(true);
        currentMove_ = NO_MOVE;
    }
    /* Particle::writeToSerialized (Particle.cpp:302-320). */
    void writeToSerialized(SerializedParticle& sp) { sp = read(); }

    /* Particle::initialize (Particle.cpp:81-183) on this particle's stream. */
    void initialize(bool initInvar = false, bool initCat = true) {
        const int T = batch_->numTaxa(), N = numNodes_, S = batch_->numChar();
        std::uniform_real_distribution<double> unif(0.0, 1.0);
        std::normal_distribution<double> normal(0.0, 1.0);
        SerializedParticle sp;
        if (batch_->lg()) {
            check(smccat_lg_exchangeabilities(sp.baseMatrix.data()));
        } else {
            for (double& b : sp.baseMatrix) b = normal(rng_);
        }
        // Tree(rng, names) (Tree.cpp:10-77): split the edge above a random
        // existing tip for each new taxon; branch lengths ~ Exp(rate 10).
        sp.parent.assign(N, -1);
        sp.parent[0] = sp.parent[1] = T;
        int next = T + 1;
        for (int i = 2; i < T; ++i) {
            const int tip = std::min(i - 1, (int)(unif(rng_) * i));
            const int fresh = next++;
            sp.parent[fresh] = sp.parent[tip];
            sp.parent[tip] = fresh;
            sp.parent[i] = fresh;
        }
        std::exponential_distribution<double> expo(10.0);
        sp.branchLengths.assign(N, 0.0);
        for (int n = 0; n < N; ++n) sp.branchLengths[n] = sp.parent[n] < 0 ? 0.0 : expo(rng_);
        sp.pInvar = initInvar ? unif(rng_) : 0.0;
        sp.shape = batch_->numRates() > 1 ? std::gamma_distribution<double>(3.0, 2.0)(rng_) : 1.0;
        // Chinese restaurant process with concentration dppAlpha (Particle.cpp:134-158).
        sp.assignments.assign(S, 0);
        std::vector<int> sizes;
        if (initCat && batch_->cat()) {
            for (int i = 0; i < S; ++i) {
                const double u = unif(rng_);
                double total = dppAlpha / (i + dppAlpha);
                if (total > u && (int)sizes.size() < batch_->maxClasses()) {
                    sp.assignments[i] = (int)sizes.size();
                    sizes.push_back(1);
                    continue;
                }
                int k = (int)sizes.size() - 1;
                for (int c = 0; c < (int)sizes.size(); ++c) {
                    total += sizes[c] / (i + dppAlpha);
                    if (total > u) { k = c; break; }
                }
                sp.assignments[i] = std::max(k, 0);
                if (sizes.empty()) sizes.push_back(0);
                sizes[std::max(k, 0)]++;
            }
        } else {
            sizes.assign(1, S);
        }
        // sampleStationaryLogits (TransitionProbabilityClass.cpp:26-35):
        // 19 standard normal logits and a 0.
        for (size_t k = 0; k < sizes.size(); ++k) {
            std::array<double, 20> l{};
            for (int j = 0; j < 19; ++j) l[j] = normal(rng_);
            sp.stationaries.push_back(l);
        }
        sp.categorySize = sizes;
        copyFromSerialized(sp);
    }

    /* refreshLikelihood (Particle.cpp:530-675): dirty nodes only, or
     * everything with forceUpdate. */
    void refreshLikelihood(bool forceUpdate = false) {
        check(smccat_refresh(ctx(), slot_, 1, forceUpdate ? SMCCAT_REFRESH_FULL : SMCCAT_REFRESH_DIRTY));
    }
    void setAssignments(std::vector<int>& assignments) {
        SerializedParticle sp = read();
        if (assignments.size() != sp.assignments.size()) throw Error(SMCCAT_EINVAL, "one class per site");
        sp.assignments = assignments;
        copyFromSerialized(sp);
    }
    void setInvariance(double i) {
        check(smccat_set_pinv(ctx(), slot_, i));
        refreshLikelihood();
        const uint8_t m = 1;
        check(smccat_accept(ctx(), slot_, 1, &m));
    }

    std::array<int, 10> moveCount{};
    std::array<int, 10> acceptCount{};
    double aNNIEpsilon = 0.01;
    double shapeDelta = 1.0;
    double scaleDelta = 1.0;
    double subtreeScaleDelta = 1.0;
    double stationaryDelta = 0.25;
    double rateMatrixDelta = 0.25;
    std::vector<double> rateMatrixCholesky;  /* 190 x 190 lower, row-major; 0.5 I */
    double invarAlpha = 100.0;
    double dppAlpha = 0.01;

    int slot() const { return slot_; }
    ParticleBatch& batch() { return *batch_; }

   private:
    void setup() {
        numNodes_ = 2 * batch_->numTaxa() - 1;
        rateMatrixCholesky.assign(190 * 190, 0.0);
        for (int i = 0; i < 190; ++i) rateMatrixCholesky[(size_t)i * 190 + i] = 0.5;
    }
    smccat_ctx* ctx() const { return batch_->ctx(); }
    uint64_t next_seed() { return ((uint64_t)rng_() << 32) ^ rng_(); }
    void syncTuning() {
        smccat_tuning t;
        t.adaptive_nni_epsilon = aNNIEpsilon;
        t.shape_delta = shapeDelta;
        t.scale_delta = scaleDelta;
        t.subtree_scale_delta = subtreeScaleDelta;
        t.stationary_delta = stationaryDelta;
        t.rate_matrix_delta = rateMatrixDelta;
        t.invar_alpha = invarAlpha;
        t.dpp_alpha = dppAlpha;
        batch_->setTuning(t);
    }
    double propose(int family) {
        syncTuning();
        int32_t kind = NO_MOVE;
        double hastings = 0.0;
        check(smccat_propose(ctx(), slot_, family, next_seed(), &kind, &hastings));
        currentMove_ = kind;
        return hastings;
    }
    SerializedParticle read() const {
        const int N = numNodes_, S = batch_->numChar(), Kmax = batch_->maxClasses();
        SerializedParticle sp;
        sp.parent.resize(N);
        sp.branchLengths.resize(N);
        std::vector<int32_t> assign(S);
        std::vector<double> logits((size_t)Kmax * 20);
        int32_t K = 0;
        check(smccat_get_particles(ctx(), slot_, 1, sp.parent.data(), sp.branchLengths.data(),
                                   sp.baseMatrix.data(), &K, logits.data(), assign.data(), &sp.pInvar,
                                   &sp.shape));
        sp.assignments.assign(assign.begin(), assign.end());
        sp.categorySize.assign(K, 0);
        for (int a : sp.assignments)
            if (a >= 0 && a < K) sp.categorySize[a]++;
        for (int k = 0; k < K; ++k) {
            std::array<double, 20> l;
            std::copy(&logits[(size_t)k * 20], &logits[(size_t)k * 20] + 20, l.begin());
            sp.stationaries.push_back(l);
        }
        return sp;
    }

    std::shared_ptr<ParticleBatch> own_;
    ParticleBatch* batch_;
    int slot_;
    std::mt19937 rng_;
    int numNodes_ = 0;
    int currentMove_ = NO_MOVE;
};

/* class Mcmc (Mcmc.hpp:15-26, Mcmc.cpp:1-73). */
class Mcmc {
   public:
    using Move = std::tuple<double, std::function<int(Particle&)>, std::function<double(Particle&)>>;

    Mcmc(void) : totalMoveWeight(0.0) {}

    void emplaceMove(Move&& move) {
        totalMoveWeight += std::get<0>(move);
        moves.emplace_back(std::move(move));
    }
    void initMoveProbs() {
        moveProbs.clear();
        double cum = 0.0;
        for (const auto& m : moves) {
            cum += std::get<0>(m);
            moveProbs.push_back(cum / totalMoveWeight);
        }
    }

    /* Mcmc::operator() (Mcmc.cpp:25-73): `iterations` draws from the move
     * registry, each repeated its count of times as a Metropolis-Hastings step
     * on tempering * lnL + lnPrior + log Hastings. */
    void operator()(Particle& model, int iterations, double tempering) {
        if (moveProbs.empty())
            throw Error(SMCCAT_ESTATE, "the move probabilities are not initialized (initMoveProbs)");
        std::mt19937& rng = model.getRng();
        std::uniform_real_distribution<double> unif(0.0, 1.0);
        model.refreshLikelihood();
        double currentPosterior = model.lnLikelihood() * tempering + model.lnPrior();
        for (int i = 0; i < iterations; ++i) {
            const double choice = unif(rng);
            std::function<double(Particle&)> proposal;
            int repeats = 3;
            for (size_t j = 0; j < moveProbs.size(); ++j) {
                if (choice < moveProbs[j]) {
                    proposal = std::get<2>(moves[j]);
                    repeats = std::get<1>(moves[j])(model);
                    break;
                }
            }
            if (!proposal) continue;
            for (int j = 0; j < repeats; ++j) {
                const double hastings = proposal(model);
                model.refreshLikelihood();
                const double newPosterior = model.lnPrior() + model.lnLikelihood() * tempering;
                if (std::log(unif(rng)) <= newPosterior - currentPosterior + hastings) {
                    model.accept();
                    currentPosterior = newPosterior;
                } else {
                    model.reject();
                }
            }
        }
    }

    /* The same sweep for every particle of a batch at once: the engine's
     * smccat_rejuvenate, whose registry is the reference's (main.cpp:55-106:
     * tree 3 x floor(T/4), stationary 1 x 2K, shape 1 x 2 with nR > 1,
     * invariant 1 x 2 with +I, rate matrix 1 x 5 without LG), all particles
     * in lockstep with one batched dirty refresh per step. The moves emplaced
     * here do not apply to it. Returns the move counts. */
    smccat_move_stats operator()(ParticleBatch& batch, int iterations, double tempering, uint64_t seed) {
        smccat_move_stats st{};
        check(smccat_rejuvenate(batch.ctx(), 0, batch.size(), iterations, tempering, seed, &st));
        return st;
    }

   private:
    std::vector<Move> moves;
    std::vector<double> moveProbs;
    double totalMoveWeight;
};

/* The reference's move registry (main.cpp:55-106) on `mcmc`, with the split
 * posteriors the tree move reads. */
inline void standardMoves(Mcmc& mcmc, const Alignment& aln, int numRates, bool invar, bool lg,
                          const SplitPosteriors& splitPosteriors) {
    const int treeRepeats = static_cast<int>(aln.getNumTaxa() * 0.25);
    mcmc.emplaceMove(Mcmc::Move{3.0, [treeRepeats](Particle&) { return treeRepeats; },
                                [&splitPosteriors](Particle& m) { return m.treeMove(splitPosteriors); }});
    mcmc.emplaceMove(Mcmc::Move{1.0, [](Particle& m) { return m.getNumCategories() * 2; },
                                [](Particle& m) { return m.stationaryMove(); }});
    if (numRates > 1)
        mcmc.emplaceMove(Mcmc::Move{1.0, [](Particle&) { return 2; }, [](Particle& m) { return m.shapeMove(); }});
    if (invar)
        mcmc.emplaceMove(Mcmc::Move{1.0, [](Particle&) { return 2; }, [](Particle& m) { return m.invarMove(); }});
    if (!lg)
        mcmc.emplaceMove(Mcmc::Move{1.0, [](Particle&) { return 5; }, [](Particle& m) { return m.rateMatrixMove(); }});
    mcmc.initMoveProbs();
}

}  // namespace smccat

#endif /* SMCCAT_PARTICLE_HPP */
