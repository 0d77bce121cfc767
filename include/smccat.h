/*
 * smccat.h -- C-ABI of the B200 likelihood engine for Smc-CAT.
 *
 * One context (smccat_ctx) holds, on one GPU, a batch of SMC particles over a
 * fixed alignment: their tree, model parameters, conditional-likelihood (CL)
 * buffers, transition matrices and per-class spectral data. The calls below
 * replace the reference's per-particle C++ likelihood interface
 * (class Particle, src/analysis/Particle.hpp:48-125) with batched calls over a
 * range of particles [first, first + count).
 *
 * Conventions
 *   - Every call returns an int status: SMCCAT_OK (0) or one of the error
 *     codes below; smccat_last_error() gives a one-line message. The reference
 *     exits the process on bad input instead (Alignment.cpp:79-96, Tree.cpp:104,
 *     main.cpp:158-174).
 *   - The caller owns every host array; the context owns all device memory.
 *   - Calls on one context are not thread-safe; each context uses one CUDA
 *     stream. Contexts on different devices are independent.
 *   - Trees are rooted and binary, flattened as a parent array over
 *     2T-1 nodes: tips 0..T-1 (taxon order of the alignment), internal nodes
 *     T..2T-2, parent[root] = -1 (the reference's node-id convention,
 *     Tree.cpp:61-74). branch[n] is the length of the edge above node n.
 *   - Residue codes are the reference's alignment codes (Alignment.cpp:7-31):
 *     0-19 = ARNDCQEGHILKMFPSTWYV, 20 = '-', 21 = 'X', 22 = '?'.
 */
#ifndef SMCCAT_H
#define SMCCAT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMCCAT_OK        0
#define SMCCAT_EINVAL    1  /* bad argument or inconsistent particle state   */
#define SMCCAT_ECUDA     2  /* a CUDA runtime call failed                   */
#define SMCCAT_ENOMEM    3  /* device or host allocation failed / too large */
#define SMCCAT_ESTATE    4  /* call out of protocol order                   */
#define SMCCAT_ENUMERIC  5  /* a likelihood came out NaN                     */
#define SMCCAT_ENODEV    6  /* no usable CUDA device                         */
#define SMCCAT_ETIMEOUT  7  /* a bounded device-side wait gave up            */

/* model_flags */
#define SMCCAT_MODEL_LG     1  /* LG exchangeabilities (else GTR, inferred)  */
#define SMCCAT_MODEL_INVAR  2  /* +I invariant-site mixture                  */
#define SMCCAT_MODEL_CAT    4  /* Dirichlet-process (CAT) class mixture      */
#define SMCCAT_MODEL_PATTERNS 8 /* site-pattern compression (no counterpart in
                                  the reference, which evaluates every site):
                                  each particle evaluates every distinct
                                  (alignment column, class) pair once and
                                  weights it by its number of sites. Results
                                  are the same up to rounding; per-site
                                  log-likelihoods are still given for every
                                  site                                        */

/* precision */
#define SMCCAT_PREC_FP64    0  /* plain FP64 pruning                         */
#define SMCCAT_PREC_FP32    1  /* mixed: FP32 partials, transition matrices and
                                  pruning arithmetic (the reference's
                                  MIXED_PRECISION CL_TYPE = float,
                                  Miscellaneous.hpp:13-17); eigensystems, the
                                  exp(Lambda t) reconstruction, log-scalers and
                                  the site / particle sums stay FP64          */

/* refresh modes */
#define SMCCAT_REFRESH_DIRTY 0 /* refreshLikelihood(false): dirty nodes only */
#define SMCCAT_REFRESH_FULL  1 /* refreshLikelihood(true): everything        */

typedef struct smccat_ctx smccat_ctx;

typedef struct smccat_config {
    int32_t num_taxa;       /* T >= 3                                          */
    int32_t num_sites;      /* S >= 1                                          */
    int32_t num_rates;      /* R in [1, 8]: discrete-gamma categories          */
    int32_t max_particles;  /* particles resident on the device at once        */
    int32_t max_classes;    /* per-particle class capacity (1 without CAT)     */
    int32_t model_flags;    /* SMCCAT_MODEL_*                                  */
    int32_t precision;      /* SMCCAT_PREC_*                                   */
    int32_t device;         /* CUDA device ordinal                             */
} smccat_config;

/* Library version string, e.g. "smccat-b200 0.1". */
const char* smccat_version(void);

/* Message for the last error raised on this thread. */
const char* smccat_last_error(void);

/* discretizeGamma (src/core/Miscellaneous.hpp:22-37): the R midpoint
 * quantiles (2i+1)/(2R) of Gamma(shape, scale 1/shape), rescaled to mean 1.
 * Host-only; needs no device. */
int smccat_discretize_gamma(double shape, int32_t num_rates, double* out);

/* The 190 LG exchangeabilities in the reference's lower-triangle order
 * (src/analysis/RateMatrices.hpp:7-111): (i, j) for i = 1..19, j < i. The
 * reference feeds these raw values as the base vector of LG runs
 * (Particle.cpp:84-94). Host-only. */
int smccat_lg_exchangeabilities(double* out190);

/* Batched transition matrices for callers that cannot allocate device memory.
 * No counterpart in the reference. Some hosts of this library may not call
 * cudaMalloc at all -- code living inside another framework's memory budget or
 * custom allocator, or a plugin that is only handed pre-allocated buffers --
 * so this entry point allocates nothing: the caller passes device buffers for
 * every input and output, and the intermediate spectral data go to a
 * fixed-size array compiled into the library (3.5 MB, kept on every GPU that
 * loads the library's kernels until the process exits).
 *   base    [num_classes][190]  log-exchangeabilities (device)
 *   logits  [num_classes][20]   stationary logits (device)
 *   times   [num_classes][num_times]  branch length x rate (device)
 *   p_out   [num_classes][num_times][20][20]  row-major P(t) (device)
 * num_classes may be at most 512; larger requests return SMCCAT_EINVAL. Work
 * is queued on `stream` (a cudaStream_t, NULL = legacy default stream) on the
 * current device and the call returns without waiting. Set-up: a call outside
 * stream capture resolves the array's device address in the CUDA context
 * current at the call (the device's primary context, or a context the host
 * made current itself); a call under stream capture uses the address recorded
 * by that context's last call outside capture, so make one call in each
 * context before capturing (else SMCCAT_ESTATE). Launch errors are reported
 * without clearing the runtime's last-error state. Every call reuses the same
 * array, so calls whose work overlaps on the GPU (e.g. on two streams at once)
 * race; order them on one stream. */
int smccat_transition_matrices_noalloc(int32_t num_classes, const double* base,
                                       const double* logits, int32_t num_times,
                                       const double* times, double* p_out, void* stream);

/* Create a context over the alignment `codes` [T][S] (row-major, taxon-major).
 * Replaces the data half of Particle::Particle (Particle.cpp:21-73): tip
 * encoding and the invariant-site flags are derived once and shared by all
 * particles. */
int smccat_create(const smccat_config* cfg, const uint8_t* codes, smccat_ctx** out);

int smccat_destroy(smccat_ctx* ctx);

/* Device bytes the context holds. */
int smccat_device_bytes(const smccat_ctx* ctx, uint64_t* bytes);

/* Load full particle states into slots [first, first+count). Replaces
 * Particle::copyFromSerialized (Particle.cpp:218-300) minus its refresh: the
 * SerializedParticle fields (SerializedParticle.hpp:8-17) with the Newick
 * tree given as parent/branch arrays. Arrays are packed per particle:
 *   parent [count][2T-1], branch [count][2T-1], base [count][190],
 *   num_classes [count], logits [count][max_classes][20],
 *   assign [count][S] (class index of each site), pinv [count], shape [count].
 * The loaded particles are marked fully dirty; call smccat_refresh next. */
int smccat_set_particles(smccat_ctx* ctx, int32_t first, int32_t count,
                         const int32_t* parent, const double* branch,
                         const double* base, const int32_t* num_classes,
                         const double* logits, const int32_t* assign,
                         const double* pinv, const double* shape);

/* Read back particle states in the same packed layout (any pointer may be
 * NULL). Replaces Particle::writeToSerialized (Particle.cpp:302-320). */
int smccat_get_particles(smccat_ctx* ctx, int32_t first, int32_t count,
                         int32_t* parent, double* branch, double* base,
                         int32_t* num_classes, double* logits, int32_t* assign,
                         double* pinv, double* shape);

/* Recompute the likelihood of particles [first, first+count).
 * mode SMCCAT_REFRESH_FULL = refreshLikelihood(true): every spectral
 * decomposition, transition matrix and internal CL is rebuilt.
 * mode SMCCAT_REFRESH_DIRTY = refreshLikelihood(false): only what the last
 * edit calls touched (Particle.cpp:537-571); the root reduction always runs.
 * Returns SMCCAT_ENUMERIC if any likelihood is NaN (the values are still
 * stored). Replaces Particle::refreshLikelihood (Particle.cpp:530-675). */
int smccat_refresh(smccat_ctx* ctx, int32_t first, int32_t count, int32_t mode);

/* Copy the current log-likelihoods of [first, first+count) to `out`.
 * Replaces Particle::lnLikelihood (Particle.cpp:480-482). */
int smccat_get_lnl(smccat_ctx* ctx, int32_t first, int32_t count, double* out);

/* Per-site log-likelihoods of particle `p` from its last refresh (S values).
 * The reference keeps no per-site output; this is the parity probe. */
int smccat_get_site_lnl(smccat_ctx* ctx, int32_t p, double* out);

/* Transition matrix P(t r) of particle p, class k, the edge above `node`
 * and rate category r, as 400 row-major doubles (P[i][j] = Pr(j | i)), from
 * the current state after its last refresh. Parity probe for
 * TransitionProbabilityClass::transitionProbabilities
 * (TransitionProbabilityClass.hpp:25, filled at .cpp:83-95). */
int smccat_get_transition_matrix(smccat_ctx* ctx, int32_t p, int32_t k, int32_t node,
                                 int32_t r, double* out400);

/* ---- edits that mark dirty state (the proposal side of the moves) ------ */

/* Set branch lengths of `n` nodes of particle p. Marks the transition
 * matrices of those nodes and the CLs on their paths to the root dirty
 * (Tree::scaleBranchMove / scaleSubtreeMove, Tree.cpp:553-612). */
int smccat_set_branch_lengths(smccat_ctx* ctx, int32_t p, int32_t n,
                              const int32_t* nodes, const double* lengths);

/* Replace the topology of particle p (NNI / SPR, Tree.cpp:625-812). Nodes
 * whose children changed, and their ancestors, are marked CL-dirty. */
int smccat_set_topology(smccat_ctx* ctx, int32_t p, const int32_t* parent,
                        const double* branch);

/* Proportion of invariant sites (Particle::invarMove, Particle.cpp:744-766):
 * only the root reduction reruns. */
int smccat_set_pinv(smccat_ctx* ctx, int32_t p, double pinv);

/* Gamma shape (Particle::shapeMove, Particle.cpp:768-783): rates are
 * re-discretised and every transition matrix and CL is rebuilt. */
int smccat_set_shape(smccat_ctx* ctx, int32_t p, double shape);

/* Exchangeabilities (190 log-rates) of particle p. Every class is
 * re-decomposed and everything downstream rebuilt. */
int smccat_set_base(smccat_ctx* ctx, int32_t p, const double* base);

/* Logits of class k of particle p: that class is re-decomposed and its
 * transition matrices and every CL rebuilt (STATIONARY_SINGLE,
 * Particle.cpp:537-548). */
int smccat_set_class_logits(smccat_ctx* ctx, int32_t p, int32_t k, const double* logits);

/* Accept (mask[i] != 0) or reject (mask[i] == 0) the pending edits of
 * particles [first, first+count) after a refresh. Accept keeps the new state;
 * reject restores the previous state and its likelihood. Both are O(nodes)
 * flag flips on the device -- no buffer copies (the reference copies the whole
 * rescale buffer, Particle.cpp:343-478). */
int smccat_accept(smccat_ctx* ctx, int32_t first, int32_t count, const uint8_t* mask);

/* Synchronise the context's stream. */
int smccat_sync(smccat_ctx* ctx);

/* ---- rejuvenation (MCMC) and the SMC weight step ------------------------ */

/* Proposal tunables shared by the particles of a context: the public members
 * of class Particle (Particle.hpp:87-94) and the DPP concentration
 * (Particle.hpp:106). Defaults: 0.01, 1.0, 1.0, 1.0, 0.25, 0.25, 100.0, 0.01. */
typedef struct smccat_tuning {
    double adaptive_nni_epsilon;   /* aNNIEpsilon                          */
    double shape_delta;            /* shapeDelta                           */
    double scale_delta;            /* scaleDelta (one branch)              */
    double subtree_scale_delta;    /* subtreeScaleDelta                    */
    double stationary_delta;       /* stationaryDelta (logit shift sd)     */
    double rate_matrix_delta;      /* rateMatrixDelta (single-entry move)  */
    double invar_alpha;            /* invarAlpha (beta proposal concentration) */
    double dpp_alpha;              /* dppAlpha                             */
} smccat_tuning;

int smccat_set_tuning(smccat_ctx* ctx, const smccat_tuning* t);
int smccat_get_tuning(smccat_ctx* ctx, smccat_tuning* t);

/* rateMatrixCholesky (Particle.hpp:93, set by main.cpp:267-289): lower
 * triangular 190 x 190, row-major; default 0.5 I. */
int smccat_set_rate_cholesky(smccat_ctx* ctx, const double* lower190x190);
/* The factor in use (190 x 190 row-major, zeros above the diagonal). */
int smccat_get_rate_cholesky(smccat_ctx* ctx, double* lower190x190);

/* Split posterior probabilities for the adaptive NNI move
 * (Tree::adaptiveNNIMove, Tree.cpp:673-766; computeSplitPosteriors,
 * Miscellaneous.hpp:115-150). Split i is a taxon bit set in 2 words
 * (bits[2i] holds taxa 0..63, bits[2i+1] taxa 64..127), canonicalised so that
 * taxon 0 is set (Tree.cpp:511-516). Replaces the previous table. */
int smccat_set_split_posteriors(smccat_ctx* ctx, int32_t n, const uint64_t* bits,
                                const double* prob);

/* computeSplitPosteriors (Miscellaneous.hpp:115-150) over the trees of
 * particles [first, first+count): each particle contributes its clade set
 * (Tree::getSplitSet, Tree.cpp:485-541: the taxon set of every non-root node,
 * canonicalised so that taxon 0 is set, each distinct set once) with weight
 * weights[i], or 1/count when weights is NULL (the resampled-assignment form,
 * Miscellaneous.hpp:135-150). The result replaces the split posteriors the
 * adaptive NNI move reads, as smccat_set_split_posteriors would. *n_out gets
 * the number of distinct splits; if bits and prob are not NULL, the first
 * min(n, cap) of them are written in the layout of smccat_set_split_posteriors,
 * by decreasing probability (ties by bits). At most 128 taxa. */
int smccat_compute_split_posteriors(smccat_ctx* ctx, int32_t first, int32_t count,
                                    const double* weights, int32_t cap, int32_t* n_out,
                                    uint64_t* bits, double* prob);

/* The resampling and proposal-tuning half of an SMC step (main.cpp:176-301).
 * Systematic resampling of [first, first+count) with the normalised weights
 * norm_weights and a uniform draw u in [0, 1) (main.cpp:178-192, the same
 * walk); ancestors[i] (relative to first) is the particle slot i descends from.
 * Then, over the resampled population, the reference's proposal tuning
 * (main.cpp:197-291), installed for smccat_propose / smccat_rejuvenate:
 * shape_delta = max(0.5 var(log shape), 0.01); scale_delta =
 * subtree_scale_delta = max(var(log branch length) over every non-root
 * branch, 0.01); stationary_delta = max(var over every class's 20 logits, 0.01);
 * invar_alpha = 0.5 mean(pinv) (+I models only); and without SMCCAT_MODEL_LG
 * the exchangeability proposal: the uncentred X^T X of the resampled base
 * vectors times 2.38^2/190 * 0.21, shrunk by 0.2 toward its mean diagonal,
 * plus 1e-6 I, Cholesky-factored (SMCCAT_ENUMERIC if not positive definite),
 * with rate_matrix_delta = max(shrinkage, 0.01). Variances are population
 * variances. The split posteriors of the resampled population become the
 * adaptive NNI table (T <= 128). With copy != 0 every slot then takes its
 * ancestor's state (copyFromSerialized, main.cpp:299-301); the next refresh
 * rebuilds the partials. */
int smccat_resample_tune(smccat_ctx* ctx, int32_t first, int32_t count, const double* norm_weights,
                         double u, int32_t copy, int32_t* ancestors);

/* Tree rejuvenation with everything on the device: `steps` lockstep
 * Metropolis-Hastings steps of Particle::treeMove (Particle.cpp:677-701: NNI
 * 0.1, adaptive NNI 0.3, SPR 0.1, scaleBranch 0.4, scaleSubtree 0.1;
 * Tree.cpp:553-812) on every particle of [first, first+count), at
 * `temperature`, with the tuned scale_delta / subtree_scale_delta /
 * adaptive_nni_epsilon and the installed split posteriors. Each step's
 * proposal, dirty-node plan, transition matrices, pruning, reduction and
 * accept/reject run as device kernels with fixed launch shapes; with
 * use_graph != 0 the whole sweep is captured as one CUDA graph and launched
 * once. Draws come from a Philox stream per particle seeded by `seed`.
 * Afterwards the host state holds the final trees and branch lengths. Needs
 * refreshed, committed particles. stats (may be NULL, else 10 entries):
 * stats[2k] proposed and stats[2k+1] accepted moves of kind k =
 * SMCCAT_MOVE_ADAPTIVE_NNI .. SMCCAT_MOVE_SCALE_SUBTREE. */
int smccat_tree_sweep(smccat_ctx* ctx, int32_t first, int32_t count, int32_t steps,
                      double temperature, uint64_t seed, int32_t use_graph, int64_t* stats);

/* Particle::lnPrior (Particle.cpp:484-517) of the current states. */
int smccat_ln_prior(smccat_ctx* ctx, int32_t first, int32_t count, double* out);

/* Move families of the reference's MCMC registry (main.cpp:55-106). */
#define SMCCAT_FAMILY_TREE         0  /* treeMove: NNI / adaptive NNI / SPR / branch / subtree */
#define SMCCAT_FAMILY_STATIONARY   1  /* stationaryMove                    */
#define SMCCAT_FAMILY_SHAPE        2  /* shapeMove                         */
#define SMCCAT_FAMILY_INVAR        3  /* invarMove                         */
#define SMCCAT_FAMILY_RATE_MATRIX  4  /* rateMatrixMove                    */

/* Move kinds, numbered like the reference's UpdateType (Particle.hpp:18-30). */
#define SMCCAT_MOVE_ADAPTIVE_NNI        0
#define SMCCAT_MOVE_NNI                 1
#define SMCCAT_MOVE_SPR                 2
#define SMCCAT_MOVE_BRANCH_LENGTH       3
#define SMCCAT_MOVE_SCALE_SUBTREE       4
#define SMCCAT_MOVE_INVAR               5
#define SMCCAT_MOVE_RATE_SHAPE          6
#define SMCCAT_MOVE_STATIONARY_SINGLE   7
#define SMCCAT_MOVE_RATE_MATRIX_SINGLE  8
#define SMCCAT_MOVE_RATE_MATRIX_FULL    9

typedef struct smccat_move_stats {
    uint64_t proposed[10];   /* per move kind (Particle::moveCount)         */
    uint64_t accepted[10];   /* per move kind (Particle::acceptCount)       */
    uint64_t lockstep_steps; /* batched refreshes issued                     */
} smccat_move_stats;

/* Apply one proposal of `family` to particle p (seeded), leaving it pending:
 * the caller refreshes and accepts/rejects. Writes the move kind and the log
 * Hastings ratio. The proposal half of one MH step of Mcmc::operator(). */
int smccat_propose(smccat_ctx* ctx, int32_t p, int32_t family, uint64_t seed, int32_t* kind,
                   double* hastings);

/* Mcmc::operator()(particle, iterations, tempering) (Mcmc.cpp:25-73) for
 * every particle of [first, first+count), all advancing in lockstep with one
 * batched dirty refresh per MH step. Move weights and repeat counts follow the
 * reference's registry (main.cpp:55-106): tree 3 x floor(T/4), stationary
 * 1 x 2K, shape 1 x 2 (R > 1), invariant 1 x 2 (+I), rate matrix 1 x 5 (GTR).
 * The particles must have no pending edits. */
int smccat_rejuvenate(smccat_ctx* ctx, int32_t first, int32_t count, int32_t iterations,
                      double temperature, uint64_t seed, smccat_move_stats* stats);

/* Mcmc::operator()(particle, iterations, tempering) (Mcmc.cpp:25-73) for every
 * particle of [first, first+count) with everything on the device. Each
 * particle's sequence of moves -- per iteration one draw from the registry of
 * main.cpp:55-106 (tree 3 x floor(T/4), stationary 1 x 2K, shape 1 x 2 when
 * R > 1, invariant 1 x 2 with +I, rate matrix 1 x 5 without LG), repeated its
 * count of times -- is drawn on the host from `seed`; then all particles
 * advance in lockstep through as many steps as the longest sequence (a
 * particle whose sequence has ended idles). Every step's proposals
 * (Particle::treeMove, invarMove, shapeMove, stationaryMove, rateMatrixMove:
 * Particle.cpp:677-783, with the same rules as smccat_propose), spectral
 * decompositions, transition matrices, pruning, reduction and
 * Metropolis-Hastings decisions on temperature * lnL + lnPrior + log Hastings
 * run as device kernels with fixed launch shapes; with use_graph != 0 the
 * whole sweep is captured as one CUDA graph and launched once. Draws come from
 * a Philox stream per particle. Afterwards the host state holds every
 * particle's final tree, branch lengths, exchangeabilities, logits, pinv and
 * shape. Needs refreshed, committed particles (+I models: pinv > 0). stats
 * (may be NULL) gets the per-kind counts and, as lockstep_steps, the number
 * of steps. */
int smccat_mcmc_sweep(smccat_ctx* ctx, int32_t first, int32_t count, int32_t iterations,
                      double temperature, uint64_t seed, int32_t use_graph,
                      smccat_move_stats* stats);

typedef struct smccat_gibbs_stats {
    int64_t particles;       /* particles reassigned                         */
    int64_t classes_before;  /* summed class counts before                   */
    int64_t classes_after;   /* summed class counts after                    */
    int64_t created;         /* classes created from auxiliary draws         */
} smccat_gibbs_stats;

/* Particle::gibbsPartitionMove(temperature) followed by refreshLikelihood(true)
 * (Particle.cpp:785-995, main.cpp:303-306) for the particles of
 * [first, first+count) whose mask byte is non-zero (mask may be NULL = all):
 * Neal's Algorithm 8 with m = 5 auxiliary classes, floor(S/2) random-site
 * iterations per particle, run on the device: every iteration's auxiliary
 * classes evaluated at once, then each particle's iterations in order with the
 * classes' site log-likelihoods from a table the pruning kernels fill. The
 * particles run in groups sized to half the free device memory (the result
 * does not depend on the grouping). Emptied classes are removed and the
 * survivors renumbered in order; new classes are appended. Needs
 * SMCCAT_MODEL_CAT and no pending edits; fails with SMCCAT_ENOMEM if a
 * particle would exceed max_classes. */
int smccat_gibbs(smccat_ctx* ctx, int32_t first, int32_t count, const uint8_t* mask,
                 double temperature, uint64_t seed, smccat_gibbs_stats* stats);

/* The unnormalised log weights one Gibbs iteration would draw from for site
 * `site` of particle p, with the site taken out of its class and the 5
 * auxiliary classes given as logits (5 x 20): K + 5 values, -inf for a class
 * that the removal empties. Nothing is changed. Parity probe for
 * Particle.cpp:857-941. */
int smccat_gibbs_weights(smccat_ctx* ctx, int32_t p, int32_t site, const double* aux_logits,
                         double temperature, double* out);

/* ---- learned CAT class proposal (no reference counterpart: the reference's
 * only reassignment move is the Gibbs sweep above) ----------------------- */

/* Parameter count of the scoring MLP: 44 inputs, two ReLU layers of 128,
 * one linear output; layout W1[44][128], b1, W2[128][128], b2, w3[128], b3. */
#define SMCCAT_MLP_PARAMS 22401
#define SMCCAT_MLP_INPUTS 44

/* Train the scoring MLP (FP32, Adam) on the class assignments of particles
 * [first, first+count) -- the samples plain Gibbs reassignment produces during
 * warm-up -- for `epochs` passes in batches of `batch_sites` sites. The first
 * call initialises the weights (Glorot, seeded). Writes the last epoch's mean
 * softmax cross-entropy. Needs SMCCAT_MODEL_CAT. */
int smccat_learned_train(smccat_ctx* ctx, int32_t first, int32_t count, int32_t epochs,
                         int32_t batch_sites, double lr, uint64_t seed, double* loss_out);

/* Mean softmax cross-entropy and its gradient for a given batch: n_sites
 * groups, group g owning feature rows [group_off[g], group_off[g+1]) of x
 * (rows of SMCCAT_MLP_INPUTS floats) with the correct row labels[g] (relative
 * to the group). Uses the current parameters; changes nothing. */
int smccat_learned_gradients(smccat_ctx* ctx, int32_t n_sites, const int32_t* group_off,
                             const float* x, const int32_t* labels, float* grad_out,
                             double* loss_out);

/* Read (get_out) and/or replace (set_in) the SMCCAT_MLP_PARAMS parameters. */
int smccat_learned_params(smccat_ctx* ctx, float* get_out, const float* set_in);

typedef struct smccat_learned_stats {
    int64_t proposed;
    int64_t accepted;
} smccat_learned_stats;

/* Metropolis-Hastings class reassignment with the learned proposal for the
 * masked particles of [first, first+count): `updates` random-site updates per
 * particle; each proposes a class from the softmax of the MLP scores among the
 * existing classes and accepts with the tempered likelihood ratio, the CRP
 * prior ratio n_b / (n_a - 1) and the proposal ratio, so the posterior is
 * unchanged. Sites whose class would empty are not moved. Then
 * refreshLikelihood(true). The scores run on the tensor cores: BF16 weights,
 * feature rows and hidden activations, FP32 accumulation. */
int smccat_learned_move(smccat_ctx* ctx, int32_t first, int32_t count, const uint8_t* mask,
                        int32_t updates, double temperature, uint64_t seed,
                        smccat_learned_stats* stats);

/* The learned proposal's scores of every class of particle p at `site` (the
 * values smccat_learned_move draws from), into out[num_classes of p]. */
int smccat_learned_scores(smccat_ctx* ctx, int32_t p, int32_t site, double* out);

/* computeNextStep (Miscellaneous.hpp:42-109) in FP64 on the device, on the
 * current log-likelihoods of [first, first+count): bisects the temperature
 * for `target_ess`, updates raw_weights in place and writes the normalised
 * weights, the new temperature and the ESS. */
int smccat_smc_step(smccat_ctx* ctx, int32_t first, int32_t count, double* raw_weights,
                    double target_ess, double last_temp, double* cur_temp, double* ess,
                    double* norm_weights);

/* ---- measurement (no reference counterpart: the reference only has the
 * compile-time TIME_PROFILE wall-clock prints, Particle.cpp:533-631) ----- */

/* The cudaStream_t the context launches on, so a caller can record its own
 * CUDA events on it. */
int smccat_get_stream(smccat_ctx* ctx, void** stream);

#define SMCCAT_KERNEL_SPEC   0
#define SMCCAT_KERNEL_PMAT   1
#define SMCCAT_KERNEL_PRUNE  2
#define SMCCAT_KERNEL_REDUCE 3
#define SMCCAT_KERNEL_ACCEPT 4
#define SMCCAT_NUM_KERNELS   5

typedef struct smccat_profile {
    uint64_t launches[SMCCAT_NUM_KERNELS];  /* kernel launches by kind          */
    double ms[SMCCAT_NUM_KERNELS];          /* summed CUDA-event durations (ms)
                                               when timing is enabled, else 0   */
    uint64_t h2d_bytes;                     /* host->device bytes copied        */
    uint64_t d2h_bytes;                     /* device->host bytes copied        */
} smccat_profile;

/* Time every instantiated pruning-kernel variant (sites per lane, mat-vec
 * schedule, register cap) with `reps` full refreshes of the loaded particles
 * [0, n) and keep the fastest for this context. Writes the chosen variant and,
 * if ms_out is not NULL, the pruning time (ms) of each variant: ms_out needs
 * one entry per variant, as many as smccat_kernel_variants reports. The
 * particles must have no pending edits; their likelihoods are recomputed. */
int smccat_autotune(smccat_ctx* ctx, int32_t reps, int32_t* variant_out, double* ms_out);

/* Number of pruning-kernel variants of this context, the one in use, and a
 * way to pin one (what smccat_autotune sets). The variants are SIMT kernels
 * of several schedules and register caps, persistent forms of the fastest of
 * them at four rate categories, then the FP64 tensor-path kernels (FP64
 * contexts) or the tcgen05 3xTF32 kernel on 128-slot tiles (FP32 contexts).
 * A new context starts on the variant measured fastest on B200. */
int smccat_kernel_variants(smccat_ctx* ctx, int32_t* count, int32_t* current);
int smccat_set_kernel_variant(smccat_ctx* ctx, int32_t variant);

/* Polls a pruning kernel's bounded device waits (for its staged transition
 * matrices, or its tensor-core products) make before giving up; polls < 0
 * restores the default (4,194,304). A wait that gives up makes the refresh
 * return SMCCAT_ETIMEOUT with NaN likelihoods, after the kernel has drained
 * the copies it had in flight; the next refresh with a sufficient limit is
 * unaffected. 0 makes every wait give up at once, which exercises that path
 * without stalling or faulting the device. No counterpart in the reference
 * (it has no device code). */
int smccat_set_wait_limit(smccat_ctx* ctx, int32_t polls);

/* Particles per device pass of smccat_gibbs / smccat_learned_move: n > 0 fixes
 * the group size, n <= 0 restores the default (groups sized to half the free
 * device memory). The results do not depend on it. No counterpart in the
 * reference. */
int smccat_set_reassign_group(smccat_ctx* ctx, int32_t n);

/* Enable (1) or disable (0) per-launch CUDA-event timing; resets counters. */
int smccat_set_profiling(smccat_ctx* ctx, int32_t enable);

/* Counters since the last smccat_set_profiling call (synchronises). */
int smccat_get_profile(smccat_ctx* ctx, smccat_profile* out);

#ifdef __cplusplus
}
#endif

#endif /* SMCCAT_H */
