// Device CAT reassignment (Neal's Algorithm 8) -- launch interface.
#pragma once
#include <cuda_runtime.h>

#include "kernels.h"

namespace smccat {

struct GibbsPart {
    int32_t p;          // particle index (seeds its random stream)
    int32_t K;          // classes on entry (slots 0..K-1)
    int32_t n_iter;     // site iterations (floor(S / 2))
    int32_t fixed_site; // >= 0: evaluate this site once and only report weights
    double pinv;
    double rates[kMaxRates];
};

// One internal node of a particle's post-order with the stash slots of its
// result and of its internal children (-1 for a tip). Slots are handed out
// from a free list in post-order, so a pass over a tree needs only as many
// slots as it ever has results waiting for their parent.
struct GibbsNode {
    int32_t n, c[2], so;
    int32_t sc[2], pad[2];
};

struct GibbsArgs {
    Dims d;
    int count;
    int Kcap;               // class slots per particle (live + retired), excluding the aux
    double temp;            // SMC tempering applied to the site log-likelihood
    double alpha;           // DPP concentration
    unsigned long long seed;
    const GibbsPart* parts; // [count]
    const GibbsNode* nodes; // [count][T-1] in post-order
    int nslots;             // stash slots a pass needs (maximum over the particles)
    const double* branch;   // [count][2T-1]
    const double* base;     // [count][190]
    double* logits;         // [count][Kcap + aux][20]: in = slots 0..K-1, out = all slots used
    int32_t* assign;        // [count][S] in / out (slot indices)
    int32_t* counts;        // [count][Kcap + aux] out
    int32_t* kout;          // [count] out: slots used
    const double* aux_in;   // weights mode: [count][aux][20] auxiliary logits (else null)
    double* weights_out;    // weights mode: [count][Kcap + aux] (else null)
    const uint8_t* codes;
    const double* isinv;
    const int32_t* invchar;
    int* status;            // bit 4: class capacity exhausted; bit 8: a bounded wait gave up
    uint32_t wait_limit;    // polls per bounded wait
    // Optional [count][Kt][S]: every site's log-likelihood (+I mixed) under each
    // class the particle enters with, evaluated beforehand by the pruning
    // kernels; those classes then need no single-site pruning per iteration.
    const double* table;
    int Kt;
    // Table mode: a pass runs in rounds. A particle stops at a birth into a
    // slot below Kt, with the new class's spectral record written to the
    // engine's spectral workspace (eng_spec, half from eng_sws) and the slot in
    // born[i]; the caller evaluates that class's table column with the pruning
    // kernels and relaunches, and the particle resumes at resume_it[i] with
    // resume_kcur[i] slots. born[i] = -1 once the particle has finished.
    int32_t* resume_it;
    int32_t* resume_kcur;
    int32_t* born;
    double* eng_spec;
    const uint8_t* eng_sws;
    // scratch, set by launch_gibbs / launch_learned_move
    double* spec;
    double* stash;
    double* aux_ls;         // [count][n_iter][aux]: site log-likelihood under each auxiliary class
    int32_t* aux_site;      // [count][n_iter]: the site each iteration draws
    double* aux_rec;        // spectral records of the auxiliary-class kernel's warps
    double* aux_stash;      // stash of the auxiliary-class kernel's warps
};

// Scratch doubles of one call: `n_iter` site iterations per particle, a
// post-order needing `nslots` stash slots; `aux` for a Gibbs pass (auxiliary
// classes evaluated beforehand), not for the learned move.
size_t gibbs_scratch_doubles(const Dims& d, int count, int Kcap, int n_iter, int nslots, bool aux);
int gibbs_aux();
// A Gibbs pass: the auxiliary-class kernel (every iteration's drawn site and
// auxiliary classes, all at once), then one sequential CTA per particle.
cudaError_t launch_gibbs(GibbsArgs a, int n_iter, double* scratch, cudaStream_t st);
// Its two parts: the auxiliary-class kernel, and one round of the sequential
// kernel (table mode runs it until no particle stops at a new class).
cudaError_t launch_gibbs_aux(GibbsArgs a, int n_iter, double* scratch, cudaStream_t st);
cudaError_t launch_gibbs_resume(GibbsArgs a, int n_iter, double* scratch, cudaStream_t st);
// The sites a learned-move pass draws (into the scratch's drawn-site array).
cudaError_t launch_draw_sites(GibbsArgs a, int n_iter, double* scratch, cudaStream_t st);
// Each particle's distinct drawn sites in increasing order into row qrow[i] of
// the evaluation site lists `list` [rows][S] (the rest of the row zero), their
// count into nv[qrow[i]]; flags: [count][S] bytes of scratch.
cudaError_t launch_visited_sites(GibbsArgs a, int n_iter, double* scratch, const int32_t* qrow, uint8_t* flags,
                                 int32_t* list, int32_t* nv, cudaStream_t st);

// Learned-proposal MH site reassignment: parts[i].n_iter updates per particle
// among its existing classes, proposals from the scoring MLP (BF16 weights
// `mlp`, site features [S][21]); accepted / proposed counts per particle.
// With a class table (GibbsArgs::table) the two classes' site values are read
// from it; without one they are pruned per update.
cudaError_t launch_learned_move(GibbsArgs a, int n_iter, const void* mlp, const float* site_feat,
                                int32_t* n_acc, int32_t* n_prop, double* scratch, cudaStream_t st);

}  // namespace smccat
