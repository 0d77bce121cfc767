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

struct GibbsArgs {
    Dims d;
    int count;
    int Kcap;               // class slots per particle (live + retired), excluding the aux
    double temp;            // SMC tempering applied to the site log-likelihood
    double alpha;           // DPP concentration
    unsigned long long seed;
    const GibbsPart* parts; // [count]
    const int32_t* tree;    // [count][T-1][3]: internal node, child 1, child 2 in post-order
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
    int* status;            // bit 4: class capacity exhausted
    // Optional [count][Kt][S]: every site's log-likelihood (+I mixed) under each
    // class the particle enters with, evaluated beforehand by the pruning
    // kernels; those classes then need no single-site pruning per iteration.
    const double* table;
    int Kt;
    // scratch, set by launch_gibbs
    double* spec;
    double* expt;
    double* stash;
};

size_t gibbs_scratch_doubles(const Dims& d, int count, int Kcap);
int gibbs_aux();
cudaError_t launch_gibbs(GibbsArgs a, double* scratch, cudaStream_t st);

// Learned-proposal MH site reassignment: parts[i].n_iter updates per particle
// among its existing classes, proposals from the scoring MLP (BF16 weights
// `mlp`, site features [S][21]); accepted / proposed counts per particle.
cudaError_t launch_learned_move(GibbsArgs a, const void* mlp, const float* site_feat,
                                int32_t* n_acc, int32_t* n_prop, double* scratch, cudaStream_t st);

}  // namespace smccat
