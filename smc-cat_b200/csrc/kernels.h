// Kernel launch interface of the B200 likelihood engine (host <-> device).
#pragma once
#include <cuda_runtime.h>

#include "smccat_internal.h"

namespace smccat {

// mbarrier polls before a bounded device wait gives up (a pruning kernel's
// wait for its staged transition matrices or tensor-core products), and the
// polls a kernel then spends draining the copies it still has in flight.
constexpr uint32_t kDrainPolls = 1u << 22;

struct Dims {
    int T, S, Spad, R, N, NI, Kmax;
};

// The byte of the spectral-workspace array of (particle p, class k): bit 0 is
// the class's spectral workspace; bits 1 and 2 flip the partial and
// transition-matrix workspaces of that class's sites and matrices. A
// class-local move (one class's stationary frequencies) rebuilds that class
// alone into the other workspaces by flipping those bits, leaving the node
// workspace indices, and so every other class, untouched.
constexpr uint8_t kSwsSpec = 1, kSwsCl = 2, kSwsP = 4;
#ifdef __CUDACC__
// NodeJob.ws bits to flip for a tile or matrix of class k: the three partial
// workspaces (node, child 1, child 2) with bit 1, the two matrix ones with bit 2.
__device__ __forceinline__ int class_ws_flip(const uint8_t* sws, int p, int Kmax, int k) {
    const int b = sws[(size_t)p * Kmax + k];
    return ((b & kSwsCl) ? 7 : 0) | ((b & kSwsP) ? 24 : 0);
}
#endif

struct PruneArgs {
    Dims d;
    int first;        // first particle of the refresh range (hdr index base)
    int tile_begin;   // first global tile of the range
    const Tile* tiles;
    const PartHdr* hdr;
    const NodeJob* nodes;
    const uint8_t* codes;
    const int32_t* perm;
    const int32_t* wt;  // sites per slot [P][S] under site-pattern compression, else null
    const void* Pm;   // double, or float when fp32
    const double* spec;
    const uint8_t* sws;
    const double* isinv;
    const int32_t* invchar;
    void* CL;         // double, or float when fp32; written and re-read inside one
                      // launch, so never read through the non-coherent path
    int fp32;         // mixed precision: FP32 partials and matrices
    double* LSC;
    double* site_lnl;
    double* partial;
    int* status;      // bit 1: NaN likelihood, bit 2: a bounded wait gave up
    uint32_t wait_limit;  // polls per bounded wait (kDrainPolls unless a test lowers it)
    // Evaluation mode (eval_k >= 0, SIMT kernels only): every tile is pruned
    // under class eval_k instead of its own class and each site's
    // log-likelihood goes to eval_out[j][Kmax][S], j = eval_map[p - first]
    // (particles with j < 0, or fewer classes, are skipped); the tile
    // partials are not written. The plan's partial workspaces are scratch.
    int eval_k = -1;
    const int32_t* eval_map = nullptr;
    double* eval_out = nullptr;
    // Per-particle evaluation: when set, particle p is evaluated under class
    // eval_kp[p - first] (any slot below Kmax whose matrices and spectral
    // record are in place; -1 skips the particle) and eval_k is not used.
    const int32_t* eval_kp = nullptr;
    // Evaluation over site lists: when set, slot j of particle p's tiles stands
    // for site eval_perm[(p - first) S + j] and slots at or past
    // eval_nv[p - first] are not evaluated. The tiles keep the committed
    // layout's columns, so each column's free workspace is the one its own
    // class's flips name.
    const int32_t* eval_perm = nullptr;
    const int32_t* eval_nv = nullptr;
};

cudaError_t launch_spec(const SpecJob* jobs, int n, double* spec, const Dims& d, cudaStream_t st);
cudaError_t launch_pmat(const PmJob* mjobs, int n, const PJob* jobs, const PartHdr* hdr, int first,
                        const uint8_t* sws, const double* spec, void* Pm, bool fp32, const Dims& d,
                        cudaStream_t st);
// Pruning kernel variants available for R rate categories: SIMT kernels at
// several register caps, then the FP64 tensor-path kernels (FP64) or the
// tcgen05 3xTF32 kernel (FP32).
int prune_variants(int R, bool fp32);
// Slots per pruning tile that a variant expects (32, 64 or 128).
int prune_variant_tile_sites(int R, bool fp32, int variant);
// The variant used until smccat_autotune or smccat_set_kernel_variant picks
// another: the fastest measured on B200 for the bench workloads.
int prune_default_variant(int R, bool fp32);
cudaError_t launch_prune(const PruneArgs& a, int ntiles, int variant, cudaStream_t st);
// Whether a variant is one of the SIMT kernels (the ones with evaluation mode).
bool prune_variant_has_eval(int R, bool fp32, int variant);
int prune_dmma_variants(int R);
cudaError_t launch_prune_dmma(const PruneArgs& a, int ntiles, int variant, cudaStream_t st);
// FP32 tensor-core (tcgen05, 3xTF32) kernels: 128-slot tiles.
int prune_tc_variants(int R);
cudaError_t launch_prune_tc(const PruneArgs& a, int ntiles, int variant, cudaStream_t st);
cudaError_t launch_reduce(const int32_t* tile_off, const double* partial, const PartHdr* hdr, int first,
                          int count, double* lnl, int* status, cudaStream_t st);
cudaError_t launch_accept(double* lnl, double* lnl_old, const uint8_t* mask, int first, int count,
                          cudaStream_t st);

}  // namespace smccat
