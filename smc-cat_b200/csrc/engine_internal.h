// Internal state of the host engine, shared by the C-ABI implementation
// (engine.cu) and the MCMC driver (mcmc.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <algorithm>
#include <vector>

#include <omp.h>
#include <nvtx3/nvToolsExt.h>

#include "kernels.h"
#include "smccat.h"

namespace smccat {

// A named NVTX range for the lifetime of the object: the entry points mark
// their work for a profiler's timeline (no cost without one attached), where
// the reference prints TIME_PROFILE timings (Particle.cpp:533-631).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Host loops over at least this many particles (state upload, plan packing,
// proposals and MH tests) run on OpenMP threads; each iteration touches only
// its own particle's slot.
constexpr int kParallelParticles = 32;
// Host threads for per-particle loops: a quarter of the cores stay free for
// the caller's and the CUDA driver's threads (a full team that loses one core
// to them stalls every parallel region for a scheduler time slice).
inline int host_team() {
    const int t = omp_get_max_threads();
    return std::max(1, t - std::max(1, t / 4));
}
constexpr int kPackThreads = 4;  // threads packing a refresh plan

// Host mirror of one particle's state and of its device workspace indices.
struct Mirror {
    std::vector<int32_t> parent;   // N
    std::vector<double> branch;    // N
    std::vector<int32_t> kids;     // 2N, -1 for tips
    std::vector<int32_t> post;     // internal nodes, post-order (root last)
    int root = -1;
    std::vector<double> base;      // 190
    int K = 0;
    std::vector<double> logits;    // Kmax * 20
    double pinv = 0.0, shape = 1.0;
    double rates[kMaxRates] = {1, 1, 1, 1, 1, 1, 1, 1};
    std::vector<uint8_t> clws, pws;  // N
    std::vector<uint8_t> sws;        // Kmax
};

struct Slot {
    Mirror cur, old;
    std::vector<int32_t> assign;
    std::vector<int32_t> class_cnt;  // slots per class, kept with `assign`
    std::vector<int32_t> site_rep;   // site-pattern compression: the site each site's
                                     // slot evaluates (its value stands for this one)
    std::vector<uint8_t> dirty_cl, dirty_p, dirty_spec;
    bool loaded = false;
    bool full = false;          // next refresh rebuilds everything
    bool commit_on_refresh = false;
    bool pending = false;       // edits since the last commit
    bool refreshed = false;     // refreshed since the last commit
    int local_class = -1;       // >= 0: the only pending edit is that class's logits,
                                // refreshed class-locally (its own workspace flips)
};

// Refresh particles [first, first+count); `active` (count bytes, may be
// null) excludes particles from the launch without touching their state.
int refresh_internal(smccat_ctx* c, int first, int count, int mode, const uint8_t* active);

// Host mirror of one slot (read-only view for the MCMC driver).
const Slot& slot_of(const smccat_ctx* c, int p);
int particles_of(const smccat_ctx* c);  // particle slots of the context
const Dims& dims_of(const smccat_ctx* c);
int model_flags_of(const smccat_ctx* c);
uint32_t wait_limit_of(const smccat_ctx* c);  // polls per bounded device wait
int device_of(const smccat_ctx* c);            // the context's CUDA device
int reassign_group_of(const smccat_ctx* c);    // smccat_set_reassign_group (0: default)
const double* lnl_device(const smccat_ctx* c);  // [max_particles] current log-likelihoods
const uint8_t* codes_device(const smccat_ctx* c);   // [T][S]
const double* isinv_device(const smccat_ctx* c);    // [S]
const int32_t* invchar_device(const smccat_ctx* c); // [S]

const uint8_t* codes_host(const smccat_ctx* c);     // [T][S]

// Drop the MCMC settings kept for a context (called by smccat_destroy).
void mcmc_release(const smccat_ctx* c);
// Drop the learned proposal kept for a context (called by smccat_destroy).
void learned_release(const smccat_ctx* c);
// BF16 MLP parameters and the device site features, or null if untrained.
const void* learned_inference_weights(const smccat_ctx* c, const float** site_feat);

// Device buffers of a particle range for kernels launched outside
// refresh_internal (the device-side moves): a pruning argument block with
// everything but hdr / nodes filled in, the launch shape, and what the
// transition-matrix and reduction kernels read. Needs a current tile list.
struct DeviceView {
    PruneArgs pa;
    int ntiles = 0, variant = 0;
    double* lnl = nullptr;
    double* lnl_old = nullptr;
    const int32_t* tile_off = nullptr;  // device
    const uint8_t* sws = nullptr;
    const double* spec = nullptr;
    void* Pm = nullptr;
    bool fp32 = false;
    int* status = nullptr;
    cudaStream_t st = nullptr;
};
int device_view(smccat_ctx* c, int first, int count, DeviceView* v);
// Mutable host mirror of one slot (the device-side moves write their results back).
Slot& slot_mut(smccat_ctx* c, int p);
// Children, internal post-order and root of a mirror from a parent array;
// false if it is not a rooted binary tree over 2T-1 nodes.
bool rebuild_tree(int T, const int32_t* parent, Mirror* m);
// Device buffer of at least `bytes` owned by the context (kept between calls,
// reallocated only to grow; freed with the context). nullptr if out of memory.
unsigned char* moves_buffer(smccat_ctx* c, size_t bytes);
// The adaptive-NNI split table in use: canonical splits (2 words each) sorted
// by (word 0, word 1), with their posterior probabilities.
void split_table(const smccat_ctx* c, std::vector<uint64_t>* keys, std::vector<double>* prob);

}  // namespace smccat
