// Shared host/device definitions of the B200 likelihood engine.
//
// Device layout (one context = one batch of particles on one GPU):
//   codes   [T][S]                      uint8 alignment codes (shared)
//   perm    [P][S]                      slot -> site, sites grouped by class
//   CL      [P][T-1][2][20][R][Spad]    internal-node partials, 2 workspaces,
//                                       state-major so a warp of 32 slots
//                                       reads 256 contiguous bytes per state
//   LSC     [P][T-1][2][R][Spad]        cumulative log scale of each node's
//                                       subtree (own scaler + children's)
//   Pm      [P][Kmax][N][2][R][20][22]  transition matrices, row-major with a
//                                       row stride of 22: column 20 holds the
//                                       row sums (P applied to the all-ones
//                                       tip vector of gap / X / ?), column 21
//                                       is padding so rows are 16-byte aligned
//   spec    [P][Kmax][2][SPEC_STRIDE]   eigenvalues, left/right factors, pi
// Every workspace index (CL, P, spectral) is chosen by the host mirror and
// shipped in the per-refresh plan, so accept/reject never touches the device.
// The partial and matrix workspace of (node, class) is the node's index XOR
// the class's flip bit (bits 1 and 2 of its spectral-workspace byte).
#pragma once
#include <stdint.h>

#include <string>

namespace smccat {

// Record the message smccat_last_error() returns on this thread.
void set_last_error(const std::string& msg);

constexpr int kStates = 20;
constexpr int kBase = 190;
constexpr int kPCols = 22;                      // P row: 20 entries, row sum, pad
constexpr int kPBlock = kStates * kPCols;       // 440 doubles per (node, rate)
constexpr int kMaxRates = 8;
constexpr int kTileSites = 32;                  // sites per pruning tile (one warp per rate)
constexpr int kSpecStride = 20 + 400 + 400 + 20 + 8;  // lam, L, Rm, pi, pad

// Offsets inside one spectral record.
constexpr int kSpecLam = 0;
constexpr int kSpecL = 20;
constexpr int kSpecRm = 420;
constexpr int kSpecPi = 820;

struct PartHdr {
    int32_t node_off;   // first NodeJob of this particle in the plan
    int32_t node_cnt;   // dirty internal nodes, post-order, root last
    int32_t root;       // root node id
    int32_t root_ws;    // CL workspace of the root after this refresh
    int32_t active;     // 0: particle not part of this refresh
    int32_t num_classes;
    int32_t cls_only;   // >= 0: a class-local refresh of that class; the other
                        // classes' tiles only re-run the root reduction
    int32_t pad1;
    double pinv;
    double rates[kMaxRates];
};

// One dirty internal node. ws bits: 0 out CL ws, 1 child1 CL ws, 2 child2
// CL ws, 3 child1 P ws, 4 child2 P ws.
struct NodeJob {
    int32_t node, c1, c2, ws;
};

// Rebuild the transition matrices of one node (all classes, all rates).
struct PJob {
    int32_t p, node, pws, pad;
    double t;           // branch length
};

// One transition-matrix CTA: class k of plan particle i, for the PJobs
// [j0, j0 + nj) of that particle (at most kPmChunk nodes).
constexpr int kPmChunk = 16;
struct PmJob {
    int32_t i, k, j0, nj;
};

// Re-decompose one class.
struct SpecJob {
    int32_t p, k, sws, pad;
    double base[kBase];
    double logits[kStates];
};

// A pruning tile: up to kTileSites consecutive slots of one class.
struct Tile {
    int32_t p, k, slot0, nslots;
};

}  // namespace smccat
