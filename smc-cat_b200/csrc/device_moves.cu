// Tree moves on the device, a whole sweep captured as one CUDA graph.
//
// The host MCMC driver (mcmc.cu) proposes every move on host mirrors and packs
// each step's plan on the host. Here three moves of the reference's tree-move
// mixture -- Tree::scaleBranchMove, Tree::scaleSubtreeMove (Tree.cpp:553-612)
// and Tree::NNIMove (Tree.cpp:625-671), 0.4, 0.1 and 0.1 of
// Particle::treeMove (Particle.cpp:682-701), so 4 : 1 : 1 here -- run for
// every particle of a range in lockstep with nothing on the host between steps:
//
//   dm_propose_kernel   one thread per particle: Philox draws, the array edit of
//                       the flattened tree (branch lengths, or for NNI the
//                       swap of one child of x with x's sibling in the parent
//                       and child tables), the dirty sets (scaled nodes'
//                       transition matrices; the subtree's internal partials,
//                       or x for NNI, and every ancestor), the plan in
//                       post-order with the next workspaces, the tree-length
//                       prior change and the log Hastings ratio;
//   pmat_kernel, prune_kernel, reduce_kernel
//                       the engine's kernels on that device-built plan, with
//                       launch shapes fixed by the range (empty job slots exit);
//   dm_mh_kernel        one thread per particle: Metropolis-Hastings on
//                       temperature * lnL + lnPrior + log Hastings (Mcmc.cpp:57-60);
//                       accept commits the new workspaces, reject restores the
//                       branch lengths or the parent / child tables (the dirty
//                       work sits in the other workspace, as on the host path).
//
// A sweep of B steps is B repetitions of this fixed sequence, captured into a
// CUDA graph and launched once. At the end the host mirrors take the final
// trees (children and post-order regenerated from the parent tables), branch
// lengths and committed workspaces back.
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <math.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "kernels.h"
#include "smccat.h"

namespace smccat {
namespace {

constexpr int kDmThreads = 64;

struct DmArgs {
    Dims d;
    int first, count, nchunk;
    int32_t* parent;     // [count][N]
    int32_t* kids;       // [count][2N]
    int32_t* nni;        // [count][6] x, a, n1, n2 and their child-slot indices
    double* branch;      // [count][N]
    uint8_t* clws;       // [count][N] committed partial workspace of each node
    uint8_t* pws;        // [count][N] committed transition-matrix workspace
    uint8_t* cur_clws;   // [count][N] workspaces of this step's proposal
    uint8_t* cur_pws;
    uint8_t* dirty;      // [count][N] bit 0: P, bit 1: partial
    int32_t* stack;      // [count][N] subtree walk
    int32_t* undo_node;  // [count][N] scaled nodes, walk order
    double* undo_len;    // [count][N] their previous lengths
    int32_t* nundo;      // [count]
    int32_t* kind;       // [count] 0 scaleBranch, 1 scaleSubtree, 2 NNI
    double* extra;       // [count] lnPrior change + log Hastings ratio
    const PartHdr* hdr0; // [count] root, classes, pinv, rates
    PartHdr* hdr;        // [count] this step's
    NodeJob* nodes;      // [count][NI]
    PJob* pjobs;         // [count][N]
    PmJob* mjobs;        // [count][Kmax][nchunk]
    curandStatePhilox4_32_10_t* rng;  // [count]
    double* lnl;         // engine arrays, [max_particles]
    double* lnl_old;
    unsigned long long* stats;  // proposed / accepted, per kind (6)
    double scale_delta, subtree_delta, temp;
};

__global__ void dm_init_kernel(curandStatePhilox4_32_10_t* rng, int count, int first, unsigned long long seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) curand_init(seed, (unsigned long long)(first + i), 0ull, &rng[i]);
}

__global__ void __launch_bounds__(kDmThreads) dm_propose_kernel(DmArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.count) return;
    const Dims& d = a.d;
    const int N = d.N, T = d.T, NI = d.NI;
    int32_t* par = a.parent + (size_t)i * N;
    int32_t* kids = a.kids + (size_t)i * 2 * N;
    double* br = a.branch + (size_t)i * N;
    uint8_t* dirty = a.dirty + (size_t)i * N;
    int32_t* stk = a.stack + (size_t)i * N;
    int32_t* un = a.undo_node + (size_t)i * N;
    double* ul = a.undo_len + (size_t)i * N;
    const PartHdr h0 = a.hdr0[i];
    const int root = h0.root;
    curandStatePhilox4_32_10_t rs = a.rng[i];

    double L0 = 0.0;
    for (int n = 0; n < N; ++n) {
        dirty[n] = 0;
        L0 += br[n];
    }
    const double v = curand_uniform_double(&rs);  // 0.4 : 0.1 : 0.1 (Particle.cpp:682-701)
    const int kind = v <= 4.0 / 6.0 ? 0 : (v <= 5.0 / 6.0 ? 1 : 2);
    const bool subtree = kind == 1;
    int x = root;
    for (int tries = 0; tries < 64 && (x == root || (kind == 2 && x < T)); ++tries)
        x = min(N - 1, (int)((1.0 - curand_uniform_double(&rs)) * N));  // uniform node
    if (x == root || (kind == 2 && x < T))  // (after 64 misses) the first admissible node
        for (int n = (kind == 2 ? T : 0); n < N; ++n)
            if (n != root) { x = n; break; }
    if (kind == 2) {
        // NNIMove (Tree.cpp:625-671): one child n1 of x trades places with x's
        // sibling n2; branch lengths stay with their nodes, so no P changes.
        const int pa = par[x];
        const int s1 = curand_uniform_double(&rs) <= 0.5 ? 0 : 1;
        const int n1 = kids[2 * x + s1];
        const int s2 = kids[2 * pa] == x ? 1 : 0;
        const int n2 = kids[2 * pa + s2];
        par[n1] = pa;
        par[n2] = x;
        kids[2 * pa + s2] = n1;
        kids[2 * x + s1] = n2;
        int32_t* u6 = a.nni + (size_t)i * 6;
        u6[0] = x; u6[1] = pa; u6[2] = n1; u6[3] = n2; u6[4] = s1; u6[5] = s2;
        a.nundo[i] = 0;
        a.kind[i] = 2;
        dirty[x] |= 2;
        for (int y = pa, g = 0; y >= 0 && g < N; y = par[y], ++g) dirty[y] |= 2;
    }
    const double sc = kind == 2 ? 1.0
                                : exp((subtree ? a.subtree_delta : a.scale_delta) * (curand_uniform_double(&rs) - 0.5));
    // Scale x's branch, or every branch of x's subtree (walk order: pre-order
    // with the second child first; reversed it is a post-order).
    int nch = 0, top = 0;
    if (kind != 2) stk[top++] = x;
    while (top > 0) {  // every node is pushed once: top <= N, nch <= N
        const int n = stk[--top];
        un[nch] = n;
        ul[nch] = br[n];
        ++nch;
        br[n] *= sc;
        dirty[n] |= 1;
        if (subtree && n >= T) {
            stk[top++] = kids[2 * n];
            stk[top++] = kids[2 * n + 1];
        }
    }
    if (kind != 2) {
        a.nundo[i] = nch;
        a.kind[i] = subtree ? 1 : 0;
        if (subtree)
            for (int q = 0; q < nch; ++q)
                if (un[q] >= T) dirty[un[q]] |= 2;
        for (int y = par[x], g = 0; y >= 0 && g < N; y = par[y], ++g) dirty[y] |= 2;
    }
    const uint8_t* kc = a.clws + (size_t)i * N;
    const uint8_t* kp = a.pws + (size_t)i * N;
    uint8_t* cc = a.cur_clws + (size_t)i * N;
    uint8_t* cp = a.cur_pws + (size_t)i * N;
    for (int n = 0; n < N; ++n) {
        cc[n] = (dirty[n] & 2) ? 1 - kc[n] : kc[n];
        cp[n] = (dirty[n] & 1) ? 1 - kp[n] : kp[n];
    }
    // Plan: the subtree's internal nodes in post-order, then x's ancestors up
    // to the root; each node's children are done before it.
    NodeJob* nj = a.nodes + (size_t)i * NI;
    int nn = 0;
    auto emit = [&](int n) {
        const int c1 = kids[2 * n], c2 = kids[2 * n + 1];
        int ws = cc[n];
        if (c1 >= T) ws |= cc[c1] << 1;
        if (c2 >= T) ws |= cc[c2] << 2;
        ws |= cp[c1] << 3;
        ws |= cp[c2] << 4;
        if (nn < NI) nj[nn++] = NodeJob{n, c1, c2, ws};
    };
    if (subtree)
        for (int q = nch - 1; q >= 0; --q)
            if (un[q] >= T) emit(un[q]);
    if (kind == 2) emit(x);  // x's new children are clean; then its ancestors
    for (int y = par[x], g = 0; y >= 0 && g < N; y = par[y], ++g) emit(y);
    PJob* pj = a.pjobs + (size_t)i * N;
    for (int q = 0; q < nch; ++q) pj[q] = PJob{a.first + i, un[q], cp[un[q]], 0, br[un[q]]};
    PmJob* mj = a.mjobs + (size_t)i * d.Kmax * a.nchunk;
    for (int k = 0; k < d.Kmax; ++k)
        for (int c = 0; c < a.nchunk; ++c) {
            const int nj_k = k < h0.num_classes ? max(0, min(kPmChunk, nch - kPmChunk * c)) : 0;
            mj[k * a.nchunk + c] = PmJob{i, k, i * N + kPmChunk * c, nj_k};
        }
    PartHdr h = h0;
    h.node_off = i * NI;
    h.node_cnt = nn;
    h.root_ws = cc[root];
    h.active = 1;
    a.hdr[i] = h;
    double L1 = 0.0;
    for (int n = 0; n < N; ++n) L1 += br[n];
    // Tree-length prior Gamma(2T-2, scale 1/10) (Particle.cpp:484-517) and the
    // Hastings ratio of a multiplicative scale of nch branches.
    a.extra[i] = (N - 2) * (log(L1) - log(L0)) - (L1 - L0) / 0.1 + nch * log(sc);
    a.rng[i] = rs;
}

__global__ void __launch_bounds__(kDmThreads) dm_mh_kernel(DmArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.count) return;
    const int N = a.d.N, p = a.first + i;
    curandStatePhilox4_32_10_t rs = a.rng[i];
    const double ratio = a.temp * (a.lnl[p] - a.lnl_old[p]) + a.extra[i];
    const bool ok = log(curand_uniform_double(&rs)) <= ratio;  // NaN ratios reject
    const uint8_t* dirty = a.dirty + (size_t)i * N;
    const int kind = a.kind[i];
    atomicAdd(&a.stats[2 * kind], 1ull);
    if (ok) {
        a.lnl_old[p] = a.lnl[p];
        uint8_t* kc = a.clws + (size_t)i * N;
        uint8_t* kp = a.pws + (size_t)i * N;
        for (int n = 0; n < N; ++n) {
            if (dirty[n] & 2) kc[n] = a.cur_clws[(size_t)i * N + n];
            if (dirty[n] & 1) kp[n] = a.cur_pws[(size_t)i * N + n];
        }
        atomicAdd(&a.stats[2 * kind + 1], 1ull);
    } else if (kind == 2) {
        a.lnl[p] = a.lnl_old[p];
        const int32_t* u6 = a.nni + (size_t)i * 6;
        int32_t* par = a.parent + (size_t)i * N;
        int32_t* kids = a.kids + (size_t)i * 2 * N;
        par[u6[2]] = u6[0];
        par[u6[3]] = u6[1];
        kids[2 * u6[1] + u6[5]] = u6[3];
        kids[2 * u6[0] + u6[4]] = u6[2];
    } else {
        a.lnl[p] = a.lnl_old[p];
        double* br = a.branch + (size_t)i * N;
        const int32_t* un = a.undo_node + (size_t)i * N;
        const double* ul = a.undo_len + (size_t)i * N;
        for (int q = a.nundo[i] - 1; q >= 0; --q) br[un[q]] = ul[q];
    }
    a.rng[i] = rs;
}

int dm_fail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

}  // namespace
}  // namespace smccat

using namespace smccat;

extern "C" int smccat_branch_sweep(smccat_ctx* c, int32_t first, int32_t count, int32_t steps,
                                   double temperature, uint64_t seed, int32_t use_graph,
                                   int64_t* stats) {
    if (!c) return dm_fail(SMCCAT_EINVAL, "null context");
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

    // Host images of the trees and committed workspaces.
    std::vector<int32_t> par((size_t)count * N), kids((size_t)count * 2 * N);
    std::vector<double> br((size_t)count * N);
    std::vector<uint8_t> clws((size_t)count * N), pws((size_t)count * N);
    std::vector<PartHdr> hdr0(count);
    for (int i = 0; i < count; ++i) {
        const Mirror& m = slot_of(c, first + i).cur;
        std::copy(m.parent.begin(), m.parent.end(), &par[(size_t)i * N]);
        std::copy(m.kids.begin(), m.kids.end(), &kids[(size_t)i * 2 * N]);
        std::copy(m.branch.begin(), m.branch.end(), &br[(size_t)i * N]);
        std::copy(m.clws.begin(), m.clws.end(), &clws[(size_t)i * N]);
        std::copy(m.pws.begin(), m.pws.end(), &pws[(size_t)i * N]);
        PartHdr& h = hdr0[i];
        std::memset(&h, 0, sizeof(h));
        h.root = m.root;
        h.num_classes = m.K;
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
    a.temp = temperature;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off = (off + bytes + 255) & ~size_t(255); return o; };
    const size_t cN = (size_t)count * N;
    const size_t o_par = take(cN * 4), o_kids = take(2 * cN * 4), o_nni = take((size_t)count * 6 * 4),
                 o_br = take(cN * 8), o_clws = take(cN),
                 o_pws = take(cN), o_cc = take(cN), o_cp = take(cN), o_dirty = take(cN), o_stack = take(cN * 4),
                 o_un = take(cN * 4), o_ul = take(cN * 8), o_nundo = take((size_t)count * 4),
                 o_kind = take((size_t)count * 4), o_extra = take((size_t)count * 8),
                 o_hdr0 = take((size_t)count * sizeof(PartHdr)), o_hdr = take((size_t)count * sizeof(PartHdr)),
                 o_nodes = take((size_t)count * NI * sizeof(NodeJob)), o_pj = take(cN * sizeof(PJob)),
                 o_mj = take((size_t)count * d.Kmax * nchunk * sizeof(PmJob)),
                 o_rng = take((size_t)count * sizeof(curandStatePhilox4_32_10_t)), o_stats = take(6 * 8);
    unsigned char* buf = moves_buffer(c, off);
    if (!buf) return dm_fail(SMCCAT_ENOMEM, "device-move buffers: out of device memory");
    a.parent = reinterpret_cast<int32_t*>(buf + o_par);
    a.kids = reinterpret_cast<int32_t*>(buf + o_kids);
    a.nni = reinterpret_cast<int32_t*>(buf + o_nni);
    a.branch = reinterpret_cast<double*>(buf + o_br);
    a.clws = buf + o_clws;
    a.pws = buf + o_pws;
    a.cur_clws = buf + o_cc;
    a.cur_pws = buf + o_cp;
    a.dirty = buf + o_dirty;
    a.stack = reinterpret_cast<int32_t*>(buf + o_stack);
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
    DM_CK(cudaMemsetAsync(a.stats, 0, 6 * 8, st));
    const int grid = (count + kDmThreads - 1) / kDmThreads;
    dm_init_kernel<<<grid, kDmThreads, 0, st>>>(a.rng, count, first, (unsigned long long)seed);
    DM_CK(cudaGetLastError());
    DM_CK(cudaStreamSynchronize(st));  // the host images may go out of scope only after their copies

    PruneArgs pa = v.pa;
    pa.hdr = a.hdr;
    pa.nodes = a.nodes;
    const int nmjobs = count * d.Kmax * nchunk;
    auto step = [&]() -> cudaError_t {
        dm_propose_kernel<<<grid, kDmThreads, 0, st>>>(a);
        cudaError_t x = cudaGetLastError();
        if (x == cudaSuccess) x = launch_pmat(a.mjobs, nmjobs, a.pjobs, a.hdr, first, v.sws, v.spec, v.Pm, v.fp32, d, st);
        if (x == cudaSuccess) x = launch_prune(pa, v.ntiles, v.variant, st);
        if (x == cudaSuccess) x = launch_reduce(v.tile_off, pa.partial, a.hdr, first, count, v.lnl, v.status, st);
        if (x == cudaSuccess) {
            dm_mh_kernel<<<grid, kDmThreads, 0, st>>>(a);
            x = cudaGetLastError();
        }
        return x;
    };
    if (steps > 0) {
        if (use_graph) {
            DM_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            cudaError_t x = cudaSuccess;
            for (int k = 0; k < steps && x == cudaSuccess; ++k) x = step();
            const cudaError_t y = cudaStreamEndCapture(st, &graph);
            DM_CK(x);
            DM_CK(y);
            DM_CK(cudaGraphInstantiate(&exec, graph, 0));
            DM_CK(cudaGraphLaunch(exec, st));
        } else {
            for (int k = 0; k < steps; ++k) DM_CK(step());
        }
    }
    unsigned long long h_stats[6];
    int status = 0;
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
        }
    }
    if (stats)
        for (int k = 0; k < 6; ++k) stats[k] = (int64_t)h_stats[k];
    return finish(SMCCAT_OK, "");
#undef DM_CK
}
