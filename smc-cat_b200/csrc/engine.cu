// Host engine behind the C-ABI (include/smccat.h).
//
// The host keeps a small mirror of every particle (tree, parameters, and the
// workspace index of each node's CL, each node's transition matrices and each
// class's spectral data) and is the only authority on which buffers are
// current. Each refresh packs a plan -- per particle: dirty internal nodes in
// post-order with their children's workspaces, transition-matrix rebuild jobs,
// spectral re-decomposition jobs -- into one pinned buffer, ships it with a
// single host->device copy and launches four kernels. Dirty work is always
// written into the workspace that is NOT the last committed one, so reject
// restores the committed state by resetting host-side indices only
// (the reference copies whole buffers, Particle.cpp:343-478).
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "host_math.h"
#include "kernels.h"
#include "smccat.h"

using namespace smccat;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

}  // namespace

void smccat::set_last_error(const std::string& msg) { g_err = msg; }

#define CK(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return fail(SMCCAT_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#include "engine_internal.h"


struct smccat_ctx {
    smccat_config cfg{};
    Dims d{};
    cudaStream_t st = nullptr;
    cudaEvent_t plan_done = nullptr;
    size_t dev_bytes = 0;

    uint8_t* d_codes = nullptr;
    double* d_isinv = nullptr;
    int32_t* d_invchar = nullptr;
    int32_t* d_perm = nullptr;
    Tile* d_tiles = nullptr;
    int32_t* d_tile_off = nullptr;
    unsigned char* d_CL = nullptr;   // partials, element size esz
    double* d_LSC = nullptr;
    unsigned char* d_Pm = nullptr;   // transition matrices, element size esz
    int esz = 8;                     // 8 (FP64) or 4 (mixed precision)
    double* d_spec = nullptr;
    uint8_t* d_sws = nullptr;
    double* d_partial = nullptr;
    double* d_lnl = nullptr;
    double* d_lnl_old = nullptr;
    double* d_site_lnl = nullptr;
    int* d_status = nullptr;
    char* d_plan = nullptr;
    unsigned char* d_moves = nullptr;  // device tree-move buffers, grow-only
    size_t moves_cap = 0;

    char* h_plan = nullptr;     // pinned
    uint8_t* h_sws = nullptr;   // pinned mirror of d_sws
    size_t plan_cap = 0;
    int tile_cap = 0;
    int prune_variant = 0;      // chosen by smccat_autotune
    uint32_t wait_limit = kDrainPolls;  // polls per bounded device wait (smccat_set_wait_limit)
    int reassign_group = 0;             // particles per reassignment pass (0: from free memory)
    int tile_sites = kTileSites;  // slots per pruning tile, as the variant expects

    std::vector<uint8_t> codes;
    std::vector<Slot> slots;
    std::vector<Tile> tiles;
    std::vector<int32_t> tile_off;
    bool tiles_dirty = false;
    int32_t* h_perm = nullptr;  // pinned staging for slot -> site maps
    Tile* h_tiles = nullptr;      // pinned staging for the tile list
    // Site-pattern compression (SMCCAT_MODEL_PATTERNS): pattern id of every
    // site (identical alignment columns share one), and per-slot site counts.
    bool patterns = false;
    std::vector<int32_t> pid;
    int npat = 0;
    int32_t* d_wt = nullptr;    // [P][S]
    int32_t* h_wt = nullptr;    // pinned staging
    int32_t* h_tile_off = nullptr;
    std::vector<int> perm_dirty;

    // measurement
    bool timing = false;
    smccat_profile prof{};
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, int>> ev_used;  // (kind, index of start event)
};

namespace {

template <class T>
int dalloc(smccat_ctx* c, T** p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(SMCCAT_ENOMEM, std::string("cudaMalloc of ") + std::to_string(n * sizeof(T)) +
                                       " bytes failed: " + cudaGetErrorString(e));
    }
    c->dev_bytes += n * sizeof(T);
    return SMCCAT_OK;
}

// Validate a rooted binary tree and derive children / internal post-order.
bool build_tree(int T, const int32_t* parent, Mirror* m) {
    const int N = 2 * T - 1;
    m->kids.assign(2 * N, -1);
    std::vector<int> nk(N, 0);
    int root = -1;
    for (int n = 0; n < N; ++n) {
        const int p = parent[n];
        if (p < 0) {
            if (root >= 0) return false;
            root = n;
            continue;
        }
        if (p < T || p >= N || nk[p] >= 2) return false;
        m->kids[2 * p + nk[p]++] = n;
    }
    if (root < T) return false;
    for (int n = T; n < N; ++n) {
        if (nk[n] != 2) return false;
        if (m->kids[2 * n] > m->kids[2 * n + 1]) std::swap(m->kids[2 * n], m->kids[2 * n + 1]);
    }
    m->post.clear();
    std::vector<std::pair<int, int>> st;
    st.push_back({root, 0});
    int visited = 0;
    while (!st.empty()) {
        auto& top = st.back();
        const int n = top.first;
        if (n >= T && top.second < 2) {
            st.push_back({m->kids[2 * n + top.second++], 0});
        } else {
            ++visited;
            if (n >= T) m->post.push_back(n);
            st.pop_back();
        }
        if (visited > N) return false;
    }
    if (visited != N) return false;
    m->parent.assign(parent, parent + N);
    m->root = root;
    return true;
}

void mark_up(Slot& s, int x) {
    while (x >= 0) {
        s.dirty_cl[x] = 1;
        x = s.cur.parent[x];
    }
}

int check_range(const smccat_ctx* c, int first, int count) {
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    if (first < 0 || count < 0 || first + count > c->cfg.max_particles)
        return fail(SMCCAT_EINVAL, "particle range out of bounds");
    return SMCCAT_OK;
}

int check_particle(const smccat_ctx* c, int p) {
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    if (p < 0 || p >= c->cfg.max_particles) return fail(SMCCAT_EINVAL, "particle index out of bounds");
    if (!c->slots[p].loaded) return fail(SMCCAT_ESTATE, "particle has no state loaded");
    return SMCCAT_OK;
}

// Host->device copy on the context stream, counted for the e2e report.
cudaError_t h2d(smccat_ctx* c, void* dst, const void* src, size_t n) {
    c->prof.h2d_bytes += n;
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, c->st);
}

cudaError_t d2h(smccat_ctx* c, void* dst, const void* src, size_t n) {
    c->prof.d2h_bytes += n;
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, c->st);
}

cudaEvent_t pool_event(smccat_ctx* c, size_t i) {
    while (c->ev_pool.size() <= i) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[i];
}

// Launch one kernel of `kind`, bracketed by CUDA events when timing is on.
template <class F>
cudaError_t launch(smccat_ctx* c, int kind, F&& f) {
    c->prof.launches[kind]++;
    if (!c->timing) return f();
    const size_t i = 2 * c->ev_used.size();
    cudaEvent_t a = pool_event(c, i), b = pool_event(c, i + 1);
    if (!a || !b) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaEventRecord(a, c->st);
    if (e != cudaSuccess) return e;
    e = f();
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(b, c->st);
    c->ev_used.push_back({kind, (int)i});
    return e;
}

// Sites grouped by class (stable), then cut into tiles of <= tile_sites; the
// per-class site counts come from the last state upload.
void rebuild_tiles(smccat_ctx* c) {
    const int P = c->cfg.max_particles, ts = c->tile_sites;
    c->tiles.clear();
    c->tile_off.assign(P + 1, 0);
    for (int p = 0; p < P; ++p) {
        c->tile_off[p] = (int)c->tiles.size();
        const Slot& s = c->slots[p];
        if (!s.loaded) continue;
        const std::vector<int32_t>& cnt = s.class_cnt;
        int slot0 = 0;
        for (int k = 0; k < s.cur.K; ++k) {
            for (int off = 0; off < cnt[k]; off += ts)
                c->tiles.push_back(Tile{p, k, slot0 + off, std::min(ts, cnt[k] - off)});
            slot0 += cnt[k];
        }
    }
    c->tile_off[P] = (int)c->tiles.size();
}

// Select pruning variant v; a different tile width rebuilds the tile list at
// the next refresh.
void select_variant(smccat_ctx* c, int v) {
    c->prune_variant = v;
    const int ts = prune_variant_tile_sites(c->d.R, c->esz == 4, v);
    if (ts != c->tile_sites) {
        c->tile_sites = ts;
        c->tiles_dirty = true;
    }
}

}  // namespace

extern "C" {

const char* smccat_version(void) { return "smccat-b200 0.1"; }

const char* smccat_last_error(void) { return g_err.c_str(); }

int smccat_discretize_gamma(double shape, int32_t num_rates, double* out) {
    if (!out) return fail(SMCCAT_EINVAL, "null argument");
    if (num_rates < 1) return fail(SMCCAT_EINVAL, "num_rates must be >= 1");
    if (num_rates > 1 && (!(shape > 0.0) || !std::isfinite(shape))) return fail(SMCCAT_EINVAL, "shape must be > 0");
    discretize_gamma(shape, num_rates, out);
    return SMCCAT_OK;
}

int smccat_lg_exchangeabilities(double* out190) {
    if (!out190) return fail(SMCCAT_EINVAL, "null argument");
    std::memcpy(out190, lg_exchangeabilities(), sizeof(double) * kBase);
    return SMCCAT_OK;
}

int smccat_destroy(smccat_ctx* c) {
    if (!c) return SMCCAT_OK;
    mcmc_release(c);
    learned_release(c);
    cudaSetDevice(c->cfg.device);
    if (c->st) cudaStreamSynchronize(c->st);
    void* dptrs[] = {c->d_codes, c->d_isinv, c->d_invchar, c->d_perm, c->d_tiles, c->d_tile_off,
                     c->d_CL, c->d_LSC, c->d_Pm, c->d_spec, c->d_sws, c->d_partial, c->d_lnl,
                     c->d_lnl_old, c->d_site_lnl, c->d_status, c->d_plan, c->d_wt, c->d_moves};
    for (void* p : dptrs) if (p) cudaFree(p);
    if (c->h_plan) cudaFreeHost(c->h_plan);
    if (c->h_sws) cudaFreeHost(c->h_sws);
    if (c->h_perm) cudaFreeHost(c->h_perm);
    if (c->h_tiles) cudaFreeHost(c->h_tiles);
    if (c->h_tile_off) cudaFreeHost(c->h_tile_off);
    if (c->h_wt) cudaFreeHost(c->h_wt);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    if (c->plan_done) cudaEventDestroy(c->plan_done);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
    return SMCCAT_OK;
}

int smccat_create(const smccat_config* cfg, const uint8_t* codes, smccat_ctx** out) {
    if (!cfg || !codes || !out) return fail(SMCCAT_EINVAL, "null argument");
    *out = nullptr;
    const int T = cfg->num_taxa, S = cfg->num_sites, R = cfg->num_rates;
    if (T < 3) return fail(SMCCAT_EINVAL, "num_taxa must be >= 3");
    if (S < 1) return fail(SMCCAT_EINVAL, "num_sites must be >= 1");
    if (R < 1 || R > kMaxRates) return fail(SMCCAT_EINVAL, "num_rates must be in [1, 8]");
    if (cfg->max_particles < 1) return fail(SMCCAT_EINVAL, "max_particles must be >= 1");
    if (cfg->max_classes < 1 || cfg->max_classes > 4096) return fail(SMCCAT_EINVAL, "max_classes must be in [1, 4096]");
    if (cfg->precision != SMCCAT_PREC_FP64 && cfg->precision != SMCCAT_PREC_FP32)
        return fail(SMCCAT_EINVAL, "unsupported precision");
    for (size_t i = 0; i < (size_t)T * S; ++i)
        if (codes[i] > 22) return fail(SMCCAT_EINVAL, "alignment code > 22 at index " + std::to_string(i));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(SMCCAT_ENODEV, "no CUDA device");
    if (cfg->device < 0 || cfg->device >= ndev) return fail(SMCCAT_ENODEV, "device ordinal out of range");

    smccat_ctx* c = new (std::nothrow) smccat_ctx();
    if (!c) return fail(SMCCAT_ENOMEM, "host allocation failed");
    c->cfg = *cfg;
    const int P = cfg->max_particles, K = cfg->max_classes, N = 2 * T - 1;
    c->d = Dims{T, S, (S + 31) / 32 * 32, R, N, T - 1, K};
    const Dims& d = c->d;

    // Capacity check against free device memory before allocating.
    const size_t cl = (size_t)P * d.NI * 2 * kStates * R * d.Spad;
    const size_t lsc = (size_t)P * d.NI * 2 * R * d.Spad;
    const size_t pm = (size_t)P * K * N * 2 * R * kPBlock;
    const size_t spec = (size_t)P * K * 2 * kSpecStride;
    const size_t esz = cfg->precision == SMCCAT_PREC_FP32 ? 4 : 8;
    const size_t need = esz * (cl + pm) + 8 * (lsc + spec);
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) { delete c; return fail(SMCCAT_ECUDA, cudaGetErrorString(e)); }
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    if (need > free_b) {
        delete c;
        return fail(SMCCAT_ENOMEM, "context needs " + std::to_string(need) + " device bytes, " +
                                       std::to_string(free_b) + " free");
    }
    int rc = SMCCAT_OK;
    auto A = [&](auto** p, size_t n) { if (rc == SMCCAT_OK) rc = dalloc(c, p, n); };
    c->tile_cap = P * ((S + kTileSites - 1) / kTileSites + K);
    A(&c->d_codes, (size_t)T * S);
    A(&c->d_isinv, (size_t)S);
    A(&c->d_invchar, (size_t)S);
    A(&c->d_perm, (size_t)P * S);
    c->patterns = (cfg->model_flags & SMCCAT_MODEL_PATTERNS) != 0;
    if (c->patterns) A(&c->d_wt, (size_t)P * S);
    A(&c->d_tiles, (size_t)c->tile_cap);
    A(&c->d_tile_off, (size_t)P + 1);
    c->esz = (int)esz;
    select_variant(c, prune_default_variant(d.R, esz == 4));
    A(&c->d_CL, cl * esz);
    A(&c->d_LSC, lsc);
    A(&c->d_Pm, pm * esz);
    A(&c->d_spec, spec);
    A(&c->d_sws, (size_t)P * K);
    A(&c->d_partial, (size_t)c->tile_cap);
    A(&c->d_lnl, (size_t)P);
    A(&c->d_lnl_old, (size_t)P);
    A(&c->d_site_lnl, (size_t)P * S);
    A(&c->d_status, 1);
    c->plan_cap = sizeof(PartHdr) * P + sizeof(NodeJob) * (size_t)P * d.NI +
                  sizeof(PJob) * (size_t)P * N +
                  sizeof(PmJob) * (size_t)P * K * ((N + kPmChunk - 1) / kPmChunk) +
                  sizeof(SpecJob) * (size_t)P * K + P + 64;
    A(&c->d_plan, c->plan_cap);
    if (rc != SMCCAT_OK) { smccat_destroy(c); return rc; }
    if (cudaMallocHost((void**)&c->h_plan, c->plan_cap) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_sws, (size_t)P * K) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_perm, (size_t)P * S * sizeof(int32_t)) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_tiles, (size_t)c->tile_cap * sizeof(Tile)) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_tile_off, ((size_t)P + 1) * sizeof(int32_t)) != cudaSuccess ||
        (c->patterns &&
         cudaMallocHost((void**)&c->h_wt, (size_t)P * S * sizeof(int32_t)) != cudaSuccess)) {
        smccat_destroy(c);
        return fail(SMCCAT_ENOMEM, "pinned host allocation failed");
    }
    std::memset(c->h_sws, 0, (size_t)P * K);
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->plan_done, cudaEventDisableTiming) != cudaSuccess) {
        smccat_destroy(c);
        return fail(SMCCAT_ECUDA, "stream/event creation failed");
    }

    // Alignment-derived data (Particle.cpp:44-73).
    c->codes.assign(codes, codes + (size_t)T * S);
    if (c->patterns) {  // pattern ids in order of first occurrence
        std::unordered_map<std::string, int32_t> seen;
        std::string col(T, '\0');
        c->pid.resize(S);
        for (int s = 0; s < S; ++s) {
            for (int t = 0; t < T; ++t) col[t] = (char)codes[(size_t)t * S + s];
            auto it = seen.emplace(col, (int32_t)seen.size()).first;
            c->pid[s] = it->second;
        }
        c->npat = (int)seen.size();
    }
    std::vector<double> isinv(S);
    std::vector<int32_t> invchar(S);
    for (int s = 0; s < S; ++s) {
        const int c1 = codes[s];
        bool inv = true;
        for (int t = 1; t < T; ++t) if (codes[(size_t)t * S + s] != c1) { inv = false; break; }
        isinv[s] = inv ? 1.0 : 0.0;
        invchar[s] = (inv && c1 < 20) ? c1 : 0;
    }
    cudaError_t ce = cudaMemcpy(c->d_codes, codes, (size_t)T * S, cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(c->d_isinv, isinv.data(), S * sizeof(double), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(c->d_invchar, invchar.data(), S * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemset(c->d_status, 0, sizeof(int));
    if (ce == cudaSuccess) ce = cudaMemset(c->d_sws, 0, (size_t)P * K);
    if (ce != cudaSuccess) { smccat_destroy(c); return fail(SMCCAT_ECUDA, cudaGetErrorString(ce)); }

    c->slots.resize(P);
    for (auto& s : c->slots) {
        for (Mirror* m : {&s.cur, &s.old}) {
            m->branch.assign(N, 0.0);
            m->base.assign(kBase, 0.0);
            m->logits.assign((size_t)K * kStates, 0.0);
            m->clws.assign(N, 0);
            m->pws.assign(N, 0);
            m->sws.assign(K, 0);
        }
        s.dirty_cl.assign(N, 0);
        s.dirty_p.assign(N, 0);
        s.dirty_spec.assign(K, 0);
    }
    c->tile_off.assign(P + 1, 0);
    *out = c;
    return SMCCAT_OK;
}

int smccat_device_bytes(const smccat_ctx* c, uint64_t* bytes) {
    if (!c || !bytes) return fail(SMCCAT_EINVAL, "null argument");
    *bytes = c->dev_bytes;
    return SMCCAT_OK;
}

int smccat_set_particles(smccat_ctx* c, int32_t first, int32_t count, const int32_t* parent,
                         const double* branch, const double* base, const int32_t* num_classes,
                         const double* logits, const int32_t* assign, const double* pinv,
                         const double* shape) {
    int rc = check_range(c, first, count);
    if (rc) return rc;
    if (!parent || !branch || !base || !num_classes || !logits || !assign || !pinv || !shape)
        return fail(SMCCAT_EINVAL, "null argument");
    const Dims& d = c->d;
    const int N = d.N, S = d.S, Kmax = d.Kmax;
    // Validate everything before touching any slot (particles in parallel;
    // the first bad particle in index order is reported).
    std::vector<Mirror> trees(count);
    std::vector<uint8_t> bad(count, 0);
#pragma omp parallel for schedule(static) num_threads(host_team()) if (count >= kParallelParticles)
    for (int i = 0; i < count; ++i) {
        uint8_t why = 0;
        const int K = num_classes[i];
        if (!build_tree(d.T, parent + (size_t)i * N, &trees[i])) why = 1;
        else if (K < 1 || K > Kmax) why = 2;
        else if (!(c->cfg.model_flags & SMCCAT_MODEL_CAT) && K != 1) why = 3;
        for (int s = 0; s < S && !why; ++s) {
            const int k = assign[(size_t)i * S + s];
            if (k < 0 || k >= K) why = 4;
        }
        const double pv = pinv[i];
        if (!why && !(pv >= 0.0 && pv < 1.0)) why = 5;
        if (!why && d.R > 1 && !(shape[i] > 0.0)) why = 6;
        for (int n = 0; n < N && !why; ++n) {
            const double b = branch[(size_t)i * N + n];
            if (!(b >= 0.0) || !std::isfinite(b)) why = 7;
        }
        bad[i] = why;
    }
    for (int i = 0; i < count; ++i) {
        const std::string who = "particle " + std::to_string(first + i) + ": ";
        switch (bad[i]) {
            case 0: continue;
            case 1: return fail(SMCCAT_EINVAL, who + "not a rooted binary tree");
            case 2: return fail(SMCCAT_EINVAL, who + "num_classes out of range");
            case 3: return fail(SMCCAT_EINVAL, "num_classes must be 1 without SMCCAT_MODEL_CAT");
            case 4: return fail(SMCCAT_EINVAL, who + "class index out of range");
            case 5: return fail(SMCCAT_EINVAL, "pinv must be in [0, 1)");
            case 6: return fail(SMCCAT_EINVAL, "shape must be > 0");
            default: return fail(SMCCAT_EINVAL, "branch lengths must be finite and >= 0");
        }
    }
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaEventSynchronize(c->plan_done));  // h_perm may still be in flight
#pragma omp parallel for schedule(static) num_threads(host_team()) if (count >= kParallelParticles)
    for (int i = 0; i < count; ++i) {
        const int p = first + i;
        Slot& s = c->slots[p];
        Mirror& m = s.cur;
        m.parent = trees[i].parent;
        m.kids = trees[i].kids;
        m.post = trees[i].post;
        m.root = trees[i].root;
        m.branch.assign(branch + (size_t)i * N, branch + (size_t)(i + 1) * N);
        m.base.assign(base + (size_t)i * kBase, base + (size_t)(i + 1) * kBase);
        m.K = num_classes[i];
        std::fill(m.logits.begin(), m.logits.end(), 0.0);
        std::copy(logits + (size_t)i * Kmax * kStates, logits + (size_t)i * Kmax * kStates + (size_t)m.K * kStates,
                  m.logits.begin());
        m.pinv = pinv[i];
        m.shape = shape[i];
        discretize_gamma(m.shape, d.R, m.rates);
        s.assign.assign(assign + (size_t)i * S, assign + (size_t)(i + 1) * S);
        // A loaded state is rebuilt and committed whole: the classes' workspace
        // flips restart at zero (class numbers may mean other classes now).
        for (Mirror* mm : {&s.cur, &s.old})
            for (auto& b : mm->sws) b &= kSwsSpec;
        s.local_class = -1;
        s.loaded = true;
        s.full = true;
        s.commit_on_refresh = true;
        s.pending = true;
        s.refreshed = false;
        // slot -> site, grouped by class (stable)
        int32_t* perm = c->h_perm + (size_t)p * S;
        std::vector<int> cnt(m.K + 1, 0);
        for (int x = 0; x < S; ++x) cnt[s.assign[x] + 1]++;
        s.class_cnt.assign(cnt.begin() + 1, cnt.end());
        for (int k = 0; k < m.K; ++k) cnt[k + 1] += cnt[k];
        for (int x = 0; x < S; ++x) perm[cnt[s.assign[x]]++] = x;
        if (c->patterns) {
            // Within each class keep the first site of every pattern; its slot
            // counts the class's sites with that column.
            int32_t* wt = c->h_wt + (size_t)p * S;
            std::vector<int32_t> slot_of(c->npat, -1), stamp(c->npat, -1);
            s.site_rep.resize(S);
            int out = 0, x0 = 0;
            for (int k = 0; k < m.K; ++k) {
                const int first_slot = out;
                for (int q = x0; q < x0 + s.class_cnt[k]; ++q) {
                    const int site = perm[q], pt = c->pid[site];
                    if (stamp[pt] != k) {
                        stamp[pt] = k;
                        slot_of[pt] = out;
                        perm[out] = site;
                        wt[out] = 0;
                        ++out;
                    }
                    wt[slot_of[pt]]++;
                    s.site_rep[site] = perm[slot_of[pt]];
                }
                x0 += s.class_cnt[k];
                s.class_cnt[k] = out - first_slot;
            }
        }
    }
    if (count > 0) {
        CK(h2d(c, c->d_perm + (size_t)first * S, c->h_perm + (size_t)first * S,
               (size_t)count * S * sizeof(int32_t)));
        if (c->patterns)
            CK(h2d(c, c->d_wt + (size_t)first * S, c->h_wt + (size_t)first * S,
                   (size_t)count * S * sizeof(int32_t)));
        CK(cudaEventRecord(c->plan_done, c->st));
    }
    c->tiles_dirty = true;
    return SMCCAT_OK;
}

int smccat_get_particles(smccat_ctx* c, int32_t first, int32_t count, int32_t* parent, double* branch,
                         double* base, int32_t* num_classes, double* logits, int32_t* assign,
                         double* pinv, double* shape) {
    int rc = check_range(c, first, count);
    if (rc) return rc;
    const Dims& d = c->d;
    for (int i = 0; i < count; ++i) {
        const Slot& s = c->slots[first + i];
        if (!s.loaded) return fail(SMCCAT_ESTATE, "particle has no state loaded");
        const Mirror& m = s.cur;
        if (parent) std::copy(m.parent.begin(), m.parent.end(), parent + (size_t)i * d.N);
        if (branch) std::copy(m.branch.begin(), m.branch.end(), branch + (size_t)i * d.N);
        if (base) std::copy(m.base.begin(), m.base.end(), base + (size_t)i * kBase);
        if (num_classes) num_classes[i] = m.K;
        if (logits) std::copy(m.logits.begin(), m.logits.end(), logits + (size_t)i * d.Kmax * kStates);
        if (assign) std::copy(s.assign.begin(), s.assign.end(), assign + (size_t)i * d.S);
        if (pinv) pinv[i] = m.pinv;
        if (shape) shape[i] = m.shape;
    }
    return SMCCAT_OK;
}

int smccat_refresh(smccat_ctx* c, int32_t first, int32_t count, int32_t mode) {
    NvtxRange range("smccat_refresh");
    return refresh_internal(c, first, count, mode, nullptr);
}

}  // extern "C"

// A pending class-local edit with nothing else dirty: the refresh can rebuild
// that class alone.
static bool local_plan(const Slot& s) {
    if (s.local_class < 0 || s.full) return false;
    for (size_t n = 0; n < s.dirty_cl.size(); ++n)
        if (s.dirty_cl[n] || s.dirty_p[n]) return false;
    return true;
}

int smccat::refresh_internal(smccat_ctx* c, int first, int count, int mode, const uint8_t* active) {
    int rc = check_range(c, first, count);
    if (rc) return rc;
    if (count == 0) return SMCCAT_OK;
    if (mode != SMCCAT_REFRESH_DIRTY && mode != SMCCAT_REFRESH_FULL)
        return fail(SMCCAT_EINVAL, "unknown refresh mode");
    for (int i = 0; i < count; ++i)
        if (!c->slots[first + i].loaded) return fail(SMCCAT_ESTATE, "particle has no state loaded");
    auto on = [&](int i) { return !active || active[i]; };
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaEventSynchronize(c->plan_done));  // previous plan copy has left the pinned buffer
    const Dims& d = c->d;
    const int N = d.N, Kmax = d.Kmax;

    if (c->tiles_dirty) {
        rebuild_tiles(c);
        if ((int)c->tiles.size() > c->tile_cap) return fail(SMCCAT_ENOMEM, "tile capacity exceeded");
        // Pinned staging: the previous tile copy is older than the plan copy
        // that plan_done (waited on above) tracks, so the buffer is free.
        std::memcpy(c->h_tiles, c->tiles.data(), c->tiles.size() * sizeof(Tile));
        std::memcpy(c->h_tile_off, c->tile_off.data(), c->tile_off.size() * sizeof(int32_t));
        CK(h2d(c, c->d_tiles, c->h_tiles, c->tiles.size() * sizeof(Tile)));
        CK(h2d(c, c->d_tile_off, c->h_tile_off, c->tile_off.size() * sizeof(int32_t)));
        c->tiles_dirty = false;
    }

    // Pack the plan: per-particle job counts, their prefix sums, then every
    // particle fills its own ranges (in parallel for large batches).
    struct Cnt { int nn, np, nm, ns; };
    std::vector<Cnt> cn(count + 1, Cnt{0, 0, 0, 0});
    // A few microseconds per particle: a small team, since waking a full one
    // after the previous refresh's GPU wait costs more than it saves.
    const int team = std::min(kPackThreads, omp_get_max_threads());
#pragma omp parallel for schedule(static) num_threads(team) if (count >= 2 * kParallelParticles)
    for (int i = 0; i < count; ++i) {
        const Slot& s = c->slots[first + i];
        Cnt x{0, 0, 0, 0};
        if (on(i)) {
            const Mirror& m = s.cur;
            if ((mode == SMCCAT_REFRESH_FULL) || s.full) {
                x.nn = (int)m.post.size();
                x.np = N - 1;
                x.ns = m.K;
            } else if (local_plan(s)) {
                x.nn = (int)m.post.size();
                x.np = N - 1;
                x.ns = 1;
                x.nm = (x.np + kPmChunk - 1) / kPmChunk;  // class local_class only
                cn[i + 1] = x;
                continue;
            } else if (s.local_class >= 0) {  // a class edit combined with others: everything
                x.nn = (int)m.post.size();
                x.np = N - 1;
                for (int k = 0; k < m.K; ++k) x.ns += s.dirty_spec[k];
            } else {
                for (int n : m.post) x.nn += s.dirty_cl[n];
                for (int n = 0; n < N; ++n) x.np += (s.dirty_p[n] && n != m.root);
                for (int k = 0; k < m.K; ++k) x.ns += s.dirty_spec[k];
            }
            x.nm = m.K * ((x.np + kPmChunk - 1) / kPmChunk);
        }
        cn[i + 1] = x;
    }
    for (int i = 1; i <= count; ++i) {
        cn[i].nn += cn[i - 1].nn;
        cn[i].np += cn[i - 1].np;
        cn[i].nm += cn[i - 1].nm;
        cn[i].ns += cn[i - 1].ns;
    }
    const int nn = cn[count].nn, np_ = cn[count].np, nm = cn[count].nm, ns = cn[count].ns;
    char* hp = c->h_plan;
    PartHdr* hdr = reinterpret_cast<PartHdr*>(hp);
    size_t off = sizeof(PartHdr) * count;
    NodeJob* nodes = reinterpret_cast<NodeJob*>(hp + off);
    off += sizeof(NodeJob) * nn;
    off = (off + 15) & ~size_t(15);
    PJob* pjobs = reinterpret_cast<PJob*>(hp + off);
    const size_t pjob_off = off;
    off += sizeof(PJob) * np_;
    off = (off + 15) & ~size_t(15);
    PmJob* mjobs = reinterpret_cast<PmJob*>(hp + off);
    const size_t mjob_off = off;
    off += sizeof(PmJob) * nm;
    off = (off + 15) & ~size_t(15);
    SpecJob* sjobs = reinterpret_cast<SpecJob*>(hp + off);
    const size_t sjob_off = off;
    std::vector<uint8_t> broken(count, 0);
#pragma omp parallel for schedule(static) num_threads(team) if (count >= 2 * kParallelParticles)
    for (int i = 0; i < count; ++i) {
        const int p = first + i;
        Slot& s = c->slots[p];
        Mirror& m = s.cur;
        int jn = cn[i].nn, jp = cn[i].np, jm = cn[i].nm, js = cn[i].ns;
        if (!on(i)) {
            PartHdr& h = hdr[i];
            std::memset(&h, 0, sizeof(h));
            h.node_off = jn;
            continue;
        }
        const bool full = (mode == SMCCAT_REFRESH_FULL) || s.full;
        if (!full && local_plan(s)) {
            // Class-local refresh (a stationary edit of one class): that class
            // is re-decomposed, its matrices of every node and its sites'
            // partials of every internal node rebuilt into its other
            // workspaces (all three workspace bits of its byte flip); node
            // workspace indices stay, and the other classes' tiles only rerun
            // the root reduction.
            const int k = s.local_class;
            m.sws[k] = s.old.sws[k] ^ (kSwsSpec | kSwsCl | kSwsP);
            SpecJob& j = sjobs[js++];
            j.p = p; j.k = k; j.sws = m.sws[k] & kSwsSpec; j.pad = 0;
            std::memcpy(j.base, m.base.data(), sizeof(j.base));
            std::memcpy(j.logits, &m.logits[(size_t)k * kStates], sizeof(j.logits));
            const int pj0 = jp;
            for (int n = 0; n < N; ++n)
                if (n != m.root) pjobs[jp++] = PJob{p, n, m.pws[n], 0, m.branch[n]};
            for (int q = pj0; q < jp; q += kPmChunk)
                mjobs[jm++] = PmJob{i, k, q, std::min(kPmChunk, jp - q)};
            PartHdr& h = hdr[i];
            h.node_off = jn;
            for (int n : m.post) {
                const int c1 = m.kids[2 * n], c2 = m.kids[2 * n + 1];
                int ws = m.clws[n];
                if (c1 >= d.T) ws |= m.clws[c1] << 1;
                if (c2 >= d.T) ws |= m.clws[c2] << 2;
                ws |= m.pws[c1] << 3;
                ws |= m.pws[c2] << 4;
                nodes[jn++] = NodeJob{n, c1, c2, ws};
            }
            h.node_cnt = jn - h.node_off;
            h.root = m.root;
            h.root_ws = m.clws[m.root];
            h.active = 1;
            h.num_classes = m.K;
            h.cls_only = k;
            h.pad1 = 0;
            h.pinv = m.pinv;
            for (int r = 0; r < kMaxRates; ++r) h.rates[r] = m.rates[r];
            std::fill(s.dirty_spec.begin(), s.dirty_spec.end(), 0);
            s.local_class = -1;
            s.full = false;
            s.refreshed = true;
            std::copy(m.sws.begin(), m.sws.end(), c->h_sws + (size_t)p * Kmax);
            continue;
        }
        if (s.local_class >= 0) {  // combined with other edits: rebuild everything
            std::fill(s.dirty_p.begin(), s.dirty_p.end(), 1);
            for (int n : m.post) s.dirty_cl[n] = 1;
            s.local_class = -1;
        }
        if (full) {
            std::fill(s.dirty_spec.begin(), s.dirty_spec.begin() + m.K, 1);
            std::fill(s.dirty_p.begin(), s.dirty_p.end(), 1);
            for (int n : m.post) s.dirty_cl[n] = 1;
            s.local_class = -1;
        }
        for (int k = 0; k < m.K; ++k) {
            if (!s.dirty_spec[k]) continue;
            m.sws[k] = s.old.sws[k] ^ kSwsSpec;
            SpecJob& j = sjobs[js++];
            j.p = p; j.k = k; j.sws = m.sws[k] & kSwsSpec; j.pad = 0;
            std::memcpy(j.base, m.base.data(), sizeof(j.base));
            std::memcpy(j.logits, &m.logits[(size_t)k * kStates], sizeof(j.logits));
        }
        const int pj0 = jp;
        for (int n = 0; n < N; ++n) {
            if (!s.dirty_p[n] || n == m.root) continue;
            m.pws[n] = 1 - s.old.pws[n];
            pjobs[jp++] = PJob{p, n, m.pws[n], 0, m.branch[n]};
        }
        for (int k = 0; k < m.K; ++k)
            for (int q = pj0; q < jp; q += kPmChunk)
                mjobs[jm++] = PmJob{i, k, q, std::min(kPmChunk, jp - q)};
        PartHdr& h = hdr[i];
        h.node_off = jn;
        for (int n : m.post) {
            if (!s.dirty_cl[n]) continue;
            m.clws[n] = 1 - s.old.clws[n];
            const int c1 = m.kids[2 * n], c2 = m.kids[2 * n + 1];
            int ws = m.clws[n];
            if (c1 >= d.T) ws |= m.clws[c1] << 1;
            if (c2 >= d.T) ws |= m.clws[c2] << 2;
            ws |= m.pws[c1] << 3;
            ws |= m.pws[c2] << 4;
            nodes[jn++] = NodeJob{n, c1, c2, ws};
        }
        h.node_cnt = jn - h.node_off;
        if (h.node_cnt > 0 && nodes[jn - 1].node != m.root) broken[i] = 1;
        h.root = m.root;
        h.root_ws = m.clws[m.root];
        h.active = 1;
        h.num_classes = m.K;
        h.cls_only = -1;
        h.pad1 = 0;
        h.pinv = m.pinv;
        for (int r = 0; r < kMaxRates; ++r) h.rates[r] = m.rates[r];
        std::fill(s.dirty_spec.begin(), s.dirty_spec.end(), 0);
        std::fill(s.dirty_p.begin(), s.dirty_p.end(), 0);
        std::fill(s.dirty_cl.begin(), s.dirty_cl.end(), 0);
        s.full = false;
        s.refreshed = true;
        std::copy(m.sws.begin(), m.sws.end(), c->h_sws + (size_t)p * Kmax);
    }
    for (int i = 0; i < count; ++i)
        if (broken[i]) return fail(SMCCAT_EINVAL, "internal error: dirty set does not reach the root");
    const size_t plan_bytes = off + sizeof(SpecJob) * ns;
    CK(h2d(c, c->d_plan, c->h_plan, plan_bytes));
    CK(h2d(c, c->d_sws + (size_t)first * Kmax, c->h_sws + (size_t)first * Kmax, (size_t)count * Kmax));
    CK(cudaEventRecord(c->plan_done, c->st));

    const PartHdr* d_hdr = reinterpret_cast<const PartHdr*>(c->d_plan);
    if (ns > 0)
        CK(launch(c, SMCCAT_KERNEL_SPEC, [&] {
            return launch_spec(reinterpret_cast<const SpecJob*>(c->d_plan + sjob_off), ns, c->d_spec, d, c->st);
        }));
    if (np_ > 0)
        CK(launch(c, SMCCAT_KERNEL_PMAT, [&] {
            return launch_pmat(reinterpret_cast<const PmJob*>(c->d_plan + mjob_off), nm,
                               reinterpret_cast<const PJob*>(c->d_plan + pjob_off), d_hdr, first,
                               c->d_sws, c->d_spec, c->d_Pm, c->esz == 4, d, c->st);
        }));
    PruneArgs a{};
    a.d = d;
    a.first = first;
    a.tile_begin = c->tile_off[first];
    a.tiles = c->d_tiles;
    a.hdr = d_hdr;
    a.nodes = reinterpret_cast<const NodeJob*>(c->d_plan + sizeof(PartHdr) * count);
    a.codes = c->d_codes;
    a.perm = c->d_perm;
    a.wt = c->patterns ? c->d_wt : nullptr;
    a.Pm = c->d_Pm;
    a.spec = c->d_spec;
    a.sws = c->d_sws;
    a.isinv = c->d_isinv;
    a.invchar = c->d_invchar;
    a.CL = c->d_CL;
    a.fp32 = c->esz == 4;
    a.LSC = c->d_LSC;
    a.site_lnl = c->d_site_lnl;
    a.partial = c->d_partial;
    a.status = c->d_status;
    a.wait_limit = c->wait_limit;
    const int ntiles = c->tile_off[first + count] - c->tile_off[first];
    if (ntiles > 0)
        CK(launch(c, SMCCAT_KERNEL_PRUNE,
                  [&] { return launch_prune(a, ntiles, c->prune_variant, c->st); }));
    CK(launch(c, SMCCAT_KERNEL_REDUCE, [&] {
        return launch_reduce(c->d_tile_off, c->d_partial, d_hdr, first, count, c->d_lnl, c->d_status, c->st);
    }));

    // Loaded particles commit their first refresh (copyFromSerialized does).
    bool any_commit = false;
    for (int i = 0; i < count; ++i) any_commit |= on(i) && c->slots[first + i].commit_on_refresh;
    if (any_commit) {
        uint8_t* mask = reinterpret_cast<uint8_t*>(c->h_plan + plan_bytes);
        for (int i = 0; i < count; ++i)
            mask[i] = (on(i) && c->slots[first + i].commit_on_refresh) ? 1 : 2;
        // The mask shares the pinned plan buffer; its copy precedes plan_done.
        uint8_t* d_mask = reinterpret_cast<uint8_t*>(c->d_plan + plan_bytes);
        CK(h2d(c, d_mask, mask, count));
        CK(cudaEventRecord(c->plan_done, c->st));
        CK(launch(c, SMCCAT_KERNEL_ACCEPT,
                  [&] { return launch_accept(c->d_lnl, c->d_lnl_old, d_mask, first, count, c->st); }));
#pragma omp parallel for schedule(static) num_threads(team) if (count >= 2 * kParallelParticles)
        for (int i = 0; i < count; ++i) {
            Slot& s = c->slots[first + i];
            if (!on(i) || !s.commit_on_refresh) continue;
            s.old = s.cur;
            s.commit_on_refresh = false;
            s.pending = false;
            s.refreshed = false;
        }
    }
    int status = 0;
    CK(d2h(c, &status, c->d_status, sizeof(int)));
    CK(cudaStreamSynchronize(c->st));
    if (status) {
        CK(cudaMemset(c->d_status, 0, sizeof(int)));
        if (status & 2)
            return fail(SMCCAT_ETIMEOUT, "a pruning warp gave up waiting for its transition matrices");
        return fail(SMCCAT_ENUMERIC, "a log-likelihood came out NaN");
    }
    return SMCCAT_OK;
}

const Slot& smccat::slot_of(const smccat_ctx* c, int p) { return c->slots[p]; }
int smccat::particles_of(const smccat_ctx* c) { return (int)c->slots.size(); }
Slot& smccat::slot_mut(smccat_ctx* c, int p) { return c->slots[p]; }
bool smccat::rebuild_tree(int T, const int32_t* parent, Mirror* m) { return build_tree(T, parent, m); }

unsigned char* smccat::moves_buffer(smccat_ctx* c, size_t bytes) {
    if (bytes > c->moves_cap) {
        cudaStreamSynchronize(c->st);
        if (c->d_moves) cudaFree(c->d_moves);
        c->d_moves = nullptr;
        c->moves_cap = 0;
        if (cudaMalloc((void**)&c->d_moves, bytes) != cudaSuccess) return nullptr;
        c->moves_cap = bytes;
    }
    return c->d_moves;
}

int smccat::device_view(smccat_ctx* c, int first, int count, DeviceView* v) {
    if (c->tiles_dirty) return fail(SMCCAT_ESTATE, "refresh the particles first");
    const Dims& d = c->d;
    PruneArgs& a = v->pa;
    a = PruneArgs{};
    a.d = d;
    a.first = first;
    a.tile_begin = c->tile_off[first];
    a.tiles = c->d_tiles;
    a.codes = c->d_codes;
    a.perm = c->d_perm;
    a.wt = c->patterns ? c->d_wt : nullptr;
    a.Pm = c->d_Pm;
    a.spec = c->d_spec;
    a.sws = c->d_sws;
    a.isinv = c->d_isinv;
    a.invchar = c->d_invchar;
    a.CL = c->d_CL;
    a.fp32 = c->esz == 4;
    a.LSC = c->d_LSC;
    a.site_lnl = c->d_site_lnl;
    a.partial = c->d_partial;
    a.status = c->d_status;
    a.wait_limit = c->wait_limit;
    v->ntiles = c->tile_off[first + count] - c->tile_off[first];
    v->variant = c->prune_variant;
    v->lnl = c->d_lnl;
    v->lnl_old = c->d_lnl_old;
    v->tile_off = c->d_tile_off;
    v->sws = c->d_sws;
    v->spec = c->d_spec;
    v->Pm = c->d_Pm;
    v->fp32 = c->esz == 4;
    v->status = c->d_status;
    v->st = c->st;
    return SMCCAT_OK;
}
const Dims& smccat::dims_of(const smccat_ctx* c) { return c->d; }
int smccat::model_flags_of(const smccat_ctx* c) { return c->cfg.model_flags; }
uint32_t smccat::wait_limit_of(const smccat_ctx* c) { return c->wait_limit; }
int smccat::device_of(const smccat_ctx* c) { return c->cfg.device; }
int smccat::reassign_group_of(const smccat_ctx* c) { return c->reassign_group; }
const double* smccat::lnl_device(const smccat_ctx* c) { return c->d_lnl; }
const uint8_t* smccat::codes_device(const smccat_ctx* c) { return c->d_codes; }
const uint8_t* smccat::codes_host(const smccat_ctx* c) { return c->codes.data(); }
const double* smccat::isinv_device(const smccat_ctx* c) { return c->d_isinv; }
const int32_t* smccat::invchar_device(const smccat_ctx* c) { return c->d_invchar; }

extern "C" {

int smccat_get_lnl(smccat_ctx* c, int32_t first, int32_t count, double* out) {
    int rc = check_range(c, first, count);
    if (rc) return rc;
    if (!out) return fail(SMCCAT_EINVAL, "null argument");
    CK(cudaSetDevice(c->cfg.device));
    CK(d2h(c, out, c->d_lnl + first, count * sizeof(double)));
    CK(cudaStreamSynchronize(c->st));
    return SMCCAT_OK;
}

int smccat_get_site_lnl(smccat_ctx* c, int32_t p, double* out) {
    int rc = check_particle(c, p);
    if (rc) return rc;
    if (!out) return fail(SMCCAT_EINVAL, "null argument");
    CK(cudaSetDevice(c->cfg.device));
    CK(d2h(c, out, c->d_site_lnl + (size_t)p * c->d.S, c->d.S * sizeof(double)));
    CK(cudaStreamSynchronize(c->st));
    if (c->patterns) {  // only each slot's own site was written
        const std::vector<int32_t>& rep = c->slots[p].site_rep;
        for (int x = 0; x < c->d.S; ++x) out[x] = out[rep[x]];
    }
    return SMCCAT_OK;
}

int smccat_get_transition_matrix(smccat_ctx* c, int32_t p, int32_t k, int32_t node, int32_t r,
                                 double* out400) {
    int rc = check_particle(c, p);
    if (rc) return rc;
    const Slot& s = c->slots[p];
    const Dims& d = c->d;
    if (!out400 || k < 0 || k >= s.cur.K || node < 0 || node >= d.N || node == s.cur.root ||
        r < 0 || r >= d.R)
        return fail(SMCCAT_EINVAL, "bad class / node / rate index");
    if (s.pending && !s.refreshed) return fail(SMCCAT_ESTATE, "particle has unrefreshed edits");
    unsigned char blk[kPBlock * 8];
    const int pws = s.cur.pws[node] ^ ((s.cur.sws[k] & kSwsP) ? 1 : 0);
    const size_t off = ((((size_t)p * d.Kmax + k) * d.N + node) * 2 + pws) *
                           (size_t)d.R * kPBlock + (size_t)r * kPBlock;
    CK(cudaSetDevice(c->cfg.device));
    CK(d2h(c, blk, c->d_Pm + off * c->esz, (size_t)kPBlock * c->esz));
    CK(cudaStreamSynchronize(c->st));
    for (int i = 0; i < kStates; ++i)
        for (int j = 0; j < kStates; ++j) {
            const size_t e = (size_t)i * kPCols + j;
            out400[i * kStates + j] = c->esz == 4 ? (double)reinterpret_cast<const float*>(blk)[e]
                                                  : reinterpret_cast<const double*>(blk)[e];
        }
    return SMCCAT_OK;
}

int smccat_set_branch_lengths(smccat_ctx* c, int32_t p, int32_t n, const int32_t* nodes,
                              const double* lengths) {
    int rc = check_particle(c, p);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!nodes || !lengths))) return fail(SMCCAT_EINVAL, "null argument");
    Slot& s = c->slots[p];
    for (int i = 0; i < n; ++i) {
        const int x = nodes[i];
        if (x < 0 || x >= c->d.N || x == s.cur.root) return fail(SMCCAT_EINVAL, "node has no edge to set");
        if (!(lengths[i] >= 0.0) || !std::isfinite(lengths[i])) return fail(SMCCAT_EINVAL, "bad branch length");
    }
    for (int i = 0; i < n; ++i) {
        const int x = nodes[i];
        s.cur.branch[x] = lengths[i];
        s.dirty_p[x] = 1;
        mark_up(s, s.cur.parent[x]);
    }
    s.pending = true;
    return SMCCAT_OK;
}

int smccat_set_topology(smccat_ctx* c, int32_t p, const int32_t* parent, const double* branch) {
    int rc = check_particle(c, p);
    if (rc) return rc;
    if (!parent || !branch) return fail(SMCCAT_EINVAL, "null argument");
    const int N = c->d.N;
    Mirror nt;
    if (!build_tree(c->d.T, parent, &nt)) return fail(SMCCAT_EINVAL, "not a rooted binary tree");
    for (int n = 0; n < N; ++n)
        if (!(branch[n] >= 0.0) || !std::isfinite(branch[n])) return fail(SMCCAT_EINVAL, "bad branch length");
    Slot& s = c->slots[p];
    std::vector<int32_t> oldpar = s.cur.parent;
    s.cur.parent = nt.parent;
    s.cur.kids = nt.kids;
    s.cur.post = nt.post;
    s.cur.root = nt.root;
    for (int n = 0; n < N; ++n) {
        if (oldpar[n] != parent[n]) {
            // both the old and the new parent now have different children
            mark_up(s, parent[n]);
            if (oldpar[n] >= 0) mark_up(s, oldpar[n]);
        }
        if (branch[n] != s.cur.branch[n]) {
            s.cur.branch[n] = branch[n];
            s.dirty_p[n] = 1;
            mark_up(s, parent[n]);
        }
    }
    s.pending = true;
    return SMCCAT_OK;
}

int smccat_set_pinv(smccat_ctx* c, int32_t p, double pinv) {
    int rc = check_particle(c, p);
    if (rc) return rc;
    if (!(pinv >= 0.0 && pinv < 1.0)) return fail(SMCCAT_EINVAL, "pinv must be in [0, 1)");
    c->slots[p].cur.pinv = pinv;
    c->slots[p].pending = true;
    return SMCCAT_OK;
}

int smccat_set_shape(smccat_ctx* c, int32_t p, double shape) {
    int rc = check_particle(c, p);
    if (rc) return rc;
    if (!(shape > 0.0) || !std::isfinite(shape)) return fail(SMCCAT_EINVAL, "shape must be > 0");
    Slot& s = c->slots[p];
    s.cur.shape = shape;
    discretize_gamma(shape, c->d.R, s.cur.rates);
    std::fill(s.dirty_p.begin(), s.dirty_p.end(), 1);
    for (int n : s.cur.post) s.dirty_cl[n] = 1;
    s.pending = true;
    return SMCCAT_OK;
}

int smccat_set_base(smccat_ctx* c, int32_t p, const double* base) {
    int rc = check_particle(c, p);
    if (rc) return rc;
    if (!base) return fail(SMCCAT_EINVAL, "null argument");
    Slot& s = c->slots[p];
    s.cur.base.assign(base, base + kBase);
    std::fill(s.dirty_spec.begin(), s.dirty_spec.begin() + s.cur.K, 1);
    std::fill(s.dirty_p.begin(), s.dirty_p.end(), 1);
    for (int n : s.cur.post) s.dirty_cl[n] = 1;
    s.pending = true;
    return SMCCAT_OK;
}

int smccat_set_class_logits(smccat_ctx* c, int32_t p, int32_t k, const double* logits) {
    int rc = check_particle(c, p);
    if (rc) return rc;
    Slot& s = c->slots[p];
    if (!logits || k < 0 || k >= s.cur.K) return fail(SMCCAT_EINVAL, "bad class index");
    std::copy(logits, logits + kStates, s.cur.logits.begin() + (size_t)k * kStates);
    // Alone, the edit is class-local: only class k's matrices and sites are
    // rebuilt, into that class's other workspaces. With other edits pending
    // (or a second class edited) everything is rebuilt.
    bool others = s.full || s.local_class >= 0;
    for (int i = 0; i < c->d.N && !others; ++i) others = s.dirty_cl[i] || s.dirty_p[i];
    for (int j = 0; j < s.cur.K && !others; ++j) others = s.dirty_spec[j] && j != k;
    s.dirty_spec[k] = 1;
    if (!others && !s.pending) {
        s.local_class = k;
    } else {
        s.local_class = -1;
        std::fill(s.dirty_p.begin(), s.dirty_p.end(), 1);
        for (int n : s.cur.post) s.dirty_cl[n] = 1;
    }
    s.pending = true;
    return SMCCAT_OK;
}

int smccat_accept(smccat_ctx* c, int32_t first, int32_t count, const uint8_t* mask) {
    int rc = check_range(c, first, count);
    if (rc) return rc;
    if (!mask) return fail(SMCCAT_EINVAL, "null argument");
    for (int i = 0; i < count; ++i) {
        const Slot& s = c->slots[first + i];
        if (!s.loaded) return fail(SMCCAT_ESTATE, "particle has no state loaded");
        if (s.pending && !s.refreshed)
            return fail(SMCCAT_ESTATE, "particle " + std::to_string(first + i) +
                                           " has edits that were never refreshed");
    }
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaEventSynchronize(c->plan_done));
    uint8_t* hm = reinterpret_cast<uint8_t*>(c->h_plan);
    for (int i = 0; i < count; ++i) hm[i] = mask[i] ? 1 : 0;
    CK(h2d(c, c->d_plan, hm, count));
    CK(cudaEventRecord(c->plan_done, c->st));
    CK(launch(c, SMCCAT_KERNEL_ACCEPT, [&] {
        return launch_accept(c->d_lnl, c->d_lnl_old, reinterpret_cast<uint8_t*>(c->d_plan), first, count, c->st);
    }));
    for (int i = 0; i < count; ++i) {
        Slot& s = c->slots[first + i];
        if (mask[i]) s.old = s.cur;
        else s.cur = s.old;
        s.local_class = -1;
        std::fill(s.dirty_spec.begin(), s.dirty_spec.end(), 0);
        std::fill(s.dirty_p.begin(), s.dirty_p.end(), 0);
        std::fill(s.dirty_cl.begin(), s.dirty_cl.end(), 0);
        s.pending = false;
        s.refreshed = false;
    }
    return SMCCAT_OK;
}

int smccat_autotune(smccat_ctx* c, int32_t reps, int32_t* variant_out, double* ms_out) {
    NvtxRange range("smccat_autotune");
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    int n = 0;
    while (n < c->cfg.max_particles && c->slots[n].loaded) ++n;
    if (n == 0) return fail(SMCCAT_ESTATE, "autotune needs loaded particles");
    for (int i = 0; i < n; ++i)
        if (c->slots[i].pending && !c->slots[i].commit_on_refresh)
            return fail(SMCCAT_ESTATE, "autotune needs particles without pending edits");
    reps = std::max(1, reps);
    const bool timing = c->timing;
    const smccat_profile saved = c->prof;
    const int nv = prune_variants(c->d.R, c->esz == 4);
    int best = 0;
    double best_ms = INFINITY;
    for (int v = 0; v < nv; ++v) {
        select_variant(c, v);
        int rc = smccat_refresh(c, 0, n, SMCCAT_REFRESH_FULL);  // warm-up, also commits loads
        if (rc) return rc;
        c->timing = true;
        c->ev_used.clear();
        c->prof = smccat_profile{};
        for (int k = 0; k < reps; ++k) {
            rc = smccat_refresh(c, 0, n, SMCCAT_REFRESH_FULL);
            if (rc) return rc;
        }
        smccat_profile pr;
        rc = smccat_get_profile(c, &pr);
        if (rc) return rc;
        const double ms = pr.ms[SMCCAT_KERNEL_PRUNE] / reps;
        if (ms_out) ms_out[v] = ms;
        if (ms < best_ms) { best_ms = ms; best = v; }
        c->timing = false;
    }
    select_variant(c, best);
    c->timing = timing;
    c->ev_used.clear();
    c->prof = saved;
    if (variant_out) *variant_out = best;
    return SMCCAT_OK;
}

int smccat_kernel_variants(smccat_ctx* c, int32_t* count, int32_t* current) {
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    if (count) *count = prune_variants(c->d.R, c->esz == 4);
    if (current) *current = c->prune_variant;
    return SMCCAT_OK;
}

int smccat_set_kernel_variant(smccat_ctx* c, int32_t variant) {
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    if (variant < 0 || variant >= prune_variants(c->d.R, c->esz == 4))
        return fail(SMCCAT_EINVAL, "kernel variant out of range");
    select_variant(c, variant);
    return SMCCAT_OK;
}

int smccat_set_wait_limit(smccat_ctx* c, int32_t polls) {
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    c->wait_limit = polls < 0 ? kDrainPolls : static_cast<uint32_t>(polls);
    return SMCCAT_OK;
}

int smccat_set_reassign_group(smccat_ctx* c, int32_t n) {
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    c->reassign_group = n > 0 ? n : 0;
    return SMCCAT_OK;
}

int smccat_sync(smccat_ctx* c) {
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->st));
    return SMCCAT_OK;
}

int smccat_get_stream(smccat_ctx* c, void** stream) {
    if (!c || !stream) return fail(SMCCAT_EINVAL, "null argument");
    *stream = (void*)c->st;
    return SMCCAT_OK;
}

int smccat_set_profiling(smccat_ctx* c, int32_t enable) {
    if (!c) return fail(SMCCAT_EINVAL, "null context");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->st));
    c->timing = enable != 0;
    c->prof = smccat_profile{};
    c->ev_used.clear();
    return SMCCAT_OK;
}

int smccat_get_profile(smccat_ctx* c, smccat_profile* out) {
    if (!c || !out) return fail(SMCCAT_EINVAL, "null argument");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->st));
    for (const auto& u : c->ev_used) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev_pool[u.second], c->ev_pool[u.second + 1]));
        c->prof.ms[u.first] += ms;
    }
    c->ev_used.clear();
    *out = c->prof;
    return SMCCAT_OK;
}

}  // extern "C"
