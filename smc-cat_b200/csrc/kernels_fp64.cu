// FP64 kernels of the B200 likelihood engine.
//
//   spec_kernel   one warp per (particle, class): spectral decomposition of the
//                 class's rate matrix (spectral.cuh).
//   pmat_kernel   one CTA per (particle, class, chunk of dirty nodes):
//                 P(t r) = L diag(exp(lambda t r)) Rm for every rate
//                 (TransitionProbabilityClass.cpp:83-95), row-major with a
//                 row-sum column, register-tiled.
//   prune_kernel  one warp per (rate, tile of <= 32 W same-class sites, W sites
//                 per lane), R warps per CTA: walks the particle's dirty
//                 internal nodes in post-order (Particle.cpp:577-626). Each warp
//                 stages its two children's P blocks into shared memory with TMA
//                 bulk copies (double-buffered, mbarrier-tracked, the next node's
//                 copy in flight while the current node computes), keeps the
//                 partial it just produced in registers (in a post-order of an
//                 upward-closed dirty set the previous node is always a child of
//                 the next one), reads at most one child partial back from
//                 memory, rescales each (site, rate) by an exact power of two,
//                 then the CTA reduces the root (Particle.cpp:634-674):
//                 log-sum-exp over rates, +I, warp sum.
//   reduce_kernel per particle, sums the tile partials in a fixed order.
#include <cuda_runtime.h>
#include <algorithm>
#include <math.h>

#include "kernels.h"
#include "spectral.cuh"

namespace smccat {

namespace {


__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bulk (non-tensor) TMA copy global -> shared, completion counted on `bar`.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar` to complete; false after `limit` polls.
__device__ __noinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

template <class T> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

// Exact power-of-two rescale: returns the exponent e with mx = f 2^e, f in [0.5, 1).
__device__ __forceinline__ int exponent_of(double mx) { int e; frexp(mx, &e); return e; }
__device__ __forceinline__ int exponent_of(float mx) { int e; frexpf(mx, &e); return e; }
__device__ __forceinline__ double pow2(double, int e) { return ldexp(1.0, e); }
__device__ __forceinline__ float pow2(float, int e) { return ldexpf(1.0f, e); }

// max(0, v[0..19]) as a depth-5 tree instead of a 20-long dependent chain.
template <class T>
__device__ __forceinline__ T max20(const T* v) {
    T m[10];
#pragma unroll
    for (int i = 0; i < 10; ++i) m[i] = fmax(v[2 * i], v[2 * i + 1]);
#pragma unroll
    for (int i = 0; i < 5; ++i) m[i] = fmax(m[2 * i], m[2 * i + 1]);
    return fmax(fmax(fmax(m[0], m[1]), fmax(m[2], m[3])), fmax(m[4], T(0)));
}

// acc[w][i] = sum_j P[i][j] x[w][j] for the W sites of a lane, P row-major
// (stride kPCols) in shared memory, every lane reading the same element.
// MUL: multiply the result into acc instead of assigning it.
// Row dot products, RB rows in flight (2 RB independent FMA chains), P read
// as pairs: each shared-memory load feeds 2 W FMAs.
// The diagonal term is added last. For the branch lengths of a tree P is close
// to the identity: summed after P_ii x_i, off-diagonal terms below half an ulp
// of the running sum would be rounded away every time -- a bias of one sign
// that, in FP32, costs ~1e-3 nats per 2,000 sites. Summed first, they keep
// their weight. (i and j are compile-time after unrolling: no run-time cost.)
template <class T, int W, bool MUL, int RB>
__device__ __forceinline__ void matvec(const T* __restrict__ P, const T (*x)[kStates],
                                       T (*acc)[kStates]) {
    static_assert(kStates % RB == 0, "rows in flight must divide the state count");
    using P2 = typename Pair<T>::type;
#pragma unroll
    for (int i0 = 0; i0 < kStates; i0 += RB) {
        T s0[RB][W], s1[RB][W], pd[RB];
#pragma unroll
        for (int b = 0; b < RB; ++b) {
            pd[b] = 0;
#pragma unroll
            for (int w = 0; w < W; ++w) s0[b][w] = s1[b][w] = 0;
        }
#pragma unroll
        for (int j = 0; j < kStates / 2; ++j) {
#pragma unroll
            for (int b = 0; b < RB; ++b) {
                const int i = i0 + b;
                const P2 p2 = reinterpret_cast<const P2*>(P + i * kPCols)[j];
                if (2 * j == i) pd[b] = p2.x;
                if (2 * j + 1 == i) pd[b] = p2.y;
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    if (2 * j != i) s0[b][w] = fma(p2.x, x[w][2 * j], s0[b][w]);
                    if (2 * j + 1 != i) s1[b][w] = fma(p2.y, x[w][2 * j + 1], s1[b][w]);
                }
            }
        }
#pragma unroll
        for (int b = 0; b < RB; ++b) {
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const T r = fma(pd[b], x[w][i0 + b], s0[b][w] + s1[b][w]);
                if (MUL) acc[w][i0 + b] *= r;
                else acc[w][i0 + b] = r;
            }
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Spectral decomposition of one class (one warp).
__global__ void __launch_bounds__(32) spec_kernel(const SpecJob* __restrict__ jobs,
                                                  double* __restrict__ spec, Dims d) {
    const SpecJob* job = jobs + blockIdx.x;
    double* rec = spec + (((size_t)job->p * d.Kmax + job->k) * 2 + (job->sws & kSwsSpec)) * kSpecStride;
    spectral_decompose_warp(job->base, job->logits, rec);
}

// ---------------------------------------------------------------------------
// Transition matrices of one class for a chunk of a particle's dirty nodes,
// every rate: P(t r) = (L diag(exp(lambda t r))) [Rm | Rm 1] with a 21st
// column of row sums and a zero pad column. The class's eigensystem is staged
// in shared memory once per CTA; each thread owns a 4 x 4 output tile of one
// rate (5 row blocks x 6 column blocks x R rates), so every shared-memory load
// feeds several FMAs. Summation order over m is that of the plain triple loop.
// Computed in FP64; stored as T (rounded once for the FP32 path).
constexpr int kPmThreads = 128;
// Position of column c in a row of nb 4-column blocks stored as [half][block][2]:
// the first pairs of all blocks, then the second pairs.
__device__ __forceinline__ int pm_ilv(int c, int nb) {
    return (((c >> 1) & 1) * nb + (c >> 2)) * 2 + (c & 1);
}
template <class T>
__global__ void __launch_bounds__(kPmThreads) pmat_kernel(const PmJob* __restrict__ mjobs,
                                                          const PJob* __restrict__ jobs,
                                                          const PartHdr* __restrict__ hdr, int first,
                                                          const uint8_t* __restrict__ sws,
                                                          const double* __restrict__ spec,
                                                          T* __restrict__ Pm, Dims d) {
    const PmJob mj = mjobs[blockIdx.x];
    if (mj.nj <= 0) return;  // fixed-shape job grids (device-side moves) leave empty entries
    const PartHdr* h = hdr + mj.i;
    const int p = first + mj.i;
    // Rows in 4-column-block interleaved order (pm_ilv): the pair loads of a
    // warp's tiles fall on distinct banks.
    __shared__ __align__(16) double Lt[kStates][kStates];  // Lt[m][ilv(i)] = L[i][m]
    __shared__ __align__(16) double Rx[kStates][24];       // Rm | row sums | zeros
    __shared__ double lam[kStates];
    __shared__ double ex[kPmChunk][kMaxRates][kStates];
    __shared__ size_t obase[kPmChunk];
    const int tid = threadIdx.x;
    const uint8_t sb = sws[(size_t)p * d.Kmax + mj.k];
    const double* rec = spec + (((size_t)p * d.Kmax + mj.k) * 2 + (sb & kSwsSpec)) * kSpecStride;
    for (int idx = tid; idx < kStates * kStates; idx += kPmThreads) {
        const int a = idx / kStates, b = idx % kStates;
        Lt[b][pm_ilv(a, 5)] = rec[kSpecL + idx];
        Rx[a][pm_ilv(b, 6)] = rec[kSpecRm + idx];
    }
    if (tid < kStates) {
        double s = 0.0;
        for (int j = 0; j < kStates; ++j) s += rec[kSpecRm + tid * kStates + j];
        Rx[tid][pm_ilv(kStates, 6)] = s;
        Rx[tid][pm_ilv(21, 6)] = Rx[tid][pm_ilv(22, 6)] = Rx[tid][pm_ilv(23, 6)] = 0.0;
        lam[tid] = rec[kSpecLam + tid];
    }
    if (tid < mj.nj) {
        const PJob pj = jobs[mj.j0 + tid];
        const int pws = pj.pws ^ ((sb & kSwsP) ? 1 : 0);  // the class's matrix-workspace flip
        obase[tid] = ((((size_t)p * d.Kmax + mj.k) * d.N + pj.node) * 2 + pws) * (size_t)d.R * kPBlock;
    }
    __syncthreads();
    // Every exponential of the chunk in one phase, then no barrier per node.
    const int per_node = d.R * kStates;
    for (int idx = tid; idx < mj.nj * per_node; idx += kPmThreads) {
        const int q = idx / per_node, r = (idx % per_node) / kStates, m = idx % kStates;
        ex[q][r][m] = exp(lam[m] * jobs[mj.j0 + q].t * h->rates[r]);
    }
    __syncthreads();
    using P2 = typename Pair<T>::type;
    const int ntile = 30 * d.R;
    for (int t = tid; t < ntile; t += kPmThreads) {
        const int r = t / 30, i0 = 4 * ((t % 30) / 6), j0 = 4 * (t % 6);
        for (int q = 0; q < mj.nj; ++q) {
            double acc[4][4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
            }
#pragma unroll 4
            for (int m = 0; m < kStates; ++m) {
                const double e = ex[q][r][m];
                const double2 a01 = *reinterpret_cast<const double2*>(&Lt[m][pm_ilv(i0, 5)]);
                const double2 a23 = *reinterpret_cast<const double2*>(&Lt[m][pm_ilv(i0 + 2, 5)]);
                const double2 b01 = *reinterpret_cast<const double2*>(&Rx[m][pm_ilv(j0, 6)]);
                const double2 b23 = *reinterpret_cast<const double2*>(&Rx[m][pm_ilv(j0 + 2, 6)]);
                const double av[4] = {a01.x * e, a01.y * e, a23.x * e, a23.y * e};
                const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
                }
            }
            // Pair stores: row offsets and j0 are even, so every pair is aligned.
            T* o = Pm + obase[q] + (size_t)r * kPBlock + j0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                P2* row = reinterpret_cast<P2*>(o + (i0 + u) * kPCols);
                row[0] = P2{static_cast<T>(acc[u][0]), static_cast<T>(acc[u][1])};
                if (j0 + 4 <= kPCols) row[1] = P2{static_cast<T>(acc[u][2]), static_cast<T>(acc[u][3])};
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Pruning + root reduction of one tile: warp r handles rate category r.
// MINB = CTAs per SM the register allocation must allow (the register cap is
// 65536 / (32 R MINB)); the autotuner picks among the instantiated values.
// W = sites per lane: the tile has up to 32 W slots, lane l owning slots
// l, l + 32, ...; W = 2 halves the shared-memory loads per FMA at the cost of
// registers. RB = mat-vec rows in flight (see matvec).
// T = storage and arithmetic type of partials and transition matrices
// (double, or float for the mixed-precision path); log-scalers and the root
// reduction are FP64 in both.
// One tile. `phase` holds each P buffer's next barrier parity; the barriers
// are initialised when `init` is set (a CTA's first tile) and reused after.
// Bounded waits: once a wait gives up (a.wait_limit polls), the warp issues no
// further copies, and lane 0 -- the lane that issued them -- drains every copy
// still in flight (waiting on its un-toggled parity, with the full limit)
// before the buffers are reused. Returns false, uniformly across the CTA,
// when any warp gave up.
// EV: the instance for evaluation mode (PruneArgs::eval_k / eval_kp and the
// site lists). The refresh instance keeps only the eval_k test: without the
// site-list and per-particle code its register allocation spills less
// (20 / 12 bytes instead of 44 / 56 at <double, 4, 3, 1, 4>).
template <class T, int R, int MINB, int W, int RB, bool EV>
__device__ __forceinline__ bool prune_tile(const PruneArgs& a, const int tile_id, uint32_t& phase, bool init) {
    const Dims d = a.d;
    const Tile tl = a.tiles[tile_id];
    const int p = tl.p;
    const PartHdr* h = a.hdr + (p - a.first);
    constexpr uint32_t kPBytes = kPBlock * sizeof(T);

    extern __shared__ __align__(128) unsigned char smem_raw[];  // [R warps][2 buffers][2 children][kPBlock]
    __shared__ __align__(8) uint64_t bars[R][2];
    __shared__ int bad;

    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
    // Evaluation mode: the class under evaluation and, over a site list, the
    // sites the tile's slots stand for.
    int nsl = tl.nslots;
    const int32_t* sperm = a.perm + (size_t)p * d.S;
    if constexpr (EV) {
        const int ek0 = a.eval_kp ? a.eval_kp[p - a.first] : a.eval_k;
        if (ek0 >= 0 && a.eval_perm != nullptr) {
            nsl = min(tl.nslots, a.eval_nv[p - a.first] - tl.slot0);
            sperm = a.eval_perm + (size_t)(p - a.first) * d.S;
        }
    }
    const bool valid = lane < nsl;  // the lane owns at least one slot
    // A lane's unused slots alias its first slot (or the tile's first): they
    // are computed like the others and never stored.
    bool vw[W];
    int site[W], col[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
        vw[w] = lane + 32 * w < nsl;
        const int slot = tl.slot0 + (vw[w] ? lane + 32 * w : (valid ? lane : 0));
        site[w] = sperm[slot];
        col[w] = r * d.Spad + slot;
    }
    T* buf = reinterpret_cast<T*>(smem_raw) + (size_t)r * 4 * kPBlock;
    // Root-reduction row of warp rr: the start of that warp's own P buffers,
    // free once the warp has left its node loop (every copy into them has been
    // waited on). Keeping it out of static shared memory lets four CTAs share
    // an SM.
    auto red = [&](int rr) {
        return reinterpret_cast<double*>(smem_raw + (size_t)rr * 4 * kPBlock * sizeof(T));
    };

    const size_t j_stride = (size_t)R * d.Spad;
    const size_t ws_stride = (size_t)kStates * j_stride;
    const size_t node_stride = 2 * ws_stride;
    const size_t lws_stride = j_stride;
    T* CLp = static_cast<T*>(a.CL) + (size_t)p * d.NI * node_stride;
    double* LSCp = a.LSC + (size_t)p * d.NI * 2 * lws_stride;
    // The class whose matrices and frequencies the tile runs: its own, or the
    // class under evaluation.
    const int ek = EV ? (a.eval_kp ? a.eval_kp[p - a.first] : a.eval_k) : a.eval_k;
    const int kc = ek >= 0 ? ek : tl.k;
    const T* Pcls = static_cast<const T*>(a.Pm) +
                    ((size_t)p * d.Kmax + kc) * d.N * 2 * (size_t)R * kPBlock + (size_t)r * kPBlock;
    auto pblock = [&](int child, int pws) {
        return Pcls + ((size_t)child * 2 + pws) * (size_t)R * kPBlock;
    };

    if (threadIdx.x == 0) bad = 0;
    if (init && lane == 0) {
        mbar_init(&bars[r][0], 1);
        mbar_init(&bars[r][1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (!h->active) return true;  // uniform across the CTA (after the barriers exist)
    const int ej = ek >= 0 ? a.eval_map[p - a.first] : 0;
    if (EV ? (a.eval_kp ? (ek < 0 || ej < 0) : (ek < 0 || ej < 0 || ek >= h->num_classes))
           : (ek >= 0 && (ej < 0 || ek >= h->num_classes)))
        return true;  // uniform as well
    if (EV && nsl <= 0) return true;  // past the end of the site list

    // A class-local refresh of another class leaves this tile's partials as
    // they are: only its root reduction reruns. In evaluation mode the plan
    // names the free partial workspaces (the tile's own class flips them like
    // the committed ones) and the evaluated class's matrices.
    const int cnt = (ek < 0 && h->cls_only >= 0 && h->cls_only != tl.k) ? 0 : h->node_cnt;
    const int wfl = ek >= 0 ? (class_ws_flip(a.sws, p, d.Kmax, tl.k) & 7) | (class_ws_flip(a.sws, p, d.Kmax, ek) & 24)
                            : class_ws_flip(a.sws, p, d.Kmax, tl.k);
    const NodeJob* nodes = a.nodes + h->node_off;
    uint32_t pend = 0;  // lane 0: bit b set while a copy into buffer b is not yet waited on
    if (cnt > 0 && lane == 0) {
        fence_proxy_async();  // a previous tile's root rows were written here
        NodeJob nj = nodes[0];
        nj.ws ^= wfl;
        mbar_expect_tx(&bars[r][0], 2 * kPBytes);
        tma_load_1d(buf, pblock(nj.c1, (nj.ws >> 3) & 1), kPBytes, &bars[r][0]);
        tma_load_1d(buf + kPBlock, pblock(nj.c2, (nj.ws >> 4) & 1), kPBytes, &bars[r][0]);
        pend = 1u;
    }

    T y[W][kStates];
    double lsc[W];
#pragma unroll
    for (int w = 0; w < W; ++w) lsc[w] = 0.0;
    int prev = -1;
    bool ok = true;
    for (int q = 0; q < cnt; ++q) {
        const int b = q & 1;
        NodeJob nj = nodes[q];
        nj.ws ^= wfl;
        if (ok && q + 1 < cnt && lane == 0) {
            // Buffer b^1 was last read at node q-1 (the warp synchronised after it).
            NodeJob nx = nodes[q + 1];
            nx.ws ^= wfl;
            fence_proxy_async();
            mbar_expect_tx(&bars[r][b ^ 1], 2 * kPBytes);
            tma_load_1d(buf + (b ^ 1) * 2 * kPBlock, pblock(nx.c1, (nx.ws >> 3) & 1), kPBytes,
                        &bars[r][b ^ 1]);
            tma_load_1d(buf + (b ^ 1) * 2 * kPBlock + kPBlock, pblock(nx.c2, (nx.ws >> 4) & 1),
                        kPBytes, &bars[r][b ^ 1]);
            pend |= 1u << (b ^ 1);
        }
        // Roles: the child computed just before (if any) is in registers; the
        // other child is a tip (gather) or a stored partial (load).
        const bool c1prev = nj.c1 == prev, c2prev = nj.c2 == prev;
        const int oi = c1prev ? 1 : 0;  // index of the "other" child (c1 when neither is prev)
        const int o = oi ? nj.c2 : nj.c1;
        const int fi = 1 - oi;          // index of the register / first child
        double lsc_o[W];
        int code_o[W];
#pragma unroll
        for (int w = 0; w < W; ++w) { lsc_o[w] = 0.0; code_o[w] = 0; }
        if (valid) {
            if (o >= d.T) {
                const int wsc = (nj.ws >> (1 + oi)) & 1;
                const double* lp = LSCp + (size_t)(o - d.T) * 2 * lws_stride + wsc * lws_stride;
#pragma unroll
                for (int w = 0; w < W; ++w) lsc_o[w] = lp[col[w]];
            } else {
                const uint8_t* cp = a.codes + (size_t)o * d.S;
#pragma unroll
                for (int w = 0; w < W; ++w) code_o[w] = cp[site[w]];
            }
        }
        if (ok) {
            if (mbar_wait_bounded(&bars[r][b], (phase >> b) & 1, a.wait_limit)) {
                phase ^= 1u << b;
                pend &= ~(1u << b);
            } else {
                ok = false;
                atomicOr(a.status, 2);
            }
        }
        if (ok && valid) {
            const T* Pf = buf + (size_t)(b * 2 + fi) * kPBlock;
            const T* Po = buf + (size_t)(b * 2 + oi) * kPBlock;
            T acc[W][kStates];
            double lsc_f[W];
            if (c1prev || c2prev) {
                matvec<T, W, false, RB>(Pf, y, acc);
#pragma unroll
                for (int w = 0; w < W; ++w) lsc_f[w] = lsc[w];
            } else {
                // Neither child was just computed (both-tip nodes, or a list that
                // is not a plain post-order): the first child comes from memory.
                const int f = fi ? nj.c2 : nj.c1;
                if (f >= d.T) {
                    const int wsf = (nj.ws >> (1 + fi)) & 1;
                    const T* fp = CLp + (size_t)(f - d.T) * node_stride + wsf * ws_stride;
                    const double* lp = LSCp + (size_t)(f - d.T) * 2 * lws_stride + wsf * lws_stride;
#pragma unroll
                    for (int w = 0; w < W; ++w) {
#pragma unroll
                        for (int j = 0; j < kStates; ++j) y[w][j] = fp[col[w] + j * j_stride];
                        lsc_f[w] = lp[col[w]];
                    }
                    matvec<T, W, false, RB>(Pf, y, acc);
                } else {
                    const uint8_t* cp = a.codes + (size_t)f * d.S;
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const int code = cp[site[w]];
                        const int cc = code < kStates ? code : kStates;
#pragma unroll
                        for (int i = 0; i < kStates; ++i) acc[w][i] = Pf[i * kPCols + cc];
                        lsc_f[w] = 0.0;
                    }
                }
            }
            if (o >= d.T) {
                // The register child is consumed; its registers now hold the
                // other child's stored partial, folded in row by row.
                const int wsc = (nj.ws >> (1 + oi)) & 1;
                const T* xp = CLp + (size_t)(o - d.T) * node_stride + wsc * ws_stride;
#pragma unroll
                for (int w = 0; w < W; ++w) {
#pragma unroll
                    for (int j = 0; j < kStates; ++j) y[w][j] = xp[col[w] + j * j_stride];
                }
                matvec<T, W, true, RB>(Po, y, acc);
            } else {
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    const int cc = code_o[w] < kStates ? code_o[w] : kStates;
#pragma unroll
                    for (int i = 0; i < kStates; ++i) acc[w][i] *= Po[i * kPCols + cc];
                }
            }
            const int wso = nj.ws & 1;
            T* out = CLp + (size_t)(nj.node - d.T) * node_stride + wso * ws_stride;
            double* lout = LSCp + (size_t)(nj.node - d.T) * 2 * lws_stride + wso * lws_stride;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const T mx = max20(acc[w]);
                double l;
                if (mx > 0) {
                    const int e = exponent_of(mx);
                    const T sc = pow2(mx, -e);
#pragma unroll
                    for (int i = 0; i < kStates; ++i) acc[w][i] *= sc;
                    l = e * 0.69314718055994530942;
                } else {
                    l = (mx == 0) ? -INFINITY : NAN;
                }
                lsc[w] = l + lsc_f[w] + lsc_o[w];
#pragma unroll
                for (int j = 0; j < kStates; ++j) y[w][j] = acc[w][j];
                if (vw[w]) {
#pragma unroll
                    for (int j = 0; j < kStates; ++j) out[col[w] + j * j_stride] = acc[w][j];
                    lout[col[w]] = lsc[w];
                }
            }
        }
        prev = nj.node;
        __syncwarp();
    }
    if (!ok) bad = 1;
    // Let every copy lane 0 issued and never waited on land before the warp's
    // buffers are reused (the root rows below) or the CTA exits. Each such
    // copy's phase is the un-toggled parity of its buffer.
    if (lane == 0 && pend) {
#pragma unroll
        for (int bb = 0; bb < 2; ++bb)
            if ((pend >> bb) & 1u) {
                if (mbar_wait_bounded(&bars[r][bb], (phase >> bb) & 1, kDrainPolls)) phase ^= 1u << bb;
                else bad = 1;
            }
    }
    __syncwarp();  // the warp's buffers are free from here on (red(r) reuses them)
    // Root reduction for this tile.
    if (cnt == 0 && valid) {
        const int rws = h->root_ws ^ (wfl & 1);
        const T* xp = CLp + (size_t)(h->root - d.T) * node_stride + rws * ws_stride;
        const double* lp = LSCp + (size_t)(h->root - d.T) * 2 * lws_stride + rws * lws_stride;
#pragma unroll
        for (int w = 0; w < W; ++w) {
#pragma unroll
            for (int j = 0; j < kStates; ++j) y[w][j] = xp[col[w] + j * j_stride];
            lsc[w] = lp[col[w]];
        }
    }
    const double* rec =
        a.spec + (((size_t)p * d.Kmax + kc) * 2 + (a.sws[(size_t)p * d.Kmax + kc] & kSwsSpec)) * kSpecStride;
    const double* pi = rec + kSpecPi;
    if (valid) {
#pragma unroll
        for (int w = 0; w < W; ++w) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < kStates; ++i) s = fma(pi[i], (double)y[w][i], s);
            red(r)[lane + 32 * w] = log(s) + lsc[w];
        }
    }
    __syncthreads();
    const bool tile_ok = bad == 0;  // read by every thread between the same two barriers
    if (r == 0) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            if (!vw[w]) continue;
            const int q = lane + 32 * w;
            double mx = red(0)[q];
#pragma unroll
            for (int rr = 1; rr < R; ++rr) mx = fmax(mx, red(rr)[q]);
            double lse = mx;
            if (mx > -INFINITY) {
                double se = 0.0;
#pragma unroll
                for (int rr = 0; rr < R; ++rr) se += exp(red(rr)[q] - mx);
                lse = mx + log(se);
            }
            // +I mixing, Particle.cpp:667-670, evaluated in log space.
            const double pinv = h->pinv;
            double u;
            if (pinv > 0.0 && a.isinv[site[w]] != 0) {
                const double la = log1p(-pinv) + lse;
                const double lb = log(pinv * pi[a.invchar[site[w]]]);
                const double m2 = fmax(la, lb);
                u = m2 + log(exp(la - m2) + exp(lb - m2));
            } else {
                u = lse + log1p(-pinv);
            }
            if (bad) u = NAN;
            if (ek >= 0) {
                a.eval_out[((size_t)ej * d.Kmax + ek) * d.S + site[w]] = u;
                continue;
            }
            a.site_lnl[(size_t)p * d.S + site[w]] = u;
            // A compressed slot stands for every site of its (column, class) pair.
            v += a.wt ? u * a.wt[(size_t)p * d.S + tl.slot0 + q] : u;
        }
        v = warp_sum(v);
        if (lane == 0 && ek < 0) a.partial[tile_id] = v;
    }
    return tile_ok;
}

template <class T, int R, int MINB, int W, int RB, bool EV>
__global__ void __launch_bounds__(32 * R, MINB) prune_kernel(const PruneArgs a) {
    uint32_t phase = 0;
    prune_tile<T, R, MINB, W, RB, EV>(a, a.tile_begin + blockIdx.x, phase, true);
}

// Persistent form: one wave of CTAs (the SMs times the CTAs each holds) walks
// the tiles in a grid-stride loop. The copy barriers are initialised once and
// their phases carried from tile to tile; every copy a tile issues is waited
// on inside that tile.
template <class T, int R, int MINB, int W, int RB, bool EV>
__global__ void __launch_bounds__(32 * R, MINB) prune_kernel_persistent(const PruneArgs a, int ntiles) {
    uint32_t phase = 0;
    bool init = true;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const bool ok = prune_tile<T, R, MINB, W, RB, EV>(a, a.tile_begin + t, phase, init);
        init = false;
        __syncthreads();
        if (!ok) break;  // a wait gave up: the CTA's remaining tiles stay unevaluated (status bit 2)
    }
}

__global__ void reduce_kernel(const int32_t* __restrict__ tile_off, const double* __restrict__ partial,
                              const PartHdr* __restrict__ hdr, int first, int count,
                              double* __restrict__ lnl, int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count || !hdr[i].active) return;
    const int p = first + i;
    double s = 0.0;
    for (int t = tile_off[p]; t < tile_off[p + 1]; ++t) s += partial[t];
    lnl[p] = s;
    if (isnan(s)) atomicOr(status, 1);
}

__global__ void accept_kernel(double* __restrict__ lnl, double* __restrict__ lnl_old,
                              const uint8_t* __restrict__ mask, int first, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int p = first + i;
    if (mask[i] == 1) lnl_old[p] = lnl[p];
    else if (mask[i] == 0) lnl[p] = lnl_old[p];
}

// ---------------------------------------------------------------------------
cudaError_t launch_spec(const SpecJob* jobs, int n, double* spec, const Dims& d, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    spec_kernel<<<n, 32, 0, st>>>(jobs, spec, d);
    return cudaGetLastError();
}

cudaError_t launch_pmat(const PmJob* mjobs, int n, const PJob* jobs, const PartHdr* hdr, int first,
                        const uint8_t* sws, const double* spec, void* Pm, bool fp32, const Dims& d,
                        cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (fp32)
        pmat_kernel<float><<<n, kPmThreads, 0, st>>>(mjobs, jobs, hdr, first, sws, spec,
                                                     static_cast<float*>(Pm), d);
    else
        pmat_kernel<double><<<n, kPmThreads, 0, st>>>(mjobs, jobs, hdr, first, sws, spec,
                                                      static_cast<double*>(Pm), d);
    return cudaGetLastError();
}

namespace {

template <class T, int R, int MINB, int W, int RB>
cudaError_t launch_prune_persistent_t(const PruneArgs& a, int ntiles, cudaStream_t st) {
    const size_t smem = sizeof(T) * 4 * (size_t)kPBlock * R;
    const bool ev = a.eval_k >= 0 || a.eval_kp != nullptr;
    auto k = ev ? prune_kernel_persistent<T, R, MINB, W, RB, true> : prune_kernel_persistent<T, R, MINB, W, RB, false>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * R, smem)) != cudaSuccess) return e;
    const int grid = std::max(1, std::min(ntiles, sms * std::max(per_sm, 1)));
    k<<<grid, 32 * R, smem, st>>>(a, ntiles);
    return cudaGetLastError();
}

template <class T, int R, int MINB, int W, int RB>
cudaError_t launch_prune_t(const PruneArgs& a, int ntiles, cudaStream_t st) {
    const size_t smem = sizeof(T) * 4 * (size_t)kPBlock * R;
    const bool ev = a.eval_k >= 0 || a.eval_kp != nullptr;
    auto k = ev ? prune_kernel<T, R, MINB, W, RB, true> : prune_kernel<T, R, MINB, W, RB, false>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // The shared-memory carveout stays at the driver's choice: forcing the
    // maximum (room for a fourth CTA's P buffers) measured slower, since the
    // register-capped variants' spills then miss the smaller L1.
    k<<<ntiles, 32 * R, smem, st>>>(a);
    return cudaGetLastError();
}

// SIMT variants as (sites per lane W, CTAs per SM MINB, mat-vec rows in flight RB):
//   R = 4:  0 (1,4,1)  1 (1,3,1)  2 (1,2,1)  3 (1,3,4)  4 (1,4,4)  5 (1,2,4)  6 (2,2,1)
//           7 (1,4,2)  8 (1,3,2)
//           FP32 only, where 40 registers hold a lane's two 20-vectors:
//           9 (1,5,1)  10 (1,6,1)  11 (1,5,4)
//           persistent (one wave, grid-stride over tiles): FP64 9 (1,3,4),
//           FP32 12 (1,4,4)
//   other:  0 (1,-,1)  1 (1,-,4)  2 (2,-,1)
// W = 2 variants take 64-slot tiles, the others 32-slot tiles.
int simt_variants(int R, bool fp32) { return R == 4 ? (fp32 ? 13 : 10) : 3; }
int simt_width(int R, int v) { return (R == 4 ? v == 6 : v == 2) ? 2 : 1; }

template <class T, int R, int MINB, int MINB2>
cudaError_t launch_prune_r(const PruneArgs& a, int ntiles, int variant, cudaStream_t st) {
    switch (variant) {
        case 1: return launch_prune_t<T, R, MINB, 1, 4>(a, ntiles, st);
        case 2: return launch_prune_t<T, R, MINB2, 2, 1>(a, ntiles, st);
        default: return launch_prune_t<T, R, MINB, 1, 1>(a, ntiles, st);
    }
}

template <class T>
cudaError_t launch_prune_r4(const PruneArgs& a, int ntiles, int variant, cudaStream_t st) {
    switch (variant) {
        case 1: return launch_prune_t<T, 4, 3, 1, 1>(a, ntiles, st);
        case 2: return launch_prune_t<T, 4, 2, 1, 1>(a, ntiles, st);
        case 3: return launch_prune_t<T, 4, 3, 1, 4>(a, ntiles, st);
        case 4: return launch_prune_t<T, 4, 4, 1, 4>(a, ntiles, st);
        case 5: return launch_prune_t<T, 4, 2, 1, 4>(a, ntiles, st);
        case 6: return launch_prune_t<T, 4, 2, 2, 1>(a, ntiles, st);
        case 7: return launch_prune_t<T, 4, 4, 1, 2>(a, ntiles, st);
        case 8: return launch_prune_t<T, 4, 3, 1, 2>(a, ntiles, st);
        case 9: return launch_prune_persistent_t<T, 4, 3, 1, 4>(a, ntiles, st);
        default: return launch_prune_t<T, 4, 4, 1, 1>(a, ntiles, st);
    }
}

template <class T>
cudaError_t launch_prune_typed(const PruneArgs& a, int ntiles, int variant, cudaStream_t st) {
    switch (a.d.R) {
        case 1: return launch_prune_r<T, 1, 4, 8>(a, ntiles, variant, st);
        case 2: return launch_prune_r<T, 2, 4, 4>(a, ntiles, variant, st);
        case 3: return launch_prune_r<T, 3, 4, 2>(a, ntiles, variant, st);
        case 4: return launch_prune_r4<T>(a, ntiles, variant, st);
        case 5: return launch_prune_r<T, 5, 2, 1>(a, ntiles, variant, st);
        case 6: return launch_prune_r<T, 6, 2, 1>(a, ntiles, variant, st);
        case 7: return launch_prune_r<T, 7, 2, 1>(a, ntiles, variant, st);
        case 8: return launch_prune_r<T, 8, 2, 1>(a, ntiles, variant, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_prune_fp32(const PruneArgs& a, int ntiles, int variant, cudaStream_t st) {
    if (a.d.R == 4) {
        switch (variant) {
            case 9: return launch_prune_t<float, 4, 5, 1, 1>(a, ntiles, st);
            case 10: return launch_prune_t<float, 4, 6, 1, 1>(a, ntiles, st);
            case 11: return launch_prune_t<float, 4, 5, 1, 4>(a, ntiles, st);
            case 12: return launch_prune_persistent_t<float, 4, 4, 1, 4>(a, ntiles, st);
            default: break;
        }
    }
    return launch_prune_typed<float>(a, ntiles, variant, st);
}

}  // namespace

// Numbered after the SIMT kernels: FP64 contexts have the FP64 tensor-path
// (DMMA) kernels, on 32-slot tiles; FP32 contexts the tcgen05 3xTF32 kernel,
// on 128-slot tiles.
int prune_variants(int R, bool fp32) {
    return simt_variants(R, fp32) + (fp32 ? prune_tc_variants(R) : prune_dmma_variants(R));
}

// FP64: one site per lane, four rows in flight (variant 3 at R = 4: 6.76 ms
// against 7.07 ms for one row in flight, 48 taxa x 2,000 sites x 256
// particles). FP32: the 128-register one-row variant.
int prune_default_variant(int R, bool fp32) {
    if (fp32) return 0;
    return R == 4 ? 3 : 1;
}

bool prune_variant_has_eval(int R, bool fp32, int variant) { return variant < simt_variants(R, fp32); }

int prune_variant_tile_sites(int R, bool fp32, int variant) {
    if (variant < simt_variants(R, fp32)) return 32 * simt_width(R, variant);
    return fp32 ? 128 : 32;
}

cudaError_t launch_prune(const PruneArgs& a, int ntiles, int variant, cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
    if (a.fp32) {
        const int ns = simt_variants(a.d.R, true);
        if (variant >= ns) return launch_prune_tc(a, ntiles, variant - ns, st);
        return launch_prune_fp32(a, ntiles, variant, st);
    }
    const int ns = simt_variants(a.d.R, false);
    if (variant >= ns) return launch_prune_dmma(a, ntiles, variant - ns, st);
    return launch_prune_typed<double>(a, ntiles, variant, st);
}

cudaError_t launch_reduce(const int32_t* tile_off, const double* partial, const PartHdr* hdr, int first,
                          int count, double* lnl, int* status, cudaStream_t st) {
    if (count <= 0) return cudaSuccess;
    reduce_kernel<<<(count + 127) / 128, 128, 0, st>>>(tile_off, partial, hdr, first, count, lnl, status);
    return cudaGetLastError();
}

cudaError_t launch_accept(double* lnl, double* lnl_old, const uint8_t* mask, int first, int count,
                          cudaStream_t st) {
    if (count <= 0) return cudaSuccess;
    accept_kernel<<<(count + 127) / 128, 128, 0, st>>>(lnl, lnl_old, mask, first, count);
    return cudaGetLastError();
}

}  // namespace smccat
