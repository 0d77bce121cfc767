// FP32 pruning on the 5th-generation tensor cores: tcgen05.mma kind::tf32 in
// a split 3xTF32 form, accumulators and the site operand in tensor memory.
//
// One CTA of 128 threads per tile of <= 128 same-class slots; thread t owns
// slot t and TMEM lane t. The rate categories run one after another, each
// walking the tile's dirty nodes in post-order. For an internal child c of a
// node, the off-diagonal part of P(c, r) X_c over the tile's sites is one
// matrix product
//   D[site][i] = sum_{j != i} X[site][j] P[i][j]    M = 128 sites, N = 24, K = 24
// (states padded from 20); the diagonal term is fused on afterwards in FP32,
// as in the SIMT kernel (for the near-identity P of short branches, small
// off-diagonal terms summed after the diagonal one would be rounded away with
// a bias of one sign). To keep FP32 accuracy the product is computed as
//   Xhi.Phi + Xhi.Plo + Xlo.Phi,  hi = rna_tf32(x), lo = x - hi,
// with FP32 accumulation: every product is exact and lo keeps 11 more bits.
// (Letting the tensor core read the raw FP32 value as hi truncates both parts
// toward zero; that one-signed error is far larger.)
//   A (X hi / lo):  TMEM columns [0, 24) / [24, 48), written by each thread
//                   for its own lane with tcgen05.st;
//   B (P hi / lo):  shared memory, K-major canonical layout without swizzle
//                   (8-row x 16-byte core matrices), built from the P block
//                   that a bulk copy (TMA) staged;
//   D:              TMEM columns [48, 72), read back with tcgen05.ld.
// Tip children need no product: their column of P is read from shared memory.
// Partials are stored in FP32 in the engine's state-major layout, log-scalers
// and the root reduction are FP64, exactly as in the SIMT kernel.
#include <cuda_runtime.h>
#include <math.h>

#include "kernels.h"

namespace smccat {
namespace {

constexpr int kTcSites = 128;
constexpr int kTcPad = 24;                         // K and N after padding
constexpr uint32_t kTcCols = 128;                  // TMEM columns per CTA
constexpr uint32_t kColHi = 0, kColLo = 24, kColD = 48;
constexpr uint32_t kCoreLbo = 128;                 // next core matrix along K
constexpr uint32_t kCoreSbo = (kTcPad / 4) * 128;  // next 8-row group
constexpr uint32_t kBBytes = kTcPad * kTcPad * 4;  // one B operand tile
constexpr uint32_t kPBytesF = kPBlock * sizeof(float);
// idesc: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2), K-major
// A and B, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcPad >> 3) << 17) |
                            ((uint32_t)(kTcSites >> 4) << 24);

__device__ __forceinline__ uint32_t sa(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Byte offset of element (row, k) of a K-major canonical tile without swizzle.
__device__ __forceinline__ uint32_t kmaj(int row, int k) {
    return (row >> 3) * kCoreSbo + (k >> 2) * kCoreLbo + (row & 7) * 16 + (k & 3) * 4;
}

// Shared-memory matrix descriptor (sm100 version 1, no swizzle).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(kCoreLbo >> 4) << 16) |
           ((uint64_t)(kCoreSbo >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sa(bar)) : "memory");
}

__device__ __forceinline__ void tc_bar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tc_bulk(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            sa(dst)),
        "l"(src), "r"(bytes), "r"(sa(bar))
        : "memory");
}

__device__ __noinline__ bool tc_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(sa(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void st8(uint32_t taddr, const uint32_t* v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}

__device__ __forceinline__ void ld8(uint32_t taddr, uint32_t* v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                   "=r"(v[7])
                 : "r"(taddr)
                 : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t d, uint32_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %4, p;\n\t}" ::"r"(d),
        "r"(a), "l"(b), "r"(acc), "r"(kIdesc)
        : "memory");
}

__device__ __forceinline__ double tc_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kTcSites, 4) prune_tc_kernel(const PruneArgs a) {
    const Dims d = a.d;
    const int R = d.R;
    const int tile_id = a.tile_begin + blockIdx.x;
    const Tile tl = a.tiles[tile_id];
    const int p = tl.p;
    const PartHdr* h = a.hdr + (p - a.first);
    if (!h->active) return;  // uniform across the CTA

    // Dynamic shared memory: P staging [2 buffers][2 children][kPBlock] floats,
    // B operands [2 children][hi, lo][kBBytes], root values [R][128] doubles.
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float* pbuf = reinterpret_cast<float*>(smem_raw);
    unsigned char* bop = smem_raw + 4 * kPBytesF;
    double* red = reinterpret_cast<double*>(bop + 4 * kBBytes);
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int bad;
    __shared__ double wsum[kTcSites / 32];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool valid = tid < tl.nslots;
    const int slot = tl.slot0 + (valid ? tid : 0);
    const int site = a.perm[(size_t)p * d.S + slot];

    const size_t j_stride = (size_t)R * d.Spad;
    const size_t ws_stride = (size_t)kStates * j_stride;
    const size_t node_stride = 2 * ws_stride;
    const size_t lws_stride = j_stride;
    float* CLp = static_cast<float*>(a.CL) + (size_t)p * d.NI * node_stride;
    double* LSCp = a.LSC + (size_t)p * d.NI * 2 * lws_stride;
    const float* Pcls = static_cast<const float*>(a.Pm) + ((size_t)p * d.Kmax + tl.k) * d.N * 2 * (size_t)R * kPBlock;
    auto pblock = [&](int child, int pws, int r) {
        return Pcls + ((size_t)child * 2 + pws) * (size_t)R * kPBlock + (size_t)r * kPBlock;
    };

    if (tid == 0) {
        bad = 0;
        tc_bar_init(&bars[0]);
        tc_bar_init(&bars[1]);
        tc_bar_init(&mma_bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa(&tmem_slot)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tm = tmem_slot;
    const uint32_t tlane = tm + ((uint32_t)(warp * 32) << 16);  // this warp's lane quarter

    const int cnt = (h->cls_only >= 0 && h->cls_only != tl.k) ? 0 : h->node_cnt;
    const int wfl = class_ws_flip(a.sws, p, d.Kmax, tl.k);
    const NodeJob* nodes = a.nodes + h->node_off;
    const int nsteps = cnt * R;  // (rate, node) pairs, rate-major
    auto issue = [&](int f) {    // thread 0: stage the P blocks of step f
        const int r = f / cnt, q = f - r * cnt;
        NodeJob nj = nodes[q];
        nj.ws ^= wfl;
        float* dst = pbuf + (size_t)(f & 1) * 2 * kPBlock;
        tc_bar_expect(&bars[f & 1], 2 * kPBytesF);
        tc_bulk(dst, pblock(nj.c1, (nj.ws >> 3) & 1, r), kPBytesF, &bars[f & 1]);
        tc_bulk(dst + kPBlock, pblock(nj.c2, (nj.ws >> 4) & 1, r), kPBytesF, &bars[f & 1]);
    };
    // Thread 0 issues every copy and product. It tracks which are still in
    // flight (copy buffers in `pend`, the last product commit in `mma_pend`),
    // stops issuing once a wait has given up, and drains the rest before the
    // CTA releases its shared and tensor memory.
    uint32_t pend = 0;
    bool mma_pend = false;
    if (tid == 0 && nsteps > 0) {
        issue(0);
        pend = 1u;
    }

    bool ok = true;
    uint32_t tphase = 0, mphase = 0;
    float y[kStates];
    double lsc = 0.0;
    int prev = -1;
    const double* rec = a.spec + (((size_t)p * d.Kmax + tl.k) * 2 + (a.sws[(size_t)p * d.Kmax + tl.k] & kSwsSpec)) * kSpecStride;
    const double* pi = rec + kSpecPi;

    for (int r = 0; r < R; ++r) {
        prev = -1;
        for (int q = 0; q < cnt; ++q) {
            const int f = r * cnt + q;
            const int b = f & 1;
            NodeJob nj = nodes[q];
            nj.ws ^= wfl;
            if (tid == 0 && ok && f + 1 < nsteps) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(f + 1);  // buffer b ^ 1 was last read at step f - 1 (synchronised since)
                pend |= 1u << (b ^ 1);
            }
            // The child computed just before (if any) is in registers; the
            // other is a tip (column of P) or a stored partial.
            const bool c1prev = nj.c1 == prev, c2prev = nj.c2 == prev;
            const int oi = c1prev ? 1 : 0;
            const int fi = 1 - oi;
            const bool has_prev = c1prev || c2prev;
            if (ok) {
                if (tc_wait(&bars[b], (tphase >> b) & 1, a.wait_limit)) {
                    tphase ^= 1u << b;
                    pend &= ~(1u << b);
                } else {
                    ok = false;
                    atomicOr(a.status, 2);
                }
            }
            const float* Pst = pbuf + (size_t)b * 2 * kPBlock;
            // B operands (P hi / lo) of the internal children.
            for (int ci = 0; ci < 2; ++ci) {
                const int c = ci ? nj.c2 : nj.c1;
                if (c < d.T) continue;
                const float* P = Pst + ci * kPBlock;
                unsigned char* bh = bop + (2 * ci) * kBBytes;
                unsigned char* bl = bop + (2 * ci + 1) * kBBytes;
                for (int e = tid; e < kTcPad * kTcPad; e += kTcSites) {
                    const int n = e / kTcPad, k = e - n * kTcPad;
                    const float v = (n < kStates && k < kStates && n != k) ? P[n * kPCols + k] : 0.f;
                    const float hi = tf32_rna(v);
                    *reinterpret_cast<float*>(bh + kmaj(n, k)) = hi;
                    *reinterpret_cast<float*>(bl + kmaj(n, k)) = v - hi;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");

            float acc[kStates];
            double lsc_f = 0.0, lsc_o = 0.0;
            for (int pass = 0; pass < 2; ++pass) {
                const int ci = pass == 0 ? fi : oi;  // child slot (0: c1, 1: c2)
                const int c = ci ? nj.c2 : nj.c1;
                float v[kStates];
                if (c < d.T) {
                    const int code = a.codes[(size_t)c * d.S + site];
                    const int cc = code < kStates ? code : kStates;
                    const float* P = Pst + ci * kPBlock;
#pragma unroll
                    for (int i = 0; i < kStates; ++i) v[i] = P[i * kPCols + cc];
                } else {
                    float x[kStates];
                    double l;
                    if (pass == 0 && has_prev) {
#pragma unroll
                        for (int j = 0; j < kStates; ++j) x[j] = y[j];
                        l = lsc;
                    } else {
                        const int wsc = (nj.ws >> (1 + ci)) & 1;
                        const float* xp = CLp + (size_t)(c - d.T) * node_stride + wsc * ws_stride;
                        const size_t col = (size_t)r * d.Spad + slot;
#pragma unroll
                        for (int j = 0; j < kStates; ++j) x[j] = xp[col + j * j_stride];
                        l = LSCp[(size_t)(c - d.T) * 2 * lws_stride + wsc * lws_stride + col];
                    }
                    if (pass == 0) lsc_f = l;
                    else lsc_o = l;
                    uint32_t hv[kTcPad], lv[kTcPad];
#pragma unroll
                    for (int j = 0; j < kTcPad; ++j) {
                        const float xv = j < kStates ? x[j] : 0.f;
                        const float hi = tf32_rna(xv);
                        hv[j] = __float_as_uint(hi);
                        lv[j] = __float_as_uint(xv - hi);
                    }
#pragma unroll
                    for (int c8 = 0; c8 < 3; ++c8) {
                        st8(tlane + kColHi + 8 * c8, hv + 8 * c8);
                        st8(tlane + kColLo + 8 * c8, lv + 8 * c8);
                    }
                    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    ok = __syncthreads_and(ok);  // one decision for the whole CTA
                    if (tid == 0 && ok) {
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint32_t bh = sa(bop + (2 * ci) * kBBytes), bl = sa(bop + (2 * ci + 1) * kBBytes);
#pragma unroll
                        for (int ks = 0; ks < 3; ++ks)  // Xhi . Phi
                            mma_tf32(tm + kColD, tm + kColHi + 8 * ks, sdesc(bh + ks * 2 * kCoreLbo), ks > 0);
#pragma unroll
                        for (int ks = 0; ks < 3; ++ks)  // Xhi . Plo
                            mma_tf32(tm + kColD, tm + kColHi + 8 * ks, sdesc(bl + ks * 2 * kCoreLbo), 1);
#pragma unroll
                        for (int ks = 0; ks < 3; ++ks)  // Xlo . Phi
                            mma_tf32(tm + kColD, tm + kColLo + 8 * ks, sdesc(bh + ks * 2 * kCoreLbo), 1);
                        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                         sa(&mma_bar))
                                     : "memory");
                        mma_pend = true;
                    }
                    if (ok) {
                        if (tc_wait(&mma_bar, mphase, a.wait_limit)) {
                            mphase ^= 1u;
                            mma_pend = false;
                        } else {
                            ok = false;
                            atomicOr(a.status, 2);
                        }
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    uint32_t dv[kTcPad];
#pragma unroll
                    for (int c8 = 0; c8 < 3; ++c8) ld8(tlane + kColD + 8 * c8, dv + 8 * c8);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    // The diagonal term last, fused onto the off-diagonal sum.
                    const float* P = Pst + ci * kPBlock;
#pragma unroll
                    for (int i = 0; i < kStates; ++i) v[i] = fmaf(P[i * kPCols + i], x[i], __uint_as_float(dv[i]));
                }
#pragma unroll
                for (int i = 0; i < kStates; ++i) acc[i] = pass == 0 ? v[i] : acc[i] * v[i];
            }
            // Rescale by an exact power of two; cumulative log-scaler.
            float mx = 0.f;
#pragma unroll
            for (int i = 0; i < kStates; ++i) mx = fmaxf(mx, acc[i]);
            double l;
            if (mx > 0.f) {
                int e;
                frexpf(mx, &e);
                const float sc = ldexpf(1.0f, -e);
#pragma unroll
                for (int i = 0; i < kStates; ++i) acc[i] *= sc;
                l = e * 0.69314718055994530942;
            } else {
                l = (mx == 0.f) ? -INFINITY : NAN;
            }
            lsc = l + lsc_f + lsc_o;
#pragma unroll
            for (int j = 0; j < kStates; ++j) y[j] = acc[j];
            if (valid) {
                const int wso = nj.ws & 1;
                const size_t col = (size_t)r * d.Spad + slot;
                float* out = CLp + (size_t)(nj.node - d.T) * node_stride + wso * ws_stride;
#pragma unroll
                for (int j = 0; j < kStates; ++j) out[col + j * j_stride] = acc[j];
                LSCp[(size_t)(nj.node - d.T) * 2 * lws_stride + wso * lws_stride + col] = lsc;
            }
            prev = nj.node;
            __syncthreads();  // P staging and B operands of this step are free
        }
        // Root value of rate r for this thread's site.
        if (cnt == 0) {
            const size_t col = (size_t)r * d.Spad + slot;
            const int rws = h->root_ws ^ (wfl & 1);
            const float* xp = CLp + (size_t)(h->root - d.T) * node_stride + rws * ws_stride;
#pragma unroll
            for (int j = 0; j < kStates; ++j) y[j] = xp[col + j * j_stride];
            lsc = LSCp[(size_t)(h->root - d.T) * 2 * lws_stride + rws * lws_stride + col];
        }
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < kStates; ++i) s = fma(pi[i], (double)y[i], s);
        red[r * kTcSites + tid] = log(s) + lsc;
    }
    if (!ok) bad = 1;
    // Let copies and products still in flight land (each on its un-toggled
    // parity) before the CTA's shared and tensor memory are released.
    if (tid == 0) {
        for (int x = 0; x < 2; ++x)
            if (((pend >> x) & 1u) && !tc_wait(&bars[x], (tphase >> x) & 1, kDrainPolls)) bad = 1;
        if (mma_pend && !tc_wait(&mma_bar, mphase, kDrainPolls)) bad = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(kTcCols) : "memory");

    double v = 0.0;
    if (valid) {
        double mx = red[tid];
        for (int r = 1; r < R; ++r) mx = fmax(mx, red[r * kTcSites + tid]);
        double lse = mx;
        if (mx > -INFINITY) {
            double se = 0.0;
            for (int r = 0; r < R; ++r) se += exp(red[r * kTcSites + tid] - mx);
            lse = mx + log(se);
        }
        // +I mixing, Particle.cpp:667-670, evaluated in log space.
        const double pinv = h->pinv;
        double u;
        if (pinv > 0.0 && a.isinv[site] != 0) {
            const double la = log1p(-pinv) + lse;
            const double lb = log(pinv * pi[a.invchar[site]]);
            const double m2 = fmax(la, lb);
            u = m2 + log(exp(la - m2) + exp(lb - m2));
        } else {
            u = lse + log1p(-pinv);
        }
        if (bad) u = NAN;
        a.site_lnl[(size_t)p * d.S + site] = u;
        v = a.wt ? u * a.wt[(size_t)p * d.S + tl.slot0 + tid] : u;
    }
    v = tc_warp_sum(v);
    if (lane == 0) wsum[warp] = v;
    __syncthreads();
    if (tid == 0) a.partial[tile_id] = wsum[0] + wsum[1] + wsum[2] + wsum[3];
}

}  // namespace

int prune_tc_variants(int R) { return R <= kMaxRates ? 1 : 0; }

cudaError_t launch_prune_tc(const PruneArgs& a, int ntiles, int variant, cudaStream_t st) {
    (void)variant;
    if (!a.fp32) return cudaErrorInvalidValue;
    const size_t smem = 4 * (size_t)kPBytesF + 4 * (size_t)kBBytes + (size_t)a.d.R * kTcSites * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(prune_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    prune_tc_kernel<<<ntiles, kTcSites, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace smccat
