// FP64 pruning on the FP64 tensor path (mma.sync m8n8k4 f64).
//
// Same work decomposition, plan and memory layout as prune_kernel (one warp
// per rate and tile of <= 32 same-class sites, TMA-staged P, register-resident
// child), but each child mat-vec of a warp is one 32 x 20 x 20 matrix product
// on the tensor pipe:  out^T[site][i] = sum_j X^T[site][j] P^T[j][i]
//   M = sites (4 tiles of 8), N = states i (3 tiles of 8, padded 20 -> 24),
//   K = states j (5 steps of 4).
// Fragment layouts (lane = 4 g + t):
//   A (X^T):  lane holds X[4 ks + t][site 8 mt + g]
//   B (P^T):  lane holds P[8 nt + g][4 ks + t]          (0 for rows >= 20)
//   D:        lane holds out[8 nt + 2 t + h][site 8 mt + g], h = 0, 1
// so a site's states live in one quad of lanes: the per-site maximum is two
// quad shuffles, and the D -> A relayout of the register child is 40 quad
// shuffles.
#include <cuda_runtime.h>
#include <math.h>

#include "kernels.h"

namespace smccat {
namespace {

constexpr uint32_t kPBytesD = kPBlock * sizeof(double);

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void bar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __noinline__ bool bar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// B fragments of one P block (row-major, stride kPCols): pf[nt][ks].
__device__ __forceinline__ void load_pfrag(const double* P, int g, int t, double (&pf)[3][5]) {
#pragma unroll
    for (int nt = 0; nt < 3; ++nt)
#pragma unroll
        for (int ks = 0; ks < 5; ++ks) {
            const int i = 8 * nt + g;
            pf[nt][ks] = (i < kStates) ? P[i * kPCols + 4 * ks + t] : 0.0;
        }
}

// A fragments of the register child for site group mt, from its D layout.
__device__ __forceinline__ void relayout(const double (&y)[4][3][2], int mt, int lane, double (&xa)[5]) {
    const int t = lane & 3, base = lane & ~3;
#pragma unroll
    for (int ks = 0; ks < 5; ++ks) {
        const int src = base + (t >> 1) + 2 * (ks & 1);
        const double v0 = __shfl_sync(0xffffffffu, y[mt][ks >> 1][0], src);
        const double v1 = __shfl_sync(0xffffffffu, y[mt][ks >> 1][1], src);
        xa[ks] = (t & 1) ? v1 : v0;
    }
}

template <int R, int MINB>
__global__ void __launch_bounds__(32 * R, MINB) prune_dmma_kernel(const PruneArgs a) {
    const Dims d = a.d;
    const int tile_id = a.tile_begin + blockIdx.x;
    const Tile tl = a.tiles[tile_id];
    const int p = tl.p;
    const PartHdr* h = a.hdr + (p - a.first);
    if (!h->active) return;

    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[R][2];
    __shared__ double red[R][32];
    __shared__ int bad;

    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    double* buf = reinterpret_cast<double*>(smem_raw) + (size_t)r * 4 * kPBlock;

    const size_t j_stride = (size_t)R * d.Spad;
    const size_t ws_stride = (size_t)kStates * j_stride;
    const size_t node_stride = 2 * ws_stride;
    const size_t lws_stride = j_stride;
    double* CLp = static_cast<double*>(a.CL) + (size_t)p * d.NI * node_stride;
    double* LSCp = a.LSC + (size_t)p * d.NI * 2 * lws_stride;
    const int colbase = r * d.Spad + tl.slot0;  // column of local site 0
    const double* Pcls = static_cast<const double*>(a.Pm) +
                         ((size_t)p * d.Kmax + tl.k) * d.N * 2 * (size_t)R * kPBlock + (size_t)r * kPBlock;
    auto pblock = [&](int child, int pws) { return Pcls + ((size_t)child * 2 + pws) * (size_t)R * kPBlock; };

    // Sites of this lane: 8 mt + g, mt = 0..3.
    int site[4];
    bool sv[4];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
        const int ls = 8 * mt + g;
        sv[mt] = ls < tl.nslots;
        site[mt] = a.perm[(size_t)p * d.S + tl.slot0 + (sv[mt] ? ls : 0)];
    }

    if (threadIdx.x == 0) bad = 0;
    if (lane == 0) {
        bar_init(&bars[r][0]);
        bar_init(&bars[r][1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int cnt = (h->cls_only >= 0 && h->cls_only != tl.k) ? 0 : h->node_cnt;
    const int wfl = class_ws_flip(a.sws, p, d.Kmax, tl.k);
    const NodeJob* nodes = a.nodes + h->node_off;
    uint32_t pend = 0;  // lane 0: bit b set while a copy into buffer b is not yet waited on
    if (cnt > 0 && lane == 0) {
        NodeJob nj = nodes[0];
        nj.ws ^= wfl;
        bar_expect(&bars[r][0], 2 * kPBytesD);
        bulk_load(buf, pblock(nj.c1, (nj.ws >> 3) & 1), kPBytesD, &bars[r][0]);
        bulk_load(buf + kPBlock, pblock(nj.c2, (nj.ws >> 4) & 1), kPBytesD, &bars[r][0]);
        pend = 1u;
    }

    double y[4][3][2];  // D layout of the last computed node
    double lsc[4];      // its cumulative log scale per site group
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) lsc[mt] = 0.0;
    int prev = -1;
    bool ok = true;
    uint32_t phase = 0;
    for (int q = 0; q < cnt; ++q) {
        const int b = q & 1;
        NodeJob nj = nodes[q];
        nj.ws ^= wfl;
        if (ok && q + 1 < cnt && lane == 0) {  // no new copies once a wait has given up
            NodeJob nx = nodes[q + 1];
            nx.ws ^= wfl;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bar_expect(&bars[r][b ^ 1], 2 * kPBytesD);
            bulk_load(buf + (b ^ 1) * 2 * kPBlock, pblock(nx.c1, (nx.ws >> 3) & 1), kPBytesD,
                      &bars[r][b ^ 1]);
            bulk_load(buf + (b ^ 1) * 2 * kPBlock + kPBlock, pblock(nx.c2, (nx.ws >> 4) & 1), kPBytesD,
                      &bars[r][b ^ 1]);
            pend |= 1u << (b ^ 1);
        }
        if (ok) {
            if (bar_wait(&bars[r][b], (phase >> b) & 1, a.wait_limit)) {
                phase ^= 1u << b;
                pend &= ~(1u << b);
            } else {
                ok = false;
                atomicOr(a.status, 2);
            }
        }
        if (ok) {
            const bool c1prev = nj.c1 == prev, c2prev = nj.c2 == prev;
            const int oi = c1prev ? 1 : 0;
            const int fi = 1 - oi;
            const int o = oi ? nj.c2 : nj.c1, f = fi ? nj.c2 : nj.c1;
            const double* Pf = buf + (size_t)(b * 2 + fi) * kPBlock;
            const double* Po = buf + (size_t)(b * 2 + oi) * kPBlock;
            double lsc_f[4], lsc_o[4];
            // ---- first factor -> y (D layout)
            if (c1prev || c2prev || f >= d.T) {
                double pf[3][5];
                load_pfrag(Pf, g, t, pf);
                const int wsf = (nj.ws >> (1 + fi)) & 1;
                const double* fp = CLp + (size_t)(f - d.T) * node_stride + wsf * ws_stride + colbase;
#pragma unroll
                for (int mt = 0; mt < 4; ++mt) {
                    double xa[5];
                    if (c1prev || c2prev) {
                        relayout(y, mt, lane, xa);
                        lsc_f[mt] = lsc[mt];
                    } else {
#pragma unroll
                        for (int ks = 0; ks < 5; ++ks)
                            xa[ks] = sv[mt] ? fp[(size_t)(4 * ks + t) * j_stride + 8 * mt + g] : 0.0;
                        lsc_f[mt] = sv[mt] ? LSCp[(size_t)(f - d.T) * 2 * lws_stride + wsf * lws_stride +
                                                  colbase + 8 * mt + g] : 0.0;
                    }
#pragma unroll
                    for (int nt = 0; nt < 3; ++nt) {
                        double d0 = 0.0, d1 = 0.0;
#pragma unroll
                        for (int ks = 0; ks < 5; ++ks) dmma(d0, d1, xa[ks], pf[nt][ks]);
                        y[mt][nt][0] = d0;
                        y[mt][nt][1] = d1;
                    }
                }
            } else {  // tip first child: gather P[i][code]
#pragma unroll
                for (int mt = 0; mt < 4; ++mt) {
                    const int code = a.codes[(size_t)f * d.S + site[mt]];
                    const int cc = code < kStates ? code : kStates;
#pragma unroll
                    for (int nt = 0; nt < 3; ++nt)
#pragma unroll
                        for (int hh = 0; hh < 2; ++hh) {
                            const int i = 8 * nt + 2 * t + hh;
                            y[mt][nt][hh] = (i < kStates) ? Pf[i * kPCols + cc] : 0.0;
                        }
                    lsc_f[mt] = 0.0;
                }
            }
            // ---- other factor, folded into y
            if (o >= d.T) {
                double pf[3][5];
                load_pfrag(Po, g, t, pf);
                const int wso = (nj.ws >> (1 + oi)) & 1;
                const double* op = CLp + (size_t)(o - d.T) * node_stride + wso * ws_stride + colbase;
#pragma unroll
                for (int mt = 0; mt < 4; ++mt) {
                    double xa[5];
#pragma unroll
                    for (int ks = 0; ks < 5; ++ks)
                        xa[ks] = sv[mt] ? op[(size_t)(4 * ks + t) * j_stride + 8 * mt + g] : 0.0;
                    lsc_o[mt] = sv[mt] ? LSCp[(size_t)(o - d.T) * 2 * lws_stride + wso * lws_stride +
                                              colbase + 8 * mt + g] : 0.0;
#pragma unroll
                    for (int nt = 0; nt < 3; ++nt) {
                        double d0 = 0.0, d1 = 0.0;
#pragma unroll
                        for (int ks = 0; ks < 5; ++ks) dmma(d0, d1, xa[ks], pf[nt][ks]);
                        y[mt][nt][0] *= d0;
                        y[mt][nt][1] *= d1;
                    }
                }
            } else {
#pragma unroll
                for (int mt = 0; mt < 4; ++mt) {
                    const int code = a.codes[(size_t)o * d.S + site[mt]];
                    const int cc = code < kStates ? code : kStates;
#pragma unroll
                    for (int nt = 0; nt < 3; ++nt)
#pragma unroll
                        for (int hh = 0; hh < 2; ++hh) {
                            const int i = 8 * nt + 2 * t + hh;
                            y[mt][nt][hh] *= (i < kStates) ? Po[i * kPCols + cc] : 0.0;
                        }
                    lsc_o[mt] = 0.0;
                }
            }
            // ---- per-site power-of-two rescale, store
            const int wso = nj.ws & 1;
            double* out = CLp + (size_t)(nj.node - d.T) * node_stride + wso * ws_stride + colbase;
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) {
                double mx = 0.0;
#pragma unroll
                for (int nt = 0; nt < 3; ++nt) mx = fmax(mx, fmax(y[mt][nt][0], y[mt][nt][1]));
                mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
                mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
                double l;
                if (mx > 0.0) {
                    int e;
                    frexp(mx, &e);
                    const double sc = ldexp(1.0, -e);
#pragma unroll
                    for (int nt = 0; nt < 3; ++nt) { y[mt][nt][0] *= sc; y[mt][nt][1] *= sc; }
                    l = e * 0.69314718055994530942;
                } else {
                    l = (mx == 0.0) ? -INFINITY : NAN;
                }
                lsc[mt] = l + lsc_f[mt] + lsc_o[mt];
                if (sv[mt]) {
#pragma unroll
                    for (int nt = 0; nt < 3; ++nt)
#pragma unroll
                        for (int hh = 0; hh < 2; ++hh) {
                            const int i = 8 * nt + 2 * t + hh;
                            if (i < kStates) out[(size_t)i * j_stride + 8 * mt + g] = y[mt][nt][hh];
                        }
                    if (t == 0)
                        LSCp[(size_t)(nj.node - d.T) * 2 * lws_stride + wso * lws_stride + colbase + 8 * mt + g] =
                            lsc[mt];
                }
            }
        }
        prev = nj.node;
        __syncwarp();
    }
    if (!ok) bad = 1;
    // Lane 0 drains every copy it issued and never waited on (each on its
    // buffer's un-toggled parity) before the CTA's shared memory is released.
    if (lane == 0 && pend) {
        for (int bb = 0; bb < 2; ++bb)
            if (((pend >> bb) & 1u) && !bar_wait(&bars[r][bb], (phase >> bb) & 1, kDrainPolls)) bad = 1;
    }
    // ---- root reduction
    if (cnt == 0) {
        const double* rp = CLp + (size_t)(h->root - d.T) * node_stride + (h->root_ws ^ (wfl & 1)) * ws_stride + colbase;
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
#pragma unroll
            for (int nt = 0; nt < 3; ++nt)
#pragma unroll
                for (int hh = 0; hh < 2; ++hh) {
                    const int i = 8 * nt + 2 * t + hh;
                    y[mt][nt][hh] = (sv[mt] && i < kStates) ? rp[(size_t)i * j_stride + 8 * mt + g] : 0.0;
                }
            lsc[mt] = sv[mt] ? LSCp[(size_t)(h->root - d.T) * 2 * lws_stride + (h->root_ws ^ (wfl & 1)) * lws_stride +
                                    colbase + 8 * mt + g] : 0.0;
        }
    }
    const double* rec =
        a.spec + (((size_t)p * d.Kmax + tl.k) * 2 + (a.sws[(size_t)p * d.Kmax + tl.k] & kSwsSpec)) * kSpecStride;
    const double* pi = rec + kSpecPi;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
        double s = 0.0;
#pragma unroll
        for (int nt = 0; nt < 3; ++nt)
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                const int i = 8 * nt + 2 * t + hh;
                if (i < kStates) s = fma(pi[i], y[mt][nt][hh], s);
            }
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (t == 0 && sv[mt]) red[r][8 * mt + g] = log(s) + lsc[mt];
    }
    __syncthreads();
    if (r == 0) {
        double v = 0.0;
        if (lane < tl.nslots) {
            const int st = a.perm[(size_t)p * d.S + tl.slot0 + lane];
            double mx = red[0][lane];
#pragma unroll
            for (int rr = 1; rr < R; ++rr) mx = fmax(mx, red[rr][lane]);
            double lse = mx;
            if (mx > -INFINITY) {
                double se = 0.0;
#pragma unroll
                for (int rr = 0; rr < R; ++rr) se += exp(red[rr][lane] - mx);
                lse = mx + log(se);
            }
            const double pinv = h->pinv;
            if (pinv > 0.0 && a.isinv[st] != 0) {
                const double la = log1p(-pinv) + lse;
                const double lb = log(pinv * pi[a.invchar[st]]);
                const double m2 = fmax(la, lb);
                v = m2 + log(exp(la - m2) + exp(lb - m2));
            } else {
                v = lse + log1p(-pinv);
            }
            if (bad) v = NAN;
            a.site_lnl[(size_t)p * d.S + st] = v;
            if (a.wt) v *= a.wt[(size_t)p * d.S + tl.slot0 + lane];  // sites the slot stands for
        }
#pragma unroll
        for (int o2 = 16; o2 > 0; o2 >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o2);
        if (lane == 0) a.partial[tile_id] = v;
    }
}

template <int R, int MINB>
cudaError_t launch_dmma_t(const PruneArgs& a, int ntiles, cudaStream_t st) {
    const size_t smem = sizeof(double) * 4 * (size_t)kPBlock * R;
    cudaError_t e = cudaFuncSetAttribute(prune_dmma_kernel<R, MINB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    prune_dmma_kernel<R, MINB><<<ntiles, 32 * R, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

int prune_dmma_variants(int R) { return R == 4 ? 3 : 1; }

cudaError_t launch_prune_dmma(const PruneArgs& a, int ntiles, int variant, cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
    switch (a.d.R) {
        case 1: return launch_dmma_t<1, 4>(a, ntiles, st);
        case 2: return launch_dmma_t<2, 4>(a, ntiles, st);
        case 3: return launch_dmma_t<3, 4>(a, ntiles, st);
        case 4:
            if (variant == 1) return launch_dmma_t<4, 3>(a, ntiles, st);
            if (variant == 2) return launch_dmma_t<4, 2>(a, ntiles, st);
            return launch_dmma_t<4, 4>(a, ntiles, st);
        case 5: return launch_dmma_t<5, 2>(a, ntiles, st);
        case 6: return launch_dmma_t<6, 2>(a, ntiles, st);
        case 7: return launch_dmma_t<7, 2>(a, ntiles, st);
        case 8: return launch_dmma_t<8, 2>(a, ntiles, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace smccat
