// CAT class reassignment (Neal's Algorithm 8, m = 5 auxiliary classes) on the
// device: Particle::gibbsPartitionMove (Particle.cpp:785-995), corrected form.
//
// Each of the floor(S/2) site iterations of a particle draws a site, takes it
// out of its class (dropping the class if it empties), draws m fresh classes
// from the prior (19 N(0,1) logits + 0, TransitionProbabilityClass.cpp:26-35),
// weights every live class and every auxiliary by temperature * log L +
// log n_k (or log(alpha / m)) and draws the new class. The drawn sites and the
// auxiliary classes do not depend on the chain's state, so a pass runs in two
// kernels: gibbs_aux_kernel diagonalises every iteration's auxiliary classes
// and prunes their sites, all iterations of all particles at once (one warp per
// (particle, iteration, auxiliary), lanes = states, single-site pruning in the
// eigenbasis P(t)x = L (exp(lambda t) o (Rm x))); then gibbs_kernel walks each
// particle's iterations in order (one CTA per particle) with the site values of
// the entry classes from a table the pruning kernels fill, those of classes
// opened during the pass pruned per site, and those of the auxiliaries from
// the first kernel. Random numbers come from a Philox stream per (particle,
// iteration).
//
// Two reference quirks are not reproduced: its tip read ignores the rate
// stride (Particle.cpp:895) and its rescalers are written and read at
// different strides (Particle.cpp:880 vs :921), so its weights mix in stale
// buffer contents.
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <math.h>

#include "gibbs.h"
#include "learned.h"
#include <cuda_bf16.h>
#include "spectral.cuh"

namespace smccat {
namespace {

constexpr int kGibbsWarps = 16;
constexpr int kAux = 5;
constexpr int kAuxWarps = 4;  // warps per CTA of the auxiliary-class kernel
constexpr int kAuxCtasPerSm = 3;

// Random numbers of site iteration `it` of particle p come from the Philox
// stream (seed, subsequence (p << 24) | it), at fixed offsets (32-bit draws):
// the site at 0, auxiliary class j's 19 logits at 64 (j + 1), the class draw
// at 64 (kAux + 1). The auxiliary-class kernel and the sequential pass read
// the same draws, and no draw depends on the chain's state.
constexpr unsigned long long kOffAux = 64, kOffChoice = 64ull * (kAux + 1);
// The learned move's update `it` uses the same site draw (offset 0), its
// proposal draw at kOffProposal and its acceptance draw at kOffAccept.
constexpr unsigned long long kOffProposal = 64, kOffAccept = 128;

__device__ double draw_at(unsigned long long seed, int p, int it, unsigned long long off) {
    curandStatePhilox4_32_10_t r;
    curand_init(seed, ((unsigned long long)p << 24) | (unsigned long long)it, off, &r);
    return curand_uniform_double(&r);
}

__device__ __forceinline__ unsigned long long iter_stream(int p, int it) {
    return ((unsigned long long)p << 24) | (unsigned long long)it;
}

__device__ int draw_site(unsigned long long seed, int p, int it, int S) {
    curandStatePhilox4_32_10_t r;
    curand_init(seed, iter_stream(p, it), 0ull, &r);
    const double u = curand_uniform_double(&r);  // (0, 1]
    const int s = (int)((1.0 - u) * S);
    return s < S ? s : S - 1;
}

// 19 N(0,1) logits and a 0 (TransitionProbabilityClass.cpp:26-35).
__device__ void draw_aux_logits(unsigned long long seed, int p, int it, int j, double* out) {
    curandStatePhilox4_32_10_t r;
    curand_init(seed, iter_stream(p, it), kOffAux + 64ull * j, &r);
    for (int m = 0; m < kStates - 1; ++m) out[m] = curand_normal_double(&r);
    out[kStates - 1] = 0.0;
}

__device__ double draw_choice(unsigned long long seed, int p, int it) {
    curandStatePhilox4_32_10_t r;
    curand_init(seed, iter_stream(p, it), kOffChoice, &r);
    return curand_uniform_double(&r);
}

__device__ __forceinline__ double warp_max20(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_maxf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Inclusive prefix sum over the warp's lanes.
__device__ __forceinline__ double warp_incl_scan(double x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Rates per warp in the Gibbs weights (all of a class's rates together) and in
// the learned move.
constexpr int kRateBlock = 4;

// Log-likelihoods of one site under one class for rates [r0, r0 + RB) (those
// below R), one warp: lanes are states and the rate chains interleave.
// Single-site pruning in the eigenbasis, P(t r) x = L (exp(lambda t r) o (Rm x)),
// with exp(lambda_m t r) evaluated where it is used. The vectors every lane
// needs whole (x before Rm, z before L) pass through the warp's shared
// exchange row `xch` [RB][kStates] and are read back as broadcast pairs, not
// shuffled lane by lane. The node computed last stays in registers (in
// post-order it is a child of the next node); other internal children come
// back from the warp's stash [nslots][RB][32]. Tip codes of the site come from
// `scode` (shared). out[b] = log L of rate r0 + b.
template <int RB>
__device__ void site_class_lnl(const GibbsArgs& a, const GibbsPart& gp, int i, int r0,
                               const double* rec, double* stash, const uint8_t* scode,
                               double* xch, double* out) {
    using D2 = double2;
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31;
    const int li = lane < kStates ? lane : 0;
    const bool st_lane = lane < kStates;
    double Lrow[kStates], Rrow[kStates];
#pragma unroll
    for (int m = 0; m < kStates; ++m) {
        Lrow[m] = rec[kSpecL + li * kStates + m];   // L[lane][m]
        Rrow[m] = rec[kSpecRm + li * kStates + m];  // Rm[lane][m]
    }
    const double lam = rec[kSpecLam + li];
    double rs = 0.0;
#pragma unroll
    for (int j = 0; j < kStates; ++j) rs += Rrow[j];
    bool on[RB];
    double v[RB], lsc[RB], rate[RB];
#pragma unroll
    for (int b = 0; b < RB; ++b) {
        on[b] = r0 + b < d.R;
        rate[b] = on[b] ? gp.rates[r0 + b] : 0.0;
        v[b] = 1.0;
        lsc[b] = 0.0;
    }
    const GibbsNode* tree = a.nodes + (size_t)i * d.NI;
    const double* br = a.branch + (size_t)i * d.N;
    int prev = -1;
    for (int q = 0; q < d.NI; ++q) {
        const GibbsNode nd = tree[q];
        double vn[RB];
#pragma unroll
        for (int b = 0; b < RB; ++b) vn[b] = 1.0;
#pragma unroll 1
        for (int ci = 0; ci < 2; ++ci) {
            const int c = nd.c[ci];
            const double lt = lam * br[c];
            double e[RB], z[RB];
#pragma unroll
            for (int b = 0; b < RB; ++b) e[b] = on[b] ? exp(lt * rate[b]) : 0.0;
            if (c < d.T) {
                const int code = scode[c];
                double rc = rs;
                if (code < kStates) {
#pragma unroll
                    for (int j = 0; j < kStates; ++j) rc = (j == code) ? Rrow[j] : rc;
                }
#pragma unroll
                for (int b = 0; b < RB; ++b) z[b] = e[b] * rc;
            } else {
                const double* sx = stash + (size_t)nd.sc[ci] * RB * 32;
#pragma unroll
                for (int b = 0; b < RB; ++b) {
                    const double xv = (c == prev) ? v[b] : sx[b * 32 + lane];
                    if (st_lane) xch[b * kStates + lane] = xv;
                }
                __syncwarp();
                double acc[RB];
#pragma unroll
                for (int b = 0; b < RB; ++b) acc[b] = 0.0;
#pragma unroll
                for (int j = 0; j < kStates / 2; ++j) {
#pragma unroll
                    for (int b = 0; b < RB; ++b) {
                        const D2 x2 = reinterpret_cast<const D2*>(xch + b * kStates)[j];
                        acc[b] = fma(Rrow[2 * j], x2.x, acc[b]);
                        acc[b] = fma(Rrow[2 * j + 1], x2.y, acc[b]);
                    }
                }
                __syncwarp();
#pragma unroll
                for (int b = 0; b < RB; ++b) z[b] = e[b] * acc[b];
            }
#pragma unroll
            for (int b = 0; b < RB; ++b)
                if (st_lane) xch[b * kStates + lane] = z[b];
            __syncwarp();
            double y[RB];
#pragma unroll
            for (int b = 0; b < RB; ++b) y[b] = 0.0;
#pragma unroll
            for (int m = 0; m < kStates / 2; ++m) {
#pragma unroll
                for (int b = 0; b < RB; ++b) {
                    const D2 z2 = reinterpret_cast<const D2*>(xch + b * kStates)[m];
                    y[b] = fma(Lrow[2 * m], z2.x, y[b]);
                    y[b] = fma(Lrow[2 * m + 1], z2.y, y[b]);
                }
            }
            __syncwarp();
#pragma unroll
            for (int b = 0; b < RB; ++b) vn[b] *= y[b];
        }
        double* so = stash + (size_t)nd.so * RB * 32;
#pragma unroll
        for (int b = 0; b < RB; ++b) {
            double x = st_lane ? vn[b] : 0.0;
            const double mx = warp_max20(x);
            if (mx > 0.0) {
                int e;
                frexp(mx, &e);
                x *= ldexp(1.0, -e);
                lsc[b] += e * 0.69314718055994530942;
            } else {
                lsc[b] = -INFINITY;
            }
            v[b] = x;
            so[b * 32 + lane] = x;
        }
        prev = nd.n;
        __syncwarp();
    }
    const double pi = st_lane ? rec[kSpecPi + lane] : 0.0;
#pragma unroll
    for (int b = 0; b < RB; ++b) {
        const double sv = wsum(pi * v[b]);
        if (lane == 0 && on[b]) out[b] = log(sv) + lsc[b];
    }
}

// Site log-likelihood (+I mixed) from the per-rate values l[r]
// (Particle.cpp:931-950, corrected form).
__device__ double site_value(const GibbsArgs& a, const GibbsPart& gp, int s, const double* l,
                             const double* pi) {
    double mx = -INFINITY;
    for (int r = 0; r < a.d.R; ++r) mx = fmax(mx, l[r]);
    double lse = mx;
    if (mx > -INFINITY) {
        double se = 0.0;
        for (int r = 0; r < a.d.R; ++r) se += exp(l[r] - mx);
        lse = mx + log(se);
    }
    if (gp.pinv > 0.0 && a.isinv[s] != 0) {
        const double la = log1p(-gp.pinv) + lse;
        const double lb = log(gp.pinv * pi[a.invchar[s]]);
        const double m2 = fmax(la, lb);
        return m2 + log(exp(la - m2) + exp(lb - m2));
    }
    return lse + log1p(-gp.pinv);
}

// Every iteration's drawn site and its log-likelihood under each of the m
// auxiliary classes (Particle.cpp:823-833 and :857-930 for the auxiliaries),
// for all particles and iterations at once: one warp per (particle,
// iteration, auxiliary class) draws the site and the class's logits,
// diagonalises the class and prunes the site. In weights mode the site is the
// fixed one and the logits come from aux_in.
__global__ void __launch_bounds__(32 * kAuxWarps, kAuxCtasPerSm) gibbs_aux_kernel(GibbsArgs a, int n_iter) {
    const Dims& d = a.d;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ SpecWork work[kAuxWarps];
    __shared__ __align__(16) double xch[kAuxWarps][kRateBlock * kStates];
    __shared__ double lg[kAuxWarps][kStates];
    __shared__ double lr[kAuxWarps][kMaxRates];
    __shared__ int ssite[kAuxWarps];
    extern __shared__ uint8_t scodes[];  // [kAuxWarps][T]
    uint8_t* scode = scodes + (size_t)warp * d.T;
    const size_t gw = (size_t)blockIdx.x * kAuxWarps + warp;
    double* rec = a.aux_rec + gw * kSpecStride;
    double* stash = a.aux_stash + gw * a.nslots * kRateBlock * 32;
    const size_t tasks = (size_t)a.count * n_iter * kAux;
    for (size_t t = gw; t < tasks; t += (size_t)gridDim.x * kAuxWarps) {
        const int j = (int)(t % kAux);
        const size_t ii = t / kAux;  // particle * n_iter + iteration
        const int it = (int)(ii % n_iter), i = (int)(ii / n_iter);
        const GibbsPart& gp = a.parts[i];
        if (lane == 0) {
            int s;
            if (gp.fixed_site >= 0) {
                s = gp.fixed_site;
                for (int m = 0; m < kStates; ++m) lg[warp][m] = a.aux_in[((size_t)i * kAux + j) * kStates + m];
            } else {
                s = draw_site(a.seed, gp.p, it, d.S);
                draw_aux_logits(a.seed, gp.p, it, j, lg[warp]);
            }
            ssite[warp] = s;
            if (j == 0) a.aux_site[ii] = s;
        }
        __syncwarp();
        const int s = ssite[warp];
        for (int c = lane; c < d.T; c += 32) scode[c] = a.codes[(size_t)c * d.S + s];
        spectral_decompose_warp_ws(a.base + (size_t)i * kBase, lg[warp], rec, work[warp]);
        __syncwarp();
        for (int r0 = 0; r0 < d.R; r0 += kRateBlock)
            site_class_lnl<kRateBlock>(a, gp, i, r0, rec, stash, scode, xch[warp], lr[warp] + r0);
        __syncwarp();
        if (lane == 0) a.aux_ls[t] = site_value(a, gp, s, lr[warp], rec + kSpecPi);
        __syncwarp();
    }
}

// The sites a pass draws, without the rest of the auxiliary work (the learned
// move, whose site draws come from the same streams).
__global__ void draw_sites_kernel(GibbsArgs a, int n_iter) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)a.count * n_iter) return;
    const int it = (int)(t % n_iter), i = (int)(t / n_iter);
    a.aux_site[t] = draw_site(a.seed, a.parts[i].p, it, a.d.S);
}

// Particle i's distinct drawn sites in increasing order into row q = qrow[i]
// of the evaluation site lists (the rest of the row zero) and their count
// into nv[q]; `flags` is [count][S] scratch. One CTA per particle.
constexpr int kVisitThreads = 512;
__global__ void __launch_bounds__(kVisitThreads) visited_sites_kernel(const int32_t* sites, int n_iter,
                                                                      const int32_t* qrow, int S,
                                                                      uint8_t* flags, int32_t* list,
                                                                      int32_t* nv) {
    const int i = blockIdx.x, tid = threadIdx.x;
    uint8_t* f = flags + (size_t)i * S;
    for (int x = tid; x < S; x += kVisitThreads) f[x] = 0;
    __syncthreads();
    for (int it = tid; it < n_iter; it += kVisitThreads) f[sites[(size_t)i * n_iter + it]] = 1;
    __syncthreads();
    // Contiguous chunks per thread, an exclusive scan of the chunk counts.
    const int chunk = (S + kVisitThreads - 1) / kVisitThreads;
    const int x0 = min(S, tid * chunk), x1 = min(S, x0 + chunk);
    int c = 0;
    for (int x = x0; x < x1; ++x) c += f[x];
    __shared__ int part[kVisitThreads];
    part[tid] = c;
    __syncthreads();
    for (int o = 1; o < kVisitThreads; o <<= 1) {
        const int v = tid >= o ? part[tid - o] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int pos = part[tid] - c;
    int32_t* row = list + (size_t)qrow[i] * S;
    for (int x = x0; x < x1; ++x)
        if (f[x]) row[pos++] = x;
    const int total = part[kVisitThreads - 1];
    for (int x = total + tid; x < S; x += kVisitThreads) row[x] = 0;
    if (tid == 0) nv[qrow[i]] = total;
}

// The sequential part of a Gibbs pass, one CTA per particle over its
// iterations in order. Each iteration takes the drawn site out of its class
// (dropping the class if it empties), weights every live class by
// temperature * log L + log n_k and each auxiliary by temperature * log L +
// log(alpha / m), and draws the new class. A class's log L comes from the
// table (the classes the particle entered with), from single-site pruning
// (classes opened during this pass, one warp per class, all its rates
// together), or from the auxiliary-class kernel. An auxiliary that is drawn
// becomes class slot kcur: its logits are drawn again from the same stream
// and it is diagonalised once.
__global__ void __launch_bounds__(32 * kGibbsWarps) gibbs_kernel(GibbsArgs a) {
    const Dims& d = a.d;
    const int i = blockIdx.x;
    const GibbsPart gp = a.parts[i];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int Kcap = a.Kcap;
    double* spec = a.spec + (size_t)i * Kcap * kSpecStride;
    double* stash = a.stash + ((size_t)i * kGibbsWarps + warp) * a.nslots * kRateBlock * 32;
    __shared__ __align__(16) double xch[kGibbsWarps][kRateBlock * kStates];
    double* logits = a.logits + (size_t)i * (Kcap + kAux) * kStates;
    int32_t* assign = a.assign + (size_t)i * d.S;
    const double* base = a.base + (size_t)i * kBase;
    extern __shared__ double sh[];                   // lnl [Kcap * R]
    double* wts = sh + (size_t)Kcap * d.R;           // [Kcap + kAux]
    int* counts = reinterpret_cast<int*>(wts + (Kcap + kAux));  // [Kcap + kAux]
    uint8_t* scode = reinterpret_cast<uint8_t*>(counts + (Kcap + kAux));  // [T]: the site's column
    const bool weights_mode = gp.fixed_site >= 0;
    __shared__ int s_site, s_kcur, s_choice;
    __shared__ SpecWork work[kAux];
    const double* auxl = a.aux_ls + (size_t)i * gp.n_iter * kAux;
    const int32_t* auxs = a.aux_site + (size_t)i * gp.n_iter;

    // Table mode resumes where the particle's last round stopped.
    const bool tabmode = a.table != nullptr;
    const int it0 = tabmode ? a.resume_it[i] : 0;
    const int kstart = tabmode ? a.resume_kcur[i] : gp.K;
    if (it0 > 0 && it0 >= gp.n_iter) return;  // finished in an earlier round (uniform)
    if (threadIdx.x == 0) s_kcur = kstart;
    for (int k = threadIdx.x; k < Kcap + kAux; k += blockDim.x) counts[k] = 0;
    __syncthreads();
    for (int x = threadIdx.x; x < d.S; x += blockDim.x) atomicAdd(&counts[assign[x]], 1);
    // Classes [0, K0) read their site log-likelihoods from the table: the entry
    // classes and those opened in earlier rounds (whose columns the caller has
    // filled). The others are pruned per site below: in table mode the classes
    // opened into slots at or above Kt (diagonalised when they opened),
    // without a table every class.
    const int K0 = tabmode ? min(kstart, a.Kt) : 0;
    const double* tab = tabmode ? a.table + (size_t)i * a.Kt * d.S : nullptr;
    if (!tabmode && warp < kAux)  // one shared workspace per decomposing warp
        for (int k = warp; k < gp.K; k += kAux)
            spectral_decompose_warp_ws(base, logits + (size_t)k * kStates,
                                       spec + (size_t)k * kSpecStride, work[warp]);
    __syncthreads();

    const double alpha_split = log(a.alpha / kAux);
    int stop = gp.n_iter;  // table mode: the iteration after a birth into a table slot
    bool stopped = false;
    for (int it = it0; it < gp.n_iter; ++it) {
        // 1. the drawn site leaves its class (Particle.cpp:808-821)
        if (threadIdx.x == 0) {
            const int s = auxs[it];
            s_site = s;
            counts[assign[s]]--;
        }
        __syncthreads();
        const int s = s_site, kcur = s_kcur;
        // 2. per-site pruning of the classes not in the table (Particle.cpp:857-930)
        if (kcur > K0) {
            for (int c = threadIdx.x; c < d.T; c += blockDim.x) scode[c] = a.codes[(size_t)c * d.S + s];
            __syncthreads();
            for (int k = K0 + warp; k < kcur; k += kGibbsWarps)
                if (counts[k] > 0)
                    for (int r0 = 0; r0 < d.R; r0 += kRateBlock)
                        site_class_lnl<kRateBlock>(a, gp, i, r0, spec + (size_t)k * kSpecStride, stash,
                                                   scode, xch[warp], sh + (size_t)k * d.R + r0);
            __syncthreads();
        }
        // 3. weights and the draw (Particle.cpp:931-978), one warp: lanes take
        // classes in turn; the cumulative sum runs in class order, chunk by
        // chunk of 32 with a warp scan, and the total is that sum's end.
        if (warp == 0) {
            const int ktot = kcur + kAux;
            double wmax = -INFINITY;
            for (int k = lane; k < ktot; k += 32) {
                double w = -INFINITY;
                if (k >= kcur) {
                    w = auxl[(size_t)it * kAux + (k - kcur)] * a.temp + alpha_split;
                } else if (counts[k] > 0) {
                    const double ls = k < K0 ? tab[(size_t)k * d.S + s]
                                             : site_value(a, gp, s, sh + (size_t)k * d.R,
                                                          spec + (size_t)k * kSpecStride + kSpecPi);
                    w = ls * a.temp + log((double)counts[k]);
                }
                wts[k] = w;
                wmax = fmax(wmax, w);
            }
            wmax = warp_max20(wmax);
            __syncwarp();
            if (weights_mode)
                for (int k = lane; k < ktot; k += 32) a.weights_out[(size_t)i * (Kcap + kAux) + k] = wts[k];
            double run = 0.0;
            for (int b0 = 0; b0 < ktot; b0 += 32) {
                const int k = b0 + lane;
                const double x = warp_incl_scan((k < ktot && wts[k] > -INFINITY) ? exp(wts[k] - wmax) : 0.0);
                run += __shfl_sync(0xffffffffu, x, 31);
            }
            const double u = __shfl_sync(0xffffffffu, lane == 0 ? draw_choice(a.seed, gp.p, it) : 0.0, 0);
            const double draw = run * u;
            int choice = ktot - 1;
            run = 0.0;
            for (int b0 = 0; b0 < ktot; b0 += 32) {
                const int k = b0 + lane;
                const bool live = k < ktot && wts[k] > -INFINITY;
                const double x = warp_incl_scan(live ? exp(wts[k] - wmax) : 0.0);
                const unsigned hit = __ballot_sync(0xffffffffu, live && run + x >= draw);
                if (hit) {
                    choice = b0 + __ffs(hit) - 1;
                    break;
                }
                run += __shfl_sync(0xffffffffu, x, 31);
            }
            if (lane == 0) {
                if (choice >= kcur && kcur >= Kcap) {
                    atomicOr(a.status, 4);  // class capacity exhausted: keep the old class
                    choice = assign[s];
                }
                if (weights_mode) {
                    counts[assign[s]]++;  // leave the state as it was
                    choice = -1;
                }
                s_choice = choice;
            }
        }
        __syncthreads();
        const int choice = s_choice;
        if (choice < 0) break;  // weights mode: nothing changes
        if (choice >= kcur) {
            // The drawn auxiliary becomes class slot kcur. In table mode a slot
            // below Kt gets a table column: its spectral record also goes to the
            // engine's workspace and the round ends here.
            const bool to_table = tabmode && kcur < a.Kt;
            if (warp == 0) {
                if (lane == 0) draw_aux_logits(a.seed, gp.p, it, choice - kcur, logits + (size_t)kcur * kStates);
                __syncwarp();
                double* rec = spec + (size_t)kcur * kSpecStride;
                spectral_decompose_warp_ws(base, logits + (size_t)kcur * kStates, rec, work[0]);
                __syncwarp();
                if (to_table) {
                    const size_t ek = (size_t)gp.p * d.Kmax + kcur;
                    double* er = a.eng_spec + (ek * 2 + (a.eng_sws[ek] & kSwsSpec)) * kSpecStride;
                    for (int x = lane; x < kSpecStride; x += 32) er[x] = rec[x];
                }
                if (lane == 0) {
                    assign[s] = kcur;
                    counts[kcur] = 1;
                    s_kcur = kcur + 1;
                }
            }
            if (to_table) {
                stop = it + 1;
                stopped = true;
                break;  // uniform: every thread saw the same choice and slot
            }
        } else if (threadIdx.x == 0) {
            assign[s] = choice;
            counts[choice]++;
        }
        __syncthreads();
    }
    __syncthreads();
    if (tabmode && threadIdx.x == 0) {
        a.resume_it[i] = stop;
        a.resume_kcur[i] = s_kcur;
        // The new class's column is needed only if iterations remain.
        a.born[i] = (stopped && stop < gp.n_iter) ? s_kcur - 1 : -1;
    }
    for (int k = threadIdx.x; k < s_kcur; k += blockDim.x) a.counts[(size_t)i * (Kcap + kAux) + k] = counts[k];
    if (threadIdx.x == 0) a.kout[i] = s_kcur;
}

// ---------------------------------------------------------------------------
// Learned-proposal site reassignment.
//
// One CTA of 128 threads per particle. The scoring MLP runs on the
// 5th-generation tensor cores: the feature rows of up to 128 classes are one
// M = 128 operand in tensor memory (thread t writes row t, BF16), each layer
// is one tcgen05.mma kind::f16 product against the BF16 weights, staged once
// in shared memory in the K-major canonical layout (no swizzle), with FP32
// accumulation in tensor memory; thread t reads its row back for the bias,
// the ReLU and the next layer's operand (or the final dot product):
//   layer 1: D[c][j] = sum_i X[c][i] W1[i][j]   M = 128, N = 128, K = 48 (44 inputs)
//   layer 2: D[c][j] = sum_i H[c][i] W2[i][j]   M = 128, N = 128, K = 128
// Tensor-memory columns: X [0, 24), D [32, 160), H [160, 224).
// A class's score depends on its own row only, so the reverse scores (two
// classes with updated sizes) come from the same products as the forward ones.
constexpr int kLmThreads = 128;
constexpr int kLmK1 = 48;
constexpr uint32_t kLmCols = 256;
constexpr uint32_t kLmColX = 0, kLmColD = 32, kLmColH = 160;
constexpr uint32_t kLmLbo = 128;                   // next core matrix along K
constexpr uint32_t kLmSbo1 = (kLmK1 / 8) * 128;    // W1: next 8-row group
constexpr uint32_t kLmSbo2 = (kMlpHid / 8) * 128;  // W2: next 8-row group
constexpr uint32_t kLmW1Bytes = kMlpHid * kLmK1 * 2;
constexpr uint32_t kLmW2Bytes = kMlpHid * kMlpHid * 2;
// idesc: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), K-major A
// and B, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kLmIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kMlpHid >> 3) << 17) |
                              ((uint32_t)(kLmThreads >> 4) << 24);

__device__ __forceinline__ uint32_t lm_sa(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (n, k) of a K-major canonical BF16 tile (8-row x
// 16-byte core matrices).
__device__ __forceinline__ uint32_t lm_kmaj(int n, int k, uint32_t sbo) {
    return (n >> 3) * sbo + (k >> 3) * kLmLbo + (n & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint64_t lm_desc(uint32_t addr, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(kLmLbo >> 4) << 16) |
           ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void lm_st8(uint32_t taddr, const uint32_t* v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}

__device__ __forceinline__ void lm_ld8(uint32_t taddr, uint32_t* v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                   "=r"(v[7])
                 : "r"(taddr)
                 : "memory");
}

__device__ __forceinline__ void lm_mma(uint32_t d, uint32_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %4, p;\n\t}" ::"r"(d),
        "r"(a), "l"(b), "r"(acc), "r"(kLmIdesc)
        : "memory");
}

__device__ __forceinline__ void lm_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(lm_sa(bar))
                 : "memory");
}

__device__ __noinline__ bool lm_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(lm_sa(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const uint32_t l = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
    const uint32_t h = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
    return l | (h << 16);
}

// Shared state of the learned-move CTA's tensor-core scoring.
struct LmState {
    uint32_t tm;       // tensor-memory base
    uint64_t* bar;     // product-completion barrier
    uint32_t phase;    // its next parity
    bool pend;         // thread 0: a committed product not yet waited on
    uint32_t limit;
};

// One product of the CTA (thread 0 issues, every thread waits for it).
// `ok` is uniform on entry and on return.
__device__ bool lm_product(LmState& s, bool ok, uint32_t acol, uint32_t bbase, uint32_t sbo, int ksteps,
                           int* status) {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok);
    if (!ok) return false;
    if (threadIdx.x == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        for (int ks = 0; ks < ksteps; ++ks)
            lm_mma(s.tm + kLmColD, s.tm + acol + 8 * ks, lm_desc(bbase + ks * 2 * kLmLbo, sbo), ks > 0);
        lm_commit(s.bar);
        s.pend = true;
    }
    bool got = lm_wait(s.bar, s.phase, s.limit);
    if (got) {
        s.phase ^= 1u;
        if (threadIdx.x == 0) s.pend = false;
    } else {
        atomicOr(status, 8);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return __syncthreads_and(got);
}

// Scores of the feature rows each thread has just written to columns
// [kLmColX, +24) of its lane: both layers and the final dot product. Thread t
// gets its own row's score.
__device__ bool lm_scores(LmState& s, bool ok, const unsigned char* w1t, const unsigned char* w2t,
                          const float* b1, const float* b2, const float* w3, float b3, int* status,
                          float* out) {
    const uint32_t tl = s.tm + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);  // this warp's lane quarter
    ok = lm_product(s, ok, kLmColX, lm_sa(w1t), kLmSbo1, kLmK1 / 16, status);
    if (ok) {
        for (int c16 = 0; c16 < kMlpHid / 16; ++c16) {
            uint32_t v[16], h[8];
            lm_ld8(tl + kLmColD + 16 * c16, v);
            lm_ld8(tl + kLmColD + 16 * c16 + 8, v + 8);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int j = 16 * c16 + 2 * q;
                h[q] = pack_bf16(fmaxf(__uint_as_float(v[2 * q]) + b1[j], 0.f),
                                 fmaxf(__uint_as_float(v[2 * q + 1]) + b1[j + 1], 0.f));
            }
            lm_st8(tl + kLmColH + 8 * c16, h);
        }
    }
    ok = lm_product(s, ok, kLmColH, lm_sa(w2t), kLmSbo2, kMlpHid / 16, status);
    float sc = b3;
    if (ok) {
        for (int c16 = 0; c16 < kMlpHid / 16; ++c16) {
            uint32_t v[16];
            lm_ld8(tl + kLmColD + 16 * c16, v);
            lm_ld8(tl + kLmColD + 16 * c16 + 8, v + 8);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int j = 16 * c16 + q;
                sc = fmaf(fmaxf(__uint_as_float(v[q]) + b2[j], 0.f), w3[j], sc);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    *out = sc;
    return ok;
}

// This thread's feature row (site features sf, class stationary pi and its
// logarithm, class size n) into tensor-memory columns [kLmColX, +24) of its lane;
// zeros for a row without a class.
__device__ void lm_features(uint32_t tl, const float* sf, const float* pi, const float* lpi, int n, bool on) {
    float x[kLmK1];
#pragma unroll
    for (int i = 0; i < kLmK1; ++i) x[i] = 0.f;
    if (on) {
        float dot = 0.f;
#pragma unroll
        for (int i = 0; i < kSiteFeat; ++i) x[i] = sf[i];
#pragma unroll
        for (int m = 0; m < kStates; ++m) {
            x[kSiteFeat + m] = pi[m];
            dot = fmaf(sf[m], lpi[m], dot);
        }
        x[kSiteFeat + 20] = logf((float)(n > 1 ? n : 1));
        x[kSiteFeat + 21] = dot;
    }
    uint32_t u[kLmK1 / 2];
#pragma unroll
    for (int q = 0; q < kLmK1 / 2; ++q) u[q] = pack_bf16(x[2 * q], x[2 * q + 1]);
#pragma unroll
    for (int c8 = 0; c8 < kLmK1 / 16; ++c8) lm_st8(tl + kLmColX + 8 * c8, u + 8 * c8);
}

__global__ void __launch_bounds__(kLmThreads) learned_move_kernel(GibbsArgs a, const __nv_bfloat16* mlp,
                                                                  const float* site_feat, int32_t* n_acc,
                                                                  int32_t* n_prop) {
    const Dims& d = a.d;
    const int i = blockIdx.x;
    const GibbsPart gp = a.parts[i];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int K = gp.K;
    double* spec = a.spec + (size_t)i * a.Kcap * kSpecStride;
    double* stash = a.stash + ((size_t)i * kGibbsWarps + warp) * a.nslots * kRateBlock * 32;
    // With the class table the two classes' site values are looked up;
    // without it they are pruned per update.
    const bool tabled = a.table != nullptr;
    const double* tab = tabled ? a.table + (size_t)i * a.Kt * d.S : nullptr;
    __shared__ __align__(16) double xch[kLmThreads / 32][kRateBlock * kStates];
    const double* logits = a.logits + (size_t)i * (a.Kcap + kAux) * kStates;
    int32_t* assign = a.assign + (size_t)i * d.S;
    const double* base = a.base + (size_t)i * kBase;
    extern __shared__ __align__(1024) unsigned char lsm[];
    unsigned char* w1t = lsm;                                  // W1 tile
    unsigned char* w2t = lsm + kLmW1Bytes;                     // W2 tile
    float* bias = reinterpret_cast<float*>(w2t + kLmW2Bytes);  // b1, b2, w3 [3][kMlpHid]
    float* pis = bias + 3 * kMlpHid;                           // [Kcap][20]
    float* lpis = pis + (size_t)a.Kcap * kStates;              // [Kcap][20]
    float* score = lpis + (size_t)a.Kcap * kStates;            // [Kcap]
    int* counts = reinterpret_cast<int*>(score + a.Kcap);      // [Kcap]
    uint8_t* scode = reinterpret_cast<uint8_t*>(counts + a.Kcap);  // [T]
    __shared__ double lrate[2][kMaxRates];
    __shared__ float rev[2], sfs[kSiteFeat];
    __shared__ int s_site, s_a, s_b;
    __shared__ SpecWork work[kLmThreads / 32];
    __shared__ int acc_n, prop_n;
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ uint32_t tmem_slot;

    // Weights: the two layer tiles in the canonical layout, biases and the
    // output row in FP32.
    for (int x = tid; x < kMlpHid * kLmK1; x += kLmThreads) {
        const int n = x / kLmK1, k = x % kLmK1;
        const __nv_bfloat16 w = k < kMlpIn ? mlp[kMlpW1 + k * kMlpHid + n] : __float2bfloat16_rn(0.f);
        *reinterpret_cast<__nv_bfloat16*>(w1t + lm_kmaj(n, k, kLmSbo1)) = w;
    }
    for (int x = tid; x < kMlpHid * kMlpHid; x += kLmThreads) {
        const int n = x / kMlpHid, k = x % kMlpHid;
        *reinterpret_cast<__nv_bfloat16*>(w2t + lm_kmaj(n, k, kLmSbo2)) = mlp[kMlpW2 + k * kMlpHid + n];
    }
    for (int j = tid; j < kMlpHid; j += kLmThreads) {
        bias[j] = __bfloat162float(mlp[kMlpB1 + j]);
        bias[kMlpHid + j] = __bfloat162float(mlp[kMlpB2 + j]);
        bias[2 * kMlpHid + j] = __bfloat162float(mlp[kMlpW3 + j]);
    }
    const float b3 = __bfloat162float(mlp[kMlpB3]);
    // Class stationary distributions (softmax of the logits) and their logs.
    for (int k = tid; k < K; k += kLmThreads) {
        const double* lg = logits + (size_t)k * kStates;
        double e[kStates], tot = 0.0;
        for (int m = 0; m < kStates; ++m) { e[m] = exp(lg[m]); tot += e[m]; }
        for (int m = 0; m < kStates; ++m) {
            const double pv = e[m] / tot;
            pis[(size_t)k * kStates + m] = (float)pv;
            lpis[(size_t)k * kStates + m] = (float)log(pv);
        }
    }
    for (int k = tid; k < a.Kcap; k += kLmThreads) counts[k] = 0;
    if (tid == 0) {
        acc_n = prop_n = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(lm_sa(&mma_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(lm_sa(&tmem_slot)),
                     "r"(kLmCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // The weight tiles are read by the tensor cores (the async proxy).
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    LmState ls{tmem_slot, &mma_bar, 0u, false, a.wait_limit};
    const uint32_t tl = ls.tm + ((uint32_t)(warp * 32) << 16);
    for (int x = tid; x < d.S; x += kLmThreads) atomicAdd(&counts[assign[x]], 1);
    if (!tabled)  // per-update pruning needs every class's eigensystem
        for (int k = warp; k < K; k += kLmThreads / 32)
            spectral_decompose_warp_ws(base, logits + (size_t)k * kStates, spec + (size_t)k * kSpecStride,
                                       work[warp]);
    __syncthreads();
    bool ok = true;
    for (int it = 0; it < gp.n_iter && ok; ++it) {
        // One site, uniform over all S. A site alone in its class stays put
        // (the move never empties a class), so the site is selected with
        // probability 1/S both ways and the selection cancels from the
        // Metropolis-Hastings ratio: a draw from only the sites that may move
        // would not, since moving a site changes which sites those are.
        if (tid == 0) {
            if (gp.fixed_site >= 0) {  // scores mode
                s_site = gp.fixed_site;
            } else {
                const int c = draw_site(a.seed, gp.p, it, d.S);
                s_site = counts[assign[c]] >= 2 ? c : -1;
            }
        }
        __syncthreads();
        const int s = s_site;
        if (s < 0) continue;
        if (tid < kSiteFeat) sfs[tid] = site_feat[(size_t)s * kSiteFeat + tid];
        if (!tabled)
            for (int c = tid; c < d.T; c += kLmThreads) scode[c] = a.codes[(size_t)c * d.S + s];
        __syncthreads();
        // Forward scores, 128 classes per product.
        for (int rb = 0; rb < K && ok; rb += kLmThreads) {
            const int k = rb + tid;
            const bool on = k < K;
            lm_features(tl, sfs, pis + (size_t)(on ? k : 0) * kStates, lpis + (size_t)(on ? k : 0) * kStates,
                        on ? counts[k] : 1, on);
            float v;
            ok = lm_scores(ls, ok, w1t, w2t, bias, bias + kMlpHid, bias + 2 * kMlpHid, b3, a.status, &v);
            if (on) score[k] = v;
        }
        __syncthreads();
        if (!ok) break;
        if (gp.fixed_site >= 0) {  // scores mode: report the forward scores, move nothing
            for (int k = tid; k < K; k += kLmThreads) a.weights_out[(size_t)i * (a.Kcap + kAux) + k] = score[k];
            break;
        }
        if (warp == 0) {  // the proposal draw, in class order (warp scan over chunks of 32)
            float mx = -INFINITY;
            for (int k = lane; k < K; k += 32) mx = fmaxf(mx, score[k]);
            mx = warp_maxf(mx);
            double run = 0.0;
            for (int b0 = 0; b0 < K; b0 += 32) {
                const int k = b0 + lane;
                const double x = warp_incl_scan(k < K ? exp((double)(score[k] - mx)) : 0.0);
                run += __shfl_sync(0xffffffffu, x, 31);
            }
            const double u =
                __shfl_sync(0xffffffffu, lane == 0 ? draw_at(a.seed, gp.p, it, kOffProposal) : 0.0, 0);
            const double draw = run * u;
            int b = K - 1;
            run = 0.0;
            for (int b0 = 0; b0 < K; b0 += 32) {
                const int k = b0 + lane;
                const double x = warp_incl_scan(k < K ? exp((double)(score[k] - mx)) : 0.0);
                const unsigned hit = __ballot_sync(0xffffffffu, k < K && run + x >= draw);
                if (hit) {
                    b = b0 + __ffs(hit) - 1;
                    break;
                }
                run += __shfl_sync(0xffffffffu, x, 31);
            }
            if (lane == 0) {
                s_a = assign[s];
                s_b = b;
                prop_n++;
            }
        }
        __syncthreads();
        const int ca = s_a, cb = s_b;
        if (ca == cb) {  // proposing the current class: a no-op, always accepted
            if (tid == 0) acc_n++;
            __syncthreads();
            continue;
        }
        // Reverse scores: the two classes with their sizes after the move, from
        // the products of their row blocks.
        for (int pass = 0; pass < 2 && ok; ++pass) {
            const int rb = (pass == 0 ? ca : cb) / kLmThreads * kLmThreads;
            if (pass == 1 && rb == ca / kLmThreads * kLmThreads) break;  // same block as ca
            const int k = rb + tid;
            const bool on = (k == ca || k == cb);
            lm_features(tl, sfs, pis + (size_t)(on ? k : 0) * kStates, lpis + (size_t)(on ? k : 0) * kStates,
                        on ? counts[k] + (k == ca ? -1 : 1) : 1, on);
            float v;
            ok = lm_scores(ls, ok, w1t, w2t, bias, bias + kMlpHid, bias + 2 * kMlpHid, b3, a.status, &v);
            if (k == ca) rev[0] = v;
            if (k == cb) rev[1] = v;
        }
        // Without the table: site likelihoods under the two classes (warps
        // 0..nb-1: a, nb..2nb-1: b, kRateBlock rates each).
        const int nb = tabled ? 0 : (d.R + kRateBlock - 1) / kRateBlock;
        if (ok && warp < 2 * nb) {
            const int which = warp < nb ? 0 : 1, r0 = (warp % nb) * kRateBlock;
            const int k = which == 0 ? ca : cb;
            site_class_lnl<kRateBlock>(a, gp, i, r0, spec + (size_t)k * kSpecStride, stash, scode, xch[warp],
                                       lrate[which] + r0);
        }
        __syncthreads();
        if (ok && warp == 0) {
            float mx = -INFINITY, mx2 = -INFINITY;
            for (int k = lane; k < K; k += 32) {
                mx = fmaxf(mx, score[k]);
                mx2 = fmaxf(mx2, k == ca ? rev[0] : (k == cb ? rev[1] : score[k]));
            }
            mx = warp_maxf(mx);
            mx2 = warp_maxf(mx2);
            double z = 0.0, z2 = 0.0;
            for (int k = lane; k < K; k += 32) {
                z += exp((double)(score[k] - mx));
                z2 += exp((double)((k == ca ? rev[0] : (k == cb ? rev[1] : score[k])) - mx2));
            }
            z = wsum(z);
            z2 = wsum(z2);
            if (lane == 0) {
                const double la = tabled ? tab[(size_t)ca * d.S + s]
                                         : site_value(a, gp, s, lrate[0], spec + (size_t)ca * kSpecStride + kSpecPi);
                const double lb = tabled ? tab[(size_t)cb * d.S + s]
                                         : site_value(a, gp, s, lrate[1], spec + (size_t)cb * kSpecStride + kSpecPi);
                const double lq_fwd = (score[cb] - mx) - log(z);
                const double lq_rev = (rev[0] - mx2) - log(z2);
                // CRP prior ratio n_b / (n_a - 1); tempered likelihood ratio.
                const double lr = a.temp * (lb - la) + log((double)counts[cb]) -
                                  log((double)(counts[ca] - 1)) + lq_rev - lq_fwd;
                if (log(draw_at(a.seed, gp.p, it, kOffAccept)) <= lr) {
                    assign[s] = cb;
                    counts[ca]--;
                    counts[cb]++;
                    acc_n++;
                }
            }
        }
        __syncthreads();
    }
    // A product still in flight (after a wait gave up) lands before the
    // tensor memory is released.
    if (tid == 0 && ls.pend) lm_wait(ls.bar, ls.phase, kDrainPolls);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(ls.tm), "r"(kLmCols) : "memory");
    for (int k = tid; k < K; k += kLmThreads) a.counts[(size_t)i * (a.Kcap + kAux) + k] = counts[k];
    if (tid == 0) {
        a.kout[i] = K;
        n_acc[i] = acc_n;
        n_prop[i] = prop_n;
    }
}

}  // namespace

namespace {

// Grid of the auxiliary-class kernel: kAuxCtasPerSm CTAs per SM, or fewer
// when there are fewer tasks.
int aux_grid(size_t tasks) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        sms = 148;
    const size_t want = (tasks + kAuxWarps - 1) / kAuxWarps;
    const size_t cap = (size_t)sms * kAuxCtasPerSm;
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

struct ScratchLayout {
    size_t spec, stash, aux_ls, aux_site, aux_rec, aux_stash, total;
};

ScratchLayout scratch_layout(const Dims& d, int count, int Kcap, int n_iter, int nslots, bool aux) {
    ScratchLayout L{};
    size_t o = 0;
    auto take = [&](size_t n) { const size_t r = o; o += (n + 31) & ~size_t(31); return r; };
    L.spec = take((size_t)count * Kcap * kSpecStride);
    L.stash = take((size_t)count * kGibbsWarps * nslots * kRateBlock * 32);
    if (aux) {
        const size_t tasks = (size_t)count * n_iter * kAux;
        const size_t warps = (size_t)aux_grid(tasks) * kAuxWarps;
        L.aux_ls = take(tasks);
        L.aux_site = take(((size_t)count * n_iter + 1) / 2);  // int32 pairs
        L.aux_rec = take(warps * kSpecStride);
        L.aux_stash = take(warps * nslots * kRateBlock * 32);
    }
    L.total = o;
    return L;
}

}  // namespace

namespace {

void set_scratch(GibbsArgs& a, int n_iter, double* scratch) {
    const ScratchLayout L = scratch_layout(a.d, a.count, a.Kcap, n_iter, a.nslots, true);
    a.spec = scratch + L.spec;
    a.stash = scratch + L.stash;
    a.aux_ls = scratch + L.aux_ls;
    a.aux_site = reinterpret_cast<int32_t*>(scratch + L.aux_site);
    a.aux_rec = scratch + L.aux_rec;
    a.aux_stash = scratch + L.aux_stash;
}

size_t gibbs_smem(const GibbsArgs& a) {
    return sizeof(double) * ((size_t)a.Kcap * a.d.R + a.Kcap + kAux) + sizeof(int) * (a.Kcap + kAux) + a.d.T + 16;
}

}  // namespace

cudaError_t launch_learned_move(GibbsArgs a, int n_iter, const void* mlp, const float* site_feat,
                                int32_t* n_acc, int32_t* n_prop, double* scratch, cudaStream_t st) {
    const Dims& d = a.d;
    set_scratch(a, n_iter, scratch);
    const size_t smem = kLmW1Bytes + kLmW2Bytes + sizeof(float) * (3 * kMlpHid + (size_t)a.Kcap * (2 * kStates + 1)) +
                        sizeof(int) * a.Kcap + d.T + 16;
    cudaError_t e = cudaFuncSetAttribute(learned_move_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    learned_move_kernel<<<a.count, kLmThreads, smem, st>>>(
        a, static_cast<const __nv_bfloat16*>(mlp), site_feat, n_acc, n_prop);
    return cudaGetLastError();
}

size_t gibbs_scratch_doubles(const Dims& d, int count, int Kcap, int n_iter, int nslots, bool aux) {
    return scratch_layout(d, count, Kcap, n_iter, nslots, aux).total;
}

int gibbs_aux() { return kAux; }

cudaError_t launch_gibbs_aux(GibbsArgs a, int n_iter, double* scratch, cudaStream_t st) {
    set_scratch(a, n_iter, scratch);
    const size_t tasks = (size_t)a.count * n_iter * kAux;
    gibbs_aux_kernel<<<aux_grid(tasks), 32 * kAuxWarps, (size_t)kAuxWarps * a.d.T, st>>>(a, n_iter);
    return cudaGetLastError();
}

cudaError_t launch_draw_sites(GibbsArgs a, int n_iter, double* scratch, cudaStream_t st) {
    set_scratch(a, n_iter, scratch);
    const size_t n = (size_t)a.count * n_iter;
    draw_sites_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, n_iter);
    return cudaGetLastError();
}

cudaError_t launch_visited_sites(GibbsArgs a, int n_iter, double* scratch, const int32_t* qrow, uint8_t* flags,
                                 int32_t* list, int32_t* nv, cudaStream_t st) {
    set_scratch(a, n_iter, scratch);
    visited_sites_kernel<<<a.count, kVisitThreads, 0, st>>>(a.aux_site, n_iter, qrow, a.d.S, flags, list, nv);
    return cudaGetLastError();
}

cudaError_t launch_gibbs_resume(GibbsArgs a, int n_iter, double* scratch, cudaStream_t st) {
    set_scratch(a, n_iter, scratch);
    const size_t smem = gibbs_smem(a);
    cudaError_t e = cudaFuncSetAttribute(gibbs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    gibbs_kernel<<<a.count, 32 * kGibbsWarps, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_gibbs(GibbsArgs a, int n_iter, double* scratch, cudaStream_t st) {
    cudaError_t e = launch_gibbs_aux(a, n_iter, scratch, st);
    if (e == cudaSuccess) e = launch_gibbs_resume(a, n_iter, scratch, st);
    return e;
}

}  // namespace smccat
