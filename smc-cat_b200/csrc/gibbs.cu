// CAT class reassignment (Neal's Algorithm 8, m = 5 auxiliary classes) on the
// device: Particle::gibbsPartitionMove (Particle.cpp:785-995), corrected form.
//
// One CTA per particle runs the floor(S/2) site iterations in order. Each
// iteration: draw a site and take it out of its class (dropping the class if
// it empties), draw m fresh classes from the prior (19 N(0,1) logits + 0,
// TransitionProbabilityClass.cpp:26-35) and diagonalise them (one warp each),
// evaluate the site's likelihood under every live class and every auxiliary
// class (one warp per (class, rate) pair, lanes = states, single-site pruning
// in the eigenbasis P(t)x = L (exp(lambda t) o (Rm x))), weight each class by
// temperature * log L + log n_k (or log(alpha / m) for the auxiliaries) and
// draw the new class. Random numbers come from a per-particle Philox stream.
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

// exp(lambda_m t_n r) for every (node, rate) of class slot k.
__device__ void fill_exp(const GibbsArgs& a, int i, int k, const double* rec, double* ex) {
    const Dims& d = a.d;
    const GibbsPart& gp = a.parts[i];
    const double* br = a.branch + (size_t)i * d.N;
    for (int idx = threadIdx.x; idx < d.N * d.R * kStates; idx += blockDim.x) {
        const int m = idx % kStates, r = (idx / kStates) % d.R, n = idx / (kStates * d.R);
        ex[idx] = exp(rec[kSpecLam + m] * br[n] * gp.rates[r]);
    }
}

// Rates per warp in the Gibbs weights (all of a class's rates together) and in
// the learned move (which spreads its two classes' rates over more warps).
constexpr int kRateBlock = 4;
constexpr int kRateBlockLearned = 2;

// Log-likelihoods of one site under one class for rates [r0, r0 + RB) (those
// below R), one warp: lanes are states and the rate chains interleave.
// Single-site pruning in the eigenbasis, P(t r) x = L (exp(lambda t r) o (Rm x)).
// The vectors every lane needs whole (x before Rm, z before L) pass through the
// warp's shared exchange row `xch` [RB][kStates] and are read back as broadcast
// pairs, not shuffled lane by lane. The node computed last stays in registers
// (in post-order it is a child of the next node); other internal children come
// back from the warp's stash [NI][RB][32]. Tip codes of the site come from
// `scode` (shared). out[b] = log L of rate r0 + b.
template <int RB>
__device__ void site_class_lnl(const GibbsArgs& a, int i, int r0, const double* rec,
                               const double* ex, double* stash, const uint8_t* scode,
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
    double rs = 0.0;
#pragma unroll
    for (int j = 0; j < kStates; ++j) rs += Rrow[j];
    bool on[RB];
    double v[RB], lsc[RB];
#pragma unroll
    for (int b = 0; b < RB; ++b) {
        on[b] = r0 + b < d.R;
        v[b] = 1.0;
        lsc[b] = 0.0;
    }
    const int32_t* tree = a.tree + (size_t)i * d.NI * 3;
    int prev = -1;
    for (int q = 0; q < d.NI; ++q) {
        const int n = tree[3 * q];
        double vn[RB];
#pragma unroll
        for (int b = 0; b < RB; ++b) vn[b] = 1.0;
#pragma unroll 1
        for (int ci = 1; ci <= 2; ++ci) {
            const int c = tree[3 * q + ci];
            double e[RB], z[RB];
#pragma unroll
            for (int b = 0; b < RB; ++b)
                e[b] = on[b] ? ex[((size_t)c * d.R + r0 + b) * kStates + li] : 0.0;
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
#pragma unroll
                for (int b = 0; b < RB; ++b) {
                    const double xv = (c == prev) ? v[b]
                                                  : stash[((size_t)(c - d.T) * RB + b) * 32 + lane];
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
            stash[((size_t)(n - d.T) * RB + b) * 32 + lane] = x;
        }
        prev = n;
        __syncwarp();
    }
    const double pi = st_lane ? rec[kSpecPi + lane] : 0.0;
#pragma unroll
    for (int b = 0; b < RB; ++b) {
        const double sv = wsum(pi * v[b]);
        if (lane == 0 && on[b]) out[b] = log(sv) + lsc[b];
    }
}

__global__ void __launch_bounds__(32 * kGibbsWarps) gibbs_kernel(GibbsArgs a) {
    const Dims& d = a.d;
    const int i = blockIdx.x;
    const GibbsPart gp = a.parts[i];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int Kcap = a.Kcap;
    double* spec = a.spec + (size_t)i * (Kcap + kAux) * kSpecStride;
    double* ex = a.expt + (size_t)i * (Kcap + kAux) * d.N * d.R * kStates;
    double* stash = a.stash + ((size_t)i * kGibbsWarps + warp) * d.NI * kRateBlock * 32;
    __shared__ __align__(16) double xch[kGibbsWarps][kRateBlock * kStates];
    double* logits = a.logits + (size_t)i * (Kcap + kAux) * kStates;
    int32_t* assign = a.assign + (size_t)i * d.S;
    const double* base = a.base + (size_t)i * kBase;
    extern __shared__ double sh[];                   // lnl [(Kcap + kAux) * R]
    double* wts = sh + (size_t)(Kcap + kAux) * d.R;  // [Kcap + kAux]
    int* counts = reinterpret_cast<int*>(wts + (Kcap + kAux));  // [Kcap + kAux]
    uint8_t* scode = reinterpret_cast<uint8_t*>(counts + (Kcap + kAux));  // [T]: the site's column
    const bool weights_mode = gp.fixed_site >= 0;
    __shared__ int s_site, s_kcur, s_choice;
    __shared__ SpecWork work[kAux];
    __shared__ curandStatePhilox4_32_10_t rng_state;

    if (threadIdx.x == 0) {
        curand_init(a.seed, (unsigned long long)gp.p, 0ull, &rng_state);
        s_kcur = gp.K;
    }
    for (int k = threadIdx.x; k < Kcap + kAux; k += blockDim.x) counts[k] = 0;
    __syncthreads();
    for (int x = threadIdx.x; x < d.S; x += blockDim.x) atomicAdd(&counts[assign[x]], 1);
    // Classes [0, K0) read their site log-likelihoods from the table; the
    // others (none without a table) are pruned per site below.
    const int K0 = a.table ? gp.K : 0;
    const double* tab = a.table ? a.table + (size_t)i * a.Kt * d.S : nullptr;
    if (warp < kAux)  // one shared workspace per decomposing warp
        for (int k = K0 + warp; k < gp.K; k += kAux)
            spectral_decompose_warp_ws(base, logits + (size_t)k * kStates,
                                       spec + (size_t)k * kSpecStride, work[warp]);
    __syncthreads();
    for (int k = K0; k < gp.K; ++k)
        fill_exp(a, i, k, spec + (size_t)k * kSpecStride, ex + (size_t)k * d.N * d.R * kStates);
    __syncthreads();

    const double alpha_split = log(a.alpha / kAux);
    for (int it = 0; it < gp.n_iter; ++it) {
        // 1. draw the site and remove it from its class (Particle.cpp:808-821)
        if (threadIdx.x == 0) {
            int s;
            if (weights_mode) {
                s = gp.fixed_site;
            } else {
                const double u = curand_uniform_double(&rng_state);  // (0, 1]
                s = (int)((1.0 - u) * d.S);
                s = s < d.S ? s : d.S - 1;
            }
            s_site = s;
            counts[assign[s]]--;
            for (int j = 0; j < kAux; ++j)
                for (int m = 0; m < kStates; ++m)
                    logits[(size_t)(s_kcur + j) * kStates + m] =
                        weights_mode ? a.aux_in[((size_t)i * kAux + j) * kStates + m]
                                     : ((m < kStates - 1) ? curand_normal_double(&rng_state) : 0.0);
        }
        __syncthreads();
        const int s = s_site, kcur = s_kcur;
        for (int c = threadIdx.x; c < d.T; c += blockDim.x) scode[c] = a.codes[(size_t)c * d.S + s];
        // 2. diagonalise the auxiliary classes (Particle.cpp:823-833)
        if (warp < kAux)
            spectral_decompose_warp_ws(base, logits + (size_t)(kcur + warp) * kStates,
                                       spec + (size_t)(kcur + warp) * kSpecStride, work[warp]);
        __syncthreads();
        for (int j = 0; j < kAux; ++j)
            fill_exp(a, i, kcur + j, spec + (size_t)(kcur + j) * kSpecStride,
                     ex + (size_t)(kcur + j) * d.N * d.R * kStates);
        __syncthreads();
        // 3. site log-likelihood per (class, rate) (Particle.cpp:857-930): one
        // warp per class, all its rates together
        for (int k = K0 + warp; k < kcur + kAux; k += kGibbsWarps) {
            if (k >= kcur || counts[k] > 0) {
                for (int r0 = 0; r0 < d.R; r0 += kRateBlock)
                    site_class_lnl<kRateBlock>(a, i, r0, spec + (size_t)k * kSpecStride,
                                               ex + (size_t)k * d.N * d.R * kStates, stash, scode,
                                               xch[warp], sh + (size_t)k * d.R + r0);
            } else if (lane == 0) {
                for (int r = 0; r < d.R; ++r) sh[(size_t)k * d.R + r] = -INFINITY;
            }
        }
        __syncthreads();
        // 4. weights and the draw (Particle.cpp:931-978)
        if (threadIdx.x == 0) {
            double wmax = -INFINITY;
            for (int k = 0; k < kcur + kAux; ++k) {
                double w = -INFINITY;
                if (k < K0 && counts[k] > 0) {
                    w = tab[(size_t)k * d.S + s] * a.temp + log((double)counts[k]);
                } else if (k >= kcur || counts[k] > 0) {
                    double mx = -INFINITY;
                    for (int r = 0; r < d.R; ++r) mx = fmax(mx, sh[k * d.R + r]);
                    double lse = mx;
                    if (mx > -INFINITY) {
                        double se = 0.0;
                        for (int r = 0; r < d.R; ++r) se += exp(sh[k * d.R + r] - mx);
                        lse = mx + log(se);
                    }
                    const double* pi = spec + (size_t)k * kSpecStride + kSpecPi;
                    double ls;
                    if (gp.pinv > 0.0 && a.isinv[s] != 0) {
                        const double la = log1p(-gp.pinv) + lse;
                        const double lb = log(gp.pinv * pi[a.invchar[s]]);
                        const double m2 = fmax(la, lb);
                        ls = m2 + log(exp(la - m2) + exp(lb - m2));
                    } else {
                        ls = lse + log1p(-gp.pinv);
                    }
                    w = ls * a.temp + ((k < kcur) ? log((double)counts[k]) : alpha_split);
                }
                wts[k] = w;
                wmax = fmax(wmax, w);
            }
            if (weights_mode) {
                for (int k = 0; k < kcur + kAux; ++k)
                    a.weights_out[(size_t)i * (Kcap + kAux) + k] = wts[k];
                counts[assign[s]]++;  // leave the state as it was
            }
            double tot = 0.0;
            for (int k = 0; k < kcur + kAux; ++k) tot += exp(wts[k] - wmax);
            const double draw = tot * curand_uniform_double(&rng_state);
            double run = 0.0;
            int choice = kcur + kAux - 1;
            for (int k = 0; k < kcur + kAux; ++k) {
                const double w = wts[k];
                if (w == -INFINITY) continue;
                run += exp(w - wmax);
                if (run >= draw) { choice = k; break; }
            }
            if (choice >= kcur && kcur >= Kcap) {
                atomicOr(a.status, 4);  // class capacity exhausted: keep the old class
                choice = assign[s];
            }
            if (weights_mode) choice = -1;
            s_choice = choice;
        }
        __syncthreads();
        const int choice = s_choice;
        if (choice < 0) break;  // weights mode: nothing changes
        if (choice >= kcur) {
            // The chosen auxiliary becomes class slot kcur.
            const int src = choice;
            if (src != kcur) {
                for (int x = threadIdx.x; x < kSpecStride; x += blockDim.x)
                    spec[(size_t)kcur * kSpecStride + x] = spec[(size_t)src * kSpecStride + x];
                for (int x = threadIdx.x; x < kStates; x += blockDim.x)
                    logits[(size_t)kcur * kStates + x] = logits[(size_t)src * kStates + x];
                for (int x = threadIdx.x; x < d.N * d.R * kStates; x += blockDim.x)
                    ex[(size_t)kcur * d.N * d.R * kStates + x] = ex[(size_t)src * d.N * d.R * kStates + x];
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                assign[s] = kcur;
                counts[kcur] = 1;
                s_kcur = kcur + 1;
            }
        } else if (threadIdx.x == 0) {
            assign[s] = choice;
            counts[choice]++;
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < s_kcur; k += blockDim.x) a.counts[(size_t)i * (Kcap + kAux) + k] = counts[k];
    if (threadIdx.x == 0) a.kout[i] = s_kcur;
}

// ---------------------------------------------------------------------------
// Learned-proposal site reassignment.

// Score of one (site, class) feature row x (kMlpIn floats, shared) by one warp;
// W is the BF16 parameter vector in shared memory, h a 128-float warp buffer.
__device__ float mlp_score(const __nv_bfloat16* W, const float* x, float* h) {
    const int lane = threadIdx.x & 31;
    float h1[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = lane + 32 * q;
        float v = __bfloat162float(W[kMlpB1 + j]);
        for (int i = 0; i < kMlpIn; ++i) v = fmaf(x[i], __bfloat162float(W[kMlpW1 + i * kMlpHid + j]), v);
        h1[q] = fmaxf(v, 0.f);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q) h[lane + 32 * q] = h1[q];
    __syncwarp();
    float part = 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = lane + 32 * q;
        float v = __bfloat162float(W[kMlpB2 + j]);
        for (int i = 0; i < kMlpHid; ++i) v = fmaf(h[i], __bfloat162float(W[kMlpW2 + i * kMlpHid + j]), v);
        part = fmaf(fmaxf(v, 0.f), __bfloat162float(W[kMlpW3 + j]), part);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    return part + __bfloat162float(W[kMlpB3]);
}

// Feature row of (site features sf, class stationary pi, class size n) by one warp.
__device__ void mlp_features(const float* sf, const double* pi, int n, float* x) {
    const int lane = threadIdx.x & 31;
    if (lane < kSiteFeat) x[lane] = sf[lane];
    if (lane < kStates) x[kSiteFeat + lane] = (float)pi[lane];
    double dot = (lane < kStates) ? sf[lane] * log(pi[lane]) : 0.0;
    dot = wsum(dot);
    if (lane == 0) {
        x[kSiteFeat + 20] = logf((float)(n > 1 ? n : 1));
        x[kSiteFeat + 21] = (float)dot;
        x[kSiteFeat + 22] = 0.f;
    }
    __syncwarp();
}

// Tempered, +I-mixed site log-likelihood from per-rate values l[r].
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

__global__ void __launch_bounds__(32 * kGibbsWarps) learned_move_kernel(GibbsArgs a,
                                                                        const __nv_bfloat16* mlp,
                                                                        const float* site_feat,
                                                                        int32_t* n_acc, int32_t* n_prop) {
    const Dims& d = a.d;
    const int i = blockIdx.x;
    const GibbsPart gp = a.parts[i];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int K = gp.K;
    double* spec = a.spec + (size_t)i * (a.Kcap + kAux) * kSpecStride;
    double* ex = a.expt + (size_t)i * (a.Kcap + kAux) * d.N * d.R * kStates;
    double* stash = a.stash + ((size_t)i * kGibbsWarps + warp) * d.NI * kRateBlockLearned * 32;
    __shared__ __align__(16) double xch[kGibbsWarps][kRateBlockLearned * kStates];
    const double* logits = a.logits + (size_t)i * (a.Kcap + kAux) * kStates;
    int32_t* assign = a.assign + (size_t)i * d.S;
    const double* base = a.base + (size_t)i * kBase;
    extern __shared__ __align__(16) unsigned char lsm[];
    __nv_bfloat16* W = reinterpret_cast<__nv_bfloat16*>(lsm);              // kMlpParams
    float* xs = reinterpret_cast<float*>(lsm + ((kMlpParams * 2 + 15) & ~15));  // [warps][kMlpIn]
    float* hs = xs + kGibbsWarps * kMlpIn;                                   // [warps][kMlpHid]
    float* score = hs + kGibbsWarps * kMlpHid;                               // [Kcap]
    int* counts = reinterpret_cast<int*>(score + a.Kcap);                   // [Kcap]
    uint8_t* scode = reinterpret_cast<uint8_t*>(counts + a.Kcap);           // [T]
    __shared__ double lrate[2][kMaxRates];
    __shared__ float rev[2];
    __shared__ int s_site, s_a, s_b;
    __shared__ curandStatePhilox4_32_10_t rng_state;
    __shared__ SpecWork work[kAux];
    __shared__ int acc_n, prop_n;

    for (int x = threadIdx.x; x < kMlpParams; x += blockDim.x) W[x] = mlp[x];
    for (int k = threadIdx.x; k < a.Kcap; k += blockDim.x) counts[k] = 0;
    if (threadIdx.x == 0) {
        curand_init(a.seed, (unsigned long long)gp.p, 0ull, &rng_state);
        acc_n = prop_n = 0;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < d.S; x += blockDim.x) atomicAdd(&counts[assign[x]], 1);
    if (warp < kAux)
        for (int k = warp; k < K; k += kAux)
            spectral_decompose_warp_ws(base, logits + (size_t)k * kStates, spec + (size_t)k * kSpecStride,
                                       work[warp]);
    __syncthreads();
    for (int k = 0; k < K; ++k)
        fill_exp(a, i, k, spec + (size_t)k * kSpecStride, ex + (size_t)k * d.N * d.R * kStates);
    __syncthreads();
    for (int it = 0; it < gp.n_iter; ++it) {
        // One site, uniform over all S. A site alone in its class stays put
        // (the move never empties a class), so the site is selected with
        // probability 1/S both ways and the selection cancels from the
        // Metropolis-Hastings ratio: a draw from only the sites that may move
        // would not, since moving a site changes which sites those are.
        if (threadIdx.x == 0) {
            int c = (int)((1.0 - curand_uniform_double(&rng_state)) * d.S);
            c = c < d.S ? c : d.S - 1;
            s_site = counts[assign[c]] >= 2 ? c : -1;
        }
        __syncthreads();
        const int s = s_site;
        if (s < 0) continue;
        for (int c = threadIdx.x; c < d.T; c += blockDim.x) scode[c] = a.codes[(size_t)c * d.S + s];
        const float* sf = site_feat + (size_t)s * kSiteFeat;
        for (int k = warp; k < K; k += kGibbsWarps) {  // forward scores
            mlp_features(sf, spec + (size_t)k * kSpecStride + kSpecPi, counts[k], xs + warp * kMlpIn);
            const float v = mlp_score(W, xs + warp * kMlpIn, hs + warp * kMlpHid);
            if (lane == 0) score[k] = v;
            __syncwarp();
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            float mx = -INFINITY;
            for (int k = 0; k < K; ++k) mx = fmaxf(mx, score[k]);
            double tot = 0.0;
            for (int k = 0; k < K; ++k) tot += exp((double)(score[k] - mx));
            const double draw = tot * curand_uniform_double(&rng_state);
            double run = 0.0;
            int b = K - 1;
            for (int k = 0; k < K; ++k) {
                run += exp((double)(score[k] - mx));
                if (run >= draw) { b = k; break; }
            }
            s_a = assign[s];
            s_b = b;
            prop_n++;
        }
        __syncthreads();
        const int ca = s_a, cb = s_b;
        if (ca == cb) {  // proposing the current class: a no-op, always accepted
            if (threadIdx.x == 0) acc_n++;
            __syncthreads();
            continue;
        }
        // Site likelihoods under the two classes (warps 0..nb-1: a, nb..2nb-1:
        // b, kRateBlockLearned rates each), reverse scores with the updated
        // class sizes (warps 2nb, 2nb+1).
        const int nb = (d.R + kRateBlockLearned - 1) / kRateBlockLearned;
        if (warp < 2 * nb) {
            const int which = warp < nb ? 0 : 1, r0 = (warp % nb) * kRateBlockLearned;
            const int k = which == 0 ? ca : cb;
            site_class_lnl<kRateBlockLearned>(a, i, r0, spec + (size_t)k * kSpecStride,
                                              ex + (size_t)k * d.N * d.R * kStates, stash, scode,
                                              xch[warp], lrate[which] + r0);
        } else if (warp < 2 * nb + 2) {
            const int w = warp - 2 * nb;
            const int k = w == 0 ? ca : cb;
            mlp_features(sf, spec + (size_t)k * kSpecStride + kSpecPi, counts[k] + (w == 0 ? -1 : 1),
                         xs + warp * kMlpIn);
            const float v = mlp_score(W, xs + warp * kMlpIn, hs + warp * kMlpHid);
            if (lane == 0) rev[w] = v;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const double la = site_value(a, gp, s, lrate[0], spec + (size_t)ca * kSpecStride + kSpecPi);
            const double lb = site_value(a, gp, s, lrate[1], spec + (size_t)cb * kSpecStride + kSpecPi);
            float mx = -INFINITY, mx2 = -INFINITY;
            for (int k = 0; k < K; ++k) {
                mx = fmaxf(mx, score[k]);
                mx2 = fmaxf(mx2, k == ca ? rev[0] : (k == cb ? rev[1] : score[k]));
            }
            double z = 0.0, z2 = 0.0;
            for (int k = 0; k < K; ++k) {
                z += exp((double)(score[k] - mx));
                z2 += exp((double)((k == ca ? rev[0] : (k == cb ? rev[1] : score[k])) - mx2));
            }
            const double lq_fwd = (score[cb] - mx) - log(z);
            const double lq_rev = (rev[0] - mx2) - log(z2);
            // CRP prior ratio n_b / (n_a - 1); tempered likelihood ratio.
            const double lr = a.temp * (lb - la) + log((double)counts[cb]) - log((double)(counts[ca] - 1)) +
                              lq_rev - lq_fwd;
            if (log(curand_uniform_double(&rng_state)) <= lr) {
                assign[s] = cb;
                counts[ca]--;
                counts[cb]++;
                acc_n++;
            }
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < K; k += blockDim.x) a.counts[(size_t)i * (a.Kcap + kAux) + k] = counts[k];
    if (threadIdx.x == 0) {
        a.kout[i] = K;
        n_acc[i] = acc_n;
        n_prop[i] = prop_n;
    }
}

}  // namespace

cudaError_t launch_learned_move(GibbsArgs a, const void* mlp, const float* site_feat, int32_t* n_acc,
                                int32_t* n_prop, double* scratch, cudaStream_t st) {
    const Dims& d = a.d;
    a.spec = scratch;
    a.expt = a.spec + (size_t)a.count * (a.Kcap + kAux) * kSpecStride;
    a.stash = a.expt + (size_t)a.count * (a.Kcap + kAux) * d.N * d.R * kStates;
    const size_t smem = ((kMlpParams * 2 + 15) & ~15) +
                        sizeof(float) * (kGibbsWarps * (kMlpIn + kMlpHid) + a.Kcap) + sizeof(int) * a.Kcap +
                        d.T + 16;
    cudaError_t e = cudaFuncSetAttribute(learned_move_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    learned_move_kernel<<<a.count, 32 * kGibbsWarps, smem, st>>>(
        a, static_cast<const __nv_bfloat16*>(mlp), site_feat, n_acc, n_prop);
    return cudaGetLastError();
}

size_t gibbs_scratch_doubles(const Dims& d, int count, int Kcap) {
    const size_t spec = (size_t)count * (Kcap + kAux) * kSpecStride;
    const size_t ex = (size_t)count * (Kcap + kAux) * d.N * d.R * kStates;
    const size_t stash = (size_t)count * kGibbsWarps * d.NI * kRateBlock * 32;
    return spec + ex + stash;
}

int gibbs_aux() { return kAux; }

cudaError_t launch_gibbs(GibbsArgs a, double* scratch, cudaStream_t st) {
    const Dims& d = a.d;
    a.spec = scratch;
    a.expt = a.spec + (size_t)a.count * (a.Kcap + kAux) * kSpecStride;
    a.stash = a.expt + (size_t)a.count * (a.Kcap + kAux) * d.N * d.R * kStates;
    const size_t smem = sizeof(double) * (size_t)(a.Kcap + kAux) * (d.R + 1) +
                        sizeof(int) * (a.Kcap + kAux) + d.T + 16;
    cudaError_t e = cudaFuncSetAttribute(gibbs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    gibbs_kernel<<<a.count, 32 * kGibbsWarps, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace smccat
