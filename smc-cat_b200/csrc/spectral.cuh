// Spectral decomposition of one rate-matrix class, shared by the engine's
// spectral kernel and by the stand-alone transition-matrix entry points.
//
// softmax of the logits (TransitionProbabilityClass.cpp:101-109), the
// normalised rate matrix Q (TransitionProbabilityClass.cpp:50-75) and a
// parallel (round-robin ordering) Jacobi eigendecomposition of the symmetrised
// S = D^1/2 Q D^-1/2. The record gets lambda, L = D^-1/2 U, Rm = U^T D^1/2
// and pi, so that P(t) = L diag(exp(lambda t)) Rm.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "smccat_internal.h"

namespace smccat {

static __device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Shared-memory workspace of one decomposing warp.
struct SpecWork {
    double A[kStates][kStates + 1];
    double V[kStates][kStates + 1];
    double pi[kStates], sq[kStates];
    double cs[10], sn[10];
    int pp[10], qq[10];
};

// Run by exactly one full warp with its own workspace `w`; `rec` holds
// kSpecStride doubles.
static __device__ __noinline__ void spectral_decompose_warp_ws(const double* __restrict__ base,
                                                               const double* __restrict__ logits,
                                                               double* __restrict__ rec,
                                                               SpecWork& w) {
    const int lane = threadIdx.x & 31;
    double(&A)[kStates][kStates + 1] = w.A;
    double(&V)[kStates][kStates + 1] = w.V;
    double(&pi)[kStates] = w.pi;
    double(&sq)[kStates] = w.sq;
    double(&cs)[10] = w.cs;
    double(&sn)[10] = w.sn;
    int(&pp)[10] = w.pp;
    int(&qq)[10] = w.qq;

    double e = (lane < kStates) ? exp(logits[lane]) : 0.0;
    const double tot = warp_sum(e);
    if (lane < kStates) { pi[lane] = e / tot; sq[lane] = sqrt(pi[lane]); }
    __syncwarp();
    // Off-diagonal Q(i,j) = exp(b_ij) pi_j; the 190-vector runs over (i, j<i).
    for (int idx = lane; idx < kStates * kStates; idx += 32) {
        const int i = idx / kStates, j = idx % kStates;
        double q = 0.0;
        if (i != j) {
            const int hi = i > j ? i : j, lo = i > j ? j : i;
            q = exp(base[hi * (hi - 1) / 2 + lo]) * pi[j];
        }
        A[i][j] = q;
    }
    __syncwarp();
    double diag = 0.0;
    if (lane < kStates) {
        for (int j = 0; j < kStates; ++j) if (j != lane) diag += A[lane][j];
        diag = -diag;
    }
    const double mean = warp_sum(lane < kStates ? -diag * pi[lane] : 0.0);
    __syncwarp();
    // Symmetrise: S_ij = exp(b_ij) sqrt(pi_i pi_j) / mean (computed once per
    // unordered pair so S is exactly symmetric), S_ii = Q_ii / mean.
    for (int idx = lane; idx < kStates * kStates; idx += 32) {
        const int i = idx / kStates, j = idx % kStates;
        if (i < j) {
            const double s = exp(base[j * (j - 1) / 2 + i]) * sq[i] * sq[j] / mean;
            A[i][j] = s;
            A[j][i] = s;
        }
    }
    if (lane < kStates) A[lane][lane] = diag / mean;
    for (int idx = lane; idx < kStates * kStates; idx += 32)
        V[idx / kStates][idx % kStates] = (idx / kStates == idx % kStates) ? 1.0 : 0.0;
    __syncwarp();

    for (int sweep = 0; sweep < 40; ++sweep) {
        double off = 0.0, dg = 0.0;
        for (int idx = lane; idx < kStates * kStates; idx += 32) {
            const int i = idx / kStates, j = idx % kStates;
            if (i < j) off += A[i][j] * A[i][j];
            else if (i == j) dg += A[i][j] * A[i][j];
        }
        off = warp_sum(off);
        dg = warp_sum(dg);
        if (!(off > 1e-34 * dg)) break;
        for (int round = 0; round < kStates - 1; ++round) {
            if (lane < 10) {
                int x, y;
                if (lane == 0) { x = 0; y = 1 + round; }
                else { x = 1 + (round + lane) % 19; y = 1 + (round - lane + 19) % 19; }
                const int p = x < y ? x : y, q = x < y ? y : x;
                const double apq = A[p][q];
                double c = 1.0, s = 0.0;
                if (apq != 0.0) {
                    const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
                    double t = 1.0 / (fabs(theta) + sqrt(theta * theta + 1.0));
                    if (theta < 0.0) t = -t;
                    c = 1.0 / sqrt(t * t + 1.0);
                    s = t * c;
                }
                pp[lane] = p; qq[lane] = q; cs[lane] = c; sn[lane] = s;
            }
            __syncwarp();
            for (int idx = lane; idx < 10 * kStates; idx += 32) {  // columns
                const int m = idx / kStates, k = idx % kStates;
                const int p = pp[m], q = qq[m];
                const double c = cs[m], s = sn[m];
                const double akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - s * akq;
                A[k][q] = s * akp + c * akq;
            }
            __syncwarp();
            for (int idx = lane; idx < 10 * kStates; idx += 32) {  // rows
                const int m = idx / kStates, k = idx % kStates;
                const int p = pp[m], q = qq[m];
                const double c = cs[m], s = sn[m];
                const double apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - s * aqk;
                A[q][k] = s * apk + c * aqk;
            }
            __syncwarp();
            if (lane < 10 && sn[lane] != 0.0) { A[pp[lane]][qq[lane]] = 0.0; A[qq[lane]][pp[lane]] = 0.0; }
            for (int idx = lane; idx < 10 * kStates; idx += 32) {  // eigenvectors
                const int m = idx / kStates, k = idx % kStates;
                const int p = pp[m], q = qq[m];
                const double c = cs[m], s = sn[m];
                const double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq;
                V[k][q] = s * vkp + c * vkq;
            }
            __syncwarp();
        }
    }
    if (lane < kStates) {
        rec[kSpecLam + lane] = A[lane][lane];
        rec[kSpecPi + lane] = pi[lane];
    }
    for (int idx = lane; idx < kStates * kStates; idx += 32) {
        const int i = idx / kStates, m = idx % kStates;
        rec[kSpecL + i * kStates + m] = V[i][m] / sq[i];   // L[i][m]
        rec[kSpecRm + m * kStates + i] = V[i][m] * sq[i];  // Rm[m][i]
    }
}

// For kernels whose blocks are a single decomposing warp.
static __device__ __forceinline__ void spectral_decompose_warp(const double* __restrict__ base,
                                                               const double* __restrict__ logits,
                                                               double* __restrict__ rec) {
    __shared__ SpecWork w;
    spectral_decompose_warp_ws(base, logits, rec, w);
}

}  // namespace smccat
