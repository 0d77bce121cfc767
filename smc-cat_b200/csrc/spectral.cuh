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

// The symmetrised matrix S of a class into w.A (with w.pi, w.sq).
static __device__ __forceinline__ void spec_build(const double* __restrict__ base,
                                                  const double* __restrict__ logits, SpecWork& w) {
    const int lane = threadIdx.x & 31;
    double(&A)[kStates][kStates + 1] = w.A;
    double(&pi)[kStates] = w.pi;
    double(&sq)[kStates] = w.sq;
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
    __syncwarp();
}

// Round-robin Jacobi rotations on w.A, accumulated into w.V, until the
// off-diagonal mass is below 1e-34 of the diagonal's (at most 40 sweeps).
static __device__ __forceinline__ void spec_jacobi(SpecWork& w) {
    const int lane = threadIdx.x & 31;
    double(&A)[kStates][kStates + 1] = w.A;
    double(&V)[kStates][kStates + 1] = w.V;
    double(&cs)[10] = w.cs;
    double(&sn)[10] = w.sn;
    int(&pp)[10] = w.pp;
    int(&qq)[10] = w.qq;
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
                    // t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)), theta =
                    // (A_qq - A_pp) / (2 A_pq), written with one division.
                    const double dd = A[q][q] - A[p][p];
                    double t = 2.0 * apq / (fabs(dd) + sqrt(dd * dd + 4.0 * apq * apq));
                    if (dd < 0.0) t = -t;
                    c = rsqrt(t * t + 1.0);
                    s = t * c;
                }
                pp[lane] = p; qq[lane] = q; cs[lane] = c; sn[lane] = s;
            }
            __syncwarp();
            // A <- G^T A G block by block: the 10 pairs partition the indices, so
            // each 2 x 2 block (pair m1 rows, pair m2 columns) belongs to one lane.
            // Columns rotate by pair m2, then rows by pair m1; a rotated pair's
            // own off-diagonal entry is set to zero.
            for (int idx = lane; idx < 100; idx += 32) {
                const int m1 = idx / 10, m2 = idx % 10;
                const int p1 = pp[m1], q1 = qq[m1], p2 = pp[m2], q2 = qq[m2];
                const double c1 = cs[m1], s1 = sn[m1], c2 = cs[m2], s2 = sn[m2];
                const double a_pp = A[p1][p2], a_pq = A[p1][q2], a_qp = A[q1][p2], a_qq = A[q1][q2];
                const double b_pp = c2 * a_pp - s2 * a_pq, b_pq = s2 * a_pp + c2 * a_pq;
                const double b_qp = c2 * a_qp - s2 * a_qq, b_qq = s2 * a_qp + c2 * a_qq;
                const bool zero = m1 == m2 && s1 != 0.0;
                A[p1][p2] = c1 * b_pp - s1 * b_qp;
                A[q1][q2] = s1 * b_pq + c1 * b_qq;
                A[p1][q2] = zero ? 0.0 : c1 * b_pq - s1 * b_qq;
                A[q1][p2] = zero ? 0.0 : s1 * b_pp + c1 * b_qp;
            }
            for (int idx = lane; idx < 10 * kStates; idx += 32) {  // eigenvectors, V <- V G
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
}

// The record: lambda, L = D^-1/2 V, Rm = V^T D^1/2 and pi.
static __device__ __forceinline__ void spec_store(const SpecWork& w, double* __restrict__ rec) {
    const int lane = threadIdx.x & 31;
    if (lane < kStates) {
        rec[kSpecLam + lane] = w.A[lane][lane];
        rec[kSpecPi + lane] = w.pi[lane];
    }
    for (int idx = lane; idx < kStates * kStates; idx += 32) {
        const int i = idx / kStates, m = idx % kStates;
        rec[kSpecL + i * kStates + m] = w.V[i][m] / w.sq[i];   // L[i][m]
        rec[kSpecRm + m * kStates + i] = w.V[i][m] * w.sq[i];  // Rm[m][i]
    }
}

// Run by exactly one full warp with its own workspace `w`; `rec` holds
// kSpecStride doubles.
static __device__ __noinline__ void spectral_decompose_warp_ws(const double* __restrict__ base,
                                                               const double* __restrict__ logits,
                                                               double* __restrict__ rec,
                                                               SpecWork& w) {
    const int lane = threadIdx.x & 31;
    spec_build(base, logits, w);
    for (int idx = lane; idx < kStates * kStates; idx += 32)
        w.V[idx / kStates][idx % kStates] = (idx / kStates == idx % kStates) ? 1.0 : 0.0;
    __syncwarp();
    spec_jacobi(w);
    spec_store(w, rec);
}

// The same decomposition started from the eigenvectors of `prev`, the record
// of a nearby class (the class before a proposal changed its frequencies or
// exchangeabilities): with U = D_prev^1/2 L_prev (orthogonal), the rotations
// start from A = U^T S U, nearly diagonal, and V = U, so they converge in a few
// sweeps instead of from the identity. `rec` (not `prev`) doubles as scratch.
static __device__ __noinline__ void spectral_decompose_warp_warm(const double* __restrict__ base,
                                                                 const double* __restrict__ logits,
                                                                 const double* __restrict__ prev,
                                                                 double* __restrict__ rec, SpecWork& w) {
    const int lane = threadIdx.x & 31;
    spec_build(base, logits, w);
    for (int idx = lane; idx < kStates * kStates; idx += 32) {
        const int i = idx / kStates, m = idx % kStates;
        w.V[i][m] = sqrt(prev[kSpecPi + i]) * prev[kSpecL + idx];
    }
    __syncwarp();
    double* B = rec + kSpecL;  // S U, row-major, until the record is written
    for (int idx = lane; idx < kStates * kStates; idx += 32) {
        const int i = idx / kStates, m = idx % kStates;
        double acc = 0.0;
        for (int j = 0; j < kStates; ++j) acc = fma(w.A[i][j], w.V[j][m], acc);
        B[idx] = acc;
    }
    __syncwarp();
    for (int idx = lane; idx < kStates * kStates; idx += 32) {  // U^T (S U), upper triangle
        const int m = idx / kStates, n = idx % kStates;
        if (m > n) continue;
        double acc = 0.0, acc2 = 0.0;
        for (int i = 0; i < kStates; ++i) {
            acc = fma(w.V[i][m], B[i * kStates + n], acc);
            acc2 = fma(w.V[i][n], B[i * kStates + m], acc2);
        }
        const double v = 0.5 * (acc + acc2);  // exactly symmetric
        w.A[m][n] = v;
        w.A[n][m] = v;
    }
    __syncwarp();
    spec_jacobi(w);
    spec_store(w, rec);
}

// For kernels whose blocks are a single decomposing warp.
static __device__ __forceinline__ void spectral_decompose_warp(const double* __restrict__ base,
                                                               const double* __restrict__ logits,
                                                               double* __restrict__ rec) {
    __shared__ SpecWork w;
    spectral_decompose_warp_ws(base, logits, rec, w);
}

}  // namespace smccat
