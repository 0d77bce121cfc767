// FP64 kernels of the B200 likelihood engine.
//
//   spec_kernel   one warp per (particle, class): softmax of the logits, the
//                 normalised rate matrix Q (TransitionProbabilityClass.cpp:50-75),
//                 and a parallel (round-robin) Jacobi eigendecomposition of the
//                 symmetrised S = D^1/2 Q D^-1/2. Stores lambda, L = D^-1/2 U,
//                 Rm = U^T D^1/2 and pi.
//   pmat_kernel   one CTA per (particle, node): P(t r) = L diag(exp(lambda t r)) Rm
//                 for every class and rate (TransitionProbabilityClass.cpp:83-95),
//                 stored transposed with a 21st row of row sums.
//   prune_kernel  one CTA per (particle, tile of <= 64 same-class sites): walks the
//                 particle's dirty internal nodes in post-order
//                 (Particle.cpp:577-626), child CLs streamed from HBM, P staged in
//                 shared memory, per-(site, rate) power-of-two rescaling, then the
//                 root reduction of the tile (Particle.cpp:634-674) with a
//                 shared-memory log-sum-exp over rates and a warp-shuffle sum.
//   reduce_kernel per particle, sums the tile partials in a fixed order.
#include <cuda_runtime.h>
#include <math.h>

#include "kernels.h"
#include "spectral.cuh"

namespace smccat {


// ---------------------------------------------------------------------------
// Spectral decomposition of one class (one warp).
__global__ void __launch_bounds__(32) spec_kernel(const SpecJob* __restrict__ jobs,
                                                  double* __restrict__ spec, Dims d) {
    const SpecJob* job = jobs + blockIdx.x;
    double* rec = spec + (((size_t)job->p * d.Kmax + job->k) * 2 + job->sws) * kSpecStride;
    spectral_decompose_warp(job->base, job->logits, rec);
}

// ---------------------------------------------------------------------------
// Transition matrices of one node for every class and rate.
__global__ void __launch_bounds__(128) pmat_kernel(const PJob* __restrict__ jobs,
                                                   const PartHdr* __restrict__ hdr, int first,
                                                   const uint8_t* __restrict__ sws,
                                                   const double* __restrict__ spec,
                                                   double* __restrict__ Pm, Dims d) {
    const PJob job = jobs[blockIdx.x];
    const PartHdr* h = hdr + (job.p - first);
    __shared__ double L[kStates][kStates + 1];
    __shared__ double Rm[kStates][kStates + 1];
    __shared__ double ex[kMaxRates][kStates];
    __shared__ double rs[kStates];
    const int tid = threadIdx.x;
    for (int k = 0; k < h->num_classes; ++k) {
        const double* rec =
            spec + (((size_t)job.p * d.Kmax + k) * 2 + sws[(size_t)job.p * d.Kmax + k]) * kSpecStride;
        __syncthreads();
        for (int idx = tid; idx < kStates * kStates; idx += blockDim.x) {
            L[idx / kStates][idx % kStates] = rec[kSpecL + idx];
            Rm[idx / kStates][idx % kStates] = rec[kSpecRm + idx];
        }
        for (int idx = tid; idx < d.R * kStates; idx += blockDim.x) {
            const int r = idx / kStates, m = idx % kStates;
            ex[r][m] = exp(rec[kSpecLam + m] * job.t * h->rates[r]);
        }
        __syncthreads();
        if (tid < kStates) {
            double s = 0.0;
            for (int j = 0; j < kStates; ++j) s += Rm[tid][j];
            rs[tid] = s;
        }
        __syncthreads();
        double* out = Pm + ((((size_t)job.p * d.Kmax + k) * d.N + job.node) * 2 + job.pws) *
                               (size_t)d.R * kPBlock;
        for (int idx = tid; idx < d.R * kPBlock; idx += blockDim.x) {
            const int r = idx / kPBlock, e = idx % kPBlock;
            const int row = e / kStates, i = e % kStates;
            double v = 0.0;
            if (row < kStates) {
#pragma unroll
                for (int m = 0; m < kStates; ++m) v = fma(L[i][m] * ex[r][m], Rm[m][row], v);
            } else {
#pragma unroll
                for (int m = 0; m < kStates; ++m) v = fma(L[i][m] * ex[r][m], rs[m], v);
            }
            out[idx] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Pruning + root reduction of one tile.
template <int R>
__device__ __forceinline__ void child_vector(const PruneArgs& a, const double* __restrict__ Pt,
                                             int child, int wsc, const double* CLp,
                                             size_t node_stride, size_t ws_stride,
                                             size_t j_stride, int col, int site, double* v) {
    if (child < a.d.T) {
        const int code = a.codes[(size_t)child * a.d.S + site];
        const int row = code < kStates ? code : kStates;
#pragma unroll
        for (int i = 0; i < kStates; ++i) v[i] = Pt[row * kStates + i];
    } else {
        const double* x = CLp + (size_t)(child - a.d.T) * node_stride + wsc * ws_stride + col;
#pragma unroll
        for (int i = 0; i < kStates; ++i) v[i] = 0.0;
#pragma unroll
        for (int j = 0; j < kStates; ++j) {
            // Plain load: the child may have been written earlier in this
            // kernel by this same thread, so the read-only path is not safe.
            const double xj = x[j * j_stride];
#pragma unroll
            for (int i = 0; i < kStates; ++i) v[i] = fma(Pt[j * kStates + i], xj, v[i]);
        }
    }
}

template <int R>
__global__ void __launch_bounds__(kTileSites * R, (R <= 4 ? 2 : 1)) prune_kernel(const PruneArgs a) {
    const Dims d = a.d;
    const int tile_id = a.tile_begin + blockIdx.x;
    const Tile tl = a.tiles[tile_id];
    const int p = tl.p;
    const PartHdr* h = a.hdr + (p - a.first);
    if (!h->active) return;  // uniform across the CTA
    const int tid = threadIdx.x;
    const int r = tid / kTileSites, sl = tid % kTileSites;
    const bool valid = sl < tl.nslots;
    const int slot = tl.slot0 + (valid ? sl : 0);
    const int site = a.perm[(size_t)p * d.S + slot];

    extern __shared__ __align__(16) double sP[];  // [2 children][R][21][20]
    __shared__ double red[R][kTileSites];
    __shared__ double wsum[2];

    const size_t j_stride = (size_t)R * d.Spad;
    const size_t ws_stride = (size_t)kStates * j_stride;
    const size_t node_stride = 2 * ws_stride;
    const size_t lws_stride = (size_t)R * d.Spad;
    const double* CLp = a.CL + (size_t)p * d.NI * node_stride;
    double* CLw = a.CL + (size_t)p * d.NI * node_stride;
    double* LSCp = a.LSC + (size_t)p * d.NI * 2 * lws_stride;
    const int col = r * d.Spad + slot;

    double y[kStates];
    double lsc = 0.0;
    const int cnt = h->node_cnt;
    for (int q = 0; q < cnt; ++q) {
        const NodeJob nj = a.nodes[h->node_off + q];
        __syncthreads();
        for (int idx = tid; idx < 2 * R * kPBlock; idx += blockDim.x) {
            const int c = idx / (R * kPBlock);
            const int rem = idx - c * R * kPBlock;
            const int child = c ? nj.c2 : nj.c1;
            const int pws = (nj.ws >> (3 + c)) & 1;
            sP[idx] = a.Pm[((((size_t)p * d.Kmax + tl.k) * d.N + child) * 2 + pws) * (size_t)R * kPBlock + rem];
        }
        __syncthreads();
        if (valid) {
            const int ws1 = (nj.ws >> 1) & 1, ws2 = (nj.ws >> 2) & 1, wso = nj.ws & 1;
            child_vector<R>(a, sP + r * kPBlock, nj.c1, ws1, CLp, node_stride, ws_stride,
                            j_stride, col, site, y);
            double v2[kStates];
            child_vector<R>(a, sP + (R + r) * kPBlock, nj.c2, ws2, CLp, node_stride, ws_stride,
                            j_stride, col, site, v2);
            double mx = 0.0;
#pragma unroll
            for (int i = 0; i < kStates; ++i) { y[i] *= v2[i]; mx = fmax(mx, y[i]); }
            double l = 0.0;
            if (mx > 0.0) {
                int e;
                frexp(mx, &e);
                const double sc = ldexp(1.0, -e);
#pragma unroll
                for (int i = 0; i < kStates; ++i) y[i] *= sc;
                l = e * 0.69314718055994530942;
            } else {
                l = (mx == 0.0) ? -INFINITY : NAN;
            }
            if (nj.c1 >= d.T)
                l += LSCp[(size_t)(nj.c1 - d.T) * 2 * lws_stride + ws1 * lws_stride + col];
            if (nj.c2 >= d.T)
                l += LSCp[(size_t)(nj.c2 - d.T) * 2 * lws_stride + ws2 * lws_stride + col];
            lsc = l;
            double* out = CLw + (size_t)(nj.node - d.T) * node_stride + wso * ws_stride + col;
#pragma unroll
            for (int j = 0; j < kStates; ++j) out[j * j_stride] = y[j];
            LSCp[(size_t)(nj.node - d.T) * 2 * lws_stride + wso * lws_stride + col] = lsc;
        }
    }
    // Root reduction for this tile.
    if (cnt == 0 && valid) {
        const double* x = CLp + (size_t)(h->root - d.T) * node_stride + h->root_ws * ws_stride + col;
#pragma unroll
        for (int j = 0; j < kStates; ++j) y[j] = x[j * j_stride];
        lsc = LSCp[(size_t)(h->root - d.T) * 2 * lws_stride + h->root_ws * lws_stride + col];
    }
    const double* rec =
        a.spec + (((size_t)p * d.Kmax + tl.k) * 2 + a.sws[(size_t)p * d.Kmax + tl.k]) * kSpecStride;
    const double* pi = rec + kSpecPi;
    if (valid) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < kStates; ++i) s = fma(pi[i], y[i], s);
        red[r][sl] = log(s) + lsc;
    }
    __syncthreads();
    double v = 0.0;
    if (r == 0 && valid) {
        double mx = red[0][sl];
#pragma unroll
        for (int rr = 1; rr < R; ++rr) mx = fmax(mx, red[rr][sl]);
        double lse = mx;
        if (mx > -INFINITY) {
            double se = 0.0;
#pragma unroll
            for (int rr = 0; rr < R; ++rr) se += exp(red[rr][sl] - mx);
            lse = mx + log(se);
        }
        // +I mixing, Particle.cpp:667-670, evaluated in log space.
        const double pinv = h->pinv;
        if (pinv > 0.0 && a.isinv[site] != 0) {
            const double la = log1p(-pinv) + lse;
            const double lb = log(pinv * pi[a.invchar[site]]);
            const double m2 = fmax(la, lb);
            v = m2 + log(exp(la - m2) + exp(lb - m2));
        } else {
            v = lse + log1p(-pinv);
        }
        a.site_lnl[(size_t)p * d.S + site] = v;
    }
    if (tid < kTileSites) {
        v = warp_sum(v);
        if ((tid & 31) == 0) wsum[tid >> 5] = v;
    }
    __syncthreads();
    if (tid == 0) a.partial[tile_id] = wsum[0] + wsum[1];
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
    if (mask[i]) lnl_old[p] = lnl[p];
    else lnl[p] = lnl_old[p];
}

// ---------------------------------------------------------------------------
cudaError_t launch_spec(const SpecJob* jobs, int n, double* spec, const Dims& d, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    spec_kernel<<<n, 32, 0, st>>>(jobs, spec, d);
    return cudaGetLastError();
}

cudaError_t launch_pmat(const PJob* jobs, int n, const PartHdr* hdr, int first, const uint8_t* sws,
                        const double* spec, double* Pm, const Dims& d, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    pmat_kernel<<<n, 128, 0, st>>>(jobs, hdr, first, sws, spec, Pm, d);
    return cudaGetLastError();
}

cudaError_t launch_prune(const PruneArgs& a, int ntiles, cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
    const size_t smem = sizeof(double) * 2 * a.d.R * kPBlock;
    switch (a.d.R) {
#define SMCCAT_PRUNE_CASE(RR)                                                              \
        case RR: {                                                                         \
            cudaError_t e = cudaFuncSetAttribute(prune_kernel<RR>,                         \
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                                 (int)smem);                               \
            if (e != cudaSuccess) return e;                                                \
            prune_kernel<RR><<<ntiles, kTileSites * RR, smem, st>>>(a);                    \
            break;                                                                         \
        }
        SMCCAT_PRUNE_CASE(1) SMCCAT_PRUNE_CASE(2) SMCCAT_PRUNE_CASE(3) SMCCAT_PRUNE_CASE(4)
        SMCCAT_PRUNE_CASE(5) SMCCAT_PRUNE_CASE(6) SMCCAT_PRUNE_CASE(7) SMCCAT_PRUNE_CASE(8)
#undef SMCCAT_PRUNE_CASE
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
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
