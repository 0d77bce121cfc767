// Transition matrices for callers that cannot allocate device memory.
//
// Some hosts of this library may not call cudaMalloc at all: code that runs
// inside another framework's memory budget or custom allocator, or a plugin
// that is only handed pre-allocated buffers and must leave the device heap
// untouched. For them this file offers one entry point
// that computes batched transition matrices P(t) from exchangeabilities and
// stationary logits -- the engine's spectral decomposition followed by
// P(t) = L diag(exp(lambda t)) Rm -- with no allocation of its own. The
// caller passes device buffers for every input and output; the intermediate
// spectral records live in a fixed-size file-scope device array.
//
// The array holds kNoAllocMaxClasses records (3.5 MB). Every GPU on which the
// library's kernels get loaded keeps it until the process exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "smccat.h"
#include "spectral.cuh"

namespace smccat {
namespace {

constexpr int kNoAllocMaxClasses = 512;
constexpr size_t kMaxContexts = 64;

// Scratch for the spectral records of one call. Its contents persist from
// call to call; every record a call reads is written earlier in that call.
static __device__ __align__(256) double g_noalloc_spec[kNoAllocMaxClasses * kSpecStride];

// Device address of g_noalloc_spec per CUDA context (host code must not use
// the symbol itself: on the host it names a stand-in, not device memory). The
// key is the context current at the call, not the device ordinal: a host may
// run this library under a context of its own (not the device's primary one),
// and a context destroyed and re-created (cudaDeviceReset) gets the array at a
// new address. A call outside stream capture resolves the address afresh and
// records it; a call under capture, where resolving could trigger module
// loading, uses the address recorded for its context.
std::vector<std::pair<CUcontext, double*>> g_noalloc_ptr;
std::mutex g_noalloc_mu;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
    });
    return fn;
}

__global__ void __launch_bounds__(32) noalloc_spec_kernel(const double* __restrict__ base,
                                                          const double* __restrict__ logits,
                                                          double* __restrict__ scratch) {
    const int m = blockIdx.x;
    spectral_decompose_warp(base + (size_t)m * kBase, logits + (size_t)m * kStates,
                            scratch + (size_t)m * kSpecStride);
}

// One CTA per (class, time): P[i][j] = sum_m L[i][m] exp(lambda_m t) Rm[m][j].
__global__ void __launch_bounds__(128) noalloc_pmat_kernel(const double* __restrict__ scratch,
                                                           int num_times,
                                                           const double* __restrict__ times,
                                                           double* __restrict__ out) {
    const int m = blockIdx.x / num_times;
    const double* rec = scratch + (size_t)m * kSpecStride;
    const double t = times[blockIdx.x];
    __shared__ double L[kStates][kStates + 1];
    __shared__ double Rm[kStates][kStates + 1];
    __shared__ double ex[kStates];
    for (int idx = threadIdx.x; idx < kStates * kStates; idx += blockDim.x) {
        L[idx / kStates][idx % kStates] = rec[kSpecL + idx];
        Rm[idx / kStates][idx % kStates] = rec[kSpecRm + idx];
    }
    if (threadIdx.x < kStates) ex[threadIdx.x] = exp(rec[kSpecLam + threadIdx.x] * t);
    __syncthreads();
    double* P = out + (size_t)blockIdx.x * kStates * kStates;
    for (int idx = threadIdx.x; idx < kStates * kStates; idx += blockDim.x) {
        const int i = idx / kStates, j = idx % kStates;
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < kStates; ++k) v = fma(L[i][k] * ex[k], Rm[k][j], v);
        P[idx] = v;
    }
}

int noalloc_fail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

}  // namespace
}  // namespace smccat

using namespace smccat;

extern "C" {

int smccat_transition_matrices_noalloc(int32_t num_classes, const double* base,
                                       const double* logits, int32_t num_times,
                                       const double* times, double* p_out, void* stream) {
    if (!base || !logits || !times || !p_out)
        return noalloc_fail(SMCCAT_EINVAL, "null device pointer");
    if (num_classes < 1 || num_classes > kNoAllocMaxClasses)
        return noalloc_fail(SMCCAT_EINVAL, "num_classes must be in [1, " +
                                               std::to_string(kNoAllocMaxClasses) + "], got " +
                                               std::to_string(num_classes));
    if (num_times < 1 || (long long)num_classes * num_times > 0x7fffffffLL)
        return noalloc_fail(SMCCAT_EINVAL, "num_times must be >= 1 and num_classes * num_times < 2^31");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return noalloc_fail(SMCCAT_ECUDA, cudaGetErrorString(e));
    void* fresh = nullptr;
    if (cap == cudaStreamCaptureStatusNone) {
        // Set-up with the caller's context current (the runtime makes the
        // device's primary context current if none is): resolve the device
        // address of the scratch array in this context.
        e = cudaGetSymbolAddress(&fresh, g_noalloc_spec);
        if (e != cudaSuccess || !fresh)
            return noalloc_fail(SMCCAT_ECUDA, std::string("cudaGetSymbolAddress: ") +
                                                  cudaGetErrorString(e));
    }
    CtxGetCurrentFn get_ctx = ctx_get_current();
    CUcontext ctx = nullptr;
    if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS || !ctx)
        return noalloc_fail(SMCCAT_ECUDA, "no current CUDA context");
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        auto it = g_noalloc_ptr.begin();
        while (it != g_noalloc_ptr.end() && it->first != ctx) ++it;
        if (fresh) {
            if (it != g_noalloc_ptr.end()) {
                it->second = static_cast<double*>(fresh);
            } else {
                if (g_noalloc_ptr.size() >= kMaxContexts) g_noalloc_ptr.erase(g_noalloc_ptr.begin());
                g_noalloc_ptr.emplace_back(ctx, static_cast<double*>(fresh));
            }
            scratch = static_cast<double*>(fresh);
        } else {
            if (it == g_noalloc_ptr.end())
                return noalloc_fail(SMCCAT_ESTATE,
                                    "first call in this CUDA context must come before stream capture");
            scratch = it->second;
        }
    }
    // Launch errors are peeked, not cleared: the error state belongs to the host
    // program as much as to this call.
    noalloc_spec_kernel<<<num_classes, 32, 0, st>>>(base, logits, scratch);
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) return noalloc_fail(SMCCAT_ECUDA, cudaGetErrorString(e));
    noalloc_pmat_kernel<<<num_classes * num_times, 128, 0, st>>>(scratch, num_times, times, p_out);
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) return noalloc_fail(SMCCAT_ECUDA, cudaGetErrorString(e));
    return SMCCAT_OK;
}

}  // extern "C"
