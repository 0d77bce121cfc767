// Training of the learned CAT class proposal (hand-written FP32 kernels).
//
// Training pairs come from the particles' current class assignments -- the
// samples that plain Gibbs reassignment (Neal's Algorithm 8) leaves behind
// during warm-up: for every (particle, site), the features of the site paired
// with each of the particle's classes, and the index of the class the site is
// in. The loss is the mean softmax cross-entropy over sites. Forward and
// backward passes are tiled FP32 GEMMs with fused bias + ReLU; the optimiser
// is Adam. After training the weights are also kept as BF16 for inference
// (the proposal kernel in gibbs.cu).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include "engine_internal.h"
#include "learned.h"
#include "smccat.h"

namespace smccat {
namespace {

int lfail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

struct Learned {
    float* params = nullptr;          // [kMlpParams]
    float* m = nullptr;               // Adam moments
    float* v = nullptr;
    __nv_bfloat16* params_bf16 = nullptr;
    float* site_feat = nullptr;       // [S][kSiteFeat]
    std::vector<float> site_feat_h;
    long step = 0;
    bool trained = false;
};

std::unordered_map<const smccat_ctx*, Learned>& learned_map() {
    static std::unordered_map<const smccat_ctx*, Learned> m;
    return m;
}
std::mutex& learned_mu() {
    static std::mutex mu;
    return mu;
}

constexpr int TILE = 16;

// C[M x N] = op(A)[M x K] . op(B)[K x N] (+ C if accumulate) (+ bias[N]) (ReLU).
// op(A)[i][k] = transA ? A[k * lda + i] : A[i * lda + k]; likewise for B.
__global__ void sgemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda, int transA,
                             const float* __restrict__ B, int ldb, int transB, float* __restrict__ C,
                             int ldc, int accumulate, const float* __restrict__ bias, int relu) {
    __shared__ float As[TILE][TILE + 1], Bs[TILE][TILE + 1];
    const int row = blockIdx.y * TILE + threadIdx.y, col = blockIdx.x * TILE + threadIdx.x;
    float acc = 0.f;
    for (int k0 = 0; k0 < K; k0 += TILE) {
        const int ka = k0 + threadIdx.x, kb = k0 + threadIdx.y;
        As[threadIdx.y][threadIdx.x] =
            (row < M && ka < K) ? (transA ? A[(size_t)ka * lda + row] : A[(size_t)row * lda + ka]) : 0.f;
        Bs[threadIdx.y][threadIdx.x] =
            (kb < K && col < N) ? (transB ? B[(size_t)col * ldb + kb] : B[(size_t)kb * ldb + col]) : 0.f;
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TILE; ++kk) acc = fmaf(As[threadIdx.y][kk], Bs[kk][threadIdx.x], acc);
        __syncthreads();
    }
    if (row < M && col < N) {
        float v = acc;
        if (accumulate) v += C[(size_t)row * ldc + col];
        if (bias) v += bias[col];
        if (relu) v = fmaxf(v, 0.f);
        C[(size_t)row * ldc + col] = v;
    }
}

// One warp per site: softmax over its classes, cross-entropy against the
// label, gradient ds = (p - onehot) / n_groups.
__global__ void softmax_ce_kernel(int n_groups, const int32_t* __restrict__ off,
                                  const int32_t* __restrict__ label, const float* __restrict__ s,
                                  float* __restrict__ ds, float* __restrict__ loss) {
    const int g = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (g >= n_groups) return;
    const int a = off[g], b = off[g + 1];
    float mx = -INFINITY;
    for (int i = a + lane; i < b; i += 32) mx = fmaxf(mx, s[i]);
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    float se = 0.f;
    for (int i = a + lane; i < b; i += 32) se += expf(s[i] - mx);
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    const float inv = 1.f / n_groups;
    for (int i = a + lane; i < b; i += 32) {
        const float p = expf(s[i] - mx) / se;
        ds[i] = (p - (i - a == label[g] ? 1.f : 0.f)) * inv;
    }
    if (lane == 0) loss[g] = -(s[a + label[g]] - mx - logf(se));
}

__global__ void relu_mask_kernel(size_t n, float* __restrict__ d, const float* __restrict__ h) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(h[i] > 0.f)) d[i] = 0.f;
}

// out[j] = sum_i A[i][j] (fixed order per column).
__global__ void colsum_kernel(int M, int N, const float* __restrict__ A, float* __restrict__ out) {
    __shared__ float sh[256];
    const int j = blockIdx.x;
    float s = 0.f;
    for (int i = threadIdx.x; i < M; i += blockDim.x) s += A[(size_t)i * N + j];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = sh[0];
}

__global__ void adam_kernel(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    m[i] = b1 * m[i] + (1.f - b1) * g[i];
    v[i] = b2 * v[i] + (1.f - b2) * g[i] * g[i];
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

__global__ void to_bf16_kernel(int n, const float* __restrict__ a, __nv_bfloat16* __restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}

cudaError_t gemm(cudaStream_t st, int M, int N, int K, const float* A, int lda, int tA, const float* B,
                 int ldb, int tB, float* C, int ldc, int acc, const float* bias, int relu) {
    dim3 blk(TILE, TILE), grd((N + TILE - 1) / TILE, (M + TILE - 1) / TILE);
    sgemm_kernel<<<grd, blk, 0, st>>>(M, N, K, A, lda, tA, B, ldb, tB, C, ldc, acc, bias, relu);
    return cudaGetLastError();
}

// Forward + backward of one batch; grads (kMlpParams) are overwritten.
// Work buffers: X [M][kMlpIn] (device), H1, H2, dH [M][kMlpHid], s, ds [M].
struct Batch {
    int M = 0, G = 0;
    float* X; float* H1; float* H2; float* dH1; float* dH2; float* s; float* ds; float* loss;
    int32_t* off; int32_t* label;
};

cudaError_t fwd_bwd(cudaStream_t st, const float* P, float* grad, const Batch& b) {
    cudaError_t e;
    const int M = b.M, H = kMlpHid;
    if ((e = gemm(st, M, H, kMlpIn, b.X, kMlpIn, 0, P + kMlpW1, H, 0, b.H1, H, 0, P + kMlpB1, 1))) return e;
    if ((e = gemm(st, M, H, H, b.H1, H, 0, P + kMlpW2, H, 0, b.H2, H, 0, P + kMlpB2, 1))) return e;
    if ((e = gemm(st, M, 1, H, b.H2, H, 0, P + kMlpW3, 1, 0, b.s, 1, 0, P + kMlpB3, 0))) return e;
    softmax_ce_kernel<<<(b.G + 7) / 8, 256, 0, st>>>(b.G, b.off, b.label, b.s, b.ds, b.loss);
    // w3, b3
    if ((e = gemm(st, H, 1, M, b.H2, H, 1, b.ds, 1, 0, grad + kMlpW3, 1, 0, nullptr, 0))) return e;
    colsum_kernel<<<1, 256, 0, st>>>(M, 1, b.ds, grad + kMlpB3);
    // dH2 = ds w3^T masked
    if ((e = gemm(st, M, H, 1, b.ds, 1, 0, P + kMlpW3, H, 0, b.dH2, H, 0, nullptr, 0))) return e;
    relu_mask_kernel<<<(unsigned)(((size_t)M * H + 255) / 256), 256, 0, st>>>((size_t)M * H, b.dH2, b.H2);
    if ((e = gemm(st, H, H, M, b.H1, H, 1, b.dH2, H, 0, grad + kMlpW2, H, 0, nullptr, 0))) return e;
    colsum_kernel<<<H, 256, 0, st>>>(M, H, b.dH2, grad + kMlpB2);
    // dH1 = dH2 W2^T masked
    if ((e = gemm(st, M, H, H, b.dH2, H, 0, P + kMlpW2, H, 1, b.dH1, H, 0, nullptr, 0))) return e;
    relu_mask_kernel<<<(unsigned)(((size_t)M * H + 255) / 256), 256, 0, st>>>((size_t)M * H, b.dH1, b.H1);
    if ((e = gemm(st, kMlpIn, H, M, b.X, kMlpIn, 1, b.dH1, H, 0, grad + kMlpW1, H, 0, nullptr, 0))) return e;
    colsum_kernel<<<H, 256, 0, st>>>(M, H, b.dH1, grad + kMlpB1);
    return cudaGetLastError();
}

// Residue composition of every column (host).
std::vector<float> site_features(const smccat_ctx* c) {
    const Dims& d = dims_of(c);
    const uint8_t* codes = codes_host(c);
    std::vector<float> f((size_t)d.S * kSiteFeat, 0.f);
    for (int s = 0; s < d.S; ++s) {
        int n = 0;
        for (int t = 0; t < d.T; ++t) {
            const int x = codes[(size_t)t * d.S + s];
            if (x < 20) { f[(size_t)s * kSiteFeat + x] += 1.f; ++n; }
        }
        for (int i = 0; i < 20; ++i) f[(size_t)s * kSiteFeat + i] /= std::max(n, 1);
        f[(size_t)s * kSiteFeat + 20] = 1.f - (float)n / d.T;
    }
    return f;
}

Learned& learned_state(smccat_ctx* c, int* rc) {
    std::lock_guard<std::mutex> lk(learned_mu());
    Learned& L = learned_map()[c];
    *rc = SMCCAT_OK;
    if (!L.params) {
        const Dims& d = dims_of(c);
        cudaError_t e = cudaMalloc(&L.params, sizeof(float) * kMlpParams);
        if (e == cudaSuccess) e = cudaMalloc(&L.m, sizeof(float) * kMlpParams);
        if (e == cudaSuccess) e = cudaMalloc(&L.v, sizeof(float) * kMlpParams);
        if (e == cudaSuccess) e = cudaMalloc(&L.params_bf16, sizeof(__nv_bfloat16) * kMlpParams);
        if (e == cudaSuccess) e = cudaMalloc(&L.site_feat, sizeof(float) * (size_t)d.S * kSiteFeat);
        if (e != cudaSuccess) { *rc = lfail(SMCCAT_ENOMEM, cudaGetErrorString(e)); return L; }
        L.site_feat_h = site_features(c);
        e = cudaMemcpy(L.site_feat, L.site_feat_h.data(), sizeof(float) * L.site_feat_h.size(),
                       cudaMemcpyHostToDevice);
        if (e != cudaSuccess) *rc = lfail(SMCCAT_ECUDA, cudaGetErrorString(e));
    }
    return L;
}

// Feature row of (site s, class with stationary pi and size n) into x.
void feature_row(const float* sf, const double* pi, int n, float* x) {
    std::memcpy(x, sf, sizeof(float) * kSiteFeat);
    double dot = 0.0;
    for (int i = 0; i < 20; ++i) {
        x[kSiteFeat + i] = (float)pi[i];
        dot += sf[i] * std::log(pi[i]);
    }
    x[kSiteFeat + 20] = (float)std::log((double)std::max(n, 1));
    x[kSiteFeat + 21] = (float)dot;
    x[kSiteFeat + 22] = 0.f;
}

void softmax20d(const double* lg, double* pi) {
    double t = 0.0;
    for (int i = 0; i < 20; ++i) { pi[i] = std::exp(lg[i]); t += pi[i]; }
    for (int i = 0; i < 20; ++i) pi[i] /= t;
}

}  // namespace

void learned_release(const smccat_ctx* c) {
    std::lock_guard<std::mutex> lk(learned_mu());
    auto it = learned_map().find(c);
    if (it == learned_map().end()) return;
    Learned& L = it->second;
    void* ps[] = {L.params, L.m, L.v, L.params_bf16, L.site_feat};
    for (void* p : ps) if (p) cudaFree(p);
    learned_map().erase(it);
}

const void* learned_inference_weights(const smccat_ctx* c, const float** site_feat) {
    std::lock_guard<std::mutex> lk(learned_mu());
    auto it = learned_map().find(c);
    if (it == learned_map().end() || !it->second.trained) return nullptr;
    *site_feat = it->second.site_feat;
    return it->second.params_bf16;
}

}  // namespace smccat

using namespace smccat;

extern "C" {

int smccat_learned_params(smccat_ctx* c, float* get_out, const float* set_in) {
    if (!c) return lfail(SMCCAT_EINVAL, "null context");
    int rc;
    Learned& L = learned_state(c, &rc);
    if (rc) return rc;
    if (set_in) {
        cudaError_t e = cudaMemcpy(L.params, set_in, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(L.m, 0, sizeof(float) * kMlpParams);
        if (e == cudaSuccess) e = cudaMemset(L.v, 0, sizeof(float) * kMlpParams);
        if (e != cudaSuccess) return lfail(SMCCAT_ECUDA, cudaGetErrorString(e));
        to_bf16_kernel<<<(kMlpParams + 255) / 256, 256>>>(kMlpParams, L.params, L.params_bf16);
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return lfail(SMCCAT_ECUDA, cudaGetErrorString(e));
        L.step = 0;
        L.trained = true;
    }
    if (get_out) {
        cudaError_t e = cudaMemcpy(get_out, L.params, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return lfail(SMCCAT_ECUDA, cudaGetErrorString(e));
    }
    return SMCCAT_OK;
}

int smccat_learned_gradients(smccat_ctx* c, int32_t n_sites, const int32_t* group_off,
                             const float* x, const int32_t* labels, float* grad_out,
                             double* loss_out) {
    if (!c || n_sites < 1 || !group_off || !x || !labels || !grad_out)
        return lfail(SMCCAT_EINVAL, "bad argument");
    int rc;
    Learned& L = learned_state(c, &rc);
    if (rc) return rc;
    const int M = group_off[n_sites];
    void* stv;
    smccat_get_stream(c, &stv);
    cudaStream_t st = static_cast<cudaStream_t>(stv);
    const size_t H = kMlpHid;
    size_t bytes = sizeof(float) * ((size_t)M * (kMlpIn + 4 * H + 2) + n_sites + kMlpParams) +
                   sizeof(int32_t) * (2 * (size_t)n_sites + 1) + 1024;
    char* buf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&buf, bytes, st);
    if (e != cudaSuccess) return lfail(SMCCAT_ENOMEM, cudaGetErrorString(e));
    Batch b;
    b.M = M;
    b.G = n_sites;
    float* f = reinterpret_cast<float*>(buf);
    b.X = f; f += (size_t)M * kMlpIn;
    b.H1 = f; f += (size_t)M * H;
    b.H2 = f; f += (size_t)M * H;
    b.dH1 = f; f += (size_t)M * H;
    b.dH2 = f; f += (size_t)M * H;
    b.s = f; f += M;
    b.ds = f; f += M;
    b.loss = f; f += n_sites;
    float* grad = f; f += kMlpParams;
    b.off = reinterpret_cast<int32_t*>(f);
    b.label = b.off + n_sites + 1;
    e = cudaMemcpyAsync(b.X, x, sizeof(float) * (size_t)M * kMlpIn, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b.off, group_off, sizeof(int32_t) * (n_sites + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b.label, labels, sizeof(int32_t) * n_sites, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = fwd_bwd(st, L.params, grad, b);
    std::vector<float> loss(n_sites);
    if (e == cudaSuccess) e = cudaMemcpyAsync(grad_out, grad, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(loss.data(), b.loss, sizeof(float) * n_sites, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(buf, st);
    if (e != cudaSuccess) return lfail(SMCCAT_ECUDA, cudaGetErrorString(e));
    if (loss_out) {
        double t = 0.0;
        for (float v : loss) t += v;
        *loss_out = t / n_sites;
    }
    return SMCCAT_OK;
}

int smccat_learned_train(smccat_ctx* c, int32_t first, int32_t count, int32_t epochs,
                         int32_t batch_sites, double lr, uint64_t seed, double* loss_out) {
    NvtxRange range("smccat_learned_train");
    if (!c || first < 0 || count < 1 || epochs < 0 || batch_sites < 1)
        return lfail(SMCCAT_EINVAL, "bad argument");
    if (!(model_flags_of(c) & SMCCAT_MODEL_CAT)) return lfail(SMCCAT_EINVAL, "the learned proposal needs SMCCAT_MODEL_CAT");
    int rc;
    Learned& L = learned_state(c, &rc);
    if (rc) return rc;
    const Dims& d = dims_of(c);
    std::mt19937_64 g(seed);
    if (!L.trained) {  // Glorot-uniform initialisation
        std::vector<float> p(kMlpParams, 0.f);
        auto fill = [&](int off, int fan_in, int fan_out) {
            const float a = std::sqrt(6.f / (fan_in + fan_out));
            std::uniform_real_distribution<float> u(-a, a);
            for (int i = 0; i < fan_in * fan_out; ++i) p[off + i] = u(g);
        };
        fill(kMlpW1, kMlpIn, kMlpHid);
        fill(kMlpW2, kMlpHid, kMlpHid);
        fill(kMlpW3, kMlpHid, 1);
        rc = smccat_learned_params(c, nullptr, p.data());
        if (rc) return rc;
    }
    // Training pairs of the particles' current assignments.
    struct Item { int p, s; };
    std::vector<Item> items;
    std::vector<std::vector<double>> pis(count);
    std::vector<std::vector<int>> cnts(count);
    for (int i = 0; i < count; ++i) {
        const Slot& s = slot_of(c, first + i);
        if (!s.loaded) return lfail(SMCCAT_ESTATE, "particle has no state loaded");
        const int K = s.cur.K;
        pis[i].resize((size_t)K * 20);
        for (int k = 0; k < K; ++k) softmax20d(&s.cur.logits[(size_t)k * 20], &pis[i][(size_t)k * 20]);
        cnts[i].assign(K, 0);
        for (int v : s.assign) cnts[i][v]++;
        for (int x = 0; x < d.S; ++x) items.push_back({i, x});
    }
    void* stv;
    smccat_get_stream(c, &stv);
    cudaStream_t st = static_cast<cudaStream_t>(stv);
    const int maxM = batch_sites * d.Kmax;
    const size_t H = kMlpHid;
    size_t bytes = sizeof(float) * ((size_t)maxM * (kMlpIn + 4 * H + 2) + batch_sites + kMlpParams) +
                   sizeof(int32_t) * (2 * (size_t)batch_sites + 1) + 1024;
    char* buf = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&buf, bytes, st);
    if (e != cudaSuccess) return lfail(SMCCAT_ENOMEM, cudaGetErrorString(e));
    Batch b;
    float* f = reinterpret_cast<float*>(buf);
    b.X = f; f += (size_t)maxM * kMlpIn;
    b.H1 = f; f += (size_t)maxM * H;
    b.H2 = f; f += (size_t)maxM * H;
    b.dH1 = f; f += (size_t)maxM * H;
    b.dH2 = f; f += (size_t)maxM * H;
    b.s = f; f += maxM;
    b.ds = f; f += maxM;
    b.loss = f; f += batch_sites;
    float* grad = f; f += kMlpParams;
    b.off = reinterpret_cast<int32_t*>(f);
    b.label = b.off + batch_sites + 1;
    std::vector<float> X((size_t)maxM * kMlpIn), lossv(batch_sites);
    std::vector<int32_t> off(batch_sites + 1), lab(batch_sites);
    double last_loss = 0.0;
    for (int ep = 0; ep < epochs && e == cudaSuccess; ++ep) {
        std::shuffle(items.begin(), items.end(), g);
        double ep_loss = 0.0;
        size_t ep_sites = 0;
        for (size_t i0 = 0; i0 < items.size() && e == cudaSuccess; i0 += batch_sites) {
            const int G = (int)std::min<size_t>(batch_sites, items.size() - i0);
            int M = 0;
            for (int gi = 0; gi < G; ++gi) {
                const Item& it = items[i0 + gi];
                const Slot& s = slot_of(c, first + it.p);
                off[gi] = M;
                lab[gi] = s.assign[it.s];
                const float* sf = &L.site_feat_h[(size_t)it.s * kSiteFeat];
                for (int k = 0; k < s.cur.K; ++k, ++M)
                    feature_row(sf, &pis[it.p][(size_t)k * 20], cnts[it.p][k], &X[(size_t)M * kMlpIn]);
            }
            off[G] = M;
            b.M = M;
            b.G = G;
            e = cudaMemcpyAsync(b.X, X.data(), sizeof(float) * (size_t)M * kMlpIn, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(b.off, off.data(), sizeof(int32_t) * (G + 1), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(b.label, lab.data(), sizeof(int32_t) * G, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = fwd_bwd(st, L.params, grad, b);
            ++L.step;
            const float c1 = 1.f - std::pow(0.9f, (float)L.step), c2 = 1.f - std::pow(0.999f, (float)L.step);
            if (e == cudaSuccess) {
                adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(kMlpParams, L.params, grad, L.m, L.v,
                                                                     (float)lr, c1, c2);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaMemcpyAsync(lossv.data(), b.loss, sizeof(float) * G, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // X is reused by the next batch
            for (int gi = 0; gi < G; ++gi) ep_loss += lossv[gi];
            ep_sites += G;
        }
        last_loss = ep_loss / std::max<size_t>(ep_sites, 1);
    }
    if (e == cudaSuccess) {
        to_bf16_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(kMlpParams, L.params, L.params_bf16);
        e = cudaStreamSynchronize(st);
    }
    cudaFreeAsync(buf, st);
    if (e != cudaSuccess) return lfail(SMCCAT_ECUDA, cudaGetErrorString(e));
    L.trained = true;
    if (loss_out) *loss_out = last_loss;
    return SMCCAT_OK;
}

}  // extern "C"
