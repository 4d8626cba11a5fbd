// Learned block-size / variant selector: a 3-layer FP32 MLP (F -> 64 -> 64 -> K,
// ReLU) scoring K candidate configurations, trained on autotuner timings.
//
// Parameter layout (flat, FP32): W1 (F x H, row-major), b1 (H), W2 (H x H),
// b2 (H), W3 (H x K), b3 (K).  Training is full-batch Adam with the
// masked-softmax cross-entropy against soft targets q, run as ONE kernel
// launch per call: one CTA keeps the weights and their gradients in shared
// memory, sweeps the samples in chunks of 32 (forward, softmax, backward), and
// applies the Adam step per epoch.  Every sum is taken in a fixed order by a
// fixed thread, so results are deterministic.  The selector has no reference
// counterpart; it replaces the hand-picked block policies of
// src/potrf/double_blocked_potrf.cpp:17-20 and the per-case sweeps of
// src/potrf/benchmark/potrf_double_blocked_cases.cpp.
#include <cmath>

#include "hdbf/selector.h"
#include "internal.h"

namespace hdbf {
namespace {

constexpr int H = HDBF_SELECTOR_HIDDEN;
constexpr int kS = 32;       // samples per chunk
constexpr int kThreads = 256;

struct Dims {
    int F, K;
    int oW1, ob1, oW2, ob2, oW3, ob3, P;
};

__host__ __device__ inline Dims dims(int F, int K)
{
    Dims d;
    d.F = F;
    d.K = K;
    d.oW1 = 0;
    d.ob1 = F * H;
    d.oW2 = d.ob1 + H;
    d.ob2 = d.oW2 + H * H;
    d.oW3 = d.ob2 + H;
    d.ob3 = d.oW3 + H * K;
    d.P = d.ob3 + K;
    return d;
}

__device__ __forceinline__ unsigned long long splitmix(unsigned long long x)
{
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

// Glorot-uniform weights from the counter-based U[-1,1) stream, zero biases.
__global__ void selector_init_kernel(float* theta, int F, int K, unsigned long long seed)
{
    const Dims d = dims(F, K);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.P) return;
    const unsigned long long h =
        splitmix(seed * 0x9E3779B97F4A7C15ull + (unsigned long long)(i + 1) * 0xD1B54A32D192ED03ull);
    const float u = (float)((double)(h >> 40) / (double)(1u << 23) - 1.0);
    float s;
    if (i < d.ob1) s = sqrtf(6.0f / (float)(F + H));
    else if (i < d.oW2) s = 0.f;
    else if (i < d.ob2) s = sqrtf(6.0f / (float)(H + H));
    else if (i < d.oW3) s = 0.f;
    else if (i < d.ob3) s = sqrtf(6.0f / (float)(H + K));
    else s = 0.f;
    theta[i] = s == 0.f ? 0.f : u * s;
}

__global__ void __launch_bounds__(kThreads) selector_train_kernel(
    float* __restrict__ theta, float* __restrict__ adam_m, float* __restrict__ adam_v, int step0,
    const float* __restrict__ X, const float* __restrict__ Q, const float* __restrict__ mask, int N,
    int F, int K, int epochs, float lr, float wd, float* __restrict__ loss_out,
    float* __restrict__ grad_out)
{
    extern __shared__ __align__(16) float sm[];
    const Dims d = dims(F, K);
    float* W = sm;                   // parameters
    float* G = W + d.P;              // gradient accumulators
    float* xs = G + d.P;             // kS x F
    float* h1 = xs + kS * F;         // kS x H
    float* h2 = h1 + kS * H;         // kS x H
    float* dz = h2 + kS * H;         // kS x K (logits, then dL/dz)
    float* dh2 = dz + kS * K;        // kS x H
    float* dh1 = dh2 + kS * H;       // kS x H
    float* lossv = dh1 + kS * H;     // kS per-slot loss sums
    const int tid = threadIdx.x;
    const float invN = 1.0f / (float)N;

    for (int i = tid; i < d.P; i += kThreads) W[i] = theta[i];
    __syncthreads();
    const int rounds = epochs > 0 ? epochs : 1;
    for (int e = 0; e < rounds; ++e) {
        for (int i = tid; i < d.P; i += kThreads) G[i] = 0.f;
        if (tid < kS) lossv[tid] = 0.f;
        __syncthreads();
        for (int c0 = 0; c0 < N; c0 += kS) {
            const int cs = min(kS, N - c0);
            for (int i = tid; i < kS * F; i += kThreads) {
                const int s = i / F;
                xs[i] = s < cs ? X[(long long)(c0 + s) * F + (i - s * F)] : 0.f;
            }
            __syncthreads();
            for (int i = tid; i < kS * H; i += kThreads) {
                const int s = i / H, j = i - s * H;
                float a = W[d.ob1 + j];
                for (int f = 0; f < F; ++f) a = fmaf(xs[s * F + f], W[d.oW1 + f * H + j], a);
                h1[i] = (s < cs && a > 0.f) ? a : 0.f;
            }
            __syncthreads();
            for (int i = tid; i < kS * H; i += kThreads) {
                const int s = i / H, j = i - s * H;
                float a = W[d.ob2 + j];
#pragma unroll 8
                for (int q = 0; q < H; ++q) a = fmaf(h1[s * H + q], W[d.oW2 + q * H + j], a);
                h2[i] = (s < cs && a > 0.f) ? a : 0.f;
            }
            __syncthreads();
            for (int i = tid; i < kS * K; i += kThreads) {
                const int s = i / K, k = i - s * K;
                float a = W[d.ob3 + k];
#pragma unroll 8
                for (int q = 0; q < H; ++q) a = fmaf(h2[s * H + q], W[d.oW3 + q * K + k], a);
                dz[i] = a;
            }
            __syncthreads();
            if (tid < kS) {
                const int s = tid;
                float* z = dz + s * K;
                if (s < cs) {
                    const float* qs = Q + (long long)(c0 + s) * K;
                    const float* ms = mask + (long long)(c0 + s) * K;
                    float zmax = -INFINITY;
                    for (int k = 0; k < K; ++k)
                        if (ms[k] > 0.f) zmax = fmaxf(zmax, z[k]);
                    float den = 0.f;
                    for (int k = 0; k < K; ++k)
                        if (ms[k] > 0.f) den += expf(z[k] - zmax);
                    const float lden = logf(den);
                    float l = 0.f;
                    for (int k = 0; k < K; ++k) {
                        if (ms[k] > 0.f) {
                            const float lp = z[k] - zmax - lden;
                            l -= qs[k] * lp;
                            z[k] = (expf(lp) - qs[k]) * invN;
                        } else {
                            z[k] = 0.f;
                        }
                    }
                    lossv[s] += l;
                } else {
                    for (int k = 0; k < K; ++k) z[k] = 0.f;
                }
            }
            __syncthreads();
            // layer 3 gradients and dh2
            for (int i = tid; i < H * K; i += kThreads) {
                const int j = i / K, k = i - j * K;
                float a = G[d.oW3 + i];
                for (int s = 0; s < kS; ++s) a = fmaf(h2[s * H + j], dz[s * K + k], a);
                G[d.oW3 + i] = a;
            }
            for (int k = tid; k < K; k += kThreads) {
                float a = G[d.ob3 + k];
                for (int s = 0; s < kS; ++s) a += dz[s * K + k];
                G[d.ob3 + k] = a;
            }
            for (int i = tid; i < kS * H; i += kThreads) {
                const int s = i / H, j = i - s * H;
                float a = 0.f;
                for (int k = 0; k < K; ++k) a = fmaf(dz[s * K + k], W[d.oW3 + j * K + k], a);
                dh2[i] = h2[i] > 0.f ? a : 0.f;
            }
            __syncthreads();
            // layer 2 gradients and dh1
            for (int i = tid; i < H * H; i += kThreads) {
                const int q = i / H, j = i - q * H;
                float a = G[d.oW2 + i];
                for (int s = 0; s < kS; ++s) a = fmaf(h1[s * H + q], dh2[s * H + j], a);
                G[d.oW2 + i] = a;
            }
            for (int j = tid; j < H; j += kThreads) {
                float a = G[d.ob2 + j];
                for (int s = 0; s < kS; ++s) a += dh2[s * H + j];
                G[d.ob2 + j] = a;
            }
            for (int i = tid; i < kS * H; i += kThreads) {
                const int s = i / H, q = i - s * H;
                // rotated start: consecutive q hit distinct banks of W2
                float a = 0.f;
#pragma unroll 8
                for (int jj = 0; jj < H; ++jj) {
                    const int j = (jj + q) & (H - 1);
                    a = fmaf(dh2[s * H + j], W[d.oW2 + q * H + j], a);
                }
                dh1[i] = h1[i] > 0.f ? a : 0.f;
            }
            __syncthreads();
            // layer 1 gradients
            for (int i = tid; i < F * H; i += kThreads) {
                const int f = i / H, q = i - f * H;
                float a = G[d.oW1 + i];
                for (int s = 0; s < kS; ++s) a = fmaf(xs[s * F + f], dh1[s * H + q], a);
                G[d.oW1 + i] = a;
            }
            for (int q = tid; q < H; q += kThreads) {
                float a = G[d.ob1 + q];
                for (int s = 0; s < kS; ++s) a += dh1[s * H + q];
                G[d.ob1 + q] = a;
            }
            __syncthreads();
        }
        if (tid == 0) {
            float l = 0.f;
            for (int s = 0; s < kS; ++s) l += lossv[s];
            if (loss_out) loss_out[e] = l * invN;
        }
        if (epochs == 0) {
            if (grad_out)
                for (int i = tid; i < d.P; i += kThreads) grad_out[i] = G[i];
            break;
        }
        const int t = step0 + e + 1;
        const float c1 = 1.0f - powf(0.9f, (float)t);
        const float c2 = 1.0f - powf(0.999f, (float)t);
        for (int i = tid; i < d.P; i += kThreads) {
            const float g = G[i] + wd * W[i];
            const float m = 0.9f * adam_m[i] + 0.1f * g;
            const float v = 0.999f * adam_v[i] + 0.001f * g * g;
            adam_m[i] = m;
            adam_v[i] = v;
            W[i] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
        }
        __syncthreads();
    }
    if (epochs > 0)
        for (int i = tid; i < d.P; i += kThreads) theta[i] = W[i];
}

// One CTA (H threads) per sample: class = argmax of the masked softmax,
// confidence = its probability.
__global__ void __launch_bounds__(H) selector_predict_kernel(const float* __restrict__ theta,
                                                             const float* __restrict__ X,
                                                             const float* __restrict__ mask, int F,
                                                             int K, int* cls, float* conf,
                                                             float* probs)
{
    const Dims d = dims(F, K);
    __shared__ float x[HDBF_SELECTOR_MAX_FEATURES], a1[H], a2[H], z[HDBF_SELECTOR_MAX_CLASSES];
    const int s = blockIdx.x, j = threadIdx.x;
    if (j < F) x[j] = X[(long long)s * F + j];
    __syncthreads();
    float a = theta[d.ob1 + j];
    for (int f = 0; f < F; ++f) a = fmaf(x[f], theta[d.oW1 + f * H + j], a);
    a1[j] = fmaxf(a, 0.f);
    __syncthreads();
    a = theta[d.ob2 + j];
    for (int q = 0; q < H; ++q) a = fmaf(a1[q], theta[d.oW2 + q * H + j], a);
    a2[j] = fmaxf(a, 0.f);
    __syncthreads();
    if (j < K) {
        a = theta[d.ob3 + j];
        for (int q = 0; q < H; ++q) a = fmaf(a2[q], theta[d.oW3 + q * K + j], a);
        z[j] = a;
    }
    __syncthreads();
    if (j == 0) {
        const float* ms = mask + (long long)s * K;
        float zmax = -INFINITY;
        int best = -1;
        for (int k = 0; k < K; ++k)
            if (ms[k] > 0.f && z[k] > zmax) { zmax = z[k]; best = k; }
        float den = 0.f;
        for (int k = 0; k < K; ++k)
            if (ms[k] > 0.f) den += expf(z[k] - zmax);
        if (cls) cls[s] = best;
        if (conf) conf[s] = best >= 0 ? 1.0f / den : 0.f;
        if (probs)
            for (int k = 0; k < K; ++k)
                probs[(long long)s * K + k] = ms[k] > 0.f ? expf(z[k] - zmax) / den : 0.f;
    }
}

size_t train_smem_bytes(int F, int K)
{
    const Dims d = dims(F, K);
    return sizeof(float) * (2 * (size_t)d.P + kS * (size_t)F + 4 * kS * (size_t)H + kS * (size_t)K + kS);
}

bool dims_ok(int F, int K)
{
    return F >= 1 && F <= HDBF_SELECTOR_MAX_FEATURES && K >= 1 && K <= HDBF_SELECTOR_MAX_CLASSES;
}

}  // namespace
}  // namespace hdbf

using namespace hdbf;

extern "C" {

int hdbf_selector_num_params(int num_features, int num_classes)
{
    if (!dims_ok(num_features, num_classes)) return -1;
    return dims(num_features, num_classes).P;
}

hdbf_status hdbf_selector_init(hdbf_handle h, float* theta, int num_features, int num_classes,
                               unsigned long long seed)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (!theta || !dims_ok(num_features, num_classes)) return HDBF_STATUS_INVALID_VALUE;
    const int P = dims(num_features, num_classes).P;
    ProfScope prof(h, kClsSelector, 0.0, 4.0 * P);
    selector_init_kernel<<<(P + 255) / 256, 256, 0, h->stream>>>(theta, num_features, num_classes,
                                                                 seed);
    h->launches++;
    return h->last_status = last_cuda(h);
}

hdbf_status hdbf_selector_train(hdbf_handle h, float* theta, float* adam_m, float* adam_v,
                                int step0, const float* X, const float* Q, const float* mask,
                                int num_samples, int num_features, int num_classes, int epochs,
                                float lr, float weight_decay, float* loss_out, float* grad_out)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (!theta || !X || !Q || !mask || num_samples <= 0 || epochs < 0 || step0 < 0 ||
        !dims_ok(num_features, num_classes))
        return HDBF_STATUS_INVALID_VALUE;
    if (epochs > 0 && (!adam_m || !adam_v)) return HDBF_STATUS_INVALID_VALUE;
    const size_t smem = train_smem_bytes(num_features, num_classes);
    if (smem > h->max_smem_optin) return HDBF_STATUS_NOT_SUPPORTED;
    cudaFuncSetAttribute(selector_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    const Dims d = dims(num_features, num_classes);
    const double per_sample = 6.0 * ((double)num_features * H + H * H + (double)H * num_classes);
    ProfScope prof(h, kClsSelector, per_sample * num_samples * (epochs > 0 ? epochs : 1),
                   4.0 * d.P * 6.0);
    selector_train_kernel<<<1, kThreads, smem, h->stream>>>(
        theta, adam_m, adam_v, step0, X, Q, mask, num_samples, num_features, num_classes, epochs,
        lr, weight_decay, loss_out, grad_out);
    h->launches++;
    return h->last_status = last_cuda(h);
}

hdbf_status hdbf_selector_predict(hdbf_handle h, const float* theta, const float* X,
                                  const float* mask, int num_samples, int num_features,
                                  int num_classes, int* cls, float* conf, float* probs)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (!theta || !X || !mask || num_samples < 0 || !dims_ok(num_features, num_classes))
        return HDBF_STATUS_INVALID_VALUE;
    if (num_samples == 0) return HDBF_STATUS_SUCCESS;
    const double per_sample = 2.0 * ((double)num_features * H + H * H + (double)H * num_classes);
    ProfScope prof(h, kClsSelector, per_sample * num_samples, 0.0);
    selector_predict_kernel<<<num_samples, H, 0, h->stream>>>(theta, X, mask, num_features,
                                                              num_classes, cls, conf, probs);
    h->launches++;
    return h->last_status = last_cuda(h);
}

}  // extern "C"
