// Training and batch inference of the selector's cost model: a perceptron
// 16 -> 64 (ReLU) -> 64 (ReLU) -> 3 predicting log-microseconds of the LOP3,
// M4R and tensor-core variants of a product term from its features.
//
// Loss over the logged samples (x_n, y_n, m_n), m_nj = 1 where variant j was
// timed:  L = sum_n sum_j m_nj (f(x_n)_j - y_nj)^2 / (2 sum m).
//
// k_mlp_fb: forward and backward for 64 samples per block, one thread per
// sample for the activations, then one thread per weight (strided) for the
// gradient sums over the block's samples, added to the global gradient with
// one atomicAdd per weight and block.  k_adam: Adam step with decoupled weight
// decay, zeroing the gradient.  k_mlp_predict: one warp per sample (the same
// warp routine the selector runs inside the closure).
#include "launch.h"
#include "select_device.cuh"

namespace cfpq {

namespace {

constexpr int F = kSelFeatures, H = kSelHidden, O = kSelOutputs;
constexpr int kSamples = 64;  // samples (= threads) per block
constexpr int kPad = H + 1;

struct MlpSmem {
    float w[kSelWeights];
    float x[kSamples][F];
    float h1[kSamples][kPad], h2[kSamples][kPad];
    float d1[kSamples][kPad], d2[kSamples][kPad];
    float dout[kSamples][O];
    float loss[kSamples / 32];
};

__global__ void __launch_bounds__(kSamples) k_mlp_fb(const float *__restrict__ W, const float *__restrict__ X,
                                                     const float *__restrict__ Y, const float *__restrict__ M,
                                                     uint32_t N, float inv_msum, float *grad, float *loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(smem_raw);
    const uint32_t t = threadIdx.x, s = blockIdx.x * kSamples + t;
    for (int i = t; i < kSelWeights; i += kSamples) S.w[i] = W[i];
    __syncthreads();
    const float *W1 = S.w, *b1 = W1 + F * H, *W2 = b1 + H, *b2 = W2 + H * H, *W3 = b2 + H, *b3 = W3 + H * O;
    const bool valid = s < N;
    float l = 0.f;
#pragma unroll
    for (int i = 0; i < F; ++i) S.x[t][i] = valid ? X[(size_t)s * F + i] : 0.f;
    // forward
    for (int u = 0; u < H; ++u) {
        float a = b1[u];
#pragma unroll
        for (int i = 0; i < F; ++i) a = fmaf(W1[i * H + u], S.x[t][i], a);
        S.h1[t][u] = fmaxf(a, 0.f);
    }
    for (int u = 0; u < H; ++u) {
        float a = b2[u];
        for (int k = 0; k < H; ++k) a = fmaf(W2[k * H + u], S.h1[t][k], a);
        S.h2[t][u] = fmaxf(a, 0.f);
    }
#pragma unroll
    for (int j = 0; j < O; ++j) {
        float a = b3[j];
        for (int u = 0; u < H; ++u) a = fmaf(W3[u * O + j], S.h2[t][u], a);
        const float m = valid ? M[(size_t)s * O + j] : 0.f;
        const float e = valid ? a - Y[(size_t)s * O + j] : 0.f;
        S.dout[t][j] = m * e * inv_msum;
        l += 0.5f * m * e * e * inv_msum;
    }
    // backward through the hidden layers
    for (int u = 0; u < H; ++u) {
        float g = 0.f;
#pragma unroll
        for (int j = 0; j < O; ++j) g = fmaf(W3[u * O + j], S.dout[t][j], g);
        S.d2[t][u] = S.h2[t][u] > 0.f ? g : 0.f;
    }
    for (int k = 0; k < H; ++k) {
        float g = 0.f;
        for (int u = 0; u < H; ++u) g = fmaf(W2[k * H + u], S.d2[t][u], g);
        S.d1[t][k] = S.h1[t][k] > 0.f ? g : 0.f;
    }
    for (int d = 16; d > 0; d >>= 1) l += __shfl_xor_sync(0xffffffffu, l, d);
    if ((t & 31) == 0) S.loss[t >> 5] = l;
    __syncthreads();
    if (t == 0) {
        float bl = 0.f;
        for (int w = 0; w < kSamples / 32; ++w) bl += S.loss[w];
        if (bl != 0.f) atomicAdd(loss, bl);
    }
    // weight gradients: sums over the block's samples
    for (int w = t; w < kSelWeights; w += kSamples) {
        float g = 0.f;
        if (w < F * H) {
            const int i = w / H, u = w % H;
            for (int q = 0; q < kSamples; ++q) g = fmaf(S.x[q][i], S.d1[q][u], g);
        } else if (w < F * H + H) {
            const int u = w - F * H;
            for (int q = 0; q < kSamples; ++q) g += S.d1[q][u];
        } else if (w < F * H + H + H * H) {
            const int r = w - (F * H + H), k = r / H, u = r % H;
            for (int q = 0; q < kSamples; ++q) g = fmaf(S.h1[q][k], S.d2[q][u], g);
        } else if (w < F * H + H + H * H + H) {
            const int u = w - (F * H + H + H * H);
            for (int q = 0; q < kSamples; ++q) g += S.d2[q][u];
        } else if (w < F * H + H + H * H + H + H * O) {
            const int r = w - (F * H + H + H * H + H), u = r / O, j = r % O;
            for (int q = 0; q < kSamples; ++q) g = fmaf(S.h2[q][u], S.dout[q][j], g);
        } else {
            const int j = w - (F * H + H + H * H + H + H * O);
            for (int q = 0; q < kSamples; ++q) g += S.dout[q][j];
        }
        if (g != 0.f) atomicAdd(grad + w, g);
    }
}

__global__ void k_adam(float *W, float *grad, float *m, float *v, uint32_t n, float lr, float beta1, float beta2,
                       float eps, float wd, float c1, float c2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grad[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    W[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * W[i]);
    grad[i] = 0.f;
}

__global__ void k_mlp_predict(const float *__restrict__ W, const float *__restrict__ X, uint32_t N, float *out) {
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= N) return;
    float x[F], p[O];
#pragma unroll
    for (int i = 0; i < F; ++i) x[i] = X[(size_t)s * F + i];
    sel::selector_mlp_warp(W, x, p);
    if ((threadIdx.x & 31) == 0)
        for (int j = 0; j < O; ++j) out[(size_t)s * O + j] = p[j];
}

}  // namespace

cudaError_t mlp_loss_grad(const float *d_w, const float *d_x, const float *d_y, const float *d_m, uint32_t n,
                          float inv_msum, float *d_grad, float *d_loss, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_fb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
    if (e != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    k_mlp_fb<<<(n + kSamples - 1) / kSamples, kSamples, sizeof(MlpSmem), s>>>(d_w, d_x, d_y, d_m, n, inv_msum, d_grad,
                                                                              d_loss);
    return cudaGetLastError();
}

cudaError_t mlp_adam_step(float *d_w, float *d_grad, float *d_m, float *d_v, float lr, float wd, uint32_t step,
                          cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<(kSelWeights + 255) / 256, 256, 0, s>>>(d_w, d_grad, d_m, d_v, kSelWeights, lr, b1, b2, 1e-8f, wd, c1,
                                                     c2);
    return cudaGetLastError();
}

cudaError_t mlp_predict(const float *d_w, const float *d_x, uint32_t n, float *d_out, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_mlp_predict<<<(unsigned)(((size_t)n * 32 + 127) / 128), 128, 0, s>>>(d_w, d_x, n, d_out);
    return cudaGetLastError();
}

}  // namespace cfpq
