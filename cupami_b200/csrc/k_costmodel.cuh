// Learned cost model for the deep-level scheduler: a one-hidden-layer MLP
// (FP32, 16 features -> 64 ReLU units -> 1) that predicts log(1 + subtree
// intersections) of a root unit (one position of a top-level class) from
// cheap features.  Forward, backward and Adam kernels are written here; the
// scheduler only uses the predictions to order root units, so they never
// change which itemsets are found or their supports.
//
// Parameter vector layout (floats):
//   mu[NF] | inv_sigma[NF] | W1[H][NF] | b1[H] | w2[H] | b2 | y_mu | y_sigma
// Inputs are standardised with (mu, inv_sigma); the network predicts the
// standardised target, which is mapped back with (y_mu, y_sigma).
#pragma once
#include "common.cuh"

namespace cpm {
namespace cm {

constexpr int NF = 16;
constexpr int H = 64;
constexpr int OFF_MU = 0;
constexpr int OFF_IS = OFF_MU + NF;
constexpr int OFF_W1 = OFF_IS + NF;
constexpr int OFF_B1 = OFF_W1 + H * NF;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H;
constexpr int OFF_YMU = OFF_B2 + 1;
constexpr int OFF_YSD = OFF_YMU + 1;
constexpr int N_PARAMS = OFF_YSD + 1;
constexpr int TRAIN_FIRST = OFF_W1;            // trained slice [OFF_W1, OFF_B2]
constexpr int TRAIN_COUNT = OFF_YMU - OFF_W1;  // W1, b1, w2, b2

}  // namespace cm

// Prediction (log-cost space) for one standardised-on-the-fly sample, with
// the parameters already staged in shared memory.
__device__ __forceinline__ float mlp_eval(const float *p, const float *xin) {
    using namespace cm;
    float x[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) x[f] = (xin[f] - p[OFF_MU + f]) * p[OFF_IS + f];
    float out = p[OFF_B2];
    for (int h = 0; h < H; ++h) {
        float a = p[OFF_B1 + h];
#pragma unroll
        for (int f = 0; f < NF; ++f) a += p[OFF_W1 + h * NF + f] * x[f];
        out += p[OFF_W2 + h] * fmaxf(a, 0.f);
    }
    return out * p[OFF_YSD] + p[OFF_YMU];
}

// y[i] = prediction for sample i (standardised space when raw == 0, else
// log-cost space).  One thread per sample, parameters staged in shared memory.
__global__ void k_mlp_forward(const float *__restrict__ params, const float *__restrict__ X, uint64_t n,
                              float *__restrict__ y, int raw) {
    using namespace cm;
    __shared__ float p[N_PARAMS];
    for (int i = threadIdx.x; i < N_PARAMS; i += blockDim.x) p[i] = params[i];
    __syncthreads();
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) x[f] = (X[s * NF + f] - p[OFF_MU + f]) * p[OFF_IS + f];
    float out = p[OFF_B2];
    for (int h = 0; h < H; ++h) {
        float a = p[OFF_B1 + h];
#pragma unroll
        for (int f = 0; f < NF; ++f) a += p[OFF_W1 + h * NF + f] * x[f];
        out += p[OFF_W2 + h] * fmaxf(a, 0.f);
    }
    y[s] = raw ? out * p[OFF_YSD] + p[OFF_YMU] : out;
}

// Gradient of the mean squared error (standardised target t) with respect to
// W1, b1, w2, b2, summed over the samples into grad[TRAIN_COUNT]; *loss gets
// the summed squared error.  One thread per sample; each block reduces in
// shared memory and adds once per parameter.
__global__ void k_mlp_backward(const float *__restrict__ params, const float *__restrict__ X,
                               const float *__restrict__ t, uint64_t n, float *__restrict__ grad,
                               float *__restrict__ loss) {
    using namespace cm;
    __shared__ float p[N_PARAMS];
    __shared__ float g[TRAIN_COUNT];
    __shared__ float l_sum;
    for (int i = threadIdx.x; i < N_PARAMS; i += blockDim.x) p[i] = params[i];
    for (int i = threadIdx.x; i < TRAIN_COUNT; i += blockDim.x) g[i] = 0.f;
    if (threadIdx.x == 0) l_sum = 0.f;
    __syncthreads();
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) {
        float x[NF], a[H];
#pragma unroll
        for (int f = 0; f < NF; ++f) x[f] = (X[s * NF + f] - p[OFF_MU + f]) * p[OFF_IS + f];
        float out = p[OFF_B2];
        for (int h = 0; h < H; ++h) {
            float z = p[OFF_B1 + h];
#pragma unroll
            for (int f = 0; f < NF; ++f) z += p[OFF_W1 + h * NF + f] * x[f];
            a[h] = z;
            out += p[OFF_W2 + h] * fmaxf(z, 0.f);
        }
        const float e = out - t[s];  // d(0.5 e^2)/d out
        atomicAdd(&l_sum, e * e);
        atomicAdd(&g[OFF_B2 - TRAIN_FIRST], e);
        for (int h = 0; h < H; ++h) {
            const float r = fmaxf(a[h], 0.f);
            atomicAdd(&g[OFF_W2 - TRAIN_FIRST + h], e * r);
            if (a[h] > 0.f) {
                const float d = e * p[OFF_W2 + h];
                atomicAdd(&g[OFF_B1 - TRAIN_FIRST + h], d);
#pragma unroll
                for (int f = 0; f < NF; ++f) atomicAdd(&g[OFF_W1 - TRAIN_FIRST + h * NF + f], d * x[f]);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TRAIN_COUNT; i += blockDim.x)
        if (g[i] != 0.f) atomicAdd(grad + i, g[i]);
    if (threadIdx.x == 0) atomicAdd(loss, l_sum);
}

// Adam step on the trained slice: grad holds sums over `n` samples.
__global__ void k_adam(float *__restrict__ params, const float *__restrict__ grad, float *__restrict__ m1,
                       float *__restrict__ m2, float lr, float scale, int step) {
    using namespace cm;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= TRAIN_COUNT) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gi = grad[i] * scale;
    m1[i] = b1 * m1[i] + (1.f - b1) * gi;
    m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
    const float mh = m1[i] / (1.f - powf(b1, (float)step));
    const float vh = m2[i] / (1.f - powf(b2, (float)step));
    params[TRAIN_FIRST + i] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace cpm
