// Root units of the deep phase, enumerated, costed and ordered on the device.
//
// Root unit u is position p of top-level frame k (u = frames[k].root + p).
// k_unit_keys gives every unit its scheduling key -- plain: the number of
// later members (size order); learned: the cost model's predicted subtree
// intersections times the tidset length -- a CUB radix sort orders the keys
// (largest first, ties in unit order) and k_fill_queue writes the work queue.
// The same pass can export the cost-model features for tracing.
#pragma once
#include "common.cuh"
#include "k_costmodel.cuh"
#include "k_deep.cuh"

namespace cpm {

// Per top-level frame: pattern id of the class item (its support is the
// singleton's), transactions, threshold.
struct FrameAux {
    uint32_t sa_pid;
    float n_tx, minsup, pad;
};

__device__ __forceinline__ uint32_t frame_of_unit(const DFrame *frames, uint32_t n_frames, uint32_t u) {
    uint32_t lo = 0, hi = n_frames;  // last frame with root <= u
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (frames[mid].root <= u) lo = mid; else hi = mid;
    }
    return lo;
}

// Cost-model features of unit (frame with m members, position p); the member
// supports are the pair patterns' supports.  Same definition as the host's
// unit_features (later siblings sampled down to at most 256).
__device__ void unit_features_dev(float *x, const DFrame &f, const FrameAux &a, uint32_t p,
                                  const uint32_t *mem_pat, const uint32_t *pat_sup) {
    const uint32_t m = f.m, cnt = m - p - 1;
    const double sp = pat_sup[mem_pat[f.mem_off + p]];
    const double sa = pat_sup[a.sa_pid], N = a.n_tx;
    const double inv_n = N > 0 ? 1.0 / N : 0.0;
    const double msp = fmax((double)a.minsup, 0.0);
    const uint32_t step = cnt > 256 ? (cnt + 255) / 256 : 1;
    double hist[4] = {0, 0, 0, 0}, mean = 0, seen = 0, surv = 0;
    for (uint32_t q = p + 1; q < m; q += step) {
        const double r = sa > 0 ? pat_sup[mem_pat[f.mem_off + q]] / sa : 0.0;
        hist[min(3, (int)(r * 4))] += 1;
        mean += r;
        surv += sp * r >= msp ? 1 : 0;
        seen += 1;
    }
    surv *= seen > 0 ? cnt / seen : 0.0;
    x[0] = (float)log1p((double)cnt);
    x[1] = (float)log1p((double)m);
    x[2] = (float)((double)p / m);
    x[3] = (float)(sp * inv_n);
    x[4] = (float)(sa * inv_n);
    x[5] = (float)(msp * inv_n);
    x[6] = (float)log1p(N);
    x[7] = (float)log1p((double)f.stride);
    for (int i = 0; i < 4; ++i) x[8 + i] = (float)(seen > 0 ? hist[i] / seen : 0.0);
    x[12] = (float)(seen > 0 ? mean / seen : 0.0);
    x[13] = (float)(surv / (cnt + 1.0));
    x[14] = (float)log1p(surv);
    x[15] = (float)log1p(surv * surv * sp * inv_n);
}

__global__ void k_unit_keys(const DFrame *__restrict__ frames, uint32_t n_frames, const FrameAux *__restrict__ aux,
                            uint32_t n_units, const uint32_t *__restrict__ mem_pat,
                            const uint32_t *__restrict__ pat_sup, const float *__restrict__ model,
                            float *__restrict__ feat_out, float *__restrict__ key, uint32_t *__restrict__ uid) {
    __shared__ float p[cm::N_PARAMS];
    if (model)
        for (int i = threadIdx.x; i < cm::N_PARAMS; i += blockDim.x) p[i] = model[i];
    __syncthreads();
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_units) return;
    const uint32_t k = frame_of_unit(frames, n_frames, u);
    const DFrame f = frames[k];
    const uint32_t pos = u - f.root;
    const float later = (float)(f.m - pos - 1);
    float kv = later;
    if (model || feat_out) {
        float x[cm::NF];
        unit_features_dev(x, f, aux[k], pos, mem_pat, pat_sup);
        if (feat_out)
            for (int i = 0; i < cm::NF; ++i) feat_out[(uint64_t)u * cm::NF + i] = x[i];
        if (model) kv = expm1f(mlp_eval(p, x)) * (float)f.stride + later;
    }
    key[u] = kv;
    uid[u] = u;
}

__global__ void k_fill_queue(const DFrame *__restrict__ frames, uint32_t n_frames, const uint32_t *__restrict__ order,
                             uint32_t n_units, unsigned long long *__restrict__ queue) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_units) return;
    const uint32_t u = order[i];
    const uint32_t k = frame_of_unit(frames, n_frames, u);
    queue[i] = ((unsigned long long)k << 32) | (u - frames[k].root);
}

}  // namespace cpm
