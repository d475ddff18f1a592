// Pair level: the Gram matrix C[i][j] = |t(f_i) & t(f_j)| of the frequent
// items, thresholded into pair patterns and top-level equivalence classes.
//
// Reference: cuEclat.mine pair batches (cuEclat.py:183-193) count every pair
// of frequent items with count_supports (k = 2); cuApriori's second level
// counts the same candidates (cuApriori.py:473-499).
//
// This file holds the CUDA-core Gram (AND + popcount, 64x64 tiles) used for
// small matrices and as the cross-check of the tensor-core Gram in
// k_gram_tc.cuh, plus the threshold/emit kernels shared by both.
#pragma once
#include "common.cuh"

namespace cpm {

// Upper-triangle tile index -> (ti, tj), ti <= tj, nt tiles per side.
__device__ __forceinline__ void tri_tile(uint32_t t, uint32_t nt, uint32_t &ti, uint32_t &tj) {
    uint32_t i = 0;
    while (t >= nt - i) { t -= nt - i; ++i; }
    ti = i;
    tj = i + t;
}

// C must be zeroed when gridDim.y > 1 (split-K partial sums are added).
__global__ void __launch_bounds__(256) k_gram_simt(const uint64_t *__restrict__ bits, uint64_t stride,
                                                   const uint32_t *__restrict__ freq, uint32_t F,
                                                   uint32_t nt, uint64_t k_chunk,
                                                   uint32_t *__restrict__ C) {
    constexpr int TM = 64, KW = 16;
    __shared__ uint64_t As[KW][TM + 1];
    __shared__ uint64_t Bs[KW][TM + 1];
    uint32_t ti, tj;
    tri_tile(blockIdx.x, nt, ti, tj);
    const uint64_t k_begin = (uint64_t)blockIdx.y * k_chunk;
    const uint64_t k_end = min(stride, k_begin + k_chunk);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    uint32_t acc[4][4] = {};
    for (uint64_t k0 = k_begin; k0 < k_end; k0 += KW) {
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int idx = threadIdx.x + l * 256;
            const int r = idx >> 4, kk = idx & 15;
            const uint32_t gi = ti * TM + r, gj = tj * TM + r;
            const uint64_t k = k0 + kk;
            As[kk][r] = (gi < F && k < k_end) ? __ldg(bits + (uint64_t)freq[gi] * stride + k) : 0ull;
            Bs[kk][r] = (gj < F && k < k_end) ? __ldg(bits + (uint64_t)freq[gj] * stride + k) : 0ull;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KW; ++kk) {
            uint64_t a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { a[i] = As[kk][ty * 4 + i]; b[i] = Bs[kk][tx * 4 + i]; }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += __popcll(a[i] & b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t gi = ti * TM + ty * 4 + i, gj = tj * TM + tx * 4 + j;
            if (gi < gj && gj < F) {
                if (gridDim.y > 1) atomicAdd(C + (uint64_t)gi * F + gj, acc[i][j]);
                else C[(uint64_t)gi * F + gj] = acc[i][j];
            }
        }
}

// cnt[i] = #{ j > i : C[i][j] passes }; one warp per row.
__global__ void k_pair_count(const uint32_t *__restrict__ C, uint32_t F, long long minsup,
                             uint32_t *__restrict__ cnt) {
    const uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (i >= F) return;
    uint32_t c = 0;
    for (uint64_t j = i + 1 + lane; j < F; j += 32) c += (long long)C[i * F + j] >= minsup;
    c = warp_sum_u32(c);
    if (!lane) cnt[i] = c;
}

// Emits pair patterns in (i, j) order and the member tables of the top-level
// classes: member k of row i is pattern (F + off[i] + k) = {f_i, f_j}.
__global__ void k_pair_emit(const uint32_t *__restrict__ C, uint32_t F, long long minsup,
                            const uint32_t *__restrict__ freq, const uint64_t *__restrict__ off,
                            const uint64_t *__restrict__ bits, uint64_t stride,
                            uint32_t *__restrict__ pat_parent, uint32_t *__restrict__ pat_item,
                            uint32_t *__restrict__ pat_sup, uint32_t *__restrict__ mem_pat,
                            uint32_t *__restrict__ mem_item, const uint64_t **__restrict__ mem_bits) {
    const uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (i >= F) return;
    uint64_t pos = off[i];
    for (uint64_t j0 = i + 1; j0 < F; j0 += 32) {
        const uint64_t j = j0 + lane;
        const uint32_t s = j < F ? C[i * F + j] : 0u;
        const bool pass = j < F && (long long)s >= minsup;
        const unsigned bal = __ballot_sync(CPM_FULL, pass);
        if (pass) {
            const uint64_t k = pos + __popc(bal & ((1u << lane) - 1));
            const uint32_t pid = (uint32_t)(F + k);
            const uint32_t item = freq[j];
            pat_parent[pid] = (uint32_t)i;
            pat_item[pid] = item;
            pat_sup[pid] = s;
            mem_pat[k] = pid;
            mem_item[k] = item;
            mem_bits[k] = bits + (uint64_t)item * stride;
        }
        pos += __popc(bal);
    }
}

}  // namespace cpm
