// Horizontal rows of the frequent items, for the deep kernel's row-wise units.
//
// Row t lists the frequent indices f (0 .. F-1, in increasing order) of the
// items transaction t holds: the transpose of the F frequent tidsets.  A deep
// unit whose prefix holds few transactions and whose siblings are long lists
// counts its children by walking the prefix's rows (k_deep.cuh) instead of
// testing every sibling id; this is the same support, |t(prefix) & t(item)|,
// counted from the other side.  Built once per mine by two passes over the
// frequent tidsets (lengths, then the rows at the scanned offsets).
#pragma once
#include "common.cuh"

namespace cpm {

// One thread per transaction: bit t of frequent tidset f is read with the
// 31 other lanes of its warp from one 64-bit word (a broadcast), eight items
// in flight.  WRITE = false: len[t] = items held; true: the indices at
// rows[off[t] ...].
template <bool WRITE>
__global__ void k_hrows(const uint64_t *__restrict__ bits, uint64_t stride, const uint32_t *__restrict__ freq,
                        uint32_t F, uint64_t n_tx, uint32_t *__restrict__ len, const uint64_t *__restrict__ off,
                        uint16_t *__restrict__ rows) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tx) return;
    const uint64_t w = t >> 6;
    const unsigned b = (unsigned)(t & 63);
    uint32_t n = 0;
    uint64_t at = WRITE ? off[t] : 0ull;
    uint32_t f = 0;
    for (; f + 8 <= F; f += 8) {
        unsigned long long x[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = __ldg(reinterpret_cast<const unsigned long long *>(bits) +
                                                 (uint64_t)__ldg(freq + f + k) * stride + w);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if ((x[k] >> b) & 1ull) {
                if (WRITE) rows[at++] = (uint16_t)(f + k);
                ++n;
            }
    }
    for (; f < F; ++f)
        if ((__ldg(reinterpret_cast<const unsigned long long *>(bits) + (uint64_t)__ldg(freq + f) * stride + w) >> b) &
            1ull) {
            if (WRITE) rows[at++] = (uint16_t)f;
            ++n;
        }
    if (!WRITE) len[t] = n;
}

// fidx[col] = frequent index of column col, 0xffff for an infrequent column.
__global__ void k_hrow_fidx(const uint32_t *__restrict__ freq, uint32_t F, uint16_t *__restrict__ fidx) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < F) fidx[freq[f]] = (uint16_t)f;
}

}  // namespace cpm
