// Packing, singleton supports, ordered compaction, k-way support counting and
// the reference kernel-module API kernels.
//
// Layout: item-major tidsets, bit (r % 64) of 64-bit word (r / 64) of row c is
// set when non-empty transaction r holds column c.  Rows are `stride` words
// apart, stride = ceil(N/64) rounded up to an even count so that every row
// starts on a 16-byte boundary and can be read with 128-bit loads.
#pragma once
#include "common.cuh"

namespace cpm {

// One thread per transaction.  Threads of a warp hold 32 consecutive rows, so
// they share one 32-bit word of every tidset; threads that reach the same
// column in the same step merge their bits with __match_any_sync and one
// atomicOr (the match mask is exactly the OR of their 1 << lane bits).
// Reference: _bitsets.py:20-28 (one atomicOr per occurrence).
__global__ void k_pack(const uint64_t *__restrict__ offsets, const uint32_t *__restrict__ ids,
                       const uint32_t *__restrict__ lut, uint64_t n_tx, uint64_t stride,
                       uint32_t *__restrict__ bits32) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned lane = threadIdx.x & 31;
    const bool valid = r < n_tx;
    const uint64_t b = valid ? offsets[r] : 0;
    const uint32_t len = valid ? (uint32_t)(offsets[r + 1] - b) : 0;
    const uint32_t maxlen = warp_max_u32(len);
    const uint64_t word32 = r >> 5;
    for (uint32_t k = 0; k < maxlen; ++k) {
        uint32_t c = 0xffffffffu;
        if (k < len) {
            c = __ldg(ids + b + k);
            if (lut) c = __ldg(lut + c);
        }
        const unsigned grp = __match_any_sync(CPM_FULL, c);
        if (c != 0xffffffffu && lane == (unsigned)(__ffs(grp) - 1))
            atomicOr(bits32 + (uint64_t)c * stride * 2 + word32, grp);
    }
}

// Marks which raw ids occur (presence bitmap over the id universe).  A few
// hundred distinct ids share a few dozen words, so the bits are tested before
// the atomic: once a word is complete its readers stop issuing atomics (a
// stale zero only costs one redundant atomicOr).
__global__ void k_mark_ids(const uint32_t *__restrict__ ids, uint64_t nnz, uint32_t *__restrict__ present) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = ids[i], bit = 1u << (v & 31);
        if (!(present[v >> 5] & bit)) atomicOr(present + (v >> 5), bit);
    }
}

// Same, with the bitmap (pw words) built per block in shared memory and OR-ed
// into the global one once per non-zero word; for id ranges that fit.
__global__ void k_mark_ids_smem(const uint32_t *__restrict__ ids, uint64_t nnz, uint32_t pw,
                                uint32_t *__restrict__ present) {
    extern __shared__ uint32_t s_present[];
    for (uint32_t w = threadIdx.x; w < pw; w += blockDim.x) s_present[w] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = ids[i], bit = 1u << (v & 31);
        if (!(s_present[v >> 5] & bit)) atomicOr(s_present + (v >> 5), bit);
    }
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < pw; w += blockDim.x)
        if (s_present[w]) atomicOr(present + w, s_present[w]);
}

// support[c] = popcount of row c; one warp per row, 128-bit loads.
__global__ void k_item_support(const uint64_t *__restrict__ bits, uint64_t stride, uint32_t n_items,
                               uint32_t *__restrict__ support) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (warp >= n_items) return;
    const ulonglong2 *row = reinterpret_cast<const ulonglong2 *>(bits + warp * stride);
    uint32_t s = 0;
    for (uint64_t v = lane; v < stride / 2; v += 32) s += popc2(ld_stream(row + v));
    s = warp_sum_u32(s);
    if (!lane) support[warp] = s;
}

// Ordered compaction of the columns whose support passes: out[k] = k-th
// passing column in increasing order; *count = number passing.  One CTA.
__global__ void k_compact_frequent(const uint32_t *__restrict__ support, uint32_t n_items,
                                   long long minsup, uint32_t *__restrict__ out,
                                   uint32_t *__restrict__ count) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t start = 0; start < n_items; start += blockDim.x) {
        const uint32_t c = start + threadIdx.x;
        const bool pass = c < n_items && (long long)support[c] >= minsup;
        const unsigned bal = __ballot_sync(CPM_FULL, pass);
        if (!lane) warp_tot[wid] = __popc(bal);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (unsigned w = 0; w < nw; ++w) {
            if (w < wid) before += warp_tot[w];
            total += warp_tot[w];
        }
        if (pass) out[base + before + __popc(bal & ((1u << lane) - 1))] = c;
        __syncthreads();
        if (threadIdx.x == 0) base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = base;
}

// Writes the singleton pattern records (parent none, item, support).
__global__ void k_emit_singletons(const uint32_t *__restrict__ freq, uint32_t F,
                                  const uint32_t *__restrict__ support, uint32_t *__restrict__ pat_parent,
                                  uint32_t *__restrict__ pat_item, uint32_t *__restrict__ pat_sup) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F) return;
    pat_parent[i] = 0xffffffffu;
    pat_item[i] = freq[i];
    pat_sup[i] = support[freq[i]];
}

// ---- reference kernel-module API (32-bit word layout of _bitsets.py) ------

__global__ void k_ref_build(const uint64_t *__restrict__ rows, const uint32_t *__restrict__ cols,
                            uint64_t count, uint64_t words, uint32_t *__restrict__ bits) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x)
        atomicOr(bits + (uint64_t)cols[i] * words + rows[i] / 32, 1u << (rows[i] % 32));
}

__global__ void k_ref_count(const uint32_t *__restrict__ bits, uint64_t words,
                            const uint32_t *__restrict__ cand, uint64_t n, uint32_t width,
                            unsigned long long *__restrict__ support) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (warp >= n) return;
    const uint32_t *cc = cand + warp * width;
    unsigned long long s = 0;
    for (uint64_t w = lane; w < words; w += 32) {
        uint32_t acc = 0xffffffffu;
        for (uint32_t j = 0; j < width; ++j) acc &= __ldg(bits + (uint64_t)cc[j] * words + w);
        s += __popc(acc);
    }
    s = warp_sum_u64(s);
    if (!lane) support[warp] = s;
}

__global__ void k_ref_intersect(const uint32_t *__restrict__ prefix, const uint32_t *__restrict__ ext,
                                uint64_t words, uint64_t n, uint32_t *__restrict__ out,
                                unsigned long long *__restrict__ support) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (warp >= n) return;
    unsigned long long s = 0;
    const uint32_t *e = ext + warp * words;
    uint32_t *o = out + warp * words;
    for (uint64_t w = lane; w < words; w += 32) {
        const uint32_t v = __ldg(prefix + w) & __ldg(e + w);
        o[w] = v;
        s += __popc(v);
    }
    s = warp_sum_u64(s);
    if (!lane) support[warp] = s;
}

}  // namespace cpm

namespace cpm {

// Batched loading: databases concatenated, rows and occurrences numbered
// globally.  One descriptor per database.
struct PackDesc {
    uint32_t *bits32;      // tidsets of this database (32-bit view)
    uint32_t *support;     // per column
    const uint32_t *lut;   // id -> column
    uint64_t stride;       // 64-bit words per tidset
    uint64_t row_base;     // first global row
    uint64_t occ_base;     // first global occurrence (index into ids)
    uint64_t present_base; // first word of this database's presence bitmap
    uint32_t n_items, pad;
};

__device__ __forceinline__ uint32_t desc_of(const uint64_t *__restrict__ bases, uint32_t n, uint64_t x) {
    uint32_t lo = 0, hi = n;  // last k with bases[k] <= x
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (bases[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

// Presence bitmaps of every database (occ_bases[d] = first occurrence of d).
// With pw > 0 the whole bitmap (pw words) is staged in shared memory per
// block (dynamic shared memory of pw words), as in k_mark_ids_smem.
__global__ void k_mark_ids_b(const uint32_t *__restrict__ ids, uint64_t nnz, const uint64_t *__restrict__ occ_bases,
                             const uint64_t *__restrict__ present_bases, uint32_t n_db, uint32_t *__restrict__ present,
                             uint32_t pw) {
    extern __shared__ uint32_t s_present[];
    uint32_t *bm = pw ? s_present : present;
    for (uint32_t w = threadIdx.x; w < pw; w += blockDim.x) s_present[w] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t d = desc_of(occ_bases, n_db, i);
        const uint32_t v = ids[i], bit = 1u << (v & 31);
        const uint64_t w = present_bases[d] + (v >> 5);
        if (!(bm[w] & bit)) atomicOr(bm + w, bit);
    }
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < pw; w += blockDim.x)
        if (s_present[w]) atomicOr(present + w, s_present[w]);
}

// k_pack over all databases: one thread per global (non-empty) row; the
// warp's 32 rows may span two databases, so lanes merge by (database, column).
__global__ void k_pack_b(const uint64_t *__restrict__ offsets, const uint32_t *__restrict__ ids, uint64_t n_rows,
                         const PackDesc *__restrict__ d, const uint64_t *__restrict__ row_bases, uint32_t n_db) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned lane = threadIdx.x & 31;
    const bool valid = r < n_rows;
    const uint32_t db = valid ? desc_of(row_bases, n_db, r) : 0;
    const PackDesc D = d[db];
    const uint64_t b = valid ? offsets[r] : 0;
    const uint32_t len = valid ? (uint32_t)(offsets[r + 1] - b) : 0;
    const uint32_t maxlen = warp_max_u32(len);
    const uint64_t lr = r - D.row_base;  // row within its database
    for (uint32_t k = 0; k < maxlen; ++k) {
        uint64_t key = ~0ull;
        uint32_t c = 0;
        if (k < len) {
            c = __ldg(D.lut + __ldg(ids + b + k));
            key = ((uint64_t)db << 32) | c;
        }
        // Lanes of one database share the word only when they also share lr / 32.
        key ^= (uint64_t)(lr >> 5) << 52;
        const unsigned grp = __match_any_sync(CPM_FULL, key);
        if (k < len && lane == (unsigned)(__ffs(grp) - 1)) {
            // OR of 1 << (row % 32) over the group (rows are consecutive lanes)
            uint32_t mask = 0;
            for (unsigned g = grp; g; g &= g - 1) {
                const unsigned l = __ffs(g) - 1;
                mask |= 1u << ((lr + l - lane) & 31);
            }
            atomicOr(D.bits32 + (uint64_t)c * D.stride * 2 + (lr >> 5), mask);
        }
    }
}

// Singleton supports of every database: one warp per (database, column).
__global__ void k_item_support_b(const PackDesc *__restrict__ d, const uint64_t *__restrict__ item_bases, uint32_t n_db,
                                 uint64_t total_items) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (w >= total_items) return;
    const uint32_t db = desc_of(item_bases, n_db, w);
    const PackDesc D = d[db];
    const uint64_t c = w - item_bases[db];
    const ulonglong2 *row = reinterpret_cast<const ulonglong2 *>(reinterpret_cast<const uint64_t *>(D.bits32) + c * D.stride);
    uint32_t s = 0;
    for (uint64_t v = lane; v < D.stride / 2; v += 32) s += popc2(ld_stream(row + v));
    s = warp_sum_u32(s);
    if (!lane) D.support[c] = s;
}

}  // namespace cpm
