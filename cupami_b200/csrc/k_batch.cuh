// Pre-deep stages of Eclat over a batch of databases, one launch per stage.
//
// Each database is described by a DbDesc (its tidsets, supports, threshold and
// where its frequent list, pair Gram and pattern ids live); the kernels below
// run the singleton compaction (cuEclat.py:174-179), the pair Gram and
// threshold (cuEclat.py:183-193) and the class tables (cuEclat.py:195-200) for
// every database at once, so the launch count does not grow with the batch.
#pragma once
#include "common.cuh"
#include "k_pairs.cuh"

namespace cpm {

struct DbDesc {
    const uint64_t *bits;      // item-major tidsets
    const uint32_t *support;   // per column
    uint32_t *freq;            // frequent columns, increasing
    uint32_t *C;               // F x F pair Gram (upper triangle)
    uint64_t stride;           // words per tidset
    uint32_t n_items;
    uint32_t F;                // frequent items (set by the host after compaction)
    long long minsup;
    uint64_t pat_base;         // pattern id of the first singleton; pairs follow at pat_base + F
    uint64_t pair_base;        // global index of the first pair (= first top-level member)
    uint64_t row_base;         // global index of the first frequent row
};

// Block b compacts database b's passing columns in order; F goes to F_out[b].
__global__ void k_compact_frequent_b(const DbDesc *__restrict__ d, uint32_t *__restrict__ F_out) {
    const DbDesc D = d[blockIdx.x];
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t start = 0; start < D.n_items; start += blockDim.x) {
        const uint32_t c = start + threadIdx.x;
        const bool pass = c < D.n_items && (long long)D.support[c] >= D.minsup;
        const unsigned bal = __ballot_sync(CPM_FULL, pass);
        if (!lane) warp_tot[wid] = __popc(bal);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (unsigned w = 0; w < nw; ++w) {
            if (w < wid) before += warp_tot[w];
            total += warp_tot[w];
        }
        if (pass) D.freq[base + before + __popc(bal & ((1u << lane) - 1))] = c;
        __syncthreads();
        if (threadIdx.x == 0) base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) F_out[blockIdx.x] = base;
}

struct BTile {
    uint32_t db, ti, tj, pad;
    uint64_t k_begin, k_end;  // words
};

// CUDA-core Gram over a list of (database, 64x64 tile, K range); C zeroed.
__global__ void __launch_bounds__(256) k_gram_simt_b(const DbDesc *__restrict__ d, const BTile *__restrict__ tiles) {
    constexpr int TM = 64, KW = 16;
    __shared__ uint64_t As[KW][TM + 1];
    __shared__ uint64_t Bs[KW][TM + 1];
    const BTile t = tiles[blockIdx.x];
    const DbDesc D = d[t.db];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    uint32_t acc[4][4] = {};
    for (uint64_t k0 = t.k_begin; k0 < t.k_end; k0 += KW) {
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int idx = threadIdx.x + l * 256;
            const int r = idx >> 4, kk = idx & 15;
            const uint32_t gi = t.ti * TM + r, gj = t.tj * TM + r;
            const uint64_t k = k0 + kk;
            As[kk][r] = (gi < D.F && k < t.k_end) ? __ldg(D.bits + (uint64_t)D.freq[gi] * D.stride + k) : 0ull;
            Bs[kk][r] = (gj < D.F && k < t.k_end) ? __ldg(D.bits + (uint64_t)D.freq[gj] * D.stride + k) : 0ull;
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
            const uint32_t gi = t.ti * TM + ty * 4 + i, gj = t.tj * TM + tx * 4 + j;
            if (gi < gj && gj < D.F && acc[i][j]) atomicAdd(D.C + (uint64_t)gi * D.F + gj, acc[i][j]);
        }
}

__device__ __forceinline__ uint32_t db_of_row(const DbDesc *d, uint32_t n_db, uint64_t r) {
    uint32_t lo = 0, hi = n_db;  // last db with row_base <= r
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (d[mid].row_base <= r) lo = mid; else hi = mid;
    }
    return lo;
}

// cnt[r] = passing pairs (i, j > i) of global frequent row r; warp per row.
__global__ void k_pair_count_b(const DbDesc *__restrict__ d, uint32_t n_db, uint64_t n_rows,
                               uint32_t *__restrict__ cnt) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (r >= n_rows) return;
    const DbDesc D = d[db_of_row(d, n_db, r)];
    const uint64_t i = r - D.row_base;
    uint32_t c = 0;
    for (uint64_t j = i + 1 + lane; j < D.F; j += 32) c += (long long)D.C[i * D.F + j] >= D.minsup;
    c = warp_sum_u32(c);
    if (!lane) cnt[r] = c;
}

// Singleton and pair patterns plus top-level member tables; warp per global
// frequent row r.  off[r] = global index of row r's first pair.
__global__ void k_emit_b(const DbDesc *__restrict__ d, uint32_t n_db, uint64_t n_rows,
                         const uint64_t *__restrict__ off, uint32_t *__restrict__ pat_parent,
                         uint32_t *__restrict__ pat_item, uint32_t *__restrict__ pat_sup,
                         uint32_t *__restrict__ pat_db, uint32_t *__restrict__ mem_pat,
                         uint32_t *__restrict__ mem_item, const uint64_t **__restrict__ mem_bits,
                         const unsigned long long *__restrict__ row_list) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (r >= n_rows) return;
    const uint32_t db = db_of_row(d, n_db, r);
    const DbDesc D = d[db];
    const uint64_t i = r - D.row_base;
    const uint32_t fi = D.freq[i];
    if (lane == 0) {
        const uint64_t pid = D.pat_base + i;
        pat_parent[pid] = 0xffffffffu;
        pat_item[pid] = fi;
        pat_sup[pid] = D.support[fi];
        if (pat_db) pat_db[pid] = db;
    }
    uint64_t pos = off[r];
    for (uint64_t j0 = i + 1; j0 < D.F; j0 += 32) {
        const uint64_t j = j0 + lane;
        const uint32_t s = j < D.F ? D.C[i * D.F + j] : 0u;
        const bool pass = j < D.F && (long long)s >= D.minsup;
        const unsigned bal = __ballot_sync(CPM_FULL, pass);
        if (pass) {
            const uint64_t k = pos + __popc(bal & ((1u << lane) - 1));
            const uint64_t pid = D.pat_base + D.F + (k - D.pair_base);
            const uint32_t item = D.freq[j];
            pat_parent[pid] = (uint32_t)(D.pat_base + i);
            pat_item[pid] = item;
            pat_sup[pid] = s;
            if (pat_db) pat_db[pid] = db;
            mem_pat[k] = (uint32_t)pid;
            mem_item[k] = item;
            // The item's transaction-id list where one was built (bit 0 set), else its bitset.
            const unsigned long long lp = row_list ? row_list[D.row_base + j] : 0ull;
            mem_bits[k] = lp ? reinterpret_cast<const uint64_t *>(lp) : D.bits + (uint64_t)item * D.stride;
        }
        pos += __popc(bal);
    }
}

// Transaction-id lists of sparse frequent items (the list form of k_deep.cuh:
// 16-byte header {count, 0, 0, 0}, ascending ids, zero padding to 16 bytes).
// words[r] = 64-bit words of row r's list, or 0 when the item stays dense
// (list above 1/list_div of the bitset).
__global__ void k_list_plan(const DbDesc *__restrict__ d, uint32_t n_db, uint64_t n_rows, uint32_t list_div,
                            uint64_t *__restrict__ words) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows) return;
    const DbDesc &D = d[db_of_row(d, n_db, r)];
    const uint32_t sup = D.support[D.freq[r - D.row_base]];
    const uint64_t lw = ((uint64_t)sup + 7) / 4 * 2;
    words[r] = lw * list_div <= D.stride ? lw : 0;
}

// One warp per frequent row with a list: extracts the row's set bits in order.
// row_list[r] gets the tagged pointer (bit 0 set) or 0.
__global__ void k_item_lists(const DbDesc *__restrict__ d, uint32_t n_db, uint64_t n_rows,
                             const uint64_t *__restrict__ words, const uint64_t *__restrict__ offs,
                             uint64_t *__restrict__ buf, unsigned long long *__restrict__ row_list) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (r >= n_rows) return;
    if (!words[r]) {
        if (lane == 0) row_list[r] = 0ull;
        return;
    }
    const DbDesc &D = d[db_of_row(d, n_db, r)];
    const uint32_t item = D.freq[r - D.row_base];
    const ulonglong2 *row = reinterpret_cast<const ulonglong2 *>(D.bits + (uint64_t)item * D.stride);
    uint32_t *o32 = reinterpret_cast<uint32_t *>(buf + offs[r]);
    const uint64_t n2 = D.stride / 2;
    uint32_t written = 0;
    for (uint64_t v0 = 0; v0 < n2; v0 += 32) {
        const uint64_t v = v0 + lane;
        const ulonglong2 x = v < n2 ? ld_stream(row + v) : make_ulonglong2(0ull, 0ull);
        const uint32_t c = (uint32_t)(__popcll(x.x) + __popcll(x.y));
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(CPM_FULL, incl, o);
            if (lane >= (unsigned)o) incl += y;
        }
        uint32_t pos = 4 + written + incl - c;
        for (unsigned long long b = x.x; b; b &= b - 1) o32[pos++] = (uint32_t)(v * 128 + __ffsll((long long)b) - 1);
        for (unsigned long long b = x.y; b; b &= b - 1) o32[pos++] = (uint32_t)(v * 128 + 64 + __ffsll((long long)b) - 1);
        written += __shfl_sync(CPM_FULL, incl, 31);
    }
    const uint32_t end = 4 + written, pad_end = (uint32_t)(((uint64_t)written + 7) / 4 * 4);
    if (lane < pad_end - end) o32[end + lane] = 0u;
    if (lane == 0) {
        o32[0] = written;
        o32[1] = o32[2] = o32[3] = 0u;
        row_list[r] = reinterpret_cast<unsigned long long>(o32) | 1ull;
    }
}

}  // namespace cpm
