// Level-wise Apriori on the device (cuApriori.py:473-535).
//
// A level is a lexicographically sorted array of k-item rows (columns), with
// the pattern id of every row.  Candidates of the next level join two rows
// that share their first k-1 items (cuApriori.py:482-487) and survive only if
// every k-subset is in the level (:488-490); the join runs in row order, so the
// candidate list comes out sorted, as the reference's sorted(candidates).
// Supports are complete intersections of the original tidsets (k_count_pruned).
#pragma once
#include "common.cuh"

namespace cpm {

__device__ __forceinline__ int cmp_rows(const uint32_t *a, const uint32_t *b, uint32_t k) {
    for (uint32_t i = 0; i < k; ++i)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}

__device__ bool level_has(const uint32_t *L, uint64_t n, uint32_t k, const uint32_t *x) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        const int c = cmp_rows(L + mid * k, x, k);
        if (!c) return true;
        if (c < 0) lo = mid + 1; else hi = mid;
    }
    return false;
}

// Row a starts a prefix group when its first k-1 items differ from row a-1.
// Levels run with their row count on the device (*d_n) and grids sized by an
// upper bound n_ub on the host, so that no level waits for its own count:
// rows at or past *d_n flag nothing and have no partners.
__global__ void k_group_start(const uint32_t *__restrict__ L, uint64_t n_ub, const uint64_t *__restrict__ d_n,
                              uint32_t k, uint32_t *__restrict__ flag) {
    const uint64_t a = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_ub) return;
    const uint64_t n = *d_n;
    flag[a] = a < n && (a == 0 || cmp_rows(L + (a - 1) * k, L + a * k, k - 1)) ? 1u : 0u;
}

// Exclusive group-start scan -> each group's first row (gfirst[g]) and, per
// row, the number of later rows of its group (its join partners).
// gfirst[g] = first row of group g; the entry after the last group holds n,
// so a row's group always ends at gfirst[g + 1] (gfirst has n + 1 entries).
__global__ void k_group_first(const uint32_t *__restrict__ flag, const uint64_t *__restrict__ gid_excl,
                              const uint64_t *__restrict__ d_n, uint64_t *__restrict__ gfirst) {
    const uint64_t a = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t n = *d_n;
    if (a < n && flag[a]) gfirst[gid_excl[a]] = a;
    if (a + 1 == n) gfirst[gid_excl[a] + flag[a]] = n;
}

__global__ void k_partners(const uint32_t *__restrict__ flag, const uint64_t *__restrict__ gid_excl,
                           const uint64_t *__restrict__ gfirst, uint64_t n_ub, const uint64_t *__restrict__ d_n,
                           uint32_t *__restrict__ partners) {
    const uint64_t a = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_ub) return;
    if (a >= *d_n) {
        partners[a] = 0;
        return;
    }
    const uint64_t g = gid_excl[a] + flag[a] - 1;  // this row's group
    partners[a] = (uint32_t)(gfirst[g + 1] - a - 1);
}

// One thread per join pair t: row a = last row with poff[a] <= t, partner
// b = a + 1 + t - poff[a].  Writes the candidate and whether every k-subset
// is frequent (cuApriori.py:488-490).
// The level's rows are L[0, *d_n): the subset searches must not see the
// rows past them (left over in a buffer sized by an upper bound).
__global__ void k_join_pairs(const uint32_t *__restrict__ L, const uint64_t *__restrict__ d_n, uint32_t k,
                             const uint64_t *__restrict__ poff, uint64_t n_pairs, uint32_t *__restrict__ cand,
                             uint32_t *__restrict__ cand_left, uint32_t *__restrict__ ok_flag) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_pairs) return;
    const uint64_t n = *d_n;
    uint64_t lo = 0, hi = n;  // upper_bound(poff, t) - 1
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (poff[mid] <= t) lo = mid + 1; else hi = mid;
    }
    const uint64_t a = lo - 1;
    const uint64_t b = a + 1 + (t - poff[a]);
    const uint32_t *ra = L + a * k, *rb = L + b * k;
    const uint32_t last = rb[k - 1];
    uint32_t *dst = cand + t * (k + 1);
    for (uint32_t i = 0; i < k; ++i) dst[i] = ra[i];
    dst[k] = last;
    cand_left[t] = (uint32_t)a;
    uint32_t sub[64];
    bool ok = true;
    for (uint32_t drop = 0; drop + 1 < k && ok; ++drop) {
        uint32_t m = 0;
        for (uint32_t i = 0; i < k; ++i)
            if (i != drop) sub[m++] = ra[i];
        sub[m] = last;
        ok = level_has(L, n, k, sub);
    }
    ok_flag[t] = ok ? 1u : 0u;
}

// Complete intersection of the candidates that passed pruning (warp each);
// pass[t] = pruned-in and support >= minsup.
__global__ void k_count_pruned(const uint64_t *__restrict__ bits, uint64_t stride, const uint32_t *__restrict__ cand,
                               const uint32_t *__restrict__ ok_flag, uint64_t n, uint32_t width, long long minsup,
                               uint32_t *__restrict__ support, uint32_t *__restrict__ pass) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (warp >= n) return;
    if (!ok_flag[warp]) {
        if (!lane) { support[warp] = 0; pass[warp] = 0; }
        return;
    }
    const uint32_t *cc = cand + warp * width;
    uint32_t s = 0;
    for (uint64_t v = lane; v < stride / 2; v += 32) {
        ulonglong2 acc = make_ulonglong2(~0ull, ~0ull);
        for (uint32_t j = 0; j < width; ++j)
            acc = and2(acc, ld_stream(reinterpret_cast<const ulonglong2 *>(bits + (uint64_t)cc[j] * stride) + v));
        s += popc2(acc);
    }
    s = warp_sum_u32(s);
    if (!lane) {
        support[warp] = s;
        pass[warp] = (long long)s >= minsup ? 1u : 0u;
    }
}

// The same supports as k_count_pruned, with the prefix shared.  The
// candidates joined on left row a of the level (t in [poff[a], poff[a] +
// partners[a]), cand rows L[a] + one last item) share the k items of L[a], so
// their complete intersection is (AND of the k rows of L[a]) AND (the last
// item's row).  One CTA takes one left row at a time (grid stride): it stages
// the prefix AND in shared memory once (stride words), then each warp streams
// one candidate's last-item row against it, eight 16-byte loads in flight per
// lane.  A group of p candidates reads k + p rows instead of (k + 1) p.
// *bytes_alg gains the rows read.  Rows at or past *d_n have no partners.
__global__ void __launch_bounds__(256) k_count_grouped(const uint64_t *__restrict__ bits, uint64_t stride,
                                                       const uint32_t *__restrict__ L, const uint64_t *__restrict__ d_n,
                                                       uint32_t k, const uint64_t *__restrict__ poff,
                                                       const uint32_t *__restrict__ partners,
                                                       const uint32_t *__restrict__ cand,
                                                       const uint32_t *__restrict__ ok_flag, long long minsup,
                                                       uint32_t *__restrict__ support, uint32_t *__restrict__ pass,
                                                       unsigned long long *__restrict__ bytes_alg) {
    extern __shared__ ulonglong2 s_pre[];
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint64_t n = *d_n, n2 = stride / 2;
    const uint32_t w = k + 1;
    unsigned long long rows_read = 0;
    for (uint64_t a = blockIdx.x; a < n; a += gridDim.x) {
        const uint32_t p = partners[a];
        if (!p) continue;  // the same for every thread of the CTA
        const uint32_t *ra = L + a * k;
        for (uint64_t v = threadIdx.x; v < n2; v += blockDim.x) {
            ulonglong2 acc = ld_stream(reinterpret_cast<const ulonglong2 *>(bits + (uint64_t)ra[0] * stride) + v);
            for (uint32_t j = 1; j < k; ++j)
                acc = and2(acc, ld_stream(reinterpret_cast<const ulonglong2 *>(bits + (uint64_t)ra[j] * stride) + v));
            s_pre[v] = acc;
        }
        __syncthreads();
        const uint64_t t0 = poff[a];
        for (uint32_t j = wid; j < p; j += nw) {
            const uint64_t t = t0 + j;
            if (!ok_flag[t]) {
                if (!lane) {
                    support[t] = 0;
                    pass[t] = 0;
                }
                continue;
            }
            const ulonglong2 *row = reinterpret_cast<const ulonglong2 *>(bits + (uint64_t)cand[t * w + k] * stride);
            uint32_t s = 0;
            uint64_t v = lane;
            for (; v + 224 < n2; v += 256) {
                ulonglong2 x[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) x[u] = ld_stream(row + v + 32 * u);
#pragma unroll
                for (int u = 0; u < 8; ++u) s += popc2(and2(x[u], s_pre[v + 32 * u]));
            }
            for (; v < n2; v += 32) s += popc2(and2(ld_stream(row + v), s_pre[v]));
            s = warp_sum_u32(s);
            if (!lane) {
                support[t] = s;
                pass[t] = (long long)s >= minsup ? 1u : 0u;
                ++rows_read;  // the last item's row
            }
        }
        if (!threadIdx.x) rows_read += k;  // the prefix rows
        __syncthreads();
    }
    if (!lane && rows_read) atomicAdd(bytes_alg, rows_read * 8ull * stride);
}

// ---- one-CTA forms for small levels (fewer launches per level) ----

// Exclusive sum over a CTA of up to 1024 threads (every thread calls it);
// *total gets the CTA's sum.  s_w holds 32 partial sums.
__device__ __forceinline__ uint64_t cta_excl_sum(uint64_t v, uint64_t *s_w, uint64_t *total) {
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(CPM_FULL, incl, o);
        if (lane >= (unsigned)o) incl += y;
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    uint64_t before = 0, tot = 0;
    for (unsigned w = 0; w < nw; ++w) {
        if (w < wid) before += s_w[w];
        tot += s_w[w];
    }
    __syncthreads();
    *total = tot;
    return before + incl - v;
}

// The join partners of every row of a level and their exclusive sum, in one
// CTA (what k_group_start, the group scan, k_group_first, k_partners and the
// partner scan do in five launches).  A row's partners are the later rows of
// its prefix group: from the row up to the next row that starts a group
// (whose first k-1 items differ from its predecessor's), found last chunk
// first with a suffix minimum.  *n_pairs gets the candidate count; rows at or
// past *d_n (up to n_ub) have no partners.
__global__ void __launch_bounds__(1024) k_level_prep(const uint32_t *__restrict__ L, uint64_t n_ub,
                                                     const uint64_t *__restrict__ d_n, uint32_t k,
                                                     uint32_t *__restrict__ partners, uint64_t *__restrict__ poff,
                                                     uint64_t *__restrict__ n_pairs) {
    __shared__ uint64_t s_w[32];
    __shared__ uint64_t s_carry;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint64_t n = *d_n;
    if (threadIdx.x == 0) s_carry = n;
    __syncthreads();
    const int64_t chunks = (int64_t)((n + blockDim.x - 1) / blockDim.x);
    for (int64_t c = chunks - 1; c >= 0; --c) {
        const uint64_t a = (uint64_t)c * blockDim.x + threadIdx.x;
        // the smallest group start after row a, within this chunk's rows
        uint64_t m = (a + 1 < n && cmp_rows(L + a * k, L + (a + 1) * k, k - 1)) ? a + 1 : ~0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_down_sync(CPM_FULL, m, o);
            if (lane + o < 32) m = min(m, y);
        }
        if (lane == 0) s_w[wid] = m;
        __syncthreads();
        uint64_t end = min(m, s_carry);
        for (unsigned w = wid + 1; w < nw; ++w) end = min(end, s_w[w]);
        if (a < n) partners[a] = (uint32_t)(end - a - 1);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint64_t cm = s_carry;
            for (unsigned w = 0; w < nw; ++w) cm = min(cm, s_w[w]);
            s_carry = cm;
        }
        __syncthreads();
    }
    for (uint64_t a = n + threadIdx.x; a < n_ub; a += blockDim.x) partners[a] = 0;
    __syncthreads();
    uint64_t run = 0;
    for (uint64_t base = 0; base < n; base += blockDim.x) {
        const uint64_t a = base + threadIdx.x;
        const uint64_t v = a < n ? partners[a] : 0;
        uint64_t tot = 0;
        const uint64_t ex = cta_excl_sum(v, s_w, &tot);
        if (a < n) poff[a] = run + ex;
        run += tot;
    }
    if (threadIdx.x == 0) *n_pairs = run;
}

// k_apriori_keep and k_level_close with the scan of the pass flags, in one
// CTA: survivors become the next level's rows and pattern records, in
// candidate order, and the level's row and pattern counts move on.
__global__ void __launch_bounds__(1024) k_level_keep(const uint32_t *__restrict__ cand,
                                                     const uint32_t *__restrict__ cand_left,
                                                     const uint32_t *__restrict__ sup,
                                                     const uint32_t *__restrict__ pass, uint64_t n, uint32_t w,
                                                     const uint32_t *__restrict__ pid_prev, uint64_t *__restrict__ d_cnt2,
                                                     uint32_t *__restrict__ L_next, uint32_t *__restrict__ pid_next,
                                                     uint32_t *__restrict__ pat_parent, uint32_t *__restrict__ pat_item,
                                                     uint32_t *__restrict__ pat_sup) {
    __shared__ uint64_t s_w[32];
    const uint64_t pid_base = d_cnt2[1];
    uint64_t run = 0;
    // Each thread takes eight consecutive candidates per round, so that a
    // level of n candidates costs n / (8 * blockDim) block scans.
    constexpr uint32_t PER = 8;
    for (uint64_t base = 0; base < n; base += (uint64_t)blockDim.x * PER) {
        const uint64_t i0 = base + (uint64_t)threadIdx.x * PER;
        uint32_t f[PER], c = 0;
#pragma unroll
        for (uint32_t u = 0; u < PER; ++u) {
            f[u] = i0 + u < n ? pass[i0 + u] : 0u;
            c += f[u] ? 1u : 0u;
        }
        uint64_t tot = 0;
        uint64_t p = run + cta_excl_sum(c, s_w, &tot);
#pragma unroll
        for (uint32_t u = 0; u < PER; ++u) {
            if (!f[u]) continue;
            const uint64_t i = i0 + u;
            for (uint32_t j = 0; j < w; ++j) L_next[p * w + j] = cand[i * w + j];
            const uint64_t pid = pid_base + p;
            pid_next[p] = (uint32_t)pid;
            pat_parent[pid] = pid_prev[cand_left[i]];
            pat_item[pid] = cand[i * w + w - 1];
            pat_sup[pid] = sup[i];
            ++p;
        }
        run += tot;
    }
    __syncthreads();  // every thread has read d_cnt2[1]
    if (threadIdx.x == 0) {
        d_cnt2[0] = run;
        d_cnt2[1] = pid_base + run;
    }
}

// Survivors, in candidate order, become the next level and pattern records.
__global__ void k_apriori_keep(const uint32_t *__restrict__ cand, const uint32_t *__restrict__ cand_left,
                               const uint32_t *__restrict__ sup, const uint32_t *__restrict__ flag,
                               const uint64_t *__restrict__ pos, uint64_t n, uint32_t w,
                               const uint32_t *__restrict__ pid_prev, const uint64_t *__restrict__ d_pid_base,
                               uint32_t *__restrict__ L_next, uint32_t *__restrict__ pid_next,
                               uint32_t *__restrict__ pat_parent, uint32_t *__restrict__ pat_item,
                               uint32_t *__restrict__ pat_sup) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const uint64_t p = pos[i];
    for (uint32_t j = 0; j < w; ++j) L_next[p * w + j] = cand[i * w + j];
    const uint64_t pid = *d_pid_base + p;
    pid_next[p] = (uint32_t)pid;
    pat_parent[pid] = pid_prev[cand_left[i]];
    pat_item[pid] = cand[i * w + w - 1];
    pat_sup[pid] = sup[i];
}

// The level's survivors (exclusive scan pos of pass flags): the next level's
// row count, and the pattern count moved past them.
__global__ void k_level_close(const uint64_t *__restrict__ pos, const uint32_t *__restrict__ pass, uint64_t n_pairs,
                              uint64_t *__restrict__ d_n, uint64_t *__restrict__ d_npat) {
    if (blockIdx.x || threadIdx.x) return;
    const uint64_t nk = n_pairs ? pos[n_pairs - 1] + pass[n_pairs - 1] : 0;
    *d_n = nk;
    *d_npat += nk;
}

__global__ void k_set_u64x2(uint64_t *__restrict__ a, uint64_t va, uint64_t *__restrict__ b, uint64_t vb) {
    if (blockIdx.x || threadIdx.x) return;
    *a = va;
    *b = vb;
}

// Level 2 from the pair Gram: rows (f_i, f_j) in (i, j) order with pattern ids.
__global__ void k_pairs_to_level(const uint32_t *__restrict__ C, uint32_t F, long long minsup,
                                 const uint32_t *__restrict__ freq, const uint64_t *__restrict__ off,
                                 uint64_t pid_base, uint32_t *__restrict__ L2, uint32_t *__restrict__ pid2,
                                 uint32_t *__restrict__ pat_parent, uint32_t *__restrict__ pat_item,
                                 uint32_t *__restrict__ pat_sup) {
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
            L2[2 * k] = freq[i];
            L2[2 * k + 1] = freq[j];
            const uint64_t pid = pid_base + k;
            pid2[k] = (uint32_t)pid;
            pat_parent[pid] = (uint32_t)i;
            pat_item[pid] = freq[j];
            pat_sup[pid] = s;
        }
        pos += __popc(bal);
    }
}

// Exclusive prefix sum of n uint32 values into uint64 (one CTA, chunked);
// *total receives the sum.  Levels hold at most a few million rows.
__global__ void k_scan_u32(const uint32_t *__restrict__ in, uint64_t n, uint64_t *__restrict__ out,
                           uint64_t *__restrict__ total) {
    __shared__ unsigned long long warp_tot[32];
    __shared__ unsigned long long base;
    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (uint64_t start = 0; start < n; start += blockDim.x) {
        const uint64_t i = start + threadIdx.x;
        unsigned long long v = i < n ? in[i] : 0;
        unsigned long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(CPM_FULL, x, o);
            if (lane >= (unsigned)o) x += y;
        }
        if (lane == 31) warp_tot[wid] = x;
        __syncthreads();
        unsigned long long before = 0, all = 0;
        for (unsigned w = 0; w < nw; ++w) {
            if (w < wid) before += warp_tot[w];
            all += warp_tot[w];
        }
        if (i < n) out[i] = base + before + x - v;
        __syncthreads();
        if (threadIdx.x == 0) base += all;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = base;
}

}  // namespace cpm
