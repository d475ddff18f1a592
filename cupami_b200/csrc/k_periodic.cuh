// Periodic-frequent support counting (cupami/periodicFrequentPattern/_temporal.py:26-53).
//
// For an itemset X held by the rows r_1 < ... < r_s of a temporal database
// whose rows are sorted by timestamp ts[], the reference kernel returns the
// support s and the periodicity
//     max(ts[r_1] - 0, ts[r_2] - ts[r_1], ..., ts[r_s] - ts[r_{s-1}], end - ts[r_s])
// (end when s = 0), scanning the set bits of the AND of X's rows in order with
// one thread per candidate (_temporal.py:26-53, launch :156-165).
//
// Here one warp handles a candidate: each lane walks a contiguous share of
// the candidate's words (4 loads in flight per row) and reduces its rows to a
// segment summary (count, first and last timestamp, largest inner gap); the
// warp joins the 32 summaries once, in row order, with shuffles.  The join
//     (a, b) -> {a.cnt + b.cnt, a.first, b.last, max(a.gap, b.gap, b.first - a.last)}
// (an empty side yields the other) is associative, so the tree gives exactly
// the sequential scan's maximum -- also across warps: when a level has too
// few candidates to fill the GPU, each candidate's rows are split over several
// warps whose summaries k_periodic_join joins in order.  With kPrune (the
// miner), a candidate stops as soon as a gap is already too long -- rows are
// sorted by timestamp, so the next set row's gap is at least
// ts[first unscanned row] - last timestamp seen.
#pragma once
#include "common.cuh"

namespace cpm {

struct PSeg {
    unsigned long long cnt;
    long long first, last, gap;
};

__device__ __forceinline__ PSeg pseg_join(const PSeg &a, const PSeg &b) {
    if (!a.cnt) return b;
    if (!b.cnt) return a;
    PSeg r;
    r.cnt = a.cnt + b.cnt;
    r.first = a.first;
    r.last = b.last;
    r.gap = max(max(a.gap, b.gap), b.first - a.last);
    return r;
}

// Lane 0 receives the join of the 32 lanes' segments in lane order.
__device__ __forceinline__ PSeg pseg_warp_join(PSeg s, unsigned lane) {
#pragma unroll
    for (unsigned o = 1; o < 32; o <<= 1) {
        PSeg t;
        t.cnt = __shfl_down_sync(CPM_FULL, s.cnt, o);
        t.first = __shfl_down_sync(CPM_FULL, s.first, o);
        t.last = __shfl_down_sync(CPM_FULL, s.last, o);
        t.gap = __shfl_down_sync(CPM_FULL, s.gap, o);
        if (lane + o < 32) s = pseg_join(s, t);
    }
    return s;
}

__device__ __forceinline__ unsigned word_popc(uint32_t x) { return __popc(x); }
__device__ __forceinline__ unsigned word_popc(unsigned long long x) { return __popcll(x); }
__device__ __forceinline__ unsigned word_low(uint32_t x) { return __ffs(x) - 1; }
__device__ __forceinline__ unsigned word_low(unsigned long long x) { return __ffsll(x) - 1; }

// Words a lane loads per step (independent loads in flight), and the fewest
// words a part of a split candidate takes (PERIODIC_PL per lane).
constexpr unsigned PERIODIC_PL = 4;
constexpr uint64_t PERIODIC_TILE = 32 * PERIODIC_PL;

// `parts` warps per candidate c (warp g: candidate g / parts, part g % parts),
// each over an equal share of the words, and each lane of a warp over a
// contiguous share of its part: the AND of the width rows cand[c * width ..]
// of `bits` (Word: uint32_t or unsigned long long; rows of `stride` words;
// bit b of word v is row v * bits(Word) + b), restricted to rows < n_tx.  A
// lane summarises its rows as it goes; the warp joins the 32 summaries once,
// in lane (= row) order.  With parts = 1 the warp writes support[c] and
// period[c] (and, with kPrune, pass[c] = ok_flag[c] && support >= need &&
// period <= max_per); with parts > 1 each warp writes its summary to
// seg[c * parts + part] and k_periodic_join finishes.  With kPrune a warp
// stops as soon as one lane's rows prove the candidate fails: a gap already
// above max_per (a stretch without set rows from row a to row b gives a gap
// of at least ts[b] - ts[a - 1]; timestamps are nonnegative and sorted).  A
// stopped candidate has pass = 0, a stopped part reports gap = LLONG_MAX; only
// passing candidates have exact values.  Without kPrune every candidate is exact.
template <class Word, bool kPrune>
__global__ void __launch_bounds__(256)
k_periodic(const Word *__restrict__ bits, uint64_t stride, const uint32_t *__restrict__ cand,
           const uint32_t *__restrict__ ok_flag, uint64_t n, uint32_t width, const long long *__restrict__ ts,
           uint64_t n_tx, long long end, long long need, long long max_per, uint32_t parts, PSeg *__restrict__ seg,
           unsigned long long *__restrict__ support, long long *__restrict__ period, uint32_t *__restrict__ pass) {
    constexpr unsigned B = sizeof(Word) * 8;
    constexpr unsigned PL = PERIODIC_PL;
    const uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    const uint64_t c = g / parts;
    const uint32_t part = (uint32_t)(g % parts);
    if (c >= n) return;  // whole warps: c is the same on every lane
    if (ok_flag && !ok_flag[c]) {
        if (parts == 1 && !lane) {
            support[c] = 0;
            period[c] = end;
            if (pass) pass[c] = 0;
        }
        return;
    }
    const uint32_t *cc = cand + c * width;
    const uint64_t words = (n_tx + B - 1) / B;
    const uint64_t w0 = words * part / parts, w1 = words * (part + 1) / parts;  // this part
    const uint64_t per_lane = (w1 - w0 + 31) / 32;
    const uint64_t lo_raw = w0 + lane * per_lane;
    const uint64_t lo = lo_raw < w1 ? lo_raw : w1;
    const uint64_t hi = lo + per_lane < w1 ? lo + per_lane : w1;  // this lane: words [lo, hi)
    const long long before = kPrune && lo < hi && lo ? __ldg(ts + lo * B - 1) : 0;
    PSeg s{0, 0, 0, 0};
    bool stopped = false;
    for (uint64_t i = 0; i < per_lane; i += PL) {  // the same trip count on every lane
        const uint64_t v0 = lo + i;
        Word x[PL];
#pragma unroll
        for (unsigned q = 0; q < PL; ++q) x[q] = v0 + q < hi ? ~Word(0) : Word(0);
        for (uint32_t j = 0; j < width; ++j) {
            const Word *row = bits + (uint64_t)cc[j] * stride;
#pragma unroll
            for (unsigned q = 0; q < PL; ++q)
                if (v0 + q < hi) x[q] &= __ldg(row + v0 + q);
        }
#pragma unroll
        for (unsigned q = 0; q < PL; ++q) {
            const uint64_t row0 = (v0 + q) * B;
            if (v0 + q < hi && n_tx - row0 < B) x[q] &= (Word(1) << (unsigned)(n_tx - row0)) - Word(1);
            for (Word y = x[q]; y; y &= y - Word(1)) {  // one timestamp load per set row
                const long long t = __ldg(ts + row0 + word_low(y));
                if (s.cnt) s.gap = max(s.gap, t - s.last);
                else s.first = t;
                s.last = t;
                ++s.cnt;
            }
        }
        if (kPrune) {
            bool bad = false;
            if (lo < hi) {
                const uint64_t done = v0 + PL < hi ? v0 + PL : hi;
                const uint64_t r_end = done * B < n_tx ? done * B : n_tx;
                const long long next = r_end < n_tx ? __ldg(ts + r_end) : end;
                const long long bound = s.cnt ? max(max(s.first - before, s.gap), next - s.last) : next - before;
                bad = bound > max_per;
            }
            if (__any_sync(CPM_FULL, bad)) {
                stopped = true;
                break;
            }
        }
    }
    s = pseg_warp_join(s, lane);
    if (lane) return;
    if (parts == 1) {
        const long long per = s.cnt ? max(max(s.first, s.gap), end - s.last) : end;
        support[c] = s.cnt;
        period[c] = per;
        if (kPrune) pass[c] = !stopped && (long long)s.cnt >= need && per <= max_per ? 1u : 0u;
    } else {
        if (stopped) {
            s.cnt = s.cnt ? s.cnt : 1;
            s.gap = 0x7fffffffffffffffll;
        }
        seg[c * parts + part] = s;
    }
}

// One thread per candidate: joins its parts' summaries in row order and
// writes what k_periodic writes with one part.
__global__ void k_periodic_join(const PSeg *__restrict__ seg, uint32_t parts, const uint32_t *__restrict__ ok_flag,
                                uint64_t n, long long end, long long need, long long max_per,
                                unsigned long long *__restrict__ support, long long *__restrict__ period,
                                uint32_t *__restrict__ pass) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    if (ok_flag && !ok_flag[c]) {
        support[c] = 0;
        period[c] = end;
        if (pass) pass[c] = 0;
        return;
    }
    PSeg run{0, 0, 0, 0};
    for (uint32_t p = 0; p < parts; ++p) run = pseg_join(run, seg[c * parts + p]);
    const long long per = run.cnt ? max(max(run.first, run.gap), end - run.last) : end;
    support[c] = run.cnt;
    period[c] = per;
    if (pass) pass[c] = (long long)run.cnt >= need && per <= max_per ? 1u : 0u;
}

__global__ void k_iota_u32(uint32_t *__restrict__ out, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (uint32_t)i;
}

// Passing candidates, in candidate order, become the next level's rows and
// pattern records (pattern pid = *d_pid_base + rank among the passing ones).
// Level 1 has no previous level: pid_prev is null and the parent is none.
__global__ void k_periodic_keep(const uint32_t *__restrict__ cand, const uint32_t *__restrict__ cand_left,
                                const unsigned long long *__restrict__ sup, const long long *__restrict__ per,
                                const uint32_t *__restrict__ pass, const uint64_t *__restrict__ pos, uint64_t n,
                                uint32_t w, const uint32_t *__restrict__ pid_prev,
                                const uint64_t *__restrict__ d_pid_base, uint32_t *__restrict__ L_next,
                                uint32_t *__restrict__ pid_next, uint32_t *__restrict__ pat_parent,
                                uint32_t *__restrict__ pat_item, uint32_t *__restrict__ pat_sup,
                                long long *__restrict__ pat_per) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !pass[i]) return;
    const uint64_t p = pos[i];
    for (uint32_t j = 0; j < w; ++j) L_next[p * w + j] = cand[i * w + j];
    const uint64_t pid = *d_pid_base + p;
    pid_next[p] = (uint32_t)pid;
    pat_parent[pid] = pid_prev ? pid_prev[cand_left[i]] : 0xffffffffu;
    pat_item[pid] = cand[i * w + w - 1];
    pat_sup[pid] = (uint32_t)sup[i];
    pat_per[pid] = per[i];
}

}  // namespace cpm
