// Periodic-frequent support counting (cupami/periodicFrequentPattern/_temporal.py:26-53).
//
// For an itemset X held by the rows r_1 < ... < r_s of a temporal database
// whose rows are sorted by timestamp ts[], the reference kernel returns the
// support s and the periodicity
//     max(0, ts[r_1] - 0, ts[r_2] - ts[r_1], ..., ts[r_s] - ts[r_{s-1}], end - ts[r_s])
// (max(0, end) when s = 0; the 0 is the reference scan's starting value and
// only matters for unsorted or negative inputs), scanning the set bits of the
// AND of X's rows in order with one thread per candidate (_temporal.py:26-53,
// launch :156-165).
//
// Here one warp handles a candidate: per step its lanes load 32 * 4
// consecutive words of each of the candidate's rows (coalesced), each lane
// scans the set rows of its 4 words in order, and the gaps that cross lane and
// step boundaries come from a ballot and one shuffle per step; only the
// largest gap needs a warp reduction, once at the end.  When a level has too
// few candidates to fill the GPU, each candidate's rows are split over several
// warps, each summarising its rows as (count, first and last timestamp,
// largest inner gap), and k_periodic_join joins the summaries in row order
// with the associative join
//     (a, b) -> {a.cnt + b.cnt, a.first, b.last, max(a.gap, b.gap, b.first - a.last)}
// (an empty side yields the other).  With kPrune (the miner), a candidate
// stops as soon as a gap is already too long -- rows are sorted by timestamp,
// so the next set row's gap is at least ts[first unscanned row] - last
// timestamp seen.
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

__device__ __forceinline__ unsigned word_low(uint32_t x) { return __ffs(x) - 1; }
__device__ __forceinline__ unsigned word_low(unsigned long long x) { return __ffsll(x) - 1; }

// Words a lane loads per step (independent loads in flight); a step of a
// warp covers PERIODIC_TILE consecutive words.
constexpr unsigned PERIODIC_PL = 4;
constexpr uint64_t PERIODIC_TILE = 32 * PERIODIC_PL;

// `parts` warps per candidate c (warp g: candidate g / parts, part g % parts),
// each over an equal share of the steps: the AND of the width rows
// cand[c * width ..] of `bits` (Word: uint32_t or unsigned long long; rows of
// `stride` words; bit b of word v is row v * bits(Word) + b), restricted to
// rows < n_tx.  Per step lane l takes the PERIODIC_PL words at
// base + PERIODIC_PL * l (coalesced) and scans their set rows in order.  The
// warp needs no ordered reduction per step: every lane keeps the running
// count, first and last timestamp of the rows scanned so far (identical on all
// lanes) and its own running maximum of the gaps it has seen -- inside its
// words, and from the previous set row (the last set row of the nearest lower
// lane with one, found by a ballot and one shuffle, or of an earlier step) to
// its first -- and the maxima are reduced once at the end.
// With parts = 1 the warp writes support[c] and period[c] (and, with kPrune,
// pass[c] = ok_flag[c] && support >= need && period <= max_per); with
// parts > 1 each warp writes its summary to seg[c * parts + part] and
// k_periodic_join finishes.  With kPrune a warp stops as soon as its rows
// prove the candidate fails: a gap already above max_per (a stretch without
// set rows from row a to row b gives a gap of at least ts[b] - ts[a - 1];
// timestamps are nonnegative and sorted).  A stopped candidate has pass = 0,
// a stopped part reports gap = LLONG_MAX; only passing candidates have exact
// values.  Without kPrune every candidate is exact.
template <class Word, bool kPrune>
__global__ void __launch_bounds__(256)
k_periodic(const Word *__restrict__ bits, uint64_t stride, const uint32_t *__restrict__ cand,
           const uint32_t *__restrict__ ok_flag, uint64_t n, uint32_t width, const long long *__restrict__ ts,
           uint64_t n_tx, long long end, long long need, long long max_per, uint32_t parts, PSeg *__restrict__ seg,
           unsigned long long *__restrict__ support, long long *__restrict__ period, uint32_t *__restrict__ pass) {
    constexpr unsigned B = sizeof(Word) * 8;
    constexpr unsigned PL = PERIODIC_PL;
    constexpr uint64_t TILE = PERIODIC_TILE;
    const uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    const uint64_t c = g / parts;
    const uint32_t part = (uint32_t)(g % parts);
    if (c >= n) return;  // whole warps: c is the same on every lane
    if (ok_flag && !ok_flag[c]) {
        if (parts == 1 && !lane) {
            support[c] = 0;
            period[c] = max(0ll, end);
            if (pass) pass[c] = 0;
        }
        return;
    }
    const uint32_t *cc = cand + c * width;
    const uint64_t words = (n_tx + B - 1) / B;
    const uint64_t tiles = (words + TILE - 1) / TILE;
    const uint64_t t0 = tiles * part / parts, t1 = tiles * (part + 1) / parts;
    const uint64_t row_lo = t0 * TILE * B;  // first row of this part (< n_tx when t0 < tiles)
    const long long before = row_lo ? __ldg(ts + row_lo - 1) : 0;
    unsigned long long run_cnt = 0;  // rows scanned so far: the same on every lane
    long long run_first = 0, run_last = 0;
    long long gmax = 0;              // this lane's largest gap seen
    bool stopped = false;
    for (uint64_t base = t0 * TILE; base < t1 * TILE; base += TILE) {
        const uint64_t v0 = base + (uint64_t)lane * PL;
        Word x[PL];
#pragma unroll
        for (unsigned q = 0; q < PL; ++q) x[q] = v0 + q < words ? ~Word(0) : Word(0);
        for (uint32_t j = 0; j < width; ++j) {
            const Word *row = bits + (uint64_t)cc[j] * stride;
#pragma unroll
            for (unsigned q = 0; q < PL; ++q)
                if (v0 + q < words) x[q] &= __ldg(row + v0 + q);
        }
        unsigned lc = 0;  // this lane's set rows in this step
        long long lf = 0, ll = 0;
#pragma unroll
        for (unsigned q = 0; q < PL; ++q) {
            const uint64_t row0 = (v0 + q) * B;
            if (v0 + q < words && n_tx - row0 < B) x[q] &= (Word(1) << (unsigned)(n_tx - row0)) - Word(1);
            // One timestamp load per set row, four set rows at a time: the
            // loads are issued before their gaps are taken, so dense words
            // do not wait on one load after another.
            for (Word y = x[q]; y;) {
                long long t[4];
                unsigned m = 0;
#pragma unroll
                for (unsigned u = 0; u < 4; ++u)
                    if (y) {
                        t[u] = __ldg(ts + row0 + word_low(y));
                        y &= y - Word(1);
                        m = u + 1;
                    }
#pragma unroll
                for (unsigned u = 0; u < 4; ++u)
                    if (u < m) {
                        if (lc) gmax = max(gmax, t[u] - ll);
                        else lf = t[u];
                        ll = t[u];
                        ++lc;
                    }
            }
        }
        const unsigned mask = __ballot_sync(CPM_FULL, lc != 0);
        if (mask) {
            const unsigned below = mask & ((1u << lane) - 1u);
            const int src = below ? 31 - __clz(below) : (int)lane;
            const long long prev = __shfl_sync(CPM_FULL, ll, src);  // last set row of the nearest lower lane
            if (lc) {
                if (below) gmax = max(gmax, lf - prev);
                else if (run_cnt) gmax = max(gmax, lf - run_last);
            }
            const long long step_first = __shfl_sync(CPM_FULL, lf, __ffs(mask) - 1);
            run_last = __shfl_sync(CPM_FULL, ll, 31 - __clz(mask));
            if (!run_cnt) run_first = step_first;
            run_cnt += __reduce_add_sync(CPM_FULL, lc);
        }
        if (kPrune) {
            bool bad = gmax > max_per;
            if (!lane) {
                const uint64_t scanned = (base + TILE) * (uint64_t)B;
                const uint64_t r_end = scanned < n_tx ? scanned : n_tx;
                const long long next = r_end < n_tx ? __ldg(ts + r_end) : end;
                const long long bound = run_cnt ? max(run_first - before, next - run_last) : next - before;
                bad = bad || bound > max_per;
            }
            if (__any_sync(CPM_FULL, bad)) {
                stopped = true;
                break;
            }
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) gmax = max(gmax, __shfl_xor_sync(CPM_FULL, gmax, o));
    if (lane) return;
    if (parts == 1) {
        const long long per = run_cnt ? max(max(run_first, gmax), end - run_last) : max(0ll, end);
        support[c] = run_cnt;
        period[c] = per;
        if (kPrune) pass[c] = !stopped && (long long)run_cnt >= need && per <= max_per ? 1u : 0u;
    } else {
        PSeg out{run_cnt, run_first, run_last, gmax};
        if (stopped) {
            out.cnt = out.cnt ? out.cnt : 1;
            out.gap = 0x7fffffffffffffffll;
        }
        seg[c * parts + part] = out;
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
        period[c] = max(0ll, end);
        if (pass) pass[c] = 0;
        return;
    }
    PSeg run{0, 0, 0, 0};
    for (uint32_t p = 0; p < parts; ++p) run = pseg_join(run, seg[c * parts + p]);
    const long long per = run.cnt ? max(max(run.first, run.gap), end - run.last) : max(0ll, end);
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
