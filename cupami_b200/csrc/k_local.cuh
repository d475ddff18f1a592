// Projected deep levels: a persistent kernel with one warp per unit.
//
// Reference: the same step as k_deep -- cuEclat._searchClass
// (cuEclat.py:211-245) with intersect_extensions (_bitsets.py:55-77): unit
// (F, p) intersects member p of frame F with every later member, keeps the
// children whose support reaches the threshold and recurses into them when
// two or more pass.
//
// k_deep hands over every frame whose prefix held at most LOCAL_MAX_BITS
// transactions, with its members written as bitsets of that many bits,
// numbered by rank within the prefix (k_deep.cuh, build_rank_dir).  A
// descendant of such a frame only loses transactions, so it keeps the same
// numbering and size: every tidset of the subtree is at most 8 KB (2 KB
// below 16,384 transactions, when the prefix is staged in the warp's slot of
// shared memory), the members of a frame lie side by side in one arena
// block (member q at bits + q * stride), and no unit needs more.  One
// warp runs a unit from claim to publication without a block barrier, so
// each SM keeps dozens of units' dependent L2 round trips in flight instead
// of one.
//
// A unit: the prefix is staged in the warp's slot of shared memory; the
// later members are streamed, G lanes per member (G the power of two covering a tidset, up to
// 32), several members per step; AND, popcount and a group sum give each
// support.  Pass 1 only counts the survivors.  With one survivor its pattern
// is written from what pass 1 kept; with two or more the unit reserves its
// pattern ids, member entries and child block at once and pass 2 recounts
// (the tidsets are a few hundred bytes and in L2), writing each survivor's
// pattern, member entry and child tidset in member order.  The child frame's
// units join the same queue.  Waits are bounded by spin_limit, and capacity
// overflows set the same error bits as k_deep, after which the host reruns.
#pragma once
#include "k_deep.cuh"

namespace cpm {

// Largest projected prefix, in transactions: ranks (and the rank directory
// of k_deep) are 16-bit, and a tidset is at most 511 16-byte words.
constexpr uint32_t LOCAL_MAX_BITS = 65536 - 128;
// Tidsets of at most this many 16-byte words (16,384 transactions) are
// staged in the warp's shared-memory slot, four words per lane at most.
constexpr uint32_t LOCAL_SLOT_W2 = 128;
constexpr uint32_t LOCAL_BLOCK = 256;

// Sum over an aligned group of G lanes (G a power of two, the same on every lane).
__device__ __forceinline__ uint32_t group_sum(uint32_t c, uint32_t G) {
    for (uint32_t o = G >> 1; o; o >>= 1) c += __shfl_xor_sync(CPM_FULL, c, o);
    return c;
}

// Lane 0 claims the next projected unit: a ticket, then a bounded wait for
// its queue entry, or until no projected unit is queued or running, or an
// error.  Returns 0 with *item set, or 1 to stop.
__device__ int local_claim(const DeepParams &P, unsigned long long *item) {
    DeepState *st = P.st;
    const unsigned long long h = atomicAdd(&st->lq_head, 1ull);
    unsigned backoff = 32;
    for (unsigned long long it = 0; it < P.spin_limit; ++it) {
        if (h < P.lq_cap) {
            const unsigned long long v = ld_acquire_u64(P.lq + h);
            if (v != QUEUE_EMPTY) {
                *item = v;
                return 0;
            }
        }
        if ((it & 7) == 0) {
            if (ld_acquire_u32(&st->error)) return 1;
            if (ld_acquire_u64(&st->lq_pending) == 0) return 1;
        }
        __nanosleep(backoff);
        backoff = min(backoff * 2, 2048u);
    }
    deep_fail(st, DEEP_ERR_SPIN);
    return 1;
}

// One claimed unit, as every lane of the warp sees it.
struct LocalUnit {
    const ulonglong2 *base;  // member 0's tidset
    uint64_t mem_off;
    uint32_t m, p, w2, root, db;
    long long minsup;
};

struct LocalCounters {
    unsigned long long inter, bytes, units, surv;
};

// Lane 0 reserves ns pattern ids, member entries and a child block of
// child_words for a unit with two or more survivors; every lane gets them.
// False (an error bit set) when a table is full.
__device__ __forceinline__ bool local_reserve(const DeepParams &P, uint32_t ns, unsigned long long child_words,
                                              unsigned long long *pid0, unsigned long long *mb,
                                              unsigned long long *ab) {
    DeepState *st = P.st;
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
        *pid0 = atomicAdd(&st->n_patterns, (unsigned long long)ns);
        *mb = atomicAdd(&st->n_members, (unsigned long long)ns);
        *ab = atomicAdd(&st->arena_next, child_words);
        if (*pid0 + ns > P.pat_cap) { deep_fail(st, DEEP_ERR_PATTERNS); ok = 0; }
        if (*mb + ns > P.members_cap) { deep_fail(st, DEEP_ERR_MEMBERS); ok = 0; }
        if (*ab + child_words > P.arena_words) { deep_fail(st, DEEP_ERR_ARENA); ok = 0; }
    }
    ok = __shfl_sync(CPM_FULL, ok, 0);
    *pid0 = __shfl_sync(CPM_FULL, *pid0, 0);
    *mb = __shfl_sync(CPM_FULL, *mb, 0);
    *ab = __shfl_sync(CPM_FULL, *ab, 0);
    return ok != 0;
}

// Survivor idx of a unit: its pattern record and member entry (one lane).
__device__ __forceinline__ void local_emit(const DeepParams &P, const LocalUnit &u, uint32_t parent_pat,
                                           uint32_t item, uint32_t sup, unsigned long long pid, unsigned long long mb,
                                           uint32_t idx, const ulonglong2 *child) {
    P.pat_parent[pid] = parent_pat;
    P.pat_item[pid] = item;
    P.pat_sup[pid] = sup;
    if (P.pat_db) P.pat_db[pid] = u.db;
    P.mem_pat[mb + idx] = (uint32_t)pid;
    P.mem_item[mb + idx] = item;
    P.mem_bits[mb + idx] = reinterpret_cast<const uint64_t *>(child);
}

// The child frame of ns survivors (members mb.., tidsets at out, 2 * W2
// words each): published by lane 0, its ns - 1 units queued by the warp.
__device__ __forceinline__ void local_publish(const DeepParams &P, const LocalUnit &u, uint32_t ns,
                                              unsigned long long mb, const ulonglong2 *out, uint32_t W2) {
    DeepState *st = P.st;
    const unsigned lane = threadIdx.x & 31;
    __syncwarp();
    unsigned long long nf = 0, qb = 0;
    int pub = 0;
    if (lane == 0) {
        nf = atomicAdd(&st->n_frames, 1ull);
        qb = atomicAdd(&st->lq_tail, (unsigned long long)(ns - 1));
        if (nf >= P.frames_cap) {
            deep_fail(st, DEEP_ERR_FRAMES);
        } else if (qb + ns - 1 > P.lq_cap) {
            deep_fail(st, DEEP_ERR_QUEUE);
        } else {
            DFrame c;
            c.mask = nullptr;
            c.mem_off = mb;
            c.m = ns;
            c.root = u.root;
            c.stride = 2u * W2;
            c.db = u.db;
            c.minsup = u.minsup;
            c.bits = reinterpret_cast<const uint64_t *>(out);
            P.frames[nf] = c;
            // Its units count as pending before this unit leaves lq_pending.
            atomicAdd(&st->lq_pending, (unsigned long long)(ns - 1));
            __threadfence();
            pub = 1;
        }
    }
    __syncwarp();
    pub = __shfl_sync(CPM_FULL, pub, 0);
    if (!pub) return;
    nf = __shfl_sync(CPM_FULL, nf, 0);
    qb = __shfl_sync(CPM_FULL, qb, 0);
    for (uint32_t i = lane; i + 1 < ns; i += 32) st_release_u64(P.lq + qb + i, (nf << 32) | i);
}

// The unit, with K 16-byte words of a tidset per lane (K = 1 for tidsets of
// at most 32 words, each spread over a group of G lanes; else G = 32) and U
// steps of NG = 32 / G members each loaded before they are reduced.
template <int K>
__device__ __forceinline__ void local_unit(const DeepParams &P, const LocalUnit &u, unsigned lane,
                                           ulonglong2 *s_pre, LocalCounters &cs) {
    constexpr int U = K == 1 ? 4 : K == 2 ? 2 : 1;
    DeepState *st = P.st;
    const uint32_t W2 = u.w2;
    const uint32_t lg = W2 >= 32 ? 5u : (W2 <= 1 ? 0u : 32u - (uint32_t)__clz(W2 - 1u));
    const uint32_t G = 1u << lg, NG = 32u >> lg, gi = lane >> lg, gl = lane & (G - 1u);
    const uint32_t cnt = u.m - u.p - 1;
    const ulonglong2 *pre2 = u.base + (uint64_t)u.p * W2;
    const ulonglong2 *sib0 = pre2 + W2;  // later member q (from 0) at sib0 + q * W2
    const ulonglong2 zero = make_ulonglong2(0ull, 0ull);
    // The prefix, staged in this warp's slot of shared memory.
    for (uint32_t j = lane; j < W2; j += 32) s_pre[j] = ld_cg(pre2 + j);
    __syncwarp();
    const uint32_t parent_pat = __ldcg(P.mem_pat + u.mem_off + u.p);
    const uint64_t item_off = u.mem_off + u.p + 1;

    // Support of later member q0 + v * NG + gi on every lane of its group.
    auto step_load = [&](uint32_t q0, ulonglong2 (&x)[U][K]) {
#pragma unroll
        for (int v = 0; v < U; ++v) {
            const uint32_t q = q0 + v * NG + gi;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const uint32_t j = gl + G * k;
                x[v][k] = (q < cnt && j < W2) ? ld_cg(sib0 + (uint64_t)q * W2 + j) : zero;
            }
        }
    };
    auto support = [&](const ulonglong2 (&xv)[K]) {
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (gl + G * k < W2) c += popc2(and2(xv[k], s_pre[gl + G * k]));
        return group_sum(c, G);
    };

    // ---- pass 1: count the survivors, keep the last one ----
    uint32_t ns = 0, last_q = 0, last_c = 0;
    for (uint32_t q0 = 0; q0 < cnt; q0 += NG * U) {
        ulonglong2 x[U][K];
        step_load(q0, x);
#pragma unroll
        for (int v = 0; v < U; ++v) {
            const uint32_t q = q0 + v * NG + gi;
            const uint32_t c = support(x[v]);
            const bool sv = q < cnt && (long long)c >= u.minsup;
            const unsigned bal = __ballot_sync(CPM_FULL, sv && gl == 0);
            if (bal) {
                ns += __popc(bal);
                const int L = 31 - __clz(bal);
                last_q = __shfl_sync(CPM_FULL, q, L);
                last_c = __shfl_sync(CPM_FULL, c, L);
            }
        }
    }
    if (lane == 0) {
        cs.inter += cnt;
        cs.bytes += 16ull * W2 * (cnt + 1ull);
        cs.units += 1;
        cs.surv += ns;
    }
    if (P.root_cost && lane == 0) atomicAdd(P.root_cost + u.root, (unsigned long long)cnt);
    if (ns == 0) return;
    if (ns == 1) {
        if (lane == 0) {
            const unsigned long long pid = atomicAdd(&st->n_patterns, 1ull);
            if (pid >= P.pat_cap) {
                deep_fail(st, DEEP_ERR_PATTERNS);
            } else {
                P.pat_parent[pid] = parent_pat;
                P.pat_item[pid] = __ldcg(P.mem_item + item_off + last_q);
                P.pat_sup[pid] = last_c;
                if (P.pat_db) P.pat_db[pid] = u.db;
            }
        }
        return;
    }
    // ---- two or more survivors: reserve, then pass 2 writes them in order ----
    const unsigned long long child_words = 2ull * W2 * ns;
    unsigned long long pid0 = 0, mb = 0, ab = 0;
    if (!local_reserve(P, ns, child_words, &pid0, &mb, &ab)) return;
    ulonglong2 *out = reinterpret_cast<ulonglong2 *>(P.arena + ab);
    uint32_t run = 0;
    for (uint32_t q0 = 0; q0 < cnt; q0 += NG * U) {
        ulonglong2 x[U][K];
        step_load(q0, x);
#pragma unroll
        for (int v = 0; v < U; ++v) {
            const uint32_t q = q0 + v * NG + gi;
            const uint32_t c = support(x[v]);
            const bool sv = q < cnt && (long long)c >= u.minsup;
            const unsigned bal = __ballot_sync(CPM_FULL, sv && gl == 0);
            const uint32_t idx = run + __popc(bal & ((1u << (gi * G)) - 1u));
            if (sv && idx < ns) {
                ulonglong2 *o = out + (uint64_t)idx * W2;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const uint32_t j = gl + G * k;
                    if (j < W2) o[j] = and2(x[v][k], s_pre[j]);
                }
                if (gl == 0)
                    local_emit(P, u, parent_pat, __ldcg(P.mem_item + item_off + q), c, pid0 + idx, mb, idx, o);
            }
            run += __popc(bal);
        }
    }
    if (lane == 0) cs.bytes += 8ull * child_words;
    // The two passes read the same words: they must agree.
    if (run != ns) {
        if (lane == 0) deep_fail(st, DEEP_ERR_INTERNAL);
        return;
    }
    local_publish(P, u, ns, mb, out, W2);
}

// A unit of a frame whose tidsets exceed a warp's shared-memory slot (more
// than LOCAL_SLOT_W2 16-byte words): one later member at a time over the
// whole warp, prefix words read with it from L2 (eight loads in flight per lane).
__device__ __forceinline__ void local_unit_wide(const DeepParams &P, const LocalUnit &u, unsigned lane,
                                             LocalCounters &cs) {
    DeepState *st = P.st;
    const uint32_t W2 = u.w2, cnt = u.m - u.p - 1;
    const ulonglong2 *pre2 = u.base + (uint64_t)u.p * W2;
    const ulonglong2 *sib0 = pre2 + W2;
    const ulonglong2 zero = make_ulonglong2(0ull, 0ull);
    const uint32_t parent_pat = __ldcg(P.mem_pat + u.mem_off + u.p);
    const uint64_t item_off = u.mem_off + u.p + 1;
    auto count = [&](uint32_t q) {
        const ulonglong2 *sb = sib0 + (uint64_t)q * W2;
        uint32_t c = 0;
        for (uint32_t j0 = 0; j0 < W2; j0 += 128) {
            ulonglong2 a[4], b[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t j = j0 + lane + 32 * k;
                a[k] = j < W2 ? ld_cg(sb + j) : zero;
                b[k] = j < W2 ? ld_cg(pre2 + j) : zero;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) c += popc2(and2(a[k], b[k]));
        }
        return warp_sum_u32(c);
    };
    uint32_t ns = 0, last_q = 0, last_c = 0;
    for (uint32_t q = 0; q < cnt; ++q) {
        const uint32_t c = count(q);
        if ((long long)c >= u.minsup) {
            ++ns;
            last_q = q;
            last_c = c;
        }
    }
    if (lane == 0) {
        cs.inter += cnt;
        cs.bytes += 16ull * W2 * (cnt + 1ull);
        cs.units += 1;
        cs.surv += ns;
    }
    if (P.root_cost && lane == 0) atomicAdd(P.root_cost + u.root, (unsigned long long)cnt);
    if (ns == 0) return;
    if (ns == 1) {
        if (lane == 0) {
            const unsigned long long pid = atomicAdd(&st->n_patterns, 1ull);
            if (pid >= P.pat_cap) {
                deep_fail(st, DEEP_ERR_PATTERNS);
            } else {
                P.pat_parent[pid] = parent_pat;
                P.pat_item[pid] = __ldcg(P.mem_item + item_off + last_q);
                P.pat_sup[pid] = last_c;
                if (P.pat_db) P.pat_db[pid] = u.db;
            }
        }
        return;
    }
    const unsigned long long child_words = 2ull * W2 * ns;
    unsigned long long pid0 = 0, mb = 0, ab = 0;
    if (!local_reserve(P, ns, child_words, &pid0, &mb, &ab)) return;
    ulonglong2 *out = reinterpret_cast<ulonglong2 *>(P.arena + ab);
    uint32_t run = 0;
    for (uint32_t q = 0; q < cnt && run < ns; ++q) {
        const uint32_t c = count(q);
        if ((long long)c < u.minsup) continue;
        const ulonglong2 *sb = sib0 + (uint64_t)q * W2;
        ulonglong2 *o = out + (uint64_t)run * W2;
        for (uint32_t j = lane; j < W2; j += 32) o[j] = and2(ld_cg(sb + j), ld_cg(pre2 + j));
        if (lane == 0) local_emit(P, u, parent_pat, __ldcg(P.mem_item + item_off + q), c, pid0 + run, mb, run, o);
        ++run;
    }
    if (lane == 0) cs.bytes += 8ull * child_words;
    if (run != ns) {
        if (lane == 0) deep_fail(st, DEEP_ERR_INTERNAL);
        return;
    }
    local_publish(P, u, ns, mb, out, W2);
}

__global__ void __launch_bounds__(LOCAL_BLOCK, 4) k_local(DeepParams P) {
    const unsigned lane = threadIdx.x & 31;
    DeepState *st = P.st;
    // Per-warp statistics (lane 0), in shared memory rather than registers.
    __shared__ LocalCounters s_cs[LOCAL_BLOCK / 32];
    LocalCounters &cs = s_cs[threadIdx.x >> 5];
    if (lane == 0) cs = LocalCounters{0, 0, 0, 0};
    __shared__ ulonglong2 s_pre_all[LOCAL_BLOCK / 32][LOCAL_SLOT_W2];
    ulonglong2 *const s_pre = s_pre_all[threadIdx.x >> 5];
    for (;;) {
        unsigned long long item = 0;
        int stop = 0;
        if (lane == 0) {
            stop = local_claim(P, &item);
            // After an error nothing more is done: the host reruns the launch.
            if (!stop && ld_relaxed_u32(&st->error)) stop = 1;
        }
        stop = __shfl_sync(CPM_FULL, stop, 0);
        if (stop) break;
        item = __shfl_sync(CPM_FULL, item, 0);
        const DFrame *fp = P.frames + (uint32_t)(item >> 32);
        LocalUnit u;
        u.base = reinterpret_cast<const ulonglong2 *>(__ldcg(reinterpret_cast<const unsigned long long *>(&fp->bits)));
        u.mem_off = __ldcg(reinterpret_cast<const unsigned long long *>(&fp->mem_off));
        u.m = __ldcg(&fp->m);
        u.p = (uint32_t)item;
        u.w2 = __ldcg(&fp->stride) / 2u;
        u.root = __ldcg(&fp->root);
        u.db = __ldcg(&fp->db);
        u.minsup = __ldcg(&fp->minsup);
        if (!u.base || u.w2 == 0 || u.w2 > (LOCAL_MAX_BITS + 127) / 128 || u.p + 1 >= u.m) {
            if (lane == 0) deep_fail(st, DEEP_ERR_INTERNAL);
            break;
        }
        const uint32_t K = u.w2 > 32 ? (u.w2 + 31) / 32 : 1u;
        if (u.w2 > LOCAL_SLOT_W2) local_unit_wide(P, u, lane, cs);
        else if (K == 1) local_unit<1>(P, u, lane, s_pre, cs);
        else if (K == 2) local_unit<2>(P, u, lane, s_pre, cs);
        else if (K == 3) local_unit<3>(P, u, lane, s_pre, cs);
        else local_unit<4>(P, u, lane, s_pre, cs);
        // Any child frame was published (fenced) above; its units were added
        // to lq_pending before this unit leaves it.
        if (lane == 0) atomicAdd(&st->lq_pending, ~0ull);  // lq_pending -= 1
        __syncwarp();  // the prefix slot is free for the next unit
    }
    if (lane == 0 && cs.units) {
        atomicAdd(&st->intersections, cs.inter);
        atomicAdd(&st->bytes_alg, cs.bytes);
        atomicAdd(&st->work_items, cs.units);
        atomicAdd(&st->local_units, cs.units);
        atomicAdd(&st->survivors, cs.surv);
    }
}

}  // namespace cpm
