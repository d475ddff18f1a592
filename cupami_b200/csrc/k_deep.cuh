// Deep levels: persistent Eclat kernel over a device work queue.
//
// Reference: cuEclat._searchClass (cuEclat.py:211-245) with
// intersect_extensions (_bitsets.py:55-77).  One reference step -- frame F,
// position p: intersect member p with every later member, keep the children
// whose support passes, recurse into them when at least two pass -- is one
// work unit here.  Units run in a persistent kernel: each CTA pops a
// (frame, position) unit from a queue in device memory, stages member p (the
// prefix tidset, ANDed with the frame mask for top-level classes) in shared
// memory, streams the later members with 128-bit loads, ANDs and popcounts
// them with a warp reduction, writes surviving children into a device arena,
// emits their patterns and, when two or more survive, appends a child frame
// and its positions to the queue.  Non-surviving children are written to the
// warp's reusable scratch slot only (overwritten in L2 before eviction).
//
// Every wait is bounded by spin_limit; running out sets CPM_DEEP_ERR_SPIN and
// the kernel returns.  Capacity overflow sets an error bit and stops all CTAs;
// the host then grows the buffers and reruns the round, so output is exact.
#pragma once
#include "common.cuh"

namespace cpm {

enum : unsigned {
    DEEP_ERR_QUEUE = 1u, DEEP_ERR_ARENA = 2u, DEEP_ERR_MEMBERS = 4u, DEEP_ERR_FRAMES = 8u,
    DEEP_ERR_PATTERNS = 16u, DEEP_ERR_SPIN = 32u,
};

constexpr unsigned long long QUEUE_EMPTY = ~0ull;
constexpr uint64_t NO_SLOT = ~0ull;

struct DFrame {
    const uint64_t *mask;  // top-level classes: tidset of the class item; else null
    uint64_t mem_off;      // first member entry
    uint32_t m;            // members
    uint32_t root;         // top-level class this frame descends from
};

// Every counter that CTAs update or poll sits on its own 128-byte line, so
// that claims, allocations and statistics do not serialise on one L2 line.
#define CPM_LINE(name) unsigned long long name; unsigned long long name##_pad[15]
struct DeepState {
    CPM_LINE(q_head);       // next ticket to hand out
    CPM_LINE(q_tail);       // entries reserved by producers
    CPM_LINE(pending);      // units queued or running
    CPM_LINE(n_patterns);
    CPM_LINE(arena_next);
    CPM_LINE(n_frames);
    CPM_LINE(n_members);
    CPM_LINE(intersections);
    CPM_LINE(bytes_alg);
    CPM_LINE(work_items);
    CPM_LINE(survivors);
    unsigned int error;
    unsigned int pad[31];
};
#undef CPM_LINE

struct DeepParams {
    DFrame *frames; uint64_t frames_cap;
    uint32_t *mem_pat; uint32_t *mem_item; const uint64_t **mem_bits; uint64_t members_cap;
    unsigned long long *queue; uint64_t queue_cap;
    uint64_t *arena; uint64_t arena_slots;
    uint32_t *pat_parent; uint32_t *pat_item; uint32_t *pat_sup; uint64_t pat_cap;
    unsigned long long *root_cost;  // per top-level class: intersections in its subtree
    DeepState *st;
    uint64_t stride;                // words per tidset (even)
    long long minsup;
    unsigned long long spin_limit;
};

__device__ __forceinline__ void deep_fail(DeepState *st, unsigned bit) { atomicOr(&st->error, bit); }

// Thread 0 claims the next unit with a ticket: one atomicAdd on the head,
// then a wait on its own queue entry until a producer fills it, or until no
// unit is queued or running (the ticket will never be filled), or an error.
// Returns 0 with *item set, or 1 to stop.
__device__ int deep_claim(const DeepParams &P, unsigned long long *item) {
    DeepState *st = P.st;
    const unsigned long long h = atomicAdd(&st->q_head, 1ull);
    unsigned backoff = 32;  // ns, doubled up to 2 us while waiting
    for (unsigned long long it = 0; it < P.spin_limit; ++it) {
        if (h < P.queue_cap) {
            const unsigned long long v = ld_acquire_u64(P.queue + h);
            if (v != QUEUE_EMPTY) { *item = v; return 0; }
        }
        if ((it & 7) == 0) {
            if (ld_acquire_u32(&st->error)) return 1;
            if (ld_acquire_u64(&st->pending) == 0) return 1;
        }
        __nanosleep(backoff);
        backoff = min(backoff * 2, 2048u);
    }
    deep_fail(st, DEEP_ERR_SPIN);
    return 1;
}

template <bool SMEM_PREFIX>
__global__ void __launch_bounds__(256) k_deep(DeepParams P) {
    extern __shared__ ulonglong2 s_prefix[];
    __shared__ unsigned long long s_item;
    __shared__ int s_stop;
    __shared__ uint32_t s_surv;
    __shared__ unsigned long long s_mem_base;
    __shared__ uint64_t s_pool[32];
    __shared__ int s_pool_n;
    __shared__ unsigned long long s_fid, s_qbase;
    __shared__ int s_ok;

    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint64_t n2 = P.stride / 2;
    DeepState *st = P.st;
    uint64_t my_slot = NO_SLOT;  // warp-uniform scratch slot (kept across units)
    if (threadIdx.x == 0) s_pool_n = 0;
    // Per-CTA statistics (thread 0), added to the global counters at exit.
    unsigned long long c_inter = 0, c_bytes = 0, c_units = 0, c_surv = 0;

    for (;;) {
        if (threadIdx.x == 0) s_stop = deep_claim(P, &s_item);
        __syncthreads();
        if (s_stop) break;
        const uint32_t fid = (uint32_t)(s_item >> 32), p = (uint32_t)s_item;
        DFrame f;
        f.mask = reinterpret_cast<const uint64_t *>(__ldcg(reinterpret_cast<const unsigned long long *>(&P.frames[fid].mask)));
        f.mem_off = __ldcg(reinterpret_cast<const unsigned long long *>(&P.frames[fid].mem_off));
        f.m = __ldcg(&P.frames[fid].m);
        f.root = __ldcg(&P.frames[fid].root);
        const uint32_t cnt = f.m - p - 1;
        const ulonglong2 *pb = reinterpret_cast<const ulonglong2 *>(
            __ldcg(reinterpret_cast<const unsigned long long *>(P.mem_bits + f.mem_off + p)));
        const ulonglong2 *mk = reinterpret_cast<const ulonglong2 *>(f.mask);
        if (SMEM_PREFIX) {
            for (uint64_t v = threadIdx.x; v < n2; v += blockDim.x)
                s_prefix[v] = mk ? and2(ld_cg(pb + v), ld_cg(mk + v)) : ld_cg(pb + v);
        }
        if (threadIdx.x == 0) {
            s_surv = 0;
            const unsigned long long mb = atomicAdd(&st->n_members, (unsigned long long)cnt);
            if (mb + cnt > P.members_cap) deep_fail(st, DEEP_ERR_MEMBERS);
            s_mem_base = mb;
            s_ok = ld_acquire_u32(&st->error) == 0;
        }
        __syncthreads();
        const bool ok = s_ok != 0;
        const uint32_t parent_pat = __ldcg(P.mem_pat + f.mem_off + p);
        for (uint32_t q = wid; ok && q < cnt; q += nw) {
            if (my_slot == NO_SLOT) {
                uint64_t s = NO_SLOT;
                if (lane == 0) {
                    const int k = atomicSub(&s_pool_n, 1) - 1;
                    if (k >= 0) {
                        s = s_pool[k];
                    } else {
                        atomicAdd(&s_pool_n, 1);
                        s = atomicAdd(&st->arena_next, 1ull);
                        if (s >= P.arena_slots) { deep_fail(st, DEEP_ERR_ARENA); s = NO_SLOT; }
                    }
                }
                my_slot = __shfl_sync(CPM_FULL, s, 0);
                if (my_slot == NO_SLOT) break;
            }
            const uint64_t mi = f.mem_off + p + 1 + q;
            const ulonglong2 *sb = reinterpret_cast<const ulonglong2 *>(
                __ldcg(reinterpret_cast<const unsigned long long *>(P.mem_bits + mi)));
            const uint32_t sib_item = __ldcg(P.mem_item + mi);
            ulonglong2 *dst = reinterpret_cast<ulonglong2 *>(P.arena + my_slot * P.stride);
            uint32_t s = 0;
            uint64_t v = lane;
            for (; v + 96 < n2; v += 128) {
                ulonglong2 x0 = ld_cg(sb + v), x1 = ld_cg(sb + v + 32);
                ulonglong2 x2 = ld_cg(sb + v + 64), x3 = ld_cg(sb + v + 96);
                if (SMEM_PREFIX) {
                    x0 = and2(x0, s_prefix[v]); x1 = and2(x1, s_prefix[v + 32]);
                    x2 = and2(x2, s_prefix[v + 64]); x3 = and2(x3, s_prefix[v + 96]);
                } else {
                    x0 = and2(x0, ld_cg(pb + v)); x1 = and2(x1, ld_cg(pb + v + 32));
                    x2 = and2(x2, ld_cg(pb + v + 64)); x3 = and2(x3, ld_cg(pb + v + 96));
                    if (mk) {
                        x0 = and2(x0, ld_cg(mk + v)); x1 = and2(x1, ld_cg(mk + v + 32));
                        x2 = and2(x2, ld_cg(mk + v + 64)); x3 = and2(x3, ld_cg(mk + v + 96));
                    }
                }
                dst[v] = x0; dst[v + 32] = x1; dst[v + 64] = x2; dst[v + 96] = x3;
                s += popc2(x0) + popc2(x1) + popc2(x2) + popc2(x3);
            }
            for (; v < n2; v += 32) {
                ulonglong2 x = ld_cg(sb + v);
                if (SMEM_PREFIX) {
                    x = and2(x, s_prefix[v]);
                } else {
                    x = and2(x, ld_cg(pb + v));
                    if (mk) x = and2(x, ld_cg(mk + v));
                }
                dst[v] = x;
                s += popc2(x);
            }
            s = warp_sum_u32(s);
            if ((long long)s >= P.minsup) {
                if (lane == 0) {
                    const uint32_t idx = atomicAdd(&s_surv, 1u);
                    const uint64_t m_out = s_mem_base + idx;
                    const unsigned long long pid = atomicAdd(&st->n_patterns, 1ull);
                    if (pid >= P.pat_cap) {
                        deep_fail(st, DEEP_ERR_PATTERNS);
                    } else {
                        P.pat_parent[pid] = parent_pat;
                        P.pat_item[pid] = sib_item;
                        P.pat_sup[pid] = s;
                    }
                    if (m_out < P.members_cap) {
                        P.mem_pat[m_out] = (uint32_t)pid;
                        P.mem_item[m_out] = sib_item;
                        P.mem_bits[m_out] = P.arena + my_slot * P.stride;
                    }
                    __threadfence();
                }
                my_slot = NO_SLOT;
            }
        }
        __syncthreads();
        const uint32_t ns = s_surv;
        if (threadIdx.x == 0) {
            s_fid = ~0ull;
            if (ns >= 2 && ld_acquire_u32(&st->error) == 0) {
                const unsigned long long nf = atomicAdd(&st->n_frames, 1ull);
                const unsigned long long qb = atomicAdd(&st->q_tail, (unsigned long long)(ns - 1));
                if (nf >= P.frames_cap) deep_fail(st, DEEP_ERR_FRAMES);
                else if (qb + ns - 1 > P.queue_cap) deep_fail(st, DEEP_ERR_QUEUE);
                else {
                    DFrame c;
                    c.mask = nullptr;
                    c.mem_off = s_mem_base;
                    c.m = ns;
                    c.root = f.root;
                    P.frames[nf] = c;
                    atomicAdd(&st->pending, (unsigned long long)(ns - 1));
                    __threadfence();
                    s_fid = nf;
                    s_qbase = qb;
                }
            } else if (ns == 1 && s_mem_base < P.members_cap && ld_acquire_u32(&st->error) == 0) {
                // The lone survivor's tidset is never read again: recycle it.
                const uint64_t *b = reinterpret_cast<const uint64_t *>(
                    __ldcg(reinterpret_cast<const unsigned long long *>(P.mem_bits + s_mem_base)));
                const uint64_t slot = (uint64_t)(b - P.arena) / P.stride;
                if (s_pool_n < 32) s_pool[s_pool_n++] = slot;
            }
        }
        __syncthreads();
        if (s_fid != ~0ull) {
            for (uint32_t i = threadIdx.x; i + 1 < ns; i += blockDim.x)
                st_release_u64(P.queue + s_qbase + i, (s_fid << 32) | i);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            c_inter += cnt;
            c_bytes += 8ull * P.stride * (1ull + cnt + ns);
            c_units += 1;
            c_surv += ns;
            if (P.root_cost) atomicAdd(P.root_cost + f.root, (unsigned long long)cnt);
            __threadfence();
            atomicAdd(&st->pending, ~0ull);  // pending -= 1
        }
    }
    if (threadIdx.x == 0 && c_units) {
        atomicAdd(&st->intersections, c_inter);
        atomicAdd(&st->bytes_alg, c_bytes);
        atomicAdd(&st->work_items, c_units);
        atomicAdd(&st->survivors, c_surv);
    }
}

}  // namespace cpm
