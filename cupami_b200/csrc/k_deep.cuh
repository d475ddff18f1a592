// Deep levels: persistent Eclat kernel over a device work queue.
//
// Reference: cuEclat._searchClass (cuEclat.py:211-245) with
// intersect_extensions (_bitsets.py:55-77).  One reference step -- frame F,
// position p: intersect member p with every later member, keep the children
// whose support passes, recurse into them when at least two pass -- is one
// work unit here.  Units run in a persistent kernel: each CTA pops a
// (frame, position) unit from a queue in device memory, stages member p (the
// prefix tidset, ANDed with the frame mask for top-level classes) in shared
// memory and streams the later members with 128-bit loads, AND and popcount
// per warp (pass 1).  Child tidsets are written only when a child frame will
// exist (two or more survivors): one exact-size arena block per unit, filled
// by a second pass over the survivors' siblings (pass 2, mostly L2 hits).  A
// unit with one survivor writes nothing but its pattern record.
//
// Frames carry their database's tidset stride, threshold and id, so one launch
// can mine many databases of different sizes at once.
//
// Tidsets come in two forms, told apart by bit 0 of the member pointer.
// Dense: `stride` 64-bit words, bit r of word r/64 set when transaction r
// holds the pattern.  List (bit 0 set): a 16-byte header whose first uint32 is
// the count n, then the n transaction ids in ascending order, padded to a
// 16-byte multiple.  At one bit per transaction a bitset is the smaller form
// until fewer than one transaction in 32 holds the pattern; below that (list
// at most the dense size, by default) children are written as lists, and frequent
// items that sparse serve as list members of the top-level classes.  The
// prefix of a unit is always staged as a dense bitmap in shared memory; a
// list sibling is intersected by testing its ids against that bitmap.  Lists
// are used only when the prefix fits in shared memory (P.lists).
//
// Every wait is bounded by spin_limit; running out sets DEEP_ERR_SPIN and the
// kernel returns.  Capacity overflow sets an error bit and stops all CTAs; the
// host then grows the buffers and reruns, so the output is exact.
#pragma once
#include "common.cuh"

namespace cpm {

enum : unsigned {
    DEEP_ERR_QUEUE = 1u, DEEP_ERR_ARENA = 2u, DEEP_ERR_MEMBERS = 4u, DEEP_ERR_FRAMES = 8u,
    DEEP_ERR_PATTERNS = 16u, DEEP_ERR_SPIN = 32u, DEEP_ERR_INTERNAL = 64u,
};

// 64-bit words of a list of n transaction ids (16-byte header, 16-byte padding).
__host__ __device__ __forceinline__ uint64_t list_words(uint64_t n) { return (n + 7) / 4 * 2; }

// Largest prefix bitmap (bytes) staged in shared memory: the kernel's static
// shared memory (about 30 KB) and this fit in the 227 KB a CTA may use.
constexpr size_t DEEP_SMEM_PREFIX_MAX = 192 * 1024;

constexpr unsigned long long QUEUE_EMPTY = ~0ull;
// try_wait rounds for a bulk-staged prefix (a copy of at most 192 KB: micro-
// seconds); running out is an error, not a normal wait.
constexpr unsigned long long BULK_WAIT_LIMIT = 1ull << 24;
// Prefixes of at least this many 16-byte words (64 KB) are bulk-copied;
// shorter ones are loaded by all the threads, which measured as fast or
// faster (dense 65,536 x 128: 0.895 ms with thread loads, 0.920 ms bulk;
// planted 100,000 x 1,000: 0.238 / 0.244 ms).
constexpr uint64_t BULK_MIN_WORDS2 = 4096;
constexpr uint32_t NO_PATTERN = 0xffffffffu;

struct DFrame {
    const uint64_t *mask;  // top-level classes: tidset of the class item; else null
    uint64_t mem_off;      // first member entry
    uint32_t m;            // members
    uint32_t root;         // top-level frames: id of their first root unit (unit p has id root + p);
                           // deeper frames: the root unit whose subtree they belong to
    uint32_t stride;       // words per tidset in this frame's database (even)
    uint32_t db;           // database index within the batch
    long long minsup;      // that database's threshold
    // Projected frames only (null otherwise): the members' tidsets, each
    // `stride` words, member q at bits + q * stride.  Their transactions are
    // numbered by rank within the tidset of the unit that made the frame.
    const uint64_t *bits = nullptr;
};

// Every counter that CTAs update or poll sits on its own 128-byte line, so
// that claims, allocations and statistics do not serialise on one L2 line.
#define CPM_LINE(name) unsigned long long name; unsigned long long name##_pad[15]
struct DeepState {
    CPM_LINE(q_head);       // next ticket to hand out
    CPM_LINE(q_tail);       // entries reserved by producers
    CPM_LINE(pending);      // units queued or running
    CPM_LINE(n_patterns);
    CPM_LINE(arena_next);   // words handed out
    CPM_LINE(n_frames);
    CPM_LINE(n_members);
    CPM_LINE(intersections);
    CPM_LINE(bytes_alg);
    CPM_LINE(work_items);
    CPM_LINE(survivors);
    CPM_LINE(n_deferred);   // root units handed back to the host (memory-bounded rounds)
    CPM_LINE(admitted);     // predicted cost of the root units started (memory-bounded rounds)
    CPM_LINE(lq_head);      // projected units: next ticket (k_local)
    CPM_LINE(lq_tail);      // projected units: entries reserved
    CPM_LINE(lq_pending);   // projected units queued or running
    CPM_LINE(local_units);  // projected units run
    CPM_LINE(h_units);      // row-wise units run
    unsigned int error;
    unsigned int pad[31];
};
#undef CPM_LINE

struct DeepParams {
    DFrame *frames; uint64_t frames_cap;
    uint32_t *mem_pat; uint32_t *mem_item; const uint64_t **mem_bits; uint64_t members_cap;
    unsigned long long *queue; uint64_t queue_cap;
    uint64_t *arena; uint64_t arena_words;
    uint32_t *pat_parent; uint32_t *pat_item; uint32_t *pat_sup; uint32_t *pat_db; uint64_t pat_cap;
    unsigned long long *root_cost;  // per root unit: intersections in its subtree (null: not kept)
    DeepState *st;
    uint64_t max_stride;            // largest frame stride (shared-memory prefix size)
    unsigned long long spin_limit;
    unsigned long long *cta_time;   // optional [2 * grid]: busy ns, exit time (globaltimer)
    uint32_t shallow;               // 1: child frames are recorded, not queued
    uint32_t balance;               // pass 1: 0 a warp per sibling; 1 siblings split over warps by size
    uint32_t prefetch;              // 1: take the next queue ticket early when units are waiting
    uint32_t lists;                 // list-form threshold divisor (0: bitsets only; needs SMEM_PREFIX)
    // Memory-bounded rounds: a unit of a frame below root_frames (a root
    // unit) claimed while the arena, the member table or the frame table has
    // (or the queue) has reached its hand-back level is not run but handed back in deferred[]
    // for a later round (defer_words 0: never).
    uint32_t root_frames;
    unsigned long long defer_words, defer_members, defer_frames, defer_queue;
    unsigned long long *deferred;
    uint64_t deferred_cap;
    // Admission by predicted size (rounds only): a root unit of a top-level
    // frame (below top_frames) costs root_key[unit] (times the frame's stride
    // when keys count members); a unit whose cost would take the round's sum
    // past admit_words is handed back, unless it is the round's first.
    const float *root_key;
    uint32_t top_frames, keys_in_words;
    unsigned long long admit_words;
    // Diagnostics (null: off): per unit, UNIT_LOG_WORDS words -- claim,
    // prefix-staged, pass-1-done and end times (globaltimer ns), CTA,
    // siblings | survivors << 32, sibling bytes, largest sibling's bytes,
    // prefix bytes | list prefix << 63 | top-level << 62 | row-wise << 61, then the times the
    // survivors were compacted, the child block granted and the children
    // written (0 for units that end after pass 1).
    // unit_log[0] counts the units logged; records start at unit_log + 1.
    unsigned long long *unit_log;
    unsigned long long unit_log_cap;
    // Projection (0: off; needs SMEM_PREFIX and !shallow): a unit whose
    // prefix holds 1..local_max transactions writes its children as bitsets
    // of that many bits, numbered by rank within the prefix, and queues the
    // child frame's units in lq for k_local.  The rank directory sits at byte
    // dir_off of the dynamic shared memory.
    unsigned long long *lq;
    uint64_t lq_cap;
    uint32_t local_max;
    uint32_t dir_off;
    // Row-wise units (h_rows null: off; one database, projection on): the
    // rows of its frequent indices (k_rows.cuh: row t at h_rows[h_off[t]
    // .. h_off[t + 1])), the column -> frequent index map, the work of one
    // row visit against one sibling id or 16-byte word, a per-CTA scratch of
    // h_scratch_words transaction ids, and the byte offset in the dynamic
    // shared memory of the h_F-entry frequent index -> sibling table.
    const uint64_t *h_off;
    const uint16_t *h_rows;
    const uint16_t *h_fidx;
    uint32_t h_F;
    float h_cost;
    uint32_t *h_scratch;
    uint32_t h_scratch_words;
    uint32_t h_table_off;
};

// Row-wise units need at least this many siblings.
constexpr uint32_t H_MIN_SIBLINGS = 8;
// The projected writers' instructions per sibling id or 16-byte word (a rank
// lookup and a segmented OR, or a compress and atomics) over a row visit's
// per frequent index (a load and a table lookup): about four.
constexpr double H_P2_WEIGHT = 4.0;
constexpr uint16_t H_NONE = 0xffffu;

constexpr int UNIT_LOG_WORDS = 12;

// Child tidset form: a list when it takes at most 1/P.lists of the dense
// words (P.lists = 0: bitsets only).
__device__ __forceinline__ bool as_list(const DeepParams &P, uint64_t n, uint32_t stride) {
    return P.lists && list_words(n) * P.lists <= stride;
}

__device__ __forceinline__ unsigned long long ld_raw_ptr(const uint64_t *const *p) {
    return __ldcg(reinterpret_cast<const unsigned long long *>(p));
}

__device__ __forceinline__ uint32_t bit_of(const uint32_t *bm, uint32_t t) { return (bm[t >> 5] >> (t & 31)) & 1u; }

// Exclusive prefix sum over the block (every thread calls it); *total gets
// the block's sum.  s_w holds 32 partial sums.
__device__ __forceinline__ uint64_t block_excl_scan_u64(uint64_t v, uint64_t *s_w, uint64_t *total) {
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

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void deep_fail(DeepState *st, unsigned bit) { atomicOr(&st->error, bit); }

// Thread 0 claims the next unit with a ticket: one atomicAdd on the head,
// then a wait on its own queue entry until a producer fills it, or until no
// unit is queued or running (the ticket will never be filled), or an error.
// Returns 0 with *item set, or 1 to stop.
//
// *next is a ticket taken ahead of time (NO_TICKET: none).  When P.prefetch is
// set and the claimed entry was already filled (units are queued beyond it),
// the next ticket is taken right away, so that its atomic overlaps the unit
// that follows; a CTA that had to wait takes its tickets one at a time, and
// holds none that a free CTA could have used.
constexpr unsigned long long NO_TICKET = ~0ull;
__device__ int deep_claim(const DeepParams &P, unsigned long long *item, unsigned long long *next) {
    DeepState *st = P.st;
    const unsigned long long h = *next != NO_TICKET ? *next : atomicAdd(&st->q_head, 1ull);
    *next = NO_TICKET;
    unsigned backoff = 32;  // ns, doubled up to 2 us while waiting
    for (unsigned long long it = 0; it < P.spin_limit; ++it) {
        if (h < P.queue_cap) {
            const unsigned long long v = ld_acquire_u64(P.queue + h);
            if (v != QUEUE_EMPTY) {
                *item = v;
                if (P.prefetch && it == 0) *next = atomicAdd(&st->q_head, 1ull);
                return 0;
            }
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

// Work units of a sibling: 16-byte words of a bitset (n2), or ids of a list
// (its header's count; lists only when the prefix is in shared memory).
template <bool SMEM_PREFIX>
__device__ __forceinline__ uint64_t sibling_units(unsigned long long sraw, uint64_t n2) {
    return (SMEM_PREFIX && (sraw & 1ull)) ? (uint64_t)__ldcg(reinterpret_cast<const uint32_t *>(sraw & ~1ull)) : n2;
}

// A sibling's size in its own form (the bytes a full pass reads).
template <bool SMEM_PREFIX>
__device__ __forceinline__ uint64_t sibling_bytes(unsigned long long sraw, uint64_t units) {
    return (SMEM_PREFIX && (sraw & 1ull)) ? 8ull * list_words(units) : 16ull * units;
}

// This lane's share of |prefix & sibling| over work units [lo, hi) of the
// sibling (dense words or list ids).  Eight 16-byte loads (or sixteen ids) in
// flight per lane.
template <bool SMEM_PREFIX>
__device__ __forceinline__ uint32_t sibling_count_range(unsigned long long sraw, uint64_t lo, uint64_t hi,
                                                        const ulonglong2 *s_prefix, const uint32_t *s_p32,
                                                        const ulonglong2 *pb, const ulonglong2 *mk, unsigned lane) {
    uint32_t s = 0;
    if (SMEM_PREFIX && (sraw & 1ull)) {
        // List sibling: test its ids against the prefix bitmap.  Lanes take
        // consecutive ids (32 per warp load), so the bit tests of one
        // instruction fall in nearby, mostly distinct shared-memory banks.
        const uint32_t *I = reinterpret_cast<const uint32_t *>(sraw & ~1ull) + 4;
        uint64_t w = lo + lane;
        for (; w + 480 < hi; w += 512) {
            uint32_t t[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) t[u] = __ldcg(I + w + 32 * u);
#pragma unroll
            for (int u = 0; u < 16; ++u) s += bit_of(s_p32, t[u]);
        }
        for (; w < hi; w += 32) s += bit_of(s_p32, __ldcg(I + w));
        return s;
    }
    const ulonglong2 *sb = reinterpret_cast<const ulonglong2 *>(sraw);
    uint64_t v = lo + lane;
    for (; v + 224 < hi; v += 256) {
        ulonglong2 x[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) x[u] = ld_cg(sb + v + 32 * u);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (SMEM_PREFIX) {
                x[u] = and2(x[u], s_prefix[v + 32 * u]);
            } else {
                x[u] = and2(x[u], ld_cg(pb + v + 32 * u));
                if (mk) x[u] = and2(x[u], ld_cg(mk + v + 32 * u));
            }
            s += popc2(x[u]);
        }
    }
    for (; v < hi; v += 32) {
        ulonglong2 x = ld_cg(sb + v);
        if (SMEM_PREFIX) {
            x = and2(x, s_prefix[v]);
        } else {
            x = and2(x, ld_cg(pb + v));
            if (mk) x = and2(x, ld_cg(mk + v));
        }
        s += popc2(x);
    }
    return s;
}

// This lane's share of |prefix & sibling| over part `part` of `parts` equal
// slices of the sibling; *bytes gets the sibling's size in its own form.
template <bool SMEM_PREFIX>
__device__ __forceinline__ uint32_t sibling_count(unsigned long long sraw, uint32_t part, uint32_t parts, uint64_t n2,
                                                  const ulonglong2 *s_prefix, const uint32_t *s_p32,
                                                  const ulonglong2 *pb, const ulonglong2 *mk, unsigned lane,
                                                  uint64_t *bytes) {
    const uint64_t units = sibling_units<SMEM_PREFIX>(sraw, n2);
    *bytes = sibling_bytes<SMEM_PREFIX>(sraw, units);
    return sibling_count_range<SMEM_PREFIX>(sraw, units * part / parts, units * (part + 1) / parts, s_prefix, s_p32,
                                            pb, mk, lane);
}

// Staging of a dense prefix by the copy engine: thread 0 makes the generic
// stores it acquired visible to the async proxy, arms the CTA's mbarrier with
// the byte count and issues cp.async.bulk copies of at most 32 KB from global
// to shared memory (no multicast: the source is this GPU's own arena).
__device__ __forceinline__ void bulk_stage(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("fence.proxy.async.global;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    for (uint32_t off = 0; off < bytes; off += 32768u) {
        const uint32_t n = min(32768u, bytes - off);
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(d + off), "l"(reinterpret_cast<const char *>(src) + off), "r"(n), "r"(b)
                     : "memory");
    }
}

// Bounded wait for the mbarrier phase `parity` to complete; false if it ran out.
__device__ __forceinline__ bool bulk_wait(uint64_t *bar, uint32_t parity, unsigned long long limit) {
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    for (unsigned long long i = 0; i < limit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(b), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Child list piece: the ids of the sibling's transactions that the prefix
// bitmap holds, over work units [lo, hi) of the sibling (list ids or bitset
// words), written in ascending order to o32[4 + at ...] (never past sc ids).
// Returns the position after the last id.  Loads run eight id chunks (or
// four word chunks) ahead of the ballot compaction.
__device__ __forceinline__ uint32_t write_list_piece(unsigned long long sraw, uint64_t lo, uint64_t hi,
                                                     const ulonglong2 *s_prefix, const uint32_t *s_p32,
                                                     uint32_t *o32, uint32_t at, uint32_t sc, unsigned lane) {
    const unsigned below = (1u << lane) - 1u;
    if (sraw & 1ull) {
        const uint32_t *I = reinterpret_cast<const uint32_t *>(sraw & ~1ull) + 4;
        for (uint64_t w0 = lo; w0 < hi; w0 += 256) {
            uint32_t t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const uint64_t j = w0 + 32 * u + lane;
                t[u] = j < hi ? __ldcg(I + j) : 0u;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const bool keep = w0 + 32 * u + lane < hi && bit_of(s_p32, t[u]);
                const unsigned bal = __ballot_sync(CPM_FULL, keep);
                const uint32_t pos = at + __popc(bal & below);
                if (keep && pos < sc) o32[4 + pos] = t[u];
                at += __popc(bal);
            }
        }
        return at;
    }
    const ulonglong2 *sb = reinterpret_cast<const ulonglong2 *>(sraw);
    for (uint64_t v0 = lo; v0 < hi; v0 += 128) {
        ulonglong2 x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t v = v0 + 32 * u + lane;
            x[u] = v < hi ? and2(ld_cg(sb + v), s_prefix[v]) : make_ulonglong2(0ull, 0ull);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t v = v0 + 32 * u + lane;
            const uint32_t c = popc2(x[u]);
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(CPM_FULL, incl, o);
                if (lane >= (unsigned)o) incl += y;
            }
            uint32_t pos = at + incl - c;
            for (unsigned long long b = x[u].x; b; b &= b - 1, ++pos)
                if (pos < sc) o32[4 + pos] = (uint32_t)(v * 128 + __ffsll((long long)b) - 1);
            for (unsigned long long b = x[u].y; b; b &= b - 1, ++pos)
                if (pos < sc) o32[4 + pos] = (uint32_t)(v * 128 + 64 + __ffsll((long long)b) - 1);
            at += __shfl_sync(CPM_FULL, incl, 31);
        }
    }
    return at;
}

// Child bitset piece: words [lo, hi) of prefix & sibling (a bitset), four
// 16-byte loads in flight per lane.
template <bool SMEM_PREFIX>
__device__ __forceinline__ void write_dense_piece(unsigned long long sraw, uint64_t lo, uint64_t hi,
                                                  const ulonglong2 *s_prefix, const ulonglong2 *pb,
                                                  const ulonglong2 *mk, ulonglong2 *dst, unsigned lane) {
    const ulonglong2 *sb = reinterpret_cast<const ulonglong2 *>(sraw);
    auto with_prefix = [&](ulonglong2 x, uint64_t v) {
        if (SMEM_PREFIX) return and2(x, s_prefix[v]);
        x = and2(x, ld_cg(pb + v));
        return mk ? and2(x, ld_cg(mk + v)) : x;
    };
    uint64_t v = lo + lane;
    for (; v + 96 < hi; v += 128) {
        ulonglong2 x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = ld_cg(sb + v + 32 * u);
#pragma unroll
        for (int u = 0; u < 4; ++u) dst[v + 32 * u] = with_prefix(x[u], v + 32 * u);
    }
    for (; v < hi; v += 32) dst[v] = with_prefix(ld_cg(sb + v), v);
}

// ---- Projection: children numbered by rank within the prefix ----
// A child of unit (F, p) is t(prefix) & t(sibling), a subset of the prefix's
// n_p transactions.  Numbering them by their rank in the prefix (the j-th
// transaction of the prefix becomes j) turns every descendant tidset into a
// bitset of n_p bits: for a prefix of a few thousand transactions among a
// million that is a few hundred bytes, instead of a list of 4-byte ids, and
// its units need no million-bit bitmap.

// dir[v] = set bits of the staged prefix before its 16-byte word v (below
// 2^16: projection needs n_p <= local_max <= 65535).  Every thread calls it.
__device__ __forceinline__ void build_rank_dir(const ulonglong2 *s_prefix, uint64_t n2, uint16_t *dir,
                                               uint64_t *s_w64) {
    const uint64_t per = (n2 + blockDim.x - 1) / blockDim.x;
    const uint64_t a = min(n2, (uint64_t)threadIdx.x * per), b = min(n2, a + per);
    uint64_t c = 0;
    for (uint64_t v = a; v < b; ++v) c += popc2(s_prefix[v]);
    uint64_t tot = 0;
    uint64_t run = block_excl_scan_u64(c, s_w64, &tot);
    for (uint64_t v = a; v < b; ++v) {
        dir[v] = (uint16_t)run;
        run += popc2(s_prefix[v]);
    }
}

// The bits of x at the set positions of m, packed to the low end in order
// (the "compress" or generalized extract of H. S. Warren, Hacker's Delight,
// 2nd ed., section 7-4, parallel-suffix method, here for 64 bits): at round
// i every bit still to move by an odd multiple of 2^i moves right by 2^i.
__device__ __forceinline__ unsigned long long compress64(unsigned long long x, unsigned long long m) {
    x &= m;
    unsigned long long mk = ~m << 1;  // zeros of m to the right of each bit, counted below
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        unsigned long long mp = mk ^ (mk << 1);  // parallel suffix (XOR) of mk
        mp ^= mp << 2;
        mp ^= mp << 4;
        mp ^= mp << 8;
        mp ^= mp << 16;
        mp ^= mp << 32;
        const unsigned long long mv = mp & m;  // bits of m that move this round
        m = (m ^ mv) | (mv >> (1 << i));
        const unsigned long long t = x & mv;
        x = (x ^ t) | (t >> (1 << i));
        mk &= ~mp;
    }
    return x;
}

// Transactions of the prefix below transaction t.
__device__ __forceinline__ uint32_t rank_of(const ulonglong2 *s_prefix, const uint16_t *dir, uint32_t t) {
    const ulonglong2 w = s_prefix[t >> 7];
    const uint32_t b = t & 127u;
    uint32_t r = dir[t >> 7];
    if (b < 64) r += __popcll(w.x & ((1ull << b) - 1ull));
    else r += __popcll(w.x) + __popcll(w.y & ((1ull << (b - 64)) - 1ull));
    return r;
}

// Sets bit r of out32 for the lanes that keep theirs, one atomicOr per
// 32-bit word touched: r must not decrease from lane to lane (lanes that
// keep nothing carry the rank they would have), so lanes with the same word
// are neighbours and a segmented OR gathers their bits in the word's first lane.
__device__ __forceinline__ void or_ranks(uint32_t *out32, uint32_t nw32, uint32_t r, bool keep, unsigned lane) {
    const uint32_t w = r >> 5;
    uint32_t v = keep ? 1u << (r & 31u) : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t vo = __shfl_down_sync(CPM_FULL, v, o);
        const uint32_t wo = __shfl_down_sync(CPM_FULL, w, o);
        if (lane + o < 32 && wo == w) v |= vo;
    }
    const uint32_t wp = __shfl_up_sync(CPM_FULL, w, 1);
    if ((lane == 0 || wp != w) && v && w < nw32) atomicOr(out32 + w, v);
}

// Projected child piece: over work units [lo, hi) of the sibling (list ids
// or bitset words), every transaction t the prefix holds sets bit rank(t)
// of the child bitset out32 (nw32 words), which is zeroed before the pass.
// Ranks stay below the prefix's count, which the caller checks against the
// bitset's size; the writes are bounded by nw32 all the same.
__device__ __forceinline__ void write_proj_piece(unsigned long long sraw, uint64_t lo, uint64_t hi,
                                                 const ulonglong2 *s_prefix, const uint32_t *s_p32,
                                                 const uint16_t *dir, uint32_t *out32, uint32_t nw32, unsigned lane) {
    if (sraw & 1ull) {
        const uint32_t *I = reinterpret_cast<const uint32_t *>(sraw & ~1ull) + 4;
        for (uint64_t w0 = lo; w0 < hi; w0 += 256) {
            uint32_t t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const uint64_t j = w0 + 32 * u + lane;
                t[u] = j < hi ? __ldcg(I + j) : 0u;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const bool in = w0 + 32 * u + lane < hi;
                // Ids ascend from lane to lane and past the end come last: ranks never fall.
                const uint32_t r = in ? rank_of(s_prefix, dir, t[u]) : 0xffffffffu;
                or_ranks(out32, nw32, r, in && bit_of(s_p32, t[u]), lane);
            }
        }
        return;
    }
    // Bitset sibling: the kept bits of a 64-bit half-word x under prefix
    // half-word m land on ranks r .. r + popc(m) - 1 in order, i.e. they are
    // compress(x, m) shifted to bit r.  A half-word of a few prefix bits is
    // walked bit by bit (gathered per 32-bit output word in a register);
    // a fuller one is compressed and OR-ed in with one or two 64-bit atomics.
    const ulonglong2 *sb = reinterpret_cast<const ulonglong2 *>(sraw);
    unsigned long long *out64 = reinterpret_cast<unsigned long long *>(out32);
    const uint32_t nw64 = nw32 / 2;
    uint32_t cw = 0xffffffffu, cv = 0;
    for (uint64_t v = lo + lane; v < hi; v += 32) {
        const ulonglong2 pw = s_prefix[v];
        if (!(pw.x | pw.y)) continue;  // no transaction of the prefix here: nothing to read
        const ulonglong2 x = and2(ld_cg(sb + v), pw);
        uint32_t r0 = dir[v];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const unsigned long long m = h ? pw.y : pw.x;
            const unsigned long long xh = h ? x.y : x.x;
            const uint32_t pm = __popcll(m);
            if (xh && pm > 4) {
                const unsigned long long c = compress64(xh, m);
                const uint32_t w = r0 >> 6, sh = r0 & 63u;
                if (w < nw64) atomicOr(out64 + w, c << sh);
                if (sh && (c >> (64 - sh)) && w + 1 < nw64) atomicOr(out64 + w + 1, c >> (64 - sh));
            } else {
                for (unsigned long long b = xh; b; b &= b - 1) {
                    const int bit = __ffsll((long long)b) - 1;
                    const uint32_t r = r0 + __popcll(m & ((1ull << bit) - 1ull));
                    if ((r >> 5) != cw) {
                        if (cv && cw < nw32) atomicOr(out32 + cw, cv);
                        cw = r >> 5;
                        cv = 0;
                    }
                    cv |= 1u << (r & 31u);
                }
            }
            r0 += pm;
        }
    }
    if (cv && cw < nw32) atomicOr(out32 + cw, cv);
}

template <bool SMEM_PREFIX>
__global__ void __launch_bounds__(1024) k_deep(DeepParams P) {
    extern __shared__ ulonglong2 s_prefix[];
    __shared__ unsigned long long s_item;
    __shared__ int s_stop, s_ok, s_grant, s_skip;
    __shared__ uint32_t s_surv;
    __shared__ unsigned long long s_mem_base, s_arena_base, s_fid, s_qbase;
    __shared__ uint32_t s_wtot[32];
    __shared__ uint64_t s_w64[32];
    __shared__ uint64_t s_off[1025];     // child offsets of one chunk of survivors; pass-1 work offsets
    __shared__ unsigned long long s_raw[1024];  // pass 1 (balanced): sibling pointers of one chunk
    __shared__ uint32_t s_cnt[1024];             // pass 1 (balanced): their supports; pass 2: child supports
    __shared__ uint32_t s_coff[1024];            // pass 2: arena offsets (words) of one chunk's children
    __shared__ uint32_t s_pid[1024];             // units of at most blockDim siblings: pattern id of each
    __shared__ uint16_t s_map[1024];             // ... and, after compaction, each survivor's sibling index
    __shared__ uint32_t s_clast[32];             // pass 2: ids in each warp's last piece of a split child
    __shared__ const uint32_t *s_hids;           // row-wise pass 2: the prefix's transaction ids, and their count
    __shared__ uint32_t s_hn;
    __shared__ unsigned long long s_bytes;
    __shared__ uint32_t s_nsurv;         // survivors counted in pass 1
    __shared__ uint32_t s_part[32];      // per-sibling sums when siblings are split over warps
    __shared__ unsigned long long s_maxb;  // largest sibling's bytes (diagnostics only)
    uint32_t *const s_p32 = reinterpret_cast<uint32_t *>(s_prefix);
    __shared__ __align__(8) uint64_t s_bulk_bar;  // completes when a bulk-staged prefix has landed
    __shared__ unsigned long long lg[7];   // claim, staged, pass 1 done, prefix word, compacted, granted,
                                           // children written (diagnostics only)

    const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    DeepState *st = P.st;
    if (!SMEM_PREFIX && P.lists) {
        // List tidsets are tested against a prefix bitmap in shared memory:
        // without one the host must not ask for them.
        if (threadIdx.x == 0 && blockIdx.x == 0) deep_fail(st, DEEP_ERR_INTERNAL);
        return;
    }
    __shared__ uint32_t s_bulk_phase;  // parity of s_bulk_bar's next phase
    if (SMEM_PREFIX && threadIdx.x == 0) {
        s_bulk_phase = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_bulk_bar))
                     : "memory");
    }
    // Per-CTA statistics (thread 0), added to the global counters at exit.
    // Kept in shared memory, not registers: only thread 0 touches them.
    __shared__ unsigned long long c_inter, c_bytes, c_units, c_surv, c_busy, t_unit;
    if (threadIdx.x == 0) c_inter = c_bytes = c_units = c_surv = c_busy = t_unit = 0;

    // Row-wise units' frequent index -> sibling table: empty between units.
    uint16_t *const s_tab = reinterpret_cast<uint16_t *>(reinterpret_cast<char *>(s_prefix) + P.h_table_off);
    if (SMEM_PREFIX && P.h_rows)
        for (uint32_t i = threadIdx.x; i < P.h_F; i += blockDim.x) s_tab[i] = H_NONE;

    unsigned long long next_ticket = NO_TICKET;  // thread 0's ticket taken ahead
    for (;;) {
        if (threadIdx.x == 0) {
            s_stop = deep_claim(P, &s_item, &next_ticket);
            s_skip = 0;
            bool hand_back = false;
            if (!s_stop && P.defer_words && (uint32_t)(s_item >> 32) < P.root_frames) {
                hand_back = ld_acquire_u64(&st->arena_next) >= P.defer_words ||
                            ld_acquire_u64(&st->n_members) >= P.defer_members ||
                            ld_acquire_u64(&st->n_frames) >= P.defer_frames ||
                            ld_acquire_u64(&st->q_tail) >= P.defer_queue;
                const uint32_t fid = (uint32_t)(s_item >> 32);
                if (!hand_back && P.root_key && fid < P.top_frames) {
                    const DFrame *f = P.frames + fid;
                    const uint32_t unit = __ldcg(&f->root) + (uint32_t)s_item;
                    const double k = (double)__ldg(P.root_key + unit);
                    const unsigned long long w =
                        1ull + (unsigned long long)(P.keys_in_words ? k : k * (double)__ldcg(&f->stride));
                    const unsigned long long before = atomicAdd(&st->admitted, w);
                    if (P.admit_words && before > 0 && before + w > P.admit_words) {
                        atomicAdd(&st->admitted, 0ull - w);
                        hand_back = true;
                    }
                }
            }
            if (hand_back) {
                // The round's arena is filling up: leave this root unit to the next round.
                const unsigned long long di = atomicAdd(&st->n_deferred, 1ull);
                if (di < P.deferred_cap) P.deferred[di] = s_item;
                else deep_fail(st, DEEP_ERR_QUEUE);
                atomicAdd(&st->pending, ~0ull);  // pending -= 1 (deferred[] is read after the kernel)
                s_skip = 1;
            }
        }
        __syncthreads();
        if (s_stop) break;
        if (s_skip) {
            __syncthreads();  // every thread has read s_skip before thread 0 claims again
            continue;
        }
        if (threadIdx.x == 0 && P.cta_time) t_unit = global_ns();
        // The error word, read now and looked at after the staging, so that
        // its latency overlaps the staging (thread 0 only; a hint that lets a
        // failed launch stop early, nothing is ordered by it).
        const unsigned err_seen = threadIdx.x == 0 ? ld_relaxed_u32(&st->error) : 0u;
        if (threadIdx.x == 0 && P.unit_log) {
            lg[0] = global_ns();
            s_maxb = 0;
        }
        const uint32_t fid = (uint32_t)(s_item >> 32), p = (uint32_t)s_item;
        const DFrame *fp = P.frames + fid;
        const ulonglong2 *mk = reinterpret_cast<const ulonglong2 *>(
            __ldcg(reinterpret_cast<const unsigned long long *>(&fp->mask)));
        const uint64_t mem_off = __ldcg(reinterpret_cast<const unsigned long long *>(&fp->mem_off));
        const uint32_t m = __ldcg(&fp->m), stride = __ldcg(&fp->stride);
        // Root unit of this work: top-level frames (the ones with a mask) are
        // split into one root unit per position.
        const uint32_t root = __ldcg(&fp->root) + (mk ? p : 0u);
        const uint32_t db = __ldcg(&fp->db);
        const long long minsup = __ldcg(&fp->minsup);
        const uint64_t n2 = stride / 2;
        const uint32_t cnt = m - p - 1;
        // Units of at most blockDim siblings keep every sibling's pointer,
        // support and pattern id in shared memory (s_raw, s_cnt, s_pid) and
        // reserve and write member entries for their survivors only, once
        // compacted; larger units reserve and write an entry per sibling.
        const bool fast = cnt <= blockDim.x;
        // Fewer siblings than warps: split every sibling into equal slices
        // (at least 4 KB of bitset each) so that every warp has work.
        const uint32_t parts = (cnt && cnt < nw) ? max(1u, min(nw / cnt, (uint32_t)(n2 >> 8))) : 1u;
        // Each warp's first sibling pointer is loaded now and its list
        // header after the staging, so that their latency overlaps it.
        const uint32_t first_q = parts == 1 ? wid : wid / parts;
        unsigned long long first_raw = 0;
        uint64_t first_units = 0;
        if (!P.balance && first_q < cnt) first_raw = ld_raw_ptr(P.mem_bits + mem_off + p + 1 + first_q);
        const unsigned long long praw = ld_raw_ptr(P.mem_bits + mem_off + p);
        const ulonglong2 *pb = reinterpret_cast<const ulonglong2 *>(praw);
        uint64_t prefix_bytes = 8ull * stride;
        // Row-wise unit: a list prefix of at most local_max transactions whose
        // rows (each ~h_cost work) take less work than the siblings' ids and
        // words.  Every input is the same on every thread, so is the choice.
        bool hmode = false;
        uint32_t h_np = 0;
        if (SMEM_PREFIX && P.h_rows && fast && cnt >= H_MIN_SIBLINGS && (praw & 1ull) && !P.shallow) {
            h_np = __ldcg(P.pat_sup + __ldcg(P.mem_pat + mem_off + p));
            if (h_np >= 1 && h_np <= P.local_max) {
                uint64_t work = 0;
                if (threadIdx.x < cnt) {
                    const unsigned long long raw = ld_raw_ptr(P.mem_bits + mem_off + p + 1 + threadIdx.x);
                    s_raw[threadIdx.x] = raw;
                    work = sibling_units<SMEM_PREFIX>(raw, n2);
                }
                uint64_t tot = 0;
                block_excl_scan_u64(work, s_w64, &tot);
                hmode = (double)h_np * (double)P.h_cost < (double)tot;
            }
        }
        if (SMEM_PREFIX && hmode) {
            // No bitmap: the prefix is read as its list of transactions.
            prefix_bytes = 8ull * list_words(h_np);
        } else if (SMEM_PREFIX && (praw & 1ull)) {
            // List prefix: clear the bitmap, set its transactions, then apply the mask.
            const uint32_t *L = reinterpret_cast<const uint32_t *>(praw & ~1ull);
            const uint32_t n = __ldcg(L);
            prefix_bytes = 8ull * list_words(n);
            for (uint64_t v = threadIdx.x; v < n2; v += blockDim.x) s_prefix[v] = make_ulonglong2(0ull, 0ull);
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                const uint32_t t = __ldcg(L + 4 + i);
                atomicOr(s_p32 + (t >> 5), 1u << (t & 31));
            }
            __syncthreads();
            if (mk)
                for (uint64_t v = threadIdx.x; v < n2; v += blockDim.x) s_prefix[v] = and2(s_prefix[v], ld_cg(mk + v));
        } else if (SMEM_PREFIX && !mk && n2 >= BULK_MIN_WORDS2) {
            // Long dense prefix of a deeper frame: one contiguous arena block,
            // staged by the copy engine while the threads wait.
            // (thread 0 flips s_bulk_phase after the barrier below, once every
            // thread has read it)
            const uint32_t ph = s_bulk_phase;
            if (threadIdx.x == 0) bulk_stage(s_prefix, pb, (uint32_t)(16 * n2), &s_bulk_bar);
            if (!bulk_wait(&s_bulk_bar, ph, BULK_WAIT_LIMIT)) {
                // Never leave with the copy in flight: record the error, then
                // wait (bounded again) for it to land.
                if (threadIdx.x == 0) deep_fail(st, DEEP_ERR_SPIN);
                bulk_wait(&s_bulk_bar, ph, BULK_WAIT_LIMIT);
            }
        } else if (SMEM_PREFIX) {
            for (uint64_t v = threadIdx.x; v < n2; v += blockDim.x)
                s_prefix[v] = mk ? and2(ld_cg(pb + v), ld_cg(mk + v)) : ld_cg(pb + v);
        }
        if (!P.balance && first_q < cnt) first_units = sibling_units<SMEM_PREFIX>(first_raw, n2);
        if (threadIdx.x == 0) {
            s_bytes = prefix_bytes;
            s_surv = 0;
            s_nsurv = 0;
            s_grant = 0;
            s_mem_base = 0;
            if (!fast) {
                const unsigned long long mb = atomicAdd(&st->n_members, (unsigned long long)cnt);
                if (mb + cnt > P.members_cap) deep_fail(st, DEEP_ERR_MEMBERS);
                s_mem_base = mb;
            }
            s_ok = err_seen == 0;
        }
        __syncthreads();
        if (SMEM_PREFIX && threadIdx.x == 0 && !hmode && !mk && !(praw & 1ull) && n2 >= BULK_MIN_WORDS2) s_bulk_phase ^= 1u;
        if (threadIdx.x == 0 && P.unit_log) {
            lg[1] = global_ns();
            lg[3] = prefix_bytes | (SMEM_PREFIX && (praw & 1ull) ? 1ull << 63 : 0ull) | (mk ? 1ull << 62 : 0ull) |
                    (hmode ? 1ull << 61 : 0ull);
        }
        const bool ok = s_ok != 0;
        const uint32_t parent_pat = __ldcg(P.mem_pat + mem_off + p);
        // ---- pass 1: supports of every later member ----
        // Entry q of the unit's member block: the survivor (pattern, item,
        // sibling tidset until pass 2) or a hole.
        auto emit = [&](uint32_t q, uint32_t s, uint32_t sib_item, unsigned long long sraw) {
            const uint64_t m_out = s_mem_base + q;
            uint32_t pid32 = NO_PATTERN;
            if ((long long)s >= minsup) {
                const unsigned long long pid = atomicAdd(&st->n_patterns, 1ull);
                if (pid >= P.pat_cap) {
                    deep_fail(st, DEEP_ERR_PATTERNS);
                } else {
                    P.pat_parent[pid] = parent_pat;
                    P.pat_item[pid] = sib_item;
                    P.pat_sup[pid] = s;
                    if (P.pat_db) P.pat_db[pid] = db;
                    pid32 = (uint32_t)pid;
                }
            }
            if (fast) {
                s_raw[q] = sraw;
                s_cnt[q] = s;
                s_pid[q] = pid32;
            } else if (m_out < P.members_cap) {
                P.mem_pat[m_out] = pid32;
                P.mem_item[m_out] = sib_item;
                P.mem_bits[m_out] = reinterpret_cast<const uint64_t *>(sraw);
            }
            if (pid32 != NO_PATTERN) atomicAdd(&s_nsurv, 1u);
        };
        // Row-wise units: the prefix's transactions, as ids (kept for pass 2).
        const uint32_t *h_ids = nullptr;
        uint32_t h_n = 0;
        if (SMEM_PREFIX && hmode) {
            // The member's list, or for a top-level class the ids of it that
            // the class item's tidset holds, compacted in order into this
            // CTA's scratch.
            const uint32_t *L = reinterpret_cast<const uint32_t *>(praw & ~1ull);
            const uint32_t n_m = __ldcg(L);
            if (!mk) {
                h_ids = L + 4;
                h_n = n_m;
            } else {
                uint32_t *scr = P.h_scratch + (uint64_t)blockIdx.x * P.h_scratch_words;
                const unsigned long long *m64 = reinterpret_cast<const unsigned long long *>(mk);
                const uint32_t per = (n_m + blockDim.x - 1) / blockDim.x;
                const uint32_t a = min(n_m, threadIdx.x * per), b = min(n_m, a + per);
                uint32_t c = 0;
                // Eight ids, then their eight mask words, in flight at a time.
                for (uint32_t j0 = a; j0 < b; j0 += 8) {
                    uint32_t t[8];
                    unsigned long long mw[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) t[u] = j0 + u < b ? __ldcg(L + 4 + j0 + u) : 0u;
#pragma unroll
                    for (int u = 0; u < 8; ++u) mw[u] = j0 + u < b ? __ldcg(m64 + (t[u] >> 6)) : 0ull;
#pragma unroll
                    for (int u = 0; u < 8; ++u) c += (uint32_t)(mw[u] >> (t[u] & 63)) & 1u;
                }
                uint64_t tot = 0;
                uint64_t at = block_excl_scan_u64(c, s_w64, &tot);
                for (uint32_t j0 = a; j0 < b; j0 += 8) {
                    uint32_t t[8];
                    unsigned long long mw[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) t[u] = j0 + u < b ? __ldcg(L + 4 + j0 + u) : 0u;
#pragma unroll
                    for (int u = 0; u < 8; ++u) mw[u] = j0 + u < b ? __ldcg(m64 + (t[u] >> 6)) : 0ull;
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if ((mw[u] >> (t[u] & 63)) & 1ull) {
                            if (at < P.h_scratch_words) scr[at] = t[u];
                            ++at;
                        }
                }
                h_ids = scr;
                h_n = (uint32_t)(tot < P.h_scratch_words ? tot : (uint64_t)P.h_scratch_words);
            }
            // The prefix's count sized the projection: anything else is an error,
            // and no more than that many transactions are read.
            if (h_n != h_np && threadIdx.x == 0) deep_fail(st, DEEP_ERR_INTERNAL);
            h_n = min(h_n, h_np);
            if (threadIdx.x == 0) {
                s_hids = h_ids;
                s_hn = h_n;
                atomicAdd(&st->h_units, 1ull);
            }
            uint32_t my_f = H_NONE;
            if (threadIdx.x < cnt) {
                my_f = __ldg(P.h_fidx + __ldcg(P.mem_item + mem_off + p + 1 + threadIdx.x));
                s_cnt[threadIdx.x] = 0;
                if (my_f < P.h_F) s_tab[my_f] = (uint16_t)threadIdx.x;
                else deep_fail(st, DEEP_ERR_INTERNAL);
            }
            // Counters: copies in the (unused) prefix-bitmap region, one per
            // group of warps, so that the many rows holding a popular item do
            // not all add to one shared word; else s_cnt alone.
            uint32_t copies = 1;
            {
                const uint64_t fit = (P.max_stride * 8) / (4ull * cnt);
                while (copies * 2 <= nw && copies * 2 <= fit) copies *= 2;
            }
            uint32_t *const s_wc = copies > 1 ? reinterpret_cast<uint32_t *>(s_prefix) : s_cnt;
            if (copies > 1)
                for (uint32_t i = threadIdx.x; i < copies * cnt; i += blockDim.x) s_wc[i] = 0u;
            uint32_t *const my_wc = s_wc + (wid & (copies - 1)) * cnt;
            __syncthreads();  // the table, the counters and the scratch ids are in place
            // Every row of the prefix: each frequent index that is a later
            // member adds one to that member's support.
            unsigned long long visited = 0, nrows = 0;
            for (uint32_t j = threadIdx.x; j < h_n; j += blockDim.x) {
                const uint32_t t = __ldcg(h_ids + j);
                const uint32_t ra = __ldg(P.h_off + t), rb = __ldg(P.h_off + t + 1);
                visited += rb - ra;
                ++nrows;
                // Eight frequent indices of the row in flight at a time.
                for (uint32_t k0 = ra; k0 < rb; k0 += 8) {
                    uint32_t f[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) f[u] = k0 + u < rb ? (uint32_t)__ldg(P.h_rows + k0 + u) : H_NONE;
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (f[u] != H_NONE) {
                            const uint32_t sib = s_tab[f[u]];
                            if (sib != H_NONE) atomicAdd(my_wc + sib, 1u);
                        }
                }
            }
            // Bytes read: an id and two offsets per row, two per frequent index.
            if (nrows) atomicAdd(&s_bytes, 2ull * visited + 12ull * nrows);
            __syncthreads();  // every count is in
            if (ok && threadIdx.x < cnt) {
                const uint32_t q = threadIdx.x;
                uint32_t sup = 0;
                for (uint32_t c = 0; c < copies; ++c) sup += s_wc[c * cnt + q];
                emit(q, sup, __ldcg(P.mem_item + mem_off + p + 1 + q), s_raw[q]);
            }
            if (threadIdx.x < cnt && my_f < P.h_F) s_tab[my_f] = H_NONE;  // nobody reads it before the next barrier
        } else if (P.balance) {
            // Siblings split over warps by size.  Per chunk of up to blockDim
            // siblings: every sibling's work (bitset words or list ids) is
            // laid end to end, each warp takes an equal slice of the total
            // (crossing sibling boundaries) and adds its partial counts into
            // s_cnt; then each sibling is emitted.  A unit takes as long as
            // its bytes, not as long as its largest sibling.
            for (uint32_t c0 = 0; ok && c0 < cnt; c0 += blockDim.x) {
                const uint32_t cn = min((uint32_t)blockDim.x, cnt - c0);
                uint64_t wk = 0;
                unsigned long long raw = 0;
                if (threadIdx.x < cn) {
                    raw = ld_raw_ptr(P.mem_bits + mem_off + p + 1 + c0 + threadIdx.x);
                    wk = sibling_units<SMEM_PREFIX>(raw, n2);
                    s_raw[threadIdx.x] = raw;
                    s_cnt[threadIdx.x] = 0;
                }
                uint64_t tot = 0;
                const uint64_t ex = block_excl_scan_u64(wk, s_w64, &tot);
                if (threadIdx.x < cn) s_off[threadIdx.x] = ex;
                if (threadIdx.x == 0) s_off[cn] = tot;
                __syncthreads();
                const uint64_t lo = tot * wid / nw, hi = tot * (wid + 1) / nw;
                if (lo < hi) {
                    uint32_t a = 0, b = cn;  // first sibling whose work ends past lo
                    while (a < b) {
                        const uint32_t mid = (a + b) >> 1;
                        if (s_off[mid + 1] <= lo) a = mid + 1; else b = mid;
                    }
                    for (uint32_t i = a; i < cn && s_off[i] < hi; ++i) {
                        const uint64_t u0 = max(lo, s_off[i]) - s_off[i], u1 = min(hi, s_off[i + 1]) - s_off[i];
                        if (u0 >= u1) continue;
                        uint32_t c = sibling_count_range<SMEM_PREFIX>(s_raw[i], u0, u1, s_prefix, s_p32, pb, mk, lane);
                        c = warp_sum_u32(c);
                        if (lane == 0 && c) atomicAdd(&s_cnt[i], c);
                    }
                }
                __syncthreads();
                if (threadIdx.x < cn) {
                    const uint64_t b = sibling_bytes<SMEM_PREFIX>(raw, wk);
                    atomicAdd(&s_bytes, (unsigned long long)b);
                    if (P.unit_log) atomicMax(&s_maxb, (unsigned long long)b);
                    emit(c0 + threadIdx.x, s_cnt[threadIdx.x], __ldcg(P.mem_item + mem_off + p + 1 + c0 + threadIdx.x),
                         raw);
                }
                __syncthreads();
            }
        } else if (parts == 1) {
            for (uint32_t q = wid; ok && q < cnt; q += nw) {
                const uint64_t mi = mem_off + p + 1 + q;
                const bool first = q == wid;
                const unsigned long long sraw = first ? first_raw : ld_raw_ptr(P.mem_bits + mi);
                const uint32_t sib_item = __ldcg(P.mem_item + mi);
                const uint64_t units = first ? first_units : sibling_units<SMEM_PREFIX>(sraw, n2);
                const uint64_t b = sibling_bytes<SMEM_PREFIX>(sraw, units);
                uint32_t s = sibling_count_range<SMEM_PREFIX>(sraw, 0, units, s_prefix, s_p32, pb, mk, lane);
                s = warp_sum_u32(s);
                if (lane == 0) {
                    atomicAdd(&s_bytes, (unsigned long long)b);
                    if (P.unit_log) atomicMax(&s_maxb, (unsigned long long)b);
                    emit(q, s, sib_item, sraw);
                }
            }
        } else {
            if (threadIdx.x < 32) s_part[threadIdx.x] = 0;
            __syncthreads();
            for (uint32_t it = wid; ok && it < cnt * parts; it += nw) {
                const uint32_t q = it / parts, j = it - q * parts;  // q == first_q: one part per warp
                const unsigned long long sraw = first_raw;
                const uint64_t units = first_units;
                const uint64_t b = sibling_bytes<SMEM_PREFIX>(sraw, units);
                uint32_t s = sibling_count_range<SMEM_PREFIX>(sraw, units * j / parts, units * (j + 1) / parts,
                                                              s_prefix, s_p32, pb, mk, lane);
                s = warp_sum_u32(s);
                if (lane == 0) {
                    atomicAdd(&s_part[q], s);
                    if (j == 0) atomicAdd(&s_bytes, (unsigned long long)b);
                    if (j == 0 && P.unit_log) atomicMax(&s_maxb, (unsigned long long)b);
                }
            }
            __syncthreads();
            if (ok && threadIdx.x < cnt) {
                const uint64_t mi = mem_off + p + 1 + threadIdx.x;
                emit(threadIdx.x, s_part[threadIdx.x], __ldcg(P.mem_item + mi), ld_raw_ptr(P.mem_bits + mi));
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && P.unit_log) {
            lg[2] = global_ns();
            lg[4] = lg[5] = lg[6] = 0;
        }
        // Diagnostics record of this unit (thread 0, at its end).
        auto log_unit = [&](uint32_t nsurv) {
            const unsigned long long k = atomicAdd(P.unit_log, 1ull);
            if (k >= P.unit_log_cap) return;
            unsigned long long *r = P.unit_log + 1 + k * UNIT_LOG_WORDS;
            r[0] = lg[0]; r[1] = lg[1]; r[2] = lg[2]; r[3] = global_ns(); r[4] = blockIdx.x;
            r[5] = (unsigned long long)cnt | ((unsigned long long)nsurv << 32);
            r[6] = s_bytes - (lg[3] & ((1ull << 61) - 1)); r[7] = s_maxb; r[8] = lg[3];
            r[9] = lg[4]; r[10] = lg[5]; r[11] = lg[6];
        };
        if (s_nsurv < 2) {
            // No child frame (the common case): nothing to compact, write or
            // publish, so the unit ends here without further barriers.
            if (threadIdx.x == 0) {
                if (P.unit_log) log_unit(s_nsurv);
                c_inter += cnt;
                c_bytes += s_bytes;
                c_units += 1;
                c_surv += s_nsurv;
                if (P.root_cost) atomicAdd(P.root_cost + root, (unsigned long long)cnt);
                if (P.cta_time) c_busy += global_ns() - t_unit;
                // No fence: nothing this unit wrote is read before the kernel
                // ends, and pending only falls to zero when every unit is done.
                atomicAdd(&st->pending, ~0ull);  // pending -= 1
            }
            continue;
        }
        // Survivors move to the front of the block in member order, so every
        // child frame keeps its members sorted by column (the pattern tree is
        // then a prefix tree: a pattern's parent is itself minus its last item).
        if (fast && ok) {
            const uint32_t q = threadIdx.x;
            const bool keep = q < cnt && s_pid[q] != NO_PATTERN;
            const unsigned bal = __ballot_sync(CPM_FULL, keep);
            if (lane == 0) s_wtot[wid] = __popc(bal);
            __syncthreads();
            uint32_t before = 0, total = 0;
            for (unsigned w = 0; w < nw; ++w) {
                if (w < wid) before += s_wtot[w];
                total += s_wtot[w];
            }
            if (threadIdx.x == 0) {
                s_surv = 0;
                const unsigned long long mb = atomicAdd(&st->n_members, (unsigned long long)total);
                if (mb + total > P.members_cap) {
                    deep_fail(st, DEEP_ERR_MEMBERS);
                } else {
                    s_mem_base = mb;
                    s_surv = total;
                }
            }
            __syncthreads();
            if (keep && s_surv) {
                const uint32_t pos = before + __popc(bal & ((1u << lane) - 1));
                s_map[pos] = (uint16_t)q;
                P.mem_pat[s_mem_base + pos] = s_pid[q];
                P.mem_item[s_mem_base + pos] = __ldcg(P.mem_item + mem_off + p + 1 + q);
            }
        } else if (ok && s_mem_base + cnt <= P.members_cap) {
            uint32_t base = 0;
            for (uint32_t start = 0; start < cnt; start += blockDim.x) {
                const uint32_t q = start + threadIdx.x;
                const uint64_t src = s_mem_base + q;
                uint32_t e_pat = NO_PATTERN, e_item = 0;
                const uint64_t *e_bits = nullptr;
                if (q < cnt) {
                    e_pat = __ldcg(P.mem_pat + src);
                    e_item = __ldcg(P.mem_item + src);
                    e_bits = reinterpret_cast<const uint64_t *>(ld_raw_ptr(P.mem_bits + src));
                }
                const bool keep = e_pat != NO_PATTERN;
                const unsigned bal = __ballot_sync(CPM_FULL, keep);
                if (lane == 0) s_wtot[wid] = __popc(bal);
                __syncthreads();
                uint32_t before = 0, total = 0;
                for (unsigned w = 0; w < nw; ++w) {
                    if (w < wid) before += s_wtot[w];
                    total += s_wtot[w];
                }
                if (keep) {
                    const uint64_t dst = s_mem_base + base + before + __popc(bal & ((1u << lane) - 1));
                    P.mem_pat[dst] = e_pat;
                    P.mem_item[dst] = e_item;
                    P.mem_bits[dst] = e_bits;
                }
                base += total;
                __syncthreads();
            }
            if (threadIdx.x == 0) s_surv = base;
        } else if (threadIdx.x == 0) {
            s_surv = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0 && P.unit_log) lg[4] = global_ns();
        const uint32_t ns = s_surv;
        const bool expand = ns >= 2;
        // Projected children (bitsets of lstride words, numbered by rank in
        // the prefix) when the prefix holds at most local_max transactions.
        uint32_t lstride = 0, n_pre = 0;
        if (SMEM_PREFIX && P.local_max && !P.shallow && expand) {
            n_pre = __ldcg(P.pat_sup + parent_pat);
            if (n_pre >= 1 && n_pre <= P.local_max) lstride = 2u * ((n_pre + 127u) / 128u);
        }
        const bool proj = lstride != 0;
        // Words of the survivors' child tidsets (each dense or a list, by its support).
        uint64_t child_words = (uint64_t)ns * stride;
        uint64_t fast_wtot = 0;
        if (fast && expand) {
            // The survivors' siblings and supports, moved to their compacted
            // places, with their child offsets and work offsets from one scan
            // (child words in the high half, work units in the low half: each
            // sum stays below 2^32).
            const uint32_t i = threadIdx.x;
            unsigned long long raw = 0;
            uint32_t sc = 0;
            uint64_t sz = 0, wk = 0;
            if (i < ns) {
                const uint32_t q = s_map[i];
                raw = s_raw[q];
                sc = s_cnt[q];
                sz = proj ? lstride : (SMEM_PREFIX && as_list(P, sc, stride)) ? list_words(sc) : stride;
                wk = sibling_units<SMEM_PREFIX>(raw, n2);
            }
            uint64_t tot = 0;
            const uint64_t ex = block_excl_scan_u64((sz << 32) | wk, s_w64, &tot);
            if (i < ns) {
                s_raw[i] = raw;
                s_cnt[i] = sc;
                s_coff[i] = (uint32_t)(ex >> 32);
                s_off[i] = ex & 0xffffffffull;
            }
            if (i == 0) s_off[ns] = tot & 0xffffffffull;
            if (threadIdx.x < 32) s_clast[threadIdx.x] = 0;
            child_words = tot >> 32;
            fast_wtot = tot & 0xffffffffull;
        } else if (expand && proj) {
            child_words = (uint64_t)ns * lstride;
        } else if (expand && P.lists) {
            uint64_t part = 0;
            for (uint32_t i = threadIdx.x; i < ns; i += blockDim.x) {
                const uint32_t sc = __ldcg(P.pat_sup + __ldcg(P.mem_pat + s_mem_base + i));
                part += as_list(P, sc, stride) ? list_words(sc) : stride;
            }
            uint64_t tot = 0;
            block_excl_scan_u64(part, s_w64, &tot);
            child_words = tot;
        }
        // Children written row by row (the row-wise pass 2 below): always for
        // row-wise units, and for the other projected units of one database
        // when the prefix's rows (plus a ballot per 32 transactions and
        // survivor) are less work than the projected writers' pass over the
        // survivors' siblings, weighted by H_P2_WEIGHT (units of more than
        // blockDim siblings: always).
        const bool rows_p2 =
            SMEM_PREFIX && proj && P.h_rows &&
            (hmode || !fast ||
             (double)n_pre * ((double)P.h_cost + ns / 32.0) < H_P2_WEIGHT * (double)fast_wtot);
        if (threadIdx.x == 0) {
            s_grant = 0;
            s_fid = ~0ull;
            if (expand && ld_relaxed_u32(&st->error) == 0) {
                const unsigned long long ab = atomicAdd(&st->arena_next, (unsigned long long)child_words);
                if (ab + (unsigned long long)child_words > P.arena_words) deep_fail(st, DEEP_ERR_ARENA);
                else s_grant = 1;
                s_arena_base = ab;
            }
        }
        __syncthreads();
        uint16_t *const s_dir = reinterpret_cast<uint16_t *>(reinterpret_cast<char *>(s_prefix) + P.dir_off);
        if (SMEM_PREFIX && rows_p2 && s_grant && !hmode) {
            // The prefix's transaction ids, in order, from its bitmap and rank
            // directory into this CTA's scratch, for the row-wise pass 2.
            build_rank_dir(s_prefix, n2, s_dir, s_w64);
            __syncthreads();
            uint32_t *scr = P.h_scratch + (uint64_t)blockIdx.x * P.h_scratch_words;
            for (uint64_t v = threadIdx.x; v < n2; v += blockDim.x) {
                const ulonglong2 w = s_prefix[v];
                uint32_t r = s_dir[v];
                for (unsigned long long b = w.x; b; b &= b - 1, ++r)
                    if (r < P.h_scratch_words) scr[r] = (uint32_t)(v * 128 + __ffsll((long long)b) - 1);
                for (unsigned long long b = w.y; b; b &= b - 1, ++r)
                    if (r < P.h_scratch_words) scr[r] = (uint32_t)(v * 128 + 64 + __ffsll((long long)b) - 1);
            }
            if (threadIdx.x == 0) {
                const uint32_t last = (uint32_t)n2 - 1u;
                const uint32_t tot = (uint32_t)s_dir[last] + popc2(s_prefix[last]);
                if (tot != n_pre) deep_fail(st, DEEP_ERR_INTERNAL);
                s_hids = scr;
                s_hn = min(min(tot, n_pre), P.h_scratch_words);
            }
            __syncthreads();  // the ids are in place
        }
        if (SMEM_PREFIX && proj && s_grant && !rows_p2) {
            // Rank directory of the prefix, and the child block zeroed for
            // the bits the projected writers OR in.
            build_rank_dir(s_prefix, n2, s_dir, s_w64);
            uint64_t *blk = P.arena + s_arena_base;
            for (uint64_t i = threadIdx.x; i < child_words; i += blockDim.x) blk[i] = 0ull;
            __syncthreads();
            if (threadIdx.x == 0) {
                // The directory's total is the prefix's count: it must be the
                // support the projection was sized by (the writers stay inside
                // the child bitsets either way).
                const uint32_t last = (uint32_t)n2 - 1u;
                if ((uint32_t)s_dir[last] + popc2(s_prefix[last]) != n_pre) deep_fail(st, DEEP_ERR_INTERNAL);
            }
        }
        if (threadIdx.x == 0 && P.unit_log) lg[5] = global_ns();
        // ---- pass 2: child tidsets of the survivors (only when they recurse) ----
        // Per chunk of up to blockDim survivors: their siblings' work (list
        // ids or bitset words) is laid end to end and each warp takes an
        // equal slice, crossing child boundaries, so that every warp writes
        // even when few children survive.  A list child split over warps needs
        // each piece's first output position: a warp whose slice ends inside
        // a list child first counts that last piece (s_clast), and a warp that
        // starts inside one adds up the counts of the warps before it.
        if (SMEM_PREFIX && rows_p2 && s_grant) {
            // Row-wise children (projected): survivor k's child has bit j set
            // when the j-th transaction of the prefix holds survivor k's item.
            // A warp takes 32 consecutive transactions, each lane marks the
            // survivors in its row (64 at a time), and one ballot per survivor
            // is a whole 32-bit word of its child: plain stores, every word
            // written once, the padding after the last transaction zeroed.
            uint32_t *blk32 = reinterpret_cast<uint32_t *>(P.arena + s_arena_base);
            const uint32_t *const h_ids2 = s_hids;
            const uint32_t h_n2 = s_hn;
            const uint32_t nw32 = 2u * lstride, used32 = (h_n2 + 31u) / 32u;
            for (uint32_t g0 = 0; g0 < ns; g0 += 64) {
                const uint32_t gn = min(64u, ns - g0);
                // Survivor k's frequent index, from its member entry (in survivor order).
                uint32_t gf = H_NONE;
                if (threadIdx.x < gn) {
                    gf = __ldg(P.h_fidx + __ldcg(P.mem_item + s_mem_base + g0 + threadIdx.x));
                    if (gf < P.h_F) s_tab[gf] = (uint16_t)threadIdx.x;
                    else deep_fail(st, DEEP_ERR_INTERNAL);
                }
                __syncthreads();
                for (uint32_t w = wid; w < used32; w += nw) {
                    const uint32_t j = w * 32u + lane;
                    unsigned long long mark = 0;
                    if (j < h_n2) {
                        const uint32_t t = __ldcg(h_ids2 + j);
                        const uint32_t ra = __ldg(P.h_off + t), rb = __ldg(P.h_off + t + 1);
                        for (uint32_t k0 = ra; k0 < rb; k0 += 8) {
                            uint32_t f[8];
#pragma unroll
                            for (int u = 0; u < 8; ++u)
                                f[u] = k0 + u < rb ? (uint32_t)__ldg(P.h_rows + k0 + u) : H_NONE;
#pragma unroll
                            for (int u = 0; u < 8; ++u)
                                if (f[u] != H_NONE) {
                                    const uint32_t g = s_tab[f[u]];
                                    if (g < 64u) mark |= 1ull << g;
                                }
                        }
                    }
                    for (uint32_t k = 0; k < gn; ++k) {
                        const unsigned word = __ballot_sync(CPM_FULL, (unsigned)(mark >> k) & 1u);
                        if (lane == (k & 31u)) blk32[(uint64_t)(g0 + k) * nw32 + w] = word;
                    }
                }
                __syncthreads();  // the group's rows are read
                if (threadIdx.x < gn && gf < P.h_F) s_tab[gf] = H_NONE;
                __syncthreads();  // the table is empty again
            }
            const uint32_t pad = nw32 - used32;
            for (uint64_t i = threadIdx.x; i < (uint64_t)ns * pad; i += blockDim.x)
                blk32[(i / pad) * nw32 + used32 + i % pad] = 0u;
            for (uint32_t k = threadIdx.x; k < ns; k += blockDim.x)
                P.mem_bits[s_mem_base + k] = reinterpret_cast<const uint64_t *>(P.arena + s_arena_base + (uint64_t)k * lstride);
            __threadfence();
        } else if (s_grant) {
            uint64_t chunk_base = 0;
            for (uint32_t start = 0; start < ns; start += blockDim.x) {
                const uint32_t cn = min((uint32_t)blockDim.x, ns - start);
                uint64_t ctot = 0, wtot = fast_wtot;
                if (!fast) {
                uint64_t sz = 0, wk = 0;
                if (threadIdx.x < cn) {
                    const uint64_t m_out = s_mem_base + start + threadIdx.x;
                    const unsigned long long raw = ld_raw_ptr(P.mem_bits + m_out);
                    const uint32_t sc = P.lists ? __ldcg(P.pat_sup + __ldcg(P.mem_pat + m_out)) : 0u;
                    sz = proj ? lstride : (SMEM_PREFIX && as_list(P, sc, stride)) ? list_words(sc) : stride;
                    wk = sibling_units<SMEM_PREFIX>(raw, n2);
                    s_raw[threadIdx.x] = raw;
                    s_cnt[threadIdx.x] = sc;
                }
                const uint64_t cex = block_excl_scan_u64(sz, s_w64, &ctot);
                const uint64_t wex = block_excl_scan_u64(wk, s_w64, &wtot);
                if (threadIdx.x < cn) {
                    s_coff[threadIdx.x] = (uint32_t)(chunk_base + cex);
                    s_off[threadIdx.x] = wex;
                }
                if (threadIdx.x == 0) s_off[cn] = wtot;
                if (threadIdx.x < 32) s_clast[threadIdx.x] = 0;
                }
                __syncthreads();
                const uint64_t lo = wtot * wid / nw, hi = wtot * (wid + 1) / nw;
                uint32_t first = cn;  // first child whose work ends past lo
                if (lo < hi) {
                    uint32_t a = 0, b = cn;
                    while (a < b) {
                        const uint32_t mid = (a + b) >> 1;
                        if (s_off[mid + 1] <= lo) a = mid + 1; else b = mid;
                    }
                    first = a;
                    // The child this slice ends in, when it goes on past the slice.
                    uint32_t z = first;
                    while (z + 1 < cn && s_off[z + 1] < hi) ++z;
                    const bool list_child = SMEM_PREFIX && !proj && as_list(P, s_cnt[z], stride);
                    if (list_child && s_off[z + 1] > hi) {
                        uint32_t c = sibling_count_range<SMEM_PREFIX>(s_raw[z], max(lo, s_off[z]) - s_off[z],
                                                                      hi - s_off[z], s_prefix, s_p32, pb, mk, lane);
                        c = warp_sum_u32(c);
                        if (lane == 0) s_clast[wid] = c;
                    }
                }
                __syncthreads();
                for (uint32_t i = first; i < cn && s_off[i] < hi; ++i) {
                    const uint64_t u0 = max(lo, s_off[i]) - s_off[i], u1 = min(hi, s_off[i + 1]) - s_off[i];
                    const uint64_t units = s_off[i + 1] - s_off[i];
                    uint64_t *out = P.arena + s_arena_base + s_coff[i];
                    const uint32_t sc = s_cnt[i];
                    if (SMEM_PREFIX && proj) {
                        if (u0 < u1)
                            write_proj_piece(s_raw[i], u0, u1, s_prefix, s_p32, s_dir, reinterpret_cast<uint32_t *>(out),
                                             2u * lstride, lane);
                    } else if (SMEM_PREFIX && as_list(P, sc, stride)) {
                        uint32_t *o32 = reinterpret_cast<uint32_t *>(out);
                        uint32_t at = 0;
                        if (u0 > 0) {
                            // Ids written by the earlier warps that hold parts of this child.
                            for (uint32_t w = wid; w-- > 0;) {
                                at += s_clast[w];
                                if (wtot * w / nw <= s_off[i]) break;
                            }
                        }
                        if (u0 < u1) at = write_list_piece(s_raw[i], u0, u1, s_prefix, s_p32, o32, at, sc, lane);
                        if (u0 == 0 && lane == 0) {
                            o32[0] = sc;
                            o32[1] = o32[2] = o32[3] = 0u;
                        }
                        if (u1 == units) {
                            if (lane == 0 && at != sc) deep_fail(st, DEEP_ERR_INTERNAL);
                            // Ids the count promised but the pass did not find (only when the
                            // counts disagree, an error) become 0, an in-range id.
                            for (uint32_t j = at + lane; j < sc; j += 32) o32[4 + j] = 0u;
                            // Zero the padding after the last id.
                            const uint32_t end = 4 + sc, pad_end = (uint32_t)(list_words(sc) * 2);
                            if (lane < pad_end - end) o32[end + lane] = 0u;
                        }
                    } else if (u0 < u1) {
                        write_dense_piece<SMEM_PREFIX>(s_raw[i], u0, u1, s_prefix, pb, mk,
                                                       reinterpret_cast<ulonglong2 *>(out), lane);
                    }
                }
                __syncthreads();  // every piece of this chunk is written
                if (threadIdx.x < cn) {
                    const uint64_t *out = P.arena + s_arena_base + s_coff[threadIdx.x];
                    const bool lst = SMEM_PREFIX && !proj && as_list(P, s_cnt[threadIdx.x], stride);
                    P.mem_bits[s_mem_base + start + threadIdx.x] = reinterpret_cast<const uint64_t *>(
                        reinterpret_cast<unsigned long long>(out) | (lst ? 1ull : 0ull));
                }
                chunk_base += ctot;
                __syncthreads();
            }
            __threadfence();
            // Child blocks may later be staged by cp.async.bulk (async proxy).
            asm volatile("fence.proxy.async.global;" ::: "memory");
        }
        if (threadIdx.x == 0 && P.unit_log) lg[6] = global_ns();
        __syncthreads();
        if (threadIdx.x == 0 && s_grant) {
            const unsigned long long nf = atomicAdd(&st->n_frames, 1ull);
            // Shallow launches keep the child frame for the host (its
            // positions become root units of later rounds) instead of
            // queueing them.  A projected frame's units go to k_local's queue.
            const unsigned long long qb =
                P.shallow ? 0ull : atomicAdd(proj ? &st->lq_tail : &st->q_tail, (unsigned long long)(ns - 1));
            if (nf >= P.frames_cap) deep_fail(st, DEEP_ERR_FRAMES);
            else if (!P.shallow && qb + ns - 1 > (proj ? P.lq_cap : P.queue_cap)) deep_fail(st, DEEP_ERR_QUEUE);
            else {
                DFrame c;
                c.mask = nullptr;
                c.mem_off = s_mem_base;
                c.m = ns;
                c.root = root;
                c.stride = proj ? lstride : stride;
                c.db = db;
                c.minsup = minsup;
                c.bits = proj ? P.arena + s_arena_base : nullptr;
                P.frames[nf] = c;
                if (!P.shallow) {
                    atomicAdd(proj ? &st->lq_pending : &st->pending, (unsigned long long)(ns - 1));
                    __threadfence();
                    s_fid = nf;
                    s_qbase = qb;
                } else {
                    __threadfence();
                }
            }
        }
        __syncthreads();
        if (s_fid != ~0ull) {
            for (uint32_t i = threadIdx.x; i + 1 < ns; i += blockDim.x)
                st_release_u64((proj ? P.lq : P.queue) + s_qbase + i, (s_fid << 32) | i);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (P.unit_log) log_unit(ns);
            c_inter += cnt;
            c_bytes += s_bytes + (s_grant ? 8ull * child_words : 0ull);
            c_units += 1;
            c_surv += ns;
            if (P.root_cost) atomicAdd(P.root_cost + root, (unsigned long long)cnt);
            if (P.cta_time) c_busy += global_ns() - t_unit;
            // The child frame was published (fenced) above; its units were
            // added to pending before this unit leaves it.
            atomicAdd(&st->pending, ~0ull);  // pending -= 1
        }
    }
    if (threadIdx.x == 0 && P.cta_time) {
        P.cta_time[2 * blockIdx.x] = c_busy;
        P.cta_time[2 * blockIdx.x + 1] = global_ns();
    }
    if (threadIdx.x == 0 && c_units) {
        atomicAdd(&st->intersections, c_inter);
        atomicAdd(&st->bytes_alg, c_bytes);
        atomicAdd(&st->work_items, c_units);
        atomicAdd(&st->survivors, c_surv);
    }
}

}  // namespace cpm
