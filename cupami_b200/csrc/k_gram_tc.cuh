// Tensor-core pair Gram: C[i][j] = |t(f_i) & t(f_j)| for i < j as an exact
// INT8 GEMM D^T D on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Reference: the pair level of cuEclat.mine (cuEclat.py:183-193) and the
// second Apriori level (cuApriori.py:519-526) count every pair of frequent
// items with count_supports, one CUDA block per pair (_bitsets.py:30-53).
// Here the 0/1 matrix D (transactions x items) never exists in HBM: producer
// warps read 16 bytes of tidset bits per row and expand them to 128 int8
// 0/1 values directly in shared memory, in the UMMA K-major SWIZZLE_128B
// layout.  One elected thread issues tcgen05.mma.kind::i8 (M=128, N=256,
// K=32 per instruction, INT32 accumulators in TMEM).  Counts are exact.
//
// CTA: 12 producer warps (one A or B row each per stage: 128 + 256 rows) +
// 1 MMA warp; 4 pipeline stages of 48 KB.  Units: upper-triangle output tiles
// x K-splits; partial sums are added into C with atomics (C zeroed first).
// Every mbarrier wait is bounded; a wait that runs out raises a shared abort
// flag, the CTA drains its issued MMAs (bounded), frees TMEM and returns, and
// the host sees the error word.
#pragma once
#include "common.cuh"
#include "k_batch.cuh"

namespace cpm {
namespace tc {

constexpr int BM = 128;           // A rows (items) per tile
constexpr int BN = 256;           // B rows (items) per tile
constexpr int BK = 128;           // transactions (int8 K elements) per stage
constexpr int STAGES = 4;
constexpr int A_BYTES = BM * BK;  // 16 KB
constexpr int B_BYTES = BN * BK;  // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int PRODUCER_WARPS = (BM + BN) / 32;  // 12: one row per producer thread
constexpr int MMA_WARP = PRODUCER_WARPS;
constexpr int THREADS = (PRODUCER_WARPS + 1) * 32;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + alignment slack
constexpr uint32_t TMEM_COLS = BN;  // 256 int32 accumulator columns
constexpr unsigned long long WAIT_LIMIT = 1ull << 22;  // try_wait rounds

// kind::i8 instruction descriptor: D S32, A/B unsigned 8-bit, both K-major,
// N = 256 (N >> 3 at bit 17), M = 128 (M >> 4 at bit 24).
constexpr uint32_t IDESC = (2u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

// Shared-memory matrix descriptor, K-major SWIZZLE_128B: 8-row atoms of
// 128-byte rows, 1024 bytes apart (SBO), LBO unused (1), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; returns false (and raises *abort) if it ran out or another
// thread aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort) {
    for (unsigned long long i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try(bar, parity)) return true;
        if (*abort) return false;
    }
    *abort = 1;
    return false;
}

__device__ __forceinline__ uint32_t expand4(uint32_t nib) {
    // bits b0..b3 -> bytes 0..3 (0x00 or 0x01): nib * (1 + 2^7 + 2^14 + 2^21)
    return (nib * 0x00204081u) & 0x01010101u;
}

}  // namespace tc

// One unit: database db, A block ti (128 rows), B block tj (256 columns),
// words [kw_begin, kw_end) of the tidsets (a whole number of 2-word stages).
struct GramUnit {
    uint32_t db, ti, tj, pad;
    uint64_t kw_begin, kw_end;
};

// C of every database must be zeroed.  *err gets a nonzero word if any wait
// ran out.
__global__ void __launch_bounds__(tc::THREADS, 1)
    k_gram_tc(const DbDesc *__restrict__ dbs, const GramUnit *__restrict__ units, unsigned int *__restrict__ err) {
    using namespace tc;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];
    __shared__ __align__(8) uint64_t empty_bar[STAGES];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_base_slot;
    __shared__ int abort_flag;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const GramUnit tile = units[blockIdx.x];
    const DbDesc D = dbs[tile.db];
    const uint64_t *__restrict__ bits = D.bits;
    const uint64_t stride = D.stride;
    const uint32_t *__restrict__ freq = D.freq;
    const uint32_t F = D.F;
    uint32_t *__restrict__ C = D.C;
    const uint64_t kw_begin = tile.kw_begin;
    const uint64_t kw_end = min(stride, tile.kw_end);
    const uint32_t n_k = kw_end > kw_begin ? (uint32_t)((kw_end - kw_begin + 1) / 2) : 0;  // 2 words per stage

    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            tc::mbar_init(tc::smem_u32(&full_bar[s]), PRODUCER_WARPS * 32);
            tc::mbar_init(tc::smem_u32(&empty_bar[s]), 1);
        }
        tc::mbar_init(tc::smem_u32(&done_bar), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == MMA_WARP) {
        const uint32_t slot = tc::smem_u32(&tmem_base_slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;
    volatile int *abort = &abort_flag;

    if (warp < PRODUCER_WARPS) {
        // ---- producers: one row of A (r < 128) or B per thread per stage ----
        const uint32_t r = threadIdx.x;
        const bool is_a = r < BM;
        const uint32_t row = is_a ? r : r - BM;
        const uint64_t g = is_a ? (uint64_t)tile.ti * BM + row : (uint64_t)tile.tj * BN + row;
        const ulonglong2 *src =
            g < F ? reinterpret_cast<const ulonglong2 *>(bits + (uint64_t)freq[g] * stride + kw_begin) : nullptr;
        const uint32_t atom = row >> 3, rr = row & 7;
        const uint32_t row_off = (is_a ? 0u : (uint32_t)A_BYTES) + atom * 1024u + rr * 128u;
        // Loads run three stages ahead of the expansion, so that their latency
        // overlaps the wait for a free stage and the expansions before it.
        const ulonglong2 zero = make_ulonglong2(0, 0);
        ulonglong2 w1 = (src && n_k > 0) ? src[0] : zero;
        ulonglong2 w2 = (src && n_k > 1) ? src[1] : zero;
        ulonglong2 w3 = (src && n_k > 2) ? src[2] : zero;
        for (uint32_t kt = 0; kt < n_k; ++kt) {
            const uint32_t s = kt % STAGES, ph = (kt / STAGES) & 1u;
            const ulonglong2 w = w1;
            w1 = w2;
            w2 = w3;
            w3 = (src && kt + 3 < n_k) ? src[kt + 3] : zero;
            if (!tc::mbar_wait(tc::smem_u32(&empty_bar[s]), ph ^ 1u, abort)) break;
            unsigned char *dst = smem + (uint32_t)s * STAGE_BYTES + row_off;
#pragma unroll
            for (uint32_t c = 0; c < 8; ++c) {
                const uint64_t word = c < 4 ? w.x : w.y;
                const uint32_t b16 = (uint32_t)(word >> (16 * (c & 3))) & 0xFFFFu;
                uint4 v;
                v.x = tc::expand4(b16 & 0xF);
                v.y = tc::expand4((b16 >> 4) & 0xF);
                v.z = tc::expand4((b16 >> 8) & 0xF);
                v.w = tc::expand4(b16 >> 12);
                *reinterpret_cast<uint4 *>(dst + ((c ^ rr) << 4)) = v;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc::mbar_arrive(tc::smem_u32(&full_bar[s]));
        }
    } else {
        // ---- MMA issuer: one elected thread ----
        if (lane == 0) {
            const uint32_t base = tc::smem_u32(smem);
            uint32_t kt = 0;
            for (; kt < n_k; ++kt) {
                const uint32_t s = kt % STAGES, ph = (kt / STAGES) & 1u;
                if (!tc::mbar_wait(tc::smem_u32(&full_bar[s]), ph, abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_addr = base + s * STAGE_BYTES;
                const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
                for (uint32_t kk = 0; kk < BK / 32; ++kk) {
                    const uint64_t ad = tc::smem_desc(a_addr + kk * 32);
                    const uint64_t bd = tc::smem_desc(b_addr + kk * 32);
                    const uint32_t acc = (kt | kk) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                        ::"r"(tmem), "l"(ad), "l"(bd), "r"(IDESC), "r"(acc)
                        : "memory");
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 tc::smem_u32(&empty_bar[s]))
                             : "memory");
            }
            // Signals the epilogue once every issued MMA has completed (also on abort).
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             tc::smem_u32(&done_bar))
                         : "memory");
        }
        __syncwarp();
    }

    // ---- epilogue: warps 0..7, lane quarter (warp % 4), column half (warp / 4) ----
    if (warp < 8) {
        // done_bar is committed even after an abort: waiting on it (bounded,
        // whatever the abort flag says) drains every issued MMA before TMEM
        // is read or freed.
        bool done = false;
        for (unsigned long long i = 0; i < WAIT_LIMIT && !done; ++i) done = tc::mbar_try(tc::smem_u32(&done_bar), 0);
        if (!done) *abort = 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const bool ok = done && !*abort && n_k > 0;
        if (ok) {
            const uint32_t quarter = warp & 3, half = warp >> 2;
            const uint64_t gi = (uint64_t)tile.ti * BM + quarter * 32 + lane;
            for (uint32_t cc = 0; cc < BN / 2; cc += 32) {
                const uint32_t col0 = half * (BN / 2) + cc;
                const uint32_t taddr = tmem + ((quarter * 32u) << 16) + col0;
                uint32_t v[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (gi < F) {
#pragma unroll
                    for (uint32_t j = 0; j < 32; ++j) {
                        const uint64_t gj = (uint64_t)tile.tj * BN + col0 + j;
                        if (gi < gj && gj < F && v[j]) atomicAdd(C + gi * F + gj, v[j]);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0 && abort_flag) atomicOr(err, 1u);
    if (warp == MMA_WARP) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
    }
}

// Use the tensor cores when the Gram is large enough to fill the GPU.
inline bool gram_tc_worthwhile(uint32_t F, uint64_t n_tx) {
    return F >= 96 && (double)n_tx * F * F >= 2e9;
}

}  // namespace cpm
