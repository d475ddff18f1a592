// cupami_b200 runtime: the C ABI declared in include/cupami_b200.h.
//
// Host side of the vertical-bitset miner: device memory, database loading,
// the Eclat and Apriori drivers, and result ordering.  All arithmetic on
// transactions runs in the CUDA kernels included below; the host only plans
// (buffer sizes, class order) and moves counts and results.
#include "../../include/cupami_b200.h"
#include "common.cuh"
#include "k_basic.cuh"
#include "k_pairs.cuh"
#include "k_batch.cuh"
#include "k_gram_tc.cuh"
#include "k_deep.cuh"
#include "k_local.cuh"
#include "k_rows.cuh"
#include "k_apriori.cuh"
#include "k_periodic.cuh"
#include "k_costmodel.cuh"
#include "k_units.cuh"
#include "k_text.cuh"
#include <cub/device/device_radix_sort.cuh>

#include <cub/device/device_scan.cuh>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_set>
#include <vector>
#include <map>
#include <memory>
#include <array>
#include <chrono>
#include <cstdlib>
#include <mutex>
#include <deque>
#include <cmath>

using namespace cpm;

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

struct cpm_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    std::string err;
    bool tc_ok = true;        // tensor-core Gram usable on this device
    size_t mem_free = 0;      // free device memory when the context was made
    int deep_occ_smem = -1;   // k_deep<true> CTAs per SM, for deep_occ_bytes of prefix
    size_t deep_occ_bytes = 0;
    int deep_occ_global = -1; // k_deep<false> CTAs per SM
    int local_occ = -1;       // k_local CTAs per SM
    unsigned deep_occ_block = 0;  // block size the occupancies above were taken for
    std::vector<float> model;  // cost-model parameters (empty: none loaded)
    float last_deep_ms = 0.f;  // deep-phase kernel time of the last bounded-round run
    uint32_t deep_balance = 0;  // k_deep pass 1 of the current mine: 1 siblings split by size, 0 warp each
    int last_deep_block = 0, last_deep_ctas = 0;  // launch shape of the last deep phase
    size_t l2_bytes = 126ull << 20;               // device L2 size (cpm_init)
    void *pinned = nullptr;                       // host staging for uploads (stage_upload)
    size_t pinned_bytes = 0;
    std::map<int, std::pair<int, int>> tune;      // log2(stride) -> (threads per CTA, CTAs per SM), cpm_autotune
    std::map<int, int> tune_lists;                // log2(stride) -> list divisor (0: bitsets only), cpm_autotune
    // Deep-level buffer sizes the last Eclat mine of a database of this shape
    // needed (transactions, items, frequent pairs, threshold), so that a
    // database loaded again (the drop-in reloads per mine()) starts there.
    std::map<std::array<uint64_t, 4>, std::array<uint64_t, 5>> plan_hints;
};

struct cpm_db {
    cpm_ctx *ctx = nullptr;
    uint64_t n_tx = 0, words = 0, stride = 2;
    uint32_t n_items = 0;
    uint64_t *d_bits = nullptr;
    uint32_t *d_support = nullptr;
    std::vector<uint32_t> labels;  // raw ids in column order (cpm_db_from_ids)
    // Temporal databases (cpm_tdb_from_csr): every row kept, with its timestamp.
    long long *d_ts = nullptr;
    long long end = 0;
    bool temporal = false;
    // Deep-level buffer sizes that the last mine() of this database needed.
    uint64_t hint_frames = 0, hint_members = 0, hint_queue = 0, hint_patterns = 0, hint_arena = 0;
};

struct cpm_result {
    std::vector<uint32_t> parent, item, support;
    std::vector<int64_t> period;  // periodic-frequent results only (cpm_mine_periodic)
    cpm_stats stats{};
    int algo = CPM_ECLAT;
    // Per root unit, when traced: cost-model features and log1p(subtree intersections)
    std::vector<float> trace_x, trace_y;
};

static int set_err(cpm_ctx *ctx, int code, const char *fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? CPM_ENOMEM : CPM_ECUDA,      \
                           "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,  \
                           __LINE__);                                                          \
    } while (0)

#define CKR(expr)                 \
    do {                          \
        int r_ = (expr);          \
        if (r_ != CPM_OK) return r_; \
    } while (0)

template <class T>
static int dalloc(cpm_ctx *ctx, T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocAsync((void **)p, count * sizeof(T), ctx->stream);
    if (e == cudaErrorMemoryAllocation) {
        // Blocks freed earlier stay reserved by the stream-ordered pool: once
        // the stream has passed their frees, hand them back and try again.
        cudaGetLastError();
        cudaMemPool_t pool;
        if (cudaStreamSynchronize(ctx->stream) == cudaSuccess &&
            cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess)
            cudaMemPoolTrimTo(pool, 0);
        e = cudaMallocAsync((void **)p, count * sizeof(T), ctx->stream);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return set_err(ctx, CPM_ENOMEM, "device allocation of %zu bytes failed: %s",
                       count * sizeof(T), cudaGetErrorString(e));
    }
    return CPM_OK;
}

template <class T>
static void dfree(cpm_ctx *ctx, T *&p) {
    if (p) cudaFreeAsync((void *)p, ctx->stream);
    p = nullptr;
}

// RAII list of device buffers freed at scope exit (stream ordered).
struct DevScope {
    cpm_ctx *ctx;
    std::vector<void *> ptrs;
    explicit DevScope(cpm_ctx *c) : ctx(c) {}
    template <class T>
    int alloc(T **p, size_t count) {
        int r = dalloc(ctx, p, count);
        if (r == CPM_OK) ptrs.push_back((void *)*p);
        return r;
    }
    ~DevScope() {
        for (void *p : ptrs) cudaFreeAsync(p, ctx->stream);
    }
};

extern "C" const char *cpm_version(void) { return "cupami_b200 0.1 (sm_100a)"; }

extern "C" int cpm_default_opts(cpm_opts *o) {
    if (!o) return CPM_EINVAL;
    memset(o, 0, sizeof *o);
    o->scheduler = CPM_SCHED_PLAIN;
    o->spin_limit = 1ull << 26;
    return CPM_OK;
}

extern "C" int cpm_init(int device, cpm_ctx **out) {
    if (!out) return CPM_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return CPM_ENODEV;
    }
    if (device < 0 || device >= n) return CPM_EINVAL;
    cpm_ctx *ctx = new cpm_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    for (int i = 0; i < 8 && e == cudaSuccess; ++i) e = cudaEventCreate(&ctx->ev[i]);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    int l2 = 0;
    if (e == cudaSuccess && cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device) == cudaSuccess && l2 > 0)
        ctx->l2_bytes = (size_t)l2;
    int major = 0, minor = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device);
    if (e == cudaSuccess) {
        // Keep freed blocks in the stream-ordered pool between calls.
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return CPM_ECUDA;
    }
    ctx->tc_ok = (major == 10 && minor == 0);
    size_t total = 0;
    cudaMemGetInfo(&ctx->mem_free, &total);
    // The deep kernel stages prefixes of up to DEEP_SMEM_PREFIX_MAX bytes in shared memory.
    cudaFuncSetAttribute(k_deep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DEEP_SMEM_PREFIX_MAX);
    cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES);
    cudaGetLastError();
    *out = ctx;
    return CPM_OK;
}

// Databases made on the context must be freed first (they point to it).
extern "C" void cpm_shutdown(cpm_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    delete ctx;
}

extern "C" const char *cpm_last_error(const cpm_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

extern "C" void *cpm_stream(const cpm_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" int cpm_synchronize(cpm_ctx *ctx) {
    if (!ctx) return CPM_EINVAL;
    CK(cudaStreamSynchronize(ctx->stream));
    return CPM_OK;
}

// ---------------------------------------------------------------------------
// databases
// ---------------------------------------------------------------------------

// Offsets of the non-empty rows only (empty baskets are dropped and the rest
// renumbered in order, cuApriori.py:391-392).
// Presence bitmaps up to this many 32-bit words (id range 0..393,215) are
// built in shared memory (48 KB, the default dynamic shared-memory limit).
constexpr uint64_t CPM_MARK_SMEM_WORDS = 12288;

static int compact_offsets(cpm_ctx *ctx, const uint64_t *offsets, uint64_t n_rows, uint64_t nnz,
                           std::vector<uint64_t> &out) {
    out.clear();
    out.reserve(n_rows + 1);
    if (n_rows == 0) {
        if (nnz) return set_err(ctx, CPM_EINVAL, "nnz must be 0 when there are no rows");
        out.push_back(0);
        return CPM_OK;
    }
    if (offsets[0] != 0 || offsets[n_rows] != nnz)
        return set_err(ctx, CPM_EINVAL, "offsets must start at 0 and end at nnz");
    out.push_back(0);
    for (uint64_t r = 0; r < n_rows; ++r) {
        if (offsets[r + 1] < offsets[r]) return set_err(ctx, CPM_EINVAL, "offsets must be nondecreasing");
        if (offsets[r + 1] > offsets[r]) out.push_back(offsets[r + 1]);
    }
    return CPM_OK;
}

// The offsets as uploaded: the caller's own array when no basket is empty
// (checked in parallel), else the compacted copy in `storage`.
static int offsets_view(cpm_ctx *ctx, const uint64_t *offsets, uint64_t n_rows, uint64_t nnz,
                        std::vector<uint64_t> &storage, const uint64_t **view, uint64_t *n_view) {
    if (n_rows && offsets[0] == 0 && offsets[n_rows] == nnz) {
        int bad = 0, empty = 0;
#pragma omp parallel for reduction(| : bad, empty) schedule(static) if (n_rows > (1u << 16))
        for (int64_t r = 0; r < (int64_t)n_rows; ++r) {
            bad |= offsets[r + 1] < offsets[r];
            empty |= offsets[r + 1] == offsets[r];
        }
        if (bad) return set_err(ctx, CPM_EINVAL, "offsets must be nondecreasing");
        if (!empty) {
            *view = offsets;
            *n_view = n_rows + 1;
            return CPM_OK;
        }
    }
    CKR(compact_offsets(ctx, offsets, n_rows, nnz, storage));
    *view = storage.data();
    *n_view = storage.size();
    return CPM_OK;
}

// Uploads of 16-256 MB go through pinned memory the context keeps, filled by
// a parallel copy; smaller and larger ones are copied from pageable memory.  The staging buffer is reused
// only after the caller has synchronised the stream (every loader does).
static int stage_upload(cpm_ctx *ctx, const std::vector<std::pair<void *, std::pair<const void *, size_t>>> &parts) {
    size_t total = 0;
    for (auto &pt : parts) total += (pt.second.second + 255) & ~(size_t)255;
    if (total == 0) return CPM_OK;
    // Small uploads: the driver's own pageable path is as fast (measured);
    // very large ones would pin too much host memory.
    if (total < (16ull << 20) || total > (256ull << 20)) {
        for (auto &pt : parts)
            if (pt.second.second)
                CK(cudaMemcpyAsync(pt.first, pt.second.first, pt.second.second, cudaMemcpyHostToDevice, ctx->stream));
        return CPM_OK;
    }
    if (ctx->pinned_bytes < total) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        const size_t want = std::max<size_t>(total, 16ull << 20);
        if (cudaHostAlloc(&ctx->pinned, want, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            ctx->pinned = nullptr;
            for (auto &pt : parts)
                if (pt.second.second)
                    CK(cudaMemcpyAsync(pt.first, pt.second.first, pt.second.second, cudaMemcpyHostToDevice,
                                       ctx->stream));
            return CPM_OK;
        }
        ctx->pinned_bytes = want;
    }
    size_t at = 0;
    for (auto &pt : parts) {
        unsigned char *dst = static_cast<unsigned char *>(ctx->pinned) + at;
        const unsigned char *src = static_cast<const unsigned char *>(pt.second.first);
        const size_t n = pt.second.second, chunk = 1u << 20;
#pragma omp parallel for schedule(static) if (n > (1u << 20))
        for (int64_t c = 0; c < (int64_t)((n + chunk - 1) / chunk); ++c)
            memcpy(dst + c * chunk, src + c * chunk, std::min(chunk, n - c * chunk));
        if (n) CK(cudaMemcpyAsync(pt.first, dst, n, cudaMemcpyHostToDevice, ctx->stream));
        at += (n + 255) & ~(size_t)255;
    }
    return CPM_OK;
}

static int db_alloc_bits(cpm_ctx *ctx, cpm_db *db) {
    db->words = (db->n_tx + 63) / 64;
    db->stride = std::max<uint64_t>(2, (db->words + 1) & ~1ull);
    CKR(dalloc(ctx, &db->d_bits, (size_t)std::max<uint32_t>(1, db->n_items) * db->stride));
    CKR(dalloc(ctx, &db->d_support, db->n_items));
    CK(cudaMemsetAsync(db->d_bits, 0, (size_t)std::max<uint32_t>(1, db->n_items) * db->stride * 8, ctx->stream));
    return CPM_OK;
}

static int db_pack(cpm_ctx *ctx, cpm_db *db, const uint64_t *d_off, const uint32_t *d_ids,
                   const uint32_t *d_lut) {
    if (db->n_tx) {
        const unsigned threads = 256;
        const unsigned blocks = (unsigned)((db->n_tx + threads - 1) / threads);
        k_pack<<<blocks, threads, 0, ctx->stream>>>(d_off, d_ids, d_lut, db->n_tx, db->stride,
                                                    reinterpret_cast<uint32_t *>(db->d_bits));
        CK(cudaGetLastError());
    }
    if (db->n_items) {
        const unsigned threads = 256;
        const unsigned blocks = (unsigned)(((uint64_t)db->n_items * 32 + threads - 1) / threads);
        k_item_support<<<blocks, threads, 0, ctx->stream>>>(db->d_bits, db->stride, db->n_items, db->d_support);
        CK(cudaGetLastError());
    }
    return CPM_OK;
}

extern "C" int cpm_db_from_csr(cpm_ctx *ctx, const uint64_t *offsets, uint64_t n_rows,
                               const uint32_t *cols, uint64_t nnz, uint32_t n_items, cpm_db **out) {
    if (!ctx || !out || (!offsets && n_rows) || (!cols && nnz)) return CPM_EINVAL;
    *out = nullptr;
    CK(cudaSetDevice(ctx->device));
    std::vector<uint64_t> off;
    CKR(compact_offsets(ctx, offsets, n_rows, nnz, off));
    for (uint64_t k = 0; k < nnz; ++k)
        if (cols[k] >= n_items) return set_err(ctx, CPM_EINVAL, "column %u out of range (n_items %u)", cols[k], n_items);
    cpm_db *db = new cpm_db();
    db->ctx = ctx;
    db->n_tx = off.size() - 1;
    db->n_items = n_items;
    int r = db_alloc_bits(ctx, db);
    DevScope tmp(ctx);
    uint64_t *d_off = nullptr;
    uint32_t *d_ids = nullptr;
    if (r == CPM_OK) r = tmp.alloc(&d_off, off.size());
    if (r == CPM_OK) r = tmp.alloc(&d_ids, nnz);
    if (r == CPM_OK && cudaMemcpyAsync(d_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        r = set_err(ctx, CPM_ECUDA, "offset upload failed");
    if (r == CPM_OK && nnz && cudaMemcpyAsync(d_ids, cols, nnz * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        r = set_err(ctx, CPM_ECUDA, "column upload failed");
    if (r == CPM_OK) r = db_pack(ctx, db, d_off, d_ids, nullptr);
    if (r == CPM_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        r = set_err(ctx, CPM_ECUDA, "pack failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (r != CPM_OK) {
        cpm_db_free(db);
        return r;
    }
    *out = db;
    return CPM_OK;
}

// Temporal database (cupami/periodicFrequentPattern/_temporal.py:109-147):
// rows in timestamp order and every row kept -- an empty basket keeps its
// timestamp and counts in the support denominator -- with the timestamps on
// the device beside the tidsets.  The periodic miner prunes on the timestamps
// being sorted and nonnegative (as the reference requires, _temporal.py:89-99);
// end closes the last gap.
extern "C" int cpm_tdb_from_csr(cpm_ctx *ctx, const uint64_t *offsets, uint64_t n_rows, const uint32_t *cols,
                                uint64_t nnz, uint32_t n_items, const int64_t *timestamps, int64_t end,
                                cpm_db **out) {
    if (!ctx || !out || (!offsets && n_rows) || (!cols && nnz) || (!timestamps && n_rows)) return CPM_EINVAL;
    *out = nullptr;
    CK(cudaSetDevice(ctx->device));
    if (!n_rows && nnz) return set_err(ctx, CPM_EINVAL, "nnz must be 0 when there are no rows");
    if (n_rows) {
        if (offsets[0] != 0 || offsets[n_rows] != nnz)
            return set_err(ctx, CPM_EINVAL, "offsets must start at 0 and end at nnz");
        for (uint64_t r = 0; r < n_rows; ++r) {
            if (offsets[r + 1] < offsets[r]) return set_err(ctx, CPM_EINVAL, "offsets must be nondecreasing");
            if (r && timestamps[r] < timestamps[r - 1])
                return set_err(ctx, CPM_EINVAL, "timestamps must be nondecreasing (rows sorted by timestamp)");
        }
        if (timestamps[0] < 0) return set_err(ctx, CPM_EINVAL, "timestamps must be nonnegative");
        if (end < timestamps[n_rows - 1]) return set_err(ctx, CPM_EINVAL, "end must be at least the last timestamp");
    }
    for (uint64_t k = 0; k < nnz; ++k)
        if (cols[k] >= n_items) return set_err(ctx, CPM_EINVAL, "column %u out of range (n_items %u)", cols[k], n_items);
    cpm_db *db = new cpm_db();
    db->ctx = ctx;
    db->n_tx = n_rows;
    db->n_items = n_items;
    db->temporal = true;
    db->end = end;
    int r = db_alloc_bits(ctx, db);
    if (r == CPM_OK) r = dalloc(ctx, &db->d_ts, n_rows);
    DevScope tmp(ctx);
    uint64_t *d_off = nullptr;
    uint32_t *d_ids = nullptr;
    if (r == CPM_OK) r = tmp.alloc(&d_off, n_rows + 1);
    if (r == CPM_OK) r = tmp.alloc(&d_ids, nnz);
    if (r == CPM_OK && n_rows)
        r = stage_upload(ctx, {{d_off, {offsets, (n_rows + 1) * 8}}, {d_ids, {cols, nnz * 4}},
                               {db->d_ts, {timestamps, n_rows * 8}}});
    if (r == CPM_OK) r = db_pack(ctx, db, d_off, d_ids, nullptr);
    if (r == CPM_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        r = set_err(ctx, CPM_ECUDA, "pack failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (r != CPM_OK) {
        cpm_db_free(db);
        return r;
    }
    *out = db;
    return CPM_OK;
}

// Decimal-string order of integer labels: "1" < "10" < "100" < "11" < "2".
static inline uint64_t decimal_key(uint32_t v) {
    char d[10];
    int n = 0;
    do { d[n++] = (char)(v % 10); v /= 10; } while (v);
    uint64_t key = 0;
    for (int i = 0; i < 10; ++i) key = key * 11 + (i < n ? (uint64_t)d[n - 1 - i] + 1 : 0);
    return key;
}

extern "C" int cpm_db_from_ids(cpm_ctx *ctx, const uint64_t *offsets, uint64_t n_rows,
                               const uint32_t *ids, uint64_t nnz, cpm_db **out) {
    if (!ctx || !out || (!offsets && n_rows) || (!ids && nnz)) return CPM_EINVAL;
    *out = nullptr;
    const bool dbg = getenv("CPM_DEBUG") != nullptr;
    auto t0 = std::chrono::steady_clock::now();
    auto lap = [&](const char *what) {
        if (!dbg) return;
        const auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "cpm: load %-20s %.3f ms\n", what, std::chrono::duration<double, std::milli>(now - t0).count());
        t0 = now;
    };
    CK(cudaSetDevice(ctx->device));
    std::vector<uint64_t> off_store;
    const uint64_t *offv = nullptr;
    uint64_t n_off = 0;
    CKR(offsets_view(ctx, offsets, n_rows, nnz, off_store, &offv, &n_off));
    lap("offsets");
    uint32_t max_id = 0;
#pragma omp parallel for reduction(max : max_id) schedule(static) if (nnz > (1u << 18))
    for (int64_t k = 0; k < (int64_t)nnz; ++k) max_id = std::max(max_id, ids[k]);
    DevScope tmp(ctx);
    uint64_t *d_off = nullptr;
    uint32_t *d_ids = nullptr, *d_lut = nullptr, *d_present = nullptr;
    CKR(tmp.alloc(&d_off, n_off));
    CKR(tmp.alloc(&d_ids, nnz));
    CKR(stage_upload(ctx, {{d_off, {offv, n_off * 8}}, {d_ids, {ids, nnz * 4}}}));
    // Distinct ids: a presence bitmap over [0, max_id] built on the device.
    const uint64_t pw = (uint64_t)max_id / 32 + 1;
    CKR(tmp.alloc(&d_present, pw));
    CK(cudaMemsetAsync(d_present, 0, pw * 4, ctx->stream));
    if (nnz) {
        if (pw <= CPM_MARK_SMEM_WORDS) {
            const unsigned blocks = (unsigned)std::min<uint64_t>((nnz + 1023) / 1024, (uint64_t)ctx->sms * 2);
            k_mark_ids_smem<<<blocks, 1024, pw * 4, ctx->stream>>>(d_ids, nnz, (uint32_t)pw, d_present);
        } else {
            const unsigned blocks = (unsigned)std::min<uint64_t>((nnz + 255) / 256, (uint64_t)ctx->sms * 16);
            k_mark_ids<<<blocks, 256, 0, ctx->stream>>>(d_ids, nnz, d_present);
        }
        CK(cudaGetLastError());
    }
    lap("max id, upload, mark");
    std::vector<uint32_t> present(pw);
    CK(cudaMemcpyAsync(present.data(), d_present, pw * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    lap("presence sync");
    std::vector<uint32_t> uniq;
    for (uint64_t w = 0; w < pw; ++w)
        for (uint32_t m = present[w]; m; m &= m - 1) uniq.push_back((uint32_t)(w * 32 + __builtin_ctz(m)));
    std::vector<uint64_t> keys(uniq.size());
    for (size_t i = 0; i < uniq.size(); ++i) keys[i] = decimal_key(uniq[i]);
    std::vector<uint32_t> order(uniq.size());
    std::iota(order.begin(), order.end(), 0u);
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    cpm_db *db = new cpm_db();
    db->ctx = ctx;
    db->n_tx = n_off - 1;
    db->n_items = (uint32_t)uniq.size();
    db->labels.resize(uniq.size());
    // Column lookup: dense table over the id range when it is small enough,
    // otherwise ids are first replaced by their rank among the distinct ids.
    std::vector<uint32_t> rank(uniq.size());
    for (size_t c = 0; c < order.size(); ++c) {
        db->labels[c] = uniq[order[c]];
        rank[order[c]] = (uint32_t)c;
    }
    int r = db_alloc_bits(ctx, db);
    if (r == CPM_OK) {
        if ((uint64_t)max_id < (1ull << 26)) {
            std::vector<uint32_t> lut((uint64_t)max_id + 1, 0);
            for (size_t i = 0; i < uniq.size(); ++i) lut[uniq[i]] = rank[i];
            r = tmp.alloc(&d_lut, lut.size());
            if (r == CPM_OK &&
                cudaMemcpyAsync(d_lut, lut.data(), lut.size() * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
                r = set_err(ctx, CPM_ECUDA, "lookup upload failed");
            if (r == CPM_OK) r = db_pack(ctx, db, d_off, d_ids, d_lut);
            if (r == CPM_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                r = set_err(ctx, CPM_ECUDA, "pack failed");
        } else {
            std::vector<uint32_t> cols(nnz);
            for (uint64_t k = 0; k < nnz; ++k)
                cols[k] = rank[std::lower_bound(uniq.begin(), uniq.end(), ids[k]) - uniq.begin()];
            if (nnz && cudaMemcpyAsync(d_ids, cols.data(), nnz * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
                r = set_err(ctx, CPM_ECUDA, "column upload failed");
            if (r == CPM_OK) r = db_pack(ctx, db, d_off, d_ids, nullptr);
            if (r == CPM_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                r = set_err(ctx, CPM_ECUDA, "pack failed");
        }
    }
    if (r != CPM_OK) {
        cpm_db_free(db);
        return r;
    }
    lap("labels, table, pack");
    *out = db;
    return CPM_OK;
}

extern "C" int cpm_db_from_ids_batch(cpm_ctx *ctx, uint32_t n_db, const uint64_t *const *offsets,
                                     const uint64_t *n_rows, const uint32_t *const *ids, const uint64_t *nnz,
                                     cpm_db **out) {
    if (!ctx || !out || (n_db && (!offsets || !n_rows || !ids || !nnz))) return CPM_EINVAL;
    for (uint32_t d = 0; d < n_db; ++d) out[d] = nullptr;
    if (!n_db) return CPM_OK;
    const bool dbg = getenv("CPM_DEBUG") != nullptr;
    auto t0 = std::chrono::steady_clock::now();
    auto lap = [&](const char *what) {
        if (!dbg) return;
        const auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "cpm: batch load %-24s %.3f ms\n", what,
                std::chrono::duration<double, std::milli>(now - t0).count());
        t0 = now;
    };
    CK(cudaSetDevice(ctx->device));
    // ---- host: compacted offsets and largest id of every database ----
    std::vector<std::vector<uint64_t>> off(n_db);
    std::vector<uint32_t> max_id(n_db, 0);
    std::vector<int> bad(n_db, 0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t d = 0; d < (int64_t)n_db; ++d) {
        if ((!offsets[d] && n_rows[d]) || (!ids[d] && nnz[d])) { bad[d] = 1; continue; }
        cpm_ctx tmp;  // errors are reported below
        if (compact_offsets(&tmp, offsets[d], n_rows[d], nnz[d], off[d]) != CPM_OK) { bad[d] = 2; continue; }
        uint32_t m = 0;
        for (uint64_t k = 0; k < nnz[d]; ++k) m = std::max(m, ids[d][k]);
        max_id[d] = m;
    }
    for (uint32_t d = 0; d < n_db; ++d) {
        if (bad[d]) return set_err(ctx, CPM_EINVAL, "database %u: invalid CSR arrays", d);
        if (max_id[d] >= (1u << 26)) {
            // Ids this large take the one-database path (sorted ranks).
            for (uint32_t e = 0; e < n_db; ++e) {
                const int r = cpm_db_from_ids(ctx, offsets[e], n_rows[e], ids[e], nnz[e], &out[e]);
                if (r != CPM_OK) {
                    for (uint32_t f = 0; f < e; ++f) { cpm_db_free(out[f]); out[f] = nullptr; }
                    return r;
                }
            }
            return CPM_OK;
        }
    }
    lap("offsets, max ids");
    std::vector<uint64_t> row_base(n_db + 1, 0), occ_base(n_db + 1, 0), pres_base(n_db + 1, 0);
    for (uint32_t d = 0; d < n_db; ++d) {
        row_base[d + 1] = row_base[d] + off[d].size() - 1;
        occ_base[d + 1] = occ_base[d] + nnz[d];
        pres_base[d + 1] = pres_base[d] + (uint64_t)max_id[d] / 32 + 1;
    }
    const uint64_t R = row_base[n_db], NNZ = occ_base[n_db], PW = pres_base[n_db];
    // Every database's rebased offsets and ids, back to back in host memory
    // the context keeps pinned (reused by later loads), filled in parallel and
    // sent with two copies.  Without pinned memory: ordinary vectors.
    const size_t off_bytes = (R + 1) * 8, ids_bytes = NNZ * 4;
    const size_t stage_bytes = ((off_bytes + 255) & ~(size_t)255) + ids_bytes;
    std::vector<uint64_t> v_off;
    std::vector<uint32_t> v_ids;
    uint64_t *h_off = nullptr;
    uint32_t *h_ids = nullptr;
    if (ctx->pinned_bytes < stage_bytes) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        if (cudaHostAlloc(&ctx->pinned, std::max<size_t>(stage_bytes, 16ull << 20), cudaHostAllocDefault) ==
            cudaSuccess)
            ctx->pinned_bytes = std::max<size_t>(stage_bytes, 16ull << 20);
        else
            cudaGetLastError(), ctx->pinned = nullptr;
    }
    if (ctx->pinned) {
        h_off = static_cast<uint64_t *>(ctx->pinned);
        h_ids = reinterpret_cast<uint32_t *>(static_cast<unsigned char *>(ctx->pinned) +
                                             ((off_bytes + 255) & ~(size_t)255));
    } else {
        v_off.resize(R + 1);
        v_ids.resize(NNZ);
        h_off = v_off.data();
        h_ids = v_ids.data();
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t d = 0; d < (int64_t)n_db; ++d) {
        for (uint64_t r = 0; r + 1 < off[d].size(); ++r) h_off[row_base[d] + r] = occ_base[d] + off[d][r];
        if (nnz[d]) memcpy(h_ids + occ_base[d], ids[d], nnz[d] * 4);
    }
    h_off[R] = NNZ;
    lap("concatenate");
    DevScope tmp(ctx);
    uint64_t *d_off = nullptr, *d_occ = nullptr, *d_pres_base = nullptr, *d_rows = nullptr, *d_items = nullptr;
    uint32_t *d_ids = nullptr, *d_present = nullptr, *d_lut = nullptr;
    CKR(tmp.alloc(&d_off, R + 1));
    CKR(tmp.alloc(&d_ids, NNZ));
    CKR(tmp.alloc(&d_occ, n_db));
    CKR(tmp.alloc(&d_pres_base, n_db));
    CKR(tmp.alloc(&d_present, PW));
    CK(cudaMemcpyAsync(d_off, h_off, (R + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    if (NNZ) CK(cudaMemcpyAsync(d_ids, h_ids, NNZ * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_occ, occ_base.data(), n_db * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_pres_base, pres_base.data(), n_db * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(d_present, 0, PW * 4, ctx->stream));
    if (NNZ) {
        const unsigned blocks = (unsigned)std::min<uint64_t>((NNZ + 255) / 256, (uint64_t)ctx->sms * 16);
        const uint32_t spw = PW <= CPM_MARK_SMEM_WORDS ? (uint32_t)PW : 0u;
        k_mark_ids_b<<<spw ? std::min(blocks, (unsigned)ctx->sms * 2) : blocks, 256, spw * 4, ctx->stream>>>(
            d_ids, NNZ, d_occ, d_pres_base, n_db, d_present, spw);
        CK(cudaGetLastError());
    }
    std::vector<uint32_t> present(PW);
    CK(cudaMemcpyAsync(present.data(), d_present, PW * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    lap("upload, presence");
    // ---- host: label order and id -> column table of every database ----
    std::vector<uint64_t> lut_base(n_db + 1, 0);
    for (uint32_t d = 0; d < n_db; ++d) lut_base[d + 1] = lut_base[d] + (uint64_t)max_id[d] + 1;
    std::vector<uint32_t> h_lut(lut_base[n_db], 0);
    std::vector<std::vector<uint32_t>> labels(n_db);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t d = 0; d < (int64_t)n_db; ++d) {
        std::vector<uint32_t> uniq;
        for (uint64_t w = pres_base[d]; w < pres_base[d + 1]; ++w)
            for (uint32_t m = present[w]; m; m &= m - 1)
                uniq.push_back((uint32_t)((w - pres_base[d]) * 32 + __builtin_ctz(m)));
        std::vector<uint64_t> keys(uniq.size());
        for (size_t i = 0; i < uniq.size(); ++i) keys[i] = decimal_key(uniq[i]);
        std::vector<uint32_t> order(uniq.size());
        std::iota(order.begin(), order.end(), 0u);
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
        labels[d].resize(uniq.size());
        for (size_t c = 0; c < order.size(); ++c) {
            labels[d][c] = uniq[order[c]];
            h_lut[lut_base[d] + uniq[order[c]]] = (uint32_t)c;
        }
    }
    lap("labels");
    // ---- device: tidsets of every database, packed in one pass ----
    std::vector<cpm_db *> dbs(n_db, nullptr);
    auto cleanup = [&]() {
        for (cpm_db *x : dbs)
            if (x) cpm_db_free(x);
    };
    std::vector<PackDesc> pd(n_db);
    std::vector<uint64_t> item_base(n_db + 1, 0);
    for (uint32_t d = 0; d < n_db; ++d) {
        cpm_db *db = new cpm_db();
        dbs[d] = db;
        db->ctx = ctx;
        db->n_tx = off[d].size() - 1;
        db->n_items = (uint32_t)labels[d].size();
        db->labels = std::move(labels[d]);
        const int r = db_alloc_bits(ctx, db);
        if (r != CPM_OK) {
            cleanup();
            return r;
        }
        pd[d] = PackDesc{reinterpret_cast<uint32_t *>(db->d_bits), db->d_support, nullptr, db->stride,
                         row_base[d], occ_base[d], pres_base[d], db->n_items, 0};
        item_base[d + 1] = item_base[d] + db->n_items;
    }
    lap("allocate tidsets");
    PackDesc *d_pd = nullptr;
    int r = tmp.alloc(&d_lut, lut_base[n_db]);
    if (r == CPM_OK) r = tmp.alloc(&d_pd, n_db);
    if (r == CPM_OK) r = tmp.alloc(&d_rows, n_db);
    if (r == CPM_OK) r = tmp.alloc(&d_items, n_db);
    if (r != CPM_OK) {
        cleanup();
        return r;
    }
    for (uint32_t d = 0; d < n_db; ++d) pd[d].lut = d_lut + lut_base[d];
    cudaMemcpyAsync(d_lut, h_lut.data(), lut_base[n_db] * 4, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(d_pd, pd.data(), n_db * sizeof(PackDesc), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(d_rows, row_base.data(), n_db * 8, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(d_items, item_base.data(), n_db * 8, cudaMemcpyHostToDevice, ctx->stream);
    if (R) k_pack_b<<<(unsigned)((R + 255) / 256), 256, 0, ctx->stream>>>(d_off, d_ids, R, d_pd, d_rows, n_db);
    if (item_base[n_db])
        k_item_support_b<<<(unsigned)((item_base[n_db] * 32 + 255) / 256), 256, 0, ctx->stream>>>(d_pd, d_items, n_db,
                                                                                                 item_base[n_db]);
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        cleanup();
        return set_err(ctx, CPM_ECUDA, "batched pack failed: %s", cudaGetErrorString(e));
    }
    for (uint32_t d = 0; d < n_db; ++d) out[d] = dbs[d];
    lap("pack");
    return CPM_OK;
}

extern "C" int cpm_db_info(const cpm_db *db, uint64_t *n_tx, uint32_t *n_items, uint64_t *words) {
    if (!db) return CPM_EINVAL;
    if (n_tx) *n_tx = db->n_tx;
    if (n_items) *n_items = db->n_items;
    if (words) *words = db->words;
    return CPM_OK;
}

extern "C" int cpm_db_labels(const cpm_db *db, uint32_t *ids_out) {
    if (!db || !ids_out) return CPM_EINVAL;
    if (db->labels.size() != db->n_items) return CPM_EINVAL;
    std::copy(db->labels.begin(), db->labels.end(), ids_out);
    return CPM_OK;
}

extern "C" void cpm_db_free(cpm_db *db) {
    if (!db) return;
    cpm_ctx *ctx = db->ctx;
    cudaSetDevice(ctx->device);
    dfree(ctx, db->d_bits);
    dfree(ctx, db->d_support);
    dfree(ctx, db->d_ts);
    cudaStreamSynchronize(ctx->stream);
    delete db;
}

// ---------------------------------------------------------------------------
// mining
// ---------------------------------------------------------------------------

static double elapsed_ms(cpm_ctx *ctx, int a, int b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[b]);
    return ms;
}

// Frequent singletons: ordered list of columns whose support passes.
static int mine_singletons(cpm_ctx *ctx, cpm_db *db, long long ms, DevScope &ds, uint32_t **d_freq,
                           uint32_t &F, uint64_t &launches) {
    uint32_t *d_count = nullptr;
    CKR(ds.alloc(d_freq, db->n_items));
    CKR(ds.alloc(&d_count, 1));
    CK(cudaMemsetAsync(d_count, 0, 4, ctx->stream));
    if (db->n_items) {
        k_compact_frequent<<<1, 1024, 0, ctx->stream>>>(db->d_support, db->n_items, ms, *d_freq, d_count);
        CK(cudaGetLastError());
        launches++;
    }
    CK(cudaMemcpyAsync(&F, d_count, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CPM_OK;
}

// Tensor-core Gram of the selected databases (C zeroed here) in one launch;
// synchronous (reads the error word).  d_desc / h describe every database.
static int gram_tc_run(cpm_ctx *ctx, DevScope &ds, const DbDesc *d_desc, const std::vector<DbDesc> &h,
                       const std::vector<uint32_t> &sel, cpm_stats &st) {
    // Upper-triangle tiles of each database: A block ti (128 rows) x B block
    // tj (256 columns) whenever some column of the block lies right of some row.
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> tiles(sel.size());
    uint64_t tile_stages = 0;
    for (size_t s = 0; s < sel.size(); ++s) {
        const DbDesc &D = h[sel[s]];
        CK(cudaMemsetAsync(D.C, 0, (size_t)D.F * D.F * 4, ctx->stream));
        const uint32_t nti = (D.F + tc::BM - 1) / tc::BM, ntj = (D.F + tc::BN - 1) / tc::BN;
        for (uint32_t ti = 0; ti < nti; ++ti)
            for (uint32_t tj = 0; tj < ntj; ++tj)
                if ((uint64_t)tj * tc::BN + tc::BN - 1 > (uint64_t)ti * tc::BM) tiles[s].push_back({ti, tj});
        tile_stages += tiles[s].size() * (D.stride / 2);
    }
    // K split: about four units per SM over the whole selection, and at
    // least 32 stages per unit so the epilogue (one atomic per output) stays
    // small next to the main loop.
    const uint64_t per = std::max<uint64_t>(32, (tile_stages + (uint64_t)ctx->sms * 4 - 1) / ((uint64_t)ctx->sms * 4));
    std::vector<GramUnit> units;
    for (size_t s = 0; s < sel.size(); ++s) {
        const DbDesc &D = h[sel[s]];
        const uint64_t kstages = D.stride / 2;
        for (auto &t : tiles[s])
            for (uint64_t k = 0; k < kstages; k += per)
                units.push_back({sel[s], t.first, t.second, 0, 2 * k, 2 * std::min(kstages, k + per)});
        // Work issued to the tensor cores: every tile is a full 128x256 block.
        st.pair_ops += 2ull * (uint64_t)tc::BM * tc::BN * (kstages * 128) * tiles[s].size();
    }
    if (units.empty()) return CPM_OK;
    GramUnit *d_units = nullptr;
    unsigned int *d_err = nullptr;
    CKR(ds.alloc(&d_units, units.size()));
    CKR(ds.alloc(&d_err, 1));
    CK(cudaMemcpyAsync(d_units, units.data(), units.size() * sizeof(GramUnit), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(d_err, 0, 4, ctx->stream));
    for (size_t u0 = 0; u0 < units.size(); u0 += 1u << 30) {
        const unsigned nb = (unsigned)std::min<size_t>(units.size() - u0, 1u << 30);
        k_gram_tc<<<nb, tc::THREADS, tc::SMEM_BYTES, ctx->stream>>>(d_desc, d_units + u0, d_err);
        CK(cudaGetLastError());
        st.kernel_launches += 1;
    }
    unsigned int herr = 0;
    CK(cudaMemcpyAsync(&herr, d_err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (herr) return set_err(ctx, CPM_ETIMEOUT, "tensor-core Gram pipeline wait ran out");
    return CPM_OK;
}

// Pair Gram C[F][F] (upper triangle) on the tensor cores or the CUDA cores.
static int pair_gram(cpm_ctx *ctx, cpm_db *db, const uint32_t *d_freq, uint32_t F, const cpm_opts &o,
                     DevScope &ds, uint32_t **d_C, cpm_stats &st) {
    CKR(ds.alloc(d_C, (size_t)F * F));
    const bool use_tc = o.pair_engine == 1 || (o.pair_engine == 0 && ctx->tc_ok && gram_tc_worthwhile(F, db->n_tx));
    CK(cudaEventRecord(ctx->ev[5], ctx->stream));
    if (use_tc) {
        if (!ctx->tc_ok) return set_err(ctx, CPM_EINVAL, "the tensor-core Gram needs an sm_100 device");
        std::vector<DbDesc> h(1);
        h[0].bits = db->d_bits;
        h[0].support = db->d_support;
        h[0].freq = const_cast<uint32_t *>(d_freq);
        h[0].C = *d_C;
        h[0].stride = db->stride;
        h[0].n_items = db->n_items;
        h[0].F = F;
        DbDesc *d_desc = nullptr;
        CKR(ds.alloc(&d_desc, 1));
        CK(cudaMemcpyAsync(d_desc, h.data(), sizeof(DbDesc), cudaMemcpyHostToDevice, ctx->stream));
        CKR(gram_tc_run(ctx, ds, d_desc, h, std::vector<uint32_t>{0u}, st));
        CK(cudaEventRecord(ctx->ev[6], ctx->stream));
        return CPM_OK;
    }
    CK(cudaMemsetAsync(*d_C, 0, (size_t)F * F * 4, ctx->stream));
    const uint32_t nt = (F + 63) / 64;
    const uint32_t tiles = nt * (nt + 1) / 2;
    // Split K so that the grid covers the GPU a few times over.
    uint64_t ksplit = std::max<uint64_t>(1, (uint64_t)ctx->sms * 4 / tiles);
    ksplit = std::min<uint64_t>(ksplit, std::max<uint64_t>(1, db->stride / 64));
    const uint64_t k_chunk = ((db->stride + ksplit - 1) / ksplit + 15) / 16 * 16;
    ksplit = (db->stride + k_chunk - 1) / k_chunk;
    dim3 grid(tiles, (unsigned)ksplit);
    k_gram_simt<<<grid, 256, 0, ctx->stream>>>(db->d_bits, db->stride, d_freq, F, nt, k_chunk, *d_C);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[6], ctx->stream));
    st.kernel_launches += 1;
    st.pair_ops += 2ull * db->n_tx * F * (uint64_t)F;
    return CPM_OK;
}

struct DeepBuffers {
    DFrame *frames = nullptr;
    uint32_t *mem_pat = nullptr, *mem_item = nullptr;
    const uint64_t **mem_bits = nullptr;
    unsigned long long *queue = nullptr;
    unsigned long long *lq = nullptr;  // projected units (k_local), queue_cap entries
    uint64_t *arena = nullptr;
    uint32_t *pat_parent = nullptr, *pat_item = nullptr, *pat_sup = nullptr, *pat_db = nullptr;
    unsigned long long *root_cost = nullptr;
    DeepState *st = nullptr;
    uint64_t frames_cap = 0, members_cap = 0, queue_cap = 0, arena_words = 0, pat_cap = 0;
    cpm_ctx *owner = nullptr;  // released on every exit path
    ~DeepBuffers() {
        if (owner) release(owner);
    }
    void release(cpm_ctx *ctx) {
        dfree(ctx, frames); dfree(ctx, mem_pat); dfree(ctx, mem_item); dfree(ctx, mem_bits);
        dfree(ctx, queue); dfree(ctx, lq); dfree(ctx, arena); dfree(ctx, pat_parent); dfree(ctx, pat_item);
        dfree(ctx, pat_sup); dfree(ctx, pat_db); dfree(ctx, root_cost); dfree(ctx, st);
    }
};

static int grow(cpm_ctx *ctx, DeepBuffers &b, uint64_t frames_cap, uint64_t members_cap, uint64_t queue_cap,
                uint64_t arena_words, uint64_t pat_cap, uint64_t n_roots, bool with_db) {
    b.release(ctx);
    b.frames_cap = frames_cap; b.members_cap = members_cap; b.queue_cap = queue_cap;
    b.arena_words = arena_words; b.pat_cap = pat_cap;
    CKR(dalloc(ctx, &b.frames, frames_cap));
    CKR(dalloc(ctx, &b.mem_pat, members_cap));
    CKR(dalloc(ctx, &b.mem_item, members_cap));
    CKR(dalloc(ctx, &b.mem_bits, members_cap));
    CKR(dalloc(ctx, &b.queue, queue_cap));
    CKR(dalloc(ctx, &b.lq, queue_cap));
    CKR(dalloc(ctx, &b.arena, arena_words));
    CKR(dalloc(ctx, &b.pat_parent, pat_cap));
    CKR(dalloc(ctx, &b.pat_item, pat_cap));
    CKR(dalloc(ctx, &b.pat_sup, pat_cap));
    if (with_db) CKR(dalloc(ctx, &b.pat_db, pat_cap));
    CKR(dalloc(ctx, &b.root_cost, std::max<uint64_t>(1, n_roots)));
    CKR(dalloc(ctx, &b.st, 1));
    return CPM_OK;
}


// Projection of small prefixes by k_deep and the projected levels (k_local):
// only where the prefix bitmap and its rank directory (2 bytes per 16-byte
// word) fit in shared memory.  deep_project >= 128 sets the largest
// projected prefix; 0 projects prefixes of up to LOCAL_MAX_BITS transactions
// when there are at least PROJECT_MIN_ROOTS_PER_SM root units per SM.  A
// search of fewer is short and bound by its chain of dependent units, which
// a warp per unit only lengthens (planted 100,000 x 1,000, ~1,000 root units:
// deep phase 0.22 ms without projection, 1.11 ms with it; 1M x 20k, 65,000
// root units: 718 -> 384 ms).
constexpr uint64_t PROJECT_MIN_ROOTS_PER_SM = 16;
static uint32_t deep_local_max(const cpm_ctx *ctx, const cpm_opts &o, bool smem_prefix, uint64_t max_stride,
                               uint64_t n_roots) {
    if (o.deep_project == 1 || !smem_prefix) return 0;
    if (max_stride * 8 + max_stride > DEEP_SMEM_PREFIX_MAX) return 0;
    if (o.deep_project >= 128) return std::min<uint32_t>((uint32_t)o.deep_project, LOCAL_MAX_BITS);
    return n_roots >= PROJECT_MIN_ROOTS_PER_SM * (uint64_t)ctx->sms ? LOCAL_MAX_BITS : 0;
}

// k_deep<true>'s dynamic shared memory: the prefix bitmap, then the rank directory.
static size_t deep_smem_bytes(uint64_t max_stride, uint32_t local_max) {
    return max_stride * 8 + (local_max ? max_stride : 0);
}

// Projection fields of a launch (local_max 0: off).
static void deep_set_local(DeepParams &P, const DeepBuffers &b, uint64_t max_stride, uint32_t local_max) {
    P.local_max = local_max;
    P.lq = local_max ? b.lq : nullptr;
    P.lq_cap = local_max ? b.queue_cap : 0;
    P.dir_off = (uint32_t)(max_stride * 8);
    // Row-wise units off unless the caller sets them (one database only).
    P.h_off = nullptr; P.h_rows = nullptr; P.h_fidx = nullptr; P.h_F = 0; P.h_cost = 0.f;
    P.h_scratch = nullptr; P.h_scratch_words = 0; P.h_table_off = 0;
}

// The projected units k_deep queued, after it (same stream).
static int launch_local(cpm_ctx *ctx, const DeepParams &P, cpm_stats &st) {
    if (!P.local_max) return CPM_OK;
    if (ctx->local_occ < 0) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->local_occ, k_local, (int)LOCAL_BLOCK, 0));
        ctx->local_occ = std::max(1, ctx->local_occ);
    }
    CK(cudaEventRecord(ctx->ev[7], ctx->stream));  // k_local's start (it ends at the caller's ev[3])
    k_local<<<(unsigned)(ctx->sms * ctx->local_occ), LOCAL_BLOCK, 0, ctx->stream>>>(P);
    CK(cudaGetLastError());
    st.kernel_launches++;
    return CPM_OK;
}

// Part of the arena kept free for frames that shallow expansion keeps.

// Memory-bounded deep phase.  Root units (in scheduler order: d_uid/d_key,
// largest first) are admitted into rounds while their cost keys fit a share
// of the arena; each round is one persistent launch with the arena reset to
// the persistent region.  A round that overflows is discarded (its counters
// rewound) and retried with half as many units; a single unit that still
// overflows runs shallow -- only its own intersections -- and its child
// frame, kept in the persistent region, contributes its positions as new
// root units, processed next (depth first, so the region stays small).
static int deep_rounds_run(cpm_ctx *ctx, DevScope &ds, DeepBuffers &b, const std::vector<DFrame> &top_frames,
                           const uint32_t *d_uid, const float *d_key, const float *d_unit_key, uint64_t n_units,
                           uint64_t P2_total,
                           uint64_t max_stride, unsigned grid, unsigned block, bool smem_prefix, uint64_t spin,
                           bool keys_in_words, uint32_t lists, uint32_t local_max, const std::vector<unsigned long long> *cont,
                           uint64_t arena_words, uint64_t pat_cap, DeepState &hs, cpm_stats &st);

static int deep_rounds(cpm_ctx *ctx, DevScope &ds, DeepBuffers &b, const std::vector<DFrame> &top_frames,
                       const uint32_t *d_uid, const float *d_key, const float *d_unit_key, uint64_t n_units,
                       uint64_t base_patterns,
                       uint64_t P2_total, uint64_t max_stride, unsigned grid, unsigned block, bool smem_prefix,
                       uint64_t spin,
                       uint64_t pat_need, bool with_db, uint64_t arena_limit_words, bool keys_in_words,
                       uint32_t lists, uint32_t local_max, const std::vector<unsigned long long> *cont, DeepState &hs, cpm_stats &st) {
    const bool dbg = getenv("CPM_DEBUG") != nullptr;
    if (cont) return deep_rounds_run(ctx, ds, b, top_frames, nullptr, nullptr, d_unit_key, 0, P2_total, max_stride,
                                     grid, block,
                                     smem_prefix, spin, keys_in_words, lists, local_max, cont, b.arena_words, b.pat_cap, hs, st);
    // Fixed tables large enough for any round; the arena takes the rest.
    const uint64_t frames_cap = 32ull << 20, members_cap = 256ull << 20, queue_cap = 64ull << 20;
    const uint64_t pat_cap = std::max<uint64_t>(pat_need, 96ull << 20);
    const uint64_t fixed = frames_cap * sizeof(DFrame) + members_cap * 16 + queue_cap * 8 + pat_cap * 16 + (1ull << 30);
    uint64_t arena_words = ctx->mem_free > fixed * 2 ? (uint64_t)(ctx->mem_free * 0.75 - fixed) / 8 : 0;
    if (arena_limit_words) arena_words = std::min(arena_words, arena_limit_words);
    if (arena_words < 64 * max_stride) return set_err(ctx, CPM_ENOMEM, "no device memory left for deep rounds");
    // Patterns, members and frames of the top level must survive the regrow.
    std::vector<uint32_t> par(base_patterns), item(base_patterns), sup(base_patterns), pdb, mp(P2_total), mi(P2_total);
    std::vector<const uint64_t *> mb(P2_total);
    CK(cudaMemcpyAsync(par.data(), b.pat_parent, base_patterns * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(item.data(), b.pat_item, base_patterns * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(sup.data(), b.pat_sup, base_patterns * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (with_db) {
        pdb.resize(base_patterns);
        CK(cudaMemcpyAsync(pdb.data(), b.pat_db, base_patterns * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaMemcpyAsync(mp.data(), b.mem_pat, P2_total * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(mi.data(), b.mem_item, P2_total * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(mb.data(), b.mem_bits, P2_total * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // The unit order (d_uid / d_key) lives in the caller's scratch, not in b.
    CKR(grow(ctx, b, frames_cap, members_cap, queue_cap, arena_words, pat_cap, 1, with_db));
    CK(cudaMemcpyAsync(b.pat_parent, par.data(), base_patterns * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b.pat_item, item.data(), base_patterns * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b.pat_sup, sup.data(), base_patterns * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (with_db) CK(cudaMemcpyAsync(b.pat_db, pdb.data(), base_patterns * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b.mem_pat, mp.data(), P2_total * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b.mem_item, mi.data(), P2_total * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b.mem_bits, mb.data(), P2_total * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(b.frames, top_frames.data(), top_frames.size() * sizeof(DFrame), cudaMemcpyHostToDevice,
                       ctx->stream));
    hs = DeepState{};
    hs.n_patterns = base_patterns;
    return deep_rounds_run(ctx, ds, b, top_frames, d_uid, d_key, d_unit_key, n_units, P2_total, max_stride, grid,
                           block,
                           smem_prefix, spin, keys_in_words, lists, local_max, nullptr, arena_words, pat_cap, hs, st);
}

// The rounds themselves.  Fresh start (cont null): every root unit d_uid /
// d_key, largest first, after the top level was rebuilt in b.  Continuation
// (cont): the root units a first launch deferred, in queue order, with the
// top level and the patterns found so far (hs.n_patterns) kept in b.
static int deep_rounds_run(cpm_ctx *ctx, DevScope &ds, DeepBuffers &b, const std::vector<DFrame> &top_frames,
                           const uint32_t *d_uid, const float *d_key, const float *d_unit_key, uint64_t n_units,
                           uint64_t P2_total,
                           uint64_t max_stride, unsigned grid, unsigned block, bool smem_prefix, uint64_t spin,
                           bool keys_in_words, uint32_t lists, uint32_t local_max, const std::vector<unsigned long long> *cont,
                           uint64_t arena_words, uint64_t pat_cap, DeepState &hs, cpm_stats &st) {
    const bool dbg = getenv("CPM_DEBUG") != nullptr;
    const uint64_t queue_cap = b.queue_cap;
    std::vector<uint32_t> uid(n_units);
    std::vector<float> key(n_units);
    if (n_units) {
        CK(cudaMemcpyAsync(uid.data(), d_uid, n_units * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(key.data(), d_key, n_units * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    // Root units as (frame, position, key), front = next.
    struct Root {
        uint32_t frame, p;
        double key;
    };
    std::deque<Root> roots;
    if (cont)
        for (unsigned long long it : *cont) roots.push_back({(uint32_t)(it >> 32), (uint32_t)it, 1.0});
    for (uint64_t i = 0; i < n_units; ++i) {
        uint32_t k = (uint32_t)(std::upper_bound(top_frames.begin(), top_frames.end(), uid[i],
                                                 [](uint32_t u, const DFrame &f) { return u < f.root; }) -
                                top_frames.begin()) - 1;
        // Learned keys already estimate words touched; plain keys are member
        // counts, scaled by the tidset length.
        const double words = keys_in_words ? (double)key[i] : (double)key[i] * top_frames[k].stride;
        roots.push_back({k, uid[i] - top_frames[k].root, std::max(1.0, words)});
    }
    uint64_t persist_frames = top_frames.size(), persist_members = P2_total, persist_arena = 0;
    uint64_t committed = hs.n_patterns;
    // Child frames kept by shallow expansions form a stack at the front of
    // the arena: (frame id, arena start, root units still queued).  A frame's
    // block is released once every root unit taken from it has run.
    struct Kept {
        uint32_t fid;
        uint64_t arena_start;
        uint64_t left;
    };
    std::vector<Kept> kept;
    uint64_t limit = ~0ull;  // units per round
    std::vector<unsigned long long> q;
    DeepParams P;
    P.frames = b.frames; P.frames_cap = b.frames_cap;
    P.mem_pat = b.mem_pat; P.mem_item = b.mem_item; P.mem_bits = b.mem_bits; P.members_cap = b.members_cap;
    P.queue = b.queue; P.queue_cap = b.queue_cap;
    P.arena = b.arena; P.arena_words = b.arena_words;
    P.pat_parent = b.pat_parent; P.pat_item = b.pat_item; P.pat_sup = b.pat_sup; P.pat_db = b.pat_db;
    P.pat_cap = b.pat_cap;
    P.root_cost = nullptr; P.st = b.st; P.max_stride = max_stride; P.spin_limit = spin; P.cta_time = nullptr;
    P.unit_log = nullptr; P.unit_log_cap = 0;
    P.lists = lists;
    deep_set_local(P, b, max_stride, local_max);
    if (local_max) CK(cudaMemsetAsync(b.lq, 0xff, b.queue_cap * 8, ctx->stream));
    P.root_frames = 0; P.defer_words = 0; P.defer_members = 0; P.defer_frames = 0; P.defer_queue = 0;
    P.root_key = nullptr; P.top_frames = 0; P.keys_in_words = 0; P.admit_words = 0;
    P.deferred = nullptr; P.deferred_cap = 0;
    const size_t smem_bytes = deep_smem_bytes(max_stride, local_max);
    uint64_t rounds = 0, failed = 0, shallow = 0;
    float deep_ms = 0.f;
    auto launch = [&](size_t n_take, uint32_t shallow_mode) -> int {
        q.clear();
        for (size_t i = 0; i < n_take; ++i) q.push_back(((unsigned long long)roots[i].frame << 32) | roots[i].p);
        CK(cudaMemsetAsync(b.queue, 0xff, std::min<uint64_t>(queue_cap, q.size() * 64 + (1u << 20)) * 8, ctx->stream));
        CK(cudaMemcpyAsync(b.queue, q.data(), q.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
        DeepState s0{};
        s0.q_tail = q.size();
        s0.pending = q.size();
        s0.n_patterns = committed;
        s0.n_frames = persist_frames;
        s0.n_members = persist_members;
        s0.arena_next = persist_arena;
        CK(cudaMemcpyAsync(b.st, &s0, sizeof s0, cudaMemcpyHostToDevice, ctx->stream));
        P.shallow = shallow_mode;
        P.balance = ctx->deep_balance;
        // Next ticket taken early when units are queued: measured 1M x 20k
        // 768 -> 756 ms, dense 65,536 x 128 0.887 -> 0.844 ms, planted equal.
        P.prefetch = 1;
        // Queue entries beyond the memset stay stale: bound the round's queue.
        P.queue_cap = std::min<uint64_t>(queue_cap, q.size() * 64 + (1u << 20));
        CK(cudaEventRecord(ctx->ev[2], ctx->stream));
        if (smem_prefix) k_deep<true><<<grid, block, smem_bytes, ctx->stream>>>(P);
        else k_deep<false><<<grid, block, 0, ctx->stream>>>(P);
        CK(cudaGetLastError());
        CKR(launch_local(ctx, P, st));
        CK(cudaEventRecord(ctx->ev[3], ctx->stream));
        CK(cudaMemcpyAsync(&hs, b.st, sizeof hs, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        // The projected queue is empty again for the next round.
        if (local_max && hs.lq_tail)
            CK(cudaMemsetAsync(b.lq, 0xff, std::min<uint64_t>(hs.lq_tail, b.queue_cap) * 8, ctx->stream));
        const float round_ms = (float)elapsed_ms(ctx, 2, 3);
        deep_ms += round_ms;
        if (P.local_max) st.ms_local += elapsed_ms(ctx, 7, 3);
        if (dbg)
            fprintf(stderr, "cpm: round %llu: %zu units, %.3f ms, %.3g bytes, %.0f GB/s, deferred %llu, error 0x%x, "
                    "admitted %llu of %llu, arena %llu (hand back at %llu), members %llu (%llu), frames %llu (%llu), "
                    "queue %llu (%llu)\n",
                    (unsigned long long)rounds, n_take, round_ms, (double)hs.bytes_alg,
                    round_ms > 0 ? hs.bytes_alg / (round_ms * 1e6) : 0.0, (unsigned long long)hs.n_deferred, hs.error,
                    (unsigned long long)hs.admitted, (unsigned long long)P.admit_words,
                    (unsigned long long)hs.arena_next, (unsigned long long)P.defer_words,
                    (unsigned long long)hs.n_members, (unsigned long long)P.defer_members,
                    (unsigned long long)hs.n_frames, (unsigned long long)P.defer_frames,
                    (unsigned long long)hs.q_tail, (unsigned long long)P.defer_queue);
        st.kernel_launches++;
        if (!hs.error) {  // a discarded round's work is not counted (its time is)
            st.intersections += hs.intersections;
            st.bytes_alg += hs.bytes_alg;
            st.work_items += hs.work_items;
            st.projected_units += hs.local_units;
        }
        ++rounds;
        return CPM_OK;
    };
    // Each round queues the next root units (all of them unless a round
    // overflowed) and lets the kernel defer root units once the round has
    // filled `frac` of the free arena; deferred units return to the front.
    // A round that still overflows is discarded and retried with half the
    // units and half the fill level.
    double frac = 0.5;
    double words_per_key = 0.0;  // arena words per admitted key unit (0: not known yet)
    uint64_t deferred_total = 0;
    unsigned long long *d_deferred = nullptr;
    uint64_t deferred_cap = 0;
    std::vector<unsigned long long> deferred_h;
    while (!roots.empty()) {
        const size_t take = (size_t)std::min<uint64_t>(roots.size(), limit);
        if (take > deferred_cap) {
            deferred_cap = std::max<uint64_t>(take, deferred_cap * 2);
            CKR(ds.alloc(&d_deferred, deferred_cap));
        }
        P.root_frames = (uint32_t)persist_frames;
        P.root_key = d_unit_key;
        P.top_frames = (uint32_t)top_frames.size();
        P.keys_in_words = keys_in_words ? 1u : 0u;
        // Admission budget in key units: 80% of the free arena over the
        // arena words a key unit has cost so far (none before a round has run).
        const uint64_t round_start_arena = persist_arena;
        P.admit_words = words_per_key > 0
                            ? (uint64_t)(0.8 * (double)(arena_words - persist_arena) / words_per_key)
                            : 0ull;
        P.defer_words = persist_arena + std::max<uint64_t>(1, (uint64_t)(frac * (double)(arena_words - persist_arena)));
        P.defer_members = persist_members + (uint64_t)(frac * (double)(b.members_cap - persist_members));
        P.defer_frames = persist_frames + (uint64_t)(frac * (double)(b.frames_cap - persist_frames));
        P.defer_queue = take + (uint64_t)(frac * (double)(std::min<uint64_t>(queue_cap, take * 64 + (1u << 20)) - take));
        P.deferred = d_deferred;
        P.deferred_cap = deferred_cap;
        CKR(launch(take, 0));
        if (!hs.error) {
            committed = hs.n_patterns;
            const uint64_t n_def = hs.n_deferred;
            if (n_def >= take) return set_err(ctx, CPM_EINTERNAL, "a deep round deferred every root unit");
            deferred_h.resize(n_def);
            if (n_def) {
                CK(cudaMemcpyAsync(deferred_h.data(), d_deferred, n_def * 8, cudaMemcpyDeviceToHost, ctx->stream));
                CK(cudaStreamSynchronize(ctx->stream));
            }
            std::unordered_set<unsigned long long> def(deferred_h.begin(), deferred_h.end());
            std::vector<Root> back;
            for (size_t i = 0; i < take; ++i) {
                if (def.count(((unsigned long long)roots[i].frame << 32) | roots[i].p)) {
                    back.push_back(roots[i]);
                    continue;
                }
                for (Kept &k : kept)
                    if (k.fid == roots[i].frame) --k.left;
            }
            roots.erase(roots.begin(), roots.begin() + take);
            roots.insert(roots.begin(), back.begin(), back.end());
            while (!kept.empty() && kept.back().left == 0) {
                persist_arena = kept.back().arena_start;
                kept.pop_back();
            }
            deferred_total += n_def;
            if (limit != ~0ull) limit = limit >= (1ull << 40) ? ~0ull : limit * 2;  // saturating
            frac = std::min(0.5, frac * 1.25);
            // Arena words per admitted key unit: follow a round that used
            // more at once, decay slowly after rounds that used less.
            if (hs.admitted)
                words_per_key = std::max(0.7 * words_per_key,
                                         (double)(hs.arena_next - round_start_arena) / (double)hs.admitted);
            continue;
        }
        if (hs.error & DEEP_ERR_SPIN) return set_err(ctx, CPM_ETIMEOUT, "deep-level kernel wait ran out of spins");
        if (hs.error & DEEP_ERR_INTERNAL)
            return set_err(ctx, CPM_EINTERNAL, "deep-level kernel: a child list disagrees with its support");
        if (hs.error & DEEP_ERR_PATTERNS) {
            // Grow the pattern records (keeping the committed ones) and rerun the round.
            const uint64_t cap = std::max<uint64_t>(b.pat_cap * 2, committed + (hs.n_patterns - committed) * 2);
            uint32_t *np_[4] = {nullptr, nullptr, nullptr, nullptr};
            uint32_t **old_[4] = {&b.pat_parent, &b.pat_item, &b.pat_sup, &b.pat_db};
            for (int a = 0; a < 4; ++a) {
                if (!*old_[a]) continue;
                CKR(dalloc(ctx, &np_[a], cap));
                if (committed)
                    CK(cudaMemcpyAsync(np_[a], *old_[a], committed * 4, cudaMemcpyDeviceToDevice, ctx->stream));
                dfree(ctx, *old_[a]);
                *old_[a] = np_[a];
            }
            b.pat_cap = cap;
            P.pat_parent = b.pat_parent; P.pat_item = b.pat_item; P.pat_sup = b.pat_sup; P.pat_db = b.pat_db;
            P.pat_cap = b.pat_cap;
            ++failed;
            continue;
        }
        ++failed;
        if (take > 1) {
            limit = std::max<size_t>(1, take / 2);
            frac = std::max(0.05, frac / 2);
            words_per_key *= 2;  // the keys under-predicted this round's arena
            continue;
        }
        // One root unit whose subtree does not fit: expand it by one level.
        P.root_frames = 0;
        P.defer_words = 0;
        CKR(launch(1, 1));
        if (hs.error)
            return set_err(ctx, CPM_EOVERFLOW,
                           "the child tidsets of one class position exceed the device arena (%llu of %llu words "
                           "free, error 0x%x)", (unsigned long long)(arena_words - persist_arena),
                           (unsigned long long)arena_words, hs.error);
        ++shallow;
        committed = hs.n_patterns;
        const Root parent = roots.front();
        roots.pop_front();
        for (Kept &k : kept)
            if (k.fid == parent.frame) --k.left;
        if (hs.n_frames > persist_frames) {
            DFrame c;
            CK(cudaMemcpy(&c, b.frames + persist_frames, sizeof c, cudaMemcpyDeviceToHost));
            const uint64_t cid = persist_frames;
            kept.push_back({(uint32_t)cid, persist_arena, (uint64_t)c.m - 1});
            persist_frames = hs.n_frames;
            persist_members = hs.n_members;
            persist_arena = hs.arena_next;
            for (uint32_t p = c.m - 1; p-- > 0;)
                roots.push_front({(uint32_t)cid, p, parent.key * (c.m - 1 - p) / std::max(1u, c.m)});
        }
        while (!kept.empty() && kept.back().left == 0) {
            persist_arena = kept.back().arena_start;
            kept.pop_back();
        }
        limit = ~0ull;
    }
    if (dbg)
        fprintf(stderr, "cpm: deep rounds %llu (failed %llu, shallow %llu, deferred units %llu), arena %.1f GB, "
                "%.3f ms\n", (unsigned long long)rounds, (unsigned long long)failed, (unsigned long long)shallow,
                (unsigned long long)deferred_total, arena_words * 8 / 1e9, deep_ms);
    st.retries += failed;
    st.deep_rounds = rounds;
    // The caller reads patterns up to hs.n_patterns and the deep time from
    // these counters.
    hs.n_patterns = committed;
    hs.work_items = st.work_items;
    hs.local_units = st.projected_units;
    hs.intersections = st.intersections;
    hs.bytes_alg = st.bytes_alg;
    hs.n_frames = persist_frames;
    ctx->last_deep_ms = deep_ms;
    return CPM_OK;
}

// Eclat over a batch of databases (a single database is a batch of one).
// Host syncs: frequent counts; pair counts; end of the deep phase.
static int scan_u32(cpm_ctx *ctx, DevScope &ds, const uint32_t *in, uint64_t *out, uint64_t n, uint64_t *total,
                    uint64_t *d_tot = nullptr);

static int mine_eclat_batch(cpm_ctx *ctx, cpm_db **dbs, uint32_t n_db, const long long *ms, const cpm_opts &o,
                            cpm_result **res) {
    cpm_stats st{};
    const bool dbg = getenv("CPM_DEBUG") != nullptr;
    auto t_start = std::chrono::steady_clock::now();
    auto lap = [&](const char *what) {
        if (!dbg) return;
        const auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "cpm: host %-24s %.3f ms\n", what,
                std::chrono::duration<double, std::milli>(now - t_start).count());
        t_start = now;
    };
    DevScope ds(ctx);
    if (o.deep_balance < 0 || o.deep_balance > 2)
        return set_err(ctx, CPM_EINVAL, "deep_balance must be 0, 1 or 2 (got %d)", o.deep_balance);
    // Measured (deep phase, 1M x 20k / dense 65,536 x 128 / planted 100k):
    // a warp per sibling 782 / 0.895 / 0.238 ms, split by size 870 / 0.989 /
    // 0.269 ms -- the split's scan and barriers cost more than the balance it
    // buys -- so the automatic choice is a warp per sibling.
    ctx->deep_balance = o.deep_balance == 2 ? 1u : 0u;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    // ---- singletons ----
    std::vector<DbDesc> h(n_db);
    uint64_t items_total = 0, max_stride = 2;
    for (uint32_t d = 0; d < n_db; ++d) items_total += dbs[d]->n_items;
    uint32_t *freq_all = nullptr, *d_F = nullptr;
    DbDesc *d_desc = nullptr;
    CKR(ds.alloc(&freq_all, items_total));
    CKR(ds.alloc(&d_F, n_db));
    CKR(ds.alloc(&d_desc, n_db));
    std::vector<uint64_t> item_off(n_db + 1, 0);
    for (uint32_t d = 0; d < n_db; ++d) {
        cpm_db *db = dbs[d];
        h[d] = DbDesc{};
        h[d].bits = db->d_bits;
        h[d].support = db->d_support;
        h[d].freq = freq_all + item_off[d];
        h[d].stride = db->stride;
        h[d].n_items = db->n_items;
        h[d].minsup = ms[d];
        item_off[d + 1] = item_off[d] + db->n_items;
        max_stride = std::max<uint64_t>(max_stride, db->stride);
    }
    // Transaction-id lists need the prefix bitmap in shared memory (k_deep.cuh);
    // decided once the frequent items are known (below).
    bool use_lists = false;
    CK(cudaMemcpyAsync(d_desc, h.data(), n_db * sizeof(DbDesc), cudaMemcpyHostToDevice, ctx->stream));
    k_compact_frequent_b<<<n_db, 1024, 0, ctx->stream>>>(d_desc, d_F);
    CK(cudaGetLastError());
    st.kernel_launches++;
    std::vector<uint32_t> F(n_db);
    CK(cudaMemcpyAsync(F.data(), d_F, n_db * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    lap("singletons");
    // Lists halve the bytes of sparse tidsets but cost more instructions per
    // byte: they pay where the deep phase streams from HBM, i.e. where one
    // database's frequent tidsets exceed half the L2 (126 MB on B200).
    {
        uint64_t biggest = 0;
        for (uint32_t d = 0; d < n_db; ++d) biggest = std::max<uint64_t>(biggest, (uint64_t)F[d] * dbs[d]->stride * 8);
        use_lists = o.tidsets != 1 && max_stride * 8 <= DEEP_SMEM_PREFIX_MAX &&
                    (o.tidsets == 2 || biggest > (uint64_t)ctx->l2_bytes / 2);
    }
    // A tidset becomes a list when its list takes at most 1/list_div of its
    // bitset (set by the options or the autotuner; 1 by default: measured on
    // the 1M x 20k workload, deep phase 740 / 752 / 851 ms for divisors
    // 1 / 2 / 4).
    uint32_t list_div = o.list_div > 0 ? (uint32_t)o.list_div : 1u;
    if (o.tidsets == 0 && !o.list_div && o.autotune) {
        const auto it = ctx->tune_lists.find(63 - __builtin_clzll(std::max<uint64_t>(1, max_stride)));
        if (it != ctx->tune_lists.end()) {
            use_lists = it->second > 0 && max_stride * 8 <= DEEP_SMEM_PREFIX_MAX;
            if (it->second > 0) list_div = (uint32_t)it->second;
        }
    }
    // ---- pair Grams ----
    uint64_t rows = 0, c_total = 0;
    std::vector<uint64_t> c_off(n_db, 0);
    for (uint32_t d = 0; d < n_db; ++d) {
        h[d].F = F[d];
        h[d].row_base = rows;
        rows += F[d];
        c_off[d] = c_total;
        c_total += (uint64_t)F[d] * F[d];
        st.n_frequent_items += F[d];
    }
    uint32_t *C_all = nullptr, *cnt_all = nullptr;
    uint64_t *off_all = nullptr;
    CKR(ds.alloc(&C_all, c_total));
    CKR(ds.alloc(&cnt_all, rows));
    CKR(ds.alloc(&off_all, rows + 1));
    if (c_total) CK(cudaMemsetAsync(C_all, 0, c_total * 4, ctx->stream));
    for (uint32_t d = 0; d < n_db; ++d) h[d].C = C_all + c_off[d];
    CK(cudaMemcpyAsync(d_desc, h.data(), n_db * sizeof(DbDesc), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->ev[5], ctx->stream));
    std::vector<BTile> tiles;
    std::vector<uint32_t> tc_dbs;
    for (uint32_t d = 0; d < n_db; ++d) {
        if (F[d] < 2) continue;
        const bool tc = o.pair_engine == 1 ||
                        (o.pair_engine == 0 && ctx->tc_ok && gram_tc_worthwhile(F[d], dbs[d]->n_tx));
        if (tc) {
            if (!ctx->tc_ok) return set_err(ctx, CPM_EINVAL, "the tensor-core Gram needs an sm_100 device");
            tc_dbs.push_back(d);
            continue;
        }
        const uint32_t nt = (F[d] + 63) / 64;
        const uint64_t n_tri = (uint64_t)nt * (nt + 1) / 2;
        // Split K so the batch covers the GPU a few times over.
        const uint64_t words = h[d].stride;
        uint64_t ksplit = std::max<uint64_t>(1, (uint64_t)ctx->sms * 4 / std::max<uint64_t>(1, n_tri * n_db));
        ksplit = std::min<uint64_t>(ksplit, std::max<uint64_t>(1, words / 64));
        const uint64_t chunk = ((words + ksplit - 1) / ksplit + 15) / 16 * 16;
        for (uint32_t ti = 0; ti < nt; ++ti)
            for (uint32_t tj = ti; tj < nt; ++tj)
                for (uint64_t k = 0; k < words; k += chunk) tiles.push_back({d, ti, tj, 0, k, std::min(words, k + chunk)});
        st.pair_ops += 2ull * dbs[d]->n_tx * F[d] * (uint64_t)F[d];
    }
    CKR(gram_tc_run(ctx, ds, d_desc, h, tc_dbs, st));
    if (!tiles.empty()) {
        BTile *d_tiles = nullptr;
        CKR(ds.alloc(&d_tiles, tiles.size()));
        CK(cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(BTile), cudaMemcpyHostToDevice, ctx->stream));
        for (size_t t0 = 0; t0 < tiles.size(); t0 += 1u << 30) {
            const unsigned nb = (unsigned)std::min<size_t>(tiles.size() - t0, 1u << 30);
            k_gram_simt_b<<<nb, 256, 0, ctx->stream>>>(d_desc, d_tiles + t0);
            CK(cudaGetLastError());
            st.kernel_launches++;
        }
    }
    CK(cudaEventRecord(ctx->ev[6], ctx->stream));
    std::vector<uint32_t> cnt(rows), hfreq(items_total);
    std::vector<uint64_t> list_words_h;
    uint64_t *d_list_words = nullptr;
    if (rows) {
        k_pair_count_b<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, ctx->stream>>>(d_desc, n_db, rows, cnt_all);
        CK(cudaGetLastError());
        st.kernel_launches++;
        CK(cudaMemcpyAsync(cnt.data(), cnt_all, rows * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(hfreq.data(), freq_all, items_total * 4, cudaMemcpyDeviceToHost, ctx->stream));
        if (use_lists) {
            CKR(ds.alloc(&d_list_words, rows));
            k_list_plan<<<(unsigned)((rows + 255) / 256), 256, 0, ctx->stream>>>(d_desc, n_db, rows, list_div,
                                                                               d_list_words);
            CK(cudaGetLastError());
            st.kernel_launches++;
            list_words_h.resize(rows);
            CK(cudaMemcpyAsync(list_words_h.data(), d_list_words, rows * 8, cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    CK(cudaStreamSynchronize(ctx->stream));
    lap("pairs");
    // Transaction-id lists of the sparse frequent items (members of the top-level classes).
    unsigned long long *d_row_list = nullptr;
    if (!list_words_h.empty()) {
        std::vector<uint64_t> loff(rows);
        uint64_t lw_total = 0;
        for (uint64_t r = 0; r < rows; ++r) {
            loff[r] = lw_total;
            lw_total += list_words_h[r];
        }
        if (lw_total) {
            uint64_t *d_lbuf = nullptr, *d_loff = nullptr;
            CKR(ds.alloc(&d_lbuf, lw_total));
            CKR(ds.alloc(&d_loff, rows));
            CKR(ds.alloc(&d_row_list, rows));
            CK(cudaMemcpyAsync(d_loff, loff.data(), rows * 8, cudaMemcpyHostToDevice, ctx->stream));
            k_item_lists<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, ctx->stream>>>(d_desc, n_db, rows, d_list_words,
                                                                                     d_loff, d_lbuf, d_row_list);
            CK(cudaGetLastError());
            st.kernel_launches++;
        }
    }
    // Pair numbering and pattern ids: per database, singletons then pairs.
    std::vector<uint64_t> off(rows + 1, 0);
    for (uint64_t r = 0; r < rows; ++r) off[r + 1] = off[r] + cnt[r];
    const uint64_t P2_total = off[rows];
    st.n_frequent_pairs = P2_total;
    uint64_t pat_next = 0;
    for (uint32_t d = 0; d < n_db; ++d) {
        h[d].pat_base = pat_next;
        h[d].pair_base = off[h[d].row_base];
        const uint64_t p2 = off[h[d].row_base + F[d]] - off[h[d].row_base];
        pat_next += F[d] + p2;
    }
    const uint64_t base_patterns = pat_next;
    CK(cudaMemcpyAsync(d_desc, h.data(), n_db * sizeof(DbDesc), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(off_all, off.data(), (rows + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    // ---- top-level classes (cuEclat.py:195-200) ----
    std::vector<DFrame> frames;
    std::vector<FrameAux> aux;
    for (uint32_t d = 0; d < n_db; ++d)
        for (uint32_t i = 0; i < F[d]; ++i) {
            const uint64_t r = h[d].row_base + i;
            if (cnt[r] < 2) continue;
            DFrame f;
            f.mask = h[d].bits + (uint64_t)hfreq[item_off[d] + i] * h[d].stride;
            f.mem_off = off[r];
            f.m = cnt[r];
            f.root = 0;
            f.stride = (uint32_t)h[d].stride;
            f.db = d;
            f.minsup = ms[d];
            frames.push_back(f);
            aux.push_back({(uint32_t)(h[d].pat_base + i), (float)dbs[d]->n_tx, (float)ms[d], 0.f});
        }
    // Root units: position p of top-level frame k has id frames[k].root + p;
    // they are costed, ordered and queued on the device (k_units.cuh).
    uint64_t n_units = 0;
    for (DFrame &f : frames) {
        f.root = (uint32_t)n_units;
        n_units += f.m - 1;
    }
    const bool learned = o.scheduler == CPM_SCHED_LEARNED && !ctx->model.empty();
    lap("frames and units");
    // ---- deep phase, grown and rerun on overflow ----
    cpm_db *db0 = dbs[0];
    DeepBuffers b;
    b.owner = ctx;
    const bool with_db = n_db > 1;
    const std::array<uint64_t, 4> plan_key{db0->n_tx, db0->n_items, P2_total, (uint64_t)ms[0]};
    if (n_db == 1 && !db0->hint_members) {
        const auto it = ctx->plan_hints.find(plan_key);
        if (it != ctx->plan_hints.end()) {
            db0->hint_frames = it->second[0];
            db0->hint_members = it->second[1];
            db0->hint_queue = it->second[2];
            db0->hint_patterns = it->second[3];
            db0->hint_arena = it->second[4];
        }
    }
    uint64_t frames_cap = std::max<uint64_t>({1024, frames.size() * 8 + P2_total * 2,
                                              n_db == 1 ? db0->hint_frames : 0});
    // Member entries are reserved for every sibling of every unit (~ the
    // intersections), several times the pair count on deep lattices.
    // Every unit reserves an entry per sibling: the third level alone takes
    // sum m(m-1)/2 over the top-level classes; deeper levels add to it.
    uint64_t level3 = 0;
    for (const DFrame &f : frames) level3 += (uint64_t)f.m * (f.m - 1) / 2;
    uint64_t members_cap = std::max<uint64_t>({4096, P2_total * 64, level3 * 4, n_db == 1 ? db0->hint_members : 0});
    uint64_t queue_cap = std::max<uint64_t>({4096, n_units * 8 + P2_total * 4, level3,
                                             n_db == 1 ? db0->hint_queue : 0});
    frames_cap = std::max<uint64_t>(frames_cap, level3 / 8);
    uint64_t pat_cap = std::max<uint64_t>({4096, base_patterns * 16, n_db == 1 ? db0->hint_patterns : 0});
    const uint64_t arena_budget = o.arena_bytes ? o.arena_bytes / 8 : (uint64_t)(ctx->mem_free * 0.6) / 8;
    // First arena: what the database needed before, else a guess capped at
    // 16 GB (a launch that fills it hands the rest to rounds).
    uint64_t arena_words = o.arena_bytes ? o.arena_bytes / 8
                                         : std::min<uint64_t>(arena_budget, std::max<uint64_t>(
                                               {(uint64_t)4096 * max_stride,
                                                std::min<uint64_t>(P2_total * 8 * max_stride, 2ull << 30),
                                                n_db == 1 ? db0->hint_arena : 0}));
    const uint64_t spin = o.spin_limit ? o.spin_limit : (1ull << 26);
    const size_t prefix_bytes = max_stride * 8;
    const bool smem_prefix = prefix_bytes <= DEEP_SMEM_PREFIX_MAX;
    const uint32_t local_max = deep_local_max(ctx, o, smem_prefix, max_stride, n_units);
    // Row-wise units (k_rows.cuh): one database, projection on, frequent
    // indices below 2^16, and their F-entry table after the rank directory.
    const uint32_t F0 = n_db == 1 ? F[0] : 0u;
    const size_t h_table_bytes = ((size_t)F0 * 2 + 15) / 16 * 16;
    const bool h_on = n_db == 1 && local_max && o.deep_rows != 1 && F0 >= 2 && F0 < H_NONE &&
                      deep_smem_bytes(max_stride, local_max) + h_table_bytes <= DEEP_SMEM_PREFIX_MAX;
    const size_t smem_bytes = deep_smem_bytes(max_stride, local_max) + (h_on ? h_table_bytes : 0);
    // Long tidsets leave room for fewer CTAs per SM: give each 16 or 32 warps
    // so that enough loads stay in flight; short ones run up to four 8-warp
    // CTAs.  Measured (deep phase): 1,564-word tidsets (planted-100k) 0.25 ms
    // with 16-warp CTAs against 0.32 ms with 8-warp ones; 1,024-word tidsets
    // (dense 65,536 x 128) 1.10 ms with 8-warp CTAs against 1.85 ms.
    unsigned block = max_stride >= 8192 ? 1024 : max_stride >= 1536 ? 512 : 256;
    int want_ctas = 4;
    if (o.autotune) {
        const auto it = ctx->tune.find(63 - __builtin_clzll(std::max<uint64_t>(1, max_stride)));
        if (it != ctx->tune.end()) {
            block = (unsigned)it->second.first;
            want_ctas = it->second.second;
        }
    }
    if (o.deep_block) {
        if (o.deep_block != 128 && o.deep_block != 256 && o.deep_block != 512 && o.deep_block != 1024)
            return set_err(ctx, CPM_EINVAL, "deep_block must be 128, 256, 512 or 1024 (got %d)", o.deep_block);
        block = (unsigned)o.deep_block;
    }
    if (o.deep_rows < 0 || o.deep_rows > 1)
        return set_err(ctx, CPM_EINVAL, "deep_rows must be 0 or 1 (got %d)", o.deep_rows);
    if (o.deep_project < 0 || (o.deep_project > 1 && o.deep_project < 128))
        return set_err(ctx, CPM_EINVAL, "deep_project must be 0, 1 or 128-65408 (got %d)", o.deep_project);
    if (o.deep_ctas_per_sm) {
        if (o.deep_ctas_per_sm < 1 || o.deep_ctas_per_sm > 4)
            return set_err(ctx, CPM_EINVAL, "deep_ctas_per_sm must be 1-4 (got %d)", o.deep_ctas_per_sm);
        want_ctas = o.deep_ctas_per_sm;
    }
    if (smem_prefix && (ctx->deep_occ_smem < 0 || ctx->deep_occ_bytes != smem_bytes || ctx->deep_occ_block != block)) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->deep_occ_smem, k_deep<true>, block, smem_bytes));
        ctx->deep_occ_bytes = smem_bytes;
        ctx->deep_occ_block = block;
    } else if (!smem_prefix && (ctx->deep_occ_global < 0 || ctx->deep_occ_block != block)) {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->deep_occ_global, k_deep<false>, block, 0));
        ctx->deep_occ_block = block;
    }
    const int cta_per_sm = std::min(want_ctas, std::max(1, smem_prefix ? ctx->deep_occ_smem : ctx->deep_occ_global));
    const unsigned grid = (unsigned)(ctx->sms * cta_per_sm);
    ctx->last_deep_block = (int)block;
    ctx->last_deep_ctas = cta_per_sm;
    // Rows of the frequent indices and the row-wise units' other inputs.
    uint64_t *d_hoff = nullptr;
    uint16_t *d_hrows = nullptr, *d_hfidx = nullptr;
    uint32_t *d_hscr = nullptr;
    float h_cost = 0.f;
    if (h_on) {
        const cpm_db *d0 = dbs[0];
        uint32_t *d_hlen = nullptr;
        CKR(ds.alloc(&d_hlen, d0->n_tx + 1));
        CKR(ds.alloc(&d_hoff, d0->n_tx + 1));
        CK(cudaMemsetAsync(d_hlen + d0->n_tx, 0, 4, ctx->stream));
        const unsigned nb = (unsigned)((d0->n_tx + 255) / 256);
        if (d0->n_tx) {
            k_hrows<false><<<nb, 256, 0, ctx->stream>>>(d0->d_bits, d0->stride, freq_all, F0, d0->n_tx, d_hlen,
                                                        nullptr, nullptr);
            CK(cudaGetLastError());
        }
        uint64_t nnz_f = 0;
        CKR(scan_u32(ctx, ds, d_hlen, d_hoff, d0->n_tx + 1, &nnz_f));
        CKR(ds.alloc(&d_hrows, std::max<uint64_t>(1, nnz_f)));
        if (d0->n_tx) {
            k_hrows<true><<<nb, 256, 0, ctx->stream>>>(d0->d_bits, d0->stride, freq_all, F0, d0->n_tx, nullptr,
                                                       d_hoff, d_hrows);
            CK(cudaGetLastError());
        }
        CKR(ds.alloc(&d_hfidx, std::max<uint32_t>(1, d0->n_items)));
        CK(cudaMemsetAsync(d_hfidx, 0xff, (size_t)std::max<uint32_t>(1, d0->n_items) * 2, ctx->stream));
        k_hrow_fidx<<<(F0 + 255) / 256, 256, 0, ctx->stream>>>(freq_all, F0, d_hfidx);
        CK(cudaGetLastError());
        CKR(ds.alloc(&d_hscr, (uint64_t)grid * local_max));
        // A row visit: its frequent indices plus about three for the id and offsets.
        h_cost = d0->n_tx ? (float)((double)nnz_f / (double)d0->n_tx) + 3.f : 0.f;
        st.kernel_launches += 4;
    }
    DeepState hs{};
    bool rounds = false, arena_exceeded = false;
    std::vector<float> features;  // per root unit, when traced (cost-model inputs)
    FrameAux *d_aux = nullptr;
    float *d_key = nullptr, *d_key2 = nullptr, *d_feat = nullptr, *d_model = nullptr;
    uint32_t *d_uid = nullptr, *d_uid2 = nullptr;
    void *d_sort_tmp = nullptr;
    size_t sort_bytes = 0;
    if (n_units) {
        CKR(ds.alloc(&d_aux, aux.size()));
        CKR(ds.alloc(&d_key, n_units));
        CKR(ds.alloc(&d_key2, n_units));
        CKR(ds.alloc(&d_uid, n_units));
        CKR(ds.alloc(&d_uid2, n_units));
        if (o.collect_trace) CKR(ds.alloc(&d_feat, n_units * cm::NF));
        if (learned) {
            CKR(ds.alloc(&d_model, cm::N_PARAMS));
            CK(cudaMemcpyAsync(d_model, ctx->model.data(), cm::N_PARAMS * 4, cudaMemcpyHostToDevice, ctx->stream));
        }
        CK(cudaMemcpyAsync(d_aux, aux.data(), aux.size() * sizeof(FrameAux), cudaMemcpyHostToDevice, ctx->stream));
        CK(cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_bytes, d_key, d_key2, d_uid, d_uid2,
                                                     (int64_t)n_units, 0, 32, ctx->stream));
        CKR(ds.alloc(reinterpret_cast<unsigned char **>(&d_sort_tmp), sort_bytes));
    }

    unsigned long long *d_deferred = nullptr;
    if (n_units) CKR(ds.alloc(&d_deferred, n_units));
    for (int attempt = 0;; ++attempt) {
        CKR(grow(ctx, b, frames_cap, members_cap, queue_cap, arena_words, pat_cap + base_patterns, n_units,
                 with_db));
        if (members_cap < P2_total) return set_err(ctx, CPM_EINTERNAL, "member table too small");
        if (rows) {
            k_emit_b<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, ctx->stream>>>(
                d_desc, n_db, rows, off_all, b.pat_parent, b.pat_item, b.pat_sup, b.pat_db, b.mem_pat, b.mem_item,
                b.mem_bits, d_row_list);
            CK(cudaGetLastError());
            st.kernel_launches++;
        }
        if (frames.empty()) {
            hs = DeepState{};
            hs.n_patterns = base_patterns;
            break;
        }
        CK(cudaMemcpyAsync(b.frames, frames.data(), frames.size() * sizeof(DFrame), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(cudaMemsetAsync(b.queue, 0xff, b.queue_cap * 8, ctx->stream));
        if (local_max) CK(cudaMemsetAsync(b.lq, 0xff, b.queue_cap * 8, ctx->stream));
        // Key every root unit (size, or predicted cost), sort largest first
        // (stable), write the queue -- all on the device.
        k_unit_keys<<<(unsigned)((n_units + 127) / 128), 128, 0, ctx->stream>>>(
            b.frames, (uint32_t)frames.size(), d_aux, (uint32_t)n_units, b.mem_pat, b.pat_sup, d_model, d_feat, d_key,
            d_uid);
        CK(cudaGetLastError());
        CK(cub::DeviceRadixSort::SortPairsDescending(d_sort_tmp, sort_bytes, d_key, d_key2, d_uid, d_uid2,
                                                     (int64_t)n_units, 0, 32, ctx->stream));
        k_fill_queue<<<(unsigned)((n_units + 255) / 256), 256, 0, ctx->stream>>>(b.frames, (uint32_t)frames.size(),
                                                                               d_uid2, (uint32_t)n_units, b.queue);
        CK(cudaGetLastError());
        st.kernel_launches += 3;
        if (attempt == 0 && n_db == 1 && db0->hint_arena > arena_budget) {
            // This database's child tidsets did not fit in one launch before.
            rounds = true;
            break;
        }
        if (d_feat && features.empty()) {
            features.resize(n_units * cm::NF);
            CK(cudaMemcpyAsync(features.data(), d_feat, n_units * cm::NF * 4, cudaMemcpyDeviceToHost, ctx->stream));
        }
        CK(cudaMemsetAsync(b.root_cost, 0, std::max<size_t>(1, n_units) * 8, ctx->stream));

        hs = DeepState{};
        hs.q_tail = n_units;
        hs.pending = n_units;
        hs.n_patterns = base_patterns;
        hs.n_frames = frames.size();
        hs.n_members = P2_total;
        CK(cudaMemcpyAsync(b.st, &hs, sizeof hs, cudaMemcpyHostToDevice, ctx->stream));
        DeepParams P;
        P.frames = b.frames; P.frames_cap = b.frames_cap;
        P.mem_pat = b.mem_pat; P.mem_item = b.mem_item; P.mem_bits = b.mem_bits; P.members_cap = b.members_cap;
        P.queue = b.queue; P.queue_cap = b.queue_cap;
        P.arena = b.arena; P.arena_words = b.arena_words;
        P.pat_parent = b.pat_parent; P.pat_item = b.pat_item; P.pat_sup = b.pat_sup; P.pat_db = b.pat_db;
        P.pat_cap = b.pat_cap;
        P.root_cost = b.root_cost; P.st = b.st; P.max_stride = max_stride; P.spin_limit = spin;
        unsigned long long *d_ct = nullptr;
        const bool timing = getenv("CPM_DEBUG") != nullptr;
        if (timing) {
            CKR(ds.alloc(&d_ct, 2ull * grid));
            CK(cudaMemsetAsync(d_ct, 0, 16ull * grid, ctx->stream));
        }
        P.cta_time = d_ct;
        // CPM_UNIT_LOG=<file>: write one record per deep-level unit (k_deep.cuh) there.
        const char *log_path = getenv("CPM_UNIT_LOG");
        P.unit_log = nullptr;
        P.unit_log_cap = 0;
        if (log_path) {
            P.unit_log_cap = 8ull << 20;
            CKR(ds.alloc(&P.unit_log, 1 + P.unit_log_cap * UNIT_LOG_WORDS));
            CK(cudaMemsetAsync(P.unit_log, 0, 8, ctx->stream));
        }
        P.shallow = 0;
        P.balance = ctx->deep_balance;
        // Next ticket taken early when units are queued: measured 1M x 20k
        // 768 -> 756 ms, dense 65,536 x 128 0.887 -> 0.844 ms, planted equal.
        P.prefetch = 1;
        P.lists = use_lists ? list_div : 0u;
        // Root units claimed once the arena is three-quarters full are handed
        // back and finished in memory-bounded rounds after this launch.
        P.root_frames = (uint32_t)frames.size();
        P.defer_words = std::max<uint64_t>(1, b.arena_words / 4 * 3);
        P.defer_members = P2_total + (b.members_cap - P2_total) / 4 * 3;
        P.defer_frames = frames.size() + (b.frames_cap - frames.size()) / 4 * 3;
        P.defer_queue = n_units + (b.queue_cap - n_units) / 4 * 3;
        P.deferred = d_deferred;
        P.deferred_cap = n_units;
        P.root_key = nullptr; P.top_frames = 0; P.keys_in_words = 0; P.admit_words = 0;
        deep_set_local(P, b, max_stride, local_max);
        P.h_off = d_hoff; P.h_rows = d_hrows; P.h_fidx = d_hfidx; P.h_F = F0; P.h_cost = h_cost;
        P.h_scratch = d_hscr; P.h_scratch_words = local_max;
        P.h_table_off = (uint32_t)deep_smem_bytes(max_stride, local_max);
        CK(cudaEventRecord(ctx->ev[2], ctx->stream));
        if (smem_prefix) k_deep<true><<<grid, block, smem_bytes, ctx->stream>>>(P);
        else k_deep<false><<<grid, block, 0, ctx->stream>>>(P);
        CK(cudaGetLastError());
        CKR(launch_local(ctx, P, st));
        CK(cudaEventRecord(ctx->ev[3], ctx->stream));
        st.kernel_launches++;
        CK(cudaMemcpyAsync(&hs, b.st, sizeof hs, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        st.ms_local = local_max ? elapsed_ms(ctx, 7, 3) : 0.0;
        if (P.unit_log) {
            unsigned long long n_log = 0;
            CK(cudaMemcpy(&n_log, P.unit_log, 8, cudaMemcpyDeviceToHost));
            n_log = std::min<unsigned long long>(n_log, P.unit_log_cap);
            std::vector<unsigned long long> rec(n_log * UNIT_LOG_WORDS);
            CK(cudaMemcpy(rec.data(), P.unit_log + 1, rec.size() * 8, cudaMemcpyDeviceToHost));
            if (FILE *f = fopen(log_path, "wb")) {
                fwrite(rec.data(), 8, rec.size(), f);
                fclose(f);
            }
        }
        if (timing) {
            std::vector<unsigned long long> ct(2ull * grid);
            CK(cudaMemcpy(ct.data(), d_ct, 16ull * grid, cudaMemcpyDeviceToHost));
            unsigned long long busy = 0, first = ~0ull, last = 0;
            std::vector<unsigned long long> exits;
            for (unsigned c = 0; c < grid; ++c) {
                busy += ct[2 * c];
                if (ct[2 * c + 1]) {
                    first = std::min(first, ct[2 * c + 1]);
                    last = std::max(last, ct[2 * c + 1]);
                    exits.push_back(ct[2 * c + 1]);
                }
            }
            std::sort(exits.begin(), exits.end());
            const double span = (double)elapsed_ms(ctx, 2, 3) * 1e6;
            fprintf(stderr, "cpm: deep %.3f ms, grid %u, busy %.1f%% of grid x span, exits: first %.3f ms before "
                    "last, median %.3f ms before last, units %llu\n", span / 1e6, grid,
                    100.0 * busy / (span * grid), (last - first) / 1e6,
                    exits.empty() ? 0.0 : (last - exits[exits.size() / 2]) / 1e6, hs.work_items);
        }
        if (!hs.error) break;
        if (hs.error & DEEP_ERR_SPIN)
            return set_err(ctx, CPM_ETIMEOUT, "deep-level kernel wait ran out of spins (limit %llu)",
                           (unsigned long long)spin);
        if (hs.error & DEEP_ERR_INTERNAL)
            return set_err(ctx, CPM_EINTERNAL, "deep-level kernel: a child list disagrees with its support");
        if (attempt >= 12)
            return set_err(ctx, CPM_EOVERFLOW,
                           "deep-level buffers still too small after retries (error 0x%x, frames %llu/%llu, "
                           "members %llu/%llu, queue %llu/%llu, arena %llu/%llu, patterns %llu/%llu)",
                           hs.error, hs.n_frames, (unsigned long long)b.frames_cap, hs.n_members,
                           (unsigned long long)b.members_cap, hs.q_tail, (unsigned long long)b.queue_cap,
                           hs.arena_next, (unsigned long long)b.arena_words, hs.n_patterns,
                           (unsigned long long)b.pat_cap);
        if (getenv("CPM_DEBUG"))
            fprintf(stderr, "cpm: deep retry %d error 0x%x frames %llu members %llu queue %llu arena %llu patterns %llu\n",
                    attempt, hs.error, hs.n_frames, hs.n_members, hs.q_tail, hs.arena_next, hs.n_patterns);
        st.retries++;
        // Counters at the failure are lower bounds of the final need: grow
        // every buffer past them (one overflow usually means several).
        frames_cap = std::max<uint64_t>(frames_cap * 8, hs.n_frames * 8);
        members_cap = std::max<uint64_t>(members_cap * 8, hs.n_members * 8);
        queue_cap = std::max<uint64_t>(queue_cap * 8, std::max(hs.q_tail, hs.lq_tail) * 8);
        pat_cap = std::max<uint64_t>(pat_cap * 8, hs.n_patterns * 8);
        if ((hs.error & DEEP_ERR_ARENA) && arena_words >= arena_budget) {
            rounds = true;  // the child tidsets do not fit at once: bounded rounds below
            arena_exceeded = true;
            break;
        }
        arena_words = std::min<uint64_t>(arena_budget, std::max<uint64_t>(arena_words * 4, hs.arena_next * 4));
    }
    float first_ms = 0.f;
    bool continued = false;
    if (!rounds && !frames.empty() && hs.n_deferred) {
        // The first launch filled its arena and handed root units back: finish
        // them in rounds over the same buffers.
        std::vector<unsigned long long> cont(hs.n_deferred);
        CK(cudaMemcpyAsync(cont.data(), d_deferred, cont.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        first_ms = (float)elapsed_ms(ctx, 2, 3);
        st.intersections = hs.intersections;
        st.bytes_alg = hs.bytes_alg;
        st.work_items = hs.work_items;
        st.projected_units = hs.local_units;
        st.row_units = hs.h_units;
        CKR(deep_rounds(ctx, ds, b, frames, nullptr, nullptr, d_key, 0, base_patterns, P2_total, max_stride, grid, block,
                        smem_prefix, spin, 0, with_db, 0, learned, use_lists ? list_div : 0u, local_max, &cont, hs, st));
        rounds = continued = true;
        ++st.deep_rounds;  // the first launch
    } else if (rounds) {
        st.ms_local = 0.0;  // the first launch's time is not part of ms_deep either
        CKR(deep_rounds(ctx, ds, b, frames, d_uid2, d_key2, d_key, n_units, base_patterns, P2_total, max_stride, grid,
                        block,
                        smem_prefix, spin, pat_cap + base_patterns, with_db, o.arena_bytes ? o.arena_bytes / 8 : 0,
                        learned, use_lists ? list_div : 0u, local_max, nullptr, hs, st));
    }
    lap("deep phase");
    if (n_db == 1) {
        // Remember what this database needed so that the next mine() starts there.
        db0->hint_frames = std::max<uint64_t>(db0->hint_frames, hs.n_frames + hs.n_frames / 4 + 64);
        db0->hint_members = std::max<uint64_t>(db0->hint_members, hs.n_members + hs.n_members / 4 + 64);
        const uint64_t q_used = std::max(hs.q_tail, hs.lq_tail);
        db0->hint_queue = std::max<uint64_t>(db0->hint_queue, q_used + q_used / 4 + 64);
        db0->hint_patterns = std::max<uint64_t>(db0->hint_patterns, hs.n_patterns + hs.n_patterns / 4 + 64);
        // After rounds the arena counter covers one round only; what is known
        // then is whether one launch overflowed the whole budget.
        if (!rounds) db0->hint_arena = std::max<uint64_t>(db0->hint_arena, hs.arena_next + hs.arena_next / 4 + 64);
        else if (arena_exceeded) db0->hint_arena = std::max<uint64_t>(db0->hint_arena, arena_budget + 1);
        else if (continued && !o.arena_bytes)
            db0->hint_arena = std::max<uint64_t>(db0->hint_arena, arena_budget);  // did not fit: take the budget next time
        ctx->plan_hints[plan_key] = {db0->hint_frames, db0->hint_members, db0->hint_queue, db0->hint_patterns,
                                     db0->hint_arena};
    }
    const uint64_t n = hs.n_patterns;
    std::vector<uint32_t> par(n), item(n), sup(n), pdb;
    if (n) {
        CK(cudaMemcpyAsync(par.data(), b.pat_parent, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(item.data(), b.pat_item, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(sup.data(), b.pat_sup, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
        if (with_db) {
            pdb.resize(n);
            CK(cudaMemcpyAsync(pdb.data(), b.pat_db, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    std::vector<unsigned long long> rc;
    if (o.collect_trace && n_units) {
        rc.resize(n_units);
        CK(cudaMemcpyAsync(rc.data(), b.root_cost, n_units * 8, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaEventRecord(ctx->ev[4], ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    st.frames = hs.n_frames;
    st.work_items = hs.work_items;
    st.projected_units = hs.local_units;
    if (!rounds) st.row_units = hs.h_units;  // (rounds run no row-wise units)
    st.intersections = hs.intersections;
    st.bytes_alg = hs.bytes_alg;
    st.ms_pairs = rows ? elapsed_ms(ctx, 5, 6) : 0.0;
    st.ms_deep = frames.empty() ? 0.0 : rounds ? first_ms + ctx->last_deep_ms : elapsed_ms(ctx, 2, 3);
    st.ms_total = elapsed_ms(ctx, 0, 4);
    st.deep_gbs = st.ms_deep > 0 ? st.bytes_alg / (st.ms_deep * 1e6) : 0.0;
    st.pair_tops = st.ms_pairs > 0 ? st.pair_ops / (st.ms_pairs * 1e9) : 0.0;
    st.n_patterns = n;
    lap("pattern download");
    // ---- split the pattern tree per database (parents precede children) ----
    if (n_db == 1) {
        res[0]->parent.swap(par);
        res[0]->item.swap(item);
        res[0]->support.swap(sup);
    } else {
        std::vector<uint32_t> local(n);
        for (uint32_t d = 0; d < n_db; ++d) {
            res[d]->parent.clear(); res[d]->item.clear(); res[d]->support.clear();
        }
        for (uint64_t g = 0; g < n; ++g) {
            cpm_result *r = res[pdb[g]];
            local[g] = (uint32_t)r->parent.size();
            r->parent.push_back(par[g] == 0xffffffffu ? 0xffffffffu : local[par[g]]);
            r->item.push_back(item[g]);
            r->support.push_back(sup[g]);
        }
    }
    for (uint32_t d = 0; d < n_db; ++d) {
        res[d]->stats = st;
        res[d]->stats.n_patterns = res[d]->parent.size();
        if (!rc.empty()) {
            res[d]->trace_x.clear();
            res[d]->trace_y.clear();
            for (uint32_t k = 0; k < frames.size(); ++k) {
                if (frames[k].db != d) continue;
                for (uint32_t p = 0; p + 1 < frames[k].m; ++p) {
                    const uint64_t u = frames[k].root + p;
                    res[d]->trace_x.insert(res[d]->trace_x.end(), &features[u * cm::NF], &features[u * cm::NF] + cm::NF);
                    res[d]->trace_y.push_back((float)std::log1p((double)rc[u]));
                }
            }
        }
    }
    return CPM_OK;
}

static int mine_eclat(cpm_ctx *ctx, cpm_db *db, long long ms, const cpm_opts &o, cpm_result *res) {
    return mine_eclat_batch(ctx, &db, 1, &ms, o, &res);
}


// Exclusive sum of n uint32 counts into uint64 offsets (CUB decoupled
// look-back scan); *total gets the sum (one small read-back, synchronous).
struct U32ToU64 {
    __host__ __device__ uint64_t operator()(uint32_t v) const { return v; }
};

// Exclusive sum of n counts into out; with total, also its sum (one
// device-to-host copy and a sync), without it nothing leaves the device.
static int scan_u32(cpm_ctx *ctx, DevScope &ds, const uint32_t *in, uint64_t *out, uint64_t n, uint64_t *total,
                    uint64_t *d_tot) {
    if (total) *total = 0;
    if (!n) return CPM_OK;
    if (n <= 4096) {
        // Small scans (most Apriori levels): one single-block launch of at
        // most four passes instead of CUB's two launches.
        if (!d_tot) CKR(ds.alloc(&d_tot, 1));
        k_scan_u32<<<1, 1024, 0, ctx->stream>>>(in, n, out, d_tot);
        CK(cudaGetLastError());
        if (!total) return CPM_OK;
        CK(cudaMemcpyAsync(total, d_tot, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        return CPM_OK;
    }
    thrust::transform_iterator<U32ToU64, const uint32_t *, uint64_t> it(in, U32ToU64());
    size_t bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, it, out, (int64_t)n, ctx->stream));
    void *tmp = nullptr;
    CKR(ds.alloc(reinterpret_cast<unsigned char **>(&tmp), bytes));
    CK(cub::DeviceScan::ExclusiveSum(tmp, bytes, it, out, (int64_t)n, ctx->stream));
    if (!total) return CPM_OK;
    uint64_t last_off = 0;
    uint32_t last_in = 0;
    CK(cudaMemcpyAsync(&last_off, out + n - 1, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&last_in, in + n - 1, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *total = last_off + last_in;
    return CPM_OK;
}

// Apriori (cuApriori.py:501-535): level 2 from the pair Gram, then each
// level joined, pruned and counted on the device (k_apriori.cuh).  Two small
// counts come back per level (candidates, survivors) to size the next.
struct PatternArrays {
    uint32_t *parent = nullptr, *item = nullptr, *sup = nullptr;
    uint64_t cap = 0;
};

static int patterns_reserve(cpm_ctx *ctx, PatternArrays &pa, uint64_t used, uint64_t need) {
    if (need <= pa.cap) return CPM_OK;
    uint64_t cap = std::max<uint64_t>(need, pa.cap * 2);
    PatternArrays nw;
    nw.cap = cap;
    CKR(dalloc(ctx, &nw.parent, cap));
    CKR(dalloc(ctx, &nw.item, cap));
    CKR(dalloc(ctx, &nw.sup, cap));
    if (used) {
        CK(cudaMemcpyAsync(nw.parent, pa.parent, used * 4, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(nw.item, pa.item, used * 4, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(nw.sup, pa.sup, used * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    dfree(ctx, pa.parent);
    dfree(ctx, pa.item);
    dfree(ctx, pa.sup);
    pa = nw;
    return CPM_OK;
}

// Grow-only device buffers reused from one Apriori level to the next (one
// slot per array; freed when the mine ends): levels are small and many, and
// allocating every array per level cost more host time than their kernels.
struct LevelScratch {
    cpm_ctx *ctx;
    std::vector<std::pair<void *, size_t>> bufs;  // (pointer, bytes)
    explicit LevelScratch(cpm_ctx *c) : ctx(c) {}
    ~LevelScratch() {
        for (auto &b : bufs)
            if (b.first) cudaFreeAsync(b.first, ctx->stream);
    }
    template <class T>
    int get(size_t slot, T **p, size_t count) {
        if (bufs.size() <= slot) bufs.resize(slot + 1, {nullptr, 0});
        const size_t bytes = std::max<size_t>(1, count) * sizeof(T);
        if (bufs[slot].second < bytes) {
            if (bufs[slot].first) cudaFreeAsync(bufs[slot].first, ctx->stream);
            bufs[slot] = {nullptr, 0};
            const size_t n = (bytes + bytes / 2) / sizeof(T) + 1;
            T *q = nullptr;
            CKR(dalloc(ctx, &q, n));
            bufs[slot] = {q, n * sizeof(T)};
        }
        *p = static_cast<T *>(bufs[slot].first);
        return CPM_OK;
    }
};

// One level's join, shared by the Apriori and the periodic miners
// (cuApriori.py:482-490): the prefix groups of the level's rows L[0, d_cnt2[0])
// of k items, the join partners of every row, then every joined candidate of
// k + 1 items (scratch slot 5), its left row (slot 6) and whether all of its
// k-subsets are in the level (slot 7).  One host round trip: n_pairs is the
// candidate count (0: the search is over) and n_pat the pattern count so far
// (d_cnt2[1]).  Scratch slots 0-7 are used.
// Levels of at most this many rows (and candidate sets of at most this many)
// go through the one-CTA kernels k_level_prep / k_level_keep.
constexpr uint64_t APRIORI_SMALL_LEVEL = 65536;

static int level_join(cpm_ctx *ctx, LevelScratch &scratch, DevScope &lvl, const uint32_t *L, uint64_t n_ub,
                      const uint64_t *d_cnt2, uint32_t k, uint64_t *d_tot, uint64_t &n_pairs, uint64_t &n_pat,
                      uint32_t *&cand, uint32_t *&left, uint32_t *&okf, uint64_t &launches) {
    uint32_t *gflag = nullptr, *partners = nullptr;
    uint64_t *gid = nullptr, *gfirst = nullptr, *poff = nullptr;
    if (n_ub <= APRIORI_SMALL_LEVEL) {
        // One CTA does the prefix groups, the partners and their sum.
        CKR(scratch.get(2, &partners, n_ub));
        CKR(scratch.get(3, &poff, n_ub));
        k_level_prep<<<1, 1024, 0, ctx->stream>>>(L, n_ub, d_cnt2, k, partners, poff, d_tot);
        CK(cudaGetLastError());
        uint64_t counts[3] = {0, 0, 0};
        CK(cudaMemcpyAsync(counts, d_cnt2, 16, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(counts + 2, d_tot, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        n_pat = counts[1];
        n_pairs = counts[2];
        launches += 1;
    } else {
    CKR(scratch.get(0, &gflag, n_ub));
    CKR(scratch.get(1, &gid, n_ub));
    CKR(scratch.get(2, &partners, n_ub));
    CKR(scratch.get(3, &poff, n_ub));
    CKR(scratch.get(4, &gfirst, n_ub + 1));
    const unsigned nb = (unsigned)((n_ub + 255) / 256);
    k_group_start<<<nb, 256, 0, ctx->stream>>>(L, n_ub, d_cnt2, k, gflag);
    CK(cudaGetLastError());
    CKR(scan_u32(ctx, lvl, gflag, gid, n_ub, nullptr, d_tot));
    k_group_first<<<nb, 256, 0, ctx->stream>>>(gflag, gid, d_cnt2, gfirst);
    CK(cudaGetLastError());
    k_partners<<<nb, 256, 0, ctx->stream>>>(gflag, gid, gfirst, n_ub, d_cnt2, partners);
    CK(cudaGetLastError());
    uint64_t counts[2] = {0, 0};
    CK(cudaMemcpyAsync(counts, d_cnt2, 16, cudaMemcpyDeviceToHost, ctx->stream));
    CKR(scan_u32(ctx, lvl, partners, poff, n_ub, &n_pairs, d_tot));  // synchronises: counts are in
    n_pat = counts[1];
    launches += 7;
    }
    cand = left = okf = nullptr;
    if (!n_pairs) return CPM_OK;
    CKR(scratch.get(5, &cand, n_pairs * (k + 1)));
    CKR(scratch.get(6, &left, n_pairs));
    CKR(scratch.get(7, &okf, n_pairs));
    k_join_pairs<<<(unsigned)((n_pairs + 255) / 256), 256, 0, ctx->stream>>>(L, d_cnt2, k, poff, n_pairs, cand, left,
                                                                             okf);
    CK(cudaGetLastError());
    launches++;
    return CPM_OK;
}

// Largest prefix k_count_grouped stages in shared memory.
constexpr size_t APRIORI_GROUP_SMEM = 160 * 1024;

static int mine_apriori(cpm_ctx *ctx, cpm_db *db, long long ms, const cpm_opts &o, cpm_result *res) {
    cpm_stats &st = res->stats;
    DevScope ds(ctx);
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    uint32_t *d_freq = nullptr;
    uint32_t F = 0;
    CKR(mine_singletons(ctx, db, ms, ds, &d_freq, F, st.kernel_launches));
    st.n_frequent_items = F;
    PatternArrays pa;
    struct Free {
        cpm_ctx *c; PatternArrays *p;
        ~Free() { dfree(c, p->parent); dfree(c, p->item); dfree(c, p->sup); }
    } free_patterns{ctx, &pa};
    uint64_t n_pat = 0;
    CKR(patterns_reserve(ctx, pa, 0, std::max<uint64_t>(1024, (uint64_t)F * 4 + db->hint_patterns)));
    if (F) {
        k_emit_singletons<<<(F + 255) / 256, 256, 0, ctx->stream>>>(d_freq, F, db->d_support, pa.parent, pa.item,
                                                                    pa.sup);
        CK(cudaGetLastError());
        st.kernel_launches++;
    }
    n_pat = F;
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    uint64_t *d_total = nullptr;
    CKR(ds.alloc(&d_total, 2));
    if (F >= 2) {
        uint32_t *d_C = nullptr, *d_cnt = nullptr;
        uint64_t *d_off = nullptr;
        CKR(pair_gram(ctx, db, d_freq, F, o, ds, &d_C, st));
        CKR(ds.alloc(&d_cnt, F));
        CKR(ds.alloc(&d_off, F + 1));
        k_pair_count<<<(unsigned)(((uint64_t)F * 32 + 255) / 256), 256, 0, ctx->stream>>>(d_C, F, ms, d_cnt);
        CK(cudaGetLastError());
        k_scan_u32<<<1, 1024, 0, ctx->stream>>>(d_cnt, F, d_off, d_total);
        CK(cudaGetLastError());
        uint64_t P2 = 0;
        CK(cudaMemcpyAsync(&P2, d_total, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        st.kernel_launches += 2;
        st.n_frequent_pairs = P2;
        CKR(patterns_reserve(ctx, pa, n_pat, n_pat + P2));
        uint32_t *L = nullptr, *pid = nullptr;
        CKR(dalloc(ctx, &L, 2 * P2));
        CKR(dalloc(ctx, &pid, P2));
        k_pairs_to_level<<<(unsigned)(((uint64_t)F * 32 + 255) / 256), 256, 0, ctx->stream>>>(
            d_C, F, ms, d_freq, d_off, n_pat, L, pid, pa.parent, pa.item, pa.sup);
        CK(cudaGetLastError());
        st.kernel_launches++;
        n_pat += P2;
        // Row and pattern counts stay on the device (d_cnt2[0], d_cnt2[1]);
        // the host keeps upper bounds (n_ub, pat_ub) for grids and buffers
        // and learns the true counts with each level's one round trip.
        uint64_t *d_cnt2 = nullptr;
        CKR(ds.alloc(&d_cnt2, 2));
        k_set_u64x2<<<1, 1, 0, ctx->stream>>>(d_cnt2, P2, d_cnt2 + 1, n_pat);
        CK(cudaGetLastError());
        uint64_t n_ub = P2, pat_ub = n_pat;
        uint32_t k = 2;
        LevelScratch scratch(ctx);
        uint64_t *d_tot = nullptr;
        CKR(ds.alloc(&d_tot, 1));
        // Candidates sharing a left row share its prefix AND (k_count_grouped)
        // when that prefix fits in shared memory; else every candidate ANDs
        // all of its rows (k_count_pruned).
        const size_t pre_bytes = db->stride * 8;
        const bool grouped = pre_bytes <= APRIORI_GROUP_SMEM;
        unsigned long long *d_bytes = nullptr;
        CKR(ds.alloc(&d_bytes, 1));
        CK(cudaMemsetAsync(d_bytes, 0, 8, ctx->stream));
        int group_ctas = 1;
        if (grouped) {
            CK(cudaFuncSetAttribute(k_count_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)APRIORI_GROUP_SMEM));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&group_ctas, k_count_grouped, 256, pre_bytes));
            group_ctas = std::max(1, group_ctas);
        }
        while (n_ub >= 2) {
            if (k + 1 > 64) {
                dfree(ctx, L);
                dfree(ctx, pid);
                return set_err(ctx, CPM_EINVAL, "patterns longer than 64 items are not supported");
            }
            const uint32_t w = k + 1;
            DevScope lvl(ctx);  // large-scan temporaries only
            // Join and prune, then count and keep.
            uint64_t n_pairs = 0;
            uint32_t *cand = nullptr, *left = nullptr, *okf = nullptr, *sup = nullptr, *pass = nullptr;
            uint64_t *pos = nullptr;
            CKR(level_join(ctx, scratch, lvl, L, n_ub, d_cnt2, k, d_tot, n_pairs, n_pat, cand, left, okf,
                           st.kernel_launches));
            if (!n_pairs) break;
            CKR(scratch.get(8, &sup, n_pairs));
            CKR(scratch.get(9, &pass, n_pairs));
            CKR(scratch.get(10, &pos, n_pairs));
            if (grouped) {
                uint64_t *poff = nullptr;
                uint32_t *partners = nullptr;
                CKR(scratch.get(2, &partners, n_ub));  // written by level_join
                CKR(scratch.get(3, &poff, n_ub));
                const uint64_t grid = std::min<uint64_t>(n_ub, (uint64_t)ctx->sms * group_ctas);
                k_count_grouped<<<(unsigned)grid, 256, pre_bytes, ctx->stream>>>(
                    db->d_bits, db->stride, L, d_cnt2, k, poff, partners, cand, okf, ms, sup, pass, d_bytes);
            } else {
                k_count_pruned<<<(unsigned)((n_pairs * 32 + 255) / 256), 256, 0, ctx->stream>>>(
                    db->d_bits, db->stride, cand, okf, n_pairs, w, ms, sup, pass);
                st.bytes_alg += n_pairs * w * db->stride * 8;
            }
            CK(cudaGetLastError());
            if (n_pairs > APRIORI_SMALL_LEVEL) CKR(scan_u32(ctx, lvl, pass, pos, n_pairs, nullptr, d_tot));
            st.kernel_launches += n_pairs > APRIORI_SMALL_LEVEL ? 3 : 1;
            st.intersections += n_pairs * (w - 1);
            // Survivors: at most n_pairs rows and patterns.
            uint32_t *L2 = nullptr, *pid2 = nullptr;
            CKR(patterns_reserve(ctx, pa, n_pat, pat_ub + n_pairs));
            CKR(dalloc(ctx, &L2, n_pairs * w));
            CKR(dalloc(ctx, &pid2, n_pairs));
            if (n_pairs <= APRIORI_SMALL_LEVEL) {
                k_level_keep<<<1, 1024, 0, ctx->stream>>>(cand, left, sup, pass, n_pairs, w, pid, d_cnt2, L2, pid2,
                                                          pa.parent, pa.item, pa.sup);
                CK(cudaGetLastError());
                st.kernel_launches += 1;
            } else {
                k_apriori_keep<<<(unsigned)((n_pairs + 255) / 256), 256, 0, ctx->stream>>>(
                    cand, left, sup, pass, pos, n_pairs, w, pid, d_cnt2 + 1, L2, pid2, pa.parent, pa.item, pa.sup);
                CK(cudaGetLastError());
                k_level_close<<<1, 1, 0, ctx->stream>>>(pos, pass, n_pairs, d_cnt2, d_cnt2 + 1);
                CK(cudaGetLastError());
                st.kernel_launches += 2;
            }
            dfree(ctx, L);
            dfree(ctx, pid);
            L = L2;
            pid = pid2;
            pat_ub += n_pairs;
            n_ub = n_pairs;
            k = w;
        }
        uint64_t final_pat = 0;
        unsigned long long grouped_bytes = 0;
        CK(cudaMemcpyAsync(&final_pat, d_cnt2 + 1, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(&grouped_bytes, d_bytes, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        n_pat = final_pat;
        st.bytes_alg += grouped_bytes;
        dfree(ctx, L);
        dfree(ctx, pid);
    }
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    res->parent.resize(n_pat);
    res->item.resize(n_pat);
    res->support.resize(n_pat);
    if (n_pat) {
        CK(cudaMemcpyAsync(res->parent.data(), pa.parent, n_pat * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(res->item.data(), pa.item, n_pat * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(res->support.data(), pa.sup, n_pat * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    db->hint_patterns = std::max<uint64_t>(db->hint_patterns, n_pat + n_pat / 4);
    st.n_patterns = n_pat;
    st.ms_pairs = F >= 2 ? elapsed_ms(ctx, 5, 6) : 0.0;
    st.ms_deep = elapsed_ms(ctx, 2, 3);
    st.ms_total = elapsed_ms(ctx, 0, 3);
    st.deep_gbs = st.ms_deep > 0 ? st.bytes_alg / (st.ms_deep * 1e6) : 0.0;
    st.pair_tops = st.ms_pairs > 0 ? st.pair_ops / (st.ms_pairs * 1e9) : 0.0;
    return CPM_OK;
}

// Periodic-frequent itemsets (cuPFEclat.mine, cupami/periodicFrequentPattern/cuPFEclat.py:146-175;
// cuPFApriori.mine, cuPFApriori.py:141-157): an itemset is kept when its
// support is positive and at least min_sup and its periodicity is at most
// max_per (_temporal.py:166-171).  Adding an item only removes rows, so the
// support falls and gaps merge: the kept itemsets are closed under taking
// subsets, and one level-wise search finds them for both miners.  Level 1
// evaluates every item; each later level joins two kept itemsets that share
// all but their last item, drops a candidate with a subset that was not kept
// (k_join_pairs) and evaluates the rest (k_periodic, pruning early).  The
// miners differ only in insertion order, which cpm_result_copy rebuilds
// (CPM_ORDER_DEPTH_FIRST for cuPFEclat, CPM_ORDER_APRIORI for cuPFApriori).
// Warps per candidate for k_periodic: enough for about 32 resident warps per
// SM when a level has few candidates, at most one per step of a row.
// Candidates are split into parts (segments of their rows, joined by
// k_periodic_join): levels of few candidates into enough parts to fill the
// GPU, and every other level into PERIODIC_OVERSPLIT parts, so that the
// densest candidates (pairs of the most frequent items hold tens of thousands
// of rows, against a few hundred on average) do not leave a tail of single
// warps walking their rows.
constexpr uint64_t PERIODIC_OVERSPLIT = 4;

static uint32_t periodic_parts(const cpm_ctx *ctx, uint64_t n, uint64_t words) {
    const uint64_t tiles = (words + PERIODIC_TILE - 1) / PERIODIC_TILE;
    const uint64_t target = (uint64_t)ctx->sms * 32;
    if (!n || tiles <= 1) return 1;
    const uint64_t want = n >= target ? PERIODIC_OVERSPLIT : (target + n - 1) / n;
    return (uint32_t)std::min<uint64_t>(std::min<uint64_t>(want, tiles), 1024);
}

// k_periodic over n candidates, split `parts` ways (seg: n * parts summaries),
// plus k_periodic_join when split.
template <class Word, bool kPrune>
static int periodic_launch(cpm_ctx *ctx, uint32_t parts, PSeg *seg, const Word *bits, uint64_t stride,
                           const uint32_t *cand, const uint32_t *okf, uint64_t n, uint32_t width, const long long *ts,
                           uint64_t n_tx, long long end, long long need, long long max_per, unsigned long long *sup,
                           long long *per, uint32_t *pass, uint64_t &launches) {
    const uint64_t warps = n * parts;
    k_periodic<Word, kPrune><<<(unsigned)((warps + 7) / 8), 256, 0, ctx->stream>>>(
        bits, stride, cand, okf, n, width, ts, n_tx, end, need, max_per, parts, seg, sup, per, pass);
    CK(cudaGetLastError());
    launches++;
    if (parts > 1) {
        k_periodic_join<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(seg, parts, okf, n, end, need, max_per,
                                                                              sup, per, pass);
        CK(cudaGetLastError());
        launches++;
    }
    return CPM_OK;
}

static int mine_periodic(cpm_ctx *ctx, cpm_db *db, long long ms, long long max_per, cpm_result *res) {
    cpm_stats &st = res->stats;
    DevScope ds(ctx);
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    const long long need = std::max<long long>(ms, 1);
    const auto *bits = reinterpret_cast<const unsigned long long *>(db->d_bits);
    const uint32_t n_items = db->n_items;
    const uint64_t words = (db->n_tx + 63) / 64;
    PatternArrays pa;
    long long *pat_per = nullptr;
    uint64_t per_cap = 0;
    uint32_t *L = nullptr, *pid = nullptr;
    struct Free {
        cpm_ctx *c; PatternArrays *p; long long **per; uint32_t **L, **pid;
        ~Free() {
            dfree(c, p->parent); dfree(c, p->item); dfree(c, p->sup);
            dfree(c, *per); dfree(c, *L); dfree(c, *pid);
        }
    } free_all{ctx, &pa, &pat_per, &L, &pid};
    // Pattern records and their periods grow together.
    auto reserve = [&](uint64_t used, uint64_t want) -> int {
        CKR(patterns_reserve(ctx, pa, used, want));
        if (per_cap < pa.cap) {
            long long *nw = nullptr;
            CKR(dalloc(ctx, &nw, pa.cap));
            if (used) CK(cudaMemcpyAsync(nw, pat_per, used * 8, cudaMemcpyDeviceToDevice, ctx->stream));
            dfree(ctx, pat_per);
            pat_per = nw;
            per_cap = pa.cap;
        }
        return CPM_OK;
    };
    uint64_t *d_cnt2 = nullptr, *d_tot = nullptr;  // (rows of the level, patterns so far); scan total
    CKR(ds.alloc(&d_cnt2, 2));
    CKR(ds.alloc(&d_tot, 1));
    k_set_u64x2<<<1, 1, 0, ctx->stream>>>(d_cnt2, 0, d_cnt2 + 1, 0);
    CK(cudaGetLastError());
    st.kernel_launches++;
    CKR(reserve(0, std::max<uint64_t>(1024, db->hint_patterns)));
    uint64_t n_ub = 0, pat_ub = 0;
    if (n_items) {
        uint32_t *cand = nullptr, *pass = nullptr;
        unsigned long long *sup = nullptr;
        long long *per = nullptr;
        uint64_t *pos = nullptr;
        CKR(ds.alloc(&cand, n_items));
        CKR(ds.alloc(&pass, n_items));
        CKR(ds.alloc(&sup, n_items));
        CKR(ds.alloc(&per, n_items));
        CKR(ds.alloc(&pos, n_items));
        k_iota_u32<<<(n_items + 255) / 256, 256, 0, ctx->stream>>>(cand, n_items);
        CK(cudaGetLastError());
        const uint32_t parts = periodic_parts(ctx, n_items, words);
        PSeg *seg = nullptr;
        if (parts > 1) CKR(ds.alloc(&seg, (uint64_t)n_items * parts));
        CKR((periodic_launch<unsigned long long, true>(ctx, parts, seg, bits, db->stride, cand, nullptr, n_items, 1,
                                                        db->d_ts, db->n_tx, db->end, need, max_per, sup, per, pass,
                                                        st.kernel_launches)));
        uint64_t F1 = 0;
        CKR(scan_u32(ctx, ds, pass, pos, n_items, &F1, d_tot));
        st.n_frequent_items = F1;
        CKR(reserve(0, F1 * 4 + db->hint_patterns));
        CKR(dalloc(ctx, &L, F1));
        CKR(dalloc(ctx, &pid, F1));
        k_periodic_keep<<<(n_items + 255) / 256, 256, 0, ctx->stream>>>(
            cand, nullptr, sup, per, pass, pos, n_items, 1, nullptr, d_cnt2 + 1, L, pid, pa.parent, pa.item, pa.sup,
            pat_per);
        CK(cudaGetLastError());
        k_level_close<<<1, 1, 0, ctx->stream>>>(pos, pass, n_items, d_cnt2, d_cnt2 + 1);
        CK(cudaGetLastError());
        st.kernel_launches += 4;
        st.intersections += n_items;
        n_ub = pat_ub = F1;
    }
    LevelScratch scratch(ctx);
    uint32_t k = 1;
    while (n_ub >= 2) {
        if (k + 1 > 64) return set_err(ctx, CPM_EINVAL, "patterns longer than 64 items are not supported");
        const uint32_t w = k + 1;
        DevScope lvl(ctx);  // large-scan temporaries only
        uint64_t n_pairs = 0, n_pat = 0;
        uint32_t *cand = nullptr, *left = nullptr, *okf = nullptr, *pass = nullptr;
        unsigned long long *sup = nullptr;
        long long *per = nullptr;
        uint64_t *pos = nullptr;
        CKR(level_join(ctx, scratch, lvl, L, n_ub, d_cnt2, k, d_tot, n_pairs, n_pat, cand, left, okf,
                       st.kernel_launches));
        if (!n_pairs) break;
        CKR(scratch.get(8, &sup, n_pairs));
        CKR(scratch.get(9, &pass, n_pairs));
        CKR(scratch.get(10, &pos, n_pairs));
        CKR(scratch.get(11, &per, n_pairs));
        const uint32_t parts = periodic_parts(ctx, n_pairs, words);
        PSeg *seg = nullptr;
        if (parts > 1) CKR(scratch.get(12, &seg, n_pairs * parts));
        CKR((periodic_launch<unsigned long long, true>(ctx, parts, seg, bits, db->stride, cand, okf, n_pairs, w,
                                                        db->d_ts, db->n_tx, db->end, need, max_per, sup, per, pass,
                                                        st.kernel_launches)));
        CKR(scan_u32(ctx, lvl, pass, pos, n_pairs, nullptr, d_tot));
        st.kernel_launches += 2;
        st.intersections += n_pairs * (w - 1);
        uint32_t *L2 = nullptr, *pid2 = nullptr;
        CKR(reserve(n_pat, pat_ub + n_pairs));
        CKR(dalloc(ctx, &L2, n_pairs * w));
        CKR(dalloc(ctx, &pid2, n_pairs));
        k_periodic_keep<<<(unsigned)((n_pairs + 255) / 256), 256, 0, ctx->stream>>>(
            cand, left, sup, per, pass, pos, n_pairs, w, pid, d_cnt2 + 1, L2, pid2, pa.parent, pa.item, pa.sup,
            pat_per);
        CK(cudaGetLastError());
        k_level_close<<<1, 1, 0, ctx->stream>>>(pos, pass, n_pairs, d_cnt2, d_cnt2 + 1);
        CK(cudaGetLastError());
        st.kernel_launches += 2;
        dfree(ctx, L);
        dfree(ctx, pid);
        L = L2;
        pid = pid2;
        pat_ub += n_pairs;
        n_ub = n_pairs;
        k = w;
    }
    uint64_t n_pat = 0;
    CK(cudaMemcpyAsync(&n_pat, d_cnt2 + 1, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    res->parent.resize(n_pat);
    res->item.resize(n_pat);
    res->support.resize(n_pat);
    res->period.resize(n_pat);
    if (n_pat) {
        CK(cudaMemcpyAsync(res->parent.data(), pa.parent, n_pat * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(res->item.data(), pa.item, n_pat * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(res->support.data(), pa.sup, n_pat * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(res->period.data(), pat_per, n_pat * 8, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    db->hint_patterns = std::max<uint64_t>(db->hint_patterns, n_pat + n_pat / 4);
    st.n_patterns = n_pat;
    st.ms_total = st.ms_deep = elapsed_ms(ctx, 0, 3);
    return CPM_OK;
}

extern "C" int cpm_mine_periodic(cpm_ctx *ctx, cpm_db *db, int64_t min_sup, int64_t max_per, int algo,
                                 cpm_result **out) {
    if (!ctx || !db || !out || db->ctx != ctx) return CPM_EINVAL;
    *out = nullptr;
    if (!db->temporal) return set_err(ctx, CPM_EINVAL, "periodic mining needs a temporal database (cpm_tdb_from_csr)");
    if (algo != CPM_ECLAT && algo != CPM_APRIORI) return set_err(ctx, CPM_EINVAL, "unknown algorithm %d", algo);
    CK(cudaSetDevice(ctx->device));
    // Supports are 32-bit counts; thresholds beyond every count pass nothing.
    const long long ms = (long long)std::min<int64_t>(min_sup, (int64_t)1 << 40);
    cpm_result *res = new cpm_result();
    res->algo = algo;
    const int r = mine_periodic(ctx, db, ms, (long long)max_per, res);
    if (r != CPM_OK) {
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        delete res;
        return r;
    }
    *out = res;
    return CPM_OK;
}

extern "C" int cpm_mine(cpm_ctx *ctx, cpm_db *db, int64_t min_sup, int algo, const cpm_opts *opts,
                        cpm_result **out) {
    if (!ctx || !db || !out || db->ctx != ctx) return CPM_EINVAL;
    if (algo != CPM_ECLAT && algo != CPM_APRIORI) return set_err(ctx, CPM_EINVAL, "unknown algorithm %d", algo);
    *out = nullptr;
    CK(cudaSetDevice(ctx->device));
    cpm_opts o;
    if (opts) o = *opts;
    else cpm_default_opts(&o);
    // Supports are 32-bit counts; thresholds beyond every count pass nothing.
    const long long ms = (long long)std::max<int64_t>(std::min<int64_t>(min_sup, (int64_t)1 << 40), -1);
    cpm_result *res = new cpm_result();
    res->algo = algo;
    const auto t0 = std::chrono::steady_clock::now();
    int r = algo == CPM_ECLAT ? mine_eclat(ctx, db, ms, o, res) : mine_apriori(ctx, db, ms, o, res);
    if (r != CPM_OK) {
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        delete res;
        return r;
    }
    (void)t0;
    *out = res;
    return CPM_OK;
}

extern "C" int cpm_mine_batch(cpm_ctx *ctx, cpm_db **dbs, uint32_t n_db, const int64_t *min_sups,
                              const cpm_opts *opts, cpm_result **out) {
    if (!ctx || !out || (n_db && (!dbs || !min_sups))) return CPM_EINVAL;
    for (uint32_t d = 0; d < n_db; ++d) {
        out[d] = nullptr;
        if (!dbs[d] || dbs[d]->ctx != ctx) return set_err(ctx, CPM_EINVAL, "database %u is not on this context", d);
    }
    if (!n_db) return CPM_OK;
    CK(cudaSetDevice(ctx->device));
    cpm_opts o;
    if (opts) o = *opts;
    else cpm_default_opts(&o);
    std::vector<long long> ms(n_db);
    std::vector<cpm_result *> res(n_db);
    for (uint32_t d = 0; d < n_db; ++d) {
        ms[d] = (long long)std::max<int64_t>(std::min<int64_t>(min_sups[d], (int64_t)1 << 40), -1);
        res[d] = new cpm_result();
        res[d]->algo = CPM_ECLAT;
    }
    const int r = mine_eclat_batch(ctx, dbs, n_db, ms.data(), o, res.data());
    if (r != CPM_OK) {
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        for (cpm_result *x : res) delete x;
        return r;
    }
    for (uint32_t d = 0; d < n_db; ++d) out[d] = res[d];
    return CPM_OK;
}

extern "C" int cpm_autotune(cpm_ctx *ctx, cpm_db *db, int64_t min_sup, const cpm_opts *opts, int32_t *block,
                            int32_t *ctas_per_sm, int32_t *list_div, double *ms_deep) {
    if (!ctx || !db) return CPM_EINVAL;
    cpm_opts o;
    if (opts) o = *opts;
    else cpm_default_opts(&o);
    o.autotune = 0;
    o.collect_trace = 0;
    static const int blocks[4] = {128, 256, 512, 1024};
    double best = 1e300;
    int best_block = 0, best_ctas = 0;
    for (int bi = 0; bi < 4; ++bi) {
        for (int c = 1; c <= 4; ++c) {
            o.deep_block = blocks[bi];
            o.deep_ctas_per_sm = c;
            double t = 1e300;
            int used = c;
            for (int rep = 0; rep < 2; ++rep) {
                cpm_result *r = nullptr;
                const int rc = cpm_mine(ctx, db, min_sup, CPM_ECLAT, &o, &r);
                if (rc != CPM_OK) return rc;
                t = std::min(t, r->stats.ms_deep);
                used = ctx->last_deep_ctas;
                cpm_result_free(r);
            }
            if (t < best) {
                best = t;
                best_block = blocks[bi];
                best_ctas = used;
            }
            if (used < c) break;  // occupancy allows no more CTAs of this size
        }
    }
    const int bucket = 63 - __builtin_clzll(std::max<uint64_t>(1, db->stride));
    ctx->tune[bucket] = {best_block, best_ctas};
    // Tidset forms at that shape: bitsets only, or lists below 1/1 .. 1/8 of the bitset.
    if (db->stride * 8 <= DEEP_SMEM_PREFIX_MAX) {
        o.deep_block = best_block;
        o.deep_ctas_per_sm = best_ctas;
        int best_div = -1;
        double best_l = 1e300;
        static const int divs[5] = {0, 1, 2, 4, 8};
        for (int di = 0; di < 5; ++di) {
            o.tidsets = divs[di] ? 2 : 1;
            o.list_div = divs[di];
            double t = 1e300;
            for (int rep = 0; rep < 2; ++rep) {
                cpm_result *r = nullptr;
                const int rc = cpm_mine(ctx, db, min_sup, CPM_ECLAT, &o, &r);
                if (rc != CPM_OK) return rc;
                t = std::min(t, r->stats.ms_deep);
                cpm_result_free(r);
            }
            if (t < best_l) {
                best_l = t;
                best_div = divs[di];
            }
        }
        ctx->tune_lists[bucket] = best_div;
        best = std::min(best, best_l);
    }
    if (block) *block = best_block;
    if (ctas_per_sm) *ctas_per_sm = best_ctas;
    if (list_div) {
        const auto it = ctx->tune_lists.find(bucket);
        *list_div = it == ctx->tune_lists.end() ? 0 : it->second;
    }
    if (ms_deep) *ms_deep = best;
    return CPM_OK;
}

extern "C" int cpm_result_size(const cpm_result *res, uint64_t *n_patterns, uint64_t *n_item_slots) {
    if (!res) return CPM_EINVAL;
    const uint64_t n = res->parent.size();
    if (n_patterns) *n_patterns = n;
    if (n_item_slots) {
        // depth of every pattern (parents always precede children)
        std::vector<uint32_t> depth(n);
        uint64_t tot = 0;
        for (uint64_t k = 0; k < n; ++k) {
            depth[k] = res->parent[k] == 0xffffffffu ? 1 : depth[res->parent[k]] + 1;
            tot += depth[k];
        }
        *n_item_slots = tot;
    }
    return CPM_OK;
}

extern "C" int cpm_result_tree(const cpm_result *res, int64_t *parent, uint32_t *item, uint64_t *support) {
    if (!res) return CPM_EINVAL;
    for (size_t k = 0; k < res->parent.size(); ++k) {
        if (parent) parent[k] = res->parent[k] == 0xffffffffu ? -1 : (int64_t)res->parent[k];
        if (item) item[k] = res->item[k];
        if (support) support[k] = res->support[k];
    }
    return CPM_OK;
}

// Patterns of a result in the requested order.  A pattern is its parent's
// items plus its own.  The device builds a prefix tree (every pattern extends
// its parent by a larger item), so the insertion orders are traversals of
// that tree; any other tree is ordered by comparing item lists.
static int result_copy(const cpm_result *res, int order, uint64_t *offsets, uint32_t *items, uint64_t *supports,
                       int64_t *periods) {
    if (!res || !offsets || !supports) return CPM_EINVAL;
    if (order != CPM_ORDER_ECLAT && order != CPM_ORDER_APRIORI && order != CPM_ORDER_NONE &&
        order != CPM_ORDER_DEPTH_FIRST)
        return CPM_EINVAL;
    if (periods && res->period.size() != res->parent.size()) return CPM_EINVAL;
    const uint64_t n = res->parent.size();
    const uint32_t *par = res->parent.data(), *itm = res->item.data();
    const bool dbg = getenv("CPM_DEBUG") != nullptr;
    auto t0 = std::chrono::steady_clock::now();
    auto lap = [&](const char *what) {
        if (!dbg) return;
        const auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "cpm: order %-16s %.3f ms\n", what, std::chrono::duration<double, std::milli>(now - t0).count());
        t0 = now;
    };
    // Scratch kept per thread across calls: large fresh allocations cost a
    // page fault per 4 KB on first touch, which dominated this function.
    static thread_local std::vector<uint32_t> depth_s;
    static thread_local std::vector<uint64_t> idx_s, coff_s, kids_s, fill_s;
    if (depth_s.size() < n) depth_s.resize(n);
    uint32_t *depth = depth_s.data();
    for (uint64_t k = 0; k < n; ++k) {
        const uint32_t p = par[k];
        if (p != 0xffffffffu && p >= k) return CPM_EINTERNAL;
        depth[k] = p == 0xffffffffu ? 1 : depth[p] + 1;
    }
    bool prefix_tree = true;
    for (uint64_t k = 0; k < n && prefix_tree; ++k)
        if (par[k] != 0xffffffffu && itm[k] <= itm[par[k]]) prefix_tree = false;
    lap("depth, check");
    if (idx_s.size() < n) idx_s.resize(n);
    uint64_t *idx = idx_s.data();
    std::iota(idx, idx + n, 0ull);
    std::vector<uint64_t> start;  // item lists in device order (only for non-prefix trees)
    std::vector<uint32_t> flat;
    auto pat = [&](uint64_t k) { return flat.data() + start[k]; };
    if (prefix_tree && order != CPM_ORDER_NONE) {
        // children lists (counting sort by parent), each sorted by item
        if (coff_s.size() < n + 2) coff_s.resize(n + 2);
        uint64_t *coff = coff_s.data();
        std::fill(coff, coff + n + 2, 0ull);
        std::vector<uint64_t> roots;
        for (uint64_t k = 0; k < n; ++k)
            if (par[k] == 0xffffffffu) roots.push_back(k);
#pragma omp parallel for schedule(static, 65536)
        for (int64_t k = 0; k < (int64_t)n; ++k)
            if (par[k] != 0xffffffffu) __atomic_fetch_add(&coff[par[k] + 1], 1ull, __ATOMIC_RELAXED);
        for (uint64_t k = 0; k < n; ++k) coff[k + 1] += coff[k];
        if (kids_s.size() < coff[n] + 1) kids_s.resize(coff[n] + 1);
        if (fill_s.size() < n + 1) fill_s.resize(n + 1);
        uint64_t *kids = kids_s.data(), *fill = fill_s.data();
        std::copy(coff, coff + n, fill);
        // Children in any order here: every list is sorted by item below.
#pragma omp parallel for schedule(static, 65536)
        for (int64_t k = 0; k < (int64_t)n; ++k)
            if (par[k] != 0xffffffffu) kids[__atomic_fetch_add(&fill[par[k]], 1ull, __ATOMIC_RELAXED)] = (uint64_t)k;
        lap("children");
        auto by_item = [&](uint64_t a, uint64_t b) { return itm[a] < itm[b]; };
        std::sort(roots.begin(), roots.end(), by_item);
#pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t k = 0; k < (int64_t)n; ++k)
            if (coff[k + 1] - coff[k] > 1) std::sort(kids + coff[k], kids + coff[k + 1], by_item);
        lap("sort children");
        uint64_t w = 0;
        if (order == CPM_ORDER_APRIORI) {
            // by length, then tuple: breadth first, children in item order
            std::vector<uint64_t> level(roots), next;
            while (!level.empty()) {
                next.clear();
                for (uint64_t v : level) {
                    idx[w++] = v;
                    next.insert(next.end(), kids + coff[v], kids + coff[v + 1]);
                }
                level.swap(next);
            }
        } else {
            // Eclat: singletons, pairs, then for every pair: its children, then
            // each child's subtree in the same way (cuEclat.py:211-245).
            // Depth first: singletons, then for every singleton: its children,
            // then each child's subtree (cuPFEclat.py:160-173).
            for (uint64_t r : roots) idx[w++] = r;
            std::vector<uint64_t> pairs;
            if (order == CPM_ORDER_DEPTH_FIRST) {
                pairs = roots;
            } else {
                for (uint64_t r : roots)
                    for (uint64_t c = coff[r]; c < coff[r + 1]; ++c) pairs.push_back(kids[c]);
                for (uint64_t q : pairs) idx[w++] = q;
            }
            // Every pair's descendants take a contiguous range of the order:
            // descendant counts bottom up (deepest level first; parents
            // precede children, so the levels are the depths), then each
            // pair's range is walked on its own thread.
            std::vector<uint64_t> desc(n, 0);
            uint32_t max_depth = 0;
            for (uint64_t k = 0; k < n; ++k) max_depth = std::max(max_depth, depth[k]);
            std::vector<uint64_t> doff(max_depth + 2, 0), dnode(n);
            for (uint64_t k = 0; k < n; ++k) ++doff[depth[k] + 1];
            for (uint32_t d = 0; d <= max_depth; ++d) doff[d + 1] += doff[d];
            {
                std::vector<uint64_t> dfill(doff.begin(), doff.end() - 1);
                for (uint64_t k = 0; k < n; ++k) dnode[dfill[depth[k]]++] = k;
            }
            for (uint32_t d = max_depth; d >= 2; --d) {
#pragma omp parallel for schedule(static, 16384)
                for (int64_t i = (int64_t)doff[d]; i < (int64_t)doff[d + 1]; ++i) {
                    const uint64_t k = dnode[i];
                    __atomic_fetch_add(&desc[par[k]], desc[k] + 1, __ATOMIC_RELAXED);
                }
            }
            std::vector<uint64_t> pstart(pairs.size() + 1, w);
            for (size_t i = 0; i < pairs.size(); ++i) pstart[i + 1] = pstart[i] + desc[pairs[i]];
            if (pstart[pairs.size()] != n) return CPM_EINTERNAL;
#pragma omp parallel for schedule(dynamic, 1)
            for (int64_t i = 0; i < (int64_t)pairs.size(); ++i) {
                std::vector<std::pair<uint64_t, uint64_t>> stack;  // (node, next child to descend)
                uint64_t at = pstart[i];
                const uint64_t q = pairs[i];
                for (uint64_t c = coff[q]; c < coff[q + 1]; ++c) idx[at++] = kids[c];
                stack.push_back({q, coff[q]});
                while (!stack.empty()) {
                    auto &top = stack.back();
                    if (top.second == coff[top.first + 1]) {
                        stack.pop_back();
                        continue;
                    }
                    const uint64_t child = kids[top.second++];
                    for (uint64_t c = coff[child]; c < coff[child + 1]; ++c) idx[at++] = kids[c];
                    stack.push_back({child, coff[child]});
                }
            }
            w = n;
        }
        if (w != n) return CPM_EINTERNAL;
    } else if (order != CPM_ORDER_NONE || !prefix_tree) {
        // Item lists, sorted ascending within each pattern (parents precede
        // children, so a parent's list is sorted when a child copies it).
        start.assign(n + 1, 0);
        for (uint64_t k = 0; k < n; ++k) start[k + 1] = start[k] + depth[k];
        flat.resize(start[n]);
        for (uint64_t k = 0; k < n; ++k) {
            uint32_t *a = flat.data() + start[k];
            const uint32_t p = par[k];
            const uint32_t d = depth[k];
            if (p != 0xffffffffu) memcpy(a, flat.data() + start[p], (d - 1) * 4);
            a[d - 1] = itm[k];
            for (uint32_t i = d - 1; i > 0 && a[i] < a[i - 1]; --i) std::swap(a[i], a[i - 1]);
        }
        if (order == CPM_ORDER_APRIORI) {
            std::sort(idx, idx + n, [&](uint64_t a, uint64_t b) {
                if (depth[a] != depth[b]) return depth[a] < depth[b];
                return std::lexicographical_compare(pat(a), pat(a) + depth[a], pat(b), pat(b) + depth[b]);
            });
        } else if (order == CPM_ORDER_ECLAT || order == CPM_ORDER_DEPTH_FIRST) {
            // cuEclat inserts singletons, then pairs, then every deeper pattern in
            // the order of its class search: key (x1..x_{k-1}, -1, x_k).  The
            // depth-first order uses that key from the pairs on.
            const uint32_t deep = order == CPM_ORDER_ECLAT ? 3 : 2;
            std::sort(idx, idx + n, [&](uint64_t a, uint64_t b) {
                const uint32_t ga = std::min<uint32_t>(depth[a], deep), gb = std::min<uint32_t>(depth[b], deep);
                if (ga != gb) return ga < gb;
                if (ga < deep) return std::lexicographical_compare(pat(a), pat(a) + depth[a], pat(b), pat(b) + depth[b]);
                const uint32_t *x = pat(a), *y = pat(b);
                const int64_t la = depth[a] + 1, lb = depth[b] + 1;
                for (int64_t i = 0; i < std::min(la, lb); ++i) {
                    const int64_t u = i < la - 2 ? (int64_t)x[i] : (i == la - 2 ? (int64_t)-1 : (int64_t)x[la - 2]);
                    const int64_t v = i < lb - 2 ? (int64_t)y[i] : (i == lb - 2 ? (int64_t)-1 : (int64_t)y[lb - 2]);
                    if (u != v) return u < v;
                }
                return la < lb;
            });
        }
    }
    lap("order");
    // offsets: exclusive sum of the depths in order (two parallel passes)
    offsets[0] = 0;
    {
        const int64_t chunk = 1 << 18, nc = (int64_t)((n + chunk - 1) / chunk);
        std::vector<uint64_t> part(nc + 1, 0);
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < nc; ++c) {
            uint64_t sum = 0;
            for (int64_t r = c * chunk; r < std::min<int64_t>((int64_t)n, (c + 1) * chunk); ++r) sum += depth[idx[r]];
            part[c + 1] = sum;
        }
        for (int64_t c = 0; c < nc; ++c) part[c + 1] += part[c];
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < nc; ++c) {
            uint64_t sum = part[c];
            for (int64_t r = c * chunk; r < std::min<int64_t>((int64_t)n, (c + 1) * chunk); ++r) {
                sum += depth[idx[r]];
                offsets[r + 1] = sum;
            }
        }
    }
    lap("offsets");
#pragma omp parallel for schedule(static, 65536)
    for (int64_t r = 0; r < (int64_t)n; ++r) {
        const uint64_t k = idx[r];
        supports[r] = res->support[k];
        if (periods) periods[r] = res->period[k];
        if (!items) continue;
        uint32_t *a = items + offsets[r];
        if (!flat.empty()) {
            memcpy(a, pat(k), depth[k] * 4);
        } else {
            // prefix tree: walk up the parents, last item first (already ascending)
            uint64_t v = k;
            for (uint32_t i = depth[k]; i-- > 0; v = par[v]) a[i] = itm[v];
        }
    }
    lap("items");
    return CPM_OK;
}

extern "C" int cpm_result_copy(const cpm_result *res, int order, uint64_t *offsets, uint32_t *items,
                               uint64_t *supports) {
    return result_copy(res, order, offsets, items, supports, nullptr);
}

extern "C" int cpm_result_copy_periodic(const cpm_result *res, int order, uint64_t *offsets, uint32_t *items,
                                        uint64_t *supports, int64_t *periods) {
    if (!periods) return CPM_EINVAL;
    return result_copy(res, order, offsets, items, supports, periods);
}

extern "C" int cpm_results_copy(cpm_result *const *res, uint32_t n, int order, uint64_t *sizes,
                                uint64_t *offsets, uint32_t *items, uint64_t *supports) {
    if (!res || !sizes) return CPM_EINVAL;
    // sizes[2k], sizes[2k+1] = patterns and item slots of result k; with
    // output arrays, result k's rows follow result k-1's (offsets restart at 0
    // for every result and take n_k + 1 entries).
    for (uint32_t k = 0; k < n; ++k)
        if (!res[k] || cpm_result_size(res[k], &sizes[2 * k], &sizes[2 * k + 1]) != CPM_OK) return CPM_EINVAL;
    if (!offsets || !supports) return CPM_OK;
    // Every result's place in the outputs first, then the results ordered in
    // parallel (each ordering keeps its scratch per thread).
    std::vector<uint64_t> o(n + 1, 0), it(n + 1, 0), sp(n + 1, 0);
    for (uint32_t k = 0; k < n; ++k) {
        o[k + 1] = o[k] + sizes[2 * k] + 1;
        it[k + 1] = it[k] + sizes[2 * k + 1];
        sp[k + 1] = sp[k] + sizes[2 * k];
    }
    int status = CPM_OK;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t k = 0; k < (int64_t)n; ++k) {
        const int r = cpm_result_copy(res[k], order, offsets + o[k], items ? items + it[k] : nullptr, supports + sp[k]);
        if (r != CPM_OK) {
#pragma omp critical
            status = r;
        }
    }
    return status;
}

extern "C" int cpm_result_from_tree(const int64_t *parent, const uint32_t *item, const uint64_t *support,
                                    uint64_t n, cpm_result **out) {
    if (!out || (n && (!parent || !item || !support))) return CPM_EINVAL;
    *out = nullptr;
    cpm_result *res = new cpm_result();
    res->parent.resize(n);
    res->item.assign(item, item + n);
    res->support.resize(n);
    for (uint64_t k = 0; k < n; ++k) {
        if (parent[k] >= (int64_t)k || parent[k] < -1 || support[k] > 0xffffffffull) {
            delete res;
            return CPM_EINVAL;
        }
        res->parent[k] = parent[k] < 0 ? 0xffffffffu : (uint32_t)parent[k];
        res->support[k] = (uint32_t)support[k];
    }
    res->stats.n_patterns = n;
    *out = res;
    return CPM_OK;
}

extern "C" int cpm_result_from_tree_periodic(const int64_t *parent, const uint32_t *item, const uint64_t *support,
                                             const int64_t *period, uint64_t n, cpm_result **out) {
    if (!out || (n && !period)) return CPM_EINVAL;
    const int r = cpm_result_from_tree(parent, item, support, n, out);
    if (r != CPM_OK) return r;
    (*out)->period.assign(period, period + n);
    return CPM_OK;
}

extern "C" int cpm_result_stats(const cpm_result *res, cpm_stats *stats) {
    if (!res || !stats) return CPM_EINVAL;
    *stats = res->stats;
    return CPM_OK;
}

extern "C" void cpm_result_free(cpm_result *res) { delete res; }

// ---------------------------------------------------------------------------
// reference kernel-module API
// ---------------------------------------------------------------------------

extern "C" int cpm_build_bitsets(cpm_ctx *ctx, const uint64_t *d_rows, const uint32_t *d_columns, uint64_t count,
                                 uint64_t transactions, uint32_t items, uint32_t *d_bitsets) {
    if (!ctx || (count && (!d_rows || !d_columns)) || (items && !d_bitsets)) return CPM_EINVAL;
    CK(cudaSetDevice(ctx->device));
    const uint64_t words = (transactions + 31) / 32;
    if (items && words) CK(cudaMemsetAsync(d_bitsets, 0, (size_t)items * words * 4, ctx->stream));
    if (count) {
        const unsigned blocks = (unsigned)std::min<uint64_t>((count + 255) / 256, (uint64_t)ctx->sms * 32);
        k_ref_build<<<blocks, 256, 0, ctx->stream>>>(d_rows, d_columns, count, words, d_bitsets);
        CK(cudaGetLastError());
    }
    return CPM_OK;
}

extern "C" int cpm_count_supports(cpm_ctx *ctx, const uint32_t *d_bitsets, uint64_t words32,
                                  const uint32_t *d_candidates, uint64_t n_candidates, uint32_t width,
                                  uint64_t *d_supports) {
    if (!ctx || (n_candidates && (!d_candidates || !d_supports || !width))) return CPM_EINVAL;
    CK(cudaSetDevice(ctx->device));
    if (!n_candidates) return CPM_OK;
    k_ref_count<<<(unsigned)((n_candidates * 32 + 255) / 256), 256, 0, ctx->stream>>>(
        d_bitsets, words32, d_candidates, n_candidates, width, reinterpret_cast<unsigned long long *>(d_supports));
    CK(cudaGetLastError());
    return CPM_OK;
}

// periodic_counts of cupami/periodicFrequentPattern/_temporal.py:26-53, called
// by TemporalInput._evaluate (:156-165): exact supports and periodicities of
// every candidate (k_periodic without early stopping).
extern "C" int cpm_periodic_counts(cpm_ctx *ctx, const uint32_t *d_bitsets, uint64_t words32,
                                   const uint32_t *d_candidates, uint64_t n_candidates, uint32_t width,
                                   const int64_t *d_timestamps, uint64_t n_transactions, int64_t end,
                                   uint64_t *d_supports, int64_t *d_periods) {
    if (!ctx || (n_candidates && (!d_candidates || !d_supports || !d_periods || !width))) return CPM_EINVAL;
    if (n_candidates && n_transactions && (!d_bitsets || !d_timestamps)) return CPM_EINVAL;
    CK(cudaSetDevice(ctx->device));
    if (!n_candidates) return CPM_OK;
    // Rows past the bitsets' words hold no bits (the reference kernel scans
    // words32 words and skips rows >= n_transactions).
    const uint64_t rows = std::min<uint64_t>(n_transactions, words32 * 32);
    const uint32_t parts = periodic_parts(ctx, n_candidates, (rows + 31) / 32);
    DevScope ds(ctx);
    PSeg *seg = nullptr;
    if (parts > 1) CKR(ds.alloc(&seg, n_candidates * parts));
    uint64_t launches = 0;
    return periodic_launch<uint32_t, false>(ctx, parts, seg, d_bitsets, words32, d_candidates, nullptr, n_candidates,
                                            width, reinterpret_cast<const long long *>(d_timestamps), rows,
                                            (long long)end, 0, 0, reinterpret_cast<unsigned long long *>(d_supports),
                                            reinterpret_cast<long long *>(d_periods), nullptr, launches);
}

extern "C" int cpm_intersect_extensions(cpm_ctx *ctx, const uint32_t *d_prefix, const uint32_t *d_extensions,
                                        uint64_t words32, uint64_t n_extensions, uint32_t *d_out,
                                        uint64_t *d_supports) {
    if (!ctx || (n_extensions && (!d_prefix || !d_extensions || !d_out || !d_supports))) return CPM_EINVAL;
    CK(cudaSetDevice(ctx->device));
    if (!n_extensions) return CPM_OK;
    k_ref_intersect<<<(unsigned)((n_extensions * 32 + 255) / 256), 256, 0, ctx->stream>>>(
        d_prefix, d_extensions, words32, n_extensions, d_out, reinterpret_cast<unsigned long long *>(d_supports));
    CK(cudaGetLastError());
    return CPM_OK;
}

// ---------------------------------------------------------------------------
// learned cost model (scheduler)
// ---------------------------------------------------------------------------

extern "C" int cpm_costmodel_params(uint32_t *n_features, uint32_t *n_params) {
    if (n_features) *n_features = cm::NF;
    if (n_params) *n_params = cm::N_PARAMS;
    return CPM_OK;
}

extern "C" int cpm_costmodel_gradient(cpm_ctx *ctx, const float *params, const float *X, const float *y, uint64_t n,
                                      float *grad, float *loss) {
    if (!ctx || !params || !grad || (n && (!X || !y))) return CPM_EINVAL;
    CK(cudaSetDevice(ctx->device));
    DevScope ds(ctx);
    float *d_p = nullptr, *d_x = nullptr, *d_t = nullptr, *d_g = nullptr, *d_l = nullptr;
    CKR(ds.alloc(&d_p, cm::N_PARAMS));
    CKR(ds.alloc(&d_x, std::max<uint64_t>(1, n) * cm::NF));
    CKR(ds.alloc(&d_t, std::max<uint64_t>(1, n)));
    CKR(ds.alloc(&d_g, cm::TRAIN_COUNT));
    CKR(ds.alloc(&d_l, 1));
    std::vector<float> t(n);
    const float ysd = params[cm::OFF_YSD] != 0.f ? params[cm::OFF_YSD] : 1.f;
    for (uint64_t i = 0; i < n; ++i) t[i] = (y[i] - params[cm::OFF_YMU]) / ysd;
    CK(cudaMemcpyAsync(d_p, params, cm::N_PARAMS * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (n) {
        CK(cudaMemcpyAsync(d_x, X, n * cm::NF * 4, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(d_t, t.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
    }
    CK(cudaMemsetAsync(d_g, 0, cm::TRAIN_COUNT * 4, ctx->stream));
    CK(cudaMemsetAsync(d_l, 0, 4, ctx->stream));
    if (n) {
        k_mlp_backward<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(d_p, d_x, d_t, n, d_g, d_l);
        CK(cudaGetLastError());
    }
    std::vector<float> g(cm::TRAIN_COUNT);
    float l = 0.f;
    CK(cudaMemcpyAsync(g.data(), d_g, cm::TRAIN_COUNT * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&l, d_l, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // d/dtheta of (1 / 2n) sum (f - t)^2
    const float inv = n ? 1.f / (float)n : 0.f;
    for (int i = 0; i < cm::N_PARAMS; ++i) grad[i] = 0.f;
    for (int i = 0; i < cm::TRAIN_COUNT; ++i) grad[cm::TRAIN_FIRST + i] = g[i] * inv;
    if (loss) *loss = 0.5f * l * inv;
    return CPM_OK;
}

static uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static double gauss(uint64_t &s) {
    const double u1 = ((splitmix(s) >> 11) + 1.0) / 9007199254740993.0;
    const double u2 = (splitmix(s) >> 11) / 9007199254740992.0;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

extern "C" int cpm_costmodel_train(cpm_ctx *ctx, const float *X, const float *y, uint64_t n, uint32_t epochs,
                                   float lr, uint64_t seed, float *params, float *loss_history) {
    if (!ctx || !params || !n || !X || !y || !epochs) return CPM_EINVAL;
    CK(cudaSetDevice(ctx->device));
    // Standardisation from the training data; He-initialised weights.
    std::vector<float> P(cm::N_PARAMS, 0.f);
    for (int f = 0; f < cm::NF; ++f) {
        double m = 0, v = 0;
        for (uint64_t i = 0; i < n; ++i) m += X[i * cm::NF + f];
        m /= n;
        for (uint64_t i = 0; i < n; ++i) v += (X[i * cm::NF + f] - m) * (X[i * cm::NF + f] - m);
        const double sd = std::sqrt(v / n);
        P[cm::OFF_MU + f] = (float)m;
        P[cm::OFF_IS + f] = (float)(sd > 1e-6 ? 1.0 / sd : 0.0);
    }
    double ym = 0, yv = 0;
    for (uint64_t i = 0; i < n; ++i) ym += y[i];
    ym /= n;
    for (uint64_t i = 0; i < n; ++i) yv += (y[i] - ym) * (y[i] - ym);
    const double ysd = std::max(std::sqrt(yv / n), 1e-6);
    P[cm::OFF_YMU] = (float)ym;
    P[cm::OFF_YSD] = (float)ysd;
    uint64_t rng = seed * 0x2545F4914F6CDD1Dull + 1;
    for (int i = 0; i < cm::H * cm::NF; ++i) P[cm::OFF_W1 + i] = (float)(gauss(rng) * std::sqrt(2.0 / cm::NF));
    for (int i = 0; i < cm::H; ++i) P[cm::OFF_W2 + i] = (float)(gauss(rng) * std::sqrt(1.0 / cm::H));
    std::vector<float> t(n);
    for (uint64_t i = 0; i < n; ++i) t[i] = (float)((y[i] - ym) / ysd);
    DevScope ds(ctx);
    float *d_p = nullptr, *d_x = nullptr, *d_t = nullptr, *d_g = nullptr, *d_m1 = nullptr, *d_m2 = nullptr,
          *d_l = nullptr;
    CKR(ds.alloc(&d_p, cm::N_PARAMS));
    CKR(ds.alloc(&d_x, n * cm::NF));
    CKR(ds.alloc(&d_t, n));
    CKR(ds.alloc(&d_g, cm::TRAIN_COUNT));
    CKR(ds.alloc(&d_m1, cm::TRAIN_COUNT));
    CKR(ds.alloc(&d_m2, cm::TRAIN_COUNT));
    CKR(ds.alloc(&d_l, epochs));
    CK(cudaMemcpyAsync(d_p, P.data(), cm::N_PARAMS * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_x, X, n * cm::NF * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_t, t.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(d_m1, 0, cm::TRAIN_COUNT * 4, ctx->stream));
    CK(cudaMemsetAsync(d_m2, 0, cm::TRAIN_COUNT * 4, ctx->stream));
    CK(cudaMemsetAsync(d_l, 0, epochs * 4, ctx->stream));
    const unsigned blocks = (unsigned)((n + 255) / 256);
    for (uint32_t e = 0; e < epochs; ++e) {
        CK(cudaMemsetAsync(d_g, 0, cm::TRAIN_COUNT * 4, ctx->stream));
        k_mlp_backward<<<blocks, 256, 0, ctx->stream>>>(d_p, d_x, d_t, n, d_g, d_l + e);
        k_adam<<<(cm::TRAIN_COUNT + 255) / 256, 256, 0, ctx->stream>>>(d_p, d_g, d_m1, d_m2, lr, 1.f / (float)n,
                                                                     (int)e + 1);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(params, d_p, cm::N_PARAMS * 4, cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<float> lh(epochs);
    CK(cudaMemcpyAsync(lh.data(), d_l, epochs * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (loss_history)
        for (uint32_t e = 0; e < epochs; ++e) loss_history[e] = 0.5f * lh[e] / (float)n;
    return CPM_OK;
}

extern "C" int cpm_costmodel_predict(cpm_ctx *ctx, const float *params, const float *X, uint64_t n, float *y) {
    if (!ctx || !params || (n && (!X || !y))) return CPM_EINVAL;
    if (!n) return CPM_OK;
    CK(cudaSetDevice(ctx->device));
    DevScope ds(ctx);
    float *d_p = nullptr, *d_x = nullptr, *d_y = nullptr;
    CKR(ds.alloc(&d_p, cm::N_PARAMS));
    CKR(ds.alloc(&d_x, n * cm::NF));
    CKR(ds.alloc(&d_y, n));
    CK(cudaMemcpyAsync(d_p, params, cm::N_PARAMS * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_x, X, n * cm::NF * 4, cudaMemcpyHostToDevice, ctx->stream));
    k_mlp_forward<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(d_p, d_x, n, d_y, 1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(y, d_y, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CPM_OK;
}

extern "C" int cpm_costmodel_set(cpm_ctx *ctx, const float *params) {
    if (!ctx) return CPM_EINVAL;
    if (!params) ctx->model.clear();
    else ctx->model.assign(params, params + cm::N_PARAMS);
    return CPM_OK;
}

extern "C" int cpm_result_trace(const cpm_result *res, float *X, float *y, uint64_t *n) {
    if (!res || !n) return CPM_EINVAL;
    *n = res->trace_y.size();
    if (X) std::copy(res->trace_x.begin(), res->trace_x.end(), X);
    if (y) std::copy(res->trace_y.begin(), res->trace_y.end(), y);
    return CPM_OK;
}

// ---------------------------------------------------------------------------
// Eclat with no device allocation
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory when they mine: their device
// memory belongs to another runtime's pool, or their process forbids
// allocation after start-up.  cpm_mine_eclat_noalloc takes the tidsets and the
// output arrays from the caller and keeps every intermediate buffer (frequent
// list, pair Gram, class tables, work queue, child tidsets) in the one static
// device array below, CPM_NOALLOC_SCRATCH_BYTES long, which every GPU that
// loads this library holds until the process exits.

static __device__ __align__(256) unsigned char g_noalloc_scratch[CPM_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per device.  In host code the symbol
// name is only a host-side stand-in, so the address must come from
// cudaGetSymbolAddress with the device current.  Resolved on the first call
// for each device, which is why that first call should come before any
// stream capture.
static std::mutex g_noalloc_mutex;
static unsigned char *g_noalloc_addr[256] = {};

static int noalloc_scratch(cpm_ctx *ctx, unsigned char **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (ctx->device < 0 || ctx->device >= 256) return set_err(ctx, CPM_EINVAL, "device index out of range");
    if (!g_noalloc_addr[ctx->device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return set_err(ctx, CPM_ECUDA, "cudaGetSymbolAddress of the static scratch failed: %s",
                           cudaGetErrorString(e));
        }
        g_noalloc_addr[ctx->device] = static_cast<unsigned char *>(p);
    }
    *out = g_noalloc_addr[ctx->device];
    return CPM_OK;
}

// 256-byte aligned pieces of the static scratch.
struct NoallocCarve {
    unsigned char *base;
    uint64_t used;
    uint64_t left() const {
        const uint64_t off = (used + 255) & ~255ull;
        return off >= CPM_NOALLOC_SCRATCH_BYTES ? 0 : CPM_NOALLOC_SCRATCH_BYTES - off;
    }
    template <class T>
    T *take(uint64_t count) {
        const uint64_t off = (used + 255) & ~255ull;
        const uint64_t bytes = std::max<uint64_t>(1, count) * sizeof(T);
        if (off > CPM_NOALLOC_SCRATCH_BYTES || bytes > CPM_NOALLOC_SCRATCH_BYTES - off) return nullptr;
        used = off + bytes;
        return reinterpret_cast<T *>(base + off);
    }
};

extern "C" int cpm_mine_eclat_noalloc(cpm_ctx *ctx, const uint64_t *d_bits, uint64_t stride, uint32_t n_items,
                                      uint64_t n_transactions, int64_t min_sup, const cpm_opts *opts,
                                      uint32_t *d_parent, uint32_t *d_item, uint32_t *d_support,
                                      uint64_t capacity, uint64_t *n_patterns) {
    if (!ctx || !n_patterns) return CPM_EINVAL;
    *n_patterns = 0;
    if ((n_items && !d_bits) || (capacity && (!d_parent || !d_item || !d_support)))
        return set_err(ctx, CPM_EINVAL, "null input or output pointer");
    if (n_items == 0) return CPM_OK;  // an empty database has no patterns, as with cpm_mine
    if (stride < 2 || (stride & 1) || (reinterpret_cast<uintptr_t>(d_bits) & 15))
        return set_err(ctx, CPM_EINVAL, "tidset rows need an even stride and a 16-byte aligned base");
    if (n_transactions > stride * 64) return set_err(ctx, CPM_EINVAL, "stride too small for the transactions");
    CK(cudaSetDevice(ctx->device));
    unsigned char *base = nullptr;
    CKR(noalloc_scratch(ctx, &base));
    NoallocCarve carve{base, 0};
    const long long ms = (long long)std::max<int64_t>(std::min<int64_t>(min_sup, (int64_t)1 << 40), -1);
    const unsigned long long limit_mib = CPM_NOALLOC_SCRATCH_BYTES >> 20;
    uint32_t *d_item_sup = carve.take<uint32_t>(n_items);
    uint32_t *d_freq = carve.take<uint32_t>(n_items);
    uint32_t *d_count = carve.take<uint32_t>(1);
    DeepState *d_st = carve.take<DeepState>(1);
    if (!d_item_sup || !d_freq || !d_count || !d_st)
        return set_err(ctx, CPM_EINVAL, "%u items exceed the %llu MiB static scratch", n_items, limit_mib);
    // Singletons.
    if (n_items) {
        k_item_support<<<(unsigned)(((uint64_t)n_items * 32 + 255) / 256), 256, 0, ctx->stream>>>(
            d_bits, stride, n_items, d_item_sup);
        CK(cudaGetLastError());
    }
    CK(cudaMemsetAsync(d_count, 0, 4, ctx->stream));
    if (n_items) {
        k_compact_frequent<<<1, 1024, 0, ctx->stream>>>(d_item_sup, n_items, ms, d_freq, d_count);
        CK(cudaGetLastError());
    }
    uint32_t F = 0;
    CK(cudaMemcpyAsync(&F, d_count, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (F > capacity)
        return set_err(ctx, CPM_EOVERFLOW, "output capacity %llu is below the %u frequent items",
                       (unsigned long long)capacity, F);
    if (F) {
        k_emit_singletons<<<(F + 255) / 256, 256, 0, ctx->stream>>>(d_freq, F, d_item_sup, d_parent, d_item,
                                                                    d_support);
        CK(cudaGetLastError());
    }
    if (F < 2) {
        CK(cudaStreamSynchronize(ctx->stream));
        *n_patterns = F;
        return CPM_OK;
    }
    // Pair level on the CUDA cores (the same Gram and threshold as cpm_mine).
    uint32_t *d_C = carve.take<uint32_t>((uint64_t)F * F);
    uint32_t *d_cnt = carve.take<uint32_t>(F);
    uint64_t *d_off = carve.take<uint64_t>((uint64_t)F + 1);
    if (!d_C || !d_cnt || !d_off)
        return set_err(ctx, CPM_EINVAL, "%u frequent items need a %llu-byte pair matrix, beyond the %llu MiB static "
                       "scratch", F, (unsigned long long)F * F * 4, limit_mib);
    CK(cudaMemsetAsync(d_C, 0, (size_t)F * F * 4, ctx->stream));
    {
        const uint32_t nt = (F + 63) / 64;
        const uint32_t tiles = nt * (nt + 1) / 2;
        uint64_t ksplit = std::max<uint64_t>(1, (uint64_t)ctx->sms * 4 / tiles);
        ksplit = std::min<uint64_t>(ksplit, std::max<uint64_t>(1, stride / 64));
        const uint64_t k_chunk = ((stride + ksplit - 1) / ksplit + 15) / 16 * 16;
        ksplit = (stride + k_chunk - 1) / k_chunk;
        k_gram_simt<<<dim3(tiles, (unsigned)ksplit), 256, 0, ctx->stream>>>(d_bits, stride, d_freq, F, nt, k_chunk,
                                                                              d_C);
        CK(cudaGetLastError());
    }
    k_pair_count<<<(unsigned)(((uint64_t)F * 32 + 255) / 256), 256, 0, ctx->stream>>>(d_C, F, ms, d_cnt);
    CK(cudaGetLastError());
    std::vector<uint32_t> cnt(F);
    std::vector<uint64_t> off(F + 1, 0);
    CK(cudaMemcpyAsync(cnt.data(), d_cnt, (size_t)F * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (uint32_t i = 0; i < F; ++i) off[i + 1] = off[i] + cnt[i];
    const uint64_t P2 = off[F];
    if (F + P2 > capacity)
        return set_err(ctx, CPM_EOVERFLOW, "output capacity %llu is below the %llu singletons and pairs",
                       (unsigned long long)capacity, (unsigned long long)(F + P2));
    std::vector<uint32_t> roots;
    for (uint32_t i = 0; i < F; ++i)
        if (cnt[i] >= 2) roots.push_back(i);
    std::stable_sort(roots.begin(), roots.end(), [&](uint32_t a, uint32_t b) { return cnt[a] > cnt[b]; });
    std::vector<unsigned long long> init;
    for (size_t k = 0; k < roots.size(); ++k)
        for (uint32_t p = 0; p + 1 < cnt[roots[k]]; ++p) init.push_back(((unsigned long long)k << 32) | p);
    std::stable_sort(init.begin(), init.end(), [&](unsigned long long a, unsigned long long b) {
        return cnt[roots[a >> 32]] - (uint32_t)a > cnt[roots[b >> 32]] - (uint32_t)b;
    });
    // Deep-level tables from what is left: the queue and frame tables are
    // bounded by the output capacity, members and child tidsets share the rest.
    const uint64_t rest = carve.left();
    const uint64_t frames_cap = std::min<uint64_t>(capacity + roots.size(), rest / 16 / sizeof(DFrame)) + 1;
    const uint64_t queue_cap = std::min<uint64_t>(capacity + init.size(), rest / 16 / 8) + 1;
    DFrame *d_frames = carve.take<DFrame>(frames_cap);
    unsigned long long *d_queue = carve.take<unsigned long long>(queue_cap);
    unsigned long long *d_root_cost = carve.take<unsigned long long>(roots.size());
    const uint64_t members_cap = std::max<uint64_t>(P2, carve.left() / 4 / 16);
    uint32_t *d_mem_pat = carve.take<uint32_t>(members_cap);
    uint32_t *d_mem_item = carve.take<uint32_t>(members_cap);
    const uint64_t **d_mem_bits = carve.take<const uint64_t *>(members_cap);
    const uint64_t arena_slots = d_mem_bits ? carve.left() / (stride * 8) : 0;
    uint64_t *d_arena = arena_slots ? carve.take<uint64_t>(arena_slots * stride) : nullptr;
    if (!d_frames || !d_queue || !d_root_cost || !d_mem_pat || !d_mem_item || !d_mem_bits || !d_arena ||
        init.size() > queue_cap || roots.size() > frames_cap || arena_slots < 64)
        return set_err(ctx, CPM_EINVAL, "%llu-word tidsets with %llu pairs exceed the %llu MiB static scratch",
                       (unsigned long long)stride, (unsigned long long)P2, limit_mib);
    CK(cudaMemcpyAsync(d_off, off.data(), (F + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    k_pair_emit<<<(unsigned)(((uint64_t)F * 32 + 255) / 256), 256, 0, ctx->stream>>>(
        d_C, F, ms, d_freq, d_off, d_bits, stride, d_parent, d_item, d_support, d_mem_pat, d_mem_item, d_mem_bits);
    CK(cudaGetLastError());
    if (roots.empty()) {
        CK(cudaStreamSynchronize(ctx->stream));
        *n_patterns = F + P2;
        return CPM_OK;
    }
    std::vector<uint32_t> hfreq(F);
    CK(cudaMemcpyAsync(hfreq.data(), d_freq, (size_t)F * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<DFrame> frames(roots.size());
    for (size_t k = 0; k < roots.size(); ++k) {
        frames[k].mask = d_bits + (uint64_t)hfreq[roots[k]] * stride;
        frames[k].mem_off = off[roots[k]];
        frames[k].m = cnt[roots[k]];
        frames[k].root = (uint32_t)k;
        frames[k].stride = (uint32_t)stride;
        frames[k].db = 0;
        frames[k].minsup = ms;
    }
    // Every call shares the scratch: reset what the kernel expects cleared.
    CK(cudaMemcpyAsync(d_frames, frames.data(), frames.size() * sizeof(DFrame), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(d_queue, 0xff, queue_cap * 8, ctx->stream));
    CK(cudaMemcpyAsync(d_queue, init.data(), init.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(d_root_cost, 0, std::max<size_t>(1, roots.size()) * 8, ctx->stream));
    DeepState hs{};
    hs.q_tail = init.size();
    hs.pending = init.size();
    hs.n_patterns = F + P2;
    hs.n_frames = roots.size();
    hs.n_members = P2;
    CK(cudaMemcpyAsync(d_st, &hs, sizeof hs, cudaMemcpyHostToDevice, ctx->stream));
    DeepParams P;
    P.frames = d_frames; P.frames_cap = frames_cap;
    P.mem_pat = d_mem_pat; P.mem_item = d_mem_item; P.mem_bits = d_mem_bits; P.members_cap = members_cap;
    P.queue = d_queue; P.queue_cap = queue_cap;
    P.arena = d_arena; P.arena_words = arena_slots * stride;
    P.pat_parent = d_parent; P.pat_item = d_item; P.pat_sup = d_support; P.pat_db = nullptr; P.pat_cap = capacity;
    P.root_cost = d_root_cost; P.st = d_st; P.max_stride = stride;
    P.spin_limit = opts && opts->spin_limit ? opts->spin_limit : (1ull << 26);
    P.cta_time = nullptr;
    P.unit_log = nullptr; P.unit_log_cap = 0;
    P.shallow = 0;
    P.balance = 0;
    P.prefetch = 0;
    P.lists = 0;
    P.local_max = 0; P.lq = nullptr; P.lq_cap = 0; P.dir_off = 0;  // no projection: one launch, fixed scratch
    P.h_off = nullptr; P.h_rows = nullptr; P.h_fidx = nullptr; P.h_F = 0; P.h_cost = 0.f;
    P.h_scratch = nullptr; P.h_scratch_words = 0; P.h_table_off = 0;
    P.root_frames = 0; P.defer_words = 0; P.defer_members = 0; P.defer_frames = 0; P.defer_queue = 0;
    P.root_key = nullptr; P.top_frames = 0; P.keys_in_words = 0; P.admit_words = 0;
    P.deferred = nullptr; P.deferred_cap = 0;
    // Each warp keeps one scratch tidset: leave at least half the arena to children.
    const size_t prefix_bytes = stride * 8;
    const bool smem_prefix = prefix_bytes <= DEEP_SMEM_PREFIX_MAX;
    int per_sm = 1;
    if (smem_prefix) {
        // cpm_init already allows k_deep<true> DEEP_SMEM_PREFIX_MAX bytes of dynamic shared memory;
        // the attribute is process-wide, so it is not touched here.
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_deep<true>, 256, prefix_bytes));
    } else {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_deep<false>, 256, 0));
    }
    const uint64_t grid = std::max<uint64_t>(
        1, std::min<uint64_t>((uint64_t)ctx->sms * std::max(1, per_sm), arena_slots / 16));
    if (smem_prefix) k_deep<true><<<(unsigned)grid, 256, prefix_bytes, ctx->stream>>>(P);
    else k_deep<false><<<(unsigned)grid, 256, 0, ctx->stream>>>(P);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&hs, d_st, sizeof hs, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (hs.error & DEEP_ERR_SPIN)
        return set_err(ctx, CPM_ETIMEOUT, "deep-level kernel wait ran out of spins (limit %llu)",
                       (unsigned long long)P.spin_limit);
    if (hs.error & DEEP_ERR_PATTERNS)
        return set_err(ctx, CPM_EOVERFLOW, "output capacity %llu is below the number of patterns",
                       (unsigned long long)capacity);
    if (hs.error)
        return set_err(ctx, CPM_EOVERFLOW, "the search outgrew the %llu MiB static scratch (error 0x%x)", limit_mib,
                       hs.error);
    *n_patterns = hs.n_patterns;
    return CPM_OK;
}

// ---------------------------------------------------------------------------
// delimited text of integer baskets, parsed on the device
// ---------------------------------------------------------------------------

struct cpm_csr {
    std::vector<uint64_t> offsets;  // n_rows + 1
    std::vector<uint32_t> ids;
};

extern "C" int cpm_parse_int_text(cpm_ctx *ctx, const char *text, uint64_t n_bytes, int32_t sep, cpm_csr **out) {
    if (!ctx || !out) return CPM_EINVAL;
    *out = nullptr;
    if (n_bytes && !text) return set_err(ctx, CPM_EINVAL, "null text");
    if (sep < 1 || sep > 127 || (sep >= '0' && sep <= '9') || sep == '\n')
        return set_err(ctx, CPM_EINVAL, "the separator must be one ASCII character other than a digit or newline");
    CK(cudaSetDevice(ctx->device));
    std::unique_ptr<cpm_csr> csr(new cpm_csr());
    // Lines: one per newline, plus a last one when the text does not end in a newline.
    const bool tail = n_bytes && text[n_bytes - 1] != '\n';
    if (n_bytes == 0) {
        csr->offsets.assign(1, 0);
        *out = csr.release();
        return CPM_OK;
    }
    DevScope ds(ctx);
    unsigned char *d_text = nullptr;
    uint32_t *d_flag = nullptr;
    uint64_t *d_pos = nullptr;
    unsigned int *d_reject = nullptr;
    CKR(ds.alloc(&d_text, n_bytes));
    CKR(ds.alloc(&d_flag, n_bytes));
    CKR(ds.alloc(&d_pos, n_bytes));
    CKR(ds.alloc(&d_reject, 1));
    CKR(stage_upload(ctx, {{d_text, {text, n_bytes}}}));
    CK(cudaMemsetAsync(d_reject, 0, 4, ctx->stream));
    const unsigned grid = (unsigned)std::min<uint64_t>((n_bytes + 255) / 256, (uint64_t)ctx->sms * 32);
    k_text_newlines<<<grid, 256, 0, ctx->stream>>>(d_text, n_bytes, d_flag);
    CK(cudaGetLastError());
    uint64_t n_nl = 0;
    CKR(scan_u32(ctx, ds, d_flag, d_pos, n_bytes, &n_nl));
    const uint64_t n_lines = n_nl + (tail ? 1 : 0);
    uint64_t *d_nl = nullptr, *d_off = nullptr;
    uint32_t *d_cnt = nullptr;
    CKR(ds.alloc(&d_nl, std::max<uint64_t>(1, n_nl)));
    CKR(ds.alloc(&d_cnt, std::max<uint64_t>(1, n_lines)));
    CKR(ds.alloc(&d_off, n_lines + 1));
    k_text_scatter<<<grid, 256, 0, ctx->stream>>>(d_flag, d_pos, n_bytes, d_nl);
    CK(cudaGetLastError());
    const unsigned lgrid = (unsigned)((n_lines + 255) / 256);
    if (n_lines) {
        k_text_lines<false><<<lgrid, 256, 0, ctx->stream>>>(d_text, n_bytes, d_nl, n_nl, n_lines, (unsigned char)sep,
                                                            d_cnt, nullptr, nullptr, d_reject);
        CK(cudaGetLastError());
    }
    uint64_t nnz = 0;
    CKR(scan_u32(ctx, ds, d_cnt, d_off, n_lines, &nnz));
    unsigned int reject = 0;
    CK(cudaMemcpyAsync(&reject, d_reject, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (reject)
        return set_err(ctx, CPM_EINVAL, "the text is not unquoted integer baskets (canonical ids up to 4294967295, "
                       "one separator between tokens, ASCII only)");
    uint32_t *d_ids = nullptr;
    CKR(ds.alloc(&d_ids, std::max<uint64_t>(1, nnz)));
    if (n_lines && nnz) {
        k_text_lines<true><<<lgrid, 256, 0, ctx->stream>>>(d_text, n_bytes, d_nl, n_nl, n_lines, (unsigned char)sep,
                                                           nullptr, d_off, d_ids, d_reject);
        CK(cudaGetLastError());
    }
    csr->offsets.resize(n_lines + 1);
    csr->ids.resize(nnz);
    if (n_lines) CK(cudaMemcpyAsync(csr->offsets.data(), d_off, n_lines * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (nnz) CK(cudaMemcpyAsync(csr->ids.data(), d_ids, nnz * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    csr->offsets[n_lines] = nnz;
    *out = csr.release();
    return CPM_OK;
}

extern "C" int cpm_csr_size(const cpm_csr *csr, uint64_t *n_rows, uint64_t *nnz) {
    if (!csr || !n_rows || !nnz) return CPM_EINVAL;
    *n_rows = csr->offsets.size() - 1;
    *nnz = csr->ids.size();
    return CPM_OK;
}

extern "C" int cpm_csr_copy(const cpm_csr *csr, uint64_t *offsets, uint32_t *ids) {
    if (!csr || !offsets || (!ids && !csr->ids.empty())) return CPM_EINVAL;
    memcpy(offsets, csr->offsets.data(), csr->offsets.size() * 8);
    if (!csr->ids.empty()) memcpy(ids, csr->ids.data(), csr->ids.size() * 4);
    return CPM_OK;
}

extern "C" void cpm_csr_free(cpm_csr *csr) { delete csr; }

// ---------------------------------------------------------------------------
// pattern keys for the Python dict (host only)
// ---------------------------------------------------------------------------

// Pattern k's key is its items' labels joined by `sep`; keys are written one
// after another, each followed by `end`, into out (cap bytes).  *len gets the
// bytes needed; with out null (or cap too small) nothing is written, so a
// first call sizes the buffer.  Two passes over the patterns (key lengths,
// then keys at their prefix-sum offsets), both parallel.
extern "C" int cpm_join_labels(const uint64_t *offsets, const uint32_t *items, uint64_t n_patterns,
                               const char *labels, const uint64_t *label_off, uint32_t n_labels, char sep, char end,
                               char *out, uint64_t cap, uint64_t *len) {
    if (!len || (n_patterns && (!offsets || (!items && offsets[n_patterns]))) || (n_labels && (!labels || !label_off)))
        return CPM_EINVAL;
    *len = 0;
    if (!n_patterns) return CPM_OK;
    std::vector<uint64_t> at(n_patterns + 1, 0);
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t k = 0; k < (int64_t)n_patterns; ++k) {
        uint64_t l = 1;  // `end`
        const uint64_t a = offsets[k], b = offsets[k + 1];
        if (b < a) { bad = 1; continue; }
        for (uint64_t j = a; j < b; ++j) {
            const uint32_t c = items[j];
            if (c >= n_labels) { bad = 1; break; }
            l += label_off[c + 1] - label_off[c] + (j > a ? 1 : 0);
        }
        at[k + 1] = l;
    }
    if (bad) return CPM_EINVAL;
    for (uint64_t k = 0; k < n_patterns; ++k) at[k + 1] += at[k];
    *len = at[n_patterns];
    if (!out || cap < *len) return CPM_OK;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)n_patterns; ++k) {
        char *p = out + at[k];
        for (uint64_t j = offsets[k]; j < offsets[k + 1]; ++j) {
            if (j > offsets[k]) *p++ = sep;
            const uint32_t c = items[j];
            const uint64_t n = label_off[c + 1] - label_off[c];
            memcpy(p, labels + label_off[c], n);
            p += n;
        }
        *p = end;
    }
    return CPM_OK;
}
