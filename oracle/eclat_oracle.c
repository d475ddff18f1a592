/*
 * CPU restatement of cuPAMI's vertical-bitset miners -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the CUDA path, never part of it: only the test
 * suite, the smoke check and the benchmark's CPU-baseline leg load it.
 *
 * What it restates (reference paths are relative to the cuPAMI project):
 *   - bitset packing            cupami/frequentPattern/_bitsets.py:20-28, 91-100
 *   - support counting          cupami/frequentPattern/_bitsets.py:30-53, 103-113
 *   - retained intersections    cupami/frequentPattern/_bitsets.py:55-77, 116-125
 *   - Eclat driver              cupami/frequentPattern/cuEclat.py:168-203
 *   - Eclat class search        cupami/frequentPattern/cuEclat.py:211-245
 *   - Apriori driver            cupami/frequentPattern/cuApriori.py:501-535
 *   - Apriori candidates        cupami/frequentPattern/cuApriori.py:473-492
 *   - row numbering             cupami/frequentPattern/cuApriori.py:397-404
 *     (row = position among non-empty baskets; columns are given already
 *      mapped to the lexicographic order of the string labels)
 *
 * Patterns are emitted in exactly the order the reference drivers insert them
 * into their result dictionary, so the order can be compared as well as the
 * set.  Bitsets use 64-bit words here (the reference uses 32-bit words); the
 * word width changes no support count.
 *
 * Parity pin: the Python wrapper checks this code against golden vectors that
 * were produced by running the reference drivers themselves (tests/golden).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    uint64_t n;          /* patterns */
    uint64_t cap;
    uint64_t n_items;    /* total item slots */
    uint64_t items_cap;
    uint64_t *offsets;   /* n + 1 */
    uint32_t *items;
    uint64_t *supports;
} oracle_result;

static int res_push(oracle_result *r, const uint32_t *pat, uint32_t len, uint64_t sup) {
    if (r->n + 1 >= r->cap) {
        uint64_t nc = r->cap ? r->cap * 2 : 1024;
        uint64_t *no = realloc(r->offsets, (nc + 1) * sizeof(uint64_t));
        uint64_t *ns = realloc(r->supports, nc * sizeof(uint64_t));
        if (!no || !ns) return -1;
        r->offsets = no; r->supports = ns; r->cap = nc;
    }
    if (r->n_items + len > r->items_cap) {
        uint64_t nc = r->items_cap ? r->items_cap * 2 : 4096;
        while (nc < r->n_items + len) nc *= 2;
        uint32_t *ni = realloc(r->items, nc * sizeof(uint32_t));
        if (!ni) return -1;
        r->items = ni; r->items_cap = nc;
    }
    if (r->n == 0) r->offsets[0] = 0;
    memcpy(r->items + r->n_items, pat, len * sizeof(uint32_t));
    r->n_items += len;
    r->supports[r->n] = sup;
    r->n++;
    r->offsets[r->n] = r->n_items;
    return 0;
}

void oracle_free(oracle_result *r) {
    if (!r) return;
    free(r->offsets); free(r->items); free(r->supports); free(r);
}

uint64_t oracle_count(const oracle_result *r) { return r->n; }
uint64_t oracle_item_slots(const oracle_result *r) { return r->n_items; }

void oracle_copy(const oracle_result *r, uint64_t *offsets, uint32_t *items, uint64_t *supports) {
    if (r->n) {
        memcpy(offsets, r->offsets, (r->n + 1) * sizeof(uint64_t));
        memcpy(items, r->items, r->n_items * sizeof(uint32_t));
        memcpy(supports, r->supports, r->n * sizeof(uint64_t));
    } else {
        offsets[0] = 0;
    }
}

/* Packs the CSR into item-major 64-bit bitsets; returns the row count used. */
static uint64_t *pack(uint64_t n_rows, uint32_t n_items, const uint64_t *offsets,
                      const uint32_t *cols, uint64_t *n_tx, uint64_t *words_out) {
    uint64_t n = 0;
    for (uint64_t r = 0; r < n_rows; ++r) n += offsets[r + 1] > offsets[r];
    uint64_t words = (n + 63) / 64;
    uint64_t *bits = calloc((size_t)n_items * (words ? words : 1), sizeof(uint64_t));
    if (!bits) return NULL;
    uint64_t row = 0;
    for (uint64_t r = 0; r < n_rows; ++r) {
        if (offsets[r + 1] == offsets[r]) continue;
        for (uint64_t k = offsets[r]; k < offsets[r + 1]; ++k)
            bits[(uint64_t)cols[k] * words + row / 64] |= 1ull << (row % 64);
        ++row;
    }
    *n_tx = n;
    *words_out = words;
    return bits;
}

static uint64_t popc_and(const uint64_t *a, const uint64_t *b, uint64_t words) {
    uint64_t s = 0;
    for (uint64_t w = 0; w < words; ++w) s += (uint64_t)__builtin_popcountll(a[w] & b[w]);
    return s;
}

static uint64_t popc_and_store(const uint64_t *a, const uint64_t *b, uint64_t *out, uint64_t words) {
    uint64_t s = 0;
    for (uint64_t w = 0; w < words; ++w) {
        uint64_t v = a[w] & b[w];
        out[w] = v;
        s += (uint64_t)__builtin_popcountll(v);
    }
    return s;
}

/* Support passes when support >= minsup; a minsup <= 0 lets every candidate
 * through, zero supports included, as the reference's comparison does. */
#define PASSES(s, ms) ((int64_t)(s) >= (ms))

typedef struct {
    uint32_t *prefix; uint32_t plen;
    uint32_t *labels; uint32_t m;
    uint64_t *vert;   /* m * words */
    uint32_t pos;
} frame;

oracle_result *oracle_eclat(uint64_t n_rows, uint32_t n_items, const uint64_t *offsets,
                            const uint32_t *cols, int64_t minsup, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    oracle_result *res = calloc(1, sizeof(*res));
    if (!res) return NULL;
    uint64_t n, words;
    uint64_t *bits = pack(n_rows, n_items, offsets, cols, &n, &words);
    if (!bits && n_items) { oracle_free(res); return NULL; }
    uint32_t *frequent = malloc((n_items + 1) * sizeof(uint32_t));
    uint32_t nf = 0;
    for (uint32_t i = 0; i < n_items; ++i) {
        uint64_t s = popc_and(bits + (uint64_t)i * words, bits + (uint64_t)i * words, words);
        if (PASSES(s, minsup)) {
            frequent[nf++] = i;
            res_push(res, &i, 1, s);
        }
    }
    /* Pair level (cuEclat.py:183-193): combinations(frequent, 2) in order. */
    uint64_t *pair_sup = malloc(((uint64_t)nf * nf + 1) * sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t a = 0; a < (int64_t)nf; ++a)
        for (uint32_t b = (uint32_t)a + 1; b < nf; ++b)
            pair_sup[(uint64_t)a * nf + b] = popc_and(bits + (uint64_t)frequent[a] * words,
                                                      bits + (uint64_t)frequent[b] * words, words);
    uint32_t *ext_count = calloc(nf + 1, sizeof(uint32_t));
    for (uint32_t a = 0; a < nf; ++a)
        for (uint32_t b = a + 1; b < nf; ++b) {
            uint64_t s = pair_sup[(uint64_t)a * nf + b];
            if (PASSES(s, minsup)) {
                uint32_t pat[2] = {frequent[a], frequent[b]};
                res_push(res, pat, 2, s);
                ext_count[a]++;
            }
        }
    /* Classes in first-appearance order of their left item (cuEclat.py:195-200). */
    uint32_t *pat = malloc((nf + 2) * sizeof(uint32_t));
    frame *stack = malloc((nf + 2) * sizeof(frame));
    for (uint32_t a = 0; a < nf; ++a) {
        if (ext_count[a] < 2) continue;
        uint32_t m = ext_count[a];
        frame f0;
        f0.plen = 1;
        f0.prefix = malloc(sizeof(uint32_t));
        f0.prefix[0] = frequent[a];
        f0.labels = malloc(m * sizeof(uint32_t));
        f0.vert = malloc((uint64_t)m * (words ? words : 1) * sizeof(uint64_t));
        f0.m = 0;
        f0.pos = 0;
        for (uint32_t b = a + 1; b < nf; ++b)
            if (PASSES(pair_sup[(uint64_t)a * nf + b], minsup)) f0.labels[f0.m++] = frequent[b];
#pragma omp parallel for
        for (int64_t e = 0; e < (int64_t)m; ++e)
            for (uint64_t w = 0; w < words; ++w)
                f0.vert[(uint64_t)e * words + w] =
                    bits[(uint64_t)f0.labels[e] * words + w] & bits[(uint64_t)frequent[a] * words + w];
        int depth = 0;
        stack[depth++] = f0;
        /* Explicit DFS (cuEclat.py:211-245). */
        while (depth) {
            frame *f = &stack[depth - 1];
            if (f->m < 2 || f->pos >= f->m - 1) {
                free(f->prefix); free(f->labels); free(f->vert);
                --depth;
                continue;
            }
            uint32_t p = f->pos++;
            uint32_t cnt = f->m - p - 1;
            uint64_t *child = malloc((uint64_t)cnt * (words ? words : 1) * sizeof(uint64_t));
            uint64_t *sup = malloc((cnt + 1) * sizeof(uint64_t));
            const uint64_t *pre = f->vert + (uint64_t)p * words;
#pragma omp parallel for schedule(static)
            for (int64_t q = 0; q < (int64_t)cnt; ++q)
                sup[q] = popc_and_store(pre, f->vert + (uint64_t)(p + 1 + q) * words,
                                        child + (uint64_t)q * words, words);
            uint32_t kept = 0;
            memcpy(pat, f->prefix, f->plen * sizeof(uint32_t));
            pat[f->plen] = f->labels[p];
            for (uint32_t q = 0; q < cnt; ++q) {
                if (!PASSES(sup[q], minsup)) continue;
                pat[f->plen + 1] = f->labels[p + 1 + q];
                res_push(res, pat, f->plen + 2, sup[q]);
                if (kept != q) memmove(child + (uint64_t)kept * words, child + (uint64_t)q * words,
                                       words * sizeof(uint64_t));
                sup[kept] = q;  /* remember which label survived */
                kept++;
            }
            if (kept > 1) {
                frame c;
                c.plen = f->plen + 1;
                c.prefix = malloc(c.plen * sizeof(uint32_t));
                memcpy(c.prefix, f->prefix, f->plen * sizeof(uint32_t));
                c.prefix[f->plen] = f->labels[p];
                c.m = kept;
                c.labels = malloc(kept * sizeof(uint32_t));
                for (uint32_t k = 0; k < kept; ++k) c.labels[k] = f->labels[p + 1 + sup[k]];
                c.vert = child;
                c.pos = 0;
                stack[depth++] = c;  /* f may move; not used after this point */
            } else {
                free(child);
            }
            free(sup);
        }
    }
    free(stack); free(pat); free(ext_count); free(pair_sup); free(frequent); free(bits);
    return res;
}

/* ---- Apriori (cuApriori.py:473-535) ---------------------------------------- */

typedef struct { uint32_t k; uint64_t n; uint32_t *pats; } level_t;

static int cmp_k;
static int cmp_pat(const void *a, const void *b) {
    const uint32_t *x = a, *y = b;
    for (int i = 0; i < cmp_k; ++i)
        if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
    return 0;
}

static int contains(const level_t *lv, const uint32_t *pat) {
    uint64_t lo = 0, hi = lv->n;
    while (lo < hi) {
        uint64_t mid = (lo + hi) / 2;
        const uint32_t *p = lv->pats + mid * lv->k;
        int c = 0;
        for (uint32_t i = 0; i < lv->k && !c; ++i)
            if (p[i] != pat[i]) c = p[i] < pat[i] ? -1 : 1;
        if (!c) return 1;
        if (c < 0) lo = mid + 1; else hi = mid;
    }
    return 0;
}

oracle_result *oracle_apriori(uint64_t n_rows, uint32_t n_items, const uint64_t *offsets,
                              const uint32_t *cols, int64_t minsup, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    oracle_result *res = calloc(1, sizeof(*res));
    if (!res) return NULL;
    uint64_t n, words;
    uint64_t *bits = pack(n_rows, n_items, offsets, cols, &n, &words);
    level_t cur = {1, 0, malloc((n_items + 1) * sizeof(uint32_t))};
    for (uint32_t i = 0; i < n_items; ++i) {
        uint64_t s = popc_and(bits + (uint64_t)i * words, bits + (uint64_t)i * words, words);
        if (PASSES(s, minsup)) { cur.pats[cur.n++] = i; res_push(res, &i, 1, s); }
    }
    while (cur.n) {
        uint32_t k = cur.k + 1;
        /* Prefix join over the sorted level, then every (k-1)-subset checked. */
        uint64_t cap = 1024, nc = 0;
        uint32_t *cand = malloc(cap * k * sizeof(uint32_t));
        uint32_t *sub = malloc(2 * (size_t)k * sizeof(uint32_t));
        for (uint64_t a = 0; a < cur.n; ++a) {
            const uint32_t *pa = cur.pats + a * cur.k;
            for (uint64_t b = a + 1; b < cur.n; ++b) {
                const uint32_t *pb = cur.pats + b * cur.k;
                if (memcmp(pa, pb, (cur.k - 1) * sizeof(uint32_t))) break;
                uint32_t *c = sub;
                memcpy(c, pa, cur.k * sizeof(uint32_t));
                c[cur.k] = pb[cur.k - 1];
                int ok = 1;
                uint32_t *tmp = sub + k;
                for (uint32_t drop = 0; drop < k && ok; ++drop) {
                    uint32_t t = 0;
                    for (uint32_t i = 0; i < k; ++i) if (i != drop) tmp[t++] = c[i];
                    ok = contains(&cur, tmp);
                }
                if (!ok) continue;
                if (nc == cap) { cap *= 2; cand = realloc(cand, cap * k * sizeof(uint32_t)); }
                memcpy(cand + nc * k, c, k * sizeof(uint32_t));
                nc++;
            }
        }
        free(sub);
        /* Sorted level order: the join above already emits in sorted order
         * because the level is sorted and candidates extend it in place. */
        cmp_k = (int)k;
        qsort(cand, nc, k * sizeof(uint32_t), cmp_pat);
        uint64_t *sup = malloc((nc + 1) * sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t c = 0; c < (int64_t)nc; ++c) {
            const uint32_t *pc = cand + (uint64_t)c * k;
            uint64_t s = 0;
            for (uint64_t w = 0; w < words; ++w) {
                uint64_t v = ~0ull;
                for (uint32_t j = 0; j < k; ++j) v &= bits[(uint64_t)pc[j] * words + w];
                s += (uint64_t)__builtin_popcountll(v);
            }
            sup[c] = s;
        }
        level_t nxt = {k, 0, malloc((nc + 1) * k * sizeof(uint32_t))};
        for (uint64_t c = 0; c < nc; ++c) {
            if (!PASSES(sup[c], minsup)) continue;
            memcpy(nxt.pats + nxt.n * k, cand + c * k, k * sizeof(uint32_t));
            nxt.n++;
            res_push(res, cand + c * k, k, sup[c]);
        }
        free(sup); free(cand); free(cur.pats);
        cur = nxt;
    }
    free(cur.pats); free(bits);
    return res;
}
