// Device parse of delimited text holding unquoted integer baskets.
//
// Reference: cupami/frequentPattern/_gpu_io.py:34-54 (read_text) reads a CSV
// or TSV file on the GPU when every stripped, non-empty line matches
// ^[0-9]+(\s*SEP\s*[0-9]+)*$ and otherwise leaves it to the CPU reader; its
// labels are the stripped token strings.  Here the bytes are uploaded once and
// parsed by three kernels: newline positions, one thread per line to check the
// layout and count its tokens, and one thread per line to write the tokens as
// uint32 ids (the offsets come from a scan of the counts).  A token's id is its
// value; that id names the same label as the token's string only when the
// token is canonical (no leading zero unless it is "0", at most 4294967295), so
// any other token -- like any line outside the layout, a non-ASCII byte or an
// empty token -- sets the reject flag and the caller reads the file on the CPU,
// which is what the reference does for layouts its GPU reader does not take.
#pragma once
#include "common.cuh"

namespace cpm {

__device__ __forceinline__ bool text_space(unsigned char c) {
    return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f';
}

// flag[i] = 1 where text[i] is a newline.
__global__ void k_text_newlines(const unsigned char *__restrict__ text, uint64_t n, uint32_t *__restrict__ flag) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = text[i] == '\n' ? 1u : 0u;
}

// nl[pos[i]] = i for every newline i (pos: exclusive scan of the flags).
__global__ void k_text_scatter(const uint32_t *__restrict__ flag, const uint64_t *__restrict__ pos, uint64_t n,
                               uint64_t *__restrict__ nl) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (flag[i]) nl[pos[i]] = i;
}

// Line k spans [start, end): start = 0 or one past newline k - 1, end =
// newline k, or n for a last line without one.
__device__ __forceinline__ void text_line(const uint64_t *__restrict__ nl, uint64_t n_nl, uint64_t n, uint64_t k,
                                          uint64_t *start, uint64_t *end) {
    *start = k == 0 ? 0 : nl[k - 1] + 1;
    *end = k < n_nl ? nl[k] : n;
}

// Tokens of line k (0 for a blank line); a line outside the layout sets *reject.
// With write_ids, writes the ids at ids[off[k] ...] instead of counting.
template <bool WRITE>
__global__ void k_text_lines(const unsigned char *__restrict__ text, uint64_t n, const uint64_t *__restrict__ nl,
                             uint64_t n_nl, uint64_t n_lines, unsigned char sep, uint32_t *__restrict__ count,
                             const uint64_t *__restrict__ off, uint32_t *__restrict__ ids,
                             unsigned int *__restrict__ reject) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_lines) return;
    uint64_t a, b;
    text_line(nl, n_nl, n, k, &a, &b);
    while (a < b && text_space(text[a])) ++a;
    while (b > a && text_space(text[b - 1])) --b;
    uint32_t tokens = 0;
    bool ok = true;
    uint64_t at = WRITE ? off[k] : 0;
    uint64_t i = a;
    while (i < b && ok) {
        // a token: digits only, canonical, at most 4294967295
        const uint64_t t0 = i;
        uint64_t v = 0;
        while (i < b && text[i] >= '0' && text[i] <= '9') {
            v = v * 10 + (text[i] - '0');
            if (v > 0xFFFFFFFFull) ok = false;
            ++i;
        }
        const uint64_t len = i - t0;
        if (len == 0 || (len > 1 && text[t0] == '0') || len > 10) ok = false;
        if (!ok) break;
        if (WRITE) ids[at++] = (uint32_t)v;
        ++tokens;
        if (i == b) break;
        // then optional spaces, the separator, optional spaces, and another token
        while (i < b && text[i] != sep && text_space(text[i])) ++i;
        if (i == b || text[i] != sep) {
            ok = false;
            break;
        }
        ++i;
        while (i < b && text_space(text[i])) ++i;
        if (i == b) ok = false;  // a separator must be followed by a token
    }
    for (uint64_t j = a; j < b && ok; ++j)
        if (text[j] >= 0x80) ok = false;
    if (!ok) {
        atomicOr(reject, 1u);
        tokens = 0;
    }
    if (!WRITE) count[k] = tokens;
}

}  // namespace cpm
