// Host launchers for the reference's own bitset kernels -- TEST
// INFRASTRUCTURE ONLY (the reference-GPU leg of the benchmark and its parity
// test; the product never loads this).
//
// The kernels are not restated here: oracle/build_ref.py extracts the
// reference's CUDA source strings (cupami/frequentPattern/_bitsets.py:19-78,
// cupami/periodicFrequentPattern/_temporal.py:26-53) into a temporary file
// under oracle/_ref/ and compiles this file with -DREF_KERNELS=<that path>.
// Each launcher uses the reference wrapper's launch shape: build_bitsets one
// thread per occurrence in blocks of 256 (_bitsets.py:91-100); count_supports
// and intersect_extensions one block of 256 threads per candidate
// (_bitsets.py:103-125); periodic_counts one thread per candidate in blocks of
// 128 (_temporal.py:156-165).
#include <cuda_runtime.h>
#include <stdint.h>

#include REF_KERNELS

extern "C" int ref_build_bitsets(uint64_t count, const uint64_t *rows, const uint32_t *columns, uint64_t words,
                                 uint32_t *bitsets, void *stream) {
    if (count)
        build_bitsets<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
            (unsigned long long)count, (const unsigned long long *)rows, columns, (unsigned long long)words, bitsets);
    return (int)cudaGetLastError();
}

extern "C" int ref_count_supports(const uint32_t *bitsets, uint64_t words, const uint32_t *candidates, uint32_t width,
                                  uint64_t n, uint64_t *supports, void *stream) {
    if (n)
        count_supports<<<(unsigned)n, 256, 0, (cudaStream_t)stream>>>(bitsets, (unsigned long long)words, candidates,
                                                                      width, (unsigned long long *)supports);
    return (int)cudaGetLastError();
}

extern "C" int ref_intersect_extensions(const uint32_t *prefix, const uint32_t *extensions, uint64_t words, uint64_t n,
                                        uint32_t *intersections, uint64_t *supports, void *stream) {
    if (n)
        intersect_extensions<<<(unsigned)n, 256, 0, (cudaStream_t)stream>>>(
            prefix, extensions, (unsigned long long)words, intersections, (unsigned long long *)supports);
    return (int)cudaGetLastError();
}

extern "C" int ref_periodic_counts(const uint32_t *bits, uint64_t words, const uint32_t *candidates, uint32_t width,
                                   uint32_t n, const int64_t *timestamps, uint64_t rows, int64_t end,
                                   uint64_t *supports, int64_t *periods, void *stream) {
    if (n)
        periodic_counts<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
            bits, (unsigned long long)words, candidates, width, n, (const long long *)timestamps,
            (unsigned long long)rows, (long long)end, (unsigned long long *)supports, (long long *)periods);
    return (int)cudaGetLastError();
}
