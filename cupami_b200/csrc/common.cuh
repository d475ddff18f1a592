// Shared device helpers for the cupami_b200 kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define CPM_WARP 32
#define CPM_FULL 0xffffffffu

namespace cpm {

__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(CPM_FULL, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(CPM_FULL, v, o);
    return v;
}

__device__ __forceinline__ uint32_t warp_max_u32(uint32_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(CPM_FULL, v, o));
    return v;
}

__device__ __forceinline__ uint32_t popc2(ulonglong2 v) {
    return (uint32_t)(__popcll(v.x) + __popcll(v.y));
}

__device__ __forceinline__ ulonglong2 and2(ulonglong2 a, ulonglong2 b) {
    return make_ulonglong2(a.x & b.x, a.y & b.y);
}

// Streaming 16-byte load that bypasses L1 (siblings are read once per unit).
__device__ __forceinline__ ulonglong2 ld_stream(const ulonglong2 *p) {
    ulonglong2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.u64 {%0, %1}, [%2];"
                 : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}

// Coherent 16-byte load cached in L2 only: for data that other CTAs of the
// same kernel may have written (child tidsets, member tables).
__device__ __forceinline__ ulonglong2 ld_cg(const ulonglong2 *p) {
    ulonglong2 v;
    asm volatile("ld.global.cg.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Relaxed load (no ordering): for a flag whose value is only a hint.
__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

}  // namespace cpm
