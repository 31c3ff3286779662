// prims.cuh — small device building blocks: warp/block scans and reductions,
// cache-hinted loads.  All reductions use a fixed tree so results are
// bit-reproducible from run to run.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace prg {

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// L2 eviction-priority policies (createpolicy) for cache-hinted loads.
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Streaming 16-byte load of read-only data: no L1 allocation, evict-first in
// L2, so the index stream does not push the gathered rank vector out of L2.
__device__ __forceinline__ uint4 ld_stream_u4(const uint4 *p, uint64_t pol) {
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ld_stream_f4(const float4 *p, uint64_t pol) {
    float4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double2 ld_stream_d2(const double2 *p, uint64_t pol) {
    double2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
        : "=d"(v.x), "=d"(v.y)
        : "l"(p), "l"(pol));
    return v;
}
// Gather of the rank vector: read-only path, evict-last in L2.
__device__ __forceinline__ float ld_gather(const float *p, uint64_t pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
// Gather that does not allocate in L1 (cold sources: keeps L1 for the hot prefix).
__device__ __forceinline__ float ld_gather_na(const float *p, uint64_t pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_gather_na(const double *p, uint64_t pol) {
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_gather(const double *p, uint64_t pol) {
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of two doubles (fixed tree).  `sh` needs 2*32 doubles.
// Result valid in thread 0 only.  Ends with a __syncthreads-free return;
// callers must __syncthreads() before reusing `sh`.
__device__ __forceinline__ double2 block_sum2(double a, double b, double *sh) {
    a = warp_sum(a);
    b = warp_sum(b);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sh[w] = a;
        sh[32 + w] = b;
    }
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (w == 0) {
        int nw = blockDim.x >> 5;
        double x = l < nw ? sh[l] : 0.0;
        double y = l < nw ? sh[32 + l] : 0.0;
        x = warp_sum(x);
        y = warp_sum(y);
        r = make_double2(x, y);
    }
    return r;
}

template <class T>
__device__ __forceinline__ T block_sum(T a, T *sh) {
    a = warp_sum(a);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = a;
    __syncthreads();
    T r = T(0);
    if (w == 0) {
        int nw = blockDim.x >> 5;
        T x = l < nw ? sh[l] : T(0);
        r = warp_sum(x);
    }
    return r;
}

// Inclusive warp scan (u32).
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    int l = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (l >= o) v += t;
    }
    return v;
}

// Exclusive block scan (u32), returns this thread's exclusive prefix and the
// block total through *total.  `sh` needs 33 u32.  Contains __syncthreads.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *sh, uint32_t *total) {
    int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    uint32_t inc = warp_incl_scan(v);
    if (l == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t s = l < nw ? sh[l] : 0u;
        uint32_t si = warp_incl_scan(s);
        if (l < nw) sh[l] = si - s;
        if (l == nw - 1) sh[32] = si;
    }
    __syncthreads();
    uint32_t r = sh[w] + inc - v;
    *total = sh[32];
    __syncthreads();
    return r;
}

}  // namespace prg
