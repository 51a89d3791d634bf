// Device primitives shared by the engine's kernels: CTA geometry, load flavours
// and a deterministic CTA reduction.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace nk {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// Streaming loads for single-use matrix data (evict-first), cached loads for
// the gathered vector, which stays resident in L2.
#ifndef NK_STREAM_HINT
#define NK_STREAM_HINT 1 // 1: evict-first loads for matrix entries, 0: default caching
#endif
template <class T> __device__ __forceinline__ T stream_load(const T *p) {
#if NK_STREAM_HINT
    return __ldcs(p);
#else
    return *p;
#endif
}
template <class T> __device__ __forceinline__ T gather_load(const T *p) { return __ldg(p); }

// Gather flavours: 0 read-only path (L1-allocating), 1 read-only without L1
// allocation (a gathered line is rarely reused from L1 when the vector is much
// larger than L1), 2 L2 only.
template <int G, class T> __device__ __forceinline__ T gather_as(const T *p) {
    if constexpr (G == 1 && sizeof(T) == 8) {
        double v;
        asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
        return T(v);
    } else if constexpr (G == 1 && sizeof(T) == 4) {
        float v;
        asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
        return T(v);
    } else if constexpr (G == 2) {
        return __ldcg(p);
    } else {
        return __ldg(p);
    }
}

// Deterministic CTA reduction of NV doubles (fixed tree) over a CTA of W
// warps; result in thread 0.
template <int NV, int W = kWarps>
__device__ __forceinline__ void cta_sum(double (&v)[NV], double *smem /* W*NV */) {
#pragma unroll
    for (int t = 0; t < NV; ++t)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            v[t] += __shfl_xor_sync(0xffffffffu, v[t], off);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
#pragma unroll
        for (int t = 0; t < NV; ++t)
            smem[w * NV + t] = v[t];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < NV; ++t) {
            double s = 0;
            for (int i = 0; i < W; ++i)
                s += smem[i * NV + t];
            v[t] = s;
        }
    }
    __syncthreads();
}

} // namespace nk
