// Device building blocks of the PDHG engine: CSR views, the row schedule, the
// sub-warp / warp / CTA row dot products and deterministic block reductions.
//
// Every SpMV in the engine walks a *schedule*: a list of work items, each one of
//   kind W in {2,4,8,16,32}: a tile of up to 256/W consecutive rows, one row per
//                            W-lane sub-warp (rows longer than the matrix's long
//                            threshold are skipped here and handled below);
//   kind KIND_WARP:          up to 8 long rows from the long-row list, one per warp;
//   kind KIND_CTA:           one very long row, the whole CTA on it.
// Items are visited by a persistent grid in a fixed round-robin order, and every
// reduction combines values in a fixed order, so results do not depend on
// timing.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

namespace nk {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int KIND_WARP = 64;
constexpr int KIND_CTA = 128;

template <class V, class P, class I> struct Csr {
    const P *ptr;
    const I *idx;
    const V *val;
    int64_t rows;
};

struct Schedule {
    const int4 *items;   // {kind, first, count, 0}
    const int64_t *longrows;
    int nitems;
    int64_t long_threshold; // rows with more entries are in the long list
};

// Streaming loads for single-use matrix data (evict-first), cached loads for
// the gathered vector, which stays resident in L2.
template <class T> __device__ __forceinline__ T stream_load(const T *p) { return __ldcs(p); }
template <class T> __device__ __forceinline__ T gather_load(const T *p) { return __ldg(p); }

// Sum of one row over W cooperating lanes (lane = 0..W-1); all 32 lanes of the
// warp must call it.  Lanes with valid == false contribute zero.  Returns the
// row sum in every lane of the W-group.
template <int W, class Acc, class V, class P, class I, class X>
__device__ __forceinline__ Acc group_dot(const Csr<V, P, I> &M, int64_t row, bool valid,
                                         const X *__restrict__ x, int lane) {
    Acc acc = Acc(0);
    if (valid) {
        P b = M.ptr[row], e = M.ptr[row + 1];
        P k = b + lane;
        // two independent chains keep more gathers in flight
        Acc acc2 = Acc(0);
        for (; k + W < e; k += 2 * W) {
            I j0 = stream_load(M.idx + k), j1 = stream_load(M.idx + k + W);
            V v0 = stream_load(M.val + k), v1 = stream_load(M.val + k + W);
            acc = acc + Acc(v0) * Acc(gather_load(x + j0));
            acc2 = acc2 + Acc(v1) * Acc(gather_load(x + j1));
        }
        if (k < e)
            acc = acc + Acc(stream_load(M.val + k)) * Acc(gather_load(x + stream_load(M.idx + k)));
        acc = acc + acc2;
    }
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1)
        acc = acc + __shfl_xor_sync(0xffffffffu, acc, off);
    return acc;
}

// Sum of one row over the whole CTA; result valid in every thread.
template <class Acc, class V, class P, class I, class X>
__device__ __forceinline__ Acc cta_dot(const Csr<V, P, I> &M, int64_t row,
                                       const X *__restrict__ x, Acc *smem /* kWarps */) {
    P b = M.ptr[row], e = M.ptr[row + 1];
    Acc acc = Acc(0), acc2 = Acc(0);
    P k = b + threadIdx.x;
    for (; k + kThreads < e; k += 2 * kThreads) {
        I j0 = stream_load(M.idx + k), j1 = stream_load(M.idx + k + kThreads);
        V v0 = stream_load(M.val + k), v1 = stream_load(M.val + k + kThreads);
        acc = acc + Acc(v0) * Acc(gather_load(x + j0));
        acc2 = acc2 + Acc(v1) * Acc(gather_load(x + j1));
    }
    if (k < e)
        acc = acc + Acc(stream_load(M.val + k)) * Acc(gather_load(x + stream_load(M.idx + k)));
    acc = acc + acc2;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        acc = acc + __shfl_xor_sync(0xffffffffu, acc, off);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
        smem[w] = acc;
    __syncthreads();
    Acc total = Acc(0);
#pragma unroll
    for (int i = 0; i < kWarps; ++i)
        total = total + smem[i];
    __syncthreads();
    return total;
}

// Deterministic CTA reduction of NV doubles (fixed tree); result in thread 0.
template <int NV> __device__ __forceinline__ void cta_sum(double (&v)[NV], double *smem /* kWarps*NV */) {
#pragma unroll
    for (int t = 0; t < NV; ++t)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            v[t] += __shfl_xor_sync(0xffffffffu, v[t], off);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
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
            for (int i = 0; i < kWarps; ++i)
                s += smem[i * NV + t];
            v[t] = s;
        }
    }
    __syncthreads();
}

// Visit every row of a schedule.  Every thread of the CTA calls
// f(row, sum, leader, valid, group, lane) once per row position: sum is the
// row's dot product with x (identical across the cooperating group), leader
// marks the one thread that consumes it, valid is false for padding lanes, and
// group is std::integral_constant<int, lanes per row> (kThreads for a CTA row),
// so f can run a second cooperative dot product over the same row of another
// matrix.
template <class Acc, class V, class P, class I, class X, class F>
__device__ __forceinline__ void sweep(const Csr<V, P, I> &M, const Schedule &S,
                                      const X *__restrict__ x, F &&f) {
    __shared__ Acc red[kWarps];
    const int lane32 = threadIdx.x & 31;
    for (int it = blockIdx.x; it < S.nitems; it += gridDim.x) {
        int4 item = S.items[it];
        int kind = item.x;
        if (kind <= 32) {
            switch (kind) {
#define NK_TILE(WW)                                                                                \
    case WW: {                                                                                     \
        int sub = threadIdx.x / WW, lane = threadIdx.x % WW;                                       \
        int64_t row = int64_t(item.y) + sub;                                                       \
        bool valid = sub < item.z;                                                                 \
        if (valid) {                                                                               \
            int64_t len = int64_t(M.ptr[row + 1]) - int64_t(M.ptr[row]);                           \
            valid = len <= S.long_threshold;                                                       \
        }                                                                                          \
        Acc s = group_dot<WW, Acc>(M, row, valid, x, lane);                                        \
        f(row, s, valid && lane == 0, valid, std::integral_constant<int, WW>{}, lane);                                            \
    } break;
                NK_TILE(2)
                NK_TILE(4)
                NK_TILE(8)
                NK_TILE(16)
                NK_TILE(32)
#undef NK_TILE
            default:
                break;
            }
        } else if (kind == KIND_WARP) {
            int w = threadIdx.x >> 5;
            bool valid = w < item.z;
            int64_t row = valid ? S.longrows[item.y + w] : 0;
            Acc s = group_dot<32, Acc>(M, row, valid, x, lane32);
            f(row, s, valid && lane32 == 0, valid, std::integral_constant<int, 32>{}, lane32);
        } else {
            int64_t row = S.longrows[item.y];
            Acc s = cta_dot<Acc>(M, row, x, red);
            f(row, s, threadIdx.x == 0, true, std::integral_constant<int, kThreads>{}, int(threadIdx.x));
        }
    }
}

} // namespace nk
