// SELL-32 storage of the engine's matrices and the thread-per-row dot product
// every fused PDHG kernel is built on.
//
// Layout.  The rows of a matrix are taken in engine order (sorted by length,
// longest first, stable) and cut into chunks of 32 consecutive rows; chunk c
// stores its rows column-major: entry k of the chunk's row t sits at
// cptr[c] + 32*k + t, padded to the chunk's longest row.  A warp works on one
// chunk with one row per lane, so its k-th load reads entry k of 32 rows -- a
// single coalesced access -- with no shared memory and no synchronisation.  A
// row's entries keep their CSR order, and a lane adds them up one by one, so
// the sum has the order and rounding of a sequential CPU loop.
//
// Rows longer than the split length are cut into segments ("virtual rows") of
// at most that length; the segments of split rows come first, in whole chunks.
// A row of at most 32 segments lies inside one chunk: its warp adds the
// segment sums in order through shared memory (the row's first lane leads).
// Longer rows span chunks: each segment's sum goes to a slot, and the last
// segment of the row to arrive (an atomic counter) adds the slots in order.
// Either way the result does not depend on timing.  Padding entries and padding
// virtual rows are never read (lane loops stop at their own length).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace nk {

#ifndef NK_UNROLL
#define NK_UNROLL 4
#endif
#ifndef NK_UNROLL_SPLIT
#define NK_UNROLL_SPLIT 4
#endif
constexpr int kUnroll = NK_UNROLL;            // independent loads in flight per lane
constexpr int kUnrollSplit = NK_UNROLL_SPLIT; // the same for split-row segments

template <class V, class I> struct Sell {
    const int64_t *cptr;   // nchunks + 1 element offsets
    const int32_t *len;    // length of each virtual row
    const I *idx;          // column indices (engine order of the other side)
    const V *val;
    int64_t nv;            // virtual rows
    int64_t nsv;           // leading virtual rows that are segments of split rows
    int64_t nsr;           // leading real rows that were split
    const int4 *seg;       // per split segment: {real row (-1: padding), first segment,
                           //   segments, counter (-1: the row lies in one chunk)}
    double *slots;         // per split segment: partial sum
    unsigned *counters;    // per split row: arrivals (reset by the last one)
    // The fused kernels' schedule: CTA b owns chunks clist[coff[b] .. coff[b+1]).
    const int64_t *coff = nullptr;
    const int64_t *clist = nullptr;
};

// Sequential dot product of virtual row v (entries in CSR order) starting
// from acc; U entries' loads are issued before their products are added.
// Used inside the fused PDHG kernels, where registers are scarce.
template <class Acc, int U = kUnroll, int G = 0, class V, class I, class X>
__device__ __forceinline__ Acc sell_dot(const Sell<V, I> &M, int64_t v, int len, Acc acc,
                                        const X *__restrict__ x) {
    const int64_t base = M.cptr[v >> 5] + (v & 31);
    const I *ip = M.idx + base;
    const V *vp = M.val + base;
    int k = 0;
    for (; k + U <= len; k += U) {
        I j[U];
        V w[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            j[u] = stream_load(ip + int64_t(k + u) * 32);
            w[u] = stream_load(vp + int64_t(k + u) * 32);
        }
        X g[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            g[u] = gather_as<G>(x + j[u]);
#pragma unroll
        for (int u = 0; u < U; ++u)
            acc = acc + Acc(w[u]) * Acc(g[u]);
    }
    for (; k < len; ++k)
        acc = acc + Acc(stream_load(vp + int64_t(k) * 32)) *
                        Acc(gather_as<G>(x + stream_load(ip + int64_t(k) * 32)));
    return acc;
}

// The same sum, software-pipelined: the gathers of block b are issued, then the
// index/value loads of block b+1, and only then are block b's products added,
// so each block costs about one memory round trip instead of two.  It needs
// more registers; the plain SpMV kernel uses it.
template <class Acc, int U = kUnroll, class V, class I, class X>
__device__ __forceinline__ Acc sell_dot_pipelined(const Sell<V, I> &M, int64_t v, int len, Acc acc,
                                                  const X *__restrict__ x) {
    if (len <= 0)
        return acc;
    const int64_t base = M.cptr[v >> 5] + (v & 31);
    const I *ip = M.idx + base;
    const V *vp = M.val + base;
    I j[U];
    V w[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
        if (u < len) {
            j[u] = stream_load(ip + int64_t(u) * 32);
            w[u] = stream_load(vp + int64_t(u) * 32);
        }
    for (int k = 0; k < len; k += U) {
        X g[U];
        V wc[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k + u < len) {
                g[u] = gather_load(x + j[u]);
                wc[u] = w[u];
            }
        const int kn = k + U;
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (kn + u < len) {
                j[u] = stream_load(ip + int64_t(kn + u) * 32);
                w[u] = stream_load(vp + int64_t(kn + u) * 32);
            }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k + u < len)
                acc = acc + Acc(wc[u]) * Acc(g[u]);
    }
    return acc;
}

// Sparse symmetric Q in CSR (engine order on both sides).
template <class V, class I> struct QCsr {
    const int64_t *ptr;
    const I *idx;
    const V *val;
};

// Sequential dot of row r of Q with x, from zero (Sparse::multiply order).
template <class Acc, class V, class I, class X>
__device__ __forceinline__ Acc q_dot(const QCsr<V, I> &Q, int64_t r, const X *__restrict__ x) {
    Acc acc = Acc(0);
    for (int64_t k = Q.ptr[r]; k < Q.ptr[r + 1]; ++k)
        acc = acc + Acc(Q.val[k]) * Acc(x[Q.idx[k]]);
    return acc;
}

} // namespace nk
