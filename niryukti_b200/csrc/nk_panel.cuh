// Column panels of A's long rows: the dual kernel's A dx without scattered
// global gathers for the rows that hold most of the entries.
//
// A gather from a vector much larger than L1 costs the SM's load path one
// cache-line lookup per lane, hit or miss, and the dual kernel's dx gathers are
// uniform over all columns, so that lookup rate, not DRAM, sets its pace.  The
// long rows of A (longer than the SELL split length; in engine order they are
// the first `rows` rows) are therefore also stored by column panel: panel p
// holds the entries whose engine column lies in [p*width, (p+1)*width), a slice
// of dx that fits in one CTA's shared memory.  A CTA of panel_kernel copies the
// slice once and reads every gathered dx entry of the panel from shared memory
// (a few bank cycles per warp instead of one lookup per lane).
//
// Inside a panel the rows with at least one entry there are ordered by their
// entry count (descending, stable) and cut into 32-row chunks stored
// column-major, one row per lane, as in SELL-32: entry k of the chunk's lane t
// sits at cptr[c] + 32*k + t, and a row's entries keep their CSR order.  A lane
// adds its row's entries in the panel one by one from zero and writes the sum
// to partial[p*rows + row]; (row, panel) pairs without entries are never
// written and stay zero.  The dual kernel then adds a long row's partials in
// panel order 0, 1, ..., from zero: the result does not depend on timing, and
// with a single panel it is the row's sequential CSR sum, the CPU's order.
#pragma once
#include "nk_device.cuh"
#include <cuda_runtime.h>
#include <cstdint>

#ifndef NK_PANEL
#define NK_PANEL 1 // 1: long rows of A take the panel path in the dual SpMV
#endif
#ifndef NK_PANEL_THREADS
#define NK_PANEL_THREADS 1024 // threads per CTA of panel_kernel (one CTA per SM)
#endif
#ifndef NK_PANEL_UNROLL
#define NK_PANEL_UNROLL 4
#endif

namespace nk {

constexpr int kPanelThreads = NK_PANEL_THREADS;
constexpr int kPanelWarps = kPanelThreads / 32;
constexpr int kPanelMinBlocks = 1024 / kPanelThreads;

template <class V> struct PanelView {
    int64_t rows = 0;        // long rows: engine rows [0, rows)
    int64_t cols = 0;        // columns of A
    int64_t width = 0;       // columns per panel (a multiple of 16)
    const int64_t *uoff = nullptr; // CTA b runs units[uoff[b] .. uoff[b+1])
    const int4 *units = nullptr;   // {panel, first chunk, end chunk, 0}
    const int64_t *cptr = nullptr; // chunk c: entries [cptr[c], cptr[c+1])
    const int2 *lane = nullptr;    // 32 per chunk: {row (-1: padding), entries}
    const uint16_t *lidx = nullptr; // column within the panel
    const V *val = nullptr;
    double *partial = nullptr;     // [panels][rows]
};

// One launch per trial, after primal_kernel (which writes dx) and before
// dual_kernel (which adds the partials).  Grid: one CTA per unit list.
template <class Acc, class V, class X>
__global__ void __launch_bounds__(kPanelThreads, kPanelMinBlocks)
    panel_kernel(PanelView<V> P, const X *__restrict__ dx, const Control *ctl) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    X *sdx = reinterpret_cast<X *>(dyn_smem);
    if (ctl->restart != 0) // a requested Halpern restart freezes the chunk
        return;
    const int warp = threadIdx.x >> 5, t = threadIdx.x & 31;
    const int64_t u0 = P.uoff[blockIdx.x], u1 = P.uoff[blockIdx.x + 1];
    for (int64_t u = u0; u < u1; ++u) {
        const int4 w = P.units[u];
        const int64_t col0 = int64_t(w.x) * P.width;
        const int64_t cols = P.cols - col0 < P.width ? P.cols - col0 : P.width;
        if (u > u0)
            __syncthreads(); // every warp is done with the previous slice
        stage16<kPanelThreads>(sdx, dx + col0, cols * int64_t(sizeof(X)));
        __syncthreads();
        double *out = P.partial + int64_t(w.x) * P.rows;
        for (int64_t c = w.y + warp; c < w.z; c += kPanelWarps) {
            const int2 rl = P.lane[c * 32 + t];
            const int64_t base = P.cptr[c] + t;
            const uint16_t *ip = P.lidx + base;
            const V *vp = P.val + base;
            Acc acc = Acc(0);
            int k = 0;
            constexpr int U = NK_PANEL_UNROLL;
            for (; k + U <= rl.y; k += U) {
                uint16_t j[U];
                V a[U];
#pragma unroll
                for (int q = 0; q < U; ++q) {
                    j[q] = stream_load(ip + int64_t(k + q) * 32);
                    a[q] = stream_load(vp + int64_t(k + q) * 32);
                }
#pragma unroll
                for (int q = 0; q < U; ++q)
                    acc = acc + Acc(a[q]) * Acc(sdx[j[q]]);
            }
            for (; k < rl.y; ++k)
                acc = acc + Acc(stream_load(vp + int64_t(k) * 32)) *
                                Acc(sdx[stream_load(ip + int64_t(k) * 32)]);
            if (rl.x >= 0)
                out[rl.x] = double(acc);
        }
    }
}

} // namespace nk
