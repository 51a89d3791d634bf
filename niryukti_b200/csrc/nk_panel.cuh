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
// Inside a panel each row with entries there is a segment: its entries in CSR
// order.  A segment longer than a quarter of a lane's expected stream is cut
// into runs of nearly equal length; a shorter one is one run.  Each run is
// followed by a marker entry (column 0xFFFF) whose value slot carries the run's
// slot number, and runs are packed whole into lanes, longest first onto the
// least-loaded lane, so every lane holds a stream of nearly the same length.
// A chunk's 32 lane streams are stored column-major as in SELL-32 (entry k of
// lane t of chunk c at cptr[c] + 32*k + t).  A lane adds its entries one by
// one; at a marker it writes the sum to partial[slot] and starts again from
// zero.  So a run's sum is its sequential CSR sum, and no lane waits on a
// lookup: the slot number arrives in the stream.  Slots are numbered row by
// row, then by panel, then by run, so long row i owns slots
// [roff[i], roff[i+1]); the dual kernel adds them in that order from zero.
// The result does not depend on timing, and for a row held by one run (one
// panel, not cut) it is the row's sequential CSR sum, the CPU's order.
//
// A unit is an equal share of all panels' entries, one per CTA; it holds one
// piece (one chunk per warp) per panel it touches, so a CTA copies one slice,
// or two where its share straddles a panel boundary.  CTAs take units from a
// global counter and, inside a piece, warps take chunks from a shared counter.
// Every run's sum has one writer, so which CTA or warp runs a chunk changes
// nothing in the results, and the SMs finish together whatever the estimate
// of a unit's cost was worth.
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
#ifndef NK_PANEL_MIN_RUN
#define NK_PANEL_MIN_RUN 32 // panels only when long rows average this many entries per panel
#endif
#ifndef NK_PANEL_MIN_SPLIT
#define NK_PANEL_MIN_SPLIT 64 // segments are cut into runs of no fewer entries than this
#endif
#ifndef NK_PANEL_UNROLL
#define NK_PANEL_UNROLL 8 // entries of its stream a lane loads before adding them
#endif

namespace nk {

constexpr int kPanelThreads = NK_PANEL_THREADS;
constexpr int kPanelWarps = kPanelThreads / 32;
constexpr int kPanelMinBlocks = 1024 / kPanelThreads;
constexpr uint16_t kPanelMarker = 0xFFFF; // column of a segment's closing marker
constexpr int64_t kPanelMaxWidth = 65535;  // columns 0 .. 0xFFFE

template <class V> struct PanelView {
    int64_t rows = 0;        // long rows: engine rows [0, rows)
    int64_t cols = 0;        // columns of A
    int64_t width = 0;       // columns per panel (a multiple of 16)
    int64_t nunits = 0;
    const int4 *units = nullptr;   // pieces {panel, first chunk, end chunk, unit}
    const int64_t *uoff = nullptr; // unit u: pieces [uoff[u], uoff[u+1])
    const int64_t *cptr = nullptr; // chunk c: entries [cptr[c], cptr[c+1]), 32 per step
    const uint16_t *lidx = nullptr; // column within the panel, or kPanelMarker
    const V *val = nullptr;         // value, or at a marker the slot (bits of an int)
    double *partial = nullptr;     // one per slot
    int64_t slots = 0;
    unsigned *claim = nullptr;     // [0] next unit, [1] CTAs done; zero between launches
};

// The slot a marker's value carries.
template <class V> __device__ __forceinline__ int64_t marker_slot(V a) {
    if constexpr (sizeof(V) == 8)
        return int64_t(__double_as_longlong(double(a)));
    else
        return int64_t(__float_as_int(float(a)));
}

// One launch per trial, after primal_kernel (which writes dx) and before
// dual_kernel (which adds the partials).  Persistent grid, one CTA per SM.
template <class Acc, class V, class X>
__global__ void __launch_bounds__(kPanelThreads, kPanelMinBlocks)
    panel_kernel(PanelView<V> P, const X *__restrict__ dx, const Control *ctl) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ unsigned unit, next_chunk;
    X *sdx = reinterpret_cast<X *>(dyn_smem);
    if (ctl->restart != 0) // a requested Halpern restart freezes the chunk: no claims
        return;
    const int t = threadIdx.x & 31;
    for (;;) {
        if (threadIdx.x == 0)
            unit = atomicAdd(P.claim, 1u);
        __syncthreads();
        const unsigned u = unit;
        if (u >= P.nunits)
            break; // the whole CTA
        for (int64_t pc = P.uoff[u]; pc < P.uoff[u + 1]; ++pc) {
            const int4 w = P.units[pc];
            if (threadIdx.x == 0)
                next_chunk = 0;
            const int64_t col0 = int64_t(w.x) * P.width;
            const int64_t cols = P.cols - col0 < P.width ? P.cols - col0 : P.width;
            stage16<kPanelThreads>(sdx, dx + col0, cols * int64_t(sizeof(X)));
            __syncthreads();
            double *out = P.partial;
            const int span = w.z - w.y;
            for (;;) {
                unsigned k = 0;
                if (t == 0)
                    k = atomicAdd(&next_chunk, 1u);
                k = __shfl_sync(0xffffffffu, k, 0);
                if (int(k) >= span)
                    break;
                const int64_t c = int64_t(w.y) + k;
                const int64_t base = P.cptr[c] + t;
                const int len = int((P.cptr[c + 1] - P.cptr[c]) >> 5);
                const uint16_t *ip = P.lidx + base;
                const V *vp = P.val + base;
                Acc acc = Acc(0);
                int e = 0;
                constexpr int U = NK_PANEL_UNROLL;
                for (; e + U <= len; e += U) {
                    uint16_t j[U];
                    V a[U];
#pragma unroll
                    for (int q = 0; q < U; ++q) {
                        j[q] = stream_load(ip + int64_t(e + q) * 32);
                        a[q] = stream_load(vp + int64_t(e + q) * 32);
                    }
#pragma unroll
                    for (int q = 0; q < U; ++q) {
                        if (j[q] == kPanelMarker) {
                            const int64_t sl = marker_slot(a[q]);
                            if (sl >= 0 && sl < P.slots) // a layout fault drops the sum
                                out[sl] = double(acc);
                            acc = Acc(0);
                        } else
                            acc = acc + Acc(a[q]) * Acc(sdx[j[q]]);
                    }
                }
                for (; e < len; ++e) {
                    const uint16_t j = stream_load(ip + int64_t(e) * 32);
                    const V a = stream_load(vp + int64_t(e) * 32);
                    if (j == kPanelMarker) {
                        const int64_t sl = marker_slot(a);
                        if (sl >= 0 && sl < P.slots)
                            out[sl] = double(acc);
                        acc = Acc(0);
                    } else
                        acc = acc + Acc(a) * Acc(sdx[j]);
                }
            }
            __syncthreads(); // the slice and the chunk counter are free for the next piece
        }
        __syncthreads(); // every thread has read `unit` (a unit may hold no piece)
    }
    if (threadIdx.x == 0) { // the last CTA out clears the counters for the next launch
        __threadfence();
        if (atomicAdd(P.claim + 1, 1u) == gridDim.x - 1) {
            P.claim[0] = 0;
            P.claim[1] = 0;
        }
    }
}

} // namespace nk
