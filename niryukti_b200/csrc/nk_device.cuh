// Kernels of the B200 PDHG engine (host side: nk_engine.cu).
//
// One PDHG trial is two kernels over SELL-32 matrices (nk_sell.cuh):
//   primal_kernel  g = c + A^T y (+ Q x + q.x)   -- one lane per row of A^T
//                  trial x = clamp((x - tau g)/(1 + tau q), lb, ub), dx, sum dx^2
//                  (restates primal_trial, src/cuda.cu:240-260, and the CPU loop
//                   src/cpu.cpp:107-132, fused into the SpMV)
//   dual_kernel    delta = A dx                   -- one lane per row of A
//                  trial y = interval prox of y + sigma (Ax + 2 delta), Ax + delta,
//                  sum dy^2, sum dy*delta         (dual_trial, src/cuda.cu:261-284;
//                                                  src/cpu.cpp:136-150)
//                  and, in its last CTA, the accept / step-factor / averaging decision
//                  (decide, src/cuda.cu:285-335; src/cpu.cpp:151-216)
// Iterates are double-buffered: accepting a trial flips a device-side index, and the
// running-average update of an accepted step is applied by the next trial's kernels
// (commit_primal / commit_dual, src/cuda.cu:336-370, without their own passes).
// The Halpern variant keeps a separate commit kernel.
#pragma once
#include "nk_kernels.cuh"
#include "nk_sell.cuh"
#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#ifndef NK_FUSED_THREADS
#define NK_FUSED_THREADS 1024 // threads per CTA of the fused trial kernels
#endif
#ifndef NK_SPLIT_PIPE
#define NK_SPLIT_PIPE 0 // 1: software-pipelined dot for split-row segments
#endif
#ifndef NK_DUAL_GATHER
#define NK_DUAL_GATHER 0 // gather flavour of the dual kernel's dx loads (gather_as)
#endif
#ifndef NK_PREFETCH
#define NK_PREFETCH 1 // 1: load a row's epilogue vectors before its dot product
#endif

namespace nk {

constexpr int kDualGather = NK_DUAL_GATHER;
// The fused kernels run 1024 threads per SM (64 registers each) in CTAs of
// kFusedThreads; larger CTAs give each CTA a larger slice of shared memory.
constexpr int kFusedThreads = NK_FUSED_THREADS;
constexpr int kFusedWarps = kFusedThreads / 32;
constexpr int kFusedMinBlocks = 1024 / kFusedThreads;
static_assert(kFusedThreads % 32 == 0 && 1024 % kFusedThreads == 0, "fused CTA size");

// Device-resident control state.  The first eleven fields keep the meaning of
// the reference's `state` vector (src/cuda.cu:224-225,601).
struct Control {
    double factor;    // step multiplier
    double mass;      // averaging mass
    double accepted;  // accepted trials
    double rejected;  // rejected trials
    double accept;    // last trial accepted
    double weight;    // last averaging weight
    double epoch;     // Halpern epoch steps
    double init_res;  // Halpern initial residual
    double prev_res;  // Halpern previous residual
    double restart;   // Halpern restart requested
    double lambda;    // Halpern anchor weight
    double tau, sigma;  // base steps of the current chunk (device-resident for graph replay)
    double pending_w;   // averaging weight of the accepted step not yet folded in
    int cur;            // which x / y / Ax buffer holds the current iterate
    int pending;        // 1 while pending_w must still be applied
    unsigned arrive;    // last-CTA detection in dual_kernel
    int flags;          // bit 0 adaptive, bit 1 halpern, bit 2 residual restarts
};

struct Vecs {
    const double *c, *q, *lb, *ub, *rl, *ru;
    double *x0, *x1, *y0, *y1, *ax0, *ax1, *xa, *ya;
    double *dx;           // primal displacement (FP64 gather source)
    float *dx32;          // FP32 gather source (precision FP32)
    float *y32_0, *y32_1; // FP32 copies of y (precision FP32)
    double *anchor_x, *anchor_y, *anchor_ax;
    double *part_p;       // per-CTA sum dx^2 of primal_kernel
    double *part_d;       // per-CTA (sum dy^2, sum dy*delta) of dual_kernel
    Control *ctl;
    int grid_p;           // CTAs of primal_kernel (partials to read)
    double reflection;
    // rows split across chunks: their dx^2 (A^T's rows) and dy^2, dy*delta (A's)
    double *split_p;      // [At's cross-chunk split rows]
    double *split_d;      // [2 * A's cross-chunk split rows]
    int nsplit_p, nsplit_d;
    // panel path of A's long rows (nk_panel.cuh): long row i's run sums are
    // panel_partial[panel_roff[i] .. panel_roff[i+1])
    const double *panel_partial;
    const int64_t *panel_roff;
    int64_t panel_rows;
    int npanels;
};

__device__ __forceinline__ double clampd(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v); // std::clamp
}
__device__ __forceinline__ double max0(double v) { return 0. < v ? v : 0.; } // std::max(0., v)
__device__ __forceinline__ double min0(double v) { return v < 0. ? v : 0.; } // std::min(0., v)

// Combine the segment sums of a split row: called by the lane that finished a
// segment; returns true in the lane that finished the row's last segment, with
// the row's total (init, then the segments in order) in *total.
__device__ __forceinline__ bool split_done(double *slots, unsigned *counters, int4 sg, int64_t vr,
                                           double part, double init, double *total) {
    slots[vr] = part;
    __threadfence();
    if (atomicAdd(&counters[sg.w], 1u) != unsigned(sg.z - 1))
        return false;
    __threadfence();
    double t = init;
    for (int s = 0; s < sg.z; ++s)
        t += __ldcg(slots + sg.y + s);
    counters[sg.w] = 0;
    *total = t;
    return true;
}

// Split-region chunk (all 32 lanes hold segments or padding): every lane
// publishes its segment sum.  The leader lane of a row that lies in this chunk
// adds its segments in order (from init).  For a row spanning chunks, each
// segment sum goes to a slot and the lane whose atomic arrival completes the
// row gets the total: its warp adds the row's slots cooperatively (lane-strided
// partial sums and a fixed shuffle tree, so the result is deterministic).  On
// true, *total holds the completed row of the calling lane.
__device__ __forceinline__ bool split_chunk(double *wpart /* this warp's 32 */, double *slots,
                                           unsigned *counters, int4 sg, int64_t vr, double part,
                                           double init, double *total) {
    const int lane = threadIdx.x & 31;
    wpart[lane] = part;
    __syncwarp();
    bool done = false;
    if (sg.x >= 0 && sg.w < 0 && vr == sg.y) {
        double t = init;
        for (int s = 0; s < sg.z; ++s)
            t += wpart[lane + s];
        *total = t;
        done = true;
    }
    bool last = false;
    if (sg.x >= 0 && sg.w >= 0) {
        slots[vr] = part;
        __threadfence();
        last = atomicAdd(&counters[sg.w], 1u) == unsigned(sg.z - 1);
    }
    unsigned finishers = __ballot_sync(0xffffffffu, last);
    if (finishers)
        __threadfence();
    while (finishers) {
        const int b = __ffs(finishers) - 1;
        finishers &= finishers - 1;
        const int first = __shfl_sync(0xffffffffu, sg.y, b);
        const int nseg = __shfl_sync(0xffffffffu, sg.z, b);
        double acc = 0;
        for (int s = lane; s < nseg; s += 32)
            acc += __ldcg(slots + first + s);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == b) {
            *total = init + acc;
            counters[sg.w] = 0;
            done = true;
        }
    }
    __syncwarp();
    return done;
}

// The split-region work of one lane: dot product of its segment, then the
// chunk combine.  Kept out of line so that the register budget of the kernels'
// main path does not carry it.  init_vec (may be null) gives the row sum's
// start; on true, *row and *total hold the completed row.
// *cross receives the row's counter when the row spans chunks (-1 when it
// lies in this chunk).
template <class Acc, int G = 0, class V, class I, class X>
__device__ __noinline__ bool split_lane(const Sell<V, I> M, int64_t vr, int len,
                                        const X *__restrict__ x, const double *init_vec,
                                        double *wpart, int64_t *row, double *total, int *cross) {
#if NK_SPLIT_PIPE
    const double part = double(sell_dot_pipelined<Acc, kUnrollSplit>(M, vr, len, Acc(0), x));
#else
    const double part = double(sell_dot<Acc, kUnrollSplit, G>(M, vr, len, Acc(0), x));
#endif
    const int4 sg = M.seg[vr];
    *row = sg.x;
    *cross = sg.w;
    const double init = (sg.x >= 0 && init_vec) ? init_vec[sg.x] : 0.;
    return split_chunk(wpart, M.slots, M.counters, sg, vr, part, init, total);
}

// Copies `bytes` rounded up to 16 from global `src` to shared `dst` with the
// CTA's T threads, 16-byte loads, four in flight per thread.  Both addresses
// are 16-byte aligned; the rounding reads at most 15 bytes past the end of
// `src`, which every device buffer of the engine carries as zeroed slack.
template <int T>
__device__ __forceinline__ void stage16(void *dst, const void *src, int64_t bytes) {
    const int4 *s = static_cast<const int4 *>(src);
    int4 *d = static_cast<int4 *>(dst);
    const int64_t n16 = (bytes + 15) >> 4;
    int64_t k = threadIdx.x;
    for (; k + 3 * T < n16; k += 4 * T) {
        const int4 a = __ldcg(s + k), b = __ldcg(s + k + T), c = __ldcg(s + k + 2 * T),
                   e = __ldcg(s + k + 3 * T);
        d[k] = a;
        d[k + T] = b;
        d[k + 2 * T] = c;
        d[k + 3 * T] = e;
    }
    for (; k < n16; k += T)
        d[k] = __ldcg(s + k);
}

// Index of the first SELL chunk of the calling warp and the warp stride of a
// persistent grid.
__device__ __forceinline__ int64_t first_chunk() {
    return (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
}
__device__ __forceinline__ int64_t chunk_stride() {
    return (int64_t(gridDim.x) * blockDim.x) >> 5;
}

// ------------------------------------------------------------------ schedule
// The fused kernels' schedule: CTA b owns the chunks list[off[b] .. off[b+1])
// (chosen on the host by memory work, costliest first) and its warps claim
// them one at a time from a shared counter, so no warp idles while its CTA
// has work left.  A chunk's contribution to the step rule's sums goes to its
// own slot (k, its place in the list), and the CTA adds the slots in list
// order: the sums do not depend on which warp ran which chunk.
struct CtaClaim {
    const int64_t *list;
    int64_t begin;
    int count;
    unsigned *counter; // shared, zeroed before the first claim
    __device__ __forceinline__ bool next(int *k, int64_t *ch) {
        unsigned c = 0;
        if ((threadIdx.x & 31) == 0)
            c = atomicAdd(counter, 1u);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (int(c) >= count)
            return false;
        *k = int(c);
        *ch = list[begin + c];
        return true;
    }
};

// Warp sum in a fixed shuffle tree; result in every lane.
__device__ __forceinline__ double warp_total(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// The CTA's NV sums: slots[k*NV + t] of its `count` chunks added in list
// order by warp 0 (lane-strided, then a fixed tree).  Writes out[t] from
// thread 0.  Called by every thread after a __syncthreads.
template <int NV>
__device__ __forceinline__ void ordered_slots(const double *slots, int count, double *out) {
    if (threadIdx.x >= 32)
        return;
#pragma unroll
    for (int t = 0; t < NV; ++t) {
        double s = 0;
        for (int k = threadIdx.x; k < count; k += 32)
            s += slots[k * NV + t];
        s = warp_total(s);
        if (threadIdx.x == 0)
            out[t] = s;
    }
}

// ------------------------------------------------------------------ primal
// SPLIT: the matrix has split rows (kernels without them skip that path
// entirely, which keeps their register footprint small).  A row split across
// chunks is finished by whichever warp adds its last segment; its dx^2 goes
// to that row's own slot (split_p[counter]), added by the decision in row
// order, so it too lands in the sums the same way every time.
template <class Acc, class V, class I, bool SPARSE_Q, bool FP32G, bool SPLIT>
__global__ void __launch_bounds__(kFusedThreads, kFusedMinBlocks)
    primal_kernel(Sell<V, I> At, QCsr<V, I> Q, Vecs v) {
    __shared__ double wpart[SPLIT ? kFusedWarps : 1][32];
    __shared__ unsigned claim;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    double *slots = reinterpret_cast<double *>(dyn_smem); // one per chunk of this CTA
    const Control &ctl = *v.ctl;
    const int64_t begin = At.coff[blockIdx.x];
    const int count = int(At.coff[blockIdx.x + 1] - begin);
    if (threadIdx.x == 0)
        claim = 0;
    __syncthreads();
    const bool frozen = ctl.restart != 0; // a requested Halpern restart freezes the chunk
    if (!frozen) {
        const int cur = ctl.cur;
        const bool pending = ctl.pending != 0;
        const double pw = ctl.pending_w;
        const double tau = ctl.tau * ctl.factor;
        const double *x = cur ? v.x1 : v.x0;
        double *xt = cur ? v.x0 : v.x1;
        const double *y = cur ? v.y1 : v.y0;
        const float *y32 = cur ? v.y32_1 : v.y32_0;
        // epilogue of column j; g = c_j + (A^T y)_j; returns dx_j^2 (inf if not finite)
        auto finish = [&](int64_t j, double g, double xj, double qj, double lj, double uj,
                          double aj) -> double {
            if (pending)
                v.xa[j] = aj + (xj - aj) * pw;
            if constexpr (SPARSE_Q)
                g = g + (double(q_dot<Acc>(Q, j, x)) + qj * xj);
            double t = (xj - tau * g) / (1 + tau * (SPARSE_Q ? 0. : qj));
            t = clampd(t, lj, uj);
            xt[j] = t;
            const double d = t - xj;
            if constexpr (FP32G)
                v.dx32[j] = float(d);
            else
                v.dx[j] = d;
            return isfinite(t) ? d * d : INFINITY;
        };
        const int lane = threadIdx.x & 31;
        CtaClaim cc{At.clist, begin, count, &claim};
        int k;
        for (int64_t ch; cc.next(&k, &ch);) {
            const int64_t vr = ch * 32 + lane;
            double mine = 0;
            if (vr < At.nv) {
                const int len = At.len[vr];
                if (!SPLIT || vr >= At.nsv) {
                    const int64_t j = vr - At.nsv + At.nsr;
#if NK_PREFETCH // the epilogue's loads do not depend on the dot product: issue them first
                    const double xj = x[j], cj = v.c[j], qj = v.q ? v.q[j] : 0., lj = v.lb[j],
                                 uj = v.ub[j];
                    const double aj = pending ? v.xa[j] : 0.;
#else
                    const double cj = v.c[j];
#endif
                    double g;
                    if constexpr (FP32G)
                        g = cj + double(sell_dot<Acc>(At, vr, len, Acc(0), y32));
                    else // FP64 accumulation starts from c_j, like the CPU loop (src/cpu.cpp:108-111)
                        g = double(sell_dot<Acc>(At, vr, len, Acc(cj), y));
#if NK_PREFETCH
                    mine = finish(j, g, xj, qj, lj, uj, aj);
#else
                    mine = finish(j, g, x[j], v.q ? v.q[j] : 0., v.lb[j], v.ub[j],
                                  pending ? v.xa[j] : 0.);
#endif
                }
            }
            if constexpr (SPLIT) {
                if (ch * 32 < At.nsv) { // split region: the whole warp is here
                    int64_t j;
                    double g;
                    int cross = -1;
                    bool done;
                    if constexpr (FP32G) // FP32 sums add c_j afterwards, in FP64
                        done = split_lane<Acc>(At, vr, At.len[vr], y32, nullptr,
                                               wpart[threadIdx.x >> 5], &j, &g, &cross);
                    else
                        done = split_lane<Acc>(At, vr, At.len[vr], y, v.c,
                                               wpart[threadIdx.x >> 5], &j, &g, &cross);
                    if (done) {
                        if constexpr (FP32G)
                            g = v.c[j] + g;
                        const double d2 = finish(j, g, x[j], v.q ? v.q[j] : 0., v.lb[j], v.ub[j],
                                                 pending ? v.xa[j] : 0.);
                        if (cross >= 0)
                            v.split_p[cross] = d2;
                        else
                            mine = d2;
                    }
                }
            }
            mine = warp_total(mine);
            if (lane == 0)
                slots[k] = mine;
        }
    }
    __syncthreads();
    double tot[1] = {0};
    if (!frozen)
        ordered_slots<1>(slots, count, tot);
    if (threadIdx.x == 0)
        v.part_p[blockIdx.x] = tot[0];
}

// ------------------------------------------------------------------ dual + decide
__device__ inline void decide(Vecs &v, double p, double d, double c) {
    Control &s = *v.ctl;
    const bool adaptive = s.flags & 1, halpern = s.flags & 2, residual_restarts = s.flags & 4;
    if (s.restart != 0) { // a requested Halpern restart freezes the chunk (src/cuda.cu:298-301)
        s.accept = 0;
        return;
    }
    double factor = s.factor;
    double tau = s.tau * factor, sigma = s.sigma * factor;
    double energy = p / tau + d / sigma;
    double limit = fabs(c) > 0 ? energy / (2 * fabs(c)) : INFINITY;
    bool finite = isfinite(energy) && isfinite(c);
    bool accept = finite && (!adaptive || limit >= 1);
    if (adaptive) {
        double k = s.accepted + 2;
        double mult = fmin((1 - pow(k, -.3)) * limit, 1 + pow(k, -.6));
        if (!finite || !isfinite(mult) || mult <= 0)
            mult = .5;
        s.factor = clampd(factor * mult, 1e-12, 1e12);
    }
    s.accept = accept ? 1 : 0;
    s.pending = 0;
    if (accept) {
        s.mass += factor;
        s.accepted += 1;
        s.weight = factor / s.mass;
        if (halpern) {
            double residual = sqrt(fmax(0., energy - 2 * c));
            if (s.epoch == 0)
                s.init_res = residual;
            s.lambda = 1 / (s.epoch + 2);
            s.epoch += 1;
            // integer halving as in the CPU backend (src/cpu.cpp:196)
            double half = double(int64_t(s.accepted) / 2);
            bool req = residual_restarts && s.epoch >= 10 &&
                       (residual <= .2 * s.init_res ||
                        (residual <= .8 * s.init_res && residual > s.prev_res) ||
                        s.epoch >= fmax(10., half));
            s.restart = req ? 1 : 0;
            s.prev_res = residual;
        } else {
            s.cur ^= 1;
            s.pending = 1;
            s.pending_w = s.weight;
        }
    } else
        s.rejected += 1;
}

// PANEL: A's long rows (engine rows [0, v.panel_rows)) come from panel_kernel
// as one partial sum per run (a row's entries in one column panel, or a cut
// of them); the schedule lists them as "combine chunks" (encoded -k-1 for
// rows [32k, 32k+32)) in place of their split-row chunks, and a lane adds its
// row's run sums in slot order (panel by panel, runs in CSR order).
template <class Acc, class V, class I, bool FP32G, bool SPLIT, bool PANEL = false>
__global__ void __launch_bounds__(kFusedThreads, kFusedMinBlocks)
    dual_kernel(Sell<V, I> A, Vecs v) {
    __shared__ double wpart[SPLIT ? kFusedWarps : 1][32];
    __shared__ double red[kFusedWarps * 3];
    __shared__ unsigned claim;
    __shared__ bool last;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    double *slots = reinterpret_cast<double *>(dyn_smem); // two per chunk of this CTA
    const Control &ctl = *v.ctl;
    const int64_t begin = A.coff[blockIdx.x];
    const int count = int(A.coff[blockIdx.x + 1] - begin);
    if (threadIdx.x == 0)
        claim = 0;
    __syncthreads();
    const bool frozen = ctl.restart != 0;
    if (!frozen) {
        const int cur = ctl.cur;
        const bool pending = ctl.pending != 0;
        const double pw = ctl.pending_w;
        const double sigma = ctl.sigma * ctl.factor;
        const double *y = cur ? v.y1 : v.y0;
        double *yt = cur ? v.y0 : v.y1;
        float *yt32 = cur ? v.y32_0 : v.y32_1;
        const double *ax = cur ? v.ax1 : v.ax0;
        double *axt = cur ? v.ax0 : v.ax1;
        // epilogue of row i; adds dy^2 (inf if not finite) and dy * delta
        auto finish = [&](int64_t i, double delta, double yi, double axi, double rli, double rui,
                          double ai, double &dy2, double &cpl) {
            if (pending)
                v.ya[i] = ai + (yi - ai) * pw;
            const double bar = axi + 2 * delta;
            const double z = yi + sigma * bar;
            const double t = max0(z - sigma * rui) + min0(z - sigma * rli);
            yt[i] = t;
            if constexpr (FP32G)
                yt32[i] = float(t);
            axt[i] = axi + delta;
            const double dy = t - yi;
            const bool bad = !isfinite(bar) || !isfinite(t) || !isfinite(delta);
            dy2 = bad ? INFINITY : dy * dy;
            cpl = dy * delta;
        };
        const int lane = threadIdx.x & 31;
        CtaClaim cc{A.clist, begin, count, &claim};
        int k;
        for (int64_t ch; cc.next(&k, &ch);) {
            double dy2 = 0, cpl = 0;
            bool combine = false;
            if constexpr (PANEL) {
                if (ch < 0) { // long rows: their run sums, in slot order
                    combine = true;
                    const int64_t i = (-ch - 1) * 32 + lane;
                    if (i < v.panel_rows) {
                        const double yi = y[i], axi = ax[i], rli = v.rl[i], rui = v.ru[i];
                        const double ai = pending ? v.ya[i] : 0.;
                        const int64_t s0 = v.panel_roff[i], s1 = v.panel_roff[i + 1];
                        const double *pp = v.panel_partial;
                        double delta = 0;
                        int64_t p = s0;
                        constexpr int B = 8; // loads in flight; the adds stay in slot order
                        for (; p + B <= s1; p += B) {
                            double a[B];
#pragma unroll
                            for (int q = 0; q < B; ++q)
                                a[q] = __ldcg(pp + p + q);
#pragma unroll
                            for (int q = 0; q < B; ++q)
                                delta += a[q];
                        }
                        for (; p < s1; ++p)
                            delta += __ldcg(pp + p);
                        finish(i, delta, yi, axi, rli, rui, ai, dy2, cpl);
                    }
                }
            }
            if (!combine) {
                const int64_t vr = ch * 32 + lane;
                if (vr < A.nv && (!SPLIT || vr >= A.nsv)) {
                    const int len = A.len[vr];
                    const int64_t i = vr - A.nsv + A.nsr;
#if NK_PREFETCH
                    const double yi = y[i], axi = ax[i], rli = v.rl[i], rui = v.ru[i];
                    const double ai = pending ? v.ya[i] : 0.;
#endif
                    double delta;
                    if constexpr (FP32G)
                        delta = double(sell_dot<Acc, kUnroll, kDualGather>(A, vr, len, Acc(0),
                                                                         v.dx32));
                    else
                        delta = double(sell_dot<Acc, kUnroll, kDualGather>(A, vr, len, Acc(0),
                                                                         v.dx));
#if NK_PREFETCH
                    finish(i, delta, yi, axi, rli, rui, ai, dy2, cpl);
#else
                    finish(i, delta, y[i], ax[i], v.rl[i], v.ru[i], pending ? v.ya[i] : 0., dy2,
                           cpl);
#endif
                }
                if constexpr (SPLIT) {
                    if (ch * 32 < A.nsv) { // split region: the whole warp is here
                        int64_t i;
                        double delta;
                        int cross = -1;
                        bool done;
                        if constexpr (FP32G)
                            done = split_lane<Acc, kDualGather>(A, vr, A.len[vr], v.dx32, nullptr,
                                                                wpart[threadIdx.x >> 5], &i,
                                                                &delta, &cross);
                        else
                            done = split_lane<Acc, kDualGather>(A, vr, A.len[vr], v.dx, nullptr,
                                                                wpart[threadIdx.x >> 5], &i,
                                                                &delta, &cross);
                        if (done) {
                            double a2, a3;
                            finish(i, delta, y[i], ax[i], v.rl[i], v.ru[i],
                                   pending ? v.ya[i] : 0., a2, a3);
                            if (cross >= 0) {
                                v.split_d[2 * cross] = a2;
                                v.split_d[2 * cross + 1] = a3;
                            } else {
                                dy2 = a2;
                                cpl = a3;
                            }
                        }
                    }
                }
            }
            dy2 = warp_total(dy2);
            cpl = warp_total(cpl);
            if (lane == 0) {
                slots[2 * k] = dy2;
                slots[2 * k + 1] = cpl;
            }
        }
    }
    __syncthreads();
    double tot[2] = {0, 0};
    if (!frozen)
        ordered_slots<2>(slots, count, tot);
    if (threadIdx.x == 0) {
        v.part_d[2 * blockIdx.x] = tot[0];
        v.part_d[2 * blockIdx.x + 1] = tot[1];
        __threadfence();
        unsigned prev = atomicAdd(&v.ctl->arrive, 1u);
        last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!last)
        return;
    // Last CTA: every other CTA of this launch and the whole primal launch are
    // complete; combine partials in index order (deterministic) and decide.
    __threadfence();
    double p = 0, d = 0, c = 0;
    for (int b = threadIdx.x; b < v.grid_p; b += kFusedThreads)
        p += __ldcg(v.part_p + b);
    for (int b = threadIdx.x; b < int(gridDim.x); b += kFusedThreads) {
        d += __ldcg(v.part_d + 2 * b);
        c += __ldcg(v.part_d + 2 * b + 1);
    }
    for (int r = threadIdx.x; r < v.nsplit_p; r += kFusedThreads)
        p += __ldcg(v.split_p + r);
    for (int r = threadIdx.x; r < v.nsplit_d; r += kFusedThreads) {
        d += __ldcg(v.split_d + 2 * r);
        c += __ldcg(v.split_d + 2 * r + 1);
    }
    double r3[3] = {p, d, c};
    cta_sum<3, kFusedWarps>(r3, red);
    if (threadIdx.x == 0) {
        decide(v, r3[0], r3[1], r3[2]);
        v.ctl->arrive = 0;
    }
}

// ------------------------------------------------------------------ Halpern commit
// commit_primal / commit_dual Halpern branches (src/cuda.cu:336-370), written in the
// CPU backend's form (src/cpu.cpp:174-187): T = trial, old = current.
__global__ void halpern_commit(int64_t n, int64_t m, Vecs v, bool fp32g) {
    const Control &s = *v.ctl;
    if (s.accept == 0)
        return;
    int cur = s.cur;
    double lam = s.lambda, r = v.reflection;
    double *x = cur ? v.x1 : v.x0;
    const double *xt = cur ? v.x0 : v.x1;
    double *y = cur ? v.y1 : v.y0;
    const double *yt = cur ? v.y0 : v.y1;
    double *ax = cur ? v.ax1 : v.ax0;
    const double *axt = cur ? v.ax0 : v.ax1;
    float *y32 = cur ? v.y32_1 : v.y32_0;
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += stride) {
        double T = xt[j], old = x[j];
        v.xa[j] = T;
        x[j] = lam * v.anchor_x[j] + (1 - lam) * ((1 + r) * T - r * old);
    }
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += stride) {
        double T = yt[i], old = y[i];
        v.ya[i] = T;
        double ny = lam * v.anchor_y[i] + (1 - lam) * ((1 + r) * T - r * old);
        y[i] = ny;
        if (fp32g)
            y32[i] = float(ny);
        ax[i] = lam * v.anchor_ax[i] + (1 - lam) * ((1 + r) * axt[i] - r * ax[i]);
    }
}

// Fold a pending averaging step into xa / ya (commit of the last accepted trial).
__global__ void flush_average(int64_t n, int64_t m, Vecs v) {
    const Control &s = *v.ctl;
    if (!s.pending)
        return;
    double w = s.pending_w;
    const double *x = s.cur ? v.x1 : v.x0;
    const double *y = s.cur ? v.y1 : v.y0;
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += stride)
        v.xa[j] = v.xa[j] + (x[j] - v.xa[j]) * w;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += stride)
        v.ya[i] = v.ya[i] + (y[i] - v.ya[i]) * w;
}
__global__ void clear_pending(Control *s) { s->pending = 0; }

// ------------------------------------------------------------------ plain SpMV
// out = M x (engine order on both sides, FP64 accumulation): activity rebasing
// and the monitor.
template <class V, class I>
__global__ void __launch_bounds__(kThreads) spmv_kernel(Sell<V, I> M, const double *x,
                                                        double *out) {
    __shared__ double wpart[kWarps][32];
    const int lane = threadIdx.x & 31;
    for (int64_t ch = first_chunk(); ch * 32 < M.nv; ch += chunk_stride()) {
        const int64_t vr = ch * 32 + lane;
        if (vr >= M.nv)
            continue;
        const int len = M.len[vr];
        const double s = sell_dot_pipelined<double>(M, vr, len, 0., x);
        if (vr >= M.nsv) {
            out[vr - M.nsv + M.nsr] = s;
        } else {
            const int4 sg = M.seg[vr];
            double t;
            if (split_chunk(wpart[threadIdx.x >> 5], M.slots, M.counters, sg, vr, s, 0., &t))
                out[sg.x] = t;
        }
    }
}
template <class V, class I>
__global__ void q_spmv_kernel(int64_t n, QCsr<V, I> Q, const double *x, double *out) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride)
        out[r] = q_dot<double>(Q, r, x);
}

// ------------------------------------------------------------------ monitor
// Scaled-space KKT proxy of the reference's monitor_partial / monitor_reduce
// (src/cuda.cu:387-446), one launch with a last-CTA reduction.
__global__ void monitor_kernel(int64_t n, int64_t rows, const double *x, const double *y,
                               const double *ax, const double *aty, const double *qx,
                               const double *c, const double *q, const double *lb,
                               const double *ub, const double *rl, const double *ru, double cscale,
                               double *partial, unsigned *arrive, double *result) {
    __shared__ double red[kWarps * 5];
    __shared__ bool last;
    double pr = 0, du = 0, ob = 0, co = 0, bd = 0;
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    int64_t top = n > rows ? n : rows;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < top; i += stride) {
        if (i < n) {
            double g = c[i] + q[i] * x[i] + aty[i] + (qx ? qx[i] : 0);
            pr = fmax(pr, fmax(0., fmax(lb[i] - x[i], x[i] - ub[i])) / (1 + fabs(x[i])));
            du = fmax(du, fabs(fmin(x[i] - lb[i], fmax(x[i] - ub[i], g))) / cscale);
            double o = c[i] * x[i] + .5 * q[i] * x[i] * x[i] + (qx ? .5 * qx[i] * x[i] : 0);
            ob += o;
            if (g > 0 && isfinite(lb[i]))
                co += fabs(g * (x[i] - lb[i]));
            if (g < 0 && isfinite(ub[i]))
                co += fabs(g * (ub[i] - x[i]));
            if (!isfinite(x[i]) || !isfinite(g) || !isfinite(o))
                bd = 1;
        }
        if (i < rows) {
            if (isfinite(rl[i]))
                pr = fmax(pr, fmax(0., rl[i] - ax[i]) / (1 + fabs(rl[i])));
            if (isfinite(ru[i]))
                pr = fmax(pr, fmax(0., ax[i] - ru[i]) / (1 + fabs(ru[i])));
            if (y[i] != 0) {
                double endpoint = y[i] > 0 ? ru[i] : rl[i];
                if (isfinite(endpoint))
                    co += fabs(y[i] * (endpoint - ax[i]));
                else
                    du = fmax(du, fabs(y[i]));
            }
            if (!isfinite(ax[i]) || !isfinite(y[i]))
                bd = 1;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        pr = fmax(pr, __shfl_xor_sync(0xffffffffu, pr, off));
        du = fmax(du, __shfl_xor_sync(0xffffffffu, du, off));
        bd = fmax(bd, __shfl_xor_sync(0xffffffffu, bd, off));
        ob += __shfl_xor_sync(0xffffffffu, ob, off);
        co += __shfl_xor_sync(0xffffffffu, co, off);
    }
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[w * 5 + 0] = pr;
        red[w * 5 + 1] = du;
        red[w * 5 + 2] = ob;
        red[w * 5 + 3] = co;
        red[w * 5 + 4] = bd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a[5] = {0, 0, 0, 0, 0};
        for (int i = 0; i < kWarps; ++i) {
            a[0] = fmax(a[0], red[i * 5 + 0]);
            a[1] = fmax(a[1], red[i * 5 + 1]);
            a[2] += red[i * 5 + 2];
            a[3] += red[i * 5 + 3];
            a[4] = fmax(a[4], red[i * 5 + 4]);
        }
        for (int t = 0; t < 5; ++t)
            partial[5 * blockIdx.x + t] = a[t];
        __threadfence();
        last = atomicAdd(arrive, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0)
        return;
    __threadfence();
    double a[5] = {0, 0, 0, 0, 0};
    for (unsigned b = 0; b < gridDim.x; ++b) {
        a[0] = fmax(a[0], partial[5 * b + 0]);
        a[1] = fmax(a[1], partial[5 * b + 1]);
        a[2] += partial[5 * b + 2];
        a[3] += partial[5 * b + 3];
        a[4] = fmax(a[4], partial[5 * b + 4]);
    }
    *result = a[4] ? INFINITY : fmax(fmax(a[0], a[1]), a[3] / (1 + fabs(a[2])));
    *arrive = 0;
}

// ------------------------------------------------------------------ setup kernels
__global__ void check_indices(int64_t nnz, const int64_t *idx, const double *val, int64_t cols,
                              int *bad) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz; k += stride)
        if (idx[k] < 0 || idx[k] >= cols || !isfinite(val[k]))
            atomicOr(bad, 1);
}
__global__ void fp32_flags(int64_t nnz, const double *val, int *bad) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        float f = float(val[k]);
        if (!isfinite(f) || (val[k] != 0 && f == 0))
            atomicOr(bad, 1);
    }
}
// Row id of every entry (for the transpose).
__global__ void expand_rows(int64_t rows, const int64_t *ptr, int32_t *rowid) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < rows; i += stride)
        for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
            rowid[k] = int32_t(i);
}
__global__ void iota64(int64_t n, int64_t *a) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride)
        a[k] = k;
}
__global__ void count_cols(int64_t nnz, const int64_t *idx, int64_t *counts) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz; k += stride)
        atomicAdd(reinterpret_cast<unsigned long long *>(counts + idx[k]), 1ull);
}
__global__ void gather_transpose(int64_t nnz, const int64_t *perm, const int32_t *rowid,
                                 const double *val, int64_t *tidx, double *tval) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz; p += stride) {
        int64_t k = perm[p];
        tidx[p] = rowid[k];
        tval[p] = val[k];
    }
}
// Engine-order CSR: new row i = old row perm[i], column indices mapped through
// inv (old column -> engine column); entries keep their order inside a row.
__global__ void permute_csr(int64_t rows, const int64_t *perm, const int64_t *inv,
                            const int64_t *src_ptr, const int64_t *src_idx, const double *src_val,
                            const int64_t *dst_ptr, int64_t *dst_idx, double *dst_val) {
    int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t i = warp; i < rows; i += nwarps) {
        int64_t o = perm[i], b = src_ptr[o], len = src_ptr[o + 1] - b, d = dst_ptr[i];
        for (int64_t k = lane; k < len; k += 32) {
            dst_idx[d + k] = inv[src_idx[b + k]];
            dst_val[d + k] = src_val[b + k];
        }
    }
}
// Engine-order CSR -> SELL-32: virtual row v copies entries [src[v], src[v]+len[v]).
template <class V, class I>
__global__ void fill_sell(int64_t nv, const int64_t *src, const int32_t *len, const int64_t *cptr,
                          const int64_t *cidx, const double *cval, I *idx, V *val) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < nv; v += stride) {
        int64_t base = cptr[v >> 5] + (v & 31), s = src[v];
        for (int k = 0; k < len[v]; ++k) {
            idx[base + int64_t(k) * 32] = I(cidx[s + k]);
            val[base + int64_t(k) * 32] = V(cval[s + k]);
        }
    }
}
template <class V, class I>
__global__ void convert_csr(int64_t nnz, const int64_t *cidx, const double *cval, I *idx, V *val) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        idx[k] = I(cidx[k]);
        val[k] = V(cval[k]);
    }
}
// out[i] = in[perm[i]]  (caller order -> engine order)
__global__ void gather_vec(int64_t n, const int64_t *perm, const double *in, double *out) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = in[perm[i]];
}
// out[perm[i]] = in[i]  (engine order -> caller order)
__global__ void scatter_vec(int64_t n, const int64_t *perm, const double *in, double *out) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[perm[i]] = in[i];
}
__global__ void to_float(int64_t n, const double *src, float *dst) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride)
        dst[k] = float(src[k]);
}

} // namespace nk
