// Device side of the batched PDHG engine: many independent LP / convex-QP
// instances advanced together, each with its own step sizes, acceptance state,
// restarts and termination flag.
//
// Layout.  Every instance keeps its own SELL-32 matrices (A and A^T, engine
// order inside the instance: rows sorted by length) and vectors in its own
// device allocation, described by one BInst record.  The batch is the block
// diagonal of all instances, but it is never packed into one matrix: the
// kernels walk work lists of (instance, chunk) pairs instead, so an instance
// joins or leaves the batch by editing a list, not by repacking matrices.
// A chunk never spans two instances, so each warp works for exactly one
// instance and its sums are per-instance without atomics: one partial per
// chunk, combined in list order by the per-instance decision (deterministic).
//
// One PDHG trial of the whole batch is three launches: batch_primal (A^T y,
// projected primal step), batch_dual (A dx, interval prox) and batch_decide
// (one warp per instance: the acceptance rule and step-size update of
// src/cuda.cu:285-335, i.e. the single engine's decide() without Halpern).
#pragma once

namespace nk {

struct BInst {
    // matrices: SELL-32 chunk offsets, row lengths, int32 indices, values (V)
    const int64_t *a_cptr, *t_cptr;
    const int32_t *a_len, *t_len, *a_idx, *t_idx;
    const float *a_val, *t_val;       // FP32 values (MIXED batches), else null
    const double *a_val64, *t_val64;  // FP64 values (always present)
    const int64_t *q_ptr; // Q in CSR (engine order), null for none
    const int32_t *q_idx;
    const float *q_val;
    const double *q_val64;
    const double *c, *q, *lb, *ub, *rl, *ru; // q: null when the diagonal is all zero
    double *x[2], *y[2], *ax[2], *xa, *ya, *dx;
    // evaluation: original-space constants and work vectors
    const double *cs, *olb, *oub, *rs, *shift, *orl, *oru;
    double *e_ax, *e_aty[2], *e_qx, *best_x, *best_y, *epoch_x, *epoch_y;
    int32_t n, m; // real columns / rows (chunks cover them padded to 32)
    double os, cscale;
};

struct BCtl { // per instance; the first fields mirror Control (nk_device.cuh)
    double factor, mass, accepted, rejected, accept, weight, tau, sigma, pending_w;
    int cur, pending, adaptive, active;
    int fp64; // 1: trials use the FP64 values (FP64 batches, and the refinement phase)
};

// Work item of the trial kernels: a run of `count` consecutive chunks of one
// instance starting at `chunk`, whose partial sums go to part, part+1, ...
// (partials are instance-contiguous).  A run shares one descriptor fetch.
// Items are placed on CTAs on the host by estimated memory work (runs of
// consecutive items of equal work, a few per CTA; CTA b owns list entries
// [coff[b], coff[b+1]), in instance and chunk order), and a CTA's warps claim
// its items from a shared counter, so every SM finishes its share at about
// the same time.
// Where an item runs changes no result: its partials have fixed slots.
struct BWork {
    int inst, chunk, part, count;
};

// CTA size bound of the trial kernels: every variant keeps 1024 threads of
// one SM resident (64 registers a thread), so a grid of sms * 1024 / threads
// CTAs is resident at once.
constexpr int kBatchMaxThreads = 512;

// The warp's next item of its CTA's list (lane 0 claims; false when the list
// is done).
__device__ __forceinline__ bool claim_item(unsigned *next, int count, int *w) {
    unsigned k = 0;
    if ((threadIdx.x & 31) == 0)
        k = atomicAdd(next, 1u);
    k = __shfl_sync(0xffffffffu, k, 0);
    *w = int(k);
    return int(k) < count;
}

// Sequential dot of row r of a SELL matrix (32-row chunks, column-major)
// starting from acc; U loads in flight per lane.
template <class Acc, class V, int U, class X>
__device__ __forceinline__ Acc bsell_dot(const int64_t *cptr, const int32_t *idx, const V *val,
                                         int r, int len, Acc acc, const X *__restrict__ x) {
    const int64_t base = cptr[r >> 5] + (r & 31);
    const int32_t *ip = idx + base;
    const V *vp = val + base;
    int k = 0;
    for (; k + U <= len; k += U) {
        int32_t j[U];
        V w[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            j[u] = stream_load(ip + int64_t(k + u) * 32);
            w[u] = stream_load(vp + int64_t(k + u) * 32);
        }
        X g[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            g[u] = gather_load(x + j[u]);
#pragma unroll
        for (int u = 0; u < U; ++u)
            acc = acc + Acc(w[u]) * Acc(g[u]);
    }
    for (; k < len; ++k)
        acc = acc + Acc(stream_load(vp + int64_t(k) * 32)) *
                        Acc(gather_load(x + stream_load(ip + int64_t(k) * 32)));
    return acc;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// ------------------------------------------------------------------ trial
// A SELL row dot with the instance's values in its current precision
// (warp-uniform: a chunk belongs to one instance).
template <int U>
__device__ __forceinline__ double inst_dot(bool f64, const int64_t *cptr, const int32_t *idx,
                                           const float *v32, const double *v64, int r, int len,
                                           double acc, const double *__restrict__ x) {
    return f64 ? bsell_dot<double, double, U>(cptr, idx, v64, r, len, acc, x)
               : bsell_dot<double, float, U>(cptr, idx, v32, r, len, acc, x);
}

// Q row products of one chunk (columns j of lanes), summed by the lane itself
// for rows of at most 32 entries and by the whole warp (lane-strided partial
// sums, fixed shuffle tree) for longer rows, so that no lane walks a long row
// alone.  Every lane of the warp must call it.
__device__ __forceinline__ double chunk_q(const BInst &I, bool f64, int j, bool valid,
                                          const double *__restrict__ x) {
    const int lane = threadIdx.x & 31;
    const int64_t b = valid ? I.q_ptr[j] : 0, e = valid ? I.q_ptr[j + 1] : 0;
    const bool longrow = e - b > 32;
    double qa = 0;
    if (!longrow)
        for (int64_t k = b; k < e; ++k)
            qa += (f64 ? I.q_val64[k] : double(I.q_val[k])) * x[I.q_idx[k]];
    unsigned todo = __ballot_sync(0xffffffffu, longrow);
    while (todo) {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        const int64_t sb = __shfl_sync(0xffffffffu, b, src), se = __shfl_sync(0xffffffffu, e, src);
        double part = 0;
        for (int64_t k = sb + lane; k < se; k += 32)
            part += (f64 ? I.q_val64[k] : double(I.q_val[k])) * x[I.q_idx[k]];
        part = warp_sum(part);
        if (lane == src)
            qa = part;
    }
    return qa;
}

// part[w.part + k] = sum dx^2 of chunk k of the run.  With `probe` (the
// autotuner's timed trials) a pending average is left pending: the launch then
// writes only the trial buffers, dx and the partials, which the next trial
// overwrites, so it leaves no trace in any instance's trajectory.
template <int U>
__global__ void __launch_bounds__(kBatchMaxThreads, 1024 / kBatchMaxThreads)
    batch_primal(const BInst *__restrict__ ins, const BCtl *__restrict__ ctl,
                 const BWork *__restrict__ work, const int *__restrict__ coff, double *part,
                 int probe) {
    __shared__ unsigned next;
    const int lane = threadIdx.x & 31;
    const int begin = coff[blockIdx.x], count = coff[blockIdx.x + 1] - begin;
    if (threadIdx.x == 0)
        next = 0;
    __syncthreads();
    for (int w; claim_item(&next, count, &w);) {
        const BWork it = work[begin + w];
        const BCtl &s = ctl[it.inst];
        if (!s.active) {
            if (lane < it.count)
                part[it.part + lane] = 0;
            continue;
        }
        const BInst &I = ins[it.inst];
        const bool f64 = s.fp64 != 0;
        const int cur = s.cur, n = I.n;
        const double tau = s.tau * s.factor, pw = s.pending_w;
        const bool pending = s.pending != 0 && !probe, sq = I.q_ptr != nullptr;
        const double *x = I.x[cur], *y = I.y[cur];
        double *xt = I.x[cur ^ 1];
        for (int k = 0; k < it.count; ++k) {
            const int j = (it.chunk + k) * 32 + lane;
            const bool valid = j < n;
            const double qa = sq ? chunk_q(I, f64, j, valid, x) : 0.;
            double mine = 0;
            if (valid) {
                const double xj = x[j], cj = I.c[j], qj = I.q ? I.q[j] : 0., lj = I.lb[j],
                             uj = I.ub[j];
                const double aj = pending ? I.xa[j] : 0.;
                // FP64 accumulation starts from c_j, like the CPU loop (src/cpu.cpp:108-111)
                double g = inst_dot<U>(f64, I.t_cptr, I.t_idx, I.t_val, I.t_val64, j, I.t_len[j],
                                       cj, y);
                if (pending)
                    I.xa[j] = aj + (xj - aj) * pw;
                if (sq)
                    g = g + (qa + qj * xj);
                double t = (xj - tau * g) / (1 + tau * (sq ? 0. : qj));
                t = t < lj ? lj : (uj < t ? uj : t);
                xt[j] = t;
                const double d = t - xj;
                I.dx[j] = d;
                mine = isfinite(t) ? d * d : INFINITY;
            }
            mine = warp_sum(mine);
            if (lane == 0)
                part[it.part + k] = mine;
        }
    }
}

// part[2 (w.part + k)] = sum dy^2, part[2 (w.part + k) + 1] = sum dy * delta.
// `probe` as for batch_primal.
template <int U>
__global__ void __launch_bounds__(kBatchMaxThreads, 1024 / kBatchMaxThreads)
    batch_dual(const BInst *__restrict__ ins, const BCtl *__restrict__ ctl,
               const BWork *__restrict__ work, const int *__restrict__ coff, double *part,
               int probe) {
    __shared__ unsigned next;
    const int lane = threadIdx.x & 31;
    const int begin = coff[blockIdx.x], count = coff[blockIdx.x + 1] - begin;
    if (threadIdx.x == 0)
        next = 0;
    __syncthreads();
    for (int w; claim_item(&next, count, &w);) {
        const BWork it = work[begin + w];
        const BCtl &s = ctl[it.inst];
        if (!s.active) {
            if (lane < it.count) {
                part[2 * (it.part + lane)] = 0;
                part[2 * (it.part + lane) + 1] = 0;
            }
            continue;
        }
        const BInst &I = ins[it.inst];
        const bool f64 = s.fp64 != 0;
        const int cur = s.cur, m = I.m;
        const double sigma = s.sigma * s.factor, pw = s.pending_w;
        const bool pending = s.pending != 0 && !probe;
        const double *y = I.y[cur], *ax = I.ax[cur];
        double *yt = I.y[cur ^ 1], *axt = I.ax[cur ^ 1];
        for (int k = 0; k < it.count; ++k) {
            const int i = (it.chunk + k) * 32 + lane;
            double dy2 = 0, cpl = 0;
            if (i < m) {
                const double yi = y[i], axi = ax[i], rli = I.rl[i], rui = I.ru[i];
                const double ai = pending ? I.ya[i] : 0.;
                const double delta = inst_dot<U>(f64, I.a_cptr, I.a_idx, I.a_val, I.a_val64, i,
                                                 I.a_len[i], 0., I.dx);
                if (pending)
                    I.ya[i] = ai + (yi - ai) * pw;
                const double bar = axi + 2 * delta;
                const double z = yi + sigma * bar;
                const double t = max0(z - sigma * rui) + min0(z - sigma * rli);
                yt[i] = t;
                axt[i] = axi + delta;
                const double dy = t - yi;
                const bool bad = !isfinite(bar) || !isfinite(t) || !isfinite(delta);
                dy2 = bad ? INFINITY : dy * dy;
                cpl = dy * delta;
            }
            dy2 = warp_sum(dy2);
            cpl = warp_sum(cpl);
            if (lane == 0) {
                part[2 * (it.part + k)] = dy2;
                part[2 * (it.part + k) + 1] = cpl;
            }
        }
    }
}

// One warp per active instance: combine its chunk partials in list order and
// apply the acceptance rule (decide() of nk_device.cuh without Halpern).
__global__ void batch_decide(BCtl *ctl, const int *__restrict__ slots, int nslots,
                             const int *col_first, const int *col_count, const int *row_first,
                             const int *row_count, const double *part_p, const double *part_d) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int k = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); k < nslots; k += warps) {
        const int b = slots[k];
        double p = 0, d = 0, c = 0;
        for (int t = lane; t < col_count[k]; t += 32)
            p += part_p[col_first[k] + t];
        for (int t = lane; t < row_count[k]; t += 32) {
            d += part_d[2 * (row_first[k] + t)];
            c += part_d[2 * (row_first[k] + t) + 1];
        }
        p = warp_sum(p);
        d = warp_sum(d);
        c = warp_sum(c);
        if (lane != 0)
            continue;
        BCtl &s = ctl[b];
        if (!s.active)
            continue;
        const double factor = s.factor;
        const double tau = s.tau * factor, sigma = s.sigma * factor;
        const double energy = p / tau + d / sigma;
        const double limit = fabs(c) > 0 ? energy / (2 * fabs(c)) : INFINITY;
        const bool finite = isfinite(energy) && isfinite(c);
        const bool accept = finite && (!s.adaptive || limit >= 1);
        if (s.adaptive) {
            const double kk = s.accepted + 2;
            double mult = fmin((1 - pow(kk, -.3)) * limit, 1 + pow(kk, -.6));
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
            s.cur ^= 1;
            s.pending = 1;
            s.pending_w = s.weight;
        } else
            s.rejected += 1;
    }
}

// ------------------------------------------------------------------ element work
// Per-element operations of the host driver (off the trial path).  Work items
// are the same (instance, chunk) pairs; `op` selects what the lane does with
// column j (column lists) or row i (row lists).

// Fold a pending averaging step into xa / ya (flush before candidates).
__global__ void batch_flush(const BInst *ins, const BCtl *ctl, const int2 *cols, int ncols,
                            const int2 *rows, int nrows) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int w = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); w < ncols + nrows;
         w += warps) {
        const bool col = w < ncols;
        const int2 it = col ? cols[w] : rows[w - ncols];
        const BCtl &s = ctl[it.x];
        if (!s.active || !s.pending)
            continue;
        const BInst &I = ins[it.x];
        const int e = it.y * 32 + lane;
        if (col && e < I.n)
            I.xa[e] = I.xa[e] + (I.x[s.cur][e] - I.xa[e]) * s.pending_w;
        if (!col && e < I.m)
            I.ya[e] = I.ya[e] + (I.y[s.cur][e] - I.ya[e]) * s.pending_w;
    }
}
__global__ void batch_clear_pending(BCtl *ctl, const int *slots, int nslots) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nslots; k += gridDim.x * blockDim.x)
        ctl[slots[k]].pending = 0;
}

// Which vector an element kernel reads: the current iterate, the average,
// the best point or the epoch (restart anchor) point.
enum BSrc : int { kCur = 0, kAvg = 1, kBest = 2, kEpoch = 3 };
__device__ __forceinline__ const double *bsrc_x(const BInst &I, const BCtl &s, int src) {
    return src == kCur ? I.x[s.cur] : src == kAvg ? I.xa : src == kBest ? I.best_x : I.epoch_x;
}
__device__ __forceinline__ const double *bsrc_y(const BInst &I, const BCtl &s, int src) {
    return src == kCur ? I.y[s.cur] : src == kAvg ? I.ya : src == kBest ? I.best_y : I.epoch_y;
}

// Products of a source point with the FP64 matrices (evaluation is always in
// FP64, whatever precision the trials use) for the instances with mask[b] != 0:
// e_ax = A x (row lists), e_aty[slot] = A^T y (column lists), e_qx = Q x
// (column lists, QP instances).
__global__ void batch_products(const BInst *ins, const BCtl *ctl, const int *mask, int src,
                               int slot, const int2 *cols, int ncols, const int2 *rows, int nrows) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int w = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); w < ncols + nrows;
         w += warps) {
        const bool col = w < ncols;
        const int2 it = col ? cols[w] : rows[w - ncols];
        if (!mask[it.x])
            continue;
        const BInst &I = ins[it.x];
        const BCtl &s = ctl[it.x];
        const int e = it.y * 32 + lane;
        if (col && e < I.n) {
            I.e_aty[slot][e] = bsell_dot<double, double, 4>(I.t_cptr, I.t_idx, I.t_val64, e,
                                                            I.t_len[e], 0., bsrc_y(I, s, src));
            if (I.q_ptr) {
                const double *x = bsrc_x(I, s, src);
                double qa = 0;
                for (int64_t k = I.q_ptr[e]; k < I.q_ptr[e + 1]; ++k)
                    qa += I.q_val64[k] * x[I.q_idx[k]];
                I.e_qx[e] = qa;
            }
        }
        if (!col && e < I.m)
            I.e_ax[e] = bsell_dot<double, double, 4>(I.a_cptr, I.a_idx, I.a_val64, e, I.a_len[e],
                                                     0., bsrc_x(I, s, src));
    }
}

// Original-space KKT terms of Verifier::evaluate for one source point per
// instance, one partial row of kBatchKkt values per work item (the meaning of
// values 0-9 is kkt_partial's in nk_solve.cuh), plus the Farkas screen of the
// point's dual: 10 ray impossible (max), 11 + 12 the FP64 feasibility bound,
// 13 its magnitude.
constexpr int kBatchKkt = 14;
constexpr unsigned kBatchKktMax = 0x70fu;
__global__ void batch_kkt(const BInst *ins, const BCtl *ctl, const int *mask, int src, int slot,
                          const int2 *cols, int ncols, const int2 *rows, int nrows, double *part) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int w = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); w < ncols + nrows;
         w += warps) {
        const bool col = w < ncols;
        const int2 it = col ? cols[w] : rows[w - ncols];
        double v[kBatchKkt] = {};
        if (mask[it.x]) {
            const BInst &I = ins[it.x];
            const BCtl &s = ctl[it.x];
            const int e = it.y * 32 + lane;
            if (col && e < I.n) {
                const double *xp = bsrc_x(I, s, src);
                const double cj = I.cs[e], xs = xp[e], xo = xs * cj;
                const double lo = I.olb[e], hi = I.oub[e];
                const double viol = fmax(0., fmax(lo - xo, xo - hi));
                v[0] = viol / (1 + fabs(xo));
                v[1] = viol;
                const double f = I.os / cj;
                const double qxs = I.q_ptr ? I.e_qx[e] : 0.;
                const double aty = I.e_aty[slot][e];
                const double lin = (I.c[e] + aty) * f;
                const double qe = I.q ? I.q[e] : 0.;
                const double curv = (qe * xs + qxs) * f;
                const double g = lin + curv;
                v[4] = I.c[e] * xs + .5 * qe * xs * xs + .5 * xs * qxs;
                if (!isfinite(lin) || !isfinite(g) || !isfinite(xo))
                    v[9] = 1;
                const double d = clampd(g, xo - hi, xo - lo);
                v[3] = fabs(d);
                v[2] = fabs(d) / I.cscale;
                if (g > 0 && isfinite(lo))
                    v[5] += fabs(g * (xo - lo));
                if (g < 0 && isfinite(hi))
                    v[5] += fabs(g * (hi - xo));
                double arg;
                if (I.q_ptr) {
                    arg = g > 0 ? lo : g < 0 ? hi : clampd(0., lo, hi);
                    if (!isfinite(arg))
                        v[8] = 1;
                    else
                        v[7] = g * arg - curv * xo / 2;
                } else {
                    const double qo = qe * f / cj;
                    arg = qo > 0 ? clampd(-lin / qo, lo, hi) : lin > 0 ? lo : lin < 0 ? hi
                                                                                    : clampd(0., lo, hi);
                    if (!isfinite(arg))
                        v[8] = 1;
                    else
                        v[7] = lin * arg + .5 * qo * arg * arg;
                }
                const double gy = aty * f; // (A^T y)_j in caller units
                if (gy != 0) {
                    const double b = gy > 0 ? lo : hi;
                    if (!isfinite(b))
                        v[10] = 1;
                    else {
                        v[12] = gy * b;
                        v[13] = fabs(gy * b);
                    }
                }
            }
            if (!col && e < I.m) {
                const double r = I.rs[e], yo = bsrc_y(I, s, src)[e] * r * I.os;
                const double axo = I.e_ax[e] / r + I.shift[e];
                const double lo = I.orl[e], hi = I.oru[e];
                if (isfinite(lo))
                    v[0] = fmax(v[0], fmax(0., lo - axo) / (1 + fabs(lo)));
                if (isfinite(hi))
                    v[0] = fmax(v[0], fmax(0., axo - hi) / (1 + fabs(hi)));
                v[1] = fmax(0., fmax(lo - axo, axo - hi));
                if (yo != 0) {
                    const double ep = yo > 0 ? hi : lo;
                    if (isfinite(ep)) {
                        v[6] = yo * ep;
                        v[5] += fabs(yo * (ep - axo));
                        v[11] = -yo * ep;
                        v[13] = fabs(yo * ep);
                    } else {
                        v[8] = 1;
                        v[10] = 1;
                        v[3] = fabs(yo);
                        v[2] = fabs(yo);
                    }
                    v[7] += yo * I.shift[e];
                }
                if (!isfinite(axo) || !isfinite(yo))
                    v[9] = 1;
            }
        }
#pragma unroll
        for (int t = 0; t < kBatchKkt; ++t)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double o = __shfl_xor_sync(0xffffffffu, v[t], off);
                v[t] = (kBatchKktMax >> t & 1) ? fmax(v[t], o) : v[t] + o;
            }
        if (lane == 0)
            for (int t = 0; t < kBatchKkt; ++t)
                part[int64_t(w) * kBatchKkt + t] = v[t];
    }
}

// sum (x - epoch_x)^2 and (y - epoch_y)^2 of each masked instance's source
// point src_of[b]: part[2w], part[2w+1].
__global__ void batch_displacement(const BInst *ins, const BCtl *ctl, const int *mask,
                                   const int *src_of, const int2 *cols, int ncols,
                                   const int2 *rows, int nrows, double *part) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int w = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); w < ncols + nrows;
         w += warps) {
        const bool col = w < ncols;
        const int2 it = col ? cols[w] : rows[w - ncols];
        double dx = 0, dy = 0;
        if (mask[it.x]) {
            const BInst &I = ins[it.x];
            const BCtl &s = ctl[it.x];
            const int e = it.y * 32 + lane;
            const int src = src_of[it.x];
            if (col && e < I.n) {
                const double d = bsrc_x(I, s, src)[e] - I.epoch_x[e];
                dx = d * d;
            }
            if (!col && e < I.m) {
                const double d = bsrc_y(I, s, src)[e] - I.epoch_y[e];
                dy = d * d;
            }
        }
        dx = warp_sum(dx);
        dy = warp_sum(dy);
        if (lane == 0) {
            part[2 * w] = dx;
            part[2 * w + 1] = dy;
        }
    }
}

// Combine per-item partial rows (NV values) of each listed instance in list
// order: out[k * NV + t]; one warp per instance.
template <int NV>
__global__ void batch_finish(const int *col_first, const int *col_count, int ncols_total,
                             const int *row_first, const int *row_count, int nslots,
                             unsigned max_mask, const double *part, double *out) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int k = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); k < nslots; k += warps) {
        double v[NV];
#pragma unroll
        for (int t = 0; t < NV; ++t)
            v[t] = 0;
        auto take = [&](int item) {
#pragma unroll
            for (int t = 0; t < NV; ++t) {
                const double p = part[int64_t(item) * NV + t];
                v[t] = (max_mask >> t & 1) ? fmax(v[t], p) : v[t] + p;
            }
        };
        for (int t = lane; t < col_count[k]; t += 32)
            take(col_first[k] + t);
        for (int t = lane; t < row_count[k]; t += 32)
            take(ncols_total + row_first[k] + t);
#pragma unroll
        for (int t = 0; t < NV; ++t)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double o = __shfl_xor_sync(0xffffffffu, v[t], off);
                v[t] = (max_mask >> t & 1) ? fmax(v[t], o) : v[t] + o;
            }
        if (lane == 0)
#pragma unroll
            for (int t = 0; t < NV; ++t)
                out[int64_t(k) * NV + t] = v[t];
    }
}

// Copies a source point into best (op 0) or epoch (op 1) for masked instances.
__global__ void batch_keep(const BInst *ins, const BCtl *ctl, const int *mask, const int *src_of,
                           int op, const int2 *cols, int ncols, const int2 *rows, int nrows) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int w = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); w < ncols + nrows;
         w += warps) {
        const bool col = w < ncols;
        const int2 it = col ? cols[w] : rows[w - ncols];
        if (!mask[it.x])
            continue;
        const BInst &I = ins[it.x];
        const BCtl &s = ctl[it.x];
        const int e = it.y * 32 + lane;
        const int src = src_of[it.x];
        if (col && e < I.n)
            (op ? I.epoch_x : I.best_x)[e] = bsrc_x(I, s, src)[e];
        if (!col && e < I.m)
            (op ? I.epoch_y : I.best_y)[e] = bsrc_y(I, s, src)[e];
    }
}

// Restart of masked instances from their current, averaged or best point:
// the candidate becomes the iterate, averages restart from zero
// (reset_candidate, src/cuda.cu:892-930).  The activity A x is recomputed by
// the row pass from the new iterate (after the column pass, in a second
// launch), with the values the instance's trials use.
__global__ void batch_restart_cols(const BInst *ins, BCtl *ctl, const int *mask, const int *src_of,
                                   const int2 *cols, int ncols, const int2 *rows, int nrows) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int w = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); w < ncols + nrows;
         w += warps) {
        const bool col = w < ncols;
        const int2 it = col ? cols[w] : rows[w - ncols];
        if (!mask[it.x])
            continue;
        const BInst &I = ins[it.x];
        const BCtl &s = ctl[it.x];
        const int e = it.y * 32 + lane;
        const int src = src_of[it.x];
        if (col && e < I.n) {
            if (src != kCur)
                I.x[s.cur][e] = bsrc_x(I, s, src)[e];
            I.xa[e] = 0;
        }
        if (!col && e < I.m) {
            if (src != kCur)
                I.y[s.cur][e] = bsrc_y(I, s, src)[e];
            I.ya[e] = 0;
        }
    }
}
__global__ void batch_restart_rows(const BInst *ins, const BCtl *ctl, const int *mask,
                                   const int2 *rows, int nrows) {
    const int lane = threadIdx.x & 31;
    const int warps = int((int64_t(gridDim.x) * blockDim.x) >> 5);
    for (int w = int((int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); w < nrows; w += warps) {
        const int2 it = rows[w];
        if (!mask[it.x])
            continue;
        const BInst &I = ins[it.x];
        const BCtl &s = ctl[it.x];
        const int e = it.y * 32 + lane;
        if (e < I.m)
            I.ax[s.cur][e] = inst_dot<4>(s.fp64 != 0, I.a_cptr, I.a_idx, I.a_val, I.a_val64, e,
                                         I.a_len[e], 0., I.x[s.cur]);
    }
}
// Control side of a restart; mask 2 also starts the FP64 refinement phase of
// a reduced-precision instance: fresh step-size state, as a new FP64 engine
// would have (the reference's mixed-precision refinement restarts PDHG).
__global__ void batch_restart_ctl(BCtl *ctl, const int *mask, const int *slots, int nslots) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nslots; k += gridDim.x * blockDim.x) {
        const int b = slots[k];
        if (mask[b]) {
            ctl[b].pending = 0;
            ctl[b].mass = 0;
        }
        if (mask[b] == 2) {
            ctl[b].fp64 = 1;
            ctl[b].factor = 1;
            ctl[b].accepted = 0;
            ctl[b].weight = 0;
            ctl[b].accept = 0;
        }
    }
}

} // namespace nk
