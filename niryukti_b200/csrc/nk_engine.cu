// B200 PDHG iteration engine: the replacement for the reference's CudaBackend
// (src/cuda.cu:565-950) behind the IterationBackend seam (src/internal.hpp:102-134).
//
// One PDHG trial is two kernels:
//   primal_kernel  g = c + A^T y (+ Q x + q.x)      -- CSR SpMV over the explicit transpose
//                  trial x = clamp((x - tau g)/(1 + tau q), lb, ub), dx, sum dx^2
//                  (restates primal_trial, src/cuda.cu:240-260, and the CPU loop
//                   src/cpu.cpp:107-132, fused into the SpMV epilogue)
//   dual_kernel    delta = A dx                      -- CSR SpMV
//                  trial y = interval prox of y + sigma (Ax + 2 delta), Ax + delta,
//                  sum dy^2, sum dy*delta            (dual_trial, src/cuda.cu:261-284;
//                                                     src/cpu.cpp:136-150)
//                  and, in its last CTA, the accept / step-factor / averaging decision
//                  (decide, src/cuda.cu:285-335; src/cpu.cpp:151-216)
// Iterates are double-buffered: accepting a trial flips a device-side index, and the
// running-average update of an accepted step is applied by the next trial's kernels
// (commit_primal / commit_dual, src/cuda.cu:336-370, without their own passes).
// The Halpern variant keeps a separate commit kernel.
#include "nk_common.cuh"
#include "nk_kernels.cuh"
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

namespace nk {

thread_local char g_last_error[2048] = {};
void set_last_error(const char *what) { std::snprintf(g_last_error, sizeof(g_last_error), "%s", what); }

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
    double *dx;        // primal displacement (FP64 gather source)
    float *dx32;       // FP32 gather source (precision FP32)
    float *y32_0, *y32_1; // FP32 copies of y (precision FP32)
    double *anchor_x, *anchor_y, *anchor_ax;
    double *part_p;    // per-CTA sum dx^2 of primal_kernel
    double *part_d;    // per-CTA (sum dy^2, sum dy*delta) of dual_kernel
    Control *ctl;
    int grid_p;        // CTAs of primal_kernel (partials to read)
    double reflection;
};

__device__ __forceinline__ double clampd(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v); // std::clamp
}
__device__ __forceinline__ double max0(double v) { return 0. < v ? v : 0.; } // std::max(0., v)
__device__ __forceinline__ double min0(double v) { return v < 0. ? v : 0.; } // std::min(0., v)

// ------------------------------------------------------------------ primal
template <class Acc, class V, class P, class I, bool SPARSE_Q, bool FP32G>
__global__ void __launch_bounds__(kThreads) primal_kernel(Csr<V, P, I> At, Schedule S,
                                                          Csr<V, P, I> Q, Schedule /*unused*/,
                                                          Vecs v) {
    __shared__ double red[kWarps];
    __shared__ Acc qred[kWarps];
    const Control &ctl = *v.ctl;
    double mine = 0;
    bool bad = false;
    if (ctl.restart == 0) {
        const int cur = ctl.cur;
        const bool pending = ctl.pending != 0;
        const double pw = ctl.pending_w;
        const double tau = ctl.tau * ctl.factor;
        const double *x = cur ? v.x1 : v.x0;
        double *xt = cur ? v.x0 : v.x1;
        const double *y = cur ? v.y1 : v.y0;
        const float *y32 = cur ? v.y32_1 : v.y32_0;
        auto body = [&](int64_t j, Acc s, bool leader, bool valid, auto group, int lane) {
            constexpr int G = decltype(group)::value;
            Acc qs = Acc(0);
            if constexpr (SPARSE_Q) {
                if constexpr (G == kThreads)
                    qs = cta_dot<Acc>(Q, j, x, qred);
                else
                    qs = group_dot<G, Acc>(Q, j, valid, x, lane);
            }
            if (!leader)
                return;
            double xj = x[j];
            if (pending) {
                double a = v.xa[j];
                v.xa[j] = a + (xj - a) * pw;
            }
            double g = v.c[j] + double(s);
            double qj = v.q[j];
            if constexpr (SPARSE_Q)
                g = g + (double(qs) + qj * xj);
            double t = (xj - tau * g) / (1 + tau * (SPARSE_Q ? 0. : qj));
            t = clampd(t, v.lb[j], v.ub[j]);
            xt[j] = t;
            double d = t - xj;
            if constexpr (FP32G)
                v.dx32[j] = float(d);
            else
                v.dx[j] = d;
            mine += d * d;
            bad |= !isfinite(t);
        };
        if constexpr (FP32G)
            sweep<Acc>(At, S, y32, body);
        else
            sweep<Acc>(At, S, y, body);
    }
    double tot[1] = {bad ? INFINITY : mine};
    cta_sum<1>(tot, red);
    if (threadIdx.x == 0)
        v.part_p[blockIdx.x] = tot[0];
}

// ------------------------------------------------------------------ dual + decide
__device__ void decide(Vecs &v, double p, double d, double c) {
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

template <class Acc, class V, class P, class I, bool FP32G>
__global__ void __launch_bounds__(kThreads) dual_kernel(Csr<V, P, I> A, Schedule S, Vecs v) {
    __shared__ double red[kWarps * 3];
    __shared__ bool last;
    const Control &ctl = *v.ctl;
    double dy2 = 0, cpl = 0;
    bool bad = false;
    if (ctl.restart == 0) {
        const int cur = ctl.cur;
        const bool pending = ctl.pending != 0;
        const double pw = ctl.pending_w;
        const double sigma = ctl.sigma * ctl.factor;
        const double *y = cur ? v.y1 : v.y0;
        double *yt = cur ? v.y0 : v.y1;
        float *yt32 = cur ? v.y32_0 : v.y32_1;
        const double *ax = cur ? v.ax1 : v.ax0;
        double *axt = cur ? v.ax0 : v.ax1;
        auto body = [&](int64_t i, Acc s, bool leader, bool, auto, int) {
            if (!leader)
                return;
            double yi = y[i], axi = ax[i];
            if (pending) {
                double a = v.ya[i];
                v.ya[i] = a + (yi - a) * pw;
            }
            double delta = double(s);
            double bar = axi + 2 * delta;
            double z = yi + sigma * bar;
            double t = max0(z - sigma * v.ru[i]) + min0(z - sigma * v.rl[i]);
            yt[i] = t;
            if constexpr (FP32G)
                yt32[i] = float(t);
            axt[i] = axi + delta;
            double dy = t - yi;
            dy2 += dy * dy;
            cpl += dy * delta;
            bad |= !isfinite(bar) || !isfinite(t) || !isfinite(delta);
        };
        if constexpr (FP32G)
            sweep<Acc>(A, S, v.dx32, body);
        else
            sweep<Acc>(A, S, v.dx, body);
    }
    double tot[2] = {bad ? INFINITY : dy2, cpl};
    cta_sum<2>(tot, red);
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
    for (int b = threadIdx.x; b < v.grid_p; b += kThreads)
        p += v.part_p[b];
    for (int b = threadIdx.x; b < int(gridDim.x); b += kThreads) {
        d += v.part_d[2 * b];
        c += v.part_d[2 * b + 1];
    }
    double r3[3] = {p, d, c};
    cta_sum<3>(r3, red);
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
// out = M * x (with out_shift: out written through the current-buffer index when
// `which` is non-null: out = which->cur ? out1 : out0).
template <class Acc, class V, class P, class I, class X>
__global__ void __launch_bounds__(kThreads) spmv_kernel(Csr<V, P, I> M, Schedule S, const X *x,
                                                        double *out) {
    sweep<Acc>(M, S, x, [&](int64_t r, Acc s, bool leader, bool, auto, int) {
        if (leader)
            out[r] = double(s);
    });
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
    // max-reductions: transport as sums of per-warp maxima through a fixed tree
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
template <class P> __global__ void narrow_ptr(int64_t n, const int64_t *src, P *dst) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride)
        dst[k] = P(src[k]);
}
template <class I, class V>
__global__ void convert_entries(int64_t nnz, const int64_t *idx, const double *val, I *di, V *dv) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        di[k] = I(idx[k]);
        dv[k] = V(val[k]);
    }
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
__global__ void to_float(int64_t n, const double *src, float *dst) {
    int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride)
        dst[k] = float(src[k]);
}

// ------------------------------------------------------------------ host side
inline int grid_for(int64_t n, int cap = 148 * 8) {
    int64_t g = (n + kThreads - 1) / kThreads;
    return int(std::max<int64_t>(1, std::min<int64_t>(g, cap)));
}

// A device CSR in one of the engine's storage formats, with its row schedule.
struct DeviceMatrix {
    int64_t rows = 0, cols = 0, nnz = 0;
    bool wide = false; // int64 ptr/idx
    int vbits = 64;    // 64 (double) or 32 (float) values
    DevBuf<int32_t> ptr32, idx32;
    DevBuf<int64_t> ptr64, idx64;
    DevBuf<double> val64;
    DevBuf<float> val32;
    // schedule
    DevBuf<int4> items;
    DevBuf<int64_t> longrows;
    int nitems = 0;
    int64_t long_threshold = 0;
    int width = 0; // sub-warp width of regular tiles
    std::vector<int64_t> host_ptr;

    template <class V, class P, class I> Csr<V, P, I> view() const {
        Csr<V, P, I> c;
        c.rows = rows;
        if constexpr (sizeof(P) == 8)
            c.ptr = reinterpret_cast<const P *>(ptr64.p);
        else
            c.ptr = reinterpret_cast<const P *>(ptr32.p);
        if constexpr (sizeof(I) == 8)
            c.idx = reinterpret_cast<const I *>(idx64.p);
        else
            c.idx = reinterpret_cast<const I *>(idx32.p);
        if constexpr (sizeof(V) == 8)
            c.val = reinterpret_cast<const V *>(val64.p);
        else
            c.val = reinterpret_cast<const V *>(val32.p);
        return c;
    }
    Schedule schedule() const { return Schedule{items.p, longrows.p, nitems, long_threshold}; }
    size_t device_bytes() const {
        return ptr32.bytes() + idx32.bytes() + ptr64.bytes() + idx64.bytes() + val64.bytes() +
               val32.bytes() + items.bytes() + longrows.bytes();
    }
};

// Row schedule: tiles of consecutive rows for a sub-warp width chosen from the
// mean row length, long rows split out to warp-per-row and CTA-per-row items.
void build_schedule(DeviceMatrix &M, int width_hint, int64_t threshold_hint) {
    const auto &p = M.host_ptr;
    int64_t R = M.rows;
    int W = width_hint;
    if (W <= 0) {
        // width from the body of the length distribution (rows of at most 64
        // entries); the tail goes to warp- and CTA-per-row items
        int64_t body_rows = 0, body_nnz = 0;
        for (int64_t r = 0; r < R; ++r) {
            int64_t len = p[r + 1] - p[r];
            if (len <= 64) {
                ++body_rows;
                body_nnz += len;
            }
        }
        double mean = body_rows ? double(body_nnz) / double(body_rows) : 1;
        W = 2;
        while (W < 32 && W < mean)
            W *= 2;
    }
    int64_t thr = threshold_hint > 0 ? threshold_hint : std::max<int64_t>(int64_t(4) * W, 32);
    M.width = W;
    M.long_threshold = thr;
    std::vector<int4> items;
    int per = kThreads / W;
    for (int64_t r = 0; r < R; r += per) {
        int cnt = int(std::min<int64_t>(per, R - r));
        items.push_back(make_int4(W, int(r), cnt, 0));
    }
    std::vector<int64_t> longs;
    for (int64_t r = 0; r < R; ++r)
        if (p[r + 1] - p[r] > thr)
            longs.push_back(r);
    std::stable_sort(longs.begin(), longs.end(),
                     [&](int64_t a, int64_t b) { return p[a + 1] - p[a] > p[b + 1] - p[b]; });
    const int64_t cta_threshold = 4096;
    size_t k = 0;
    for (; k < longs.size() && p[longs[k] + 1] - p[longs[k]] > cta_threshold; ++k)
        items.push_back(make_int4(KIND_CTA, int(k), 1, 0));
    for (; k < longs.size(); k += kWarps) {
        int cnt = int(std::min<size_t>(kWarps, longs.size() - k));
        items.push_back(make_int4(KIND_WARP, int(k), cnt, 0));
    }
    // Put the heavy items first so the persistent grid starts on them.
    std::stable_sort(items.begin(), items.end(), [](const int4 &a, const int4 &b) {
        return (a.x > 32) > (b.x > 32);
    });
    M.nitems = int(items.size());
    M.items.alloc(std::max<size_t>(1, items.size()));
    if (!items.empty())
        cuda_check(cudaMemcpy(M.items.p, items.data(), items.size() * sizeof(int4),
                              cudaMemcpyHostToDevice),
                   "schedule upload");
    M.longrows.alloc(std::max<size_t>(1, longs.size()));
    if (!longs.empty())
        cuda_check(cudaMemcpy(M.longrows.p, longs.data(), longs.size() * sizeof(int64_t),
                              cudaMemcpyHostToDevice),
                   "long rows upload");
}

// Upload a host CSR (int64 ptr/index, double values) into the engine format.
// `dptr/didx/dval` may already hold the int64/double arrays on the device.
void fill_matrix(DeviceMatrix &M, int64_t rows, int64_t cols, const int64_t *dptr,
                 const int64_t *didx, const double *dval, bool wide, int vbits,
                 cudaStream_t stream) {
    M.rows = rows;
    M.cols = cols;
    M.wide = wide;
    M.vbits = vbits;
    M.host_ptr.resize(size_t(rows + 1));
    cuda_check(cudaMemcpyAsync(M.host_ptr.data(), dptr, size_t(rows + 1) * sizeof(int64_t),
                               cudaMemcpyDeviceToHost, stream),
               "ptr download");
    cuda_check(cudaStreamSynchronize(stream), "ptr download");
    M.nnz = M.host_ptr[size_t(rows)];
    int g = grid_for(std::max<int64_t>(M.nnz, rows + 1), 148 * 32);
    if (wide) {
        M.ptr64.alloc(size_t(rows + 1));
        M.idx64.alloc(std::max<int64_t>(1, M.nnz));
        cuda_check(cudaMemcpyAsync(M.ptr64.p, dptr, size_t(rows + 1) * 8, cudaMemcpyDeviceToDevice,
                                   stream),
                   "ptr copy");
    } else {
        M.ptr32.alloc(size_t(rows + 1));
        M.idx32.alloc(std::max<int64_t>(1, M.nnz));
        narrow_ptr<int32_t><<<g, kThreads, 0, stream>>>(rows + 1, dptr, M.ptr32.p);
    }
    if (vbits == 64)
        M.val64.alloc(std::max<int64_t>(1, M.nnz));
    else
        M.val32.alloc(std::max<int64_t>(1, M.nnz));
    if (M.nnz) {
        if (wide && vbits == 64)
            convert_entries<int64_t, double><<<g, kThreads, 0, stream>>>(M.nnz, didx, dval,
                                                                        M.idx64.p, M.val64.p);
        else if (wide)
            convert_entries<int64_t, float><<<g, kThreads, 0, stream>>>(M.nnz, didx, dval,
                                                                       M.idx64.p, M.val32.p);
        else if (vbits == 64)
            convert_entries<int32_t, double><<<g, kThreads, 0, stream>>>(M.nnz, didx, dval,
                                                                        M.idx32.p, M.val64.p);
        else
            convert_entries<int32_t, float><<<g, kThreads, 0, stream>>>(M.nnz, didx, dval,
                                                                       M.idx32.p, M.val32.p);
    }
    cuda_check(cudaGetLastError(), "matrix conversion");
}

struct Engine {
    int64_t n = 0, m = 0;
    bool adaptive = false, halpern = false, residual_restarts = false, graphs = false;
    bool sparse_q = false, wide = false;
    int precision = NK_PRECISION_FP64;
    double reflection = 0, a_norm = 0, q_norm = 0;
    cudaStream_t stream = nullptr;
    DeviceMatrix A, At, Q;
    DevBuf<double> c, q, lb, ub, rl, ru, x[2], y[2], ax[2], xa, ya, dx, anchor_x, anchor_y,
        anchor_ax, part_p, part_d, mon_ax, mon_aty, mon_qx, mon_part, mon_out;
    DevBuf<float> dx32, y32[2];
    DevBuf<Control> ctl;
    DevBuf<unsigned> mon_arrive;
    Control *host_ctl = nullptr; // pinned mirror
    int grid_p = 1, grid_d = 1;
    int64_t accepted = 0, rejected = 0, trials = 0;
    int empty_chunks = 0;
    bool request_restart = false;
    double graph_tau = NAN, graph_sigma = NAN;
    cudaGraphExec_t graph_exec[8] = {};
    double cscale = 1;

    ~Engine() {
        if (stream)
            cudaStreamSynchronize(stream);
        for (auto &g : graph_exec)
            if (g)
                cudaGraphExecDestroy(g);
        if (host_ctl)
            cudaFreeHost(host_ctl);
        if (stream)
            cudaStreamDestroy(stream);
    }

    Vecs vecs() {
        Vecs v{};
        v.c = c.p;
        v.q = q.p;
        v.lb = lb.p;
        v.ub = ub.p;
        v.rl = rl.p;
        v.ru = ru.p;
        v.x0 = x[0].p;
        v.x1 = x[1].p;
        v.y0 = y[0].p;
        v.y1 = y[1].p;
        v.ax0 = ax[0].p;
        v.ax1 = ax[1].p;
        v.xa = xa.p;
        v.ya = ya.p;
        v.dx = dx.p;
        v.dx32 = dx32.p;
        v.y32_0 = y32[0].p;
        v.y32_1 = y32[1].p;
        v.anchor_x = anchor_x.p;
        v.anchor_y = anchor_y.p;
        v.anchor_ax = anchor_ax.p;
        v.part_p = part_p.p;
        v.part_d = part_d.p;
        v.ctl = ctl.p;
        v.grid_p = grid_p;
        v.reflection = reflection;
        return v;
    }

    // -------------------------------------------------------------- launches
    template <class V, class P, class I> void launch_trial_t() {
        Vecs v = vecs();
        auto at = At.view<V, P, I>();
        auto a = A.view<V, P, I>();
        auto qm = sparse_q ? Q.view<V, P, I>() : Csr<V, P, I>{nullptr, nullptr, nullptr, 0};
        Schedule qs = sparse_q ? Q.schedule() : Schedule{};
        if (ev[0])
            cudaEventRecord(ev[0], stream);
        if (precision == NK_PRECISION_FP32) {
            if (sparse_q)
                primal_kernel<float, V, P, I, true, true>
                    <<<grid_p, kThreads, 0, stream>>>(at, At.schedule(), qm, qs, v);
            else
                primal_kernel<float, V, P, I, false, true>
                    <<<grid_p, kThreads, 0, stream>>>(at, At.schedule(), qm, qs, v);
            if (ev[1])
                cudaEventRecord(ev[1], stream);
            dual_kernel<float, V, P, I, true><<<grid_d, kThreads, 0, stream>>>(a, A.schedule(), v);
        } else {
            if (sparse_q)
                primal_kernel<double, V, P, I, true, false>
                    <<<grid_p, kThreads, 0, stream>>>(at, At.schedule(), qm, qs, v);
            else
                primal_kernel<double, V, P, I, false, false>
                    <<<grid_p, kThreads, 0, stream>>>(at, At.schedule(), qm, qs, v);
            if (ev[1])
                cudaEventRecord(ev[1], stream);
            dual_kernel<double, V, P, I, false><<<grid_d, kThreads, 0, stream>>>(a, A.schedule(), v);
        }
        if (ev[2])
            cudaEventRecord(ev[2], stream);
        if (halpern)
            halpern_commit<<<grid_for(std::max(n, m)), kThreads, 0, stream>>>(
                n, m, v, precision == NK_PRECISION_FP32);
    }
    // Per-kernel timing hooks: when non-null, events are recorded around the
    // primal and dual launches of each trial (profiling mode, no graphs).
    cudaEvent_t ev[4] = {};
    void launch_trial() {
        if (precision == NK_PRECISION_FP64) {
            if (wide)
                launch_trial_t<double, int64_t, int64_t>();
            else
                launch_trial_t<double, int32_t, int32_t>();
        } else {
            if (wide)
                launch_trial_t<float, int64_t, int64_t>();
            else
                launch_trial_t<float, int32_t, int32_t>();
        }
    }

    template <class V, class P, class I>
    void spmv_t(const DeviceMatrix &M, const double *xin, double *out) {
        if (M.rows == 0)
            return;
        int g = std::max(1, std::min(M.nitems, 148 * 8));
        spmv_kernel<double, V, P, I, double>
            <<<g, kThreads, 0, stream>>>(M.view<V, P, I>(), M.schedule(), xin, out);
    }
    // out = M * xin with the FP64 accumulation path (used for activity rebasing,
    // the monitor and tests).
    void spmv(const DeviceMatrix &M, const double *xin, double *out) {
        if (M.vbits == 64) {
            if (M.wide)
                spmv_t<double, int64_t, int64_t>(M, xin, out);
            else
                spmv_t<double, int32_t, int32_t>(M, xin, out);
        } else {
            if (M.wide)
                spmv_t<float, int64_t, int64_t>(M, xin, out);
            else
                spmv_t<float, int32_t, int32_t>(M, xin, out);
        }
        cuda_check(cudaGetLastError(), "spmv launch");
    }

    void sync_ctl() {
        cuda_check(cudaMemcpyAsync(host_ctl, ctl.p, sizeof(Control), cudaMemcpyDeviceToHost,
                                   stream),
                   "control download");
        cuda_check(cudaStreamSynchronize(stream), "control sync");
    }
    void push_ctl() {
        cuda_check(cudaMemcpyAsync(ctl.p, host_ctl, sizeof(Control), cudaMemcpyHostToDevice,
                                   stream),
                   "control upload");
    }
    void flush() {
        Vecs v = vecs();
        flush_average<<<grid_for(std::max(n, m)), kThreads, 0, stream>>>(n, m, v);
        clear_pending<<<1, 1, 0, stream>>>(ctl.p);
        cuda_check(cudaGetLastError(), "flush");
    }
    // Recompute the resident activity A*x of the current iterate.
    void refresh_activity(int cur) {
        if (m)
            spmv(A, x[cur].p, ax[cur].p);
    }
    void refresh_y32(int cur) {
        if (precision == NK_PRECISION_FP32 && m)
            to_float<<<grid_for(m), kThreads, 0, stream>>>(m, y[cur].p, y32[cur].p);
    }

    void clear_graphs() {
        for (auto &g : graph_exec)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }
    // Graph k holds 2^k trials.
    cudaGraphExec_t graph_for(int k) {
        if (!graph_exec[k]) {
            cudaGraph_t g = nullptr;
            cuda_check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal),
                       "graph capture");
            try {
                for (int t = 0; t < (1 << k); ++t)
                    launch_trial();
            } catch (...) {
                cudaStreamEndCapture(stream, &g);
                if (g)
                    cudaGraphDestroy(g);
                throw;
            }
            cuda_check(cudaStreamEndCapture(stream, &g), "graph end capture");
            cudaError_t e = cudaGraphInstantiate(&graph_exec[k], g, 0);
            cudaGraphDestroy(g);
            cuda_check(e, "graph instantiate");
        }
        return graph_exec[k];
    }

    int advance(int count, double tau, double sigma) {
        if (count < 0)
            throw Error(NK_ERR_INVALID, "negative trial count");
        if (sparse_q) { // QP step safety, src/cpu.cpp:97-102 / src/cuda.cu:817-822
            double safety = std::sqrt(tau * sigma) * a_norm + tau * q_norm;
            double scale = safety > 0 ? std::min(1., .9 / safety) : 1.;
            tau *= scale;
            sigma *= scale;
        }
        sync_ctl();
        double before_rej = host_ctl->rejected;
        if (host_ctl->tau != tau || host_ctl->sigma != sigma) {
            host_ctl->tau = tau;
            host_ctl->sigma = sigma;
            push_ctl();
        }
        int left = count;
        if (graphs) {
            for (int k = 7; k >= 0 && left > 0; --k)
                while (left >= (1 << k)) {
                    cuda_check(cudaGraphLaunch(graph_for(k), stream), "graph launch");
                    left -= 1 << k;
                }
        } else {
            for (; left > 0; --left)
                launch_trial();
        }
        cuda_check(cudaGetLastError(), "trial launch");
        trials += count;
        sync_ctl();
        int64_t now = int64_t(host_ctl->accepted);
        int progress = int(now - accepted);
        accepted = now;
        rejected = int64_t(host_ctl->rejected);
        request_restart = host_ctl->restart != 0;
        empty_chunks = progress ? 0 : empty_chunks + 1;
        bool nonfinite_fixed = !adaptive && host_ctl->rejected != before_rej;
        if (empty_chunks >= 4 || nonfinite_fixed)
            throw Error(NK_ERR_STALLED,
                        "CUDA PDHG backtracking stalled or produced nonfinite steps");
        return progress;
    }

    void download(double *dst, const double *src, int64_t count) {
        if (count && dst)
            cuda_check(cudaMemcpyAsync(dst, src, size_t(count) * 8, cudaMemcpyDeviceToHost, stream),
                       "candidate download");
    }
    void upload(double *dst, const double *src, int64_t count) {
        if (count)
            cuda_check(cudaMemcpyAsync(dst, src, size_t(count) * 8, cudaMemcpyHostToDevice, stream),
                       "upload");
    }

    void candidates(double *hx, double *hy, double *hxa, double *hya) {
        flush();
        sync_ctl();
        int cur = host_ctl->cur;
        download(hx, x[cur].p, n);
        download(hy, y[cur].p, m);
        download(hxa, xa.p, n);
        download(hya, ya.p, m);
        refresh_activity(cur); // rebase A*x like the reference (src/cuda.cu:874-891)
        cuda_check(cudaStreamSynchronize(stream), "candidates");
    }

    void zero_average() {
        if (n)
            cuda_check(cudaMemsetAsync(xa.p, 0, size_t(n) * 8, stream), "zero xa");
        if (m)
            cuda_check(cudaMemsetAsync(ya.p, 0, size_t(m) * 8, stream), "zero ya");
    }

    void restart_state(int cur) {
        // common tail of reset / reset_candidate (src/cuda.cu:911-930,941-948)
        if (halpern) {
            if (n)
                cuda_check(cudaMemcpyAsync(anchor_x.p, x[cur].p, size_t(n) * 8,
                                           cudaMemcpyDeviceToDevice, stream), "anchor x");
            if (m) {
                cuda_check(cudaMemcpyAsync(anchor_y.p, y[cur].p, size_t(m) * 8,
                                           cudaMemcpyDeviceToDevice, stream), "anchor y");
                cuda_check(cudaMemcpyAsync(anchor_ax.p, ax[cur].p, size_t(m) * 8,
                                           cudaMemcpyDeviceToDevice, stream), "anchor ax");
            }
        }
        zero_average();
        sync_ctl();
        host_ctl->cur = cur;
        host_ctl->pending = 0;
        host_ctl->mass = 0;
        if (halpern) {
            host_ctl->epoch = 0;
            host_ctl->init_res = INFINITY;
            host_ctl->prev_res = INFINITY;
            host_ctl->restart = 0;
            host_ctl->lambda = 0;
            request_restart = false;
        }
        push_ctl();
        cuda_check(cudaStreamSynchronize(stream), "restart");
    }

    void reset_candidate(bool average) {
        flush();
        sync_ctl();
        int cur = host_ctl->cur;
        if (average) {
            if (n)
                cuda_check(cudaMemcpyAsync(x[cur].p, xa.p, size_t(n) * 8, cudaMemcpyDeviceToDevice,
                                           stream), "restart x");
            if (m)
                cuda_check(cudaMemcpyAsync(y[cur].p, ya.p, size_t(m) * 8, cudaMemcpyDeviceToDevice,
                                           stream), "restart y");
        }
        refresh_y32(cur);
        refresh_activity(cur);
        restart_state(cur);
    }

    void reset(const double *hx, const double *hy) {
        sync_ctl();
        int cur = host_ctl->cur;
        upload(x[cur].p, hx, n);
        upload(y[cur].p, hy, m);
        refresh_y32(cur);
        refresh_activity(cur);
        restart_state(cur);
    }

    double monitor() {
        if (!mon_ax.p) {
            mon_ax.alloc(std::max<int64_t>(1, m));
            mon_aty.alloc(std::max<int64_t>(1, n));
            mon_qx.alloc(std::max<int64_t>(1, n));
            mon_part.alloc(size_t(5 * 148 * 8));
            mon_out.alloc(1);
            mon_arrive.alloc(1);
            cuda_check(cudaMemsetAsync(mon_arrive.p, 0, sizeof(unsigned), stream), "monitor");
            std::vector<double> hc(static_cast<size_t>(n));
            if (n)
                cuda_check(cudaMemcpy(hc.data(), c.p, size_t(n) * 8, cudaMemcpyDeviceToHost), "c");
            cscale = 1;
            for (double v : hc)
                cscale = std::max(cscale, 1 + std::abs(v));
        }
        flush();
        sync_ctl();
        int cur = host_ctl->cur;
        double best = INFINITY;
        for (int which = 0; which < 2; ++which) {
            const double *px = which ? xa.p : x[cur].p;
            const double *py = which ? ya.p : y[cur].p;
            if (m && A.nnz)
                spmv(A, px, mon_ax.p);
            else if (m)
                cuda_check(cudaMemsetAsync(mon_ax.p, 0, size_t(m) * 8, stream), "monitor ax");
            if (n && At.nnz)
                spmv(At, py, mon_aty.p);
            else if (n)
                cuda_check(cudaMemsetAsync(mon_aty.p, 0, size_t(n) * 8, stream), "monitor aty");
            if (sparse_q)
                spmv(Q, px, mon_qx.p);
            if (std::max(n, m) == 0)
                return 0;
            int g = grid_for(std::max(n, m));
            monitor_kernel<<<g, kThreads, 0, stream>>>(
                n, m, px, py, mon_ax.p, mon_aty.p, sparse_q ? mon_qx.p : nullptr, c.p, q.p, lb.p,
                ub.p, rl.p, ru.p, cscale, mon_part.p, mon_arrive.p, mon_out.p);
            cuda_check(cudaGetLastError(), "monitor");
            double r = 0;
            cuda_check(cudaMemcpyAsync(&r, mon_out.p, 8, cudaMemcpyDeviceToHost, stream),
                       "monitor result");
            cuda_check(cudaStreamSynchronize(stream), "monitor sync");
            best = std::min(best, r);
        }
        return best;
    }

    // snapshot parts: x, y, xa, ya, ax, anchor_x, anchor_y, anchor_ax, control(11),
    // counters {accepted, rejected, empty_chunks, request_restart}
    std::vector<int64_t> layout() const {
        int64_t hn = halpern ? n : 0, hm = halpern ? m : 0;
        return {n, m, n, m, m, hn, hm, hm, 11, 4};
    }
    void snapshot(double *out) {
        flush();
        sync_ctl();
        int cur = host_ctl->cur;
        auto L = layout();
        int64_t at = 0;
        const double *src[8] = {x[cur].p, y[cur].p, xa.p, ya.p, ax[cur].p,
                                anchor_x.p, anchor_y.p, anchor_ax.p};
        for (int i = 0; i < 8; ++i) {
            download(out + at, src[i], L[size_t(i)]);
            at += L[size_t(i)];
        }
        cuda_check(cudaStreamSynchronize(stream), "snapshot");
        const Control &s = *host_ctl;
        double st[11] = {s.factor, s.mass, s.accepted, s.rejected, s.accept, s.weight,
                         s.epoch, s.init_res, s.prev_res, s.restart, s.lambda};
        std::memcpy(out + at, st, sizeof(st));
        at += 11;
        double cnt[4] = {double(accepted), double(rejected), double(empty_chunks),
                         request_restart ? 1. : 0.};
        std::memcpy(out + at, cnt, sizeof(cnt));
    }
    void restore(const double *in, const int64_t *sizes, int parts) {
        auto L = layout();
        if (parts != int(L.size()))
            throw Error(NK_ERR_INVALID, "GPU checkpoint state count");
        for (int i = 0; i < parts; ++i)
            if (sizes[i] != L[size_t(i)])
                throw Error(NK_ERR_INVALID, "GPU checkpoint state dimensions");
        int64_t at = 0;
        for (int i = 0; i < 10; ++i)
            at += L[size_t(i)];
        const double *cnt = in + at - 4;
        for (int i = 0; i < 4; ++i)
            if (!std::isfinite(cnt[i]) || cnt[i] < 0)
                throw Error(NK_ERR_INVALID, "GPU checkpoint counters");
        const double *st = in + at - 15;
        if (!(st[0] > 0) || st[2] < 0 || st[3] < 0)
            throw Error(NK_ERR_INVALID, "GPU checkpoint counters");
        sync_ctl();
        int cur = 0;
        double *dst[8] = {x[cur].p, y[cur].p, xa.p, ya.p, ax[cur].p,
                          anchor_x.p, anchor_y.p, anchor_ax.p};
        at = 0;
        for (int i = 0; i < 8; ++i) {
            upload(dst[i], in + at, L[size_t(i)]);
            at += L[size_t(i)];
        }
        refresh_y32(cur);
        Control &s = *host_ctl;
        s.factor = st[0];
        s.mass = st[1];
        s.accepted = st[2];
        s.rejected = st[3];
        s.accept = st[4];
        s.weight = st[5];
        s.epoch = st[6];
        s.init_res = st[7];
        s.prev_res = st[8];
        s.restart = st[9];
        s.lambda = st[10];
        s.cur = cur;
        s.pending = 0;
        accepted = int64_t(cnt[0]);
        rejected = int64_t(cnt[1]);
        empty_chunks = int(cnt[2]);
        request_restart = cnt[3] != 0;
        push_ctl();
        cuda_check(cudaStreamSynchronize(stream), "restore");
    }

    // Runs `count` trials one by one with events around each kernel; returns the
    // mean primal and dual kernel durations in milliseconds.
    void profile(int count, double tau, double sigma, double *ms_primal, double *ms_dual) {
        if (count <= 0)
            throw Error(NK_ERR_INVALID, "profile needs a positive trial count");
        sync_ctl();
        host_ctl->tau = tau;
        host_ctl->sigma = sigma;
        push_ctl();
        for (auto &e : ev)
            cuda_check(cudaEventCreate(&e), "event");
        double tp = 0, td = 0;
        try {
            for (int t = 0; t < count; ++t) {
                launch_trial();
                cuda_check(cudaEventSynchronize(ev[2]), "profile sync");
                float a = 0, b = 0;
                cudaEventElapsedTime(&a, ev[0], ev[1]);
                cudaEventElapsedTime(&b, ev[1], ev[2]);
                tp += a;
                td += b;
            }
        } catch (...) {
            for (auto &e : ev) {
                cudaEventDestroy(e);
                e = nullptr;
            }
            throw;
        }
        for (auto &e : ev) {
            cudaEventDestroy(e);
            e = nullptr;
        }
        trials += count;
        sync_ctl();
        accepted = int64_t(host_ctl->accepted);
        rejected = int64_t(host_ctl->rejected);
        *ms_primal = tp / count;
        *ms_dual = td / count;
    }

    size_t device_bytes() const {
        size_t b = A.device_bytes() + At.device_bytes() + Q.device_bytes();
        for (auto *d : {&c, &q, &lb, &ub, &rl, &ru, &x[0], &x[1], &y[0], &y[1], &ax[0], &ax[1],
                        &xa, &ya, &dx, &anchor_x, &anchor_y, &anchor_ax, &part_p, &part_d})
            b += d->bytes();
        b += dx32.bytes() + y32[0].bytes() + y32[1].bytes();
        return b;
    }
};

// Build the explicit transpose on the device: stable radix sort of the column
// indices carries every entry to its row of A^T in increasing row order, the
// order Sparse::transpose produces (src/model.cpp:39-58).
void device_transpose(int64_t rows, int64_t cols, int64_t nnz, const int64_t *dptr,
                      const int64_t *didx, const double *dval, DevBuf<int64_t> &tptr,
                      DevBuf<int64_t> &tidx, DevBuf<double> &tval, cudaStream_t stream) {
    tptr.alloc(size_t(cols + 1));
    tidx.alloc(std::max<int64_t>(1, nnz));
    tval.alloc(std::max<int64_t>(1, nnz));
    DevBuf<int64_t> counts(static_cast<size_t>(cols + 1));
    cuda_check(cudaMemsetAsync(counts.p, 0, size_t(cols + 1) * 8, stream), "counts");
    if (nnz) {
        int g = grid_for(nnz, 148 * 32);
        count_cols<<<g, kThreads, 0, stream>>>(nnz, didx, counts.p);
        DevBuf<int32_t> rowid(static_cast<size_t>(nnz));
        expand_rows<<<grid_for(rows, 148 * 32), kThreads, 0, stream>>>(rows, dptr, rowid.p);
        DevBuf<int64_t> keys_out(static_cast<size_t>(nnz)), perm_in(static_cast<size_t>(nnz)),
            perm_out(static_cast<size_t>(nnz));
        iota64<<<g, kThreads, 0, stream>>>(nnz, perm_in.p);
        int end_bit = 1;
        while (end_bit < 63 && (int64_t(1) << end_bit) < cols)
            ++end_bit;
        size_t temp = 0;
        cuda_check(cub::DeviceRadixSort::SortPairs(nullptr, temp, didx, keys_out.p, perm_in.p,
                                                   perm_out.p, nnz, 0, end_bit, stream),
                   "transpose sort size");
        DevBuf<char> work(temp);
        cuda_check(cub::DeviceRadixSort::SortPairs(work.p, temp, didx, keys_out.p, perm_in.p,
                                                   perm_out.p, nnz, 0, end_bit, stream),
                   "transpose sort");
        gather_transpose<<<g, kThreads, 0, stream>>>(nnz, perm_out.p, rowid.p, dval, tidx.p,
                                                    tval.p);
        cuda_check(cudaGetLastError(), "transpose gather");
        size_t t2 = 0;
        cuda_check(cub::DeviceScan::ExclusiveSum(nullptr, t2, counts.p, tptr.p, cols + 1, stream),
                   "transpose scan size");
        DevBuf<char> w2(t2);
        cuda_check(cub::DeviceScan::ExclusiveSum(w2.p, t2, counts.p, tptr.p, cols + 1, stream),
                   "transpose scan");
        cuda_check(cudaStreamSynchronize(stream), "transpose");
    } else {
        cuda_check(cudaMemsetAsync(tptr.p, 0, size_t(cols + 1) * 8, stream), "empty transpose");
    }
}

int occupancy_grid(const void *kernel, int nitems) {
    int dev = 0, sms = 148, per = 4;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kThreads, 0);
    per = std::max(1, per);
    return std::max(1, std::min(nitems, sms * per));
}

void validate_csr(const nk_csr *M, int64_t rows, int64_t cols, const char *what) {
    if (!M || M->rows != rows || M->cols != cols || !M->ptr)
        throw Error(NK_ERR_INVALID, std::string("inconsistent ") + what + " dimensions");
    if (M->ptr[0] != 0)
        throw Error(NK_ERR_INVALID, std::string("invalid ") + what + " CSR storage");
    for (int64_t i = 0; i < rows; ++i)
        if (M->ptr[i + 1] < M->ptr[i])
            throw Error(NK_ERR_INVALID, std::string("invalid ") + what + " CSR offsets");
    if (M->ptr[rows] > 0 && (!M->index || !M->value))
        throw Error(NK_ERR_INVALID, std::string("missing ") + what + " entries");
}

// Upload a host CSR, check indices on the device, convert to the engine format.
void upload_matrix(DeviceMatrix &D, const nk_csr *H, bool wide, int vbits, cudaStream_t stream,
                   DevBuf<int64_t> *keep_ptr = nullptr, DevBuf<int64_t> *keep_idx = nullptr,
                   DevBuf<double> *keep_val = nullptr) {
    int64_t nnz = H->ptr[H->rows];
    DevBuf<int64_t> p(static_cast<size_t>(H->rows + 1)), ix(std::max<int64_t>(1, nnz));
    DevBuf<double> vv(std::max<int64_t>(1, nnz));
    cuda_check(cudaMemcpyAsync(p.p, H->ptr, size_t(H->rows + 1) * 8, cudaMemcpyHostToDevice, stream),
               "ptr upload");
    if (nnz) {
        cuda_check(cudaMemcpyAsync(ix.p, H->index, size_t(nnz) * 8, cudaMemcpyHostToDevice, stream),
                   "index upload");
        cuda_check(cudaMemcpyAsync(vv.p, H->value, size_t(nnz) * 8, cudaMemcpyHostToDevice, stream),
                   "value upload");
        DevBuf<int> bad(1);
        cuda_check(cudaMemsetAsync(bad.p, 0, sizeof(int), stream), "flag");
        check_indices<<<grid_for(nnz, 148 * 32), kThreads, 0, stream>>>(nnz, ix.p, vv.p, H->cols,
                                                                        bad.p);
        if (vbits == 32)
            fp32_flags<<<grid_for(nnz, 148 * 32), kThreads, 0, stream>>>(nnz, vv.p, bad.p + 0);
        int hb = 0;
        cuda_check(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, stream), "flag");
        cuda_check(cudaStreamSynchronize(stream), "index check");
        if (hb)
            throw Error(NK_ERR_INVALID,
                        vbits == 32 ? "invalid coefficient/index, or FP32 matrix conversion would "
                                      "overflow or erase a coefficient; use fp64"
                                    : "Invalid matrix coefficient/index");
    }
    fill_matrix(D, H->rows, H->cols, p.p, ix.p, vv.p, wide, vbits, stream);
    cuda_check(cudaStreamSynchronize(stream), "matrix upload");
    if (keep_ptr) {
        *keep_ptr = std::move(p);
        *keep_idx = std::move(ix);
        *keep_val = std::move(vv);
    }
}

Engine *create_engine(const nk_csr *Ah, const nk_csr *Qh, const double *hc, const double *hq,
                      const double *hlb, const double *hub, const double *hrl, const double *hru,
                      const double *hx0, const double *hy0, const nk_pdhg_options *o) {
    if (!Ah || !hc || !hlb || !hub || !hrl || !hru || !hx0 || !hy0 || !o)
        throw Error(NK_ERR_INVALID, "null argument");
    int64_t m = Ah->rows, n = Ah->cols;
    if (m < 0 || n < 0)
        throw Error(NK_ERR_INVALID, "Negative matrix dimension");
    validate_csr(Ah, m, n, "A");
    bool sparse_q = Qh && Qh->rows > 0 && Qh->ptr && Qh->ptr[Qh->rows] > 0;
    if (sparse_q)
        validate_csr(Qh, n, n, "Q");
    if (o->halpern && o->adaptive)
        throw Error(NK_ERR_UNSUPPORTED, "Halpern requires a fixed PDHG operator");
    if (!std::isfinite(o->reflection) || o->reflection < 0 || o->reflection > 1)
        throw Error(NK_ERR_INVALID, "Invalid Halpern reflection");
    if (o->precision < 0 || o->precision > 2)
        throw Error(NK_ERR_INVALID, "unknown matrix precision");
    if (sparse_q && o->precision == NK_PRECISION_MIXED)
        throw Error(NK_ERR_UNSUPPORTED, "Sparse QP requires FP64 matrices");
    int64_t nnz = Ah->ptr[m], qnnz = sparse_q ? Qh->ptr[n] : 0;
    bool fits32 = m <= INT32_MAX && n <= INT32_MAX && nnz <= INT32_MAX && qnnz <= INT32_MAX;
    if (o->index_bits == 32 && !fits32)
        throw Error(NK_ERR_INVALID, "Model exceeds 32-bit CSR limits");
    int dev = 0, count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        throw Error(NK_ERR_NO_DEVICE, "no CUDA device");
    cuda_check(cudaGetDevice(&dev), "device");
    size_t freeb = 0, total = 0;
    cuda_check(cudaMemGetInfo(&freeb, &total), "cudaMemGetInfo");
    // the reference guard (src/cuda.cu:1292-1298)
    long double estimate = 48.L * (nnz + qnnz) + 240.L * (m + n + 2);
    if (estimate > .8L * freeb)
        throw Error(NK_ERR_MEMORY,
                    "Estimated GPU storage exceeds 80% of available memory; use --device cpu");
    auto E = std::make_unique<Engine>();
    E->n = n;
    E->m = m;
    E->adaptive = o->adaptive && !sparse_q;
    E->halpern = o->halpern;
    E->residual_restarts = o->residual_restarts;
    E->graphs = o->graphs;
    E->reflection = o->reflection;
    E->precision = o->precision;
    E->sparse_q = sparse_q;
    E->wide = !fits32 || o->index_bits == 64;
    cuda_check(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking), "stream");
    cudaStream_t s = E->stream;
    int vbits = o->precision == NK_PRECISION_FP64 ? 64 : 32;
    if (sparse_q && o->precision == NK_PRECISION_FP64)
        vbits = 64;
    // A, then its transpose from the raw device copy
    DevBuf<int64_t> rp, ri;
    DevBuf<double> rv;
    upload_matrix(E->A, Ah, E->wide, vbits, s, &rp, &ri, &rv);
    {
        DevBuf<int64_t> tp, ti;
        DevBuf<double> tv;
        device_transpose(m, n, nnz, rp.p, ri.p, rv.p, tp, ti, tv, s);
        fill_matrix(E->At, n, m, tp.p, ti.p, tv.p, E->wide, vbits, s);
        cuda_check(cudaStreamSynchronize(s), "transpose convert");
    }
    rp.release();
    ri.release();
    rv.release();
    if (sparse_q)
        upload_matrix(E->Q, Qh, E->wide, vbits, s);
    build_schedule(E->A, 0, 0);
    build_schedule(E->At, 0, 0);
    if (sparse_q)
        build_schedule(E->Q, E->At.width, 1 << 30); // Q rows follow A^T's geometry
    // norms for the QP step safety (src/cpu.cpp:25-42)
    if (sparse_q) {
        std::vector<double> cols(static_cast<size_t>(n), 0.0);
        double rowmax = 0;
        for (int64_t i = 0; i < m; ++i) {
            double sum = 0;
            for (int64_t k = Ah->ptr[i]; k < Ah->ptr[i + 1]; ++k) {
                sum += std::abs(Ah->value[k]);
                cols[size_t(Ah->index[k])] += std::abs(Ah->value[k]);
            }
            rowmax = std::max(rowmax, sum);
        }
        double colmax = 0;
        for (double v : cols)
            colmax = std::max(colmax, v);
        E->a_norm = std::sqrt(rowmax) * std::sqrt(colmax);
        long double largest = 0; // Model::quadratic_norm_bound, src/model.cpp:257-267
        for (int64_t i = 0; i < n; ++i) {
            long double sum = std::abs(hq ? hq[i] : 0.0);
            for (int64_t k = Qh->ptr[i]; k < Qh->ptr[i + 1]; ++k)
                sum += std::abs(Qh->value[k]);
            largest = std::max(largest, sum);
        }
        E->q_norm = std::nextafter(double(largest), INFINITY);
    }
    auto vec = [&](DevBuf<double> &d, const double *h, int64_t len) {
        d.alloc(std::max<int64_t>(1, len));
        if (len && h)
            cuda_check(cudaMemcpyAsync(d.p, h, size_t(len) * 8, cudaMemcpyHostToDevice, s), "vector");
        else if (len)
            cuda_check(cudaMemsetAsync(d.p, 0, size_t(len) * 8, s), "vector zero");
    };
    vec(E->c, hc, n);
    vec(E->q, hq, n);
    vec(E->lb, hlb, n);
    vec(E->ub, hub, n);
    vec(E->rl, hrl, m);
    vec(E->ru, hru, m);
    vec(E->x[0], hx0, n);
    vec(E->x[1], hx0, n);
    vec(E->y[0], hy0, m);
    vec(E->y[1], hy0, m);
    vec(E->xa, nullptr, n);
    vec(E->ya, nullptr, m);
    vec(E->ax[0], nullptr, m);
    vec(E->ax[1], nullptr, m);
    if (o->precision == NK_PRECISION_FP32) {
        E->dx32.alloc(std::max<int64_t>(1, n));
        E->y32[0].alloc(std::max<int64_t>(1, m));
        E->y32[1].alloc(std::max<int64_t>(1, m));
        E->dx.alloc(1);
    } else {
        vec(E->dx, nullptr, n);
        E->dx32.alloc(1);
        E->y32[0].alloc(1);
        E->y32[1].alloc(1);
    }
    if (E->halpern) {
        vec(E->anchor_x, hx0, n);
        vec(E->anchor_y, hy0, m);
        vec(E->anchor_ax, nullptr, m);
    } else {
        E->anchor_x.alloc(1);
        E->anchor_y.alloc(1);
        E->anchor_ax.alloc(1);
    }
    // grids from occupancy
    {
        const void *pk, *dk;
        if (o->precision == NK_PRECISION_FP32) {
            pk = E->wide ? (const void *)primal_kernel<float, float, int64_t, int64_t, false, true>
                         : (const void *)primal_kernel<float, float, int32_t, int32_t, false, true>;
            dk = E->wide ? (const void *)dual_kernel<float, float, int64_t, int64_t, true>
                         : (const void *)dual_kernel<float, float, int32_t, int32_t, true>;
        } else {
            pk = E->wide ? (const void *)primal_kernel<double, double, int64_t, int64_t, false, false>
                         : (const void *)primal_kernel<double, double, int32_t, int32_t, false, false>;
            dk = E->wide ? (const void *)dual_kernel<double, double, int64_t, int64_t, false>
                         : (const void *)dual_kernel<double, double, int32_t, int32_t, false>;
        }
        E->grid_p = occupancy_grid(pk, std::max(1, E->At.nitems));
        E->grid_d = occupancy_grid(dk, std::max(1, E->A.nitems));
    }
    E->part_p.alloc(size_t(E->grid_p));
    E->part_d.alloc(size_t(2 * E->grid_d));
    E->ctl.alloc(1);
    cuda_check(cudaMallocHost(reinterpret_cast<void **>(&E->host_ctl), sizeof(Control)), "pinned");
    Control init{};
    init.factor = 1;
    init.init_res = INFINITY;
    init.prev_res = INFINITY;
    init.tau = 0;
    init.sigma = 0;
    init.flags = (E->adaptive ? 1 : 0) | (E->halpern ? 2 : 0) | (E->residual_restarts ? 4 : 0);
    *E->host_ctl = init;
    E->push_ctl();
    E->refresh_y32(0);
    E->refresh_activity(0);
    if (E->halpern && m)
        cuda_check(cudaMemcpyAsync(E->anchor_ax.p, E->ax[0].p, size_t(m) * 8,
                                   cudaMemcpyDeviceToDevice, s), "anchor activity");
    cuda_check(cudaStreamSynchronize(s), "engine init");
    return E.release();
}

} // namespace nk

using nk::guard;

struct nk_pdhg {
    nk::Engine *e;
};

extern "C" {
unsigned nk_abi_version(void) { return 1; }
const char *nk_last_error(void) { return nk::g_last_error; }

nk_status nk_pdhg_create(const nk_csr *A, const nk_csr *Q, const double *c, const double *q,
                         const double *lb, const double *ub, const double *rl, const double *ru,
                         const double *x0, const double *y0, const nk_pdhg_options *opts,
                         nk_pdhg **out) {
    return guard([&] {
        if (!out)
            throw nk::Error(NK_ERR_INVALID, "null output handle");
        *out = nullptr;
        auto *e = nk::create_engine(A, Q, c, q, lb, ub, rl, ru, x0, y0, opts);
        *out = new nk_pdhg{e};
    });
}
void nk_pdhg_destroy(nk_pdhg *h) {
    if (h) {
        delete h->e;
        delete h;
    }
}
#define NK_HANDLE                                                                                  \
    if (!h || !h->e)                                                                               \
        throw nk::Error(NK_ERR_INVALID, "null engine handle");
nk_status nk_pdhg_advance(nk_pdhg *h, int count, double tau, double sigma, int *accepted) {
    return guard([&] {
        NK_HANDLE
        int r = h->e->advance(count, tau, sigma);
        if (accepted)
            *accepted = r;
    });
}
nk_status nk_pdhg_rejected_steps(nk_pdhg *h, int64_t *out) {
    return guard([&] {
        NK_HANDLE
        *out = h->e->rejected;
    });
}
nk_status nk_pdhg_restart_requested(nk_pdhg *h, int *out) {
    return guard([&] {
        NK_HANDLE
        *out = h->e->request_restart ? 1 : 0;
    });
}
nk_status nk_pdhg_monitor(nk_pdhg *h, double *out) {
    return guard([&] {
        NK_HANDLE
        *out = h->e->monitor();
    });
}
nk_status nk_pdhg_candidates(nk_pdhg *h, double *x, double *y, double *xa, double *ya) {
    return guard([&] {
        NK_HANDLE
        h->e->candidates(x, y, xa, ya);
    });
}
nk_status nk_pdhg_reset_candidate(nk_pdhg *h, int average) {
    return guard([&] {
        NK_HANDLE
        h->e->reset_candidate(average != 0);
    });
}
nk_status nk_pdhg_reset(nk_pdhg *h, const double *x, const double *y) {
    return guard([&] {
        NK_HANDLE
        h->e->reset(x, y);
    });
}
nk_status nk_pdhg_snapshot_layout(nk_pdhg *h, int *parts, int64_t *sizes) {
    return guard([&] {
        NK_HANDLE
        auto L = h->e->layout();
        *parts = int(L.size());
        if (sizes)
            for (size_t i = 0; i < L.size(); ++i)
                sizes[i] = L[i];
    });
}
nk_status nk_pdhg_snapshot(nk_pdhg *h, double *out) {
    return guard([&] {
        NK_HANDLE
        h->e->snapshot(out);
    });
}
nk_status nk_pdhg_restore(nk_pdhg *h, const double *in, const int64_t *sizes, int parts) {
    return guard([&] {
        NK_HANDLE
        h->e->restore(in, sizes, parts);
    });
}
nk_status nk_pdhg_stats(nk_pdhg *h, int64_t *trials, int64_t *bytes) {
    return guard([&] {
        NK_HANDLE
        if (trials)
            *trials = h->e->trials;
        if (bytes)
            *bytes = int64_t(h->e->device_bytes());
    });
}
nk_status nk_pdhg_profile(nk_pdhg *h, int count, double tau, double sigma, double *ms_primal,
                          double *ms_dual) {
    return guard([&] {
        NK_HANDLE
        h->e->profile(count, tau, sigma, ms_primal, ms_dual);
    });
}
nk_status nk_pdhg_stream(nk_pdhg *h, void **stream) {
    return guard([&] {
        NK_HANDLE
        *stream = reinterpret_cast<void *>(h->e->stream);
    });
}
nk_status nk_pdhg_schedule_info(nk_pdhg *h, int *a_width, int64_t *a_long, int *at_width,
                                int64_t *at_long, int *a_items, int *at_items) {
    return guard([&] {
        NK_HANDLE
        *a_width = h->e->A.width;
        *a_long = h->e->A.long_threshold;
        *at_width = h->e->At.width;
        *at_long = h->e->At.long_threshold;
        *a_items = h->e->A.nitems;
        *at_items = h->e->At.nitems;
    });
}
int nk_cuda_available(void) {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}
nk_status nk_cuda_description(char *buffer, int length) {
    return guard([&] {
        if (!buffer || length <= 0)
            throw nk::Error(NK_ERR_INVALID, "null buffer");
        if (!nk_cuda_available()) {
            std::snprintf(buffer, size_t(length), "No CUDA device");
            return;
        }
        cudaDeviceProp p{};
        nk::cuda_check(cudaGetDeviceProperties(&p, 0), "GPU properties");
        std::snprintf(buffer, size_t(length), "%s (%zu MiB)", p.name,
                      size_t(p.totalGlobalMem / (1024 * 1024)));
    });
}
nk_status nk_hardware_info(int *available, double *free_bytes, double *total_bytes) {
    return guard([&] {
        *available = nk_cuda_available();
        *free_bytes = *total_bytes = 0;
        size_t f = 0, t = 0;
        if (*available && cudaMemGetInfo(&f, &t) == cudaSuccess) {
            *free_bytes = double(f);
            *total_bytes = double(t);
        }
    });
}
}
