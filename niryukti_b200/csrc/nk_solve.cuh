// Device-resident solve driver: the reference's continuous PDHG driver
// (solve_continuous, src/solver.cpp:213-780, method "pdhg") with the
// per-check candidate evaluation, best-point tracking, restart test and
// primal-weight update done on the GPU.  The host sees a few hundred bytes
// per check; iterates cross PCIe only when a candidate is certified (the
// outward-rounded acceptance test of Verifier::evaluate, run on the host over
// the caller's model, exactly as the reference does), for the occasional
// infeasibility-ray test, and once at the end.
//
// Original-space KKT on the device.  The engine iterates on the prepared
// (presolved, scaled) model.  For a prepared point (x_s, y_s) the caller-space
// point of Prepared::restore_x / restore_y is x_o = D_c x_s (removed columns at
// their fixed values) and y_o = y_s * row_scale * objective_scale on the row
// that supplied the active bound.  Every term of Verifier::evaluate
// (src/verify.cpp:103-240) follows from prepared-space products:
//   A_o x_o  (kept row)    = (A_s x_s) / row_scale + shift (fixed-column activity)
//   A_o^T y_o (kept column) = (A_s^T y_s) * objective_scale / column_scale
//   c_o, q_o x_o + (Q_o x_o) = prepared values * objective_scale / column_scale
// and the removed columns contribute constants (their objective terms and
// sum_i y_i * shift_i to the Lagrangian box minimum).  Removed rows are
// redundant for every point inside the bounds, so they add nothing.  The
// device evaluation ranks candidates and decides restarts; termination is
// still certified by the host verifier on the caller's model.
#pragma once
#include <exception>
#include <memory>
#include <thread>

namespace nk {

constexpr int kKktValues = 10;
// 0 primal (max)  1 primal_abs (max)  2 dual (max)  3 dual_abs (max)
// 4 objective sum  5 complementarity  6 support  7 box minimum
// 8 bound unavailable (max)  9 non-finite (max)
constexpr unsigned kKktMaxMask = 0x30fu;

struct KktArgs {
    int64_t n, m;
    const double *x, *y, *ax, *aty, *qx;   // prepared point and its products (engine order)
    const double *c, *q;                   // prepared objective
    const double *cs, *olb, *oub;          // column scale, caller bounds of kept columns
    const double *rs, *shift, *orl, *oru;  // row scale, fixed activity, caller row bounds
    double os, cscale;                     // objective scale, max(1, 1 + |c_o|)
    int sparse_q;
};

__device__ __forceinline__ double clamp_to(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

template <int NV>
__device__ void block_combine(double (&v)[NV], unsigned max_mask, double *smem /* kWarps*NV */) {
#pragma unroll
    for (int t = 0; t < NV; ++t)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            double o = __shfl_xor_sync(0xffffffffu, v[t], off);
            v[t] = (max_mask >> t & 1) ? fmax(v[t], o) : v[t] + o;
        }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
#pragma unroll
        for (int t = 0; t < NV; ++t)
            smem[w * NV + t] = v[t];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int t = 0; t < NV; ++t) {
            double s = smem[t];
            for (int i = 1; i < kWarps; ++i)
                s = (max_mask >> t & 1) ? fmax(s, smem[i * NV + t]) : s + smem[i * NV + t];
            v[t] = s;
        }
}

__global__ void __launch_bounds__(kThreads) kkt_partial(KktArgs a, double *part) {
    __shared__ double smem[kWarps * kKktValues];
    double v[kKktValues] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t top = a.n > a.m ? a.n : a.m;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < top; i += stride) {
        if (i < a.n) {
            const double cj = a.cs[i], xs = a.x[i], xo = xs * cj;
            const double lo = a.olb[i], hi = a.oub[i];
            const double viol = fmax(0., fmax(lo - xo, xo - hi));
            v[0] = fmax(v[0], viol / (1 + fabs(xo)));
            v[1] = fmax(v[1], viol);
            const double f = a.os / cj;
            const double qxs = a.qx ? a.qx[i] : 0.;
            const double lin = (a.c[i] + a.aty[i]) * f;
            const double curv = (a.q[i] * xs + qxs) * f;
            const double g = lin + curv;
            v[4] += a.c[i] * xs + .5 * a.q[i] * xs * xs + .5 * xs * qxs;
            if (!isfinite(lin) || !isfinite(g) || !isfinite(xo))
                v[9] = 1;
            const double d = clamp_to(g, xo - hi, xo - lo);
            v[3] = fmax(v[3], fabs(d));
            v[2] = fmax(v[2], fabs(d) / a.cscale);
            if (g > 0 && isfinite(lo))
                v[5] += fabs(g * (xo - lo));
            if (g < 0 && isfinite(hi))
                v[5] += fabs(g * (hi - xo));
            double arg;
            if (a.sparse_q) {
                arg = g > 0 ? lo : g < 0 ? hi : clamp_to(0., lo, hi);
                if (!isfinite(arg))
                    v[8] = 1;
                else
                    v[7] += g * arg - curv * xo / 2;
            } else {
                const double qo = a.q[i] * f / cj;
                arg = qo > 0 ? clamp_to(-lin / qo, lo, hi)
                      : lin > 0 ? lo
                      : lin < 0 ? hi
                                : clamp_to(0., lo, hi);
                if (!isfinite(arg))
                    v[8] = 1;
                else
                    v[7] += lin * arg + .5 * qo * arg * arg;
            }
        }
        if (i < a.m) {
            const double r = a.rs[i], yo = a.y[i] * r * a.os;
            const double axo = a.ax[i] / r + a.shift[i];
            const double lo = a.orl[i], hi = a.oru[i];
            if (isfinite(lo))
                v[0] = fmax(v[0], fmax(0., lo - axo) / (1 + fabs(lo)));
            if (isfinite(hi))
                v[0] = fmax(v[0], fmax(0., axo - hi) / (1 + fabs(hi)));
            v[1] = fmax(v[1], fmax(0., fmax(lo - axo, axo - hi)));
            if (yo != 0) {
                const double e = yo > 0 ? hi : lo;
                if (isfinite(e)) {
                    v[6] += yo * e;
                    v[5] += fabs(yo * (e - axo));
                } else {
                    v[8] = 1;
                    v[3] = fmax(v[3], fabs(yo));
                    v[2] = fmax(v[2], fabs(yo));
                }
                v[7] += yo * a.shift[i];
            }
            if (!isfinite(axo) || !isfinite(yo))
                v[9] = 1;
        }
    }
    block_combine<kKktValues>(v, kKktMaxMask, smem);
    if (threadIdx.x == 0)
        for (int t = 0; t < kKktValues; ++t)
            part[blockIdx.x * kKktValues + t] = v[t];
}

// Combines `blocks` rows of NV partials into out[0..NV) with one CTA, in a
// fixed order (deterministic).
template <int NV>
__global__ void __launch_bounds__(kThreads) finish_partials(const double *part, int blocks,
                                                            unsigned max_mask, double *out) {
    __shared__ double smem[kWarps * NV];
    double v[NV];
#pragma unroll
    for (int t = 0; t < NV; ++t)
        v[t] = 0;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x)
#pragma unroll
        for (int t = 0; t < NV; ++t) {
            double p = part[b * NV + t];
            v[t] = (max_mask >> t & 1) ? fmax(v[t], p) : v[t] + p;
        }
    block_combine<NV>(v, max_mask, smem);
    if (threadIdx.x == 0)
#pragma unroll
        for (int t = 0; t < NV; ++t)
            out[t] = v[t];
}

// Sum (a - b)^2 over n columns and over m rows (restart displacement).
__global__ void __launch_bounds__(kThreads) displacement_partial(int64_t n, int64_t m,
                                                                 const double *x, const double *ex,
                                                                 const double *y, const double *ey,
                                                                 double *part) {
    __shared__ double smem[kWarps * 2];
    double v[2] = {0, 0};
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t top = n > m ? n : m;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < top; i += stride) {
        if (i < n) {
            double d = x[i] - ex[i];
            v[0] += d * d;
        }
        if (i < m) {
            double d = y[i] - ey[i];
            v[1] += d * d;
        }
    }
    block_combine<2>(v, 0u, smem);
    if (threadIdx.x == 0) {
        part[blockIdx.x * 2] = v[0];
        part[blockIdx.x * 2 + 1] = v[1];
    }
}

// Farkas screen of a candidate ray r = y - ey (ey may be null) with
// A^T r = aty - atey (atey may be null), prepared space.  The caller-space ray
// is a positive row scaling of r, so signs carry over.  Values: 0 the ray is
// impossible (max) -- a sign meets an infinite caller row bound, or A^T r
// pushes a column towards an infinite bound, where the outward-rounded
// feasibility bound (lp_lower_bound, src/verify.cpp:12-88) is -infinity;
// 1 + 2 that bound in plain FP64 (-sum r_i b_i + sum_j min over the box of
// (A^T r)_j x_j); 3 the magnitude of its terms.
constexpr int kRayValues = 4;
__global__ void __launch_bounds__(kThreads) ray_screen(int64_t n, int64_t m, const double *y,
                                                       const double *ey, const double *aty,
                                                       const double *atey, KktArgs a,
                                                       double *part) {
    __shared__ double smem[kWarps * kRayValues];
    double v[kRayValues] = {0, 0, 0, 0};
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t top = n > m ? n : m;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < top; i += stride) {
        if (i < m) {
            const double r = (y[i] - (ey ? ey[i] : 0.)) * a.rs[i] * a.os;
            if (r != 0) {
                const double b = r > 0 ? a.oru[i] : a.orl[i];
                if (!isfinite(b))
                    v[0] = 1;
                else {
                    v[1] -= r * b;
                    v[3] += fabs(r * b);
                }
            }
        }
        if (i < n) {
            const double g = (aty[i] - (atey ? atey[i] : 0.)) * a.os / a.cs[i];
            if (g != 0) {
                const double b = g > 0 ? a.olb[i] : a.oub[i];
                if (!isfinite(b))
                    v[0] = 1;
                else {
                    v[2] += g * b;
                    v[3] += fabs(g * b);
                }
            }
        }
    }
    block_combine<kRayValues>(v, 1u, smem);
    if (threadIdx.x == 0)
        for (int t = 0; t < kRayValues; ++t)
            part[blockIdx.x * kRayValues + t] = v[t];
}

// ------------------------------------------------------------------ driver
struct SolveReport {
    int status = NK_SOLVE_ITERATION_LIMIT;
    int64_t iterations = 0, restarts = 0, rejected = 0, weight_updates = 0;
    int64_t device_checks = 0, host_checks = 0, refine_iterations = 0;
    int64_t removed_rows = 0, removed_columns = 0;
    double seconds = 0, preprocess = 0, transfer = 0, iteration = 0, verification = 0;
    Accuracy accuracy, mixed;
    int64_t mixed_iterations = 0;
    double mixed_seconds = 0;
    double reached[9] = {-1, -1, -1, -1, -1, -1, -1, -1, -1}; // seconds to best kkt <= 10^-k
    std::vector<double> x, y;
};

using SteadyClock = std::chrono::steady_clock;
inline double since(SteadyClock::time_point t) {
    return std::chrono::duration<double>(SteadyClock::now() - t).count();
}

// One prepared model on the device: the engine plus the driver's buffers.
struct DeviceSolve {
    const Prepared &prep;
    const HostModel &orig;
    std::unique_ptr<Engine> E;
    int64_t n = 0, m = 0;
    DevBuf<double> cs, olb, oub, rs, shift, orl, oru;       // KKT constants, engine order
    DevBuf<double> k_ax, k_aty[2], k_qx, best_x, best_y, epoch_x, epoch_y, epoch_aty, part, out;
    double *host_out = nullptr; // pinned: 2 candidates x kKktValues, 2 displacement sums,
                                // 3 rays x kRayValues
    int grid = 148;
    double os = 1, cscale = 1, offset_o = 0, offset_s = 0, cfixed = 0;
    bool orig_is_qp = false; // the caller's model has quadratic terms (cached: O(n) to test)
    std::vector<int64_t> cperm, rperm; // engine position -> prepared index

    DeviceSolve(const Prepared &p, const HostModel &o) : prep(p), orig(o) {}
    ~DeviceSolve() {
        if (host_out)
            cudaFreeHost(host_out);
    }

    void build(const std::vector<double> &x0, const std::vector<double> &y0, int precision,
               int index_bits, bool adaptive, bool graphs) {
        const HostModel &pm = prep.model;
        n = int64_t(pm.c.size());
        m = int64_t(pm.rl.size());
        nk_csr A{pm.A.rows, pm.A.cols, pm.A.ptr.data(), pm.A.index.data(), pm.A.value.data()};
        nk_csr Q{pm.Q.rows, pm.Q.cols, pm.Q.ptr.data(), pm.Q.index.data(), pm.Q.value.data()};
        nk_pdhg_options eo{};
        eo.adaptive = adaptive;
        eo.graphs = graphs;
        eo.index_bits = index_bits;
        eo.precision = precision;
        E.reset(create_engine(&A, pm.Q.value.empty() ? nullptr : &Q, pm.c.data(), pm.q.data(),
                              pm.lb.data(), pm.ub.data(), pm.rl.data(), pm.ru.data(), x0.data(),
                              y0.data(), &eo));
        cudaStream_t s = E->stream;
        cperm.resize(size_t(n));
        rperm.resize(size_t(m));
        if (n)
            cuda_check(cudaMemcpy(cperm.data(), E->col_perm.p, size_t(n) * 8, cudaMemcpyDeviceToHost),
                       "column order");
        if (m)
            cuda_check(cudaMemcpy(rperm.data(), E->row_perm.p, size_t(m) * 8, cudaMemcpyDeviceToHost),
                       "row order");
        // constants of the original-space evaluation
        orig_is_qp = orig.is_qp();
        os = prep.objective_scale;
        offset_o = orig.offset;
        offset_s = pm.offset;
        cscale = 1;
        for (double v : orig.c)
            cscale = std::max(cscale, 1 + std::abs(v));
        long double fixed_terms = 0;
        std::vector<char> kept(orig.c.size(), 0);
        for (auto j : prep.cols)
            kept[size_t(j)] = 1;
        for (size_t j = 0; j < orig.c.size(); ++j)
            if (!kept[j]) {
                long double v = prep.fixed[j];
                fixed_terms += orig.c[j] * v + .5L * orig.q[j] * v * v;
            }
        cfixed = double(fixed_terms);
        std::vector<double> h(size_t(std::max(n, m)));
        auto put = [&](DevBuf<double> &d, int64_t len, auto &&value) {
            d.alloc(size_t(std::max<int64_t>(1, len)));
            for (int64_t i = 0; i < len; ++i)
                h[size_t(i)] = value(i);
            if (len)
                cuda_check(cudaMemcpy(d.p, h.data(), size_t(len) * 8, cudaMemcpyHostToDevice), "constants");
        };
        put(cs, n, [&](int64_t i) { return prep.column_scale[size_t(cperm[size_t(i)])]; });
        put(olb, n, [&](int64_t i) { return orig.lb[size_t(prep.cols[size_t(cperm[size_t(i)])])]; });
        put(oub, n, [&](int64_t i) { return orig.ub[size_t(prep.cols[size_t(cperm[size_t(i)])])]; });
        put(rs, m, [&](int64_t i) { return prep.row_scale[size_t(rperm[size_t(i)])]; });
        put(orl, m, [&](int64_t i) { return orig.rl[size_t(prep.lower_rows[size_t(rperm[size_t(i)])])]; });
        put(oru, m, [&](int64_t i) { return orig.ru[size_t(prep.upper_rows[size_t(rperm[size_t(i)])])]; });
        // activity of the removed (fixed) columns in every kept row, the
        // reference's `shift` (long double sum, src/preprocess.cpp:200-210)
        {
            std::vector<double> sh(size_t(m), 0.0);
            std::vector<char> fixedcol(orig.c.size(), 0);
            for (size_t j = 0; j < orig.c.size(); ++j)
                fixedcol[j] = !kept[j];
            for (int64_t r = 0; r < m; ++r) {
                int64_t i = prep.rows[size_t(r)];
                long double acc = 0;
                for (int64_t k = orig.A.ptr[size_t(i)]; k < orig.A.ptr[size_t(i + 1)]; ++k) {
                    int64_t j = orig.A.index[size_t(k)];
                    if (fixedcol[size_t(j)])
                        acc += (long double)orig.A.value[size_t(k)] * prep.fixed[size_t(j)];
                }
                sh[size_t(r)] = double(acc);
            }
            put(shift, m, [&](int64_t i) { return sh[size_t(rperm[size_t(i)])]; });
        }
        auto vec = [&](DevBuf<double> &d, int64_t len) { d.alloc(size_t(std::max<int64_t>(1, len))); };
        vec(k_ax, m);
        vec(k_aty[0], n);
        vec(k_aty[1], n);
        vec(epoch_aty, n);
        vec(k_qx, n);
        vec(best_x, n);
        vec(best_y, m);
        vec(epoch_x, n);
        vec(epoch_y, m);
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        grid = int(std::max<int64_t>(1, std::min<int64_t>(int64_t(sms) * 4, (std::max(n, m) + kThreads - 1) / kThreads)));
        part.alloc(size_t(grid) * std::max(kKktValues, kRayValues));
        out.alloc(kOutValues);
        cuda_check(cudaMallocHost(reinterpret_cast<void **>(&host_out), kOutValues * sizeof(double)),
                   "pinned");
        int cur = current();
        copy(best_x.p, E->x[cur].p, n);
        copy(best_y.p, E->y[cur].p, m);
        set_epoch(cur);
        cuda_check(cudaStreamSynchronize(s), "driver setup");
    }

    static constexpr int kOutValues = 2 * kKktValues + 2 + 3 * kRayValues;
    static constexpr int kRayOut = 2 * kKktValues + 2;

    // epoch = current iterate (after a restart), with its A^T epoch_y
    void set_epoch(int cur) {
        copy(epoch_x.p, E->x[cur].p, n);
        copy(epoch_y.p, E->y[cur].p, m);
        if (n)
            E->spmv(E->At, epoch_y.p, epoch_aty.p);
    }
    void copy(double *dst, const double *src, int64_t len) {
        if (len)
            cuda_check(cudaMemcpyAsync(dst, src, size_t(len) * 8, cudaMemcpyDeviceToDevice, E->stream),
                       "device copy");
    }
    // Folds the pending average and returns the index of the current iterate.
    int current() {
        E->flush();
        E->sync_ctl();
        return E->host_ctl->cur;
    }

    // Launches the evaluation of the prepared point (x, y) into out[slot]; the
    // products A x, A^T y (and Q x) are recomputed, not taken from the
    // engine's incrementally updated activity.
    KktArgs args(const double *x, const double *y, int slot) {
        return KktArgs{n, m, x, y, k_ax.p, k_aty[slot].p, E->sparse_q ? k_qx.p : nullptr, E->c.p,
                       E->q.p, cs.p, olb.p, oub.p, rs.p, shift.p, orl.p, oru.p, os, cscale,
                       E->sparse_q ? 1 : 0};
    }
    void evaluate(const double *x, const double *y, int slot) {
        cudaStream_t s = E->stream;
        if (m)
            E->spmv(E->A, x, k_ax.p);
        if (n)
            E->spmv(E->At, y, k_aty[slot].p);
        if (E->sparse_q)
            E->q_spmv(x, k_qx.p);
        KktArgs a = args(x, y, slot);
        kkt_partial<<<grid, kThreads, 0, s>>>(a, part.p);
        finish_partials<kKktValues><<<1, kThreads, 0, s>>>(part.p, grid, kKktMaxMask,
                                                          out.p + slot * kKktValues);
        cuda_check(cudaGetLastError(), "kkt evaluation");
    }
    void displacement(const double *x, const double *y) {
        cudaStream_t s = E->stream;
        displacement_partial<<<grid, kThreads, 0, s>>>(n, m, x, epoch_x.p, y, epoch_y.p, part.p);
        finish_partials<2><<<1, kThreads, 0, s>>>(part.p, grid, 0u, out.p + 2 * kKktValues);
        cuda_check(cudaGetLastError(), "displacement");
    }
    // Screens the three candidate rays of the infeasibility test on the device:
    // ray 0 the chosen candidate's y (slot `chosen`), ray 1 the other one's,
    // ray 2 the chosen y minus the epoch y.  Returns, per ray, whether the
    // outward-rounded host bound could still be positive.
    std::array<bool, 3> screen_rays(const double *y_chosen, int chosen, const double *y_other) {
        cudaStream_t s = E->stream;
        const double *ys[3] = {y_chosen, y_other, y_chosen};
        const double *eys[3] = {nullptr, nullptr, epoch_y.p};
        const double *atys[3] = {k_aty[chosen].p, k_aty[1 - chosen].p, k_aty[chosen].p};
        const double *ateys[3] = {nullptr, nullptr, epoch_aty.p};
        KktArgs a = args(nullptr, nullptr, 0);
        for (int r = 0; r < 3; ++r) {
            ray_screen<<<grid, kThreads, 0, s>>>(n, m, ys[r], eys[r], atys[r], ateys[r], a, part.p);
            finish_partials<kRayValues><<<1, kThreads, 0, s>>>(part.p, grid, 1u,
                                                               out.p + kRayOut + r * kRayValues);
        }
        cuda_check(cudaGetLastError(), "ray screen");
        cuda_check(cudaMemcpyAsync(host_out + kRayOut, out.p + kRayOut, 3 * kRayValues * 8,
                                   cudaMemcpyDeviceToHost, s), "ray screen");
        cuda_check(cudaStreamSynchronize(s), "ray screen");
        std::array<bool, 3> ok{};
        for (int r = 0; r < 3; ++r) {
            const double *v = host_out + kRayOut + r * kRayValues;
            // FP64 sums of the bound's terms err by far less than 1e-9 of their
            // magnitude: at or below that margin the exact bound cannot be
            // positive (a zero ray has bound 0 and magnitude 0)
            ok[size_t(r)] = v[0] == 0 && v[1] + v[2] + 1e-9 * v[3] > 0;
        }
        return ok;
    }
    void fetch(int values) {
        cuda_check(cudaMemcpyAsync(host_out, out.p, size_t(values) * 8, cudaMemcpyDeviceToHost, E->stream),
                   "evaluation result");
        cuda_check(cudaStreamSynchronize(E->stream), "evaluation sync");
    }

    // Verifier::evaluate(x, y, false) assembled from the device partials.
    Accuracy finish(const double *v) const {
        Accuracy a;
        if (v[9] != 0)
            return a;
        a.primal = v[0];
        a.primal_absolute = v[1];
        a.dual = v[2];
        a.dual_absolute = v[3];
        a.objective = os * (offset_s + v[4]);
        a.complementarity = v[5];
        a.gap = a.complementarity / (1 + std::abs(a.objective - offset_o));
        if (v[8] == 0) {
            const double support = v[6], box = v[7] + cfixed;
            long double lower = (long double)offset_o - support + box;
            long double guard = 64 * std::numeric_limits<double>::epsilon() *
                                (1 + std::abs((long double)offset_o) + std::abs((long double)support) +
                                 std::abs((long double)box));
            a.lower_bound = double(lower - guard);
            a.gap = std::max(a.gap, std::abs(a.objective - a.lower_bound) /
                                        (1 + std::abs(a.objective) + std::abs(a.lower_bound)));
        }
        if (!orig_is_qp)
            a.lower_bound = -kInf;
        a.kkt = std::max({a.primal, a.dual, a.gap});
        a.finite = std::isfinite(a.objective) && std::isfinite(a.kkt) && std::isfinite(a.gap) &&
                   std::isfinite(a.primal) && std::isfinite(a.dual);
        if (!a.finite) {
            a.kkt = kInf;
            a.lower_bound = -kInf;
        }
        return a;
    }

    // Prepared-space vectors (prepared order) of a device vector in engine order.
    std::vector<double> download_cols(const double *d) {
        std::vector<double> h(static_cast<size_t>(n));
        E->download_x(h.data(), d);
        return h;
    }
    std::vector<double> download_rows(const double *d) {
        std::vector<double> h(static_cast<size_t>(m));
        E->download_y(h.data(), d);
        return h;
    }
};

struct DriverOptions {
    double tol = 1e-6, time_limit = 60;
    int64_t iteration_limit = 100000;
    int check_every = 100;
    bool adaptive = true, restart = true, graphs = true;
    int index_bits = 0;
    bool verbose = false;
    const volatile int *cancel = nullptr; // nonzero: stop at the next check (INTERRUPTED)
};

// Iterates one DeviceSolve until its device estimate reaches `target` (and, if
// `certify`, the host verifier accepts), or a limit.  Mirrors the loop of
// solve_continuous (src/solver.cpp:510-775) with polishing off.
struct Driver {
    DeviceSolve &D;
    const Verifier &verifier;
    const DriverOptions &o;
    SolveReport &R;
    SteadyClock::time_point start;
    double step = 1, weight = 1;
    double restart_kkt;
    int64_t since_restart = 0, previous_rejected = 0, next_host_check = 0, checks = 0;
    Accuracy best;

    Driver(DeviceSolve &d, const Verifier &v, const DriverOptions &opt, SolveReport &r,
           SteadyClock::time_point t0, double initial_kkt)
        : D(d), verifier(v), o(opt), R(r), start(t0), restart_kkt(initial_kkt) {}

    // Host certification of a device candidate (caller order, original space).
    Accuracy host_check(const double *x, const double *y, std::vector<double> &ox,
                        std::vector<double> &oy, bool safe) {
        auto cx = D.download_cols(x);
        auto cy = D.download_rows(y);
        ox = D.prep.restore_x(cx);
        oy = D.prep.restore_y(cy, D.orig.rl.size());
        R.host_checks++;
        return verifier.evaluate(ox, oy, safe);
    }

    // Returns true when the model is solved (status set), false at a limit.
    // `certify` false: stop as soon as the device estimate reaches target.
    bool run(double target, bool certify, int64_t iteration_cap) {
        Engine &E = *D.E;
        const int64_t n = D.n, m = D.m;
        int stagnant = 0;
        double stagnant_ref = kInf;
        while (R.iterations < iteration_cap) {
            // stop_requested, then the time limit, as src/solver.cpp:516-523 orders them
            if (o.cancel && *o.cancel) {
                R.status = NK_SOLVE_INTERRUPTED;
                return false;
            }
            if (since(start) >= o.time_limit) {
                R.status = NK_SOLVE_TIME_LIMIT;
                return false;
            }
            int count = int(std::min<int64_t>(o.check_every, iteration_cap - R.iterations));
            auto tick = SteadyClock::now();
            int accepted = E.advance(count, step / weight, step * weight);
            R.iteration += since(tick);
            R.iterations += accepted;
            since_restart += accepted;
            R.rejected += E.rejected - previous_rejected;
            previous_rejected = E.rejected;
            tick = SteadyClock::now();
            int cur = D.current();
            D.evaluate(E.x[cur].p, E.y[cur].p, 0);
            D.evaluate(E.xa.p, E.ya.p, 1);
            D.fetch(2 * kKktValues);
            R.device_checks++;
            checks++;
            Accuracy ca = D.finish(D.host_out), aa = D.finish(D.host_out + kKktValues);
            bool avg = aa.kkt < ca.kkt;
            if (avg)
                ca = aa;
            const double *cx = avg ? E.xa.p : E.x[cur].p;
            const double *cy = avg ? E.ya.p : E.y[cur].p;
            if (ca.finite && ca.kkt < best.kkt) {
                D.copy(D.best_x.p, cx, n);
                D.copy(D.best_y.p, cy, m);
                best = ca;
                double level = 1;
                for (int k = 0; k < 9; ++k, level /= 10)
                    if (best.kkt <= level && R.reached[k] < 0)
                        R.reached[k] = since(start);
            }
            R.verification += since(tick);
            if (o.verbose)
                std::fprintf(stderr, "iter=%lld objective=%.10g primal=%.3e dual=%.3e gap=%.3e seconds=%.3f\n",
                             (long long)R.iterations, ca.objective, ca.primal, ca.dual, ca.gap,
                             since(start));
            if (!ca.finite) {
                R.status = NK_SOLVE_NUMERICAL_ERROR;
                return true;
            }
            if (ca.kkt <= target) {
                if (!certify)
                    return true;
                if (R.iterations >= next_host_check) {
                    tick = SteadyClock::now();
                    std::vector<double> ox, oy;
                    Accuracy h = host_check(cx, cy, ox, oy, true);
                    R.verification += since(tick);
                    if (h.kkt <= o.tol) {
                        R.x = std::move(ox);
                        R.y = std::move(oy);
                        R.accuracy = h;
                        R.status = NK_SOLVE_OPTIMAL;
                        return true;
                    }
                    // the estimate and the certified value disagree near the
                    // tolerance; certify again only after more progress
                    next_host_check = R.iterations + std::max<int64_t>(1000, 10 * o.check_every);
                }
            }
            // infeasibility certificates (src/solver.cpp:599-633): the rays the
            // device screen cannot rule out go to the outward-rounded host test
            if (certify && R.iterations >= 1000 && ca.primal > o.tol) {
                tick = SteadyClock::now();
                const double *other_y = avg ? E.y[cur].p : E.ya.p;
                auto ok = D.screen_rays(cy, avg ? 1 : 0, other_y);
                if ((ok[0] || ok[1] || ok[2]) &&
                    infeasible(ok[0] ? cy : nullptr, ok[1] ? other_y : nullptr,
                               ok[2] ? cy : nullptr))
                    return true;
                R.verification += since(tick);
            }
            // a mixed-precision phase ends when its estimate stops improving
            if (!certify) {
                if (best.kkt < .9 * stagnant_ref) {
                    stagnant_ref = best.kkt;
                    stagnant = 0;
                } else if (++stagnant >= 30)
                    return true;
            }
            bool restart_due = since_restart >= int64_t(o.check_every) * 2 &&
                               (ca.kkt < .5 * restart_kkt ||
                                since_restart >= std::max<int64_t>(2000, R.iterations / 2));
            if (o.restart && restart_due) {
                if (o.adaptive) {
                    D.displacement(cx, cy);
                    cuda_check(cudaMemcpyAsync(D.host_out + 2 * kKktValues, D.out.p + 2 * kKktValues,
                                               16, cudaMemcpyDeviceToHost, E.stream), "displacement");
                    cuda_check(cudaStreamSynchronize(E.stream), "displacement");
                    double dx = D.host_out[2 * kKktValues], dy = D.host_out[2 * kKktValues + 1];
                    if (dx > 1e-24 && dy > 1e-24) {
                        double target_w = std::clamp(std::sqrt(dy / dx), 1e-4, 1e4);
                        weight = std::sqrt(weight * target_w);
                        R.weight_updates++;
                    }
                }
                E.reset_candidate(avg);
                D.set_epoch(D.current());
                restart_kkt = ca.kkt;
                since_restart = 0;
                R.restarts++;
            }
        }
        return false;
    }

    // Rays from the chosen and the other candidate's dual and from the chosen
    // dual's displacement since the last restart, scaled to unit max norm and
    // certified by the outward-rounded Farkas bound; null: ruled out on the device.
    bool infeasible(const double *chosen, const double *other, const double *displaced) {
        std::vector<std::vector<double>> rays;
        if (chosen)
            rays.push_back(D.download_rows(chosen));
        if (other)
            rays.push_back(D.download_rows(other));
        if (displaced) {
            auto y = D.download_rows(displaced);
            auto e = D.download_rows(D.epoch_y.p);
            for (size_t i = 0; i < y.size(); ++i)
                y[i] -= e[i];
            rays.push_back(std::move(y));
        }
        R.host_checks++;
        for (auto &src : rays) {
            auto ray = D.prep.restore_y(src, D.orig.rl.size());
            double norm = 0;
            bool finite = true;
            for (double v : ray) {
                finite = finite && std::isfinite(v);
                norm = std::max(norm, std::abs(v));
            }
            if (!finite || !(norm > 0))
                continue;
            for (double &v : ray)
                v /= norm;
            double margin = verifier.infeasibility_bound(ray);
            if (margin > 0 && std::isfinite(margin)) {
                R.status = NK_SOLVE_INFEASIBLE;
                R.y = std::move(ray);
                return true;
            }
        }
        return false;
    }
};

// step = 0.9 / sqrt(max row l1 * max column l1), weight from ||c|| / ||b||
// (src/solver.cpp:298-333)
inline void initial_steps(const HostModel &m, bool adaptive, double &step, double &weight) {
    std::vector<double> colsum(m.c.size());
    double rowmax = 0;
    for (size_t i = 0; i < m.rl.size(); i++) {
        double s = 0;
        for (auto k = m.A.ptr[i]; k < m.A.ptr[i + 1]; k++) {
            double v = std::abs(m.A.value[size_t(k)]);
            s += v;
            colsum[size_t(m.A.index[size_t(k)])] += v;
        }
        rowmax = std::max(rowmax, s);
    }
    double colmax = 0;
    for (auto s : colsum)
        colmax = std::max(colmax, s);
    double norm = std::sqrt(rowmax) * std::sqrt(colmax);
    step = norm > 0 ? .9 / norm : 1;
    weight = 1;
    if (adaptive) {
        long double c2 = 0, b2 = 0;
        for (auto c : m.c)
            c2 += (long double)c * c;
        for (size_t i = 0; i < m.rl.size(); i++) {
            double b = std::clamp(0., m.rl[i], m.ru[i]);
            b2 += (long double)b * b;
        }
        if (c2 > 1e-24 && b2 > 1e-24)
            weight = std::clamp(std::sqrt(double(c2 / b2)), 1e-4, 1e4);
    }
}

struct SolveSettings {
    DriverOptions driver;
    PrepareOptions prepare;
    int precision = NK_PRECISION_FP64; // matrices of the first phase
    bool refine = true;                // FP64 phase after a reduced-precision one
    double phase_tol = 0;              // target of the reduced-precision phase (0: 10 * tol)
    std::vector<double> initial_x, initial_y;
};

inline SolveReport solve(const HostModel &original, const SolveSettings &S) {
    auto start = SteadyClock::now();
    SolveReport R;
    const DriverOptions &o = S.driver;
    // The verifier (its transpose of A) is built on a second host thread while
    // prepare runs: both only read the caller's model, and prepare's serial
    // stretches leave host cores free.  The thread follows this thread's
    // serial-host setting.
    std::unique_ptr<Verifier> owned_verifier;
    std::exception_ptr verifier_error;
    const bool serial = host_serial_enabled();
    std::thread build_verifier([&] {
        host_serial(serial);
        try {
            owned_verifier = std::make_unique<Verifier>(original);
        } catch (...) {
            verifier_error = std::current_exception();
        }
    });
    Prepared prep;
    try {
        prep = prepare(original, S.prepare);
    } catch (...) {
        build_verifier.join();
        throw;
    }
    build_verifier.join();
    if (verifier_error)
        std::rethrow_exception(verifier_error);
    const Verifier &verifier = *owned_verifier;
    R.preprocess = since(start);
    auto done = [&](int status) {
        R.status = status;
        R.seconds = since(start);
        return R;
    };
    if (!prep.failure.empty()) {
        if (!prep.failure_ray.empty())
            R.y = prep.failure_ray;
        return done(prep.failure == "INFEASIBLE" ? NK_SOLVE_INFEASIBLE : NK_SOLVE_NUMERICAL_ERROR);
    }
    const HostModel &pm = prep.model;
    R.removed_columns = int64_t(original.c.size() - pm.c.size());
    R.removed_rows = int64_t(original.rl.size() - pm.rl.size());
    std::vector<double> x(pm.c.size()), y(pm.rl.size());
    for (size_t j = 0; j < x.size(); j++) {
        double initial = S.initial_x.empty() ? 0 : S.initial_x[size_t(prep.cols[j])];
        x[j] = std::clamp(initial / prep.column_scale[j], pm.lb[j], pm.ub[j]);
    }
    for (size_t i = 0; i < y.size(); i++)
        if (!S.initial_y.empty())
            y[i] = S.initial_y[size_t(prep.rows[i])] / (prep.row_scale[i] * prep.objective_scale);
    R.x = prep.restore_x(x);
    R.y = prep.restore_y(y, original.rl.size());
    auto tick = SteadyClock::now();
    R.accuracy = verifier.evaluate(R.x, R.y);
    R.verification += since(tick);
    // isolated improving column at a feasible start (src/solver.cpp:268-287)
    if (R.accuracy.finite && R.accuracy.primal_absolute == 0) {
        std::vector<bool> used(pm.c.size(), false);
        for (auto j : pm.A.index)
            used[size_t(j)] = true;
        for (int64_t i = 0; i < pm.Q.rows; ++i)
            for (auto k = pm.Q.ptr[size_t(i)]; k < pm.Q.ptr[size_t(i + 1)]; ++k) {
                used[size_t(i)] = true;
                used[size_t(pm.Q.index[size_t(k)])] = true;
            }
        for (size_t j = 0; j < x.size(); j++)
            if (!used[j] && pm.q[j] == 0 &&
                ((pm.c[j] < 0 && pm.ub[j] == kInf) || (pm.c[j] > 0 && pm.lb[j] == -kInf)))
                return done(NK_SOLVE_UNBOUNDED);
    }
    if (R.accuracy.finite && R.accuracy.kkt <= o.tol)
        return done(NK_SOLVE_OPTIMAL);
    if (o.time_limit == 0)
        return done(NK_SOLVE_TIME_LIMIT);
    double step = 1, weight = 1;
    initial_steps(pm, o.adaptive, step, weight);
    const bool phased = S.precision != NK_PRECISION_FP64;
    auto transfer = SteadyClock::now();
    auto D = std::make_unique<DeviceSolve>(prep, original);
    D->build(x, y, S.precision, o.index_bits, o.adaptive, o.graphs);
    R.transfer += since(transfer);
    Driver drv(*D, verifier, o, R, start, R.accuracy.kkt);
    drv.step = step;
    drv.weight = weight;
    Accuracy best;
    if (phased) {
        double target = S.phase_tol > 0 ? S.phase_tol : 10 * o.tol;
        try {
            drv.run(S.refine ? target : o.tol, !S.refine, o.iteration_limit);
        } catch (const Error &e) {
            // backtracking that stalls on the reduced-precision values ends the
            // phase: the FP64 refinement restarts from the best point
            if (e.status != NK_ERR_STALLED || !S.refine || !drv.best.finite)
                throw;
        }
        best = drv.best;
        R.mixed_iterations = R.iterations;
        R.mixed_seconds = since(start);
        // the reduced-precision result, verified on the host (no safe bound)
        if (best.finite) {
            std::vector<double> ox, oy;
            tick = SteadyClock::now();
            R.mixed = drv.host_check(D->best_x.p, D->best_y.p, ox, oy, false);
            R.verification += since(tick);
        }
        bool stopped = R.status == NK_SOLVE_TIME_LIMIT || R.status == NK_SOLVE_INFEASIBLE ||
                       R.status == NK_SOLVE_OPTIMAL || R.status == NK_SOLVE_INTERRUPTED ||
                       R.iterations >= o.iteration_limit;
        if (S.refine && !stopped && best.finite) {
            // closing FP64 refinement, restarted from the best reduced-precision point
            auto bx = D->download_cols(D->best_x.p);
            auto by = D->download_rows(D->best_y.p);
            double w = drv.weight;
            D.reset();
            transfer = SteadyClock::now();
            D = std::make_unique<DeviceSolve>(prep, original);
            D->build(bx, by, NK_PRECISION_FP64, o.index_bits, o.adaptive, o.graphs);
            R.transfer += since(transfer);
            Driver fine(*D, verifier, o, R, start, best.kkt);
            fine.step = step;
            fine.weight = w;
            fine.best = best;
            R.status = NK_SOLVE_ITERATION_LIMIT;
            int64_t before = R.iterations;
            fine.run(o.tol, true, o.iteration_limit);
            R.refine_iterations = R.iterations - before;
            best = fine.best;
        }
    } else {
        drv.run(o.tol, true, o.iteration_limit);
        best = drv.best;
    }
    if (R.status != NK_SOLVE_OPTIMAL && R.status != NK_SOLVE_INFEASIBLE) {
        // best point seen, certified like the reference's closing evaluate
        tick = SteadyClock::now();
        if (best.finite && best.kkt < R.accuracy.kkt) {
            std::vector<double> ox, oy;
            Driver last(*D, verifier, o, R, start, best.kkt);
            Accuracy h = last.host_check(D->best_x.p, D->best_y.p, ox, oy, true);
            if (h.finite && (h.kkt < R.accuracy.kkt || !R.accuracy.finite)) {
                R.x = std::move(ox);
                R.y = std::move(oy);
                R.accuracy = h;
            }
        }
        R.verification += since(tick);
    }
    R.seconds = since(start);
    return R;
}

} // namespace nk
