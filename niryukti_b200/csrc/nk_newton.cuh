// BiCGSTAB for the barrier method's Newton systems (cuda_linear_solve,
// src/cuda.cu:1304-1434; caller src/barrier.cpp:280-300).  The optimizer logic
// stays with the reference's barrier.cpp; this solves K x = b on the GPU.
//
// Every vector and every scalar of the iteration lives on the device: the dot
// products are two-stage fixed-tree reductions, and the step scalars (rho,
// alpha, omega, beta) are formed by a one-thread kernel in the reference's
// expressions and order, so nothing but a four-flag status crosses PCIe per
// iteration.  The operator is CSR, one warp per row (lane-strided entries, a
// fixed shuffle tree), with FP64 or FP32 values and FP64 vectors and sums.
// Included by nk_engine.cu.
#pragma once
#include "nk_common.cuh"
#include "nk_kernels.cuh"
#include <chrono>
#include <cmath>
#include <cstdint>
#include <vector>

namespace nk {

struct NewtonState {
    double rho, previous, alpha, omega, beta, divisor, ss, tt, ts, rr, target;
    int stop;      // 0 running, 1 converged, 2 breakdown
    int converged; // 1 once a residual met the target
};

template <class V>
__global__ void newton_spmv(int64_t n, const int64_t *__restrict__ ptr,
                            const int64_t *__restrict__ idx, const V *__restrict__ val,
                            const double *__restrict__ x, double *__restrict__ y,
                            const NewtonState *st) {
    if (st->stop)
        return;
    const int lane = threadIdx.x & 31;
    const int64_t first = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t r = first; r < n; r += stride) {
        double acc = 0;
        for (int64_t k = ptr[r] + lane; k < ptr[r + 1]; k += 32)
            acc += double(val[k]) * x[idx[k]];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0)
            y[r] = acc;
    }
}

// part[block] = sum of a[j] * b[j] over the block's grid-stride share
__global__ void newton_dot_partial(int64_t n, const double *__restrict__ a,
                                   const double *__restrict__ b, double *__restrict__ part,
                                   const NewtonState *st) {
    __shared__ double red[kWarps];
    if (st->stop)
        return; // block-uniform
    double v = 0;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += stride)
        v += a[j] * b[j];
    double t[1] = {v};
    cta_sum<1>(t, red);
    if (threadIdx.x == 0)
        part[blockIdx.x] = t[0];
}
// *out = sum of part[0 .. blocks) in a fixed order
__global__ void newton_dot_finish(int blocks, const double *__restrict__ part, double *out,
                                  const NewtonState *st) {
    __shared__ double red[kWarps];
    if (st->stop)
        return;
    double v = 0;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x)
        v += part[b];
    double t[1] = {v};
    cta_sum<1>(t, red);
    if (threadIdx.x == 0)
        *out = t[0];
}

// The iteration's scalar steps, one thread; `step` says which point of the
// iteration has been reached (the reference's host statements in order).
__global__ void newton_scalars(NewtonState *s, int step) {
    if (s->stop)
        return;
    switch (step) {
    case 0: // rho known: breakdown test, beta
        if (!isfinite(s->rho) || fabs(s->rho) < 1e-300 || fabs(s->omega) < 1e-300) {
            s->stop = 2;
            return;
        }
        s->beta = (s->rho / s->previous) * (s->alpha / s->omega);
        break;
    case 1: // divisor known: alpha
        if (!isfinite(s->divisor) || fabs(s->divisor) < 1e-300) {
            s->stop = 2;
            return;
        }
        s->alpha = s->rho / s->divisor;
        break;
    case 2: // ss known: early exit on s (x is updated by the caller's kernel)
        if (sqrt(s->ss) <= s->target) {
            s->converged = 1;
            s->stop = 3; // x += alpha p still to do, then stop
        }
        break;
    case 3: // tt, ts known: omega
        if (!isfinite(s->tt) || s->tt < 1e-300) {
            s->stop = 2;
            return;
        }
        s->omega = s->ts / s->tt;
        break;
    case 4: // rr known
        s->converged = sqrt(s->rr) <= s->target;
        if (s->converged)
            s->stop = 1;
        s->previous = s->rho;
        break;
    }
}

// out = ca a + cb b + cc c with the coefficients of `which` (the reference's
// linear_combine calls): 0 p = r + beta p - beta omega v; 1 s = r - alpha v;
// 2 x = x + alpha p (exit on s); 3 x = x + alpha p + omega s; 4 r = s - omega t.
__global__ void newton_combine(int64_t n, double *out, const double *a, const double *b,
                               const double *c, NewtonState *st, int which) {
    const int stop = st->stop;
    if (which == 2 ? stop != 3 : stop != 0)
        return;
    double ca = 1, cb = 0, cc = 0;
    switch (which) {
    case 0: cb = st->beta; cc = -st->beta * st->omega; break;
    case 1: cb = -st->alpha; break;
    case 2: cb = st->alpha; break;
    case 3: cb = st->alpha; cc = st->omega; break;
    default: cb = -st->omega; break;
    }
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += stride)
        out[j] = ca * a[j] + cb * b[j] + cc * c[j];
}
// out = dinv * in (the right preconditioner), while the iteration runs
__global__ void newton_scale(int64_t n, double *__restrict__ out, const double *__restrict__ dinv,
                             const double *__restrict__ in, const NewtonState *st) {
    if (st->stop)
        return;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += stride)
        out[j] = dinv[j] * in[j];
}
__global__ void newton_mark_done(NewtonState *st) {
    if (st->stop == 3)
        st->stop = 1;
}

// Diagonal right preconditioner of a Newton matrix, 1 / (its scale) per row:
// |K_ii| where the diagonal carries the row; where it does not (a saddle
// point's regularised zero block, |K_ii| < 1e-8 max_j |K_ij|), the diagonal of
// the row's Schur complement, sum_j K_ij^2 / |K_jj| over the other entries.
// Rows with neither keep 1.
inline std::vector<double> newton_diagonal(const nk_csr &K) {
    const int64_t n = K.rows;
    std::vector<double> diag(static_cast<size_t>(n), 0.0), big(static_cast<size_t>(n), 0.0),
        dinv(static_cast<size_t>(n), 1.0);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t k = K.ptr[i]; k < K.ptr[i + 1]; ++k) {
            big[size_t(i)] = std::max(big[size_t(i)], std::fabs(K.value[k]));
            if (K.index[k] == i)
                diag[size_t(i)] += K.value[k];
        }
    auto carries = [&](int64_t i) {
        return std::fabs(diag[size_t(i)]) >= 1e-8 * big[size_t(i)] && diag[size_t(i)] != 0;
    };
    for (int64_t i = 0; i < n; ++i) {
        if (carries(i)) {
            dinv[size_t(i)] = 1 / std::fabs(diag[size_t(i)]);
            continue;
        }
        double schur = 0;
        for (int64_t k = K.ptr[i]; k < K.ptr[i + 1]; ++k) {
            const int64_t j = K.index[k];
            if (j != i && carries(j))
                schur += K.value[k] * K.value[k] / std::fabs(diag[size_t(j)]);
        }
        if (schur > 0 && std::isfinite(schur))
            dinv[size_t(i)] = 1 / schur;
    }
    return dinv;
}

// Solves K x = rhs (K: n x n CSR, host arrays) by BiCGSTAB, right-preconditioned
// by newton_diagonal when `precondition` (without it, the iteration is the
// reference's one exactly: every scaling is by 1).  The residual r stays the
// unpreconditioned one, so the stopping test is the reference's.  Returns true
// when a residual met the target ((fp32 ? 1e-6 : 1e-10) (1 + |rhs|)) before
// breakdown, the iteration cap (min(20000, 10 n + 100)) or the time limit; x
// gets the last iterate either way.  The arguments are checked by the caller.
inline bool newton_solve(const nk_csr &K, const double *rhs, bool fp32, bool precondition,
                         double time_limit, double *x_out, bool *timed_out) {
    const int64_t n = K.rows, nnz = K.ptr[K.rows];
    *timed_out = false;
    cudaStream_t s = nullptr;
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "Newton stream");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard_stream{s};
    const size_t nn = size_t(n), nz = size_t(std::max<int64_t>(1, nnz));
    DevBuf<int64_t> dptr(nn + 1), didx(nz);
    DevBuf<double> val64(fp32 ? 1 : nz);
    DevBuf<float> val32(fp32 ? nz : 1);
    DevBuf<double> x(nn), r(nn), anchor(nn), p(nn), v(nn), sv(nn), t(nn), y(nn), z(nn), dinv(nn);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int vgrid = int(std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads,
                                                                 int64_t(sms) * 4)));
    const int mgrid = int(std::max<int64_t>(1, std::min<int64_t>((n + kWarps - 1) / kWarps,
                                                                 int64_t(sms) * 8)));
    DevBuf<double> part(static_cast<size_t>(vgrid));
    DevBuf<NewtonState> st(1);
    cuda_check(cudaMemcpyAsync(dptr.p, K.ptr, (nn + 1) * 8, cudaMemcpyHostToDevice, s), "Newton ptr");
    if (nnz) {
        cuda_check(cudaMemcpyAsync(didx.p, K.index, size_t(nnz) * 8, cudaMemcpyHostToDevice, s),
                   "Newton idx");
        if (fp32) {
            std::vector<float> f(K.value, K.value + nnz);
            cuda_check(cudaMemcpyAsync(val32.p, f.data(), size_t(nnz) * 4, cudaMemcpyHostToDevice, s),
                       "Newton values");
            cuda_check(cudaStreamSynchronize(s), "Newton values"); // f leaves scope
        } else
            cuda_check(cudaMemcpyAsync(val64.p, K.value, size_t(nnz) * 8, cudaMemcpyHostToDevice, s),
                       "Newton values");
    }
    const std::vector<double> hdinv =
        precondition ? newton_diagonal(K) : std::vector<double>(nn, 1.0);
    cuda_check(cudaMemcpyAsync(dinv.p, hdinv.data(), nn * 8, cudaMemcpyHostToDevice, s),
               "Newton preconditioner");
    cuda_check(cudaMemcpyAsync(r.p, rhs, nn * 8, cudaMemcpyHostToDevice, s), "Newton rhs");
    cuda_check(cudaMemcpyAsync(anchor.p, rhs, nn * 8, cudaMemcpyHostToDevice, s), "Newton rhs");
    for (double *z : {x.p, p.p, v.p})
        cuda_check(cudaMemsetAsync(z, 0, nn * 8, s), "Newton zero");
    NewtonState h{};
    h.previous = h.alpha = h.omega = 1;
    cuda_check(cudaMemcpyAsync(st.p, &h, sizeof(h), cudaMemcpyHostToDevice, s), "Newton state");
    auto dot = [&](const double *a, const double *b, double *out) {
        newton_dot_partial<<<vgrid, kThreads, 0, s>>>(n, a, b, part.p, st.p);
        newton_dot_finish<<<1, kThreads, 0, s>>>(vgrid, part.p, out, st.p);
    };
    auto multiply = [&](const double *in, double *out) {
        if (fp32)
            newton_spmv<float><<<mgrid, kThreads, 0, s>>>(n, dptr.p, didx.p, val32.p, in, out, st.p);
        else
            newton_spmv<double><<<mgrid, kThreads, 0, s>>>(n, dptr.p, didx.p, val64.p, in, out, st.p);
    };
    auto combine = [&](double *out, const double *a, const double *b, const double *c, int which) {
        newton_combine<<<vgrid, kThreads, 0, s>>>(n, out, a, b, c, st.p, which);
    };
    NewtonState *d = st.p;
    // initial residual norm and target
    dot(r.p, r.p, &d->rr);
    cuda_check(cudaMemcpyAsync(&h, st.p, sizeof(h), cudaMemcpyDeviceToHost, s), "Newton state");
    cuda_check(cudaStreamSynchronize(s), "Newton norm");
    const double norm = std::sqrt(h.rr);
    h.target = (fp32 ? 1e-6 : 1e-10) * (1 + norm);
    h.converged = norm <= h.target;
    h.stop = h.converged ? 1 : 0;
    cuda_check(cudaMemcpyAsync(st.p, &h, sizeof(h), cudaMemcpyHostToDevice, s), "Newton state");
    const int64_t cap = std::min<int64_t>(20000, 10 * n + 100);
    const auto start = std::chrono::steady_clock::now();
    for (int64_t it = 0; !h.stop && it < cap; ++it) {
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count() >=
            time_limit) {
            *timed_out = true;
            break;
        }
        dot(anchor.p, r.p, &d->rho);
        newton_scalars<<<1, 1, 0, s>>>(d, 0);
        combine(p.p, r.p, p.p, v.p, 0);
        newton_scale<<<vgrid, kThreads, 0, s>>>(n, y.p, dinv.p, p.p, d); // y = M^-1 p
        multiply(y.p, v.p);
        dot(anchor.p, v.p, &d->divisor);
        newton_scalars<<<1, 1, 0, s>>>(d, 1);
        combine(sv.p, r.p, v.p, v.p, 1);
        dot(sv.p, sv.p, &d->ss);
        newton_scalars<<<1, 1, 0, s>>>(d, 2);
        combine(x.p, x.p, y.p, y.p, 2);
        newton_mark_done<<<1, 1, 0, s>>>(d);
        newton_scale<<<vgrid, kThreads, 0, s>>>(n, z.p, dinv.p, sv.p, d); // z = M^-1 s
        multiply(z.p, t.p);
        dot(t.p, t.p, &d->tt);
        dot(t.p, sv.p, &d->ts);
        newton_scalars<<<1, 1, 0, s>>>(d, 3);
        combine(x.p, x.p, y.p, z.p, 3);
        combine(r.p, sv.p, t.p, t.p, 4);
        dot(r.p, r.p, &d->rr);
        newton_scalars<<<1, 1, 0, s>>>(d, 4);
        cuda_check(cudaGetLastError(), "Newton iteration");
        cuda_check(cudaMemcpyAsync(&h, st.p, sizeof(h), cudaMemcpyDeviceToHost, s), "Newton state");
        cuda_check(cudaStreamSynchronize(s), "Newton state");
    }
    cuda_check(cudaMemcpyAsync(x_out, x.p, nn * 8, cudaMemcpyDeviceToHost, s), "Newton solution");
    cuda_check(cudaStreamSynchronize(s), "Newton solution");
    return h.converged != 0;
}

} // namespace nk
