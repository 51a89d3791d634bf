// Host side of the batched PDHG engine (kernels: nk_batch_device.cuh).
//
// A Batch holds up to `capacity` instance slots.  Each instance is prepared on
// the host exactly like a single solve (prepare(), the reference's
// presolve/scaling; its initial point, the initial verification and the
// isolated-column recession test of solve_continuous), then admitted: its
// SELL matrices and vectors go to one device allocation of its own, and its
// chunks join the work lists.  step() runs check intervals: every active
// instance gets `check_every` PDHG trials (one CUDA graph), then the driver of
// solve_continuous runs per instance on device-evaluated candidates (the
// original-space KKT of Verifier::evaluate, best point, restart test, primal
// weight, Farkas screen), certifies terminations with the host verifier, and
// retires finished instances from the work lists.  New instances join at the
// next check boundary.  Each instance keeps its own steps, acceptance state,
// restarts, counters and termination; instances never exchange data.
#pragma once

#include "nk_batch_device.cuh"

namespace nk {

struct BatchOptions {
    double tol = 1e-6, time_limit = 60;
    int64_t iteration_limit = 100000;
    int check_every = 100;
    PrepareOptions prepare;
    bool adaptive = true, restart = true, graphs = true, autotune = true;
    int precision = NK_PRECISION_FP64;
    double phase_tol = 0;     // MIXED: KKT at which an instance moves to FP64 (0: 10 * tol)
    double memory_budget = 0; // bytes; 0: 80% of the free device memory at creation
    int capacity = 4096;
};

// A prepared instance (host only; built by any thread, admitted by the batch).
struct BatchItem {
    HostModel orig;
    Prepared prep;
    std::unique_ptr<Verifier> verifier;
    SolveReport report; // early outcome (status set) or the running counters
    bool decided = false; // terminal before any iteration (presolve, start point)
    int64_t n = 0, m = 0;
    std::vector<int64_t> cperm, rperm; // engine position -> prepared index
    // SELL-32 of A (rows) and A^T (columns), engine order
    std::vector<int64_t> a_cptr, t_cptr;
    std::vector<int32_t> a_len, t_len, a_idx, t_idx;
    std::vector<double> a_val, t_val;
    std::vector<int64_t> q_ptr;
    std::vector<int32_t> q_idx;
    std::vector<double> q_val;
    std::vector<double> c, q, lb, ub, rl, ru, x0, y0, xp; // xp: x0 in prepared order
    std::vector<double> cs, olb, oub, rs, shift, orl, oru;
    double os = 1, cscale = 1, offset_o = 0, offset_s = 0, cfixed = 0;
    double step = 1, weight = 1, a_norm = 0, q_norm = 0;
    bool sparse_q = false;
    bool is_qp = false; // the caller's model has quadratic terms (cached: O(n) to test)
    size_t bytes = 0;
    int64_t iteration_limit = 100000; // this instance's limits (from its prepare options)
    double time_limit = 60;
    std::vector<int64_t> col_cost, row_cost; // estimated work per SELL chunk (work lists)
};

namespace batch_detail {

// Runs f(0 .. count-1) on up to hardware_concurrency host threads.
template <class F> void parallel_for(size_t count, F &&f) {
    const size_t threads = std::min<size_t>(count, std::max(1u, std::thread::hardware_concurrency()));
    if (threads <= 1) {
        for (size_t k = 0; k < count; ++k)
            f(k);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (size_t t = 0; t < threads; ++t)
        pool.emplace_back([&]() {
            host_serial(true); // the workers are the parallelism: no nested OpenMP teams
            for (size_t k; (k = next.fetch_add(1)) < count;)
                f(k);
        });
    for (auto &th : pool)
        th.join();
}

// SELL-32 of the rows of a CSR (ptr/index/value in prepared order) taken in
// engine order `perm`, column indices mapped through `inv`.
inline void build_sell_host(const Csr &M, const std::vector<int64_t> &perm,
                            const std::vector<int64_t> &inv, std::vector<int64_t> &cptr,
                            std::vector<int32_t> &len, std::vector<int32_t> &idx,
                            std::vector<double> &val) {
    const int64_t rows = M.rows, chunks = (rows + 31) / 32;
    len.assign(size_t(rows), 0);
    for (int64_t r = 0; r < rows; ++r) {
        const int64_t i = perm[size_t(r)];
        len[size_t(r)] = int32_t(M.ptr[size_t(i + 1)] - M.ptr[size_t(i)]);
    }
    cptr.assign(size_t(chunks + 1), 0);
    for (int64_t c = 0; c < chunks; ++c) {
        int32_t w = 0;
        for (int64_t r = c * 32; r < std::min(rows, c * 32 + 32); ++r)
            w = std::max(w, len[size_t(r)]);
        cptr[size_t(c + 1)] = cptr[size_t(c)] + 32 * int64_t(w);
    }
    idx.assign(size_t(cptr.back()), 0);
    val.assign(size_t(cptr.back()), 0.0);
    for (int64_t r = 0; r < rows; ++r) {
        const int64_t i = perm[size_t(r)];
        const int64_t base = cptr[size_t(r >> 5)] + (r & 31);
        int64_t k = 0;
        for (int64_t e = M.ptr[size_t(i)]; e < M.ptr[size_t(i + 1)]; ++e, ++k) {
            idx[size_t(base + 32 * k)] = int32_t(inv[size_t(M.index[size_t(e)])]);
            val[size_t(base + 32 * k)] = M.value[size_t(e)];
        }
    }
}

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

} // namespace batch_detail

// Prepares one instance for a batch: everything solve() does before the first
// iteration, plus the instance's SELL layout.  Thread-safe (no device calls).
// x0 / y0 (optional, the caller's n and m entries): the start point, taken into
// the prepared space as nk_solve takes Options::initial_x / initial_y.
inline std::unique_ptr<BatchItem> batch_prepare(const HostModel &original, const BatchOptions &o,
                                                const std::vector<double> *x0 = nullptr,
                                                const std::vector<double> *y0 = nullptr) {
    using namespace batch_detail;
    auto it = std::make_unique<BatchItem>();
    BatchItem &B = *it;
    B.iteration_limit = o.iteration_limit;
    B.time_limit = o.time_limit;
    auto t0 = SteadyClock::now();
    B.orig = original;
    B.is_qp = B.orig.is_qp();
    B.verifier = std::make_unique<Verifier>(B.orig);
    B.prep = prepare(B.orig, o.prepare);
    SolveReport &R = B.report;
    R.preprocess = since(t0);
    auto finish = [&](int status) {
        R.status = status;
        B.decided = true;
        R.seconds = since(t0);
        return std::move(it);
    };
    if (!B.prep.failure.empty()) {
        R.y = B.prep.failure_ray;
        return finish(B.prep.failure == "INFEASIBLE" ? NK_SOLVE_INFEASIBLE : NK_SOLVE_NUMERICAL_ERROR);
    }
    const HostModel &pm = B.prep.model;
    B.n = int64_t(pm.c.size());
    B.m = int64_t(pm.rl.size());
    if (B.n >= INT32_MAX / 2 || B.m >= INT32_MAX / 2)
        throw Error(NK_ERR_UNSUPPORTED, "batched instances are limited to 2^30 rows and columns");
    R.removed_columns = int64_t(B.orig.c.size()) - B.n;
    R.removed_rows = int64_t(B.orig.rl.size()) - B.m;
    std::vector<double> x(static_cast<size_t>(B.n)), y(static_cast<size_t>(B.m));
    for (int64_t j = 0; j < B.n; j++) {
        const double initial = x0 ? (*x0)[size_t(B.prep.cols[size_t(j)])] : 0.;
        x[size_t(j)] = std::clamp(initial / B.prep.column_scale[size_t(j)], pm.lb[size_t(j)],
                                  pm.ub[size_t(j)]);
    }
    if (y0)
        for (int64_t i = 0; i < B.m; i++)
            y[size_t(i)] = (*y0)[size_t(B.prep.rows[size_t(i)])] /
                           (B.prep.row_scale[size_t(i)] * B.prep.objective_scale);
    R.x = B.prep.restore_x(x);
    R.y = B.prep.restore_y(y, B.orig.rl.size());
    R.accuracy = B.verifier->evaluate(R.x, R.y);
    if (R.accuracy.finite && R.accuracy.primal_absolute == 0) { // src/solver.cpp:268-287
        std::vector<bool> used(size_t(B.n), false);
        for (auto j : pm.A.index)
            used[size_t(j)] = true;
        for (int64_t i = 0; i < pm.Q.rows; ++i)
            for (auto k = pm.Q.ptr[size_t(i)]; k < pm.Q.ptr[size_t(i + 1)]; ++k) {
                used[size_t(i)] = true;
                used[size_t(pm.Q.index[size_t(k)])] = true;
            }
        for (int64_t j = 0; j < B.n; j++)
            if (!used[size_t(j)] && pm.q[size_t(j)] == 0 &&
                ((pm.c[size_t(j)] < 0 && pm.ub[size_t(j)] == kInf) ||
                 (pm.c[size_t(j)] > 0 && pm.lb[size_t(j)] == -kInf)))
                return finish(NK_SOLVE_UNBOUNDED);
    }
    if (R.accuracy.finite && R.accuracy.kkt <= o.tol)
        return finish(NK_SOLVE_OPTIMAL);
    if (o.time_limit == 0)
        return finish(NK_SOLVE_TIME_LIMIT);
    initial_steps(pm, o.adaptive, B.step, B.weight);
    // engine order: rows and columns by length, longest first (stable)
    Csr at = transpose(pm.A);
    std::vector<int64_t> rlen(size_t(B.m)), clen(size_t(B.n));
    for (int64_t i = 0; i < B.m; ++i)
        rlen[size_t(i)] = pm.A.ptr[size_t(i + 1)] - pm.A.ptr[size_t(i)];
    for (int64_t j = 0; j < B.n; ++j)
        clen[size_t(j)] = at.ptr[size_t(j + 1)] - at.ptr[size_t(j)];
    B.rperm = order_by_length_desc(rlen);
    B.cperm = order_by_length_desc(clen);
    std::vector<int64_t> rinv(size_t(B.m)), cinv(size_t(B.n));
    for (int64_t i = 0; i < B.m; ++i)
        rinv[size_t(B.rperm[size_t(i)])] = i;
    for (int64_t j = 0; j < B.n; ++j)
        cinv[size_t(B.cperm[size_t(j)])] = j;
    build_sell_host(pm.A, B.rperm, cinv, B.a_cptr, B.a_len, B.a_idx, B.a_val);
    build_sell_host(at, B.cperm, rinv, B.t_cptr, B.t_len, B.t_idx, B.t_val);
    B.sparse_q = !pm.Q.value.empty();
    if (B.sparse_q) {
        B.q_ptr.assign(size_t(B.n + 1), 0);
        for (int64_t j = 0; j < B.n; ++j) {
            const int64_t r = B.cperm[size_t(j)];
            B.q_ptr[size_t(j + 1)] = B.q_ptr[size_t(j)] + pm.Q.ptr[size_t(r + 1)] - pm.Q.ptr[size_t(r)];
            for (auto k = pm.Q.ptr[size_t(r)]; k < pm.Q.ptr[size_t(r + 1)]; ++k) {
                B.q_idx.push_back(int32_t(cinv[size_t(pm.Q.index[size_t(k)])]));
                B.q_val.push_back(pm.Q.value[size_t(k)]);
            }
        }
        // QP step safety norms (src/cpu.cpp:25-42, src/model.cpp:257-267)
        std::vector<double> cols(size_t(B.n), 0.0);
        double rowmax = 0;
        for (int64_t i = 0; i < B.m; ++i) {
            double sum = 0;
            for (auto k = pm.A.ptr[size_t(i)]; k < pm.A.ptr[size_t(i + 1)]; ++k) {
                sum += std::abs(pm.A.value[size_t(k)]);
                cols[size_t(pm.A.index[size_t(k)])] += std::abs(pm.A.value[size_t(k)]);
            }
            rowmax = std::max(rowmax, sum);
        }
        double colmax = 0;
        for (double v : cols)
            colmax = std::max(colmax, v);
        B.a_norm = std::sqrt(rowmax) * std::sqrt(colmax);
        long double largest = 0;
        for (int64_t i = 0; i < B.n; ++i) {
            long double sum = std::abs(pm.q[size_t(i)]);
            for (auto k = pm.Q.ptr[size_t(i)]; k < pm.Q.ptr[size_t(i + 1)]; ++k)
                sum += std::abs(pm.Q.value[size_t(k)]);
            largest = std::max(largest, sum);
        }
        B.q_norm = std::nextafter(double(largest), INFINITY);
    }
    // estimated work per chunk for the work lists: the chunk's SELL width plus
    // its Q work (rows longer than 32 are shared by the warp, 32 entries a step)
    for (int64_t c = 0; c < (B.n + 31) / 32; ++c) {
        int64_t cost = (B.t_cptr[size_t(c + 1)] - B.t_cptr[size_t(c)]) / 32 + 4;
        if (B.sparse_q) {
            int64_t lane_max = 0, shared = 0;
            for (int64_t j = c * 32; j < std::min<int64_t>(B.n, c * 32 + 32); ++j) {
                const int64_t len = B.q_ptr[size_t(j + 1)] - B.q_ptr[size_t(j)];
                if (len > 32)
                    shared += (len + 31) / 32;
                else
                    lane_max = std::max(lane_max, len);
            }
            cost += lane_max + shared;
        }
        B.col_cost.push_back(cost);
    }
    for (int64_t c = 0; c < (B.m + 31) / 32; ++c)
        B.row_cost.push_back((B.a_cptr[size_t(c + 1)] - B.a_cptr[size_t(c)]) / 32 + 4);
    auto by_col = [&](const std::vector<double> &v) {
        std::vector<double> out(size_t(B.n));
        for (int64_t j = 0; j < B.n; ++j)
            out[size_t(j)] = v[size_t(B.cperm[size_t(j)])];
        return out;
    };
    auto by_row = [&](const std::vector<double> &v) {
        std::vector<double> out(size_t(B.m));
        for (int64_t i = 0; i < B.m; ++i)
            out[size_t(i)] = v[size_t(B.rperm[size_t(i)])];
        return out;
    };
    B.c = by_col(pm.c);
    B.q = by_col(pm.q);
    B.lb = by_col(pm.lb);
    B.ub = by_col(pm.ub);
    B.rl = by_row(pm.rl);
    B.ru = by_row(pm.ru);
    B.x0 = by_col(x);
    B.y0 = by_row(y);
    B.xp = x;
    // original-space evaluation constants (nk_solve.cuh, DeviceSolve::build)
    B.os = B.prep.objective_scale;
    B.offset_o = B.orig.offset;
    B.offset_s = pm.offset;
    B.cscale = 1;
    for (double v : B.orig.c)
        B.cscale = std::max(B.cscale, 1 + std::abs(v));
    std::vector<char> kept(B.orig.c.size(), 0);
    for (auto j : B.prep.cols)
        kept[size_t(j)] = 1;
    long double fixed_terms = 0;
    for (size_t j = 0; j < B.orig.c.size(); ++j)
        if (!kept[j]) {
            long double v = B.prep.fixed[j];
            fixed_terms += B.orig.c[j] * v + .5L * B.orig.q[j] * v * v;
        }
    B.cfixed = double(fixed_terms);
    B.cs.resize(size_t(B.n));
    B.olb.resize(size_t(B.n));
    B.oub.resize(size_t(B.n));
    for (int64_t j = 0; j < B.n; ++j) {
        const int64_t p = B.cperm[size_t(j)];
        B.cs[size_t(j)] = B.prep.column_scale[size_t(p)];
        B.olb[size_t(j)] = B.orig.lb[size_t(B.prep.cols[size_t(p)])];
        B.oub[size_t(j)] = B.orig.ub[size_t(B.prep.cols[size_t(p)])];
    }
    B.rs.resize(size_t(B.m));
    B.shift.resize(size_t(B.m));
    B.orl.resize(size_t(B.m));
    B.oru.resize(size_t(B.m));
    for (int64_t r = 0; r < B.m; ++r) {
        const int64_t p = B.rperm[size_t(r)];
        const int64_t i = B.prep.rows[size_t(p)];
        B.rs[size_t(r)] = B.prep.row_scale[size_t(p)];
        B.orl[size_t(r)] = B.orig.rl[size_t(B.prep.lower_rows[size_t(p)])];
        B.oru[size_t(r)] = B.orig.ru[size_t(B.prep.upper_rows[size_t(p)])];
        long double acc = 0;
        for (auto k = B.orig.A.ptr[size_t(i)]; k < B.orig.A.ptr[size_t(i + 1)]; ++k) {
            const auto jj = B.orig.A.index[size_t(k)];
            if (!kept[size_t(jj)])
                acc += (long double)B.orig.A.value[size_t(k)] * B.prep.fixed[size_t(jj)];
        }
        B.shift[size_t(r)] = double(acc);
    }
    // device footprint: matrices (FP64 values, plus FP32 copies in MIXED
    // batches), 20 column and 19 row vectors
    const bool mixed = o.precision == NK_PRECISION_MIXED;
    size_t bytes = 0;
    for (size_t s : {B.a_cptr.size() * 8, B.t_cptr.size() * 8, B.a_len.size() * 4,
                     B.t_len.size() * 4, B.a_idx.size() * 4, B.t_idx.size() * 4,
                     B.a_val.size() * 8, B.t_val.size() * 8, B.q_ptr.size() * 8,
                     B.q_idx.size() * 4, B.q_val.size() * 8})
        bytes += align256(s);
    if (mixed)
        for (size_t s : {B.a_val.size() * 4, B.t_val.size() * 4, B.q_val.size() * 4})
            bytes += align256(s);
    bytes += 20 * align256(size_t(B.n) * 8) + 19 * align256(size_t(B.m) * 8);
    B.bytes = bytes + 4096;
    return it;
}

// Device footprint of an instance before it is prepared (admission control):
// the reference's own estimate, 48 B per nonzero and 240 B per row and column
// (src/solver.cpp:227-228).
inline double batch_estimate(const HostModel &m) {
    return 48. * double(m.A.value.size() + m.Q.value.size()) +
           240. * double(m.A.rows + m.A.cols + 2);
}

class Batch {
  public:
    struct Slot {
        std::unique_ptr<BatchItem> item;
        DevBuf<unsigned char> mem;
        BInst d{};
        int64_t id = -1;
        bool active = false, finished = false;
        int status = NK_SOLVE_ITERATION_LIMIT;
        SteadyClock::time_point start;
        double step = 1, weight = 1, restart_kkt = kInf;
        int64_t iterations = 0, since_restart = 0, next_host_check = 0, restarts = 0,
                weight_updates = 0, rejected = 0, empty = 0, checks = 0, device_checks = 0,
                host_checks = 0;
        double prev_accepted = 0, prev_rejected = 0, iteration_seconds = 0,
               verification_seconds = 0, transfer_seconds = 0;
        Accuracy best, phase_best;
        double reached[9] = {-1, -1, -1, -1, -1, -1, -1, -1, -1};
        bool fp64_phase = true;     // false while a MIXED instance runs on FP32 values
        double stall_ref = kInf;    // best KKT when the reduced phase last improved by 10%
        int64_t stall = 0, phase_iterations = 0;
    };

    explicit Batch(const BatchOptions &o) : o_(o) {
        if (o.capacity <= 0 || o.capacity > (1 << 20))
            throw Error(NK_ERR_INVALID, "batch capacity must be in [1, 2^20]");
        if (o.check_every <= 0 || !(o.tol > 0))
            throw Error(NK_ERR_INVALID, "invalid batch options");
        if (o.precision != NK_PRECISION_FP64 && o.precision != NK_PRECISION_MIXED)
            throw Error(NK_ERR_UNSUPPORTED, "batched matrices are FP64 or MIXED (FP32 values)");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
            throw Error(NK_ERR_NO_DEVICE, "no CUDA device");
        cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
        size_t freeb = 0, total = 0;
        cuda_check(cudaMemGetInfo(&freeb, &total), "cudaMemGetInfo");
        budget_ = o.memory_budget > 0 ? o.memory_budget : .8 * double(freeb);
        slots_.resize(size_t(o.capacity));
        d_ins_.alloc(size_t(o.capacity));
        d_ctl_.alloc(size_t(o.capacity));
        d_mask_.alloc(size_t(o.capacity));
        d_src_.alloc(size_t(o.capacity));
        cuda_check(cudaMemset(d_ctl_.p, 0, sizeof(BCtl) * size_t(o.capacity)), "controls");
        cuda_check(cudaMallocHost(reinterpret_cast<void **>(&h_ctl_), sizeof(BCtl) * size_t(o.capacity)),
                   "pinned");
        std::memset(h_ctl_, 0, sizeof(BCtl) * size_t(o.capacity));
        cuda_check(cudaMallocHost(reinterpret_cast<void **>(&h_mask_), sizeof(int) * size_t(o.capacity) * 2),
                   "pinned");
        h_src_ = h_mask_ + o.capacity;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev);
        const void *kernels[] = {(const void *)batch_primal<2>, (const void *)batch_primal<4>,
                                 (const void *)batch_primal<8>, (const void *)batch_dual<2>,
                                 (const void *)batch_dual<4>, (const void *)batch_dual<8>};
        for (int t = 0; t < kCtaSizes; ++t) {
            int least = 1 << 30;
            for (const void *k : kernels) {
                int per = 1;
                cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kCtaSize[t], 0),
                           "occupancy");
                least = std::min(least, per);
            }
            resident_[t] = std::max(1, least);
        }
    }
    ~Batch() {
        if (stream_)
            cudaStreamSynchronize(stream_);
        if (graph_)
            cudaGraphExecDestroy(graph_);
        if (h_ctl_)
            cudaFreeHost(h_ctl_);
        if (h_mask_)
            cudaFreeHost(h_mask_);
        if (h_out_)
            cudaFreeHost(h_out_);
        if (stream_)
            cudaStreamDestroy(stream_);
    }

    double budget() const { return budget_; }
    double used() const { return used_; }
    int active() const { return int(order_.size()) + int(joining_.size()); }
    int variant_primal() const { return vp_; }
    double tuned_ms_primal() const { return ms_primal_; }
    const double *phase_seconds() const { return phase_; }
    double tuned_ms_dual() const { return ms_dual_; }
    int variant_dual() const { return vd_; }

    // Admits a prepared instance under `id`; returns false (nothing changed)
    // when the instance does not fit the memory budget or the slot table.
    // The item is taken only when admitted.
    bool admit(std::unique_ptr<BatchItem> &item, int64_t id) {
        if (!item)
            throw Error(NK_ERR_INVALID, "null batch item");
        if (by_id_.count(id))
            throw Error(NK_ERR_INVALID, "duplicate batch instance id");
        int free_slot = -1;
        for (int b = 0; b < int(slots_.size()); ++b)
            if (!slots_[size_t(b)].item && slots_[size_t(b)].id < 0) {
                free_slot = b;
                break;
            }
        if (free_slot < 0)
            return false;
        Slot &S = slots_[size_t(free_slot)];
        if (item->decided) { // terminal before the first iteration
            S.item = std::move(item);
            S.id = id;
            S.finished = true;
            S.status = S.item->report.status;
            by_id_[id] = free_slot;
            return true;
        }
        if (used_ + double(item->bytes) > budget_)
            return false;
        auto t0 = SteadyClock::now();
        upload(S, *item);
        S.item = std::move(item);
        S.id = id;
        S.active = true;
        S.finished = false;
        S.status = NK_SOLVE_ITERATION_LIMIT;
        S.start = t0;
        S.step = S.item->step;
        S.weight = S.item->weight;
        S.restart_kkt = S.item->report.accuracy.kkt;
        S.fp64_phase = o_.precision == NK_PRECISION_FP64;
        S.stall_ref = kInf;
        S.stall = 0;
        S.phase_iterations = 0;
        S.transfer_seconds = since(t0);
        used_ += double(S.item->bytes);
        by_id_[id] = free_slot;
        joining_.push_back(free_slot);
        return true;
    }

    // Runs up to `checks` check intervals; returns the ids that finished.
    std::vector<int64_t> step(int checks) {
        std::vector<int64_t> done;
        for (auto &[id, b] : by_id_)
            if (slots_[size_t(b)].finished && !reported_.count(id)) {
                done.push_back(id);
                reported_.insert(id);
            }
        for (int c = 0; c < checks; ++c) {
            auto tl = SteadyClock::now();
            rebuild_lists();
            phase_[6] += since(tl);
            if (order_.empty())
                break;
            run_interval();
            for (int b : order_)
                if (slots_[size_t(b)].finished && !reported_.count(slots_[size_t(b)].id)) {
                    done.push_back(slots_[size_t(b)].id);
                    reported_.insert(slots_[size_t(b)].id);
                }
            if (!done.empty())
                break;
        }
        return done;
    }

    // Progress of an instance: iterations, restarts, best KKT estimate, primal
    // weight, step, iterations since restart, KKT at the last restart, phase.
    void progress(int64_t id, double *out) const {
        auto f = by_id_.find(id);
        if (f == by_id_.end())
            throw Error(NK_ERR_INVALID, "unknown batch instance id");
        const Slot &S = slots_[size_t(f->second)];
        const double v[8] = {double(S.iterations), double(S.restarts), S.best.kkt, S.weight,
                             S.step, double(S.since_restart), S.restart_kkt,
                             S.fp64_phase ? 1. : 0.};
        std::memcpy(out, v, sizeof(v));
    }

    // Result of a finished instance; frees its slot.
    SolveReport take(int64_t id) {
        auto f = by_id_.find(id);
        if (f == by_id_.end())
            throw Error(NK_ERR_INVALID, "unknown batch instance id");
        Slot &S = slots_[size_t(f->second)];
        if (!S.finished)
            throw Error(NK_ERR_INVALID, "batch instance has not finished");
        SolveReport R = std::move(S.item->report);
        if (!S.item->decided) {
            R.status = S.status;
            R.iterations = S.iterations;
            R.restarts = S.restarts;
            R.rejected = S.rejected;
            R.weight_updates = S.weight_updates;
            R.device_checks = S.device_checks;
            R.host_checks = S.host_checks;
            R.iteration = S.iteration_seconds;
            if (o_.precision != NK_PRECISION_FP64) {
                R.mixed_iterations = S.fp64_phase ? S.phase_iterations : S.iterations;
                R.refine_iterations = S.fp64_phase ? S.iterations - S.phase_iterations : 0;
                R.mixed = S.fp64_phase ? S.phase_best : S.best;
            }
            R.verification += S.verification_seconds;
            R.transfer = S.transfer_seconds;
            for (int k = 0; k < 9; ++k)
                R.reached[k] = S.reached[k];
        }
        if (S.mem.p)
            used_ -= double(S.item->bytes);
        S.mem.release();
        S.item.reset();
        S.id = -1;
        S.finished = false;
        S.active = false;
        by_id_.erase(f);
        reported_.erase(id);
        return R;
    }

    // Time `trials` PDHG trials of the whole batch (no driver work), milliseconds.
    double time_trials(int trials) {
        rebuild_lists();
        if (order_.empty())
            return 0;
        push_steps();
        cudaEvent_t e0, e1;
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        cuda_check(cudaEventRecord(e0, stream_), "event");
        for (int t = 0; t < trials; ++t)
            launch_trial(vp_, vd_);
        cuda_check(cudaEventRecord(e1, stream_), "event");
        cuda_check(cudaEventSynchronize(e1), "event");
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        sync_progress(false);
        return double(ms);
    }
    int64_t matrix_bytes_per_trial() const { return trial_bytes_; }
    cudaStream_t stream() const { return stream_; }

  private:
    BatchOptions o_;
    cudaStream_t stream_ = nullptr;
    double budget_ = 0, used_ = 0;
    int sms_ = 148;
    std::vector<Slot> slots_;
    std::map<int64_t, int> by_id_;
    std::set<int64_t> reported_;
    std::vector<int> order_, joining_; // active slots in list order; admitted, not yet listed
    DevBuf<BInst> d_ins_;
    DevBuf<BCtl> d_ctl_;
    DevBuf<int> d_mask_, d_src_, d_slots_, d_cf_, d_cc_, d_rf_, d_rc_;
    DevBuf<int2> d_cols_, d_rows_;     // instance-contiguous (element kernels, partial layout)
    static constexpr int kRunLengths = 3;
    static constexpr int kRunLength[kRunLengths] = {1, 4, 16};
    static constexpr int kCtaSizes = 3;
    static constexpr int kCtaSize[kCtaSizes] = {128, 256, 512};
    // trial items of each (run length, CTA size): per-CTA lists, CTA b's items
    // [coff[b], coff[b+1]) costliest first, over a resident grid of ncta CTAs
    struct WorkList {
        DevBuf<BWork> items;
        DevBuf<int> coff;
        int count = 0, ncta = 0;
    };
    WorkList wcols_[kRunLengths][kCtaSizes], wrows_[kRunLengths][kCtaSizes];
    int resident_[kCtaSizes] = {}; // CTAs of each size one SM holds (every variant)
    DevBuf<double> d_pp_, d_pd_, d_pk_, d_out_;
    BCtl *h_ctl_ = nullptr;
    int *h_mask_ = nullptr, *h_src_ = nullptr;
    double *h_out_ = nullptr;
    size_t h_out_n_ = 0;
    int ncols_ = 0, nrows_ = 0;
    int64_t trial_bytes_ = 0;
    bool dirty_ = true, tuned_ = false;
    int vp_ = 13, vd_ = 13; // kernel variants (autotuned, see launch_half)
    float ms_primal_ = 0, ms_dual_ = 0; // their best times when tuned
    // wall seconds per part of a check interval: control upload, trials,
    // candidate evaluation, per-instance driver logic (host), best/restart
    // kernels, closing certification of finished instances
    double phase_[7] = {}; // ... and work-list rebuilds (with tuning and graph capture)
    int tuned_chunks_ = 0;
    cudaGraphExec_t graph_ = nullptr;

    // ---------------------------------------------------------------- admission
    void upload(Slot &S, const BatchItem &B) {
        using batch_detail::align256;
        const bool f64 = o_.precision == NK_PRECISION_FP64;
        S.mem.alloc(B.bytes);
        cudaMemsetAsync(S.mem.p, 0, B.bytes, stream_);
        unsigned char *p = S.mem.p;
        auto take = [&](size_t bytes) {
            unsigned char *r = p;
            p += align256(bytes);
            return r;
        };
        auto put = [&](const void *src, size_t bytes) {
            unsigned char *dst = take(bytes);
            if (bytes)
                cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), "upload");
            return dst;
        };
        auto put32 = [&](const std::vector<double> &v) -> const float * {
            if (f64)
                return nullptr;
            std::vector<float> f(v.begin(), v.end());
            const void *r = put(f.data(), f.size() * 4);
            cuda_check(cudaStreamSynchronize(stream_), "upload");
            return static_cast<const float *>(r);
        };
        auto put64 = [&](const std::vector<double> &v) {
            return reinterpret_cast<const double *>(put(v.data(), v.size() * 8));
        };
        BInst &d = S.d;
        d = BInst{};
        d.n = int32_t(B.n);
        d.m = int32_t(B.m);
        d.a_cptr = reinterpret_cast<const int64_t *>(put(B.a_cptr.data(), B.a_cptr.size() * 8));
        d.t_cptr = reinterpret_cast<const int64_t *>(put(B.t_cptr.data(), B.t_cptr.size() * 8));
        d.a_len = reinterpret_cast<const int32_t *>(put(B.a_len.data(), B.a_len.size() * 4));
        d.t_len = reinterpret_cast<const int32_t *>(put(B.t_len.data(), B.t_len.size() * 4));
        d.a_idx = reinterpret_cast<const int32_t *>(put(B.a_idx.data(), B.a_idx.size() * 4));
        d.t_idx = reinterpret_cast<const int32_t *>(put(B.t_idx.data(), B.t_idx.size() * 4));
        d.a_val64 = put64(B.a_val);
        d.t_val64 = put64(B.t_val);
        d.a_val = put32(B.a_val);
        d.t_val = put32(B.t_val);
        if (B.sparse_q) {
            d.q_ptr = reinterpret_cast<const int64_t *>(put(B.q_ptr.data(), B.q_ptr.size() * 8));
            d.q_idx = reinterpret_cast<const int32_t *>(put(B.q_idx.data(), B.q_idx.size() * 4));
            d.q_val64 = put64(B.q_val);
            d.q_val = put32(B.q_val);
        }
        auto cvec = [&](const std::vector<double> &v) {
            return reinterpret_cast<double *>(put(v.data(), v.size() * 8));
        };
        auto zn = [&]() { return reinterpret_cast<double *>(take(size_t(B.n) * 8)); };
        auto zm = [&]() { return reinterpret_cast<double *>(take(size_t(B.m) * 8)); };
        // 20 column vectors
        d.c = cvec(B.c);
        d.q = cvec(B.q);
        if (std::all_of(B.q.begin(), B.q.end(), [](double v) { return v == 0; }))
            d.q = nullptr; // an LP: the kernels skip the diagonal's loads
        d.lb = cvec(B.lb);
        d.ub = cvec(B.ub);
        d.x[0] = cvec(B.x0);
        d.x[1] = cvec(B.x0);
        d.xa = zn();
        d.dx = zn();
        d.cs = cvec(B.cs);
        d.olb = cvec(B.olb);
        d.oub = cvec(B.oub);
        d.e_aty[0] = zn();
        d.e_aty[1] = zn();
        d.e_qx = zn();
        d.best_x = cvec(B.x0);
        d.epoch_x = cvec(B.x0);
        zn(); zn(); zn(); zn(); // spare (alignment headroom of the estimate)
        // 19 row vectors
        d.rl = cvec(B.rl);
        d.ru = cvec(B.ru);
        d.y[0] = cvec(B.y0);
        d.y[1] = cvec(B.y0);
        d.ax[0] = zm();
        d.ax[1] = zm();
        d.ya = zm();
        d.rs = cvec(B.rs);
        d.shift = cvec(B.shift);
        d.orl = cvec(B.orl);
        d.oru = cvec(B.oru);
        d.e_ax = zm();
        d.best_y = cvec(B.y0);
        d.epoch_y = cvec(B.y0);
        zm(); zm(); zm(); zm(); zm();
        d.os = B.os;
        d.cscale = B.cscale;
        if (size_t(p - S.mem.p) > B.bytes)
            throw Error(NK_ERR_MEMORY, "batch instance layout exceeds its estimate");
        cuda_check(cudaStreamSynchronize(stream_), "instance upload");
        const int b = int(&S - slots_.data());
        cuda_check(cudaMemcpy(d_ins_.p + b, &d, sizeof(BInst), cudaMemcpyHostToDevice), "descriptor");
        // initial activity A x0 and control
        BCtl c{};
        c.factor = 1;
        c.adaptive = (o_.adaptive && !B.sparse_q) ? 1 : 0;
        c.active = 1;
        c.fp64 = f64 ? 1 : 0;
        h_ctl_[b] = c;
        cuda_check(cudaMemcpy(d_ctl_.p + b, &c, sizeof(BCtl), cudaMemcpyHostToDevice), "control");
        // initial activity A x0 with the values the trials use, each row summed
        // in CSR order (the device SpMV's order)
        std::vector<double> ax0(static_cast<size_t>(B.m), 0.0);
        const Csr &A = B.prep.model.A;
        for (int64_t r = 0; r < B.m; ++r) {
            const int64_t i = B.rperm[size_t(r)];
            double sum = 0;
            for (auto k = A.ptr[size_t(i)]; k < A.ptr[size_t(i + 1)]; ++k) {
                const double a = f64 ? A.value[size_t(k)] : double(float(A.value[size_t(k)]));
                sum += a * B.xp[size_t(A.index[size_t(k)])];
            }
            ax0[size_t(r)] = sum;
        }
        if (B.m) {
            cuda_check(cudaMemcpy(d.ax[0], ax0.data(), size_t(B.m) * 8, cudaMemcpyHostToDevice), "activity");
            cuda_check(cudaMemcpy(d.ax[1], ax0.data(), size_t(B.m) * 8, cudaMemcpyHostToDevice), "activity");
        }
    }

    // ---------------------------------------------------------------- lists
    // Device buffers of the work lists only grow: a shrinking batch reuses them.
    template <class T> static void ensure(DevBuf<T> &d, size_t count) {
        if (d.n < count)
            d.alloc(count + count / 4);
    }

    void rebuild_lists() {
        if (!joining_.empty()) {
            for (int b : joining_)
                order_.push_back(b);
            joining_.clear();
            dirty_ = true;
        }
        std::vector<int> keep;
        for (int b : order_)
            if (slots_[size_t(b)].active)
                keep.push_back(b);
            else
                dirty_ = true;
        order_.swap(keep);
        if (!dirty_)
            return;
        std::vector<int2> cols, rows;
        std::vector<int> cf, cc, rf, rc;
        std::vector<int64_t> ccost, rcost; // per chunk, in list order
        trial_bytes_ = 0;
        const int64_t vb = o_.precision == NK_PRECISION_FP64 ? 8 : 4;
        for (int b : order_) {
            const BatchItem &B = *slots_[size_t(b)].item;
            cf.push_back(int(cols.size()));
            for (int64_t c = 0; c < (B.n + 31) / 32; ++c) {
                ccost.push_back(B.col_cost[size_t(c)]);
                cols.push_back(make_int2(b, int(c)));
            }
            cc.push_back(int(cols.size()) - cf.back());
            rf.push_back(int(rows.size()));
            for (int64_t c = 0; c < (B.m + 31) / 32; ++c) {
                rcost.push_back(B.row_cost[size_t(c)]);
                rows.push_back(make_int2(b, int(c)));
            }
            rc.push_back(int(rows.size()) - rf.back());
            const int64_t nnz = int64_t(B.prep.model.A.value.size());
            trial_bytes_ += 2 * (nnz * (vb + 4) + 4 * (B.m + B.n)) + 8 * (B.m + B.n);
        }
        // trial work lists for each run length K: runs of K consecutive chunks
        // of one instance, in instance and chunk order, with their estimated
        // costs
        auto runs = [&](const std::vector<int2> &list, const std::vector<int64_t> &cost,
                        const std::vector<int> &first, const std::vector<int> &count, int K,
                        std::vector<int64_t> &icost) {
            std::vector<BWork> items;
            icost.clear();
            for (size_t k = 0; k < first.size(); ++k)
                for (int c = 0; c < count[k]; c += K) {
                    const int len = std::min(K, count[k] - c);
                    int64_t total = 0;
                    for (int t = 0; t < len; ++t)
                        total += cost[size_t(first[k] + c + t)];
                    const int2 head = list[size_t(first[k] + c)];
                    items.push_back(BWork{head.x, head.y, first[k] + c, len});
                    icost.push_back(total);
                }
            return items;
        };
        // Items onto a resident grid of CTAs of size t.  With many instances
        // (kSegmentInstances or more) the items, in instance and chunk order,
        // are cut into kSegments * G consecutive segments of equal estimated
        // work, and segment s goes to CTA s mod G.  A CTA's warps then work on
        // a few runs of one instance's consecutive chunks at a time, gathering
        // from the same x or dx lines in L1, while each CTA's share mixes
        // instances from across the batch, so that errors of the cost
        // estimate even out.  On the 512-instance batch an FP64 trial took
        // 0.846 ms so, against 1.007 ms with all items sorted by cost and
        // dealt one per CTA in turn, 0.909 ms with one segment per CTA for the
        // rows (columns dealt), and 0.871 ms with two per CTA for both.  With
        // few instances a CTA's segments come from one or two instances and
        // the estimate's errors no longer even out (the served stream, about
        // 45 active instances: 115 requests completed against 135 dealt), and
        // the items are sorted by cost, costliest first (a stable counting
        // sort), and dealt one per CTA per round, alternating direction (round
        // k to CTAs 0..G-1 when k is even, G-1..0 when odd).
        constexpr int kSegments = 4, kSegmentInstances = 64;
        const bool segmented = int(order_.size()) >= kSegmentInstances;
        auto place = [&](WorkList &W, const std::vector<BWork> &items,
                         const std::vector<int64_t> &icost, int t) {
            const int ncta = std::max(1, std::min<int>(int(items.size()), sms_ * resident_[t]));
            std::vector<int> owner(items.size());
            std::vector<int> coff(size_t(ncta + 1), 0);
            std::vector<size_t> seq(items.size()); // the order the lists are filled in
            std::iota(seq.begin(), seq.end(), size_t(0));
            if (segmented) {
                double total = 0;
                for (int64_t c : icost)
                    total += double(c);
                const int nseg = kSegments * ncta;
                const double share = std::max(1e-9, total / nseg);
                double before = 0;
                for (size_t k = 0; k < items.size(); ++k) {
                    const int seg =
                        std::min(nseg - 1, int((before + 0.5 * double(icost[k])) / share));
                    owner[k] = seg % ncta;
                    before += double(icost[k]);
                    ++coff[size_t(owner[k] + 1)];
                }
            } else {
                int64_t top = 0;
                for (int64_t c : icost)
                    top = std::max(top, c);
                std::vector<int64_t> start(size_t(top + 2), 0);
                for (int64_t c : icost)
                    ++start[size_t(top - c + 1)];
                for (size_t b = 1; b < start.size(); ++b)
                    start[b] += start[b - 1];
                for (size_t k = 0; k < items.size(); ++k)
                    seq[size_t(start[size_t(top - icost[k])]++)] = k;
                for (size_t r = 0; r < seq.size(); ++r) {
                    const int round = int(r / size_t(ncta)), at = int(r % size_t(ncta));
                    owner[seq[r]] = round % 2 ? ncta - 1 - at : at;
                    ++coff[size_t(owner[seq[r]] + 1)];
                }
            }
            for (int b = 0; b < ncta; ++b)
                coff[size_t(b + 1)] += coff[size_t(b)];
            // each CTA's list: in instance and chunk order (segments) or
            // costliest first (dealt)
            std::vector<BWork> out(std::max<size_t>(1, items.size()));
            std::vector<int> fill(coff.begin(), coff.end() - 1);
            for (size_t k : seq)
                out[size_t(fill[size_t(owner[k])]++)] = items[k];
            ensure(W.items, out.size());
            ensure(W.coff, coff.size());
            cuda_check(cudaMemcpy(W.items.p, out.data(), out.size() * sizeof(BWork),
                                  cudaMemcpyHostToDevice), "lists");
            cuda_check(cudaMemcpy(W.coff.p, coff.data(), coff.size() * sizeof(int),
                                  cudaMemcpyHostToDevice), "lists");
            W.count = int(items.size());
            W.ncta = ncta;
        };
        for (int r = 0; r < kRunLengths; ++r) {
            // after tuning only the chosen variants' lists are launched
            std::vector<int64_t> icost;
            if (!tuned_ || r == vp_ / 9) {
                auto wc = runs(cols, ccost, cf, cc, kRunLength[r], icost);
                for (int t = 0; t < kCtaSizes; ++t)
                    if (!tuned_ || t == vp_ % 3)
                        place(wcols_[r][t], wc, icost, t);
            }
            if (!tuned_ || r == vd_ / 9) {
                auto wr = runs(rows, rcost, rf, rc, kRunLength[r], icost);
                for (int t = 0; t < kCtaSizes; ++t)
                    if (!tuned_ || t == vd_ % 3)
                        place(wrows_[r][t], wr, icost, t);
            }
        }
        ncols_ = int(cols.size());
        nrows_ = int(rows.size());
        auto up = [&](auto &d, const auto &h) {
            ensure(d, std::max<size_t>(1, h.size()));
            if (!h.empty())
                cuda_check(cudaMemcpy(d.p, h.data(), h.size() * sizeof(h[0]), cudaMemcpyHostToDevice),
                           "lists");
        };
        up(d_cols_, cols);
        up(d_rows_, rows);
        up(d_slots_, order_);
        up(d_cf_, cf);
        up(d_cc_, cc);
        up(d_rf_, rf);
        up(d_rc_, rc);
        ensure(d_pp_, size_t(std::max(1, ncols_)));
        ensure(d_pd_, size_t(std::max(1, 2 * nrows_)));
        ensure(d_pk_, size_t(std::max(1, ncols_ + nrows_)) * kBatchKkt);
        ensure(d_out_, size_t(std::max<size_t>(1, order_.size())) * kBatchKkt * 2);
        const size_t need = std::max<size_t>(1, order_.size()) * kBatchKkt * 2;
        if (h_out_n_ < need) {
            if (h_out_)
                cudaFreeHost(h_out_);
            cuda_check(cudaMallocHost(reinterpret_cast<void **>(&h_out_), need * 8), "pinned");
            h_out_n_ = need;
        }
        if (graph_) {
            cudaGraphExecDestroy(graph_);
            graph_ = nullptr;
        }
        dirty_ = false;
        // tuned once, on the first work list: later tuning would insert trials
        // into running instances' check intervals and change their trajectories
        if (o_.autotune && !tuned_)
            autotune();
    }

    // ---------------------------------------------------------------- launches
    // kernel variant v (autotuned): run length {1, 4, 16}[v / 9], unroll
    // {2, 4, 8}[v / 3 % 3], CTA size {128, 256, 512}[v % 3]
    static constexpr int kVariants = 27;
    void launch_half(int v, bool primal, bool probe = false) {
        const int t = v % 3, u = v / 3 % 3, r = v / 9;
        const WorkList &W = primal ? wcols_[r][t] : wrows_[r][t];
        if (W.count == 0)
            return;
        if (primal) {
            auto *k = u == 0 ? batch_primal<2> : u == 1 ? batch_primal<4> : batch_primal<8>;
            k<<<W.ncta, kCtaSize[t], 0, stream_>>>(d_ins_.p, d_ctl_.p, W.items.p, W.coff.p,
                                                   d_pp_.p, int(probe));
        } else {
            auto *k = u == 0 ? batch_dual<2> : u == 1 ? batch_dual<4> : batch_dual<8>;
            k<<<W.ncta, kCtaSize[t], 0, stream_>>>(d_ins_.p, d_ctl_.p, W.items.p, W.coff.p,
                                                   d_pd_.p, int(probe));
        }
    }
    void launch_decide() {
        const int n = int(order_.size());
        batch_decide<<<std::max(1, (n + 7) / 8), 256, 0, stream_>>>(
            d_ctl_.p, d_slots_.p, n, d_cf_.p, d_cc_.p, d_rf_.p, d_rc_.p, d_pp_.p, d_pd_.p);
    }
    // One trial: an instance without columns (rows) contributes no partials,
    // and its decision reads none.
    void launch_trial(int vp, int vd) {
        launch_half(vp, true);
        launch_half(vd, false);
        launch_decide();
        cuda_check(cudaGetLastError(), "batch trial");
    }

    // Autotuner: times every kernel variant on the batch as it stands and
    // keeps the fastest primal and dual variants (every variant computes the
    // same sums in the same order).  The timed launches are probe trials: they
    // do a trial's work on the current iterates but apply no pending average
    // and make no decision, so the instances' iterates, averages and step
    // state come out of tuning untouched and every trajectory is the one it
    // would have been without it.
    void autotune() {
        push_steps();
        cudaEvent_t e0, e1;
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        // a timed dual launch follows a probe primal launch (it reads that dx)
        auto time_half = [&](int v, bool primal) {
            float best = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                if (!primal)
                    launch_half(vp_, true, true);
                cuda_check(cudaEventRecord(e0, stream_), "event");
                launch_half(v, primal, true);
                cuda_check(cudaEventRecord(e1, stream_), "event");
                cuda_check(cudaEventSynchronize(e1), "event");
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                best = std::min(best, ms);
            }
            return best;
        };
        const int vp0 = vp_, vd0 = vd_;
        float bp = 1e30f, bd = 1e30f;
        int bvp = vp0, bvd = vd0;
        for (int v = 0; v < kVariants; ++v) {
            const float tp = time_half(v, true);
            if (tp < bp) {
                bp = tp;
                bvp = v;
            }
            const float td = time_half(v, false);
            if (td < bd) {
                bd = td;
                bvd = v;
            }
        }
        vp_ = bvp;
        vd_ = bvd;
        ms_primal_ = bp;
        ms_dual_ = bd;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cuda_check(cudaGetLastError(), "autotune");
        sync_progress(false);
        tuned_ = true;
        tuned_chunks_ = ncols_ + nrows_;
    }

    cudaGraphExec_t graph() {
        if (!graph_) {
            cudaGraph_t g = nullptr;
            cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
            try {
                for (int t = 0; t < o_.check_every; ++t)
                    launch_trial(vp_, vd_);
            } catch (...) {
                cudaStreamEndCapture(stream_, &g);
                if (g)
                    cudaGraphDestroy(g);
                throw;
            }
            cuda_check(cudaStreamEndCapture(stream_, &g), "capture end");
            cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
            cudaGraphDestroy(g);
            cuda_check(e, "graph instantiate");
        }
        return graph_;
    }

    // Per-instance steps for the next interval (QP step safety as in
    // Engine::advance, src/cpu.cpp:97-102).
    void push_steps() {
        cuda_check(cudaMemcpyAsync(h_ctl_, d_ctl_.p, sizeof(BCtl) * slots_.size(),
                                   cudaMemcpyDeviceToHost, stream_), "controls");
        cuda_check(cudaStreamSynchronize(stream_), "controls");
        for (int b : order_) {
            Slot &S = slots_[size_t(b)];
            double tau = S.step / S.weight, sigma = S.step * S.weight;
            if (S.item->sparse_q) {
                double safety = std::sqrt(tau * sigma) * S.item->a_norm + tau * S.item->q_norm;
                double scale = safety > 0 ? std::min(1., .9 / safety) : 1.;
                tau *= scale;
                sigma *= scale;
            }
            h_ctl_[b].tau = tau;
            h_ctl_[b].sigma = sigma;
        }
        cuda_check(cudaMemcpyAsync(d_ctl_.p, h_ctl_, sizeof(BCtl) * slots_.size(),
                                   cudaMemcpyHostToDevice, stream_), "controls");
    }
    // Reads the controls back and books each instance's accepted progress.
    void sync_progress(bool count) {
        cuda_check(cudaMemcpyAsync(h_ctl_, d_ctl_.p, sizeof(BCtl) * slots_.size(),
                                   cudaMemcpyDeviceToHost, stream_), "controls");
        cuda_check(cudaStreamSynchronize(stream_), "controls");
        for (int b : order_) {
            Slot &S = slots_[size_t(b)];
            const int64_t progress = int64_t(h_ctl_[b].accepted - S.prev_accepted);
            S.prev_accepted = h_ctl_[b].accepted;
            S.rejected += int64_t(h_ctl_[b].rejected - S.prev_rejected);
            S.prev_rejected = h_ctl_[b].rejected;
            S.iterations += progress;
            S.since_restart += progress;
            if (count)
                S.empty = progress ? 0 : S.empty + 1;
        }
    }

    Accuracy finish_accuracy(const BatchItem &B, const double *v) const {
        Accuracy a;
        if (v[9] != 0)
            return a;
        a.primal = v[0];
        a.primal_absolute = v[1];
        a.dual = v[2];
        a.dual_absolute = v[3];
        a.objective = B.os * (B.offset_s + v[4]);
        a.complementarity = v[5];
        a.gap = a.complementarity / (1 + std::abs(a.objective - B.offset_o));
        if (v[8] == 0) {
            const double support = v[6], box = v[7] + B.cfixed;
            long double lower = (long double)B.offset_o - support + box;
            long double guard = 64 * std::numeric_limits<double>::epsilon() *
                                (1 + std::abs((long double)B.offset_o) +
                                 std::abs((long double)support) + std::abs((long double)box));
            a.lower_bound = double(lower - guard);
            a.gap = std::max(a.gap, std::abs(a.objective - a.lower_bound) /
                                        (1 + std::abs(a.objective) + std::abs(a.lower_bound)));
        }
        if (!B.is_qp)
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

    // Uploads a per-instance mask and source table.  The pinned host copy is
    // reused, so wait until the stream has consumed the previous upload.
    void set_mask(const std::vector<int> &on, const std::vector<int> &src,
                  const std::vector<int> &value = {}) {
        cuda_check(cudaStreamSynchronize(stream_), "mask");
        std::fill(h_mask_, h_mask_ + slots_.size(), 0);
        for (size_t k = 0; k < on.size(); ++k) {
            h_mask_[on[k]] = value.empty() ? 1 : value[k];
            h_src_[on[k]] = src.empty() ? 0 : src[k];
        }
        cuda_check(cudaMemcpyAsync(d_mask_.p, h_mask_, sizeof(int) * slots_.size(),
                                   cudaMemcpyHostToDevice, stream_), "mask");
        cuda_check(cudaMemcpyAsync(d_src_.p, h_src_, sizeof(int) * slots_.size(),
                                   cudaMemcpyHostToDevice, stream_), "mask");
    }
    int grid_items(int items) const {
        return std::max(1, std::min((items + 7) / 8, sms_ * 8));
    }
    void evaluate(int src, int slot) {
        batch_products<<<grid_items(ncols_ + nrows_), 256, 0, stream_>>>(
            d_ins_.p, d_ctl_.p, d_mask_.p, src, slot, d_cols_.p, ncols_, d_rows_.p, nrows_);
        batch_kkt<<<grid_items(ncols_ + nrows_), 256, 0, stream_>>>(
            d_ins_.p, d_ctl_.p, d_mask_.p, src, slot, d_cols_.p, ncols_, d_rows_.p, nrows_, d_pk_.p);
        const int n = int(order_.size());
        batch_finish<kBatchKkt><<<std::max(1, (n + 7) / 8), 256, 0, stream_>>>(
            d_cf_.p, d_cc_.p, ncols_, d_rf_.p, d_rc_.p, n, kBatchKktMax, d_pk_.p,
            d_out_.p + size_t(slot) * size_t(n) * kBatchKkt);
        cuda_check(cudaGetLastError(), "batch evaluation");
    }

    // Host copies (caller order, original units) of an instance's device point.
    void host_point(Slot &S, const double *dx, const double *dy, std::vector<double> &ox,
                    std::vector<double> &oy) {
        const BatchItem &B = *S.item;
        std::vector<double> ex(static_cast<size_t>(B.n)), ey(static_cast<size_t>(B.m));
        if (B.n)
            cuda_check(cudaMemcpyAsync(ex.data(), dx, size_t(B.n) * 8, cudaMemcpyDeviceToHost, stream_), "point");
        if (B.m)
            cuda_check(cudaMemcpyAsync(ey.data(), dy, size_t(B.m) * 8, cudaMemcpyDeviceToHost, stream_), "point");
        cuda_check(cudaStreamSynchronize(stream_), "point");
        std::vector<double> px(static_cast<size_t>(B.n)), py(static_cast<size_t>(B.m));
        for (int64_t j = 0; j < B.n; ++j)
            px[size_t(B.cperm[size_t(j)])] = ex[size_t(j)];
        for (int64_t i = 0; i < B.m; ++i)
            py[size_t(B.rperm[size_t(i)])] = ey[size_t(i)];
        ox = B.prep.restore_x(px);
        oy = B.prep.restore_y(py, B.orig.rl.size());
    }
    const double *point_x(Slot &S, int src) {
        const int cur = h_ctl_[&S - slots_.data()].cur;
        return src == kCur ? S.d.x[cur] : src == kAvg ? S.d.xa : S.d.best_x;
    }
    const double *point_y(Slot &S, int src) {
        const int cur = h_ctl_[&S - slots_.data()].cur;
        return src == kCur ? S.d.y[cur] : src == kAvg ? S.d.ya : S.d.best_y;
    }

    void retire(Slot &S, int status) {
        S.status = status;
        S.active = false;
        S.finished = true;
        const size_t b = size_t(&S - slots_.data());
        h_ctl_[b].active = 0;
        cuda_check(cudaMemcpyAsync(&d_ctl_.p[b].active, &h_ctl_[b].active, sizeof(int),
                                   cudaMemcpyHostToDevice, stream_), "retire");
        dirty_ = true;
    }

    // The closing evaluation of solve_continuous for every instance that
    // finished without a certificate: host copies of the best points, then the
    // verifier on host threads.
    void close_finished() {
        std::vector<int> todo;
        for (int b : order_) {
            const Slot &S = slots_[size_t(b)];
            const SolveReport &R = S.item->report;
            if (S.finished && S.status != NK_SOLVE_OPTIMAL && S.status != NK_SOLVE_INFEASIBLE &&
                S.best.finite && S.best.kkt < R.accuracy.kkt)
                todo.push_back(b);
        }
        if (todo.empty())
            return;
        const size_t nc = todo.size();
        std::vector<std::vector<double>> ox(nc), oy(nc);
        std::vector<Accuracy> acc(nc);
        for (size_t k = 0; k < nc; ++k) {
            Slot &S = slots_[size_t(todo[k])];
            host_point(S, S.d.best_x, S.d.best_y, ox[k], oy[k]);
        }
        batch_detail::parallel_for(nc, [&](size_t k) {
            acc[k] = slots_[size_t(todo[k])].item->verifier->evaluate(ox[k], oy[k], true);
        });
        for (size_t k = 0; k < nc; ++k) {
            Slot &S = slots_[size_t(todo[k])];
            SolveReport &R = S.item->report;
            S.host_checks++;
            if (acc[k].finite && (acc[k].kkt < R.accuracy.kkt || !R.accuracy.finite)) {
                R.x = std::move(ox[k]);
                R.y = std::move(oy[k]);
                R.accuracy = acc[k];
            }
        }
    }

    // One check interval for every listed instance.
    void run_interval() {
        auto tp = SteadyClock::now();
        push_steps();
        phase_[0] += since(tp);
        auto t0 = SteadyClock::now();
        if (o_.graphs)
            cuda_check(cudaGraphLaunch(graph(), stream_), "graph launch");
        else
            for (int t = 0; t < o_.check_every; ++t)
                launch_trial(vp_, vd_);
        sync_progress(true);
        const double dt = since(t0);
        phase_[1] += dt;
        auto t1 = SteadyClock::now();
        const int n = int(order_.size());
        // fold pending averages, then evaluate current (slot 0) and average (slot 1)
        batch_flush<<<grid_items(ncols_ + nrows_), 256, 0, stream_>>>(d_ins_.p, d_ctl_.p, d_cols_.p,
                                                                     ncols_, d_rows_.p, nrows_);
        batch_clear_pending<<<std::max(1, (n + 255) / 256), 256, 0, stream_>>>(d_ctl_.p, d_slots_.p, n);
        std::vector<int> all(order_.begin(), order_.end());
        set_mask(all, {});
        evaluate(kCur, 0);
        evaluate(kAvg, 1);
        cuda_check(cudaMemcpyAsync(h_out_, d_out_.p, size_t(n) * kBatchKkt * 2 * 8,
                                   cudaMemcpyDeviceToHost, stream_), "evaluation");
        cuda_check(cudaMemcpyAsync(h_ctl_, d_ctl_.p, sizeof(BCtl) * slots_.size(),
                                   cudaMemcpyDeviceToHost, stream_), "controls");
        cuda_check(cudaStreamSynchronize(stream_), "evaluation");
        const double de = since(t1);
        phase_[2] += de;
        auto t2h = SteadyClock::now();
        std::vector<int> keep_on, keep_src, restart_on, restart_src, refine_on;
        std::vector<std::pair<int, int>> certify; // (slot, candidate) for the host verifier
        const double phase_tol = o_.phase_tol > 0 ? o_.phase_tol : 10 * o_.tol;
        std::vector<Accuracy> chosen(static_cast<size_t>(n));
        for (int k = 0; k < n; ++k) {
            const int b = order_[size_t(k)];
            Slot &S = slots_[size_t(b)];
            S.iteration_seconds += dt / n;
            S.verification_seconds += de / n;
            S.device_checks++;
            S.checks++;
            const BatchItem &B = *S.item;
            const double *v0 = h_out_ + size_t(k) * kBatchKkt;
            const double *v1 = h_out_ + size_t(n + k) * kBatchKkt;
            Accuracy ca = finish_accuracy(B, v0), aa = finish_accuracy(B, v1);
            const bool avg = aa.kkt < ca.kkt;
            const double *ray = avg ? v1 : v0;
            const double *other_ray = avg ? v0 : v1;
            if (avg)
                ca = aa;
            const int src = avg ? kAvg : kCur;
            chosen[size_t(k)] = ca;
            if (ca.finite && ca.kkt < S.best.kkt) {
                keep_on.push_back(b);
                keep_src.push_back(src);
                S.best = ca;
                double level = 1;
                for (int e = 0; e < 9; ++e, level /= 10)
                    if (S.best.kkt <= level && S.reached[e] < 0)
                        S.reached[e] = since(S.start);
            }
            if ((S.empty >= 4 || !ca.finite) && !S.fp64_phase && S.best.finite) {
                // stalled backtracking or a nonfinite candidate on the FP32 values
                // ends the reduced-precision phase: FP64 refinement restarts from
                // the best point
                S.empty = 0;
                refine_on.push_back(b);
                continue;
            }
            if (S.empty >= 4) {
                retire(S, NK_SOLVE_NUMERICAL_ERROR);
                continue;
            }
            if (!ca.finite) {
                retire(S, NK_SOLVE_NUMERICAL_ERROR);
                continue;
            }
            if (ca.kkt <= o_.tol && S.iterations >= S.next_host_check) {
                // certified below, for all such instances at once, in parallel;
                // an instance certified there retires (its restart, if any, is moot)
                certify.push_back({b, src});
                S.next_host_check = S.iterations + std::max<int64_t>(1000, 10 * o_.check_every);
            }
            if (S.iterations >= 1000 && ca.primal > o_.tol) {
                // Farkas rays from the chosen and the other candidate's dual,
                // where the device screen cannot rule them out
                bool found = false;
                for (int r = 0; r < 2 && !found; ++r) {
                    const double *sv = r ? other_ray : ray;
                    // as in the single driver: only a bound that may be positive
                    if (!(sv[10] == 0 && sv[11] + sv[12] + 1e-9 * sv[13] > 0))
                        continue;
                    auto t2 = SteadyClock::now();
                    std::vector<double> ox, oy;
                    const int s2 = (r == 0) == avg ? kAvg : kCur;
                    host_point(S, point_x(S, s2), point_y(S, s2), ox, oy);
                    S.host_checks++;
                    double norm = 0;
                    bool fin = true;
                    for (double vv : oy) {
                        fin = fin && std::isfinite(vv);
                        norm = std::max(norm, std::abs(vv));
                    }
                    if (fin && norm > 0) {
                        for (double &vv : oy)
                            vv /= norm;
                        const double margin = B.verifier->infeasibility_bound(oy);
                        if (margin > 0 && std::isfinite(margin)) {
                            S.item->report.y = std::move(oy);
                            found = true;
                        }
                    }
                    S.verification_seconds += since(t2);
                }
                if (found) {
                    retire(S, NK_SOLVE_INFEASIBLE);
                    continue;
                }
            }
            if (S.iterations >= B.iteration_limit) {
                retire(S, NK_SOLVE_ITERATION_LIMIT);
                continue;
            }
            if (since(S.start) >= B.time_limit) {
                retire(S, NK_SOLVE_TIME_LIMIT);
                continue;
            }
            if (!S.fp64_phase) {
                // the reduced-precision phase ends when its best point reaches the
                // phase target or stops improving; FP64 refinement restarts from it
                if (S.best.kkt < .9 * S.stall_ref) {
                    S.stall_ref = S.best.kkt;
                    S.stall = 0;
                } else
                    ++S.stall;
                if (S.best.finite && (S.best.kkt <= phase_tol || S.stall >= 30)) {
                    refine_on.push_back(b);
                    continue;
                }
            }
            const bool due = S.since_restart >= int64_t(o_.check_every) * 2 &&
                             (ca.kkt < .5 * S.restart_kkt ||
                              S.since_restart >= std::max<int64_t>(2000, S.iterations / 2));
            if (o_.restart && due) {
                restart_on.push_back(b);
                restart_src.push_back(src);
            }
        }
        if (!certify.empty()) {
            // candidates to host memory (before any restart kernel moves them),
            // then the outward-rounded verifier on host threads
            const size_t nc = certify.size();
            std::vector<std::vector<double>> ox(nc), oy(nc);
            std::vector<Accuracy> acc(nc);
            for (size_t k = 0; k < nc; ++k) {
                Slot &S = slots_[size_t(certify[k].first)];
                host_point(S, point_x(S, certify[k].second), point_y(S, certify[k].second), ox[k],
                           oy[k]);
            }
            batch_detail::parallel_for(nc, [&](size_t k) {
                const Slot &S = slots_[size_t(certify[k].first)];
                acc[k] = S.item->verifier->evaluate(ox[k], oy[k], true);
            });
            for (size_t k = 0; k < nc; ++k) {
                Slot &S = slots_[size_t(certify[k].first)];
                S.host_checks++;
                if (acc[k].kkt <= o_.tol) {
                    S.item->report.x = std::move(ox[k]);
                    S.item->report.y = std::move(oy[k]);
                    S.item->report.accuracy = acc[k];
                    retire(S, NK_SOLVE_OPTIMAL);
                }
            }
        }
        phase_[3] += since(t2h);
        auto t3 = SteadyClock::now();
        // best points (before any restart moves the iterate)
        if (!keep_on.empty()) {
            set_mask(keep_on, keep_src);
            batch_keep<<<grid_items(ncols_ + nrows_), 256, 0, stream_>>>(
                d_ins_.p, d_ctl_.p, d_mask_.p, d_src_.p, 0, d_cols_.p, ncols_, d_rows_.p, nrows_);
        }
        if (!restart_on.empty() && o_.adaptive) {
            // primal weight from the displacement since the last restart
            set_mask(restart_on, restart_src);
            batch_displacement<<<grid_items(ncols_ + nrows_), 256, 0, stream_>>>(
                d_ins_.p, d_ctl_.p, d_mask_.p, d_src_.p, d_cols_.p, ncols_, d_rows_.p, nrows_,
                d_pk_.p);
            batch_finish<2><<<std::max(1, (n + 7) / 8), 256, 0, stream_>>>(
                d_cf_.p, d_cc_.p, ncols_, d_rf_.p, d_rc_.p, n, 0u, d_pk_.p, d_out_.p);
            cuda_check(cudaMemcpyAsync(h_out_, d_out_.p, size_t(n) * 2 * 8,
                                       cudaMemcpyDeviceToHost, stream_), "displacement");
            cuda_check(cudaStreamSynchronize(stream_), "displacement");
            for (int k = 0; k < n; ++k) {
                Slot &S = slots_[size_t(order_[size_t(k)])];
                if (!h_mask_[order_[size_t(k)]])
                    continue;
                const double dx = h_out_[2 * k], dy = h_out_[2 * k + 1];
                if (dx > 1e-24 && dy > 1e-24) {
                    const double target = std::clamp(std::sqrt(dy / dx), 1e-4, 1e4);
                    S.weight = std::sqrt(S.weight * target);
                    S.weight_updates++;
                }
            }
        }
        if (!restart_on.empty() || !refine_on.empty()) {
            // restarts (mask 1, from the chosen candidate) and FP64 refinements
            // (mask 2, from the best point) in one pass
            std::vector<int> on = restart_on, src = restart_src, val(restart_on.size(), 1);
            for (int b : refine_on) {
                on.push_back(b);
                src.push_back(kBest);
                val.push_back(2);
            }
            set_mask(on, src, val);
            batch_restart_cols<<<grid_items(ncols_ + nrows_), 256, 0, stream_>>>(
                d_ins_.p, d_ctl_.p, d_mask_.p, d_src_.p, d_cols_.p, ncols_, d_rows_.p, nrows_);
            // control first: the activity of a refined instance uses FP64 values
            batch_restart_ctl<<<std::max(1, (n + 255) / 256), 256, 0, stream_>>>(
                d_ctl_.p, d_mask_.p, d_slots_.p, n);
            batch_restart_rows<<<grid_items(nrows_), 256, 0, stream_>>>(
                d_ins_.p, d_ctl_.p, d_mask_.p, d_rows_.p, nrows_);
            // the epoch is the restarted iterate
            std::vector<int> cur_src(on.size(), kCur);
            set_mask(on, cur_src);
            batch_keep<<<grid_items(ncols_ + nrows_), 256, 0, stream_>>>(
                d_ins_.p, d_ctl_.p, d_mask_.p, d_src_.p, 1, d_cols_.p, ncols_, d_rows_.p, nrows_);
            for (size_t k = 0; k < restart_on.size(); ++k) {
                Slot &S = slots_[size_t(restart_on[k])];
                const int pos = int(std::find(order_.begin(), order_.end(), restart_on[k]) - order_.begin());
                S.restart_kkt = chosen[size_t(pos)].kkt;
                S.since_restart = 0;
                S.restarts++;
            }
            for (int b : refine_on) {
                Slot &S = slots_[size_t(b)];
                S.fp64_phase = true;
                S.phase_iterations = S.iterations;
                S.phase_best = S.best;
                S.prev_accepted = 0; // the device restarts its accepted count
                S.restart_kkt = S.best.kkt;
                S.since_restart = 0;
            }
            cuda_check(cudaGetLastError(), "batch restart");
        }
        cuda_check(cudaStreamSynchronize(stream_), "interval");
        phase_[4] += since(t3);
        auto t4 = SteadyClock::now();
        close_finished();
        phase_[5] += since(t4);
    }
};

} // namespace nk
