// The reference's CUDA plugin seam implemented over the B200 engine's C ABI.
//
// Built into the reference's library in place of src/cuda.cu (or
// src/cuda_stub.cpp), this file provides vantage::cuda_backend() and the
// device-information functions declared in src/internal.hpp:125-134 and
// include/vantage/vantage.hpp:76,145-146.  The reference's host code --
// solve_continuous, presolve, the Verifier, the branch-and-bound driver, the
// CLI, the C API and NativeSession -- is unchanged and reaches the engine
// through this adapter.  Engine errors become std::runtime_error, the
// reference's convention (src/cuda.cu:10-17), so the driver's automatic CPU
// fallback on memory-guard failures (src/solver.cpp:356-367) keeps working.
//
// cuda_batch_relaxations (the box variants of one LP relaxation that the
// branch-and-bound driver scores for strong branching) runs on the engine's
// batched solver, the two GPU presolve steps of --gpu-presolve
// (cuda_compact_matrix, cuda_propagate_integer_bounds) on its presolve kernels,
// and the barrier method's Newton solve (cuda_linear_solve) on its BiCGSTAB.
#include "internal.hpp"
#include "nk_pdhg.h"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace vantage {
namespace {

void check(nk_status status) {
    if (status != NK_OK)
        throw std::runtime_error(nk_last_error());
}

class NkBackend final : public IterationBackend {
  public:
    NkBackend(const Model &m, const std::vector<double> &x, const std::vector<double> &y,
              const nk_pdhg_options &o)
        : n_(m.c.size()), m_(m.rl.size()) {
        if (x.size() != n_ || y.size() != m_)
            throw std::runtime_error("CUDA PDHG starting point dimensions");
        nk_csr a{m.A.rows, m.A.cols, m.A.ptr.data(), m.A.index.data(), m.A.value.data()};
        nk_csr q{m.Q.rows, m.Q.cols, m.Q.ptr.data(), m.Q.index.data(), m.Q.value.data()};
        check(nk_pdhg_create(&a, m.Q.value.empty() ? nullptr : &q, m.c.data(), m.q.data(),
                             m.lb.data(), m.ub.data(), m.rl.data(), m.ru.data(), x.data(),
                             y.data(), &o, &h_));
    }
    ~NkBackend() override { nk_pdhg_destroy(h_); }
    NkBackend(const NkBackend &) = delete;
    NkBackend &operator=(const NkBackend &) = delete;

    int advance(int count, double tau, double sigma) override {
        int accepted = 0;
        check(nk_pdhg_advance(h_, count, tau, sigma, &accepted));
        return accepted;
    }
    std::vector<std::vector<double>> snapshot() override {
        int parts = 0;
        int64_t sizes[16] = {};
        check(nk_pdhg_snapshot_layout(h_, &parts, sizes));
        size_t total = 0;
        for (int i = 0; i < parts; ++i)
            total += size_t(sizes[i]);
        std::vector<double> flat(total);
        check(nk_pdhg_snapshot(h_, flat.data()));
        std::vector<std::vector<double>> out(static_cast<size_t>(parts));
        size_t at = 0;
        for (int i = 0; i < parts; ++i) {
            out[size_t(i)].assign(flat.begin() + long(at), flat.begin() + long(at + size_t(sizes[i])));
            at += size_t(sizes[i]);
        }
        return out;
    }
    void restore(const std::vector<std::vector<double>> &state) override {
        std::vector<int64_t> sizes;
        std::vector<double> flat;
        for (const auto &part : state) {
            sizes.push_back(int64_t(part.size()));
            flat.insert(flat.end(), part.begin(), part.end());
        }
        check(nk_pdhg_restore(h_, flat.data(), sizes.data(), int(sizes.size())));
    }
    int64_t rejected_steps() const override {
        int64_t r = 0;
        check(nk_pdhg_rejected_steps(h_, &r));
        return r;
    }
    bool restart_requested() const override {
        int r = 0;
        check(nk_pdhg_restart_requested(h_, &r));
        return r != 0;
    }
    double monitor() override {
        double v = 0;
        check(nk_pdhg_monitor(h_, &v));
        return v;
    }
    void candidates(std::vector<double> &x, std::vector<double> &y, std::vector<double> &ax,
                    std::vector<double> &ay) override {
        x.resize(n_);
        y.resize(m_);
        ax.resize(n_);
        ay.resize(m_);
        check(nk_pdhg_candidates(h_, x.data(), y.data(), ax.data(), ay.data()));
    }
    bool reset_candidate(bool average) override {
        check(nk_pdhg_reset_candidate(h_, average ? 1 : 0));
        return true;
    }
    void reset(const std::vector<double> &x, const std::vector<double> &y) override {
        if (x.size() != n_ || y.size() != m_)
            throw std::runtime_error("CUDA PDHG reset dimensions");
        check(nk_pdhg_reset(h_, x.data(), y.data()));
    }

  private:
    size_t n_, m_;
    nk_pdhg *h_ = nullptr;
};

} // namespace

std::unique_ptr<IterationBackend> cuda_backend(const Model &m, const std::vector<double> &x,
                                               const std::vector<double> &y, bool adaptive,
                                               bool halpern, double reflection,
                                               bool residual_restarts, bool graphs,
                                               const std::string &indices,
                                               const std::string &precision) {
    nk_pdhg_options o{};
    o.adaptive = adaptive;
    o.halpern = halpern;
    o.reflection = reflection;
    o.residual_restarts = residual_restarts;
    o.graphs = graphs;
    if (indices == "auto")
        o.index_bits = 0;
    else if (indices == "32")
        o.index_bits = 32;
    else if (indices == "64")
        o.index_bits = 64;
    else
        throw std::runtime_error("GPU indices must be auto, 32, or 64");
    if (precision == "fp64")
        o.precision = NK_PRECISION_FP64;
    else if (precision == "mixed")
        o.precision = NK_PRECISION_MIXED;
    else
        throw std::runtime_error("Matrix precision must be fp64 or mixed");
    return std::make_unique<NkBackend>(m, x, y, o);
}

Hardware hardware_info() {
    Hardware h;
    int available = 0;
    double free_bytes = 0, total_bytes = 0;
    if (nk_hardware_info(&available, &free_bytes, &total_bytes) == NK_OK) {
        h.gpu_available = available != 0;
        h.free_gpu_bytes = free_bytes;
        h.total_gpu_bytes = total_bytes;
    }
    return h;
}

bool cuda_available() { return nk_cuda_available() != 0; }

std::string cuda_description() {
    char buffer[256] = {};
    if (nk_cuda_description(buffer, sizeof(buffer)) != NK_OK)
        return "CUDA description unavailable";
    return buffer;
}

// cuda_compact_matrix (src/cuda.cu:978-1032), the CSR step of prepare with
// --gpu-presolve: the reference's argument checks and messages, then the
// engine's count / scan / ordered-scatter compaction (nk_compact_csr).
Sparse cuda_compact_matrix(const Sparse &matrix, const std::vector<int64_t> &rows,
                           const std::vector<int64_t> &columns, int64_t output_columns) {
    if (columns.size() != size_t(matrix.cols) || output_columns < 0 || rows.size() >= INT_MAX)
        throw std::runtime_error("GPU compaction dimensions");
    int64_t previous = -1;
    for (auto row : rows) {
        if (row <= previous || row >= matrix.rows)
            throw std::runtime_error("GPU compaction row map");
        previous = row;
    }
    previous = -1;
    for (auto column : columns)
        if (column >= 0) {
            if (column <= previous || column >= output_columns)
                throw std::runtime_error("GPU compaction column map");
            previous = column;
        }
    Sparse result;
    result.rows = int64_t(rows.size());
    result.cols = output_columns;
    if (rows.empty()) {
        result.ptr = {0};
        return result;
    }
    int64_t capacity = 0;
    for (auto row : rows)
        capacity += matrix.ptr[size_t(row + 1)] - matrix.ptr[size_t(row)];
    result.ptr.resize(rows.size() + 1);
    result.index.resize(size_t(capacity));
    result.value.resize(size_t(capacity));
    nk_csr a{matrix.rows, matrix.cols, matrix.ptr.data(), matrix.index.data(), matrix.value.data()};
    int64_t kept = 0;
    check(nk_compact_csr(&a, int64_t(rows.size()), rows.data(), columns.data(), output_columns,
                         result.ptr.data(), result.index.data(), result.value.data(), capacity,
                         &kept));
    result.index.resize(size_t(kept));
    result.value.resize(size_t(kept));
    return result;
}
// cuda_propagate_integer_bounds (src/cuda.cu:1033-1135): the reference's checks
// and messages, then `passes` rounds of directed-rounding proposals on the GPU
// (nk_propagate_bounds).  Integer and binary columns round inward.
bool cuda_propagate_integer_bounds(const Model &m, std::vector<double> &lb,
                                   std::vector<double> &ub, int passes) {
    m.validate();
    if (lb.size() != m.c.size() || ub.size() != m.c.size() || passes < 0 || passes > 100)
        throw std::runtime_error("GPU propagation dimensions/pass limit");
    for (size_t j = 0; j < lb.size(); ++j)
        if (std::isnan(lb[j]) || std::isnan(ub[j]) || lb[j] < m.lb[j] || ub[j] > m.ub[j] ||
            lb[j] > ub[j])
            throw std::runtime_error("Invalid GPU propagation bounds");
    if (m.A.rows == 0 || passes == 0)
        return true;
    std::vector<int> integer(m.c.size(), 0);
    for (size_t j = 0; j < m.types.size() && j < integer.size(); ++j)
        integer[j] = m.types[j] != VarType::Continuous;
    nk_csr a{m.A.rows, m.A.cols, m.A.ptr.data(), m.A.index.data(), m.A.value.data()};
    int feasible = 0;
    check(nk_propagate_bounds(&a, integer.data(), m.rl.data(), m.ru.data(), lb.data(), ub.data(),
                              passes, &feasible));
    return feasible != 0;
}
// cuda_batch_relaxations (src/cuda.cu:1136-1266): the same argument checks,
// start point (initial_x clamped into each box, initial_y), limits and result
// fields as the reference.  Where the reference advances all boxes with one
// fixed-step PDHG and keeps the better of the average and the current point,
// each box here is an instance of the engine's batch -- its own presolve,
// scaling, adaptive steps and restarts, FP64 matrices -- and returns its best
// point.  Either way the box's status comes from the reference's own
// verify(child, x, y): OPTIMAL when the KKT error is within tol, else the limit
// that ended the run.
std::vector<Result> cuda_batch_relaxations(const Model &m,
                                           const std::vector<std::vector<double>> &lower,
                                           const std::vector<std::vector<double>> &upper,
                                           const Options &o) {
    m.validate();
    if (m.is_qp() || m.is_mip() || lower.empty() || lower.size() != upper.size() ||
        lower.size() > 32 || m.c.empty())
        throw std::runtime_error("Invalid CUDA LP relaxation batch");
    using Clock = std::chrono::steady_clock;
    const auto start = Clock::now();
    auto elapsed = [&] { return std::chrono::duration<double>(Clock::now() - start).count(); };
    const size_t n = m.c.size(), rows = m.rl.size(), boxes = lower.size();
    for (size_t b = 0; b < boxes; ++b) {
        if (lower[b].size() != n || upper[b].size() != n)
            throw std::runtime_error("Batch bound dimensions");
        for (size_t j = 0; j < n; ++j)
            if (std::isnan(lower[b][j]) || std::isnan(upper[b][j]) || lower[b][j] > upper[b][j] ||
                lower[b][j] < m.lb[j] || upper[b][j] > m.ub[j])
                throw std::runtime_error("Invalid batch bounds");
    }
    nk_batch_options bo;
    nk_batch_defaults(&bo);
    bo.tol = o.tol;
    bo.time_limit = o.time_limit;
    bo.iteration_limit = o.iteration_limit;
    bo.check_every = o.check_every;
    bo.presolve = o.presolve;
    bo.scaling_combined = o.scaling == "combined";
    bo.scaling_passes = o.scaling_passes;
    bo.adaptive = o.adaptive;
    bo.restart = o.restart;
    bo.graphs = o.cuda_graphs;
    bo.precision = NK_PRECISION_FP64;
    nk_batch *batch = nullptr;
    check(nk_batch_create(&bo, &batch));
    struct Closer {
        nk_batch *b;
        ~Closer() { nk_batch_destroy(b); }
    } closer{batch};
    nk_csr a{m.A.rows, m.A.cols, m.A.ptr.data(), m.A.index.data(), m.A.value.data()};
    nk_csr noq{0, 0, nullptr, nullptr, nullptr};
    std::vector<double> x0(n);
    for (size_t b = 0; b < boxes; ++b) {
        nk_model child{a, noq, m.c.data(), m.q.size() == n ? m.q.data() : nullptr, lower[b].data(), upper[b].data(),
                       m.rl.data(), m.ru.data(), m.offset};
        for (size_t j = 0; j < n; ++j)
            x0[j] = std::clamp(o.initial_x.empty() ? 0 : o.initial_x.at(j), lower[b][j],
                               upper[b][j]);
        if (!o.initial_y.empty() && o.initial_y.size() != rows)
            throw std::runtime_error("Batch initial dual dimensions");
        nk_batch_item *item = nullptr;
        double bytes = 0;
        check(nk_batch_prepare_from(&child, &bo, x0.data(),
                                    o.initial_y.empty() ? nullptr : o.initial_y.data(), &item,
                                    &bytes));
        int admitted = 0;
        nk_status st = nk_batch_admit(batch, item, int64_t(b), &admitted);
        if (st != NK_OK || !admitted) {
            nk_batch_item_free(item);
            if (st != NK_OK)
                check(st);
            throw std::runtime_error("GPU relaxation batch exceeds available memory");
        }
    }
    std::vector<Result> results(boxes);
    std::vector<int64_t> finished(boxes);
    size_t collected = 0;
    std::vector<double> x(n), y(rows);
    while (collected < boxes) {
        int count = 0;
        check(nk_batch_step(batch, 1 << 30, finished.data(), int(finished.size()), &count));
        for (int k = 0; k < count; ++k) {
            const size_t b = size_t(finished[size_t(k)]);
            nk_solve_result sr{};
            check(nk_batch_result(batch, int64_t(b), &sr, x.data(), y.data()));
            Model child = m;
            child.lb = lower[b];
            child.ub = upper[b];
            Result &r = results[b];
            r.backend = gpu_backend_name();
            r.device_name = cuda_description();
            r.method_selected = "batched-pdhg";
            r.x = x;
            r.y = y;
            r.accuracy = verify(child, r.x, r.y);
            r.status = r.accuracy.finite && r.accuracy.kkt <= o.tol ? "OPTIMAL"
                       : stop_requested(o)                          ? "INTERRUPTED"
                       : elapsed() >= o.time_limit                  ? "TIME_LIMIT"
                                                                    : "ITERATION_LIMIT";
            r.iterations = sr.iterations;
            r.restarts = sr.restarts;
            r.rejected_steps = sr.rejected_steps;
            r.preprocess_seconds = sr.preprocess_seconds;
            r.iteration_seconds = sr.iteration_seconds;
            r.verification_seconds = sr.verification_seconds;
            ++collected;
        }
        if (count == 0 && collected < boxes)
            throw std::runtime_error("GPU relaxation batch stopped without finishing");
    }
    for (auto &r : results)
        r.seconds = elapsed();
    return results;
}
// cuda_linear_solve (src/cuda.cu:1328-1434): the barrier's Newton systems on the
// engine's device-resident BiCGSTAB (nk_linear_solve), diagonally right-
// preconditioned -- the barrier's Newton matrices scale their rows over many
// decades as the iterates approach the boundary -- then the reference's own
// acceptance test of the solution (finite, max-norm residual within tolerance).
std::vector<double> cuda_linear_solve(const Sparse &matrix, const std::vector<double> &rhs,
                                      const Options &o, bool fp32_matrix, double tolerance) {
    if (matrix.rows != matrix.cols || rhs.size() != size_t(matrix.rows))
        throw std::runtime_error("Newton matrix dimensions");
    const size_t n = rhs.size();
    if (!n)
        return {};
    if (stop_requested(o))
        throw std::runtime_error("GPU Newton solve interrupted or time-limited");
    nk_csr a{matrix.rows, matrix.cols, matrix.ptr.data(), matrix.index.data(), matrix.value.data()};
    std::vector<double> solution(n);
    int converged = 0, timed_out = 0;
    check(nk_linear_solve(&a, rhs.data(), fp32_matrix ? 1 : 0, 1, std::max(0., o.time_limit),
                          solution.data(), &converged, &timed_out));
    if (timed_out)
        throw std::runtime_error("GPU Newton solve interrupted or time-limited");
    auto activity = matrix.multiply(solution);
    long double error = 0, rhsnorm = 0;
    for (size_t j = 0; j < n; ++j) {
        if (!std::isfinite(solution[j]))
            throw std::runtime_error("Nonfinite GPU Newton solution");
        error = std::max(error, std::abs((long double)activity[j] - rhs[j]));
        rhsnorm = std::max(rhsnorm, std::abs((long double)rhs[j]));
    }
    if (!converged || error > (long double)tolerance * (1 + rhsnorm))
        throw std::runtime_error("GPU Newton residual/breakdown check failed");
    return solution;
}

} // namespace vantage
