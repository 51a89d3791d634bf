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
// The side entries of the CUDA build that are not part of the PDHG path
// (cuda_batch_relaxations, cuda_linear_solve, cuda_propagate_integer_bounds,
// cuda_compact_matrix) report that the B200 engine does not provide them,
// exactly where a CPU build reports that CUDA is missing.
#include "internal.hpp"
#include "nk_pdhg.h"

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

Sparse cuda_compact_matrix(const Sparse &, const std::vector<int64_t> &,
                           const std::vector<int64_t> &, int64_t) {
    throw std::runtime_error("GPU matrix compaction is not provided by the B200 PDHG engine");
}
bool cuda_propagate_integer_bounds(const Model &, std::vector<double> &, std::vector<double> &,
                                   int) {
    throw std::runtime_error("GPU propagation is not provided by the B200 PDHG engine");
}
std::vector<Result> cuda_batch_relaxations(const Model &, const std::vector<std::vector<double>> &,
                                           const std::vector<std::vector<double>> &,
                                           const Options &) {
    throw std::runtime_error("Batched relaxations are not provided by the B200 PDHG engine");
}
std::vector<double> cuda_linear_solve(const Sparse &, const std::vector<double> &,
                                      const Options &, bool, double) {
    throw std::runtime_error("GPU Newton solve is not provided by the B200 PDHG engine");
}

} // namespace vantage
