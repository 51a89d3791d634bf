// Host-side model, presolve/scaling and verifier of the solve path.  These are
// the reference's host stages around the iteration backend (prepare,
// src/preprocess.cpp:133-346; Verifier, src/verify.cpp:6-244), restated so
// that the prepared model and the acceptance test are bit-identical to the
// reference's.  Compiled as plain C++ (no CUDA), with FMA contraction off.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace nk {

struct Csr { // CSR with 64-bit offsets and indices (vantage::Sparse)
    int64_t rows = 0, cols = 0;
    std::vector<int64_t> ptr{0}, index;
    std::vector<double> value;
};

struct Entry {
    int64_t row, col;
    double value;
};

struct HostModel { // the continuous part of vantage::Model
    Csr A, Q;
    std::vector<double> c, q, lb, ub, rl, ru;
    double offset = 0;
    bool is_qp() const;
};

struct PrepareOptions {
    bool presolve = true;
    std::string scaling = "ruiz"; // "ruiz" or "combined"
    int scaling_passes = 5;
};

struct Prepared { // vantage::Prepared (src/internal.hpp:16-25)
    HostModel model;
    std::vector<int64_t> cols, rows, lower_rows, upper_rows;
    std::vector<double> fixed, column_scale, row_scale, failure_ray;
    double objective_scale = 1;
    std::string failure, reason;
    std::vector<double> restore_x(const std::vector<double> &x) const;
    std::vector<double> restore_y(const std::vector<double> &y, size_t n) const;
};

constexpr double kInf = __builtin_huge_val();

struct Accuracy { // vantage::Accuracy (include/vantage/vantage.hpp:78-82)
    double objective = kInf, primal = kInf, dual = kInf, gap = kInf, kkt = kInf;
    double primal_absolute = kInf, dual_absolute = kInf, complementarity = kInf,
           lower_bound = -kInf;
    bool finite = false;
};

// When set (per thread), host loops (presolve, scaling, verifier products) run
// serially: callers that already run one model per thread keep OpenMP from
// nesting teams inside them.
void host_serial(bool serial);
bool host_serial_enabled();
struct HostSerialScope { // serial host loops on this thread until the scope ends
    bool was;
    HostSerialScope() : was(host_serial_enabled()) { host_serial(true); }
    ~HostSerialScope() { host_serial(was); }
};

Csr build_csr(int64_t rows, int64_t cols, std::vector<Entry> e);
Csr transpose(const Csr &a);
// The entry checks of Model::validate (src/model.cpp:107-123) for a model whose
// CSR offsets are already valid: every coefficient of A and Q finite and every
// column index inside [0, cols); Q's columns strictly increase within a row and
// Q equals its transpose exactly.  Throws std::runtime_error with the
// reference's message.
void validate_entries(const HostModel &m);
Prepared prepare(const HostModel &src, const PrepareOptions &o);

// Verifier over one original model; keeps A^T like the reference's Verifier.
class Verifier {
  public:
    explicit Verifier(const HostModel &m);
    Accuracy evaluate(const std::vector<double> &x, const std::vector<double> &y,
                      bool safe_bound = true) const;
    double infeasibility_bound(const std::vector<double> &y) const;

  private:
    const HostModel &m_;
    Csr at_;
};

} // namespace nk
