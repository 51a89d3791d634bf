// Test infrastructure only: a plain C shim over the reference's own C++ API
// (vantage::Model, vantage::solve, vantage::cpu_backend, vantage::Verifier,
// vantage::prepare).  It is compiled together with the reference sources into
// oracle/_ref/ by oracle/Makefile and is loaded only by tests, by smoke() and
// by bench.py's CPU-baseline / reference arm.  Nothing in niryukti_b200/ links it.
//
// Interfaces wrapped (reference paths):
//   Sparse::build / Model          include/vantage/vantage.hpp:17-39, src/model.cpp:11-73
//   solve                          src/solver.cpp:55-105 (PDHG: solve_continuous :106-735)
//   cpu_backend / IterationBackend src/internal.hpp:102-128, src/cpu.cpp:249-259
//   cuda_backend                   src/internal.hpp:129-134 (the seam the engine plugs into)
//   Verifier::evaluate / verify    src/verify.cpp:103-244
//   prepare / Prepared             src/preprocess.cpp:133-346, src/internal.hpp:16-25
#include "internal.hpp"
#include <cstdio>
#include <cstring>
#include <map>
#include <sstream>
#include <string>

using namespace vantage;

namespace {
thread_local char g_error[2048] = {};
void set_error(const char *what) { std::snprintf(g_error, sizeof(g_error), "%s", what); }

std::map<std::string, std::string> parse_kv(const char *text) {
    std::map<std::string, std::string> kv;
    if (!text)
        return kv;
    std::stringstream ss(text);
    std::string item;
    while (std::getline(ss, item, ';')) {
        auto eq = item.find('=');
        if (eq == std::string::npos)
            continue;
        kv[item.substr(0, eq)] = item.substr(eq + 1);
    }
    return kv;
}

double parse_double(const std::string &s) {
    if (s == "inf")
        return inf;
    if (s == "-inf")
        return -inf;
    return std::stod(s);
}

Options make_options(const char *text) {
    Options o;
    for (auto &[k, v] : parse_kv(text)) {
        if (k == "device") o.device = v;
        else if (k == "method") o.method = v;
        else if (k == "tol") o.tol = parse_double(v);
        else if (k == "time_limit") o.time_limit = parse_double(v);
        else if (k == "iteration_limit") o.iteration_limit = std::stoll(v);
        else if (k == "check_every") o.check_every = std::stoi(v);
        else if (k == "scaling_passes") o.scaling_passes = std::stoi(v);
        else if (k == "threads") o.threads = std::stoi(v);
        else if (k == "presolve") o.presolve = v == "1";
        else if (k == "restart") o.restart = v == "1";
        else if (k == "adaptive") o.adaptive = v == "1";
        else if (k == "verbose") o.verbose = v == "1";
        else if (k == "scaling") o.scaling = v;
        else if (k == "primal_weight") o.primal_weight = v;
        else if (k == "cuda_graphs") o.cuda_graphs = v == "1";
        else if (k == "gpu_monitor") o.gpu_monitor = v == "1";
        else if (k == "gpu_indices") o.gpu_indices = v;
        else if (k == "matrix_precision") o.matrix_precision = v;
        else if (k == "polishing") o.polishing = v == "1";
        else if (k == "gpu_presolve") o.gpu_presolve = v == "1";
        else throw std::runtime_error("unknown option " + k);
    }
    return o;
}

Sparse make_csr(int64_t rows, int64_t cols, const int64_t *ptr, const int64_t *idx,
                const double *val) {
    // Route through Sparse::build so the reference's own canonicalisation applies.
    std::vector<Entry> e;
    if (ptr) {
        e.reserve(size_t(ptr[rows]));
        for (int64_t i = 0; i < rows; ++i)
            for (int64_t k = ptr[i]; k < ptr[i + 1]; ++k)
                e.push_back({i, idx[k], val[k]});
    }
    return Sparse::build(rows, cols, std::move(e));
}
} // namespace

struct ref_model {
    Model m;
};
struct ref_backend {
    std::unique_ptr<IterationBackend> b;
    size_t n, m;
};
struct ref_prepared {
    Prepared p;
};

extern "C" {
const char *ref_last_error(void) { return g_error; }

ref_model *ref_model_new(int64_t m, int64_t n, const int64_t *ptr, const int64_t *idx,
                         const double *val, const double *c, const double *q, const double *lb,
                         const double *ub, const double *rl, const double *ru, const int64_t *qptr,
                         const int64_t *qidx, const double *qval, double offset) {
    try {
        auto *r = new ref_model;
        auto &M = r->m;
        M.A = make_csr(m, n, ptr, idx, val);
        M.c.assign(c, c + n);
        M.q = q ? std::vector<double>(q, q + n) : std::vector<double>(size_t(n), 0.0);
        M.lb.assign(lb, lb + n);
        M.ub.assign(ub, ub + n);
        M.rl.assign(rl, rl + m);
        M.ru.assign(ru, ru + m);
        M.types.assign(size_t(n), VarType::Continuous);
        M.names.reserve(size_t(n));
        for (int64_t j = 0; j < n; ++j)
            M.names.push_back("x" + std::to_string(j));
        M.row_names.reserve(size_t(m));
        for (int64_t i = 0; i < m; ++i)
            M.row_names.push_back("r" + std::to_string(i));
        if (qptr && qptr[n] > 0)
            M.Q = make_csr(n, n, qptr, qidx, qval);
        else {
            M.Q.rows = M.Q.cols = 0;
        }
        M.offset = offset;
        M.validate();
        return r;
    } catch (const std::exception &e) {
        set_error(e.what());
        return nullptr;
    }
}
void ref_model_free(ref_model *r) { delete r; }

// Canonical CSR of the model as the reference stores it (after Sparse::build).
int64_t ref_model_nnz(ref_model *r) { return int64_t(r->m.A.value.size()); }
void ref_model_csr(ref_model *r, int64_t *ptr, int64_t *idx, double *val) {
    auto &A = r->m.A;
    std::memcpy(ptr, A.ptr.data(), A.ptr.size() * sizeof(int64_t));
    std::memcpy(idx, A.index.data(), A.index.size() * sizeof(int64_t));
    std::memcpy(val, A.value.data(), A.value.size() * sizeof(double));
}
void ref_model_transpose(ref_model *r, int64_t *ptr, int64_t *idx, double *val) {
    auto t = r->m.A.transpose();
    std::memcpy(ptr, t.ptr.data(), t.ptr.size() * sizeof(int64_t));
    std::memcpy(idx, t.index.data(), t.index.size() * sizeof(int64_t));
    std::memcpy(val, t.value.data(), t.value.size() * sizeof(double));
}
void ref_model_multiply(ref_model *r, const double *x, double *out) {
    std::vector<double> xv(x, x + r->m.A.cols);
    auto y = r->m.A.multiply(xv);
    std::memcpy(out, y.data(), y.size() * sizeof(double));
}
double ref_model_quadratic_norm_bound(ref_model *r) { return r->m.quadratic_norm_bound(); }

// The reference's own model reader (read_model, src/io.cpp:800-814: JSON,
// MPS, LP or QPLIB by file extension).
ref_model *ref_model_read(const char *path) {
    try {
        auto *r = new ref_model;
        r->m = read_model(path);
        return r;
    } catch (const std::exception &e) {
        set_error(e.what());
        return nullptr;
    }
}
// {m, n, nnz, qnnz, integer columns} of a model.
void ref_model_dims(ref_model *r, int64_t *dims) {
    const Model &M = r->m;
    dims[0] = int64_t(M.rl.size());
    dims[1] = int64_t(M.c.size());
    dims[2] = int64_t(M.A.value.size());
    dims[3] = M.Q.ptr.empty() ? 0 : int64_t(M.Q.value.size());
    int64_t integer = 0;
    for (auto t : M.types)
        integer += t != VarType::Continuous;
    dims[4] = integer;
}
// The continuous arrays of a model; q is zero when the model has none, and
// Q's arrays are written only when it has entries.
void ref_model_arrays(ref_model *r, double *c, double *q, double *lb, double *ub, double *rl,
                      double *ru, double *offset, int64_t *qptr, int64_t *qidx, double *qval) {
    const Model &M = r->m;
    auto put = [](double *dst, const std::vector<double> &v) {
        std::memcpy(dst, v.data(), v.size() * sizeof(double));
    };
    put(c, M.c);
    if (M.q.size() == M.c.size())
        put(q, M.q);
    else
        std::fill(q, q + M.c.size(), 0.0);
    put(lb, M.lb);
    put(ub, M.ub);
    put(rl, M.rl);
    put(ru, M.ru);
    *offset = M.offset;
    if (!M.Q.ptr.empty() && !M.Q.value.empty()) {
        std::memcpy(qptr, M.Q.ptr.data(), M.Q.ptr.size() * sizeof(int64_t));
        std::memcpy(qidx, M.Q.index.data(), M.Q.index.size() * sizeof(int64_t));
        put(qval, M.Q.value);
    }
}

// stats: [objective, primal, dual, gap, kkt, primal_abs, dual_abs, complementarity,
//         lower_bound, finite, iterations, restarts, rejected_steps, seconds,
//         iteration_seconds, verification_seconds, preprocess_seconds, weight_updates,
//         host_candidate_checks, removed_columns, removed_rows]
int ref_solve(ref_model *r, const char *opts, double *x_out, double *y_out, double *stats,
              char *status, int status_len) {
    try {
        auto o = make_options(opts);
        interrupted = 0;
        auto res = solve(r->m, o);
        const auto &a = res.accuracy;
        double s[] = {a.objective,
                      a.primal,
                      a.dual,
                      a.gap,
                      a.kkt,
                      a.primal_absolute,
                      a.dual_absolute,
                      a.complementarity,
                      a.lower_bound,
                      a.finite ? 1.0 : 0.0,
                      double(res.iterations),
                      double(res.restarts),
                      double(res.rejected_steps),
                      res.seconds,
                      res.iteration_seconds,
                      res.verification_seconds,
                      res.preprocess_seconds,
                      double(res.weight_updates),
                      double(res.host_candidate_checks),
                      double(res.removed_columns),
                      double(res.removed_rows)};
        std::memcpy(stats, s, sizeof(s));
        if (x_out && res.x.size() == r->m.c.size())
            std::memcpy(x_out, res.x.data(), res.x.size() * sizeof(double));
        if (y_out && res.y.size() == r->m.rl.size())
            std::memcpy(y_out, res.y.data(), res.y.size() * sizeof(double));
        std::snprintf(status, size_t(status_len), "%s", res.status.c_str());
        set_error(res.message.c_str()); // the result's message (empty on success)
        return 0;
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}

// acc: [objective, primal, dual, gap, kkt, primal_abs, dual_abs, complementarity,
//       lower_bound, finite]
int ref_verify(ref_model *r, const double *x, const double *y, int safe, double *acc) {
    try {
        Verifier v(r->m);
        std::vector<double> xv(x, x + r->m.c.size()), yv(y, y + r->m.rl.size());
        auto a = v.evaluate(xv, yv, safe != 0);
        double s[] = {a.objective,       a.primal,          a.dual,   a.gap,
                      a.kkt,             a.primal_absolute, a.dual_absolute,
                      a.complementarity, a.lower_bound,     a.finite ? 1.0 : 0.0};
        std::memcpy(acc, s, sizeof(s));
        return 0;
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}
double ref_infeasibility_bound(ref_model *r, const double *y) {
    Verifier v(r->m);
    return v.infeasibility_bound(std::vector<double>(y, y + r->m.rl.size()));
}

// Step-level access to an IterationBackend built by the reference's own factories.
// device: 0 = cpu_backend, 1 = cuda_backend (whatever the linked library provides).
ref_backend *ref_backend_new(ref_model *r, int device, const double *x, const double *y,
                             int adaptive, int halpern, double reflection, int restarts, int graphs,
                             const char *indices, const char *precision) {
    try {
        std::vector<double> xv(x, x + r->m.c.size()), yv(y, y + r->m.rl.size());
        auto *h = new ref_backend;
        h->n = xv.size();
        h->m = yv.size();
        if (device == 0)
            h->b = cpu_backend(r->m, xv, yv, adaptive != 0, halpern != 0, reflection, restarts != 0);
        else
            h->b = cuda_backend(r->m, xv, yv, adaptive != 0, halpern != 0, reflection,
                                restarts != 0, graphs != 0, indices ? indices : "auto",
                                precision ? precision : "fp64");
        return h;
    } catch (const std::exception &e) {
        set_error(e.what());
        return nullptr;
    }
}
void ref_backend_free(ref_backend *h) { delete h; }
int ref_backend_advance(ref_backend *h, int count, double tau, double sigma) {
    try {
        return h->b->advance(count, tau, sigma);
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}
int64_t ref_backend_rejected(ref_backend *h) { return h->b->rejected_steps(); }
int ref_backend_restart_requested(ref_backend *h) { return h->b->restart_requested() ? 1 : 0; }
double ref_backend_monitor(ref_backend *h) {
    try {
        return h->b->monitor();
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}
int ref_backend_candidates(ref_backend *h, double *x, double *y, double *xa, double *ya) {
    try {
        std::vector<double> a, b, c, d;
        h->b->candidates(a, b, c, d);
        std::memcpy(x, a.data(), a.size() * sizeof(double));
        std::memcpy(y, b.data(), b.size() * sizeof(double));
        std::memcpy(xa, c.data(), c.size() * sizeof(double));
        std::memcpy(ya, d.data(), d.size() * sizeof(double));
        return 0;
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}
int ref_backend_reset(ref_backend *h, const double *x, const double *y) {
    try {
        h->b->reset(std::vector<double>(x, x + h->n), std::vector<double>(y, y + h->m));
        return 0;
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}
int ref_backend_reset_candidate(ref_backend *h, int average) {
    try {
        return h->b->reset_candidate(average != 0) ? 1 : 0;
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}
// Snapshot flattened: returns the number of doubles written (or needed when out is null).
int64_t ref_backend_snapshot(ref_backend *h, double *out, int64_t *sizes, int max_parts) {
    auto s = h->b->snapshot();
    int64_t total = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        if (sizes && int(i) < max_parts)
            sizes[i] = int64_t(s[i].size());
        if (out)
            std::memcpy(out + total, s[i].data(), s[i].size() * sizeof(double));
        total += int64_t(s[i].size());
    }
    return total;
}

// Presolve + scaling exactly as solve_continuous runs it.
ref_prepared *ref_prepare(ref_model *r, const char *opts) {
    try {
        auto o = make_options(opts);
        auto *h = new ref_prepared;
        h->p = prepare(r->m, o);
        return h;
    } catch (const std::exception &e) {
        set_error(e.what());
        return nullptr;
    }
}
void ref_prepared_free(ref_prepared *h) { delete h; }
// dims: [rows, cols, nnz, qnnz, failure(0/1)]
void ref_prepared_dims(ref_prepared *h, int64_t *dims) {
    auto &m = h->p.model;
    dims[0] = int64_t(m.rl.size());
    dims[1] = int64_t(m.c.size());
    dims[2] = int64_t(m.A.value.size());
    dims[3] = int64_t(m.Q.value.size());
    dims[4] = h->p.failure.empty() ? 0 : 1;
}
const char *ref_prepared_failure(ref_prepared *h) { return h->p.failure.c_str(); }
// Copies every array of the prepared model; any pointer may be null to skip it.
void ref_prepared_get(ref_prepared *h, int64_t *ptr, int64_t *idx, double *val, double *c,
                      double *q, double *lb, double *ub, double *rl, double *ru, int64_t *cols,
                      int64_t *rows, int64_t *lower_rows, int64_t *upper_rows, double *fixed,
                      double *column_scale, double *row_scale, double *scalars /*objective_scale, offset*/,
                      int64_t *qptr, int64_t *qidx, double *qval) {
    auto &p = h->p;
    auto &m = p.model;
    auto cp = [](auto *dst, const auto &v) {
        if (dst && !v.empty())
            std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(ptr, m.A.ptr);
    cp(idx, m.A.index);
    cp(val, m.A.value);
    cp(c, m.c);
    cp(q, m.q);
    cp(lb, m.lb);
    cp(ub, m.ub);
    cp(rl, m.rl);
    cp(ru, m.ru);
    cp(cols, p.cols);
    cp(rows, p.rows);
    cp(lower_rows, p.lower_rows);
    cp(upper_rows, p.upper_rows);
    cp(fixed, p.fixed);
    cp(column_scale, p.column_scale);
    cp(row_scale, p.row_scale);
    if (scalars) {
        scalars[0] = p.objective_scale;
        scalars[1] = m.offset;
    }
    cp(qptr, m.Q.ptr);
    cp(qidx, m.Q.index);
    cp(qval, m.Q.value);
}
int ref_cuda_available(void) { return cuda_available() ? 1 : 0; }

// cuda_linear_solve(matrix, rhs, options, fp32_matrix, tolerance) --
// src/internal.hpp:49-50: K (n x n CSR) x = rhs; x_out gets the solution.
int ref_linear_solve(int64_t n, const int64_t *ptr, const int64_t *idx, const double *val,
                     const double *rhs, int fp32_matrix, double tolerance, double *x_out) {
    try {
        Sparse k;
        k.rows = k.cols = n;
        k.ptr.assign(ptr, ptr + n + 1);
        k.index.assign(idx, idx + ptr[n]);
        k.value.assign(val, val + ptr[n]);
        Options o;
        auto x = cuda_linear_solve(k, std::vector<double>(rhs, rhs + n), o, fp32_matrix != 0,
                                   tolerance);
        std::memcpy(x_out, x.data(), x.size() * sizeof(double));
        return 0;
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}

// cuda_batch_relaxations(model, lower, upper, options) -- src/internal.hpp:60-62.
// lower / upper: `boxes` rows of n bounds; x0 / y0 (may be NULL) become
// Options::initial_x / initial_y.  Per box, stats[10 * b ...] = [objective,
// kkt, finite, iterations, restarts, seconds, 0, 0, 0, 0], status[b] in
// {0 OPTIMAL, 1 INTERRUPTED, 2 TIME_LIMIT, 3 ITERATION_LIMIT, 4 other}; x_out
// (boxes * n) and y_out (boxes * m) may be NULL.
int ref_batch_relaxations(ref_model *r, int boxes, const double *lower, const double *upper,
                          const double *x0, const double *y0, const char *opts, double *stats,
                          int *status, double *x_out, double *y_out) {
    try {
        auto o = make_options(opts);
        const size_t n = r->m.c.size(), m = r->m.rl.size();
        if (x0)
            o.initial_x.assign(x0, x0 + n);
        if (y0)
            o.initial_y.assign(y0, y0 + m);
        std::vector<std::vector<double>> lo(static_cast<size_t>(boxes)), up(static_cast<size_t>(boxes));
        for (int b = 0; b < boxes; ++b) {
            lo[size_t(b)].assign(lower + size_t(b) * n, lower + size_t(b + 1) * n);
            up[size_t(b)].assign(upper + size_t(b) * n, upper + size_t(b + 1) * n);
        }
        auto res = cuda_batch_relaxations(r->m, lo, up, o);
        for (size_t b = 0; b < res.size(); ++b) {
            const auto &q = res[b];
            double s[10] = {q.accuracy.objective, q.accuracy.kkt, q.accuracy.finite ? 1. : 0.,
                            double(q.iterations), double(q.restarts), q.seconds, 0, 0, 0, 0};
            std::memcpy(stats + 10 * b, s, sizeof(s));
            status[b] = q.status == "OPTIMAL"           ? 0
                        : q.status == "INTERRUPTED"     ? 1
                        : q.status == "TIME_LIMIT"      ? 2
                        : q.status == "ITERATION_LIMIT" ? 3
                                                        : 4;
            if (x_out && q.x.size() == n)
                std::memcpy(x_out + b * n, q.x.data(), n * sizeof(double));
            if (y_out && q.y.size() == m)
                std::memcpy(y_out + b * m, q.y.data(), m * sizeof(double));
        }
        return 0;
    } catch (const std::exception &e) {
        set_error(e.what());
        return -1;
    }
}
}
