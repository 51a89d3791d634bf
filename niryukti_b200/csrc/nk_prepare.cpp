// Host side of the solve path: presolve + scaling (the reference's prepare(),
// src/preprocess.cpp:6-346), the maps back to the caller's model
// (Prepared::restore_x / restore_y, src/preprocess.cpp:121-132) and the FP64 /
// long double verifier used for the final, outward-rounded acceptance test
// (Verifier::evaluate and lp_lower_bound, src/verify.cpp:6-244).
//
// Every operation is restated in the reference's order and precision (double,
// long double where the reference uses it), compiled without FMA contraction,
// so the prepared model is bit-identical to the reference's.
#include "nk_host.hpp"
#include <omp.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>

namespace nk {
namespace {
constexpr double INF = std::numeric_limits<double>::infinity();
// When set (per thread), host loops run serially: callers that already run
// one presolve or verifier per thread keep OpenMP from nesting teams inside.
thread_local bool g_host_serial = false;

bool representable(double before, double after) {
    return std::isfinite(before) ? std::isfinite(after) && (before == 0 || after != 0)
                                 : before == after;
}

// extra_scale, src/preprocess.cpp:12-65 (reference built with VANTAGE_SPARSE_LU).
//
// Every loop below is element-wise (each row, column or entry is decided and
// scaled from its own values), so the row-, column- and entry-parallel loops
// compute exactly what the sequential ones do.  An entry that cannot take its
// column's factor sets the column's factor to 1; the sequential loop reaches
// the same verdict (once a column's factor is 1 every later entry takes it),
// so the verdicts are gathered per column first and applied after.
//
// The column half is scale_columns.  `colmax` / `colmin` (optional) hold, as
// bit patterns, each column's largest |a| and smallest nonzero |a| of the
// current values; with them the entry verdicts need no pass over the entries:
// rounding is monotone and sign-symmetric, so every finite a of a column has a
// finite a*f iff its largest |a| does, and every nonzero a a nonzero a*f iff its
// smallest nonzero |a| does (all of A's values are finite, Model::validate).
void scale_columns(Prepared &p, std::vector<double> col, const uint64_t *colmax,
                   const uint64_t *colmin);

void extra_scale(Prepared &p, const std::vector<double> &row, std::vector<double> col) {
    HostModel &m = p.model;
    const bool par = m.A.value.size() > 200000 && !g_host_serial;
    // A side whose factors are all 1 changes nothing (x * 1 == x, and every
    // representability test passes), so its loops are skipped.
    const bool rows_one = std::all_of(row.begin(), row.end(), [](double f) { return f == 1; });
#pragma omp parallel for schedule(dynamic, 1024) if (par && !rows_one)
    for (int64_t ii = 0; ii < (rows_one ? 0 : int64_t(row.size())); ii++) {
        const size_t i = size_t(ii);
        double f = row[i];
        bool safe = representable(p.row_scale[i], p.row_scale[i] * f) &&
                    representable(m.rl[i], m.rl[i] * f) && representable(m.ru[i], m.ru[i] * f);
        for (int64_t k = m.A.ptr[i]; k < m.A.ptr[i + 1]; k++)
            safe &= representable(m.A.value[k], m.A.value[k] * f);
        if (!safe)
            continue;
        p.row_scale[i] *= f;
        m.rl[i] *= f;
        m.ru[i] *= f;
        for (int64_t k = m.A.ptr[i]; k < m.A.ptr[i + 1]; k++)
            m.A.value[k] *= f;
    }
    scale_columns(p, std::move(col), nullptr, nullptr);
}

void scale_columns(Prepared &p, std::vector<double> col, const uint64_t *colmax,
                   const uint64_t *colmin) {
    HostModel &m = p.model;
    const bool par = m.A.value.size() > 200000 && !g_host_serial;
    if (std::all_of(col.begin(), col.end(), [](double f) { return f == 1; }))
        return;
#pragma omp parallel for if (par)
    for (int64_t jj = 0; jj < int64_t(col.size()); jj++) {
        const size_t j = size_t(jj);
        double f = col[j];
        if (!representable(p.column_scale[j], p.column_scale[j] * f) ||
            !representable(m.c[j], m.c[j] * f) || !representable(m.q[j], m.q[j] * (f * f)) ||
            !representable(m.lb[j], m.lb[j] / f) || !representable(m.ub[j], m.ub[j] / f))
            col[j] = 1;
    }
    std::vector<unsigned char> refuse(col.size(), 0);
    if (colmax && colmin) {
#pragma omp parallel for if (par)
        for (int64_t jj = 0; jj < int64_t(col.size()); jj++) {
            const size_t j = size_t(jj);
            double hi, lo;
            std::memcpy(&hi, &colmax[j], 8);
            std::memcpy(&lo, &colmin[j], 8);
            const bool any_nonzero = colmin[j] != ~uint64_t(0);
            if (!std::isfinite(hi * col[j]) || (any_nonzero && lo * col[j] == 0))
                refuse[j] = 1;
        }
    } else {
#pragma omp parallel for if (par)
        for (int64_t kk = 0; kk < int64_t(m.A.value.size()); kk++) {
            const size_t k = size_t(kk);
            auto j = m.A.index[k];
            if (!representable(m.A.value[k], m.A.value[k] * col[size_t(j)])) {
#pragma omp atomic write
                refuse[size_t(j)] = 1;
            }
        }
    }
    for (size_t j = 0; j < col.size(); j++)
        if (refuse[j])
            col[j] = 1;
    bool qsafe = true;
    for (int64_t i = 0; i < m.Q.rows; ++i)
        for (auto k = m.Q.ptr[i]; k < m.Q.ptr[i + 1]; ++k)
            qsafe &= representable(m.Q.value[k], (m.Q.value[k] * col[i]) * col[m.Q.index[k]]);
    if (!qsafe)
        std::fill(col.begin(), col.end(), 1);
    for (int64_t i = 0; i < m.Q.rows; ++i)
        for (auto k = m.Q.ptr[i]; k < m.Q.ptr[i + 1]; ++k)
            m.Q.value[k] *= col[i] * col[m.Q.index[k]];
#pragma omp parallel for if (par)
    for (int64_t jj = 0; jj < int64_t(col.size()); jj++) {
        const size_t j = size_t(jj);
        double f = col[j];
        p.column_scale[j] *= f;
        m.c[j] *= f;
        m.q[j] *= f * f;
        m.lb[j] /= f;
        m.ub[j] /= f;
    }
#pragma omp parallel for if (par)
    for (int64_t kk = 0; kk < int64_t(m.A.value.size()); kk++)
        m.A.value[size_t(kk)] *= col[size_t(m.A.index[size_t(kk)])];
}

// One Ruiz pass's row half in one sweep (src/preprocess.cpp:310-319: the row
// norms, the first extra_scale call, then the column norms): each row's
// largest |a| gives its factor clamp(1/sqrt(norm), 1e-3, 1e3) (1 for a row
// without nonzeros), the row is scaled exactly as extra_scale's row loop scales
// it, and the scaled values update the column extremes scale_columns takes --
// largest |a| and smallest nonzero |a|, as bit patterns, which order like
// non-negative values, so the maxima and minima do not depend on the order the
// rows are taken in.  A row whose factor is 1 is left as it is, which is what
// multiplying it by 1 does.
void ruiz_rows(Prepared &p, bool par, std::vector<uint64_t> &colmax,
               std::vector<uint64_t> &colmin) {
    HostModel &m = p.model;
#pragma omp parallel for schedule(dynamic, 1024) if (par)
    for (int64_t ii = 0; ii < int64_t(m.rl.size()); ++ii) {
        const size_t i = size_t(ii);
        const int64_t b = m.A.ptr[i], e = m.A.ptr[i + 1];
        double norm = 0;
        for (auto k = b; k < e; ++k)
            norm = std::max(norm, std::abs(m.A.value[size_t(k)]));
        const double f = norm > 0 ? std::clamp(1 / std::sqrt(norm), 1e-3, 1e3) : 1.;
        if (f != 1) {
            bool safe = representable(p.row_scale[i], p.row_scale[i] * f) &&
                        representable(m.rl[i], m.rl[i] * f) && representable(m.ru[i], m.ru[i] * f);
            for (auto k = b; k < e; k++)
                safe &= representable(m.A.value[size_t(k)], m.A.value[size_t(k)] * f);
            if (safe) {
                p.row_scale[i] *= f;
                m.rl[i] *= f;
                m.ru[i] *= f;
                for (auto k = b; k < e; k++)
                    m.A.value[size_t(k)] *= f;
            }
        }
        for (auto k = b; k < e; ++k) {
            const double v = std::abs(m.A.value[size_t(k)]);
            if (v == 0)
                continue;
            uint64_t bits;
            std::memcpy(&bits, &v, 8);
            const size_t j = size_t(m.A.index[size_t(k)]);
            uint64_t cur = __atomic_load_n(&colmax[j], __ATOMIC_RELAXED);
            while (bits > cur && !__atomic_compare_exchange_n(&colmax[j], &cur, bits, true,
                                                              __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
            }
            cur = __atomic_load_n(&colmin[j], __ATOMIC_RELAXED);
            while (bits < cur && !__atomic_compare_exchange_n(&colmin[j], &cur, bits, true,
                                                              __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
            }
        }
    }
}

double geometric_factor(double low, double high) {
    if (high == 0)
        return 1;
    return std::exp(
        std::clamp(-.5 * (std::log(low) + std::log(high)), std::log(1e-3), std::log(1e3)));
}

// geometric_scale, src/preprocess.cpp:73-101
void geometric_scale(Prepared &p) {
    auto &m = p.model;
    std::vector<double> row(m.rl.size(), 1), col(m.c.size(), 1);
    for (size_t i = 0; i < row.size(); i++) {
        double low = INF, high = 0;
        for (auto k = m.A.ptr[i]; k < m.A.ptr[i + 1]; k++) {
            double v = std::abs(m.A.value[k]);
            if (v > 0) {
                low = std::min(low, v);
                high = std::max(high, v);
            }
        }
        row[i] = geometric_factor(low, high);
    }
    extra_scale(p, row, col);
    std::vector<double> low(col.size(), INF), high(col.size());
    for (size_t k = 0; k < m.A.value.size(); k++) {
        auto j = m.A.index[k];
        double v = std::abs(m.A.value[k]);
        if (v > 0) {
            low[j] = std::min(low[j], v);
            high[j] = std::max(high[j], v);
        }
    }
    for (size_t j = 0; j < col.size(); j++)
        col[j] = geometric_factor(low[j], high[j]);
    std::fill(row.begin(), row.end(), 1);
    extra_scale(p, row, col);
}

// pock_chambolle_scale, src/preprocess.cpp:102-119
void pock_chambolle_scale(Prepared &p) {
    auto &m = p.model;
    std::vector<long double> rows(m.rl.size()), cols(m.c.size());
    for (size_t i = 0; i < rows.size(); i++)
        for (auto k = m.A.ptr[i]; k < m.A.ptr[i + 1]; k++) {
            long double v = std::abs(m.A.value[k]);
            rows[i] += v;
            cols[m.A.index[k]] += v;
        }
    auto factor = [](long double sum) {
        return sum > 0 && std::isfinite(sum) ? double(std::clamp(1 / std::sqrt(sum), 1e-3L, 1e3L))
                                             : 1.;
    };
    std::vector<double> row(rows.size()), col(cols.size());
    std::transform(rows.begin(), rows.end(), row.begin(), factor);
    std::transform(cols.begin(), cols.end(), col.begin(), factor);
    extra_scale(p, row, col);
}

// Hash of row [b, en) of A as a duplicate-row key (its mapped columns and
// values, in order; FNV-1a over their bits), without building the key.  The
// reference keys a std::map on the same (column, value) vectors; a hash bucket
// is only a shortlist here, the keys themselves are compared by same_row_key,
// so equal keys are found alike.
// `map` null: the identity (no column removed).
uint64_t row_key_hash(const Csr &A, const int64_t *map, int64_t b, int64_t en) {
    uint64_t h = 1469598103934665603ULL;
    for (auto k = b; k < en; ++k) {
        uint64_t bits;
        std::memcpy(&bits, &A.value[size_t(k)], 8);
        const int64_t j = A.index[size_t(k)];
        h = (h ^ uint64_t(map ? map[j] : j)) * 1099511628211ULL;
        h = (h ^ bits) * 1099511628211ULL;
    }
    return h;
}

// Equal keys (mapped columns and values, in order) of source rows a and b --
// the equality the reference's std::map of key vectors applies.
bool same_row_key(const Csr &A, const int64_t *map, int64_t a, int64_t b) {
    const int64_t ba = A.ptr[size_t(a)], ea = A.ptr[size_t(a + 1)];
    const int64_t bb = A.ptr[size_t(b)], eb = A.ptr[size_t(b + 1)];
    if (ea - ba != eb - bb)
        return false;
    for (int64_t t = 0; t < ea - ba; ++t) {
        const int64_t ja = A.index[size_t(ba + t)], jb = A.index[size_t(bb + t)];
        if ((map ? map[ja] : ja) != (map ? map[jb] : jb) ||
            !(A.value[size_t(ba + t)] == A.value[size_t(bb + t)]))
            return false;
    }
    return true;
}
} // namespace

// Sparse::build for entries that are already unique: sort (row, col), drop zeros.
Csr build_csr(int64_t rows, int64_t cols, std::vector<Entry> e) {
    auto before = [](const Entry &a, const Entry &b) {
        return a.row < b.row || (a.row == b.row && a.col < b.col);
    };
    // Entries in strictly increasing (row, col) order -- the usual case, a CSR
    // restricted to kept rows and columns -- have exactly one sorted order, so
    // the sort is skipped; otherwise std::sort as in Sparse::build.
    bool sorted = true;
    for (size_t k = 1; k < e.size() && sorted; ++k)
        sorted = before(e[k - 1], e[k]);
    if (!sorted)
        std::sort(e.begin(), e.end(), before);
    Csr s;
    s.rows = rows;
    s.cols = cols;
    s.ptr.assign(size_t(rows + 1), 0);
    s.index.reserve(e.size());
    s.value.reserve(e.size());
    for (size_t k = 0; k < e.size();) {
        auto a = e[k++];
        while (k < e.size() && e[k].row == a.row && e[k].col == a.col)
            a.value += e[k++].value;
        if (!std::isfinite(a.value))
            throw std::runtime_error("Coefficient sum overflow");
        if (a.value != 0) {
            s.ptr[size_t(a.row + 1)]++;
            s.index.push_back(a.col);
            s.value.push_back(a.value);
        }
    }
    for (int64_t i = 0; i < rows; i++)
        s.ptr[size_t(i + 1)] += s.ptr[size_t(i)];
    return s;
}

// Transpose with each column's entries in increasing row order (the order of
// a sequential row sweep).  Large matrices are swept by contiguous row blocks
// in parallel: block b places its entries of column j after those of blocks
// before it, so the result is the sequential one entry for entry.
void validate_entries(const HostModel &m) {
    const int64_t n = int64_t(m.c.size()), nnz = int64_t(m.A.value.size());
    int bad = 0;
#pragma omp parallel for reduction(max : bad) if (nnz > 200000 && !g_host_serial)
    for (int64_t k = 0; k < nnz; ++k)
        if (m.A.index[size_t(k)] < 0 || m.A.index[size_t(k)] >= n ||
            !std::isfinite(m.A.value[size_t(k)]))
            bad = 1;
    if (bad)
        throw std::runtime_error("Invalid matrix coefficient/index");
    if (m.Q.value.empty())
        return;
    for (int64_t i = 0; i < m.Q.rows; ++i) {
        int64_t previous = -1;
        for (auto k = m.Q.ptr[size_t(i)]; k < m.Q.ptr[size_t(i + 1)]; ++k) {
            const int64_t j = m.Q.index[size_t(k)];
            if (j <= previous || j >= n || !std::isfinite(m.Q.value[size_t(k)]))
                throw std::runtime_error("Invalid quadratic coefficient/index");
            previous = j;
        }
    }
    const Csr t = transpose(m.Q);
    if (t.ptr != m.Q.ptr || t.index != m.Q.index || t.value != m.Q.value)
        throw std::runtime_error("Quadratic matrix must be exactly symmetric");
}

Csr transpose(const Csr &a) {
    Csr t;
    t.rows = a.cols;
    t.cols = a.rows;
    t.ptr.assign(size_t(a.cols + 1), 0);
    t.index.resize(a.value.size());
    t.value.resize(a.value.size());
    const size_t nnz = a.value.size();
    const int blocks = omp_get_max_threads();
    if (nnz > (1u << 20) && nnz < (size_t(1) << 32) && blocks > 1 && !g_host_serial &&
        a.cols < (int64_t(1) << 31)) {
        const size_t cols = size_t(a.cols);
        std::vector<int64_t> first(size_t(blocks) + 1);
        for (int b = 0; b <= blocks; ++b) // row blocks of about equal entry counts
            first[size_t(b)] = int64_t(std::lower_bound(a.ptr.begin(), a.ptr.end(),
                                                        int64_t(nnz * size_t(b) / size_t(blocks))) -
                                       a.ptr.begin());
        first[size_t(blocks)] = a.rows;
        std::vector<uint32_t> count(size_t(blocks) * cols, 0);
#pragma omp parallel for num_threads(blocks) schedule(static, 1)
        for (int b = 0; b < blocks; ++b) {
            uint32_t *mine = count.data() + size_t(b) * cols;
            for (auto k = a.ptr[size_t(first[size_t(b)])]; k < a.ptr[size_t(first[size_t(b + 1)])];
                 ++k)
                ++mine[size_t(a.index[size_t(k)])];
        }
        // column lengths, column offsets, then each block's start inside each column
#pragma omp parallel for num_threads(blocks)
        for (int64_t jj = 0; jj < int64_t(cols); ++jj) {
            int64_t total = 0;
            for (int b = 0; b < blocks; ++b)
                total += count[size_t(b) * cols + size_t(jj)];
            t.ptr[size_t(jj) + 1] = total;
        }
        for (size_t j = 0; j < cols; ++j)
            t.ptr[j + 1] += t.ptr[j];
#pragma omp parallel for num_threads(blocks)
        for (int64_t jj = 0; jj < int64_t(cols); ++jj) {
            uint32_t run = 0;
            for (int b = 0; b < blocks; ++b) {
                const uint32_t c = count[size_t(b) * cols + size_t(jj)];
                count[size_t(b) * cols + size_t(jj)] = run;
                run += c;
            }
        }
#pragma omp parallel for num_threads(blocks) schedule(static, 1)
        for (int b = 0; b < blocks; ++b) {
            uint32_t *at = count.data() + size_t(b) * cols;
            for (int64_t i = first[size_t(b)]; i < first[size_t(b + 1)]; ++i)
                for (auto k = a.ptr[size_t(i)]; k < a.ptr[size_t(i + 1)]; ++k) {
                    const size_t j = size_t(a.index[size_t(k)]);
                    const size_t p = size_t(t.ptr[j]) + at[j]++;
                    t.index[p] = i;
                    t.value[p] = a.value[size_t(k)];
                }
        }
        return t;
    }
    for (auto j : a.index)
        t.ptr[size_t(j + 1)]++;
    for (int64_t j = 0; j < a.cols; j++)
        t.ptr[size_t(j + 1)] += t.ptr[size_t(j)];
    auto pos = t.ptr;
    for (int64_t i = 0; i < a.rows; i++)
        for (auto k = a.ptr[size_t(i)]; k < a.ptr[size_t(i + 1)]; k++) {
            auto p = pos[size_t(a.index[size_t(k)])]++;
            t.index[size_t(p)] = i;
            t.value[size_t(p)] = a.value[size_t(k)];
        }
    return t;
}

// prepare, src/preprocess.cpp:133-346 (host presolve; no GPU compaction)
Prepared prepare(const HostModel &src, const PrepareOptions &o) {
    Prepared p;
    const int64_t n = int64_t(src.c.size()), mrows = int64_t(src.rl.size());
    p.fixed.assign(size_t(n), 0);
    HostModel &m = p.model;
    m.offset = src.offset;
    std::vector<int64_t> map(size_t(n), -1);
    std::vector<bool> used(size_t(n), false);
    for (auto j : src.A.index)
        used[size_t(j)] = true;
    for (auto j : src.Q.index)
        used[size_t(j)] = true;
    for (int64_t i = 0; i < src.Q.rows; ++i)
        if (src.Q.ptr[size_t(i)] != src.Q.ptr[size_t(i + 1)])
            used[size_t(i)] = true;
    for (int64_t j = 0; j < n; j++) {
        double chosen = src.lb[j];
        bool removable = src.lb[j] == src.ub[j];
        if (!used[size_t(j)]) {
            chosen = src.q[j] > 0   ? std::clamp(-src.c[j] / src.q[j], src.lb[j], src.ub[j])
                     : src.c[j] > 0 ? src.lb[j]
                     : src.c[j] < 0 ? src.ub[j]
                                    : std::clamp(0., src.lb[j], src.ub[j]);
            removable = std::isfinite(chosen);
        }
        if (o.presolve && removable) {
            p.fixed[size_t(j)] = chosen;
            m.offset += src.c[j] * chosen + .5 * src.q[j] * chosen * chosen;
        } else {
            map[size_t(j)] = int64_t(p.cols.size());
            p.cols.push_back(j);
            m.c.push_back(src.c[j]);
            m.q.push_back(src.q[j]);
            m.lb.push_back(src.lb[j]);
            m.ub.push_back(src.ub[j]);
        }
    }
    std::vector<Entry> qe;
    for (int64_t i = 0; i < src.Q.rows; ++i)
        for (auto k = src.Q.ptr[size_t(i)]; k < src.Q.ptr[size_t(i + 1)]; ++k) {
            auto j = src.Q.index[size_t(k)];
            auto v = src.Q.value[size_t(k)];
            if (map[size_t(i)] >= 0 && map[size_t(j)] >= 0)
                qe.push_back({map[size_t(i)], map[size_t(j)], v});
            else if (map[size_t(i)] >= 0)
                m.c[size_t(map[size_t(i)])] += v * p.fixed[size_t(j)];
            else if (map[size_t(j)] < 0)
                m.offset += .5 * v * p.fixed[size_t(i)] * p.fixed[size_t(j)];
        }
    const int64_t nk = int64_t(m.c.size());
    m.Q = build_csr(nk, nk, std::move(qe));
    // No column removed: kept columns are numbered in order, so map[j] == j
    // and no entry has a fixed-column shift; the loops below skip the map.
    const bool identity = nk == n;
    const int64_t *key_map = identity ? nullptr : map.data();
    // Rows in two passes.  The first, row-parallel, does each row's own
    // arithmetic exactly as the reference's loop does (same operations, same
    // order within the row): fixed-column shift, activity bounds, and the
    // verdict (infeasible, dropped, or kept with bounds l, u), plus the hash of
    // the row's key for duplicate detection.  The second walks the rows in
    // order, so the first failure, the first occurrence of a duplicate key and
    // the emitted order are the reference's.
    enum : char { KEEP = 0, DROP = 1, FAIL_EMPTY = 2, FAIL_DISJOINT = 3 };
    std::vector<char> verdict(size_t(mrows), KEEP), dupcand(size_t(mrows), 0);
    std::vector<double> row_l(static_cast<size_t>(mrows)), row_u(static_cast<size_t>(mrows));
    std::vector<uint64_t> key_hash(size_t(mrows), 0);
    std::vector<int64_t> kept_in_row(size_t(mrows), 0); // entries in kept columns
    const long double eps = std::numeric_limits<long double>::epsilon();
#pragma omp parallel for schedule(dynamic, 1024) if (src.A.value.size() > 200000 && !g_host_serial)
    for (int64_t i = 0; i < mrows; i++) {
        long double shift = 0, shift_magnitude = 0;
        int64_t count = 0;
        const int64_t b = src.A.ptr[size_t(i)], en = src.A.ptr[size_t(i + 1)];
        if (identity)
            count = en - b;
        else
            for (auto k = b; k < en; k++) {
                auto j = src.A.index[size_t(k)];
                if (map[size_t(j)] < 0) {
                    long double term = (long double)src.A.value[size_t(k)] * p.fixed[size_t(j)];
                    shift += term;
                    shift_magnitude += std::abs(term);
                } else
                    count++;
            }
        kept_in_row[size_t(i)] = count;
        double l = src.rl[i] - double(shift), u = src.ru[i] - double(shift);
        row_l[size_t(i)] = l;
        row_u[size_t(i)] = u;
        if (count == 0 && o.presolve) {
            long double guard = 8 * eps * (en - b + 1) * (1 + shift_magnitude);
            if (shift + guard < src.rl[i] || shift - guard > src.ru[i]) {
                verdict[size_t(i)] = FAIL_EMPTY;
                continue;
            }
            if (l <= 0 && u >= 0) {
                verdict[size_t(i)] = DROP;
                continue;
            }
        }
        // Activity bounds.  A column with an infinite bound makes amin or amax
        // infinite or NaN (for either sign of v), an infinite or NaN sum stays
        // so, and the verdicts below use the bounds only when both are finite:
        // such a row's verdict is settled at that column, so the sum stops
        // there.  (Carrying long double infinities through the rest of every
        // such row took most of prepare's time on models with free columns.)
        long double amin = 0, amax = 0, magnitude = 0;
        for (auto k = b; k < en; k++) {
            auto j = src.A.index[size_t(k)];
            double v = src.A.value[size_t(k)];
            if (!std::isfinite(src.lb[j]) || !std::isfinite(src.ub[j])) {
                amin = -std::numeric_limits<long double>::infinity();
                break;
            }
            amin += (long double)v * (v > 0 ? src.lb[j] : src.ub[j]);
            amax += (long double)v * (v > 0 ? src.ub[j] : src.lb[j]);
            magnitude += std::abs((long double)v * (v > 0 ? src.lb[j] : src.ub[j])) +
                         std::abs((long double)v * (v > 0 ? src.ub[j] : src.lb[j]));
        }
        if (o.presolve) {
            long double slack = 8 * eps * (en - b + 1) * (1 + magnitude);
            if (std::isfinite(amin) && std::isfinite(amax) &&
                (amin > src.ru[i] + slack || amax < src.rl[i] - slack)) {
                verdict[size_t(i)] = FAIL_DISJOINT;
                continue;
            }
        }
        if (o.presolve && std::isfinite(amin) && std::isfinite(amax)) {
            long double guard = 8 * eps * (en - b + 1) * (1 + magnitude);
            if (amin - guard >= src.rl[i] && amax + guard <= src.ru[i]) {
                verdict[size_t(i)] = DROP;
                continue;
            }
        }
        if (o.presolve && count == en - b) {
            dupcand[size_t(i)] = 1;
            key_hash[size_t(i)] = row_key_hash(src.A, key_map, b, en);
        }
    }
    // first occurrence (prepared row) of each key, by hash; keys are compared in
    // full.  An open-addressing table (linear probing, at most half full): a
    // lookup visits every stored row whose hash is equal before it reaches an
    // empty slot, where a new key goes.
    size_t slots = 16;
    while (slots < 2 * size_t(mrows))
        slots *= 2;
    std::vector<uint64_t> slot_hash(slots);
    std::vector<size_t> slot_row(slots, ~size_t(0));
    size_t kept_entries = 0;
    for (int64_t i = 0; i < mrows; i++) {
        const char v = verdict[size_t(i)];
        if (v == FAIL_EMPTY) {
            p.failure = "INFEASIBLE";
            p.reason = "Empty row after fixed-variable substitution: r" + std::to_string(i);
            return p;
        }
        if (v == FAIL_DISJOINT) {
            p.failure = "INFEASIBLE";
            p.reason = "Verified disjoint row activity bounds: r" + std::to_string(i);
            return p;
        }
        if (v == DROP)
            continue;
        const double l = row_l[size_t(i)], u = row_u[size_t(i)];
        if (dupcand[size_t(i)]) {
            const uint64_t h = key_hash[size_t(i)];
            bool merged = false;
            size_t slot = size_t(h) & (slots - 1);
            for (; slot_row[slot] != ~size_t(0); slot = (slot + 1) & (slots - 1)) {
                if (slot_hash[slot] != h)
                    continue;
                const size_t r = slot_row[slot];
                if (!same_row_key(src.A, key_map, p.rows[r], i))
                    continue;
                if (l > m.rl[r]) {
                    m.rl[r] = l;
                    p.lower_rows[r] = i;
                }
                if (u < m.ru[r]) {
                    m.ru[r] = u;
                    p.upper_rows[r] = i;
                }
                if (m.rl[r] > m.ru[r]) {
                    p.failure = "INFEASIBLE";
                    p.reason = "Disjoint bounds on identical constraint rows";
                    p.failure_ray.assign(size_t(mrows), 0);
                    p.failure_ray[size_t(p.lower_rows[r])] = -1;
                    p.failure_ray[size_t(p.upper_rows[r])] += 1;
                    if (!(Verifier(src).infeasibility_bound(p.failure_ray) > 0))
                        p.failure_ray.clear();
                    return p;
                }
                merged = true;
                break;
            }
            if (merged)
                continue;
            slot_hash[slot] = h;
            slot_row[slot] = p.rows.size();
        }
        p.rows.push_back(i);
        p.lower_rows.push_back(i);
        p.upper_rows.push_back(i);
        m.rl.push_back(l);
        m.ru.push_back(u);
        kept_entries += size_t(kept_in_row[size_t(i)]);
    }
    // The kept entries.  When every kept row's columns strictly increase (a
    // canonical CSR: the map keeps column order), Sparse::build would only drop
    // zero values, so the CSR is written directly, rows in parallel; otherwise
    // the entries go through build_csr (sort, merge, drop zeros).
    const int64_t kept_rows = int64_t(p.rows.size());
    std::vector<int64_t> row_len(static_cast<size_t>(kept_rows), 0);
    int canonical = 1;
#pragma omp parallel for reduction(min : canonical) if (kept_entries > 200000 && !g_host_serial)
    for (int64_t r = 0; r < kept_rows; ++r) {
        const int64_t i = p.rows[size_t(r)];
        int64_t last = -1, len = 0;
        for (auto k = src.A.ptr[size_t(i)]; k < src.A.ptr[size_t(i + 1)]; k++) {
            const int64_t source = src.A.index[size_t(k)];
            const int64_t j = identity ? source : map[size_t(source)];
            if (j < 0)
                continue;
            if (j <= last)
                canonical = 0;
            last = j;
            len += src.A.value[size_t(k)] != 0;
        }
        row_len[size_t(r)] = len;
    }
    if (canonical) {
        Csr &A = m.A;
        A.rows = kept_rows;
        A.cols = nk;
        A.ptr.assign(size_t(kept_rows + 1), 0);
        for (int64_t r = 0; r < kept_rows; ++r)
            A.ptr[size_t(r + 1)] = A.ptr[size_t(r)] + row_len[size_t(r)];
        A.index.resize(size_t(A.ptr.back()));
        A.value.resize(size_t(A.ptr.back()));
#pragma omp parallel for if (kept_entries > 200000 && !g_host_serial)
        for (int64_t r = 0; r < kept_rows; ++r) {
            const int64_t i = p.rows[size_t(r)];
            int64_t at = A.ptr[size_t(r)];
            for (auto k = src.A.ptr[size_t(i)]; k < src.A.ptr[size_t(i + 1)]; k++) {
                const int64_t source = src.A.index[size_t(k)];
                const int64_t j = identity ? source : map[size_t(source)];
                if (j >= 0 && src.A.value[size_t(k)] != 0) {
                    A.index[size_t(at)] = j;
                    A.value[size_t(at++)] = src.A.value[size_t(k)];
                }
            }
        }
    } else {
        std::vector<Entry> e;
        e.reserve(kept_entries);
        for (size_t r = 0; r < p.rows.size(); ++r) {
            const int64_t i = p.rows[r];
            for (auto k = src.A.ptr[size_t(i)]; k < src.A.ptr[size_t(i + 1)]; k++)
                if (map[size_t(src.A.index[size_t(k)])] >= 0)
                    e.push_back({int64_t(r), map[size_t(src.A.index[size_t(k)])],
                                 src.A.value[size_t(k)]});
        }
        m.A = build_csr(int64_t(m.rl.size()), nk, std::move(e));
    }
    p.column_scale.assign(size_t(nk), 1);
    p.row_scale.assign(m.rl.size(), 1);
    if (o.scaling == "combined" && o.scaling_passes > 0)
        geometric_scale(p);
    // Ruiz passes (src/preprocess.cpp:306-323): the row half and the column
    // norms in one sweep (ruiz_rows), then the column half (scale_columns)
    const bool par = m.A.value.size() > 200000 && !g_host_serial;
    for (int pass = 0; pass < o.scaling_passes; pass++) {
        std::vector<uint64_t> colmax(m.c.size(), 0), colmin(m.c.size(), ~uint64_t(0));
        ruiz_rows(p, par, colmax, colmin);
        std::vector<double> col(m.c.size());
#pragma omp parallel for if (par)
        for (int64_t jj = 0; jj < int64_t(col.size()); ++jj) {
            const size_t j = size_t(jj);
            double norm;
            std::memcpy(&norm, &colmax[j], 8);
            col[j] = norm > 0 ? std::clamp(1 / std::sqrt(norm), 1e-3, 1e3) : 1.;
        }
        scale_columns(p, std::move(col), colmax.data(), colmin.data());
    }
    if (o.scaling == "combined" && o.scaling_passes > 0)
        pock_chambolle_scale(p);
    if (o.scaling_passes > 0) {
        double cnorm = 0;
        for (auto c : m.c)
            cnorm = std::max(cnorm, std::abs(c));
        for (auto q : m.q)
            cnorm = std::max(cnorm, std::abs(q));
        for (auto q : m.Q.value)
            cnorm = std::max(cnorm, std::abs(q));
        p.objective_scale = cnorm > 0 ? cnorm : 1;
        for (auto &c : m.c)
            c /= p.objective_scale;
        for (auto &q : m.q)
            q /= p.objective_scale;
        for (auto &q : m.Q.value)
            q /= p.objective_scale;
        m.offset /= p.objective_scale;
    }
    return p;
}

std::vector<double> Prepared::restore_x(const std::vector<double> &x) const {
    auto out = fixed;
    for (size_t j = 0; j < cols.size(); j++)
        out[size_t(cols[j])] = x[j] * column_scale[j];
    return out;
}
std::vector<double> Prepared::restore_y(const std::vector<double> &y, size_t n) const {
    std::vector<double> out(n);
    for (size_t i = 0; i < rows.size(); i++)
        out[size_t(y[i] >= 0 ? upper_rows[i] : lower_rows[i])] += y[i] * row_scale[i] * objective_scale;
    return out;
}

// ------------------------------------------------------------------ verifier
namespace {
long double down(long double v) { return std::nextafter(v, -std::numeric_limits<long double>::infinity()); }
long double up(long double v) { return std::nextafter(v, std::numeric_limits<long double>::infinity()); }
bool has_q(const HostModel &m) { return !m.Q.value.empty(); }

std::vector<double> multiply(const Csr &a, const std::vector<double> &x) {
    std::vector<double> y(size_t(a.rows));
#pragma omp parallel for if (a.rows > 10000 && !g_host_serial)
    for (int64_t i = 0; i < a.rows; i++) {
        double v = 0;
        for (auto k = a.ptr[size_t(i)]; k < a.ptr[size_t(i + 1)]; k++)
            v += a.value[size_t(k)] * x[size_t(a.index[size_t(k)])];
        y[size_t(i)] = v;
    }
    return y;
}

// lp_lower_bound, src/verify.cpp:12-88
double lp_lower_bound(const HostModel &m, const Csr &at, const std::vector<double> &y,
                      bool feasibility, const std::vector<double> *point) {
    long double lower = feasibility ? 0 : m.offset;
    const size_t n = m.c.size();
    if (point) {
        for (size_t i = 0; i < n; ++i) {
            long double square = up((long double)(*point)[i] * (*point)[i]);
            if (m.q[i] != 0) {
                long double lo = down((long double)(*point)[i] * (*point)[i]);
                long double term = m.q[i] >= 0 ? up(m.q[i] * square) : up(m.q[i] * lo);
                lower = down(lower - up(.5L * term));
            }
            if (has_q(m))
                for (auto k = m.Q.ptr[i]; k < m.Q.ptr[i + 1]; ++k) {
                    auto j = size_t(m.Q.index[size_t(k)]);
                    long double v = m.Q.value[size_t(k)];
                    long double lo = down((long double)(*point)[i] * (*point)[j]);
                    long double hi = up((long double)(*point)[i] * (*point)[j]);
                    long double term = up(v * (v >= 0 ? hi : lo));
                    lower = down(lower - up(.5L * term));
                }
        }
    }
    for (size_t i = 0; i < y.size(); i++)
        if (y[i] != 0) {
            double b = y[i] > 0 ? m.ru[i] : m.rl[i];
            if (!std::isfinite(b))
                return -INF;
            if (b == 0)
                continue;
            long double term = (long double)y[i] * b;
            lower = down(lower - up(term));
        }
    for (size_t j = 0; j < n; j++) {
        long double gl = feasibility ? 0 : m.c[j], gu = gl;
        if (point) {
            auto add = [&](double coefficient, double value) {
                if (coefficient == 0 || value == 0)
                    return;
                long double term = (long double)coefficient * value;
                gl = down(gl + down(term));
                gu = up(gu + up(term));
            };
            add(m.q[j], (*point)[j]);
            if (has_q(m))
                for (auto k = m.Q.ptr[j]; k < m.Q.ptr[j + 1]; ++k)
                    add(m.Q.value[size_t(k)], (*point)[size_t(m.Q.index[size_t(k)])]);
        }
        for (auto k = at.ptr[j]; k < at.ptr[j + 1]; k++)
            if (y[size_t(at.index[size_t(k)])] != 0 && at.value[size_t(k)] != 0) {
                long double v = (long double)at.value[size_t(k)] * y[size_t(at.index[size_t(k)])];
                gl = down(gl + down(v));
                gu = up(gu + up(v));
            }
        if ((!std::isfinite(m.lb[j]) && gu > 0) || (!std::isfinite(m.ub[j]) && gl < 0))
            return -INF;
        long double term = std::numeric_limits<long double>::infinity();
        if (gl <= 0 && gu >= 0)
            term = 0;
        for (double b : {m.lb[j], m.ub[j]})
            if (std::isfinite(b)) {
                term = std::min(term, (b == 0 || gl == 0) ? 0 : down(gl * b));
                term = std::min(term, (b == 0 || gu == 0) ? 0 : down(gu * b));
            }
        if (gl == 0 && gu == 0)
            term = 0;
        if (!std::isfinite(term))
            return -INF;
        if (term != 0)
            lower = down(lower + term);
    }
    double result = double(lower);
    if (!std::isfinite(result))
        return -INF;
    return std::nextafter(result, -INF);
}
} // namespace

void host_serial(bool serial) { g_host_serial = serial; }
bool host_serial_enabled() { return g_host_serial; }

bool HostModel::is_qp() const {
    return !Q.value.empty() || std::any_of(q.begin(), q.end(), [](double v) { return v != 0; });
}

Verifier::Verifier(const HostModel &m) : m_(m), at_(transpose(m.A)) {}

// Verifier::infeasibility_bound, src/verify.cpp:93-101
double Verifier::infeasibility_bound(const std::vector<double> &y) const {
    if (y.size() != m_.rl.size())
        return -INF;
    for (auto v : y)
        if (!std::isfinite(v))
            return -INF;
    return lp_lower_bound(m_, at_, y, true, nullptr);
}

// Verifier::evaluate, src/verify.cpp:103-240
Accuracy Verifier::evaluate(const std::vector<double> &x, const std::vector<double> &y,
                            bool safe_bound) const {
    const HostModel &m = m_;
    const Csr &at = at_;
    Accuracy a;
    if (x.size() != m.c.size() || y.size() != m.rl.size())
        return a;
    for (auto v : x)
        if (!std::isfinite(v))
            return a;
    for (auto v : y)
        if (!std::isfinite(v))
            return a;
    auto ax = multiply(m.A, x);
    auto aty = multiply(at, y);
    for (auto v : ax)
        if (!std::isfinite(v))
            return Accuracy{};
    for (auto v : aty)
        if (!std::isfinite(v))
            return Accuracy{};
    a.objective = m.offset;
    a.primal = a.dual = 0;
    a.primal_absolute = a.dual_absolute = 0;
    long double support = 0, box_min = 0, complement = 0;
    bool bound_ok = true;
    for (size_t i = 0; i < y.size(); i++) {
        double v = std::max({0., m.rl[i] - ax[i], ax[i] - m.ru[i]});
        if (std::isfinite(m.rl[i]))
            a.primal = std::max(a.primal, std::max(0., m.rl[i] - ax[i]) / (1 + std::abs(m.rl[i])));
        if (std::isfinite(m.ru[i]))
            a.primal = std::max(a.primal, std::max(0., ax[i] - m.ru[i]) / (1 + std::abs(m.ru[i])));
        a.primal_absolute = std::max(a.primal_absolute, v);
        double endpoint = y[i] > 0 ? m.ru[i] : m.rl[i];
        if (y[i] != 0) {
            if (std::isfinite(endpoint)) {
                support += (long double)y[i] * endpoint;
                complement += std::abs((long double)y[i] * (endpoint - ax[i]));
            } else {
                bound_ok = false;
                a.dual_absolute = std::max(a.dual_absolute, std::abs(y[i]));
                a.dual = std::max(a.dual, std::abs(y[i]));
            }
        }
    }
    auto qx = has_q(m) ? multiply(m.Q, x) : std::vector<double>(x.size(), 0);
    double cscale = 1;
    for (auto v : m.c)
        cscale = std::max(cscale, 1 + std::abs(v));
    for (size_t j = 0; j < x.size(); j++) {
        double v = std::max({0., m.lb[j] - x[j], x[j] - m.ub[j]});
        double bs = 1 + std::abs(x[j]);
        a.primal = std::max(a.primal, v / bs);
        a.primal_absolute = std::max(a.primal_absolute, v);
        a.objective += m.c[j] * x[j] + .5 * m.q[j] * x[j] * x[j] + .5 * x[j] * qx[j];
        double linear = m.c[j] + aty[j], g = linear + m.q[j] * x[j] + qx[j];
        if (!std::isfinite(linear) || !std::isfinite(g))
            return Accuracy{};
        double d = std::clamp(g, x[j] - m.ub[j], x[j] - m.lb[j]);
        a.dual_absolute = std::max(a.dual_absolute, std::abs(d));
        a.dual = std::max(a.dual, std::abs(d) / cscale);
        if (g > 0 && std::isfinite(m.lb[j]))
            complement += std::abs((long double)g * (x[j] - m.lb[j]));
        if (g < 0 && std::isfinite(m.ub[j]))
            complement += std::abs((long double)g * (m.ub[j] - x[j]));
        if (has_q(m)) {
            double arg = g > 0 ? m.lb[j] : g < 0 ? m.ub[j] : std::clamp(0., m.lb[j], m.ub[j]);
            if (!std::isfinite(arg))
                bound_ok = false;
            else
                box_min += (long double)g * arg - (long double)(m.q[j] * x[j] + qx[j]) * x[j] / 2;
            continue;
        }
        double arg = 0;
        if (m.q[j] > 0)
            arg = std::clamp(-linear / m.q[j], m.lb[j], m.ub[j]);
        else if (linear > 0)
            arg = m.lb[j];
        else if (linear < 0)
            arg = m.ub[j];
        else
            arg = std::clamp(0., m.lb[j], m.ub[j]);
        if (!std::isfinite(arg))
            bound_ok = false;
        else
            box_min += (long double)linear * arg + .5L * m.q[j] * arg * arg;
    }
    a.complementarity = double(complement);
    a.gap = a.complementarity / (1 + std::abs(a.objective - m.offset));
    if (bound_ok) {
        long double lower = (long double)m.offset - support + box_min;
        long double guard = 64 * std::numeric_limits<double>::epsilon() *
                            (1 + std::abs((long double)m.offset) + std::abs(support) +
                             std::abs(box_min));
        a.lower_bound = double(lower - guard);
        a.gap = std::max(a.gap, std::abs(a.objective - a.lower_bound) /
                                    (1 + std::abs(a.objective) + std::abs(a.lower_bound)));
    }
    if (safe_bound)
        a.lower_bound = lp_lower_bound(m, at, y, false, m.is_qp() ? &x : nullptr);
    else if (!m.is_qp())
        a.lower_bound = -INF;
    if (std::isfinite(a.lower_bound))
        a.gap = std::max(a.gap, std::abs(a.objective - a.lower_bound) /
                                    (1 + std::abs(a.objective) + std::abs(a.lower_bound)));
    a.kkt = std::max({a.primal, a.dual, a.gap});
    a.finite = std::isfinite(a.objective) && std::isfinite(a.kkt) && std::isfinite(a.gap) &&
               std::isfinite(a.primal) && std::isfinite(a.dual);
    if (!a.finite) {
        a.kkt = INF;
        a.lower_bound = -INF;
    }
    return a;
}

} // namespace nk
