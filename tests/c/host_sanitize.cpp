// The engine's host stages under AddressSanitizer and UndefinedBehaviorSanitizer
// (the reference's CI runs its host code the same way, its VANTAGE_SANITIZE
// option).  Built by tests/test_host_sanitize.py from the library's host
// sources; each argument is a model file, loaded through nk_model_open and then
// put through the entry checks, every prepare option set, restore_x/restore_y,
// and the verifier (evaluate with and without the safe bound, and the
// infeasibility bound).  Any sanitizer report ends the process with an error.
#include "nk_host.hpp"
#include "nk_pdhg.h"

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

// nk_modelfile.cpp reports through the library's error slot, which lives in the
// CUDA translation unit; here it goes to stderr.
namespace nk {
void set_last_error(const char *what) { std::fprintf(stderr, "library error: %s\n", what); }
} // namespace nk

namespace {
nk::Csr copy_csr(const nk_csr &c) {
    nk::Csr out;
    out.rows = c.rows;
    out.cols = c.cols;
    out.ptr.assign(c.ptr, c.ptr + c.rows + 1);
    out.index.assign(c.index, c.index + c.ptr[c.rows]);
    out.value.assign(c.value, c.value + c.ptr[c.rows]);
    return out;
}

int run(const char *path) {
    nk_model_file *file = nullptr;
    nk_model v;
    int maximise = 0;
    if (nk_model_open(path, &file, &v, &maximise) != NK_OK)
        return 1;
    const size_t n = size_t(v.A.cols), m = size_t(v.A.rows);
    nk::HostModel hm;
    hm.A = copy_csr(v.A);
    if (v.Q.rows > 0) {
        hm.Q = copy_csr(v.Q);
    } else {
        hm.Q.rows = hm.Q.cols = int64_t(n);
        hm.Q.ptr.assign(n + 1, 0);
    }
    hm.c.assign(v.c, v.c + n);
    hm.q.assign(v.q, v.q + n);
    hm.lb.assign(v.lb, v.lb + n);
    hm.ub.assign(v.ub, v.ub + n);
    hm.rl.assign(v.rl, v.rl + m);
    hm.ru.assign(v.ru, v.ru + m);
    hm.offset = v.offset;
    nk_model_close(file);

    nk::validate_entries(hm);
    int prepared = 0;
    for (bool presolve : {true, false})
        for (const char *scaling : {"ruiz", "combined"})
            for (int passes : {0, 5}) {
                nk::PrepareOptions o;
                o.presolve = presolve;
                o.scaling = scaling;
                o.scaling_passes = passes;
                nk::Prepared p = nk::prepare(hm, o);
                if (!p.failure.empty())
                    continue;
                ++prepared;
                std::vector<double> x(p.model.c.size(), 0.5), y(p.model.rl.size(), -0.25);
                auto ox = p.restore_x(x);
                auto oy = p.restore_y(y, m);
                if (ox.size() != n || oy.size() != m)
                    throw std::runtime_error("restored sizes");
            }
    nk::Verifier verifier(hm);
    std::vector<double> x(n), y(m);
    for (size_t j = 0; j < n; ++j)
        x[j] = std::min(std::max(0.25, hm.lb[j]), hm.ub[j]);
    for (size_t i = 0; i < m; ++i)
        y[i] = (i % 3 == 0) ? 0.5 : (i % 3 == 1 ? -0.5 : 0.0);
    auto a = verifier.evaluate(x, y, true);
    auto b = verifier.evaluate(x, y, false);
    double bound = verifier.infeasibility_bound(y);
    std::printf("%s: prepared %d of 8 option sets; kkt %.6g / %.6g; ray bound %.6g\n", path,
                prepared, a.kkt, b.kkt, bound);
    return 0;
}
} // namespace

int main(int argc, char **argv) {
    for (int k = 1; k < argc; ++k) {
        try {
            if (run(argv[k]) != 0)
                return 1;
        } catch (const std::exception &e) {
            std::fprintf(stderr, "%s: %s\n", argv[k], e.what());
            return 1;
        }
    }
    return 0;
}
