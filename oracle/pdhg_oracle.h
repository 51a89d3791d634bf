/* Test infrastructure only -- the oracle.
 *
 * A plain-C restatement of the reference's CPU PDHG path, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg to check the CUDA
 * engine.  It is never linked into, called by, or shipped with the engine.
 *
 * Restated (reference paths):
 *   orc_transpose / orc_spmv     src/model.cpp:39-73   (Sparse::transpose, Sparse::multiply)
 *   orc_quadratic_norm_bound     src/model.cpp:257-267
 *   orc_backend_*                src/cpu.cpp:4-259     (CpuBackend, cpu_backend)
 *   orc_verify / orc_infeas...   src/verify.cpp:6-244  (lp_lower_bound, Verifier::evaluate)
 *   orc_scale                    src/preprocess.cpp:6-65,301-343 (extra_scale, Ruiz, objective)
 *   orc_solve                    src/solver.cpp:255-735 (solve_continuous, PDHG branch)
 *
 * Pinned against the reference itself: tests/test_oracle.py runs each function
 * beside the reference build in oracle/_ref (libvantage_ref.so) and against the
 * golden fixtures in tests/golden/.
 */
#ifndef NK_PDHG_ORACLE_H
#define NK_PDHG_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct orc_model orc_model;
typedef struct orc_backend orc_backend;

const char *orc_last_error(void);

void orc_transpose(int64_t rows, int64_t cols, const int64_t *ptr, const int64_t *idx,
                   const double *val, int64_t *tptr, int64_t *tidx, double *tval);
void orc_spmv(int64_t rows, const int64_t *ptr, const int64_t *idx, const double *val,
              const double *x, double *y);

/* Copies every array.  qptr may be NULL (no sparse Q). */
orc_model *orc_model_new(int64_t m, int64_t n, const int64_t *ptr, const int64_t *idx,
                         const double *val, const double *c, const double *q, const double *lb,
                         const double *ub, const double *rl, const double *ru,
                         const int64_t *qptr, const int64_t *qidx, const double *qval,
                         double offset);
void orc_model_free(orc_model *);
double orc_quadratic_norm_bound(const orc_model *);

orc_backend *orc_backend_new(const orc_model *, const double *x, const double *y, int adaptive,
                             int halpern, double reflection, int fixed_point_restarts);
void orc_backend_free(orc_backend *);
/* Returns accepted progress, or -1 with orc_last_error() set. */
int orc_backend_advance(orc_backend *, int count, double tau, double sigma);
int64_t orc_backend_rejected(const orc_backend *);
int orc_backend_restart_requested(const orc_backend *);
void orc_backend_candidates(orc_backend *, double *x, double *y, double *xa, double *ya);
void orc_backend_reset(orc_backend *, const double *x, const double *y);
/* Flattened snapshot in the reference's order; returns doubles written. */
int64_t orc_backend_snapshot(const orc_backend *, double *out);

/* acc: objective, primal, dual, gap, kkt, primal_abs, dual_abs, complementarity,
 *      lower_bound, finite */
void orc_verify(const orc_model *, const double *x, const double *y, int safe_bound, double *acc);
double orc_infeasibility_bound(const orc_model *, const double *y);

/* Ruiz equilibration + objective scaling exactly as prepare() applies them
 * (scaling="ruiz").  Returns a new model and writes column_scale[n],
 * row_scale[m], *objective_scale.  Fails (NULL) when presolve would remove a
 * column or row, since the restatement covers the scaling path only. */
orc_model *orc_scale(const orc_model *, int passes, double *column_scale, double *row_scale,
                     double *objective_scale);

/* stats: objective, primal, dual, gap, kkt, finite, iterations, restarts, rejected,
 *        weight_updates, seconds, iteration_seconds, verification_seconds,
 *        status (0 OPTIMAL, 1 ITERATION_LIMIT, 2 TIME_LIMIT, 3 NUMERICAL_ERROR) */
int orc_solve(const orc_model *, double tol, int64_t iteration_limit, double time_limit,
              int check_every, int scaling_passes, int adaptive, int restart, double *x_out,
              double *y_out, double *stats);

/* Activity-based bound proposals with directed rounding, `passes` rounds over
 * A (m x n) -- the algorithm of cuda_propagate_integer_bounds
 * (src/cuda.cu:448-529, 1033-1135), restated sequentially with the rounding
 * mode switched per operation.  lb / ub are updated in place; returns 1 when
 * feasible, 0 when a row's activity range misses [rl, ru] or bounds cross. */
int orc_propagate_bounds(int64_t m, int64_t n, const int64_t *ptr, const int64_t *idx,
                         const double *val, const int *integer, const double *rl, const double *ru,
                         double *lb, double *ub, int passes);

/* accessors for a model's arrays (used to read orc_scale results) */
void orc_model_get(const orc_model *, int64_t *ptr, int64_t *idx, double *val, double *c,
                   double *q, double *lb, double *ub, double *rl, double *ru, double *offset);
#ifdef __cplusplus
}
#endif
#endif
