/* Test infrastructure only -- the oracle.  See pdhg_oracle.h for what each
 * function restates and where.  Plain C11, sequential, FP64 with long double
 * where the reference uses long double. */
#define _GNU_SOURCE
#include "pdhg_oracle.h"
#include <fenv.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static _Thread_local char g_err[512];
static void set_err(const char *s) { snprintf(g_err, sizeof g_err, "%s", s); }
const char *orc_last_error(void) { return g_err; }

static double dmax(double a, double b) { return a < b ? b : a; } /* std::max(a,b) */
static double dmin(double a, double b) { return b < a ? b : a; } /* std::min(a,b) */
static double dclamp(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }
static long double ldmin(long double a, long double b) { return b < a ? b : a; }

typedef struct {
    int64_t rows, cols;
    int64_t *ptr, *idx;
    double *val;
} csr;

struct orc_model {
    int64_t m, n;
    csr A, At, Q; /* Q.ptr == NULL when there is no sparse Q */
    double *c, *q, *lb, *ub, *rl, *ru;
    double offset;
};

static void *xmalloc(size_t bytes) {
    void *p = malloc(bytes ? bytes : 1);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}
static double *dup_d(const double *s, int64_t n) {
    double *d = xmalloc((size_t)n * sizeof(double));
    if (n) memcpy(d, s, (size_t)n * sizeof(double));
    return d;
}
static int64_t *dup_i(const int64_t *s, int64_t n) {
    int64_t *d = xmalloc((size_t)n * sizeof(int64_t));
    if (n) memcpy(d, s, (size_t)n * sizeof(int64_t));
    return d;
}

/* Sparse::transpose, src/model.cpp:39-58: counting sort by column, rows in order. */
void orc_transpose(int64_t rows, int64_t cols, const int64_t *ptr, const int64_t *idx,
                   const double *val, int64_t *tptr, int64_t *tidx, double *tval) {
    memset(tptr, 0, (size_t)(cols + 1) * sizeof(int64_t));
    int64_t nnz = ptr[rows];
    for (int64_t k = 0; k < nnz; k++) tptr[idx[k] + 1]++;
    for (int64_t j = 0; j < cols; j++) tptr[j + 1] += tptr[j];
    int64_t *pos = dup_i(tptr, cols + 1);
    for (int64_t i = 0; i < rows; i++)
        for (int64_t k = ptr[i]; k < ptr[i + 1]; k++) {
            int64_t p = pos[idx[k]]++;
            tidx[p] = i;
            tval[p] = val[k];
        }
    free(pos);
}

/* Sparse::multiply, src/model.cpp:59-73: per-row sequential FP64 sum from 0. */
void orc_spmv(int64_t rows, const int64_t *ptr, const int64_t *idx, const double *val,
              const double *x, double *y) {
    for (int64_t i = 0; i < rows; i++) {
        double v = 0;
        for (int64_t k = ptr[i]; k < ptr[i + 1]; k++) v += val[k] * x[idx[k]];
        y[i] = v;
    }
}

static void csr_copy(csr *d, int64_t rows, int64_t cols, const int64_t *ptr, const int64_t *idx,
                     const double *val) {
    d->rows = rows;
    d->cols = cols;
    d->ptr = dup_i(ptr, rows + 1);
    d->idx = dup_i(idx, ptr[rows]);
    d->val = dup_d(val, ptr[rows]);
}
static void csr_free(csr *a) {
    free(a->ptr);
    free(a->idx);
    free(a->val);
    a->ptr = a->idx = NULL;
    a->val = NULL;
}
static void build_transpose(orc_model *M) {
    int64_t nnz = M->A.ptr[M->m];
    M->At.rows = M->n;
    M->At.cols = M->m;
    M->At.ptr = xmalloc((size_t)(M->n + 1) * sizeof(int64_t));
    M->At.idx = xmalloc((size_t)nnz * sizeof(int64_t));
    M->At.val = xmalloc((size_t)nnz * sizeof(double));
    orc_transpose(M->m, M->n, M->A.ptr, M->A.idx, M->A.val, M->At.ptr, M->At.idx, M->At.val);
}

orc_model *orc_model_new(int64_t m, int64_t n, const int64_t *ptr, const int64_t *idx,
                         const double *val, const double *c, const double *q, const double *lb,
                         const double *ub, const double *rl, const double *ru,
                         const int64_t *qptr, const int64_t *qidx, const double *qval,
                         double offset) {
    orc_model *M = calloc(1, sizeof *M);
    M->m = m;
    M->n = n;
    csr_copy(&M->A, m, n, ptr, idx, val);
    build_transpose(M);
    if (qptr && qptr[n] > 0)
        csr_copy(&M->Q, n, n, qptr, qidx, qval);
    M->c = dup_d(c, n);
    if (q)
        M->q = dup_d(q, n);
    else
        M->q = calloc((size_t)(n ? n : 1), sizeof(double));
    M->lb = dup_d(lb, n);
    M->ub = dup_d(ub, n);
    M->rl = dup_d(rl, m);
    M->ru = dup_d(ru, m);
    M->offset = offset;
    return M;
}
void orc_model_free(orc_model *M) {
    if (!M) return;
    csr_free(&M->A);
    csr_free(&M->At);
    if (M->Q.ptr) csr_free(&M->Q);
    free(M->c);
    free(M->q);
    free(M->lb);
    free(M->ub);
    free(M->rl);
    free(M->ru);
    free(M);
}
void orc_model_get(const orc_model *M, int64_t *ptr, int64_t *idx, double *val, double *c,
                   double *q, double *lb, double *ub, double *rl, double *ru, double *offset) {
    int64_t nnz = M->A.ptr[M->m];
    if (ptr) memcpy(ptr, M->A.ptr, (size_t)(M->m + 1) * sizeof(int64_t));
    if (idx) memcpy(idx, M->A.idx, (size_t)nnz * sizeof(int64_t));
    if (val) memcpy(val, M->A.val, (size_t)nnz * sizeof(double));
    if (c) memcpy(c, M->c, (size_t)M->n * sizeof(double));
    if (q) memcpy(q, M->q, (size_t)M->n * sizeof(double));
    if (lb) memcpy(lb, M->lb, (size_t)M->n * sizeof(double));
    if (ub) memcpy(ub, M->ub, (size_t)M->n * sizeof(double));
    if (rl) memcpy(rl, M->rl, (size_t)M->m * sizeof(double));
    if (ru) memcpy(ru, M->ru, (size_t)M->m * sizeof(double));
    if (offset) *offset = M->offset;
}
static int has_Q(const orc_model *M) { return M->Q.ptr != NULL && M->Q.ptr[M->n] > 0; }
static int is_qp(const orc_model *M) {
    if (has_Q(M)) return 1;
    for (int64_t j = 0; j < M->n; j++)
        if (M->q[j] != 0) return 1;
    return 0;
}

/* Model::quadratic_norm_bound, src/model.cpp:257-267 */
double orc_quadratic_norm_bound(const orc_model *M) {
    long double largest = 0;
    for (int64_t i = 0; i < M->n; i++) {
        long double sum = fabs(M->q[i]);
        if (has_Q(M))
            for (int64_t k = M->Q.ptr[i]; k < M->Q.ptr[i + 1]; k++) sum += fabs(M->Q.val[k]);
        if (largest < sum) largest = sum;
    }
    return nextafter((double)largest, INFINITY);
}

/* ---------------------------------------------------------------- CpuBackend */
struct orc_backend {
    const orc_model *M;
    int64_t n, m;
    double *x, *y, *delta_x, *xa, *ya, *gradient, *trial_x, *trial_y, *ax, *next_ax, *qx;
    double *anchor_x, *anchor_y, *anchor_ax;
    int adaptive, halpern, fixed_point_restarts, request_restart;
    double a_norm, q_norm, reflection;
    int64_t epoch_steps, accepted, rejected;
    double initial_residual, previous_residual, factor, average_mass;
};

orc_backend *orc_backend_new(const orc_model *M, const double *px, const double *py, int adaptive,
                             int halpern, double reflection, int fixed_point_restarts) {
    if (halpern && adaptive) {
        set_err("Halpern requires a fixed PDHG operator");
        return NULL;
    }
    if (!isfinite(reflection) || reflection < 0 || reflection > 1) {
        set_err("Invalid Halpern reflection");
        return NULL;
    }
    orc_backend *B = calloc(1, sizeof *B);
    int64_t n = M->n, m = M->m;
    B->M = M;
    B->n = n;
    B->m = m;
    B->x = dup_d(px, n);
    B->y = dup_d(py, m);
    B->delta_x = dup_d(px, n); /* the reference initialises delta_x with x */
    B->xa = calloc((size_t)(n ? n : 1), sizeof(double));
    B->ya = calloc((size_t)(m ? m : 1), sizeof(double));
    B->gradient = calloc((size_t)(n ? n : 1), sizeof(double));
    B->trial_x = calloc((size_t)(n ? n : 1), sizeof(double));
    B->trial_y = calloc((size_t)(m ? m : 1), sizeof(double));
    B->ax = xmalloc((size_t)(m ? m : 1) * sizeof(double));
    orc_spmv(m, M->A.ptr, M->A.idx, M->A.val, B->x, B->ax);
    B->next_ax = calloc((size_t)(m ? m : 1), sizeof(double));
    B->qx = calloc((size_t)(n ? n : 1), sizeof(double));
    B->adaptive = adaptive;
    B->halpern = halpern;
    B->reflection = reflection;
    B->fixed_point_restarts = fixed_point_restarts;
    B->initial_residual = B->previous_residual = INFINITY;
    B->factor = 1;
    if (has_Q(M)) {
        B->adaptive = 0;
        B->q_norm = orc_quadratic_norm_bound(M);
        double *cols = calloc((size_t)(n ? n : 1), sizeof(double));
        double rowmax = 0;
        for (int64_t i = 0; i < m; i++) {
            double sum = 0;
            for (int64_t k = M->A.ptr[i]; k < M->A.ptr[i + 1]; k++) {
                sum += fabs(M->A.val[k]);
                cols[M->A.idx[k]] += fabs(M->A.val[k]);
            }
            rowmax = dmax(rowmax, sum);
        }
        double colmax = 0;
        for (int64_t j = 0; j < n; j++) colmax = dmax(colmax, cols[j]);
        free(cols);
        B->a_norm = sqrt(rowmax) * sqrt(colmax);
    }
    if (halpern) {
        B->anchor_x = dup_d(B->x, n);
        B->anchor_y = dup_d(B->y, m);
        B->anchor_ax = dup_d(B->ax, m);
    }
    return B;
}
void orc_backend_free(orc_backend *B) {
    if (!B) return;
    free(B->x); free(B->y); free(B->delta_x); free(B->xa); free(B->ya); free(B->gradient);
    free(B->trial_x); free(B->trial_y); free(B->ax); free(B->next_ax); free(B->qx);
    free(B->anchor_x); free(B->anchor_y); free(B->anchor_ax);
    free(B);
}
int64_t orc_backend_rejected(const orc_backend *B) { return B->rejected; }
int orc_backend_restart_requested(const orc_backend *B) { return B->request_restart; }

#define SWAP(a, b) do { double *t_ = (a); (a) = (b); (b) = t_; } while (0)

/* CpuBackend::advance, src/cpu.cpp:96-222 */
int orc_backend_advance(orc_backend *B, int count, double primal_step, double dual_step) {
    const orc_model *M = B->M;
    int64_t n = B->n, m = B->m;
    int sparse_q = has_Q(M);
    if (sparse_q) {
        double safety = sqrt(primal_step * dual_step) * B->a_norm + primal_step * B->q_norm;
        double scale = safety > 0 ? dmin(1., .9 / safety) : 1.;
        primal_step *= scale;
        dual_step *= scale;
    }
    for (int it = 0; it < count; it++) {
        for (int64_t j = 0; j < n; j++) {
            double g = M->c[j];
            for (int64_t k = M->At.ptr[j]; k < M->At.ptr[j + 1]; k++)
                g += M->At.val[k] * B->y[M->At.idx[k]];
            B->gradient[j] = g;
        }
        if (sparse_q) {
            orc_spmv(n, M->Q.ptr, M->Q.idx, M->Q.val, B->x, B->qx);
            for (int64_t j = 0; j < n; j++) B->gradient[j] += B->qx[j] + M->q[j] * B->x[j];
        }
        int success = 0;
        for (int attempt = 0; attempt < 40; attempt++) {
            double tau = primal_step * B->factor, sigma = dual_step * B->factor;
            double dx2 = 0, dy2 = 0, coupling = 0;
            for (int64_t j = 0; j < n; j++) {
                B->trial_x[j] = dclamp((B->x[j] - tau * B->gradient[j]) /
                                           (1 + tau * (sparse_q ? 0 : M->q[j])),
                                       M->lb[j], M->ub[j]);
                double dx = B->trial_x[j] - B->x[j];
                dx2 += dx * dx;
                B->delta_x[j] = dx;
            }
            for (int64_t i = 0; i < m; i++) {
                double delta = 0;
                for (int64_t k = M->A.ptr[i]; k < M->A.ptr[i + 1]; k++)
                    delta += M->A.val[k] * B->delta_x[M->A.idx[k]];
                double bar = B->ax[i] + 2 * delta;
                double z = B->y[i] + sigma * bar;
                B->trial_y[i] = dmax(0., z - sigma * M->ru[i]) + dmin(0., z - sigma * M->rl[i]);
                double dy = B->trial_y[i] - B->y[i];
                dy2 += dy * dy;
                if (!isfinite(bar) || !isfinite(B->trial_y[i])) dy2 = INFINITY;
                coupling += dy * delta;
                B->next_ax[i] = B->ax[i] + delta;
            }
            double energy = dx2 / tau + dy2 / sigma;
            double limit = fabs(coupling) > 0 ? energy / (2 * fabs(coupling)) : INFINITY;
            int finite = isfinite(energy) && isfinite(coupling);
            double used_factor = B->factor;
            int accept = finite && (!B->adaptive || limit >= 1);
            if (B->adaptive) {
                double k = (double)(B->accepted + 2);
                double multiplier = dmin((1 - pow(k, -.3)) * limit, 1 + pow(k, -.6));
                if (!finite || !isfinite(multiplier) || multiplier <= 0) multiplier = .5;
                B->factor = dclamp(B->factor * multiplier, 1e-12, 1e12);
            }
            if (!accept) {
                B->rejected++;
                if (!B->adaptive) {
                    set_err("Nonfinite PDHG step");
                    return -1;
                }
                continue;
            }
            SWAP(B->x, B->trial_x);
            SWAP(B->y, B->trial_y);
            SWAP(B->ax, B->next_ax);
            B->accepted++;
            if (B->halpern) {
                memcpy(B->xa, B->x, (size_t)n * sizeof(double));
                memcpy(B->ya, B->y, (size_t)m * sizeof(double));
                double lambda = 1 / ((double)B->epoch_steps + 2);
                double r = B->reflection;
                for (int64_t j = 0; j < n; j++)
                    B->x[j] = lambda * B->anchor_x[j] +
                              (1 - lambda) * ((1 + r) * B->x[j] - r * B->trial_x[j]);
                for (int64_t i = 0; i < m; i++) {
                    B->y[i] = lambda * B->anchor_y[i] +
                              (1 - lambda) * ((1 + r) * B->y[i] - r * B->trial_y[i]);
                    B->ax[i] = lambda * B->anchor_ax[i] +
                               (1 - lambda) * ((1 + r) * B->ax[i] - r * B->next_ax[i]);
                }
                double residual = sqrt(dmax(0., energy - 2 * coupling));
                if (B->epoch_steps == 0) B->initial_residual = residual;
                B->epoch_steps++;
                int64_t half = B->accepted / 2;
                B->request_restart =
                    B->fixed_point_restarts && B->epoch_steps >= 10 &&
                    (residual <= .2 * B->initial_residual ||
                     (residual <= .8 * B->initial_residual && residual > B->previous_residual) ||
                     B->epoch_steps >= (half > 10 ? half : 10));
                B->previous_residual = residual;
                if (B->request_restart) return it + 1;
                success = 1;
                break;
            }
            B->average_mass += used_factor;
            double w = used_factor / B->average_mass;
            for (int64_t j = 0; j < n; j++) B->xa[j] += (B->x[j] - B->xa[j]) * w;
            for (int64_t i = 0; i < m; i++) B->ya[i] += (B->y[i] - B->ya[i]) * w;
            success = 1;
            break;
        }
        if (!success) {
            set_err("PDHG backtracking exhausted");
            return -1;
        }
    }
    return count;
}

/* CpuBackend::candidates, src/cpu.cpp:223-231 (rebases A*x) */
void orc_backend_candidates(orc_backend *B, double *x, double *y, double *xa, double *ya) {
    memcpy(x, B->x, (size_t)B->n * sizeof(double));
    memcpy(y, B->y, (size_t)B->m * sizeof(double));
    memcpy(xa, B->xa, (size_t)B->n * sizeof(double));
    memcpy(ya, B->ya, (size_t)B->m * sizeof(double));
    orc_spmv(B->m, B->M->A.ptr, B->M->A.idx, B->M->A.val, B->x, B->ax);
}

/* CpuBackend::reset, src/cpu.cpp:232-247 */
void orc_backend_reset(orc_backend *B, const double *x, const double *y) {
    memcpy(B->x, x, (size_t)B->n * sizeof(double));
    memcpy(B->y, y, (size_t)B->m * sizeof(double));
    orc_spmv(B->m, B->M->A.ptr, B->M->A.idx, B->M->A.val, B->x, B->ax);
    if (B->halpern) {
        memcpy(B->anchor_x, B->x, (size_t)B->n * sizeof(double));
        memcpy(B->anchor_y, B->y, (size_t)B->m * sizeof(double));
        memcpy(B->anchor_ax, B->ax, (size_t)B->m * sizeof(double));
        B->epoch_steps = 0;
        B->initial_residual = B->previous_residual = INFINITY;
        B->request_restart = 0;
    }
    B->average_mass = 0;
    memset(B->xa, 0, (size_t)B->n * sizeof(double));
    memset(B->ya, 0, (size_t)B->m * sizeof(double));
}

/* CpuBackend::snapshot order, src/cpu.cpp:49-61 */
int64_t orc_backend_snapshot(const orc_backend *B, double *out) {
    int64_t n = B->n, m = B->m, at = 0;
#define PUT(p, len) do { if (out && (len)) memcpy(out + at, (p), (size_t)(len) * sizeof(double)); at += (len); } while (0)
    PUT(B->x, n); PUT(B->y, m); PUT(B->delta_x, n); PUT(B->xa, n); PUT(B->ya, m); PUT(B->ax, m);
    if (B->halpern) { PUT(B->anchor_x, n); PUT(B->anchor_y, m); PUT(B->anchor_ax, m); }
    double tail[8] = {(double)B->epoch_steps, B->factor, B->average_mass, (double)B->accepted,
                      (double)B->rejected, B->initial_residual, B->previous_residual,
                      B->request_restart ? 1. : 0.};
    PUT(tail, 8);
#undef PUT
    return at;
}

/* ---------------------------------------------------------------- Verifier */
static long double down(long double v) { return nextafterl(v, -INFINITY); }
static long double up(long double v) { return nextafterl(v, INFINITY); }

/* lp_lower_bound, src/verify.cpp:12-88 */
static double lp_lower_bound(const orc_model *M, const double *y, int feasibility,
                             const double *point) {
    long double lower = feasibility ? 0 : M->offset;
    int64_t n = M->n, m = M->m;
    int sq = has_Q(M);
    if (point) {
        for (int64_t i = 0; i < n; i++) {
            long double square = up((long double)point[i] * point[i]);
            if (M->q[i] != 0) {
                long double lo = down((long double)point[i] * point[i]);
                long double term = M->q[i] >= 0 ? up(M->q[i] * square) : up(M->q[i] * lo);
                lower = down(lower - up(.5L * term));
            }
            if (sq)
                for (int64_t k = M->Q.ptr[i]; k < M->Q.ptr[i + 1]; k++) {
                    int64_t j = M->Q.idx[k];
                    long double v = M->Q.val[k];
                    long double lo = down((long double)point[i] * point[j]);
                    long double hi = up((long double)point[i] * point[j]);
                    long double term = up(v * (v >= 0 ? hi : lo));
                    lower = down(lower - up(.5L * term));
                }
        }
    }
    for (int64_t i = 0; i < m; i++)
        if (y[i] != 0) {
            double b = y[i] > 0 ? M->ru[i] : M->rl[i];
            if (!isfinite(b)) return -INFINITY;
            if (b == 0) continue;
            long double term = (long double)y[i] * b;
            lower = down(lower - up(term));
        }
    for (int64_t j = 0; j < n; j++) {
        long double gl = feasibility ? 0 : M->c[j], gu = gl;
        if (point) {
#define ADD(coef, value) do { double c_ = (coef), v_ = (value); \
            if (!(c_ == 0 || v_ == 0)) { long double t_ = (long double)c_ * v_; \
            gl = down(gl + down(t_)); gu = up(gu + up(t_)); } } while (0)
            ADD(M->q[j], point[j]);
            if (sq)
                for (int64_t k = M->Q.ptr[j]; k < M->Q.ptr[j + 1]; k++)
                    ADD(M->Q.val[k], point[M->Q.idx[k]]);
#undef ADD
        }
        for (int64_t k = M->At.ptr[j]; k < M->At.ptr[j + 1]; k++)
            if (y[M->At.idx[k]] != 0 && M->At.val[k] != 0) {
                long double v = (long double)M->At.val[k] * y[M->At.idx[k]];
                gl = down(gl + down(v));
                gu = up(gu + up(v));
            }
        if ((!isfinite(M->lb[j]) && gu > 0) || (!isfinite(M->ub[j]) && gl < 0)) return -INFINITY;
        long double term = INFINITY;
        if (gl <= 0 && gu >= 0) term = 0;
        double bs[2] = {M->lb[j], M->ub[j]};
        for (int t = 0; t < 2; t++) {
            double b = bs[t];
            if (isfinite(b)) {
                term = ldmin(term, (b == 0 || gl == 0) ? 0 : down(gl * b));
                term = ldmin(term, (b == 0 || gu == 0) ? 0 : down(gu * b));
            }
        }
        if (gl == 0 && gu == 0) term = 0;
        if (!isfinite(term)) return -INFINITY;
        if (term != 0) lower = down(lower + term);
    }
    double result = (double)lower;
    if (!isfinite(result)) return -INFINITY;
    return nextafter(result, -INFINITY);
}

double orc_infeasibility_bound(const orc_model *M, const double *y) {
    for (int64_t i = 0; i < M->m; i++)
        if (!isfinite(y[i])) return -INFINITY;
    return lp_lower_bound(M, y, 1, NULL);
}

static void acc_default(double *acc) {
    for (int i = 0; i < 8; i++) acc[i] = INFINITY;
    acc[8] = -INFINITY;
    acc[9] = 0;
}

/* Verifier::evaluate, src/verify.cpp:103-240 */
void orc_verify(const orc_model *M, const double *x, const double *y, int safe_bound,
                double *acc) {
    int64_t n = M->n, m = M->m;
    acc_default(acc);
    for (int64_t j = 0; j < n; j++)
        if (!isfinite(x[j])) return;
    for (int64_t i = 0; i < m; i++)
        if (!isfinite(y[i])) return;
    double *ax = xmalloc((size_t)(m ? m : 1) * sizeof(double));
    double *aty = xmalloc((size_t)(n ? n : 1) * sizeof(double));
    double *qx = calloc((size_t)(n ? n : 1), sizeof(double));
    orc_spmv(m, M->A.ptr, M->A.idx, M->A.val, x, ax);
    orc_spmv(n, M->At.ptr, M->At.idx, M->At.val, y, aty);
    int bad = 0;
    for (int64_t i = 0; i < m && !bad; i++) bad = !isfinite(ax[i]);
    for (int64_t j = 0; j < n && !bad; j++) bad = !isfinite(aty[j]);
    if (bad) goto done;
    double objective = M->offset, primal = 0, dual = 0, primal_abs = 0, dual_abs = 0;
    long double support = 0, box_min = 0, complement = 0;
    int bound_ok = 1;
    for (int64_t i = 0; i < m; i++) {
        double v = dmax(dmax(0., M->rl[i] - ax[i]), ax[i] - M->ru[i]);
        if (isfinite(M->rl[i]))
            primal = dmax(primal, dmax(0., M->rl[i] - ax[i]) / (1 + fabs(M->rl[i])));
        if (isfinite(M->ru[i]))
            primal = dmax(primal, dmax(0., ax[i] - M->ru[i]) / (1 + fabs(M->ru[i])));
        primal_abs = dmax(primal_abs, v);
        double endpoint = y[i] > 0 ? M->ru[i] : M->rl[i];
        if (y[i] != 0) {
            if (isfinite(endpoint)) {
                support += (long double)y[i] * endpoint;
                complement += fabsl((long double)y[i] * (endpoint - ax[i]));
            } else {
                bound_ok = 0;
                dual_abs = dmax(dual_abs, fabs(y[i]));
                dual = dmax(dual, fabs(y[i]));
            }
        }
    }
    int sq = has_Q(M), qp = is_qp(M);
    if (sq) orc_spmv(n, M->Q.ptr, M->Q.idx, M->Q.val, x, qx);
    double cscale = 1;
    for (int64_t j = 0; j < n; j++) cscale = dmax(cscale, 1 + fabs(M->c[j]));
    for (int64_t j = 0; j < n; j++) {
        double v = dmax(dmax(0., M->lb[j] - x[j]), x[j] - M->ub[j]);
        double bs = 1 + fabs(x[j]);
        primal = dmax(primal, v / bs);
        primal_abs = dmax(primal_abs, v);
        objective += M->c[j] * x[j] + .5 * M->q[j] * x[j] * x[j] + .5 * x[j] * qx[j];
        double linear = M->c[j] + aty[j], g = linear + M->q[j] * x[j] + qx[j];
        if (!isfinite(linear) || !isfinite(g)) goto done;
        double d = dclamp(g, x[j] - M->ub[j], x[j] - M->lb[j]);
        dual_abs = dmax(dual_abs, fabs(d));
        dual = dmax(dual, fabs(d) / cscale);
        if (g > 0 && isfinite(M->lb[j])) complement += fabsl((long double)g * (x[j] - M->lb[j]));
        if (g < 0 && isfinite(M->ub[j])) complement += fabsl((long double)g * (M->ub[j] - x[j]));
        if (sq) {
            double arg = g > 0 ? M->lb[j] : g < 0 ? M->ub[j] : dclamp(0., M->lb[j], M->ub[j]);
            if (!isfinite(arg))
                bound_ok = 0;
            else
                box_min += (long double)g * arg - (long double)(M->q[j] * x[j] + qx[j]) * x[j] / 2;
            continue;
        }
        double arg = 0;
        if (M->q[j] > 0)
            arg = dclamp(-linear / M->q[j], M->lb[j], M->ub[j]);
        else if (linear > 0)
            arg = M->lb[j];
        else if (linear < 0)
            arg = M->ub[j];
        else
            arg = dclamp(0., M->lb[j], M->ub[j]);
        if (!isfinite(arg))
            bound_ok = 0;
        else
            box_min += (long double)linear * arg + .5L * M->q[j] * arg * arg;
    }
    double complementarity = (double)complement;
    double gap = complementarity / (1 + fabs(objective - M->offset));
    double lower_bound = -INFINITY;
    if (bound_ok) {
        long double lower = (long double)M->offset - support + box_min;
        long double guard = 64 * __DBL_EPSILON__ *
                            (1 + fabsl((long double)M->offset) + fabsl(support) + fabsl(box_min));
        lower_bound = (double)(lower - guard);
        gap = dmax(gap, fabs(objective - lower_bound) /
                            (1 + fabs(objective) + fabs(lower_bound)));
    }
    if (safe_bound)
        lower_bound = lp_lower_bound(M, y, 0, qp ? x : NULL);
    else if (!qp)
        lower_bound = -INFINITY;
    if (isfinite(lower_bound))
        gap = dmax(gap, fabs(objective - lower_bound) / (1 + fabs(objective) + fabs(lower_bound)));
    double kkt = dmax(dmax(primal, dual), gap);
    int finite = isfinite(objective) && isfinite(kkt) && isfinite(gap) && isfinite(primal) &&
                 isfinite(dual);
    if (!finite) {
        kkt = INFINITY;
        lower_bound = -INFINITY;
    }
    acc[0] = objective;
    acc[1] = primal;
    acc[2] = dual;
    acc[3] = gap;
    acc[4] = kkt;
    acc[5] = primal_abs;
    acc[6] = dual_abs;
    acc[7] = complementarity;
    acc[8] = lower_bound;
    acc[9] = finite ? 1 : 0;
done:
    free(ax);
    free(aty);
    free(qx);
}

/* ---------------------------------------------------------------- scaling */
static int representable(double before, double after) {
    return isfinite(before) ? (isfinite(after) && (before == 0 || after != 0)) : before == after;
}

typedef struct {
    orc_model *m;
    double *cs, *rs;
} prep;

/* extra_scale, src/preprocess.cpp:12-65 (built with VANTAGE_SPARSE_LU defined) */
static void extra_scale(prep *p, const double *row, double *col) {
    orc_model *M = p->m;
    for (int64_t i = 0; i < M->m; i++) {
        double f = row[i];
        int safe = representable(p->rs[i], p->rs[i] * f) && representable(M->rl[i], M->rl[i] * f) &&
                   representable(M->ru[i], M->ru[i] * f);
        for (int64_t k = M->A.ptr[i]; k < M->A.ptr[i + 1]; k++)
            safe &= representable(M->A.val[k], M->A.val[k] * f);
        if (!safe) continue;
        p->rs[i] *= f;
        M->rl[i] *= f;
        M->ru[i] *= f;
        for (int64_t k = M->A.ptr[i]; k < M->A.ptr[i + 1]; k++) M->A.val[k] *= f;
    }
    for (int64_t j = 0; j < M->n; j++) {
        double f = col[j];
        if (!representable(p->cs[j], p->cs[j] * f) || !representable(M->c[j], M->c[j] * f) ||
            !representable(M->q[j], M->q[j] * (f * f)) || !representable(M->lb[j], M->lb[j] / f) ||
            !representable(M->ub[j], M->ub[j] / f))
            col[j] = 1;
    }
    int64_t nnz = M->A.ptr[M->m];
    for (int64_t k = 0; k < nnz; k++) {
        int64_t j = M->A.idx[k];
        if (!representable(M->A.val[k], M->A.val[k] * col[j])) col[j] = 1;
    }
    int qsafe = 1;
    if (has_Q(M))
        for (int64_t i = 0; i < M->n; i++)
            for (int64_t k = M->Q.ptr[i]; k < M->Q.ptr[i + 1]; k++)
                qsafe &= representable(M->Q.val[k], (M->Q.val[k] * col[i]) * col[M->Q.idx[k]]);
    if (!qsafe)
        for (int64_t j = 0; j < M->n; j++) col[j] = 1;
    if (has_Q(M))
        for (int64_t i = 0; i < M->n; i++)
            for (int64_t k = M->Q.ptr[i]; k < M->Q.ptr[i + 1]; k++)
                M->Q.val[k] *= col[i] * col[M->Q.idx[k]];
    for (int64_t j = 0; j < M->n; j++) {
        double f = col[j];
        p->cs[j] *= f;
        M->c[j] *= f;
        M->q[j] *= f * f;
        M->lb[j] /= f;
        M->ub[j] /= f;
    }
    for (int64_t k = 0; k < nnz; k++) M->A.val[k] *= col[M->A.idx[k]];
}

static int needs_presolve(const orc_model *S) {
    char *used = calloc((size_t)(S->n ? S->n : 1), 1);
    int64_t nnz = S->A.ptr[S->m];
    for (int64_t k = 0; k < nnz; k++) used[S->A.idx[k]] = 1;
    if (has_Q(S))
        for (int64_t i = 0; i < S->n; i++)
            for (int64_t k = S->Q.ptr[i]; k < S->Q.ptr[i + 1]; k++) used[i] = used[S->Q.idx[k]] = 1;
    int bad = 0;
    for (int64_t j = 0; j < S->n && !bad; j++) {
        if (S->lb[j] == S->ub[j]) bad = 1;
        else if (!used[j]) {
            double chosen = S->q[j] > 0 ? dclamp(-S->c[j] / S->q[j], S->lb[j], S->ub[j])
                            : S->c[j] > 0 ? S->lb[j]
                            : S->c[j] < 0 ? S->ub[j]
                                          : dclamp(0., S->lb[j], S->ub[j]);
            if (isfinite(chosen)) bad = 1;
        }
    }
    free(used);
    /* rows: empty, or provably redundant (src/preprocess.cpp:216-252) */
    for (int64_t i = 0; i < S->m && !bad; i++) {
        int64_t len = S->A.ptr[i + 1] - S->A.ptr[i];
        if (len == 0) { bad = 1; break; }
        long double amin = 0, amax = 0, magnitude = 0;
        for (int64_t k = S->A.ptr[i]; k < S->A.ptr[i + 1]; k++) {
            int64_t j = S->A.idx[k];
            double v = S->A.val[k];
            amin += (long double)v * (v > 0 ? S->lb[j] : S->ub[j]);
            amax += (long double)v * (v > 0 ? S->ub[j] : S->lb[j]);
            magnitude += fabsl((long double)v * (v > 0 ? S->lb[j] : S->ub[j])) +
                         fabsl((long double)v * (v > 0 ? S->ub[j] : S->lb[j]));
        }
        if (isfinite(amin) && isfinite(amax)) {
            long double guard = 8 * __LDBL_EPSILON__ * (len + 1) * (1 + magnitude);
            if (amin > S->ru[i] + guard || amax < S->rl[i] - guard) bad = 1;
            if (amin - guard >= S->rl[i] && amax + guard <= S->ru[i]) bad = 1;
        }
    }
    return bad;
}

orc_model *orc_scale(const orc_model *S, int passes, double *column_scale, double *row_scale,
                     double *objective_scale) {
    if (needs_presolve(S)) {
        set_err("model needs presolve reductions (fixed/unused column or empty/redundant row)");
        return NULL;
    }
    orc_model *M = orc_model_new(S->m, S->n, S->A.ptr, S->A.idx, S->A.val, S->c, S->q, S->lb,
                                 S->ub, S->rl, S->ru, has_Q(S) ? S->Q.ptr : NULL,
                                 has_Q(S) ? S->Q.idx : NULL, has_Q(S) ? S->Q.val : NULL,
                                 S->offset);
    prep p = {M, column_scale, row_scale};
    for (int64_t j = 0; j < M->n; j++) column_scale[j] = 1;
    for (int64_t i = 0; i < M->m; i++) row_scale[i] = 1;
    double *row = xmalloc((size_t)(M->m ? M->m : 1) * sizeof(double));
    double *col = xmalloc((size_t)(M->n ? M->n : 1) * sizeof(double));
    double *norm = xmalloc((size_t)(M->n ? M->n : 1) * sizeof(double));
    int64_t nnz = M->A.ptr[M->m];
    for (int pass = 0; pass < passes; pass++) {
        for (int64_t j = 0; j < M->n; j++) col[j] = 1;
        for (int64_t i = 0; i < M->m; i++) {
            double nrm = 0;
            for (int64_t k = M->A.ptr[i]; k < M->A.ptr[i + 1]; k++) nrm = dmax(nrm, fabs(M->A.val[k]));
            row[i] = nrm > 0 ? dclamp(1 / sqrt(nrm), 1e-3, 1e3) : 1.;
        }
        extra_scale(&p, row, col);
        for (int64_t j = 0; j < M->n; j++) norm[j] = 0;
        for (int64_t k = 0; k < nnz; k++)
            norm[M->A.idx[k]] = dmax(norm[M->A.idx[k]], fabs(M->A.val[k]));
        for (int64_t j = 0; j < M->n; j++)
            col[j] = norm[j] > 0 ? dclamp(1 / sqrt(norm[j]), 1e-3, 1e3) : 1.;
        for (int64_t i = 0; i < M->m; i++) row[i] = 1;
        extra_scale(&p, row, col);
    }
    double os = 1;
    if (passes > 0) {
        double cnorm = 0;
        for (int64_t j = 0; j < M->n; j++) cnorm = dmax(cnorm, fabs(M->c[j]));
        for (int64_t j = 0; j < M->n; j++) cnorm = dmax(cnorm, fabs(M->q[j]));
        if (has_Q(M))
            for (int64_t k = 0; k < M->Q.ptr[M->n]; k++) cnorm = dmax(cnorm, fabs(M->Q.val[k]));
        os = cnorm > 0 ? cnorm : 1;
        for (int64_t j = 0; j < M->n; j++) M->c[j] /= os;
        for (int64_t j = 0; j < M->n; j++) M->q[j] /= os;
        if (has_Q(M))
            for (int64_t k = 0; k < M->Q.ptr[M->n]; k++) M->Q.val[k] /= os;
        M->offset /= os;
    }
    *objective_scale = os;
    free(row);
    free(col);
    free(norm);
    /* the transpose must follow the scaled values */
    csr_free(&M->At);
    build_transpose(M);
    return M;
}

/* ---------------------------------------------------------------- driver */
static double now_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* solve_continuous PDHG branch, src/solver.cpp:255-735, for models that need no
 * presolve reductions (identity column/row maps).  Farkas-ray extraction
 * (:599-633) only changes the outcome for infeasible models and is omitted;
 * polishing, checkpoints and the device monitor are off by default there too. */
int orc_solve(const orc_model *S, double tol, int64_t iteration_limit, double time_limit,
              int check_every, int scaling_passes, int adaptive, int restart, double *x_out,
              double *y_out, double *stats) {
    double start = now_s();
    int64_t n = S->n, m = S->m;
    double *cs = xmalloc((size_t)(n ? n : 1) * sizeof(double));
    double *rs = xmalloc((size_t)(m ? m : 1) * sizeof(double));
    double os = 1;
    orc_model *M = orc_scale(S, scaling_passes, cs, rs, &os);
    if (!M) {
        free(cs);
        free(rs);
        return -1;
    }
    double *x = calloc((size_t)(n ? n : 1), sizeof(double));
    double *y = calloc((size_t)(m ? m : 1), sizeof(double));
    for (int64_t j = 0; j < n; j++) x[j] = dclamp(0. / cs[j], M->lb[j], M->ub[j]);
    double *rx = xmalloc((size_t)(n ? n : 1) * sizeof(double));
    double *ry = xmalloc((size_t)(m ? m : 1) * sizeof(double));
    double *ox = xmalloc((size_t)(n ? n : 1) * sizeof(double));
    double *oy = xmalloc((size_t)(m ? m : 1) * sizeof(double));
    double *aox = xmalloc((size_t)(n ? n : 1) * sizeof(double));
    double *aoy = xmalloc((size_t)(m ? m : 1) * sizeof(double));
    double *cx = xmalloc((size_t)(n ? n : 1) * sizeof(double));
    double *cy = xmalloc((size_t)(m ? m : 1) * sizeof(double));
    double *ax_ = xmalloc((size_t)(n ? n : 1) * sizeof(double));
    double *ay_ = xmalloc((size_t)(m ? m : 1) * sizeof(double));
    double *epochx = dup_d(x, n), *epochy = dup_d(y, m);
#define RESTORE_X(src, dst) for (int64_t j_ = 0; j_ < n; j_++) (dst)[j_] = (src)[j_] * cs[j_]
    /* restore_y: out[y >= 0 ? upper : lower] += y * rs * os; identity maps here */
#define RESTORE_Y(src, dst) for (int64_t i_ = 0; i_ < m; i_++) (dst)[i_] = 0. + (src)[i_] * rs[i_] * os
    RESTORE_X(x, rx);
    RESTORE_Y(y, ry);
    double acc[10], ca[10], aa[10];
    orc_verify(S, rx, ry, 1, acc);
    int status = 1; /* ITERATION_LIMIT */
    int64_t iterations = 0, restarts = 0, weight_updates = 0, rejected_total = 0;
    double iteration_seconds = 0, verification_seconds = 0;
    if (acc[9] != 0 && acc[4] <= tol) {
        status = 0;
        goto finish;
    }
    if (time_limit == 0) {
        status = 2;
        goto finish;
    }
    {
        double *colsum = calloc((size_t)(n ? n : 1), sizeof(double));
        double rowmax = 0;
        for (int64_t i = 0; i < m; i++) {
            double s = 0;
            for (int64_t k = M->A.ptr[i]; k < M->A.ptr[i + 1]; k++) {
                double v = fabs(M->A.val[k]);
                s += v;
                colsum[M->A.idx[k]] += v;
            }
            rowmax = dmax(rowmax, s);
        }
        double colmax = 0;
        for (int64_t j = 0; j < n; j++) colmax = dmax(colmax, colsum[j]);
        free(colsum);
        double norm = sqrt(rowmax) * sqrt(colmax);
        double step = norm > 0 ? .9 / norm : 1, weight = 1;
        if (adaptive) {
            long double c2 = 0, b2 = 0;
            for (int64_t j = 0; j < n; j++) c2 += (long double)M->c[j] * M->c[j];
            for (int64_t i = 0; i < m; i++) {
                double b = dclamp(0., M->rl[i], M->ru[i]);
                b2 += (long double)b * b;
            }
            if (c2 > 1e-24 && b2 > 1e-24) weight = dclamp(sqrt((double)(c2 / b2)), 1e-4, 1e4);
        }
        orc_backend *B = orc_backend_new(M, x, y, adaptive, 0, 0, 0);
        double restart_kkt = acc[4];
        int64_t since_restart = 0, previous_rejected = 0;
        while (iterations < iteration_limit) {
            if (now_s() - start >= time_limit) {
                status = 2;
                break;
            }
            int64_t left = iteration_limit - iterations;
            int count = (int)(left < check_every ? left : check_every);
            double tick = now_s();
            int accepted = orc_backend_advance(B, count, step / weight, step * weight);
            iteration_seconds += now_s() - tick;
            if (accepted < 0) {
                status = 3;
                break;
            }
            iterations += accepted;
            since_restart += accepted;
            int64_t rej = orc_backend_rejected(B);
            rejected_total += rej - previous_rejected;
            previous_rejected = rej;
            tick = now_s();
            orc_backend_candidates(B, cx, cy, ax_, ay_);
            RESTORE_X(cx, ox);
            RESTORE_Y(cy, oy);
            orc_verify(S, ox, oy, 0, ca);
            RESTORE_X(ax_, aox);
            RESTORE_Y(ay_, aoy);
            orc_verify(S, aox, aoy, 0, aa);
            int avg = aa[4] < ca[4];
            if (avg) {
                SWAP(cx, ax_);
                SWAP(cy, ay_);
                SWAP(ox, aox);
                SWAP(oy, aoy);
                memcpy(ca, aa, sizeof ca);
            }
            if (ca[9] != 0 && ca[4] < acc[4]) {
                memcpy(rx, ox, (size_t)n * sizeof(double));
                memcpy(ry, oy, (size_t)m * sizeof(double));
                memcpy(acc, ca, sizeof acc);
            }
            verification_seconds += now_s() - tick;
            if (ca[9] == 0) {
                status = 3;
                break;
            }
            if (ca[4] <= tol) orc_verify(S, ox, oy, 1, ca);
            if (ca[4] <= tol) {
                memcpy(rx, ox, (size_t)n * sizeof(double));
                memcpy(ry, oy, (size_t)m * sizeof(double));
                memcpy(acc, ca, sizeof acc);
                status = 0;
                break;
            }
            int64_t half = iterations / 2;
            int restart_due = since_restart >= (int64_t)check_every * 2 &&
                              (ca[4] < .5 * restart_kkt || since_restart >= (half > 2000 ? half : 2000));
            if (restart && restart_due) {
                if (adaptive) {
                    long double dx = 0, dy = 0;
                    for (int64_t j = 0; j < n; j++)
                        dx += (long double)(cx[j] - epochx[j]) * (cx[j] - epochx[j]);
                    for (int64_t i = 0; i < m; i++)
                        dy += (long double)(cy[i] - epochy[i]) * (cy[i] - epochy[i]);
                    if (dx > 1e-24 && dy > 1e-24) {
                        double target = dclamp(sqrt((double)(dy / dx)), 1e-4, 1e4);
                        weight = sqrt(weight * target);
                        weight_updates++;
                    }
                }
                orc_backend_reset(B, cx, cy);
                memcpy(epochx, cx, (size_t)n * sizeof(double));
                memcpy(epochy, cy, (size_t)m * sizeof(double));
                restart_kkt = ca[4];
                since_restart = 0;
                restarts++;
            }
        }
        orc_backend_free(B);
    }
finish:
    orc_verify(S, rx, ry, 1, acc);
    if (status == 0 && (acc[9] == 0 || acc[4] > tol)) status = 3;
    if (x_out) memcpy(x_out, rx, (size_t)n * sizeof(double));
    if (y_out) memcpy(y_out, ry, (size_t)m * sizeof(double));
    double s[14] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[9], (double)iterations,
                    (double)restarts, (double)rejected_total, (double)weight_updates,
                    now_s() - start, iteration_seconds, verification_seconds, (double)status};
    memcpy(stats, s, sizeof s);
#undef RESTORE_X
#undef RESTORE_Y
    free(x); free(y); free(rx); free(ry); free(ox); free(oy); free(aox); free(aoy);
    free(cx); free(cy); free(ax_); free(ay_); free(epochx); free(epochy); free(cs); free(rs);
    orc_model_free(M);
    return 0;
}

/* ------------------------------------------------------------------ bound propagation
 * Directed-rounding arithmetic: each operation runs under its own rounding
 * mode (the file is compiled with -frounding-math, and results pass through
 * volatile so the operation happens while the mode is set). */
static double rounded(int mode, int op, double a, double b) {
    volatile double x = a, y = b, r;
    fesetround(mode);
    switch (op) {
    case 0: r = x + y; break;
    case 1: r = x - y; break;
    case 2: r = x * y; break;
    default: r = x / y; break;
    }
    fesetround(FE_TONEAREST);
    return r;
}
#define ADD_DN(a, b) rounded(FE_DOWNWARD, 0, a, b)
#define ADD_UP(a, b) rounded(FE_UPWARD, 0, a, b)
#define SUB_DN(a, b) rounded(FE_DOWNWARD, 1, a, b)
#define SUB_UP(a, b) rounded(FE_UPWARD, 1, a, b)
#define MUL_DN(a, b) rounded(FE_DOWNWARD, 2, a, b)
#define MUL_UP(a, b) rounded(FE_UPWARD, 2, a, b)
#define DIV_DN(a, b) rounded(FE_DOWNWARD, 3, a, b)
#define DIV_UP(a, b) rounded(FE_UPWARD, 3, a, b)

/* propagate_rows and the pass loop of cuda_propagate_integer_bounds
 * (src/cuda.cu:468-529, 1110-1134): proposals of a pass read the bounds of the
 * previous pass; the tightest proposal per column wins. */
int orc_propagate_bounds(int64_t m, int64_t n, const int64_t *ptr, const int64_t *idx,
                         const double *val, const int *integer, const double *rl, const double *ru,
                         double *lb, double *ub, int passes) {
    if (m == 0 || passes == 0)
        return 1;
    double *olb = malloc(sizeof(double) * (size_t)(n ? n : 1));
    double *oub = malloc(sizeof(double) * (size_t)(n ? n : 1));
    int failed = 0;
    for (int pass = 0; pass < passes; ++pass) {
        memcpy(olb, lb, sizeof(double) * (size_t)n);
        memcpy(oub, ub, sizeof(double) * (size_t)n);
        for (int64_t row = 0; row < m; ++row) {
            double low = 0, high = 0;
            int low_inf = 0, high_inf = 0;
            for (int64_t k = ptr[row]; k < ptr[row + 1]; ++k) {
                double v = val[k];
                if (v == 0)
                    continue;
                int64_t j = idx[k];
                double lo = MUL_DN(v, v > 0 ? olb[j] : oub[j]);
                double hi = MUL_UP(v, v > 0 ? oub[j] : olb[j]);
                if (isinf(lo))
                    ++low_inf;
                else
                    low = ADD_DN(low, lo);
                if (isinf(hi))
                    ++high_inf;
                else
                    high = ADD_UP(high, hi);
            }
            if ((!low_inf && low > ru[row]) || (!high_inf && high < rl[row]))
                failed = 1;
            for (int64_t k = ptr[row]; k < ptr[row + 1]; ++k) {
                double v = val[k];
                if (v == 0)
                    continue;
                int64_t j = idx[k];
                double end_low = v > 0 ? olb[j] : oub[j], end_high = v > 0 ? oub[j] : olb[j];
                double term_low = MUL_DN(v, end_low), term_high = MUL_UP(v, end_high);
                int tl = isinf(term_low) ? 1 : 0, th = isinf(term_high) ? 1 : 0;
                double rest_low = (low_inf - tl) ? -INFINITY
                                  : tl           ? low
                                                 : SUB_DN(low, MUL_UP(v, end_low));
                double rest_high = (high_inf - th) ? INFINITY
                                   : th            ? high
                                                   : SUB_UP(high, MUL_DN(v, end_high));
                double l = -INFINITY, u = INFINITY;
                if (isfinite(rl[row]) && isfinite(rest_high)) {
                    double num = SUB_DN(rl[row], rest_high);
                    if (v > 0)
                        l = DIV_DN(num, v);
                    else
                        u = DIV_UP(num, v);
                }
                if (isfinite(ru[row]) && isfinite(rest_low)) {
                    double num = SUB_UP(ru[row], rest_low);
                    if (v > 0)
                        u = DIV_UP(num, v);
                    else
                        l = DIV_DN(num, v);
                }
                int whole = integer[j] != 0;
                if (isfinite(l) && (!whole || fabs(l) < 4503599627370496.0)) {
                    double t = whole ? ceil(l) : l;
                    if (t > lb[j])
                        lb[j] = t;
                }
                if (isfinite(u) && (!whole || fabs(u) < 4503599627370496.0)) {
                    double t = whole ? floor(u) : u;
                    if (t < ub[j])
                        ub[j] = t;
                }
            }
        }
    }
    free(olb);
    free(oub);
    if (failed)
        return 0;
    for (int64_t j = 0; j < n; ++j)
        if (lb[j] > ub[j])
            return 0;
    return 1;
}
