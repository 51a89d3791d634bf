/* nk_pdhg.h -- C ABI of the B200 PDHG engine (libnkpdhg.so).
 *
 * The engine replaces the reference's CUDA iteration backend: every function of
 * the nk_pdhg_* family implements one member of the reference's plugin
 * interface `IterationBackend` (src/internal.hpp:102-124) and its factory
 * `cuda_backend()` (src/internal.hpp:129-134), with the semantics of the
 * reference's CUDA implementation `CudaBackend` (src/cuda.cu:565-950).  The
 * C++ adapter that plugs these calls into the reference's host code lives in
 * niryukti_b200/bridge/vantage_cuda_bridge.cpp.
 *
 * Conventions (mirroring the reference's C API, src/c_api.cpp:11-37):
 *   - every call returns an nk_status; on failure nk_last_error() holds a
 *     thread-local message; no C++ exception crosses this boundary;
 *   - the caller owns every host array; the engine copies what it keeps;
 *   - a handle is single-threaded (one CUDA stream); distinct handles may be
 *     used concurrently from different threads;
 *   - matrices arrive in the reference's CSR layout (int64 ptr/index, double
 *     values, src/model.cpp:11-38), canonical: rows sorted, columns strictly
 *     increasing inside a row.
 */
#ifndef NK_PDHG_H
#define NK_PDHG_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NK_OK = 0,
    NK_ERR_INVALID = 1,     /* bad argument or inconsistent model */
    NK_ERR_CUDA = 2,        /* CUDA runtime failure */
    NK_ERR_MEMORY = 3,      /* device memory guard or allocation failure */
    NK_ERR_STALLED = 4,     /* backtracking stalled / non-finite fixed step */
    NK_ERR_UNSUPPORTED = 5, /* option combination the engine refuses */
    NK_ERR_NO_DEVICE = 6    /* no CUDA device visible */
} nk_status;

/* CSR matrix in host memory, reference layout (vantage::Sparse,
 * include/vantage/vantage.hpp:17-24). */
typedef struct {
    int64_t rows, cols;
    const int64_t *ptr;   /* rows + 1 */
    const int64_t *index; /* ptr[rows] */
    const double *value;  /* ptr[rows] */
} nk_csr;

/* Matrix precisions (the reference's --matrix-precision, src/cuda.cu:117-160). */
#define NK_PRECISION_FP64 0  /* FP64 values, FP64 accumulation */
#define NK_PRECISION_MIXED 1 /* FP32 values, FP64 vectors and accumulation (reference "mixed") */
#define NK_PRECISION_FP32 2  /* FP32 values, FP32 gathered vectors and FP32 accumulation;
                                iterates, averages, reductions and control stay FP64 */

/* Options of cuda_backend() (src/internal.hpp:129-134). */
typedef struct {
    int adaptive;          /* adaptive step acceptance (src/cuda.cu:300-312) */
    int halpern;           /* Halpern anchoring (src/cuda.cu:316-327) */
    double reflection;     /* Halpern reflection in [0, 1] */
    int residual_restarts; /* fixed-point residual restart requests */
    int graphs;            /* replay trials from CUDA graphs */
    int index_bits;        /* 0 = auto (32 when it fits), 32 or 64 (--gpu-indices) */
    int precision;         /* NK_PRECISION_* */
} nk_pdhg_options;

typedef struct nk_pdhg nk_pdhg;

/* cuda_backend(model, x, y, ...) -- src/internal.hpp:129-134, src/cuda.cu:1288-1303.
 * A is m x n; Q (n x n, exactly symmetric) may be NULL or empty.  c, q, lb, ub
 * have n entries, rl, ru m entries, x0 n and y0 m.  Applies the reference's
 * memory guard ("Estimated GPU storage exceeds 80% of available memory"). */
nk_status nk_pdhg_create(const nk_csr *A, const nk_csr *Q, const double *c, const double *q,
                         const double *lb, const double *ub, const double *rl, const double *ru,
                         const double *x0, const double *y0, const nk_pdhg_options *opts,
                         nk_pdhg **out);
void nk_pdhg_destroy(nk_pdhg *h);

/* Pointer arguments of the entries below are required unless their comment
 * says a null one is skipped; a null required pointer or handle returns
 * NK_ERR_INVALID. */

/* IterationBackend::advance(count, tau, sigma) -- src/internal.hpp:105,
 * src/cuda.cu:816-866.  Runs `count` PDHG trials with base steps tau, sigma;
 * *accepted receives the accepted progress.  Like the reference CUDA backend it
 * fails with NK_ERR_STALLED after four chunks without progress, or when a
 * fixed-step run produced a non-finite step. */
nk_status nk_pdhg_advance(nk_pdhg *h, int count, double tau, double sigma, int *accepted);

/* IterationBackend::rejected_steps / restart_requested -- src/internal.hpp:108-113. */
nk_status nk_pdhg_rejected_steps(nk_pdhg *h, int64_t *out);
nk_status nk_pdhg_restart_requested(nk_pdhg *h, int *out);

/* IterationBackend::monitor -- src/internal.hpp:114-116, src/cuda.cu:657-738:
 * scaled-space KKT proxy, min over the current and averaged points. */
nk_status nk_pdhg_monitor(nk_pdhg *h, double *out);

/* IterationBackend::candidates(x, y, xa, ya) -- src/internal.hpp:117-118,
 * src/cuda.cu:867-891: copies the current and averaged iterates to the host
 * arrays (n, m, n, m entries) and rebases the resident A*x.  A null array is
 * skipped. */
nk_status nk_pdhg_candidates(nk_pdhg *h, double *x, double *y, double *xa, double *ya);

/* IterationBackend::reset_candidate(average) -- src/internal.hpp:120-122,
 * src/cuda.cu:892-930: restart from the resident current (0) or averaged (1)
 * point without host uploads. */
nk_status nk_pdhg_reset_candidate(nk_pdhg *h, int average);

/* IterationBackend::reset(x, y) -- src/internal.hpp:123, src/cuda.cu:931-949. */
nk_status nk_pdhg_reset(nk_pdhg *h, const double *x, const double *y);

/* IterationBackend::snapshot / restore -- src/internal.hpp:106-107,
 * src/cuda.cu:739-770.  The snapshot is a list of `parts` vectors; sizes first
 * (nk_pdhg_snapshot_layout), then the flattened values.  restore() accepts only
 * a snapshot of an engine of the same shape and options. */
nk_status nk_pdhg_snapshot_layout(nk_pdhg *h, int *parts, int64_t *part_sizes /* >= 16 */);
nk_status nk_pdhg_snapshot(nk_pdhg *h, double *out);
nk_status nk_pdhg_restore(nk_pdhg *h, const double *in, const int64_t *part_sizes, int parts);

/* Engine statistics for benchmarking: trials launched so far and the device
 * memory the handle holds. */
nk_status nk_pdhg_stats(nk_pdhg *h, int64_t *trials, int64_t *device_bytes);

/* Profiling (no reference counterpart): runs `count` trials one at a time with
 * CUDA events around each kernel on the engine's stream and returns the mean
 * duration of the fused primal (A^T y + primal step) and dual (A dx + dual step
 * + decision) steps in milliseconds; the dual step includes the panel kernel
 * when A's long rows are stored by column panel.  With graphs on, each trial
 * replays one captured trial whose events are graph nodes, as the graph path
 * runs it.  The trials advance the iterate. */
nk_status nk_pdhg_profile(nk_pdhg *h, int count, double tau, double sigma, double *ms_primal,
                          double *ms_dual);
/* The same, kernel by kernel: ms[0] the primal kernel, ms[1] the panel kernel
 * (0 when A has no panels), ms[2] the dual kernel. */
nk_status nk_pdhg_profile_kernels(nk_pdhg *h, int count, double tau, double sigma,
                                  double ms[3]);
/* Layout of the dual SpMV (no reference counterpart): how many of A's rows
 * (its longest, past the SELL split length) are stored by column panel, the
 * panel width in columns, the number of panels, the number of runs (a long
 * row's entries in one panel, cut into pieces of 64 or more entries where
 * they would hold up a lane; each run has its own partial sum) (all 0 without
 * panels), and the kernel launches per trial.  Null outputs are skipped. */
nk_status nk_pdhg_layout_info(nk_pdhg *h, int64_t *long_rows, int64_t *panel_width,
                              int *panels, int64_t *runs, int *kernels_per_trial);
/* Profiling (no reference counterpart): mean duration in milliseconds of `reps`
 * plain SpMVs (no fused epilogue) with A (which = 0, input x) or A^T (which = 1,
 * input y) on the resident iterate; results go to scratch, iterates unchanged. */
nk_status nk_pdhg_time_spmv(nk_pdhg *h, int which, int reps, double *ms);
/* The CUDA stream (cudaStream_t) every kernel and copy of this handle runs on,
 * for callers that time the engine with CUDA events. */
nk_status nk_pdhg_stream(nk_pdhg *h, void **stream);
/* Row schedule chosen for A and A^T: sub-warp width, long-row threshold, items.
 * Null outputs are skipped. */
nk_status nk_pdhg_schedule_info(nk_pdhg *h, int *a_width, int64_t *a_long, int *at_width,
                                int64_t *at_long, int *a_items, int *at_items);

/* ------------------------------------------------------------------ solve
 * Device-resident continuous solve: the reference's solve_continuous for
 * method "pdhg" (src/solver.cpp:213-780) -- presolve and scaling on the host
 * (prepare, src/preprocess.cpp:133-346, bit-identical), the PDHG iterations,
 * candidate evaluation, restarts and primal-weight updates on the GPU, and
 * the reference's outward-rounded Verifier (src/verify.cpp:103-244) on the
 * host to certify termination.  Polishing and the Halpern methods stay with
 * the reference's own driver (which reaches this engine through nk_pdhg_*). */

/* Termination status (the reference's Result::status strings). */
#define NK_SOLVE_OPTIMAL 0
#define NK_SOLVE_INFEASIBLE 1
#define NK_SOLVE_UNBOUNDED 2
#define NK_SOLVE_ITERATION_LIMIT 3
#define NK_SOLVE_TIME_LIMIT 4
#define NK_SOLVE_NUMERICAL_ERROR 5
#define NK_SOLVE_INTERRUPTED 6

/* The continuous part of vantage::Model (include/vantage/vantage.hpp:26-39):
 * minimise offset + c'x + 1/2 sum q_j x_j^2 + 1/2 x'Qx
 * subject to rl <= A x <= ru, lb <= x <= ub.  Q (n x n) may have rows = 0. */
typedef struct {
    nk_csr A, Q;
    const double *c, *q, *lb, *ub, *rl, *ru;
    double offset;
} nk_model;

/* vantage::Options fields the PDHG path reads (include/vantage/vantage.hpp:41-60);
 * nk_solve_defaults() fills the reference's defaults. */
typedef struct {
    double tol;               /* relative KKT tolerance (1e-6) */
    double time_limit;        /* seconds (60) */
    int64_t iteration_limit;  /* accepted iterations (100000) */
    int check_every;          /* iterations between candidate checks (100) */
    int presolve;             /* 1 */
    int scaling_combined;     /* 0 = "ruiz", 1 = "combined" */
    int scaling_passes;       /* 5 */
    int adaptive;             /* adaptive steps (1) */
    int restart;              /* restarts (1) */
    int graphs;               /* replay trials from CUDA graphs (1) */
    int index_bits;           /* 0, 32 or 64 */
    int precision;            /* NK_PRECISION_* of the first phase (FP64) */
    int refine;               /* after a reduced-precision phase, finish in FP64 (1) */
    double phase_tol;         /* target of the reduced-precision phase (0: 10 * tol) */
    int verbose;              /* per-check line on stderr (0) */
    const double *initial_x;  /* optional, n entries */
    const double *initial_y;  /* optional, m entries */
    const volatile int *cancel; /* optional: another thread sets *cancel != 0 to stop the
                                   solve at its next check (INTERRUPTED) -- the reference's
                                   Options::cancellation token (src/internal.hpp:9-11) */
} nk_solve_options;

/* vantage::Result fields of the continuous path (include/vantage/vantage.hpp:112-140). */
typedef struct {
    int status;                 /* NK_SOLVE_* */
    int64_t iterations, restarts, rejected_steps, weight_updates;
    int64_t device_checks, host_checks, removed_rows, removed_columns;
    int64_t phase_iterations;   /* iterations of the reduced-precision phase */
    int64_t refine_iterations;  /* iterations of the FP64 refinement */
    double seconds, preprocess_seconds, transfer_seconds, iteration_seconds,
        verification_seconds, phase_seconds;
    /* certified accuracy of the returned point (Verifier::evaluate) */
    double objective, kkt, primal, dual, gap, lower_bound;
    /* accuracy of the reduced-precision phase's best point (no safe bound) */
    double phase_objective, phase_kkt, phase_primal, phase_dual, phase_gap;
    /* seconds from the call until the device estimate of the best candidate's
     * relative KKT error first fell to 10^-k (k = 0..8); -1: never */
    double reached[9];
} nk_solve_result;

/* prepare(model, options) -- src/preprocess.cpp:133-346: presolve (fixed and
 * unused columns, empty, redundant and duplicate rows) and Ruiz / combined
 * scaling, bit-identical to the reference.  dims = {rows, cols, nnz, qnnz,
 * failure}: failure 0 none, 1 INFEASIBLE (presolve proof). */
typedef struct nk_prepared nk_prepared;
nk_status nk_prepare(const nk_model *model, int presolve, int scaling_combined, int scaling_passes,
                     nk_prepared **out);
void nk_prepared_free(nk_prepared *p);
nk_status nk_prepared_dims(const nk_prepared *p, int64_t dims[5]);
/* Copies the prepared model and its maps (Prepared, src/internal.hpp:16-25);
 * any pointer may be NULL.  scalars = {objective_scale, offset}. */
nk_status nk_prepared_get(const nk_prepared *p, int64_t *ptr, int64_t *index, double *value,
                          double *c, double *q, double *lb, double *ub, double *rl, double *ru,
                          int64_t *cols, int64_t *rows, int64_t *lower_rows, int64_t *upper_rows,
                          double *fixed, double *column_scale, double *row_scale, double *scalars,
                          int64_t *qptr, int64_t *qindex, double *qvalue);

/* Verifier::evaluate(x, y, safe_bound) -- src/verify.cpp:103-240, bit-identical.
 * accuracy = {objective, primal, dual, gap, kkt, primal_absolute,
 * dual_absolute, complementarity, lower_bound, finite}. */
nk_status nk_verify(const nk_model *model, const double *x, const double *y, int safe_bound,
                    double accuracy[10]);
/* Verifier::infeasibility_bound(y) -- src/verify.cpp:93-101. */
nk_status nk_infeasibility_bound(const nk_model *model, const double *y, double *bound);

void nk_solve_defaults(nk_solve_options *options);
/* Solves the model; x (n) and y (m) receive the returned primal and dual
 * points (either may be NULL).  Errors (invalid model, CUDA failure, memory
 * guard) return a status; termination outcomes are result->status. */
nk_status nk_solve(const nk_model *model, const nk_solve_options *options,
                   nk_solve_result *result, double *x, double *y);

/* cuda_available / cuda_description / hardware_info --
 * include/vantage/vantage.hpp:76,145-146, src/cuda.cu:1267-1287. */
/* ------------------------------------------------------------------ batch
 * Many independent LP / convex-QP solves advanced together on one GPU, each
 * with its own step sizes, adaptive acceptance, restarts, primal weight and
 * termination (the driver of nk_solve per instance).  The reference has one
 * batching entry, cuda_batch_relaxations (src/cuda.cu:1136-1266: box variants
 * of a single LP, fixed steps, no restarts, no QP); this family replaces it
 * for uneven, unrelated instances and is what the serving loop runs on.
 *
 * Instances keep their own device storage and join a work list of
 * (instance, 32-row chunk) pairs; one trial of the batch is three kernel
 * launches for all instances, captured in a CUDA graph per check interval.
 * Kernel variants (unroll depth, CTA size) are chosen by an autotuner that
 * times them on the batch itself.  Instances join and leave at check
 * boundaries.  Handles are single-threaded; nk_batch_prepare is thread-safe
 * and touches no device, so requests can be prepared while the batch runs. */
typedef struct {
    double tol;               /* relative KKT tolerance of the batch (1e-6) */
    double time_limit;        /* per instance, from admission (60 s); nk_batch_prepare
                                 takes an instance's limits from its own options */
    int64_t iteration_limit;  /* per instance (100000) */
    int check_every;          /* trials between candidate checks (100) */
    int presolve, scaling_combined, scaling_passes, adaptive, restart, graphs;
    int autotune;             /* time kernel variants on the live batch (1) */
    int precision;            /* NK_PRECISION_FP64 (the default), or MIXED: FP32 values
                                 until an instance's KKT reaches phase_tol or stalls,
                                 then an FP64 refinement restarted from its best point */
    double phase_tol;         /* MIXED phase target (0: 10 * tol) */
    double memory_budget;     /* admission budget in bytes (0: 80% of free memory) */
    int capacity;             /* instance slots (4096) */
} nk_batch_options;
typedef struct nk_batch nk_batch;
typedef struct nk_batch_item nk_batch_item;

void nk_batch_defaults(nk_batch_options *options);
nk_status nk_batch_create(const nk_batch_options *options, nk_batch **out);
void nk_batch_destroy(nk_batch *batch);
/* The reference's device-memory estimate of a model (src/solver.cpp:227-228). */
nk_status nk_batch_estimate(const nk_model *model, double *bytes);
/* Presolve, scale, check the start point and lay out one instance (host only).
 * *device_bytes: what admitting it will take (0 if it terminated already). */
nk_status nk_batch_prepare(const nk_model *model, const nk_batch_options *options,
                           nk_batch_item **out, double *device_bytes);
/* nk_batch_prepare with a start point: x0 (n) and y0 (m) in the caller's
 * order (either may be NULL), taken like Options::initial_x / initial_y.  It
 * serves the warm-started box variants of cuda_batch_relaxations
 * (src/cuda.cu:1136-1160; caller src/mip.cpp:1094-1118). */
nk_status nk_batch_prepare_from(const nk_model *model, const nk_batch_options *options,
                                const double *x0, const double *y0, nk_batch_item **out,
                                double *device_bytes);
void nk_batch_item_free(nk_batch_item *item);
/* Admits a prepared instance under `id`: *admitted = 1 (the batch owns the
 * item now) or 0 (over the memory budget or no free slot; the caller keeps it). */
nk_status nk_batch_admit(nk_batch *batch, nk_batch_item *item, int64_t id, int *admitted);
/* Runs up to `checks` check intervals, stopping early once some instance
 * finished; their ids go to finished[0 .. *count). */
nk_status nk_batch_step(nk_batch *batch, int checks, int64_t *finished, int capacity, int *count);
/* Result of a finished instance (x: its n, y: its m original entries; either
 * may be NULL); releases its slot and device memory. */
nk_status nk_batch_result(nk_batch *batch, int64_t id, nk_solve_result *result, double *x,
                          double *y);
nk_status nk_batch_info(nk_batch *batch, int *active, double *used_bytes, double *budget_bytes,
                        int *variant_primal, int *variant_dual);
/* Progress of a running (or finished, not yet collected) instance: {iterations,
 * restarts, best KKT estimate, primal weight, step, iterations since the last
 * restart, KKT at the last restart, 1 when in FP64}. */
nk_status nk_batch_progress(nk_batch *batch, int64_t id, double progress[8]);
/* Profiling (no reference counterpart): mean time of `trials` batch trials,
 * and the algorithmic bytes of one trial's two SpMV passes over all instances. */
nk_status nk_batch_time_trials(nk_batch *batch, int trials, double *ms, int64_t *bytes_per_trial);
/* Profiling (no reference counterpart): the autotuner's best single-launch
 * times of the batched primal and dual kernels (0 before tuning). */
nk_status nk_batch_kernel_times(nk_batch *batch, double *primal_ms, double *dual_ms);
/* Profiling (no reference counterpart): wall seconds spent so far in the parts
 * of the check intervals: control upload, trials, candidate evaluation,
 * per-instance driver logic on the host (with certification), best-point and
 * restart kernels, closing certification of finished instances, and work-list
 * rebuilds (including kernel tuning and graph capture). */
nk_status nk_batch_phase_seconds(nk_batch *batch, double seconds[7]);

/* KKT proxy without any device allocation.  No counterpart in the reference:
 * it exists for callers that must not allocate device memory themselves --
 * a host application that hands all device memory to its own pool or budget
 * (a solve service admitting work by memory footprint), or a latency-critical
 * loop in which cudaMalloc / cudaFree would synchronise the device.
 *
 * Computes the same scaled KKT proxy as one point of nk_pdhg_monitor (the
 * monitor kernel of src/cuda.cu:387-446) for caller-provided DEVICE vectors:
 * x, c, q, lb, ub, aty (= A^T y) and qx (= Q x, or NULL) of length n; y, ax
 * (= A x), rl, ru of length m; cscale = max(1, 1 + max |c_j|).  The result
 * (one double) is written to the DEVICE pointer `result` on `stream`
 * (a cudaStream_t; NULL = the default stream); nothing is synchronised.
 *
 * The kernel's per-block partial sums and its arrival counter live in one
 * fixed array in the library (about 640 KiB, held on every GPU that loads the
 * library until the process exits), so n and m are limited to
 * NK_MONITOR_STATIC_MAX entries each; larger inputs fail with NK_ERR_INVALID.
 * The first call on each device looks up that array's device address (and
 * may load the module), so make it before any stream capture.  The address is
 * kept for the life of the process: after cudaDeviceReset (or any other
 * teardown of the device's primary context) the array may move, and calls
 * made after such a reset are not supported.  All calls share
 * the array: the counter is cleared on `stream` before every launch, and calls
 * whose kernels can overlap on the GPU (different streams, or different host
 * threads) race and must be serialised by the caller. */
#define NK_MONITOR_STATIC_MAX 4194304
nk_status nk_monitor_static(int64_t n, int64_t m, const double *x, const double *y,
                            const double *ax, const double *aty, const double *qx,
                            const double *c, const double *q, const double *lb, const double *ub,
                            const double *rl, const double *ru, double cscale, double *result,
                            void *stream);

/* cuda_compact_matrix(matrix, rows, columns, output_columns) -- src/cuda.cu:953-1032,
 * called by prepare with --gpu-presolve (src/preprocess.cpp:295-298).  The CSR
 * of the kept rows (kept_rows: `rows` strictly increasing source rows) with the
 * kept columns renumbered (column_map: one entry per source column, -1 drops
 * it, the kept ones strictly increasing below output_columns), entries in
 * their source order.  Host arrays in and out: out_ptr has rows + 1 entries,
 * out_index / out_value `capacity` (at most the kept rows' entries are
 * needed); *out_nnz receives the kept entries.  Counted, scanned and compacted
 * on the GPU. */
nk_status nk_compact_csr(const nk_csr *matrix, int64_t rows, const int64_t *kept_rows,
                         const int64_t *column_map, int64_t output_columns, int64_t *out_ptr,
                         int64_t *out_index, double *out_value, int64_t capacity,
                         int64_t *out_nnz);

/* cuda_propagate_integer_bounds(model, lb, ub, passes) -- src/cuda.cu:448-529,
 * 1033-1135; callers src/solver.cpp:227-240 (--gpu-presolve) and the
 * branch-and-bound nodes (src/mip.cpp:710-720).  `passes` rounds of
 * activity-based bound proposals over A (m x n): per row, the activity range
 * from lb / ub with directed rounding, then for each entry the bound it
 * implies on its column, rounded inward for integer[j] != 0 columns, kept when
 * tighter.  lb / ub (n, host) are updated in place; *feasible = 0 when a row's
 * activity range misses [rl, ru] or a column's bounds cross.  The results are
 * proposals: the reference proves them again on the host before using them. */
nk_status nk_propagate_bounds(const nk_csr *A, const int *integer, const double *rl,
                              const double *ru, double *lb, double *ub, int passes,
                              int *feasible);

/* cuda_linear_solve(matrix, rhs, options, fp32_matrix, tolerance) --
 * src/cuda.cu:1304-1434, the barrier method's Newton systems
 * (src/barrier.cpp:280-300).  BiCGSTAB for K x = rhs (K: n x n CSR, host
 * arrays; FP32 values with FP64 vectors and sums when fp32_matrix), from x = 0,
 * to the residual target (fp32 ? 1e-6 : 1e-10) (1 + |rhs|), at most
 * min(20000, 10 n + 100) iterations.  precondition = 0 runs the reference's
 * iteration exactly; 1 adds a diagonal right preconditioner (|K_ii|, or the
 * row's Schur-complement diagonal where a saddle point's regularised block
 * leaves K_ii near zero), which the barrier's badly scaled Newton matrices
 * need.  x (n) receives the last iterate; *converged = 1 when the target was
 * met, *timed_out = 1 when time_limit seconds ran out first.  The caller checks
 * the residual of x, as the reference does, before using it. */
nk_status nk_linear_solve(const nk_csr *K, const double *rhs, int fp32_matrix, int precondition,
                          double time_limit, double *x, int *converged, int *timed_out);

/* ------------------------------------------------------------------ model file
 * Binary model file (no reference counterpart): the arrays of an nk_model
 * stored raw, so that a large instance loads by mapping a file instead of the
 * text parse the reference does for its JSON and MPS formats
 * (src/io.cpp:84-139,299,800; its Python session passes every model through a
 * temporary JSON file, python/vantage/native.py:26-31).  The layout is given
 * at the top of niryukti_b200/csrc/nk_modelfile.cpp. */
typedef struct nk_model_file nk_model_file;
/* Writes `model` to `path` (through "<path>.tmp" and a rename).  A model
 * without q stores zeros; Q is stored when it has entries.  `maximise` != 0
 * records that the source objective was a maximisation whose minimisation
 * form `model` holds (the reference's Model::sense = -1). */
nk_status nk_model_write(const char *path, const nk_model *model, int maximise);
/* Maps `path` read-only and points *model into the mapping after checking the
 * header, the file size, the checksum and the CSR structure of A and Q;
 * *maximise (may be NULL) receives the recorded sense.  The pointers stay
 * valid until nk_model_close(*file). */
nk_status nk_model_open(const char *path, nk_model_file **file, nk_model *model, int *maximise);
void nk_model_close(nk_model_file *file);
/* The checks of nk_model_open on a file image already in memory (8-byte
 * aligned, `bytes` long); *model points into the image. */
nk_status nk_model_view(const void *image, int64_t bytes, nk_model *model, int *maximise);

int nk_cuda_available(void);
nk_status nk_cuda_description(char *buffer, int length);
/* Whether a CUDA device is present, and its free and total memory in bytes
 * (0 without a device).  Null outputs are skipped. */
nk_status nk_hardware_info(int *available, double *free_bytes, double *total_bytes);

const char *nk_last_error(void);
unsigned nk_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
