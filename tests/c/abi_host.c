/* A plain C99 caller of the engine's C ABI, runnable with or without a GPU:
 * version check, a model-file round trip, presolve/scaling and the verifier,
 * the batch family's host entries, the solve's missing-device status, and the
 * error convention.  Built and run by tests/test_abi.py; it proves that
 * include/nk_pdhg.h is valid C and that the library links without C++.
 *
 * The LP: minimise -x0 - x1 subject to x0 + 2 x1 <= 4, 3 x0 + x1 <= 6,
 * 0 <= x <= 10.  Optimum x = (1.6, 1.2), objective -2.8, row duals
 * y = (0.4, 0.2) in the reference's sign convention (Verifier::evaluate
 * pairs y_i > 0 with the upper row bound, src/verify.cpp:153). */
#include "nk_pdhg.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

static int fail(const char *what) {
    fprintf(stderr, "FAIL %s: %s\n", what, nk_last_error());
    return 1;
}

int main(int argc, char **argv) {
    if (argc != 2)
        return 2;
    if (nk_abi_version() != 1)
        return fail("abi version");

    const int64_t ptr[3] = {0, 2, 4}, index[4] = {0, 1, 0, 1};
    const double value[4] = {1, 2, 3, 1};
    const double c[2] = {-1, -1}, lb[2] = {0, 0}, ub[2] = {10, 10};
    const double rl[2] = {-INFINITY, -INFINITY}, ru[2] = {4, 6};
    nk_model model;
    memset(&model, 0, sizeof model);
    model.A.rows = 2;
    model.A.cols = 2;
    model.A.ptr = ptr;
    model.A.index = index;
    model.A.value = value;
    model.c = c;
    model.lb = lb;
    model.ub = ub;
    model.rl = rl;
    model.ru = ru;

    if (nk_model_write(argv[1], &model, 0) != NK_OK)
        return fail("nk_model_write");
    nk_model_file *file = NULL;
    nk_model view;
    int maximise = -1;
    if (nk_model_open(argv[1], &file, &view, &maximise) != NK_OK)
        return fail("nk_model_open");
    if (view.A.rows != 2 || view.A.cols != 2 || maximise != 0 || view.Q.rows != 0 ||
        memcmp(view.A.value, value, sizeof value) != 0 || memcmp(view.ru, ru, sizeof ru) != 0 ||
        !isinf(view.rl[0]) || view.q[0] != 0.0)
        return fail("model file contents");

    nk_prepared *prepared = NULL;
    int64_t dims[5];
    if (nk_prepare(&view, 1, 0, 5, &prepared) != NK_OK)
        return fail("nk_prepare");
    if (nk_prepared_dims(prepared, dims) != NK_OK)
        return fail("nk_prepared_dims");
    nk_prepared_free(prepared);

    const double x[2] = {1.6, 1.2}, y[2] = {0.4, 0.2};
    double accuracy[10];
    if (nk_verify(&view, x, y, 1, accuracy) != NK_OK)
        return fail("nk_verify");

    /* the batch family's host entries: the reference's memory estimate,
     * 48 B per nonzero + 240 B per row and column, plus two */
    nk_batch_options batch_options;
    nk_batch_defaults(&batch_options);
    double estimate = 0, device_bytes = -1;
    if (nk_batch_estimate(&view, &estimate) != NK_OK || estimate != 48.0 * 4 + 240.0 * 6)
        return fail("nk_batch_estimate");
    nk_batch_item *item = NULL;
    if (nk_batch_prepare(&view, &batch_options, &item, &device_bytes) != NK_OK || !item ||
        !(device_bytes > 0))
        return fail("nk_batch_prepare");
    nk_batch_item_free(item);

    /* the device-resident solve: OPTIMAL on a GPU, NK_ERR_NO_DEVICE without one */
    nk_solve_options solve_options;
    nk_solve_defaults(&solve_options);
    nk_solve_result result;
    double sx[2], sy[2];
    const nk_status solved = nk_solve(&view, &solve_options, &result, sx, sy);
    if (nk_cuda_available() ? (solved != NK_OK || result.status != NK_SOLVE_OPTIMAL)
                            : solved != NK_ERR_NO_DEVICE)
        return fail("nk_solve");
    nk_model_close(file);

    if (nk_model_open("/nonexistent/model.nkm", &file, &view, NULL) != NK_ERR_INVALID ||
        strstr(nk_last_error(), "cannot open") == NULL)
        return fail("error convention");
    if (nk_hardware_info(NULL, NULL, NULL) != NK_OK)
        return fail("nk_hardware_info");

    printf("rows %lld cols %lld objective %.12g kkt %.3g\n", (long long)dims[0],
           (long long)dims[1], accuracy[0], accuracy[4]);
    return 0;
}
