// SP2 density-matrix purification driver over the bml API (the consumer loop
// that PROGRESS/LATTE build on bml_multiply_x2, bml_add and bml_copy), in
// FP64 and in mixed precision (FP32 bulk iterations closed by FP64 ones).
#include "internal.h"

#include <chrono>
#include <cmath>
#include <cstdlib>

namespace {

// State carried across SP2 iterations (and from the FP32 to the FP64 phase).
struct Sp2State
{
    int it = 0;           // iterations run
    int rule = 3;         // 1 tol, 2 stall, 3 maxiter, 4 error
    double best = HUGE_VAL;
    int since_best = 0;
    double last_idem = 0.0;
    double x2_seconds = 0.0;
    int max_width = 0;
};

// Up to `iters` SP2 iterations on X (X2 is scratch of X's type, precision and
// M).  Traces come back from the multiply as FP64 sums of per-row values, and
// the branch choice and the stop tests are made on them in FP64.  Returns the
// status; s.rule is set when a stop rule fires (tol/stall/error).
int sp2_iterate(bml_matrix_t *X, bml_matrix_t *X2, double threshold, double occupation, int iters,
                double tol, int stall, Sp2State &s, bool *stopped)
{
    *stopped = false;
    for (int k = 0; k < iters; ++k)
    {
        double tr[2];
        const auto t0 = std::chrono::steady_clock::now();
        const int status = bml_b200_multiply_x2(X, X2, threshold, tr);
        s.x2_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (bml_get_type(X) == ellpack && bml_b200_last_required_M() > s.max_width)
            s.max_width = bml_b200_last_required_M();
        if (status != BML_B200_OK)
        {
            s.rule = 4;
            *stopped = true;
            return status;
        }
        const double t = tr[0], t2 = tr[1];
        s.last_idem = fabs(t - t2);
        if (fabs(t2 - occupation) <= fabs(2.0 * t - t2 - occupation))
            bml_copy(X2, X);
        else
            bml_add(X, X2, 2.0, -1.0, threshold);
        ++s.it;
        if (bml_b200_last_error())
        {
            s.rule = 4;
            *stopped = true;
            return bml_b200_last_error();
        }
        if (s.last_idem < tol)
        {
            s.rule = 1;
            *stopped = true;
            return BML_B200_OK;
        }
        if (stall > 0)
        {
            if (s.last_idem < s.best)
            {
                s.best = s.last_idem;
                s.since_best = 0;
            }
            else if (++s.since_best >= stall)
            {
                s.rule = 2;
                *stopped = true;
                return BML_B200_OK;
            }
        }
    }
    return BML_B200_OK;
}

// X0 = (emax I - H) / (emax - emin) with Gershgorin bounds, into D.
int sp2_start(bml_matrix_t *H, bml_matrix_t *D)
{
    bml_copy(H, D);
    if (bml_b200_last_error())
        return bml_b200_last_error();
    double *eb = static_cast<double *>(bml_gershgorin(H));
    if (!eb || bml_b200_last_error())
    {
        free(eb);
        return bml_b200_last_error();
    }
    bml_normalize(D, eb[0], eb[1]);
    free(eb);
    return bml_b200_last_error();
}

} // namespace

extern "C" int bml_b200_sp2(bml_matrix_t *H, bml_matrix_t *D, double threshold, double occupation,
                            int maxiter, double tol, int stall, double *info)
{
    double local_info[6] = {0, 4, 0, 0, 0, 0};
    double *inf = info ? info : local_info;
    for (int k = 0; k < 6; k++)
        inf[k] = local_info[k];
    if (!H || !D || H == D || bml_get_type(H) != bml_get_type(D) ||
        bml_get_precision(H) != bml_get_precision(D) || bml_get_N(H) != bml_get_N(D))
    {
        b200_set_error(BML_B200_ERR_INVALID, "sp2: H and D must be distinct matrices of one type, precision and N");
        return BML_B200_ERR_INVALID;
    }
    bml_b200_clear_error();
    int status = sp2_start(H, D);
    if (status)
        return status;
    bml_matrix_t *X2 = bml_zero_matrix(bml_get_type(D), bml_get_precision(D), bml_get_N(D),
                                       bml_get_M(D), sequential);
    if (!X2)
        return bml_b200_last_error();
    Sp2State s;
    bool stopped = false;
    status = sp2_iterate(D, X2, threshold, occupation, maxiter, tol, stall, s, &stopped);
    bml_deallocate(&X2);
    inf[0] = s.it;
    inf[1] = s.rule;
    inf[2] = status == BML_B200_OK ? bml_trace(D) : 0.0;
    inf[3] = s.last_idem;
    inf[4] = s.max_width;
    inf[5] = s.x2_seconds;
    return status;
}

extern "C" int bml_b200_sp2_mixed(bml_matrix_t *H, bml_matrix_t *D, double threshold, double occupation,
                                  int maxiter, double tol, int stall, int nclose, double *info)
{
    double local_info[8] = {0, 4, 0, 0, 0, 0, 0, 0};
    double *inf = info ? info : local_info;
    for (int k = 0; k < 8; k++)
        inf[k] = local_info[k];
    if (!H || !D || H == D || bml_get_type(H) != ellpack || bml_get_type(D) != ellpack ||
        bml_get_precision(H) != double_real || bml_get_precision(D) != double_real ||
        bml_get_N(H) != bml_get_N(D) || nclose < 0 || nclose > maxiter)
    {
        b200_set_error(BML_B200_ERR_INVALID,
                       "sp2_mixed: H and D must be distinct double_real ELLPACK matrices of one N, "
                       "0 <= nclose <= maxiter");
        return BML_B200_ERR_INVALID;
    }
    bml_b200_clear_error();
    int status = sp2_start(H, D); // Gershgorin bounds and X0 in FP64
    if (status)
        return status;
    const int N = bml_get_N(D), M = bml_get_M(D);
    bml_matrix_t *X = bml_zero_matrix(ellpack, single_real, N, M, sequential);
    bml_matrix_t *X2 = bml_zero_matrix(ellpack, single_real, N, M, sequential);
    bml_matrix_t *D2 = nullptr;
    Sp2State s;
    bool stopped = false;
    if (!X || !X2)
    {
        status = bml_b200_last_error();
        goto done;
    }
    // bulk: FP32 products and sums, FP64 traces, branch and stop tests
    if (!ell_convert(static_cast<bml_matrix_ellpack_t *>(D), static_cast<bml_matrix_ellpack_t *>(X)))
    {
        status = bml_b200_last_error();
        goto done;
    }
    // the FP32 products may take the dense tier's f32 reduction (subnormal
    // sums flush to zero, below the FP32 iterations' rounding anyway)
    ell_set_f32_reduce(true);
    status = sp2_iterate(X, X2, threshold, occupation, maxiter - nclose, tol, stall, s, &stopped);
    ell_set_f32_reduce(false);
    inf[6] = s.it;
    inf[7] = s.x2_seconds;
    if (status != BML_B200_OK)
        goto done;
    // closing refinement in FP64
    if (!ell_convert(static_cast<bml_matrix_ellpack_t *>(X), static_cast<bml_matrix_ellpack_t *>(D)))
    {
        status = bml_b200_last_error();
        goto done;
    }
    D2 = bml_zero_matrix(ellpack, double_real, N, M, sequential);
    if (!D2)
    {
        status = bml_b200_last_error();
        goto done;
    }
    {
        const int rule_bulk = s.rule;
        status = sp2_iterate(D, D2, threshold, occupation, nclose, -1.0, 0, s, &stopped);
        if (status == BML_B200_OK)
            s.rule = rule_bulk;
    }
done:
    if (X)
        bml_deallocate(&X);
    if (X2)
        bml_deallocate(&X2);
    if (D2)
        bml_deallocate(&D2);
    inf[0] = s.it;
    inf[1] = s.rule;
    inf[2] = status == BML_B200_OK ? bml_trace(D) : 0.0;
    inf[3] = s.last_idem;
    inf[4] = s.max_width;
    inf[5] = s.x2_seconds;
    return status;
}
