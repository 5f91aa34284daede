// SP2 density-matrix purification driver over the bml API (the consumer loop
// that PROGRESS/LATTE build on bml_multiply_x2, bml_add and bml_copy).
#include "internal.h"

#include <chrono>
#include <cmath>
#include <cstdlib>

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
    // X0 = (emax I - H) / (emax - emin) with Gershgorin bounds.
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
    if (bml_b200_last_error())
        return bml_b200_last_error();

    bml_matrix_t *X2 = bml_zero_matrix(bml_get_type(D), bml_get_precision(D), bml_get_N(D),
                                       bml_get_M(D), sequential);
    if (!X2)
        return bml_b200_last_error();

    int status = BML_B200_OK;
    int rule = 3;
    int it = 0;
    double best = HUGE_VAL;
    int since_best = 0;
    double last_idem = 0.0;
    double x2_seconds = 0.0;
    int max_width = 0;
    for (; it < maxiter; ++it)
    {
        double tr[2];
        const auto t0 = std::chrono::steady_clock::now();
        status = bml_b200_multiply_x2(D, X2, threshold, tr);
        x2_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (bml_get_type(D) == ellpack && bml_b200_last_required_M() > max_width)
            max_width = bml_b200_last_required_M();
        if (status != BML_B200_OK)
        {
            rule = 4;
            break;
        }
        const double t = tr[0], t2 = tr[1];
        last_idem = fabs(t - t2);
        if (fabs(t2 - occupation) <= fabs(2.0 * t - t2 - occupation))
            bml_copy(X2, D);
        else
            bml_add(D, X2, 2.0, -1.0, threshold);
        if (bml_b200_last_error())
        {
            status = bml_b200_last_error();
            rule = 4;
            ++it;
            break;
        }
        if (last_idem < tol)
        {
            rule = 1;
            ++it;
            break;
        }
        if (stall > 0)
        {
            if (last_idem < best)
            {
                best = last_idem;
                since_best = 0;
            }
            else if (++since_best >= stall)
            {
                rule = 2;
                ++it;
                break;
            }
        }
    }
    bml_deallocate(&X2);
    inf[0] = it;
    inf[1] = rule;
    inf[2] = status == BML_B200_OK ? bml_trace(D) : 0.0;
    inf[3] = last_idem;
    inf[4] = max_width;
    inf[5] = x2_seconds;
    return status;
}
