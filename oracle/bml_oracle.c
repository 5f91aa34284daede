/*
 * CPU oracle for the ELLPACK / ELLBLOCK thresholded-multiply path.
 * TEST INFRASTRUCTURE ONLY (see bml_oracle.h).  Serial restatement of the
 * reference loops; each function cites the loop it follows.  Built with
 * -ffp-contract=off so that `x + a*b` is a rounded product then a rounded sum,
 * as in the reference's -std=c99 build.
 */
#include "bml_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- ELLPACK X^2 / A*B: row Gustavson with a dense scatter array ---------
 * ellpack/bml_multiply_ellpack_typed.c:252-333 (X^2) and :468-542 (A*B):
 * x[k] = 0 on first touch, x[k] = x[k] + a*b after; the touched columns are
 * visited in first-touch order and kept if k == i or |x| > thr. */
#define DEFINE_GUSTAVSON(NAME, REAL)                                                       \
    static int NAME(int N, int MA, const REAL *av, const int *aix, const int *anz,        \
                    int MB, const REAL *bv, const int *bix, const int *bnz, double thr,    \
                    int MC, REAL *cv, int *cix, int *cnz, double *trace, int check_pre)    \
    {                                                                                      \
        int *ix = calloc((size_t) N, sizeof(int));                                        \
        int *jx = calloc((size_t) N, sizeof(int));                                        \
        REAL *x = calloc((size_t) N, sizeof(REAL));                                       \
        REAL trX = 0, trX2 = 0;                                                            \
        int maxw = 0;                                                                      \
        for (int i = 0; i < N; i++)                                                        \
        {                                                                                  \
            int l = 0;                                                                     \
            for (int jp = 0; jp < anz[i]; jp++)                                            \
            {                                                                              \
                REAL a = av[(size_t) i * MA + jp];                                         \
                int j = aix[(size_t) i * MA + jp];                                         \
                if (j == i)                                                                \
                    trX = trX + a;                                                         \
                for (int kp = 0; kp < bnz[j]; kp++)                                        \
                {                                                                          \
                    int k = bix[(size_t) j * MB + kp];                                     \
                    if (ix[k] == 0)                                                        \
                    {                                                                      \
                        x[k] = 0.0;                                                        \
                        jx[l++] = k;                                                       \
                        ix[k] = i + 1;                                                     \
                    }                                                                      \
                    x[k] = x[k] + a * bv[(size_t) j * MB + kp];                            \
                }                                                                          \
            }                                                                              \
            int ll = 0;                                                                    \
            for (int q = 0; q < l; q++)                                                    \
            {                                                                              \
                int k = jx[q];                                                             \
                REAL xt = x[k];                                                            \
                int keep = 0;                                                              \
                if (k == i)                                                                \
                {                                                                          \
                    trX2 = trX2 + xt;                                                      \
                    keep = 1;                                                              \
                }                                                                          \
                else if (fabs((double) xt) > (sizeof(REAL) == 4 ? (double) (float) thr : thr)) \
                    keep = 1;                                                              \
                if (keep)                                                                  \
                {                                                                          \
                    if (ll < MC)                                                           \
                    {                                                                      \
                        cv[(size_t) i * MC + ll] = xt;                                     \
                        cix[(size_t) i * MC + ll] = k;                                     \
                    }                                                                      \
                    ll++;                                                                  \
                }                                                                          \
                ix[k] = 0;                                                                 \
                x[k] = 0.0;                                                                \
            }                                                                              \
            cnz[i] = ll < MC ? ll : MC;                                                    \
            int w = check_pre ? (l > ll ? l : ll) : ll;                                    \
            if (w > maxw)                                                                  \
                maxw = w;                                                                  \
        }                                                                                  \
        if (trace)                                                                         \
        {                                                                                  \
            trace[0] = (double) trX;                                                       \
            trace[1] = (double) trX2;                                                      \
        }                                                                                  \
        free(ix);                                                                          \
        free(jx);                                                                          \
        free(x);                                                                           \
        return maxw;                                                                       \
    }

DEFINE_GUSTAVSON(gustavson_d, double)
DEFINE_GUSTAVSON(gustavson_f, float)

int oracle_ellpack_x2_d(int N, int M, const double *v, const int *ix, const int *nz,
                        double thr, int M2, double *v2, int *ix2, int *nz2, double *trace)
{
    return gustavson_d(N, M, v, ix, nz, M, v, ix, nz, thr, M2, v2, ix2, nz2, trace, 0);
}

int oracle_ellpack_x2_f(int N, int M, const float *v, const int *ix, const int *nz,
                        double thr, int M2, float *v2, int *ix2, int *nz2, double *trace)
{
    return gustavson_f(N, M, v, ix, nz, M, v, ix, nz, thr, M2, v2, ix2, nz2, trace, 0);
}

int oracle_ellpack_ab_d(int N, int MA, const double *av, const int *aix, const int *anz,
                        int MB, const double *bv, const int *bix, const int *bnz,
                        double thr, int MC, double *cv, int *cix, int *cnz)
{
    return gustavson_d(N, MA, av, aix, anz, MB, bv, bix, bnz, thr, MC, cv, cix, cnz, NULL, 1);
}

/* ---- add: ellpack/bml_add_ellpack_typed.c:161-205 --------------------------- */
void oracle_ellpack_add_d(int N, int MA, double *av, int *aix, int *anz, int MB,
                          const double *bv, const int *bix, const int *bnz, double alpha,
                          double beta, double thr)
{
    int *ix = calloc((size_t) N, sizeof(int));
    int *jx = calloc((size_t) N, sizeof(int));
    double *x = calloc((size_t) N, sizeof(double));
    for (int i = 0; i < N; i++)
    {
        int l = 0;
        if (alpha > 0.0 || alpha < 0.0)
            for (int jp = 0; jp < anz[i]; jp++)
            {
                int k = aix[(size_t) i * MA + jp];
                if (ix[k] == 0)
                {
                    x[k] = 0.0;
                    ix[k] = i + 1;
                    jx[l++] = k;
                }
                x[k] = x[k] + alpha * av[(size_t) i * MA + jp];
            }
        if (beta > 0.0 || beta < 0.0)
            for (int jp = 0; jp < bnz[i]; jp++)
            {
                int k = bix[(size_t) i * MB + jp];
                if (ix[k] == 0)
                {
                    x[k] = 0.0;
                    ix[k] = i + 1;
                    jx[l++] = k;
                }
                x[k] = x[k] + beta * bv[(size_t) i * MB + jp];
            }
        int ll = 0;
        for (int q = 0; q < l; q++)
        {
            int k = jx[q];
            double xt = x[k];
            if (fabs(xt) > thr && ll < MA)
            {
                av[(size_t) i * MA + ll] = xt;
                aix[(size_t) i * MA + ll] = k;
                ll++;
            }
            x[k] = 0.0;
            ix[k] = 0;
        }
        anz[i] = ll;
    }
    free(ix);
    free(jx);
    free(x);
}

/* ---- add_identity: ellpack/bml_add_ellpack_typed.c:492-531 ------------------ */
void oracle_ellpack_add_identity_d(int N, int M, double *v, int *ix, int *nz, double beta,
                                   double thr)
{
    double *x = malloc(sizeof(double) * (size_t) (M + 1));
    int *jx = malloc(sizeof(int) * (size_t) (M + 1));
    for (int i = 0; i < N; i++)
    {
        int l = 0, diag = -1;
        for (int jp = 0; jp < nz[i]; jp++)
        {
            int k = ix[(size_t) i * M + jp];
            if (k == i)
                diag = jp;
            x[jp] = v[(size_t) i * M + jp];
            jx[jp] = k;
            l++;
        }
        if (beta > 0.0 || beta < 0.0)
        {
            if (diag == -1)
            {
                x[l] = beta;
                jx[l] = i;
                l++;
            }
            else
                x[diag] = x[diag] + beta;
        }
        int ll = 0;
        for (int jp = 0; jp < l; jp++)
            if (fabs(x[jp]) > thr && ll < M)
            {
                v[(size_t) i * M + ll] = x[jp];
                ix[(size_t) i * M + ll] = jx[jp];
                ll++;
            }
        nz[i] = ll;
    }
    free(x);
    free(jx);
}

/* ---- threshold: ellpack/bml_threshold_ellpack_typed.c:114-131 -------------- */
void oracle_ellpack_threshold_d(int N, int M, double *v, int *ix, int *nz, double thr)
{
    for (int i = 0; i < N; i++)
    {
        int rlen = 0;
        for (int j = 0; j < nz[i]; j++)
            if (fabs(v[(size_t) i * M + j]) > thr)
            {
                v[(size_t) i * M + rlen] = v[(size_t) i * M + j];
                ix[(size_t) i * M + rlen] = ix[(size_t) i * M + j];
                rlen++;
            }
        nz[i] = rlen;
    }
}

/* ---- trace / trace_mult -------------------------------------------------- */
double oracle_ellpack_trace_d(int N, int M, const double *v, const int *ix, const int *nz)
{
    double t = 0.0;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < nz[i]; j++)
            if (ix[(size_t) i * M + j] == i)
            {
                t += v[(size_t) i * M + j];
                break;
            }
    return t;
}

/* trace_mult reads B's row i at the columns of A's row i
 * (ellpack/bml_trace_ellpack_typed.c:145-158 via bml_getVector_ellpack,
 * ellpack/bml_submatrix_ellpack_typed.c:380-406). */
double oracle_ellpack_trace_mult_d(int N, int MA, const double *av, const int *aix,
                                   const int *anz, int MB, const double *bv, const int *bix,
                                   const int *bnz)
{
    double t = 0.0;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < anz[i]; j++)
        {
            double r = 0.0;
            int col = aix[(size_t) i * MA + j];
            for (int q = 0; q < bnz[i]; q++)
                if (bix[(size_t) i * MB + q] == col)
                {
                    r = bv[(size_t) i * MB + q];
                    break;
                }
            t += av[(size_t) i * MA + j] * r;
        }
    return t;
}

/* ---- transpose: serial order of ellpack/bml_transpose_ellpack_typed.c:76-96 */
void oracle_ellpack_transpose_d(int N, int M, const double *v, const int *ix, const int *nz,
                                double *tv, int *tix, int *tnz)
{
    for (int i = 0; i < N; i++)
        tnz[i] = 0;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < nz[i]; j++)
        {
            int r = ix[(size_t) i * M + j];
            if (tnz[r] < M)
            {
                tix[(size_t) r * M + tnz[r]] = i;
                tv[(size_t) r * M + tnz[r]] = v[(size_t) i * M + j];
                tnz[r]++;
            }
        }
}

/* ---- Gershgorin: ellpack/bml_normalize_ellpack_typed.c:82-175 ------------- */
void oracle_ellpack_gershgorin_d(int N, int M, const double *v, const int *ix, const int *nz,
                                 double *bounds)
{
    double emin = DBL_MAX, emax = DBL_MIN;
    for (int i = 0; i < N; i++)
    {
        double radius = 0.0, dvalue = 0.0;
        for (int j = 0; j < nz[i]; j++)
        {
            if (i == ix[(size_t) i * M + j])
                dvalue = v[(size_t) i * M + j];
            else
                radius += fabs(v[(size_t) i * M + j]);
        }
        if (dvalue + radius > emax)
            emax = dvalue + radius;
        if (dvalue - radius < emin)
            emin = dvalue - radius;
    }
    bounds[0] = emin;
    bounds[1] = emax;
}

/* ---- SP2 (same rules as bml_b200_sp2) -------------------------------------- */
int oracle_ellpack_sp2_d(int N, int M, const double *hv, const int *hix, const int *hnz,
                         double thr, double occ, int maxiter, double tol, int stall,
                         double *dv, int *dix, int *dnz, double *info)
{
    size_t NM = (size_t) N * M;
    double *x2v = malloc(sizeof(double) * NM);
    int *x2ix = malloc(sizeof(int) * NM);
    int *x2nz = malloc(sizeof(int) * (size_t) N);
    memcpy(dv, hv, sizeof(double) * NM);
    memcpy(dix, hix, sizeof(int) * NM);
    memcpy(dnz, hnz, sizeof(int) * (size_t) N);
    double b[2];
    oracle_ellpack_gershgorin_d(N, M, hv, hix, hnz, b);
    /* normalize: scale by -1/(emax-emin), add emax/(emax-emin) on the diagonal
     * with threshold 0 (ellpack/bml_normalize_ellpack_typed.c:32-45) */
    double mm = b[1] - b[0];
    double s = -1.0 / mm;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < dnz[i]; j++)
            dv[(size_t) i * M + j] = s * dv[(size_t) i * M + j];
    oracle_ellpack_add_identity_d(N, M, dv, dix, dnz, b[1] / mm, 0.0);
    int it = 0, rule = 3, since = 0, maxw = 0;
    double best = HUGE_VAL, idem = 0.0;
    for (; it < maxiter; it++)
    {
        double tr[2];
        int w = oracle_ellpack_x2_d(N, M, dv, dix, dnz, thr, M, x2v, x2ix, x2nz, tr);
        if (w > maxw)
            maxw = w;
        if (w > M)
        {
            rule = 4;
            break;
        }
        idem = fabs(tr[0] - tr[1]);
        if (fabs(tr[1] - occ) <= fabs(2.0 * tr[0] - tr[1] - occ))
        {
            memcpy(dv, x2v, sizeof(double) * NM);
            memcpy(dix, x2ix, sizeof(int) * NM);
            memcpy(dnz, x2nz, sizeof(int) * (size_t) N);
        }
        else
            oracle_ellpack_add_d(N, M, dv, dix, dnz, M, x2v, x2ix, x2nz, 2.0, -1.0, thr);
        if (idem < tol)
        {
            rule = 1;
            it++;
            break;
        }
        if (stall > 0)
        {
            if (idem < best)
            {
                best = idem;
                since = 0;
            }
            else if (++since >= stall)
            {
                rule = 2;
                it++;
                break;
            }
        }
    }
    if (info)
    {
        info[0] = it;
        info[1] = rule;
        info[2] = oracle_ellpack_trace_d(N, M, dv, dix, dnz);
        info[3] = idem;
        info[4] = maxw;
        info[5] = 0.0;
    }
    free(x2v);
    free(x2ix);
    free(x2nz);
    return it;
}

/* ---- ELLBLOCK X^2 in both real precisions ---------------------------------- */
#define EB_REAL double
#define EB_X2_NAME oracle_ellblock_x2_d
#include "bml_oracle_eb_x2.inc"
#undef EB_REAL
#undef EB_X2_NAME
#define EB_REAL float
#define EB_X2_NAME oracle_ellblock_x2_s
#include "bml_oracle_eb_x2.inc"
#undef EB_REAL
#undef EB_X2_NAME
