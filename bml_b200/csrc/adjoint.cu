// Adjoint of SP2 purification: the density-matrix response dL/dH of
// L = sum_ij D_ij V_ij, D = X_K after K SP2 iterations from H (no reference
// counterpart; the reference library has no derivatives).
//
// Forward, as bml_b200_sp2 with a fixed iteration count and no stop test:
//   X0 = (emax I - H) / (emax - emin)          (Gershgorin bounds of H)
//   X_{n+1} = T(X_n^2)                         (X^2 branch)
//   X_{n+1} = T'(2 X_n - T(X_n^2))             (2X - X^2 branch)
// where T keeps |x| > threshold (and the diagonal) and T' keeps |x| >
// threshold.  The thresholds and the branch choices are held fixed in the
// derivative: a retained entry passes its gradient, a dropped one none.
// Backward, with G the gradient on the pattern of X_{n+1}:
//   X^2 branch:    G_n = P_n(G X_n^T + X_n^T G)
//   2X - X^2:      G_n = P_n(2 G - (Q_n G) X_n^T - X_n^T (Q_n G))
// where Q_n keeps the entries of G on the pattern of T(X_n^2) and P_n keeps
// the pattern of X_n (entries outside it were dropped by an earlier
// threshold, so no gradient reaches them).  The products are the library's
// sparse products; where the unordered kernel takes them, their masked form
// forms only the entries on X_n's pattern (the rest would be dropped by P_n),
// so no product wider than X_n is ever stored; otherwise (the ordered form,
// or rows the dense tier takes) they are formed at threshold 0 and then
// restricted, one kernel.
// Memory: X is checkpointed every `every` iterations in the forward pass and
// each segment is recomputed before its backward steps (bit-identically with
// the ordered products and on the dense tier; the unordered sparse products
// may add in another order, so a recomputed iterate can differ from the first
// pass in the last bits), so at most K/every + every iterates are held.
// Finally dL/dH = -G_0/d + a * d(emax)/dH + b * d(emin)/dH, with d = emax -
// emin, a = (tr G_0 - <G_0, X0>)/d and b = <G_0, X0>/d; emax = h_k + r_k of
// its maximising row k (diagonal + sum of |off-diagonals|), so d(emax)/dH is
// 1 on H_kk and sign(H_kj) on row k's other entries, and likewise for emin
// = h_m - r_m with -sign(H_mj).
#include "internal.h"

#include <cmath>
#include <cstdlib>
#include <vector>

namespace {

struct Mat
{
    bml_matrix_t *m = nullptr;
    Mat() = default;
    explicit Mat(bml_matrix_t *p) : m(p) {}
    Mat(const Mat &) = delete;
    Mat &operator=(const Mat &) = delete;
    Mat(Mat &&o) noexcept : m(o.m) { o.m = nullptr; }
    Mat &operator=(Mat &&o) noexcept
    {
        reset();
        m = o.m;
        o.m = nullptr;
        return *this;
    }
    ~Mat() { reset(); }
    void reset()
    {
        if (m)
            bml_deallocate(&m);
        m = nullptr;
    }
    bml_matrix_ellpack_t *e() const { return static_cast<bml_matrix_ellpack_t *>(m); }
};

int err() { return bml_b200_last_error(); }

Mat zero(bml_matrix_precision_t prec, int N, int M)
{
    return Mat(bml_zero_matrix(ellpack, prec, N, M, sequential));
}

Mat copy_of(bml_matrix_t *A, int M)
{
    Mat C = zero(bml_get_precision(A), bml_get_N(A), M);
    if (C.m)
        bml_copy(A, C.m);
    return C;
}

// A*B (threshold 0) into a matrix wide enough for it: retried once at the
// width the first attempt reports.
Mat product(bml_matrix_t *A, bml_matrix_t *B, int M0)
{
    const int N = bml_get_N(A);
    int M = M0 < N ? M0 : N;
    for (int attempt = 0; attempt < 3; ++attempt)
    {
        Mat C = zero(bml_get_precision(A), N, M);
        if (!C.m)
            return Mat();
        bml_multiply_AB(A, B, C.m, 0.0);
        const int e = err();
        if (!e)
            return C;
        if (e != BML_B200_ERR_ROW_OVERFLOW || M >= N)
            return Mat();
        const int need = bml_b200_last_required_M();
        bml_b200_clear_error();
        M = need > M ? need : 2 * M;
        M = (M + 31) / 32 * 32;
        if (M > N)
            M = N;
    }
    return Mat();
}

// A*B at P's pattern (C with P's M), through the masked form of the unordered
// product; an empty Mat with no status set where that form does not apply.
Mat masked_product(bml_matrix_t *A, bml_matrix_t *B, bml_matrix_t *P)
{
    Mat C = zero(bml_get_precision(A), bml_get_N(A), bml_get_M(P));
    if (!C.m)
        return Mat();
    bool taken = false;
    if (!ell_multiply_masked(static_cast<bml_matrix_ellpack_t *>(A), static_cast<bml_matrix_ellpack_t *>(B),
                             static_cast<bml_matrix_ellpack_t *>(P), C.e(), &taken))
        return Mat();
    return C;
}

// One SP2 step X -> X_next (X2 is scratch of X's shape); returns the branch
// (0: X^2, 1: 2X - X^2).  Same calls, in the same order, as bml_b200_sp2.
int sp2_step(bml_matrix_t *X, bml_matrix_t *X2, double threshold, double occupation)
{
    double tr[2];
    if (bml_b200_multiply_x2(X, X2, threshold, tr) != BML_B200_OK)
        return -1;
    const double t = tr[0], t2 = tr[1];
    if (fabs(t2 - occupation) <= fabs(2.0 * t - t2 - occupation))
    {
        bml_copy(X2, X);
        return err() ? -1 : 0;
    }
    bml_add(X, X2, 2.0, -1.0, threshold);
    return err() ? -1 : 1;
}

// Gradient through one SP2 step: G (on X_{n+1}'s pattern) -> G_n (on Xn's
// pattern).  X2 is scratch of Xn's shape.
Mat step_back(bml_matrix_t *Xn, const Mat &G, int branch, double threshold, bml_matrix_t *X2)
{
    const int N = bml_get_N(Xn), M = bml_get_M(Xn);
    const bml_matrix_precision_t prec = bml_get_precision(Xn);
    Mat Xt(bml_transpose_new(Xn));
    if (!Xt.m)
        return Mat();
    Mat Gh; // gradient of T(X_n^2), on its pattern
    if (branch == 0)
        Gh = copy_of(G.m, bml_get_M(G.m));
    else
    {
        double tr[2];
        if (bml_b200_multiply_x2(Xn, X2, threshold, tr) != BML_B200_OK)
            return Mat();
        Gh = zero(prec, N, bml_get_M(X2));
        if (!Gh.m || !ell_restrict(static_cast<bml_matrix_ellpack_t *>(G.m),
                                   static_cast<bml_matrix_ellpack_t *>(X2), Gh.e()))
            return Mat();
        double minus1 = -1.0;
        float minus1f = -1.0f;
        bml_scale_inplace(prec == double_real ? (void *) &minus1 : (void *) &minus1f, Gh.m);
    }
    // on X_n's pattern where the masked form applies, else whole
    Mat T1 = masked_product(Gh.m, Xt.m, Xn);
    Mat T2 = T1.m ? masked_product(Xt.m, Gh.m, Xn) : Mat();
    if (err())
        return Mat();
    const bool on_pattern = T1.m && T2.m;
    if (!on_pattern)
    {
        T1 = product(Gh.m, Xt.m, 2 * M);
        if (!T1.m)
            return Mat();
        T2 = product(Xt.m, Gh.m, bml_get_M(T1.m));
        if (!T2.m)
            return Mat();
    }
    // T1 + T2 (+ 2G).  On X_n's pattern T1 and T2 share it, and G is first
    // restricted to it, so the sum is no wider than X_n.
    Mat Gr;
    if (on_pattern && branch)
    {
        Gr = zero(prec, N, M);
        if (!Gr.m || !ell_restrict(static_cast<bml_matrix_ellpack_t *>(G.m), static_cast<bml_matrix_ellpack_t *>(Xn),
                                   Gr.e()))
            return Mat();
    }
    int MS = on_pattern ? M : bml_get_M(T1.m) + bml_get_M(T2.m) + (branch ? bml_get_M(G.m) : 0);
    MS = MS < N ? MS : N;
    Mat S = copy_of(T1.m, MS);
    if (!S.m || err())
        return Mat();
    bml_add(S.m, T2.m, 1.0, 1.0, 0.0);
    if (branch)
        bml_add(S.m, on_pattern ? Gr.m : G.m, 1.0, 2.0, 0.0);
    if (err())
        return Mat();
    Mat Gn = zero(prec, N, M);
    if (!Gn.m || !ell_restrict(S.e(), static_cast<bml_matrix_ellpack_t *>(Xn), Gn.e()))
        return Mat();
    return Gn;
}

// Rows of H whose Gershgorin discs reach emax (h + r) and emin (h - r),
// computed on the host mirror with the device kernel's arithmetic.
template <typename T>
void gershgorin_rows(bml_matrix_ellpack_t *H, int *kmax, int *kmin)
{
    const T *v = static_cast<const T *>(H->value);
    double best_hi = -HUGE_VAL, best_lo = HUGE_VAL;
    *kmax = *kmin = 0;
    for (int i = 0; i < H->N; ++i)
    {
        T radius = T(0), d = T(0);
        for (int p = 0; p < H->nnz[i]; ++p)
        {
            const int k = H->index[(size_t) i * H->M + p];
            const T x = v[(size_t) i * H->M + p];
            if (k == i)
                d = x;
            else
                radius = (T) ((double) radius + (double) fabs(x));
        }
        const double hi = (double) (T) (d + radius), lo = (double) (T) (d - radius);
        if (hi > best_hi)
        {
            best_hi = hi;
            *kmax = i;
        }
        if (lo < best_lo)
        {
            best_lo = lo;
            *kmin = i;
        }
    }
}

// dH row `row` += c * (1 on the diagonal, sgn * sign(H_rj) elsewhere).
template <typename T>
void add_disc_gradient(bml_matrix_ellpack_t *H, bml_matrix_ellpack_t *dH, int row, double c, double sgn)
{
    const T *hv = static_cast<const T *>(H->value);
    T *gv = static_cast<T *>(dH->value);
    for (int p = 0; p < dH->nnz[row]; ++p)
    {
        const int k = dH->index[(size_t) row * dH->M + p];
        double s = 0.0;
        if (k == row)
            s = 1.0;
        else
            for (int q = 0; q < H->nnz[row]; ++q)
                if (H->index[(size_t) row * H->M + q] == k)
                {
                    const T x = hv[(size_t) row * H->M + q];
                    s = sgn * (x > T(0) ? 1.0 : (x < T(0) ? -1.0 : 0.0));
                    break;
                }
        gv[(size_t) row * dH->M + p] = (T) ((double) gv[(size_t) row * dH->M + p] + c * s);
    }
}

} // namespace

extern "C" int bml_b200_sp2_adjoint(bml_matrix_t *H, bml_matrix_t *V, double threshold, double occupation,
                                    int iters, int every, int M, bml_matrix_t *dH, double *loss)
{
    if (!H || !V || !dH || bml_get_type(H) != ellpack || bml_get_type(V) != ellpack ||
        bml_get_type(dH) != ellpack || bml_get_precision(V) != bml_get_precision(H) ||
        bml_get_precision(dH) != bml_get_precision(H) || bml_get_N(V) != bml_get_N(H) ||
        bml_get_N(dH) != bml_get_N(H) || iters < 0 || every < 1 || M < 1 || dH == H || dH == V)
    {
        b200_set_error(BML_B200_ERR_INVALID,
                       "sp2_adjoint: H, V, dH must be ELLPACK of one precision and N (dH distinct), "
                       "iters >= 0, every >= 1, M >= 1");
        return BML_B200_ERR_INVALID;
    }
    bml_b200_clear_error();
    const int N = bml_get_N(H);
    const bml_matrix_precision_t prec = bml_get_precision(H);

    // X0 and the bounds
    Mat X = zero(prec, N, M);
    if (!X.m)
        return err();
    bml_copy(H, X.m);
    double *eb = static_cast<double *>(bml_gershgorin(H));
    if (!eb || err())
    {
        free(eb);
        return err() ? err() : BML_B200_ERR_INVALID;
    }
    const double emin = eb[0], emax = eb[1];
    free(eb);
    bml_normalize(X.m, emin, emax);
    if (err())
        return err();

    // forward with checkpoints
    std::vector<Mat> cps;
    std::vector<int> branch(iters);
    Mat X2 = zero(prec, N, M);
    if (!X2.m)
        return err();
    for (int n = 0; n < iters; ++n)
    {
        if (n % every == 0)
        {
            cps.push_back(copy_of(X.m, M));
            if (!cps.back().m || err())
                return err();
        }
        branch[n] = sp2_step(X.m, X2.m, threshold, occupation);
        if (branch[n] < 0)
            return err();
    }
    if (iters == 0)
        cps.push_back(copy_of(X.m, M));

    // L and its gradient on D = X_K
    Mat G = zero(prec, N, M);
    if (!G.m || !ell_restrict(static_cast<bml_matrix_ellpack_t *>(V), X.e(), G.e()))
        return err();
    const double L = bml_trace_mult(X.m, G.m);
    if (err())
        return err();

    // backward, segment by segment from the last checkpoint
    for (int s = (int) cps.size() - 1; s >= 0 && iters > 0; --s)
    {
        const int n0 = s * every;
        const int n1 = n0 + every < iters ? n0 + every : iters;
        std::vector<Mat> seg;
        seg.push_back(copy_of(cps[s].m, M));
        for (int n = n0; n + 1 < n1; ++n)
        {
            Mat Xn = copy_of(seg.back().m, M);
            if (!Xn.m || sp2_step(Xn.m, X2.m, threshold, occupation) != branch[n])
            {
                if (!err())
                    b200_set_error(BML_B200_ERR_INVALID, "sp2_adjoint: recomputation took another branch");
                return err();
            }
            seg.push_back(std::move(Xn));
        }
        for (int n = n1 - 1; n >= n0; --n)
        {
            Mat Gn = step_back(seg[n - n0].m, G, branch[n], threshold, X2.m);
            if (!Gn.m)
                return err() ? err() : BML_B200_ERR_INVALID;
            G = std::move(Gn);
        }
    }

    // through X0 = (emax I - H)/d to H
    const double d = emax - emin;
    const double trG = bml_trace(G.m);
    const double gx = bml_trace_mult(G.m, cps[0].m);
    if (err())
        return err();
    bml_matrix_ellpack_t *He = static_cast<bml_matrix_ellpack_t *>(H);
    bml_matrix_ellpack_t *De = static_cast<bml_matrix_ellpack_t *>(dH);
    if (!ell_restrict(G.e(), He, De))
        return err();
    double sc = -1.0 / d;
    float scf = (float) sc;
    bml_scale_inplace(prec == double_real ? (void *) &sc : (void *) &scf, dH);
    if (err() || !ell_to_host(He) || !ell_to_host(De))
        return err();
    int kmax = 0, kmin = 0;
    const double a = (trG - gx) / d, b = gx / d;
    if (prec == double_real)
    {
        gershgorin_rows<double>(He, &kmax, &kmin);
        add_disc_gradient<double>(He, De, kmax, a, 1.0);
        add_disc_gradient<double>(He, De, kmin, b, -1.0);
    }
    else
    {
        gershgorin_rows<float>(He, &kmax, &kmin);
        add_disc_gradient<float>(He, De, kmax, a, 1.0);
        add_disc_gradient<float>(He, De, kmin, b, -1.0);
    }
    ell_mark_host(De);
    if (loss)
        *loss = L;
    return BML_B200_OK;
}
